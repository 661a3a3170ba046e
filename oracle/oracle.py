"""ctypes wrapper of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg are the only callers.  The product (rusty_h264_b200) never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

u8p = C.POINTER(C.c_uint8)
i16p = C.POINTER(C.c_int16)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
u16p = C.POINTER(C.c_uint16)


class MeParamsFlat(C.Structure):
    """Mirror of or_me_params_flat (oracle/h264_oracle_par.c)."""

    _fields_ = [
        ("fast", C.c_int32), ("mb_use_satd", C.c_int32), ("sadfp", C.c_int32), ("mv_cost_kind", C.c_int32),
        ("sadfp_lambda", C.c_double),
        ("me_snap", C.c_int32), ("me_fc", C.c_int32),
        ("dia_mask", C.c_uint32), ("dia_sub_mask", C.c_uint32),
        ("subpel", C.c_int32), ("subpel_pat", C.c_int32), ("sp_single_pass", C.c_int32), ("sub_pat", C.c_int32),
        ("me_subpel_iter", C.c_int32), ("sp_maxit", C.c_int32), ("sp_fc", C.c_int32),
    ]


def balanced_params(**kw) -> MeParamsFlat:
    """The Balanced-preset motion_search settings (config.rs:448-571 defaults)."""
    p = MeParamsFlat(fast=0, mb_use_satd=0, sadfp=0, mv_cost_kind=0, sadfp_lambda=0.5, me_snap=1, me_fc=1,
                     dia_mask=0b11100, dia_sub_mask=0b10000, subpel=1, subpel_pat=-1, sp_single_pass=1, sub_pat=2,
                     me_subpel_iter=1, sp_maxit=0, sp_fc=0)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_satd4x4_wels.restype = C.c_int32
        L.or_satd_region_wels.restype = C.c_int32
        L.or_sad.restype = C.c_int32
        L.or_satd_px.restype = C.c_int64
        L.or_satd_avg.restype = C.c_uint32
        L.or_sad_avg.restype = C.c_int64
        L.or_median3.restype = C.c_int32
        L.or_luma_sample.restype = C.c_int32
        L.or_mvbits.restype = C.c_uint32
        L.or_mc_satd_hp.restype = C.c_int64
        L.or_mc_sad_hp.restype = C.c_int64
        L.or_intra_cost.restype = C.c_int32
        L.or_la_mc_satd.restype = C.c_int64
        L.or_candidate_dist.restype = C.c_int64
        L.or_num_threads.restype = C.c_int
        L.or_chroma_qp.restype = C.c_int
        L.or_motion_search_flat.argtypes = [u8p, u8p, u8p, C.c_int, C.c_int, C.c_int, C.POINTER(MeParamsFlat), u16p,
                                            C.c_int, C.c_int, C.c_int, C.c_int, i32p, C.c_int, C.c_double, i32p,
                                            i32p, i64p, i32p]
        L.or_me_frame_flat.argtypes = [u8p, u8p, u8p, C.c_int, C.c_int, C.c_int, C.POINTER(MeParamsFlat), u16p,
                                       C.c_double, C.c_int64, i32p, i64p]
        L.or_me_frame_learned_flat.argtypes = [u8p, u8p, u8p, C.c_int, C.c_int, C.c_int, C.POINTER(MeParamsFlat),
                                               u16p, C.c_double, C.c_int64, i32p, C.c_int32, i32p, i64p, i32p]
        L.or_me_frame_multiref_flat.argtypes = [u8p, u8p, u8p, C.c_int, C.c_int, C.c_int, C.c_int,
                                                C.POINTER(MeParamsFlat), u16p, C.c_double, C.c_int64, i32p, i64p]
        L.or_closed_loop_clip.argtypes = [u8p, u8p, u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(MeParamsFlat),
                                          u16p, C.c_double, C.c_int64, C.c_int, C.c_int, i32p, C.c_int32, i32p, i64p,
                                          i16p, i16p, u8p, u8p, u8p, i32p]
        L.or_pixel_path_clip.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(MeParamsFlat), u16p,
                                         C.c_double, C.c_int64, C.c_int, C.c_int, i32p, i64p, i16p, i32p, i32p, i32p,
                                         C.c_int]
        _lib = L
    return _lib


def ptr(a: np.ndarray, t=u8p):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


# ---- convenience wrappers ---------------------------------------------------

def satd_px(src, ss, pred, ps, w, h) -> int:
    return lib().or_satd_px(ptr(src), ss, ptr(pred), ps, w, h)


def pad_plane(y: np.ndarray, pad: int) -> np.ndarray:
    h, w = y.shape
    f = np.empty((h + 2 * pad, w + 2 * pad), np.uint8)
    lib().or_pad_plane(ptr(np.ascontiguousarray(y)), w, h, pad, ptr(f))
    return f


def hpel_fused(f: np.ndarray):
    ph, pw = f.shape
    h, v, c = (np.empty_like(f) for _ in range(3))
    lib().or_hpel_fused(ptr(f), pw, ph, ptr(h), ptr(v), ptr(c))
    return h, v, c


def hpel_tiles(f: np.ndarray):
    ph, pw = f.shape
    h, v, c = (np.empty_like(f) for _ in range(3))
    lib().or_hpel_tiles(ptr(f), pw, ph, ptr(h), ptr(v), ptr(c))
    return h, v, c


def build_planes4(y: np.ndarray, pad: int = 32) -> np.ndarray:
    """F|H|V|C padded planes of a luma frame, shape (4, ph, pw)."""
    ch, cw = y.shape
    out = np.empty((4, ch + 2 * pad, cw + 2 * pad), np.uint8)
    lib().or_build_planes4(ptr(np.ascontiguousarray(y)), cw, ch, pad, ptr(out))
    return out


def mc_luma(ref: np.ndarray, x0, y0, bw, bh, mvx, mvy) -> np.ndarray:
    ch, cw = ref.shape
    out = np.empty((bh, bw), np.uint8)
    lib().or_mc_luma(ptr(ref), cw, ch, x0, y0, bw, bh, mvx, mvy, ptr(out))
    return out


def luma_sample(ref: np.ndarray, ix, iy, fx, fy) -> int:
    ch, cw = ref.shape
    return lib().or_luma_sample(ptr(ref), cw, ch, ix, iy, fx, fy)


def mv_cost_table() -> np.ndarray:
    t = np.empty(4096, np.uint16)
    lib().or_build_mv_cost(ptr(t, u16p))
    return t


def motion_search(src, ref, planes4, params, lx, ly, rw, rh, preds, lambda_me, start=None, tab=None, pad=32):
    ch, cw = src.shape
    pr = np.ascontiguousarray(np.asarray(preds, np.int32).reshape(-1))
    mv = np.zeros(2, np.int32)
    cost = np.zeros(1, np.int64)
    ev = np.zeros(1, np.int32)
    st = None if start is None else np.asarray(start, np.int32)
    tab = mv_cost_table() if tab is None else tab
    lib().or_motion_search_flat(ptr(src), ptr(ref), ptr(planes4), cw, ch, pad, C.byref(params), ptr(tab, u16p),
                                lx, ly, rw, rh, ptr(pr, i32p), len(pr) // 2, float(lambda_me),
                                None if st is None else ptr(st, i32p), ptr(mv, i32p), ptr(cost, i64p), ptr(ev, i32p))
    return (int(mv[0]), int(mv[1])), int(cost[0]), int(ev[0])


def candidate_dist(src, ref, planes4, kind, lx, ly, rw, rh, mvx, mvy, pad=32) -> int:
    ch, cw = src.shape
    return lib().or_candidate_dist(ptr(src), ptr(ref), ptr(planes4), cw, ch, pad, kind, lx, ly, rw, rh, mvx, mvy)


def me_frame(src, ref, planes4, params, lambda_me, split_gate=-1, tab=None, pad=32):
    ch, cw = src.shape
    nmb = (cw // 16) * (ch // 16)
    picks = np.zeros((nmb, 6), np.int32)
    costs = np.zeros((nmb, 2), np.int64)
    tab = mv_cost_table() if tab is None else tab
    lib().or_me_frame_flat(ptr(src), ptr(ref), ptr(planes4), cw, ch, pad, C.byref(params), ptr(tab, u16p),
                           float(lambda_me), int(split_gate), ptr(picks, i32p), ptr(costs, i64p))
    return picks, costs


def me_frame_multiref(src, refs, planes, params, lambda_me, split_gate=-1, tab=None, pad=32):
    """The plain-ME frame model over len(refs) references (refs (nref, ch, cw)
    u8, reference 0 the nearest; planes (nref, 4, ph, pw) their planes):
    picks (nmb, 8) i32 (shape, ref0, mv0x, mv0y, ref1, mv1x, mv1y, 0) and
    costs (nmb, 2) i64."""
    ch, cw = src.shape
    nmb = (cw // 16) * (ch // 16)
    refs = np.ascontiguousarray(refs, np.uint8)
    planes = np.ascontiguousarray(planes, np.uint8)
    picks = np.zeros((nmb, 8), np.int32)
    costs = np.zeros((nmb, 2), np.int64)
    tab = mv_cost_table() if tab is None else tab
    lib().or_me_frame_multiref_flat(ptr(src), ptr(refs), ptr(planes), len(refs), cw, ch, pad, C.byref(params),
                                    ptr(tab, u16p), float(lambda_me), int(split_gate), ptr(picks, i32p),
                                    ptr(costs, i64p))
    return picks, costs


def me_frame_learned(src, ref, planes4, params, lambda_me, props, prop_t, split_gate=-1, tab=None, pad=32):
    """me_frame with the learned 16x16 search over props (nmb, 16) i32;
    returns (picks, costs, fallback flags)."""
    ch, cw = src.shape
    nmb = (cw // 16) * (ch // 16)
    picks = np.zeros((nmb, 6), np.int32)
    costs = np.zeros((nmb, 2), np.int64)
    fell = np.zeros(nmb, np.int32)
    props = np.ascontiguousarray(props, np.int32)
    assert props.shape == (nmb, 16)
    tab = mv_cost_table() if tab is None else tab
    lib().or_me_frame_learned_flat(ptr(src), ptr(ref), ptr(planes4), cw, ch, pad, C.byref(params), ptr(tab, u16p),
                                   float(lambda_me), int(split_gate), ptr(props, i32p), int(prop_t), ptr(picks, i32p),
                                   ptr(costs, i64p), ptr(fell, i32p))
    return picks, costs, fell


def mc_tq_frame(src, ref, picks, qp, dz_div=6):
    ch, cw = src.shape
    nmb = (cw // 16) * (ch // 16)
    out = np.zeros((nmb, 256), np.int16)
    lib().or_mc_tq_frame(ptr(src), ptr(ref), cw, ch, ptr(np.ascontiguousarray(picks), i32p), qp, dz_div,
                         ptr(out, i16p))
    return out


def mc_tq_rec_frame(src, ref, picks, qp, dz_div=6):
    """(coeffs, rec): MC + luma T/Q and the luma reconstruction of a frame."""
    ch, cw = src.shape
    nmb = (cw // 16) * (ch // 16)
    out = np.zeros((nmb, 256), np.int16)
    rec = np.zeros((ch, cw), np.uint8)
    lib().or_mc_tq_rec_frame(ptr(src), ptr(ref), cw, ch, ptr(np.ascontiguousarray(picks), i32p), qp, dz_div,
                             ptr(out, i16p), ptr(rec))
    return out, rec


def mc_tq_chroma_frame(src_u, src_v, ref_u, ref_v, picks, qp, rec=True):
    """(coeffs (nmb, 128) i16, rec_u, rec_v): the inter MBs' chroma MC, T/Q and
    reconstruction of a frame."""
    cch, ccw = src_u.shape
    nmb = (ccw // 8) * (cch // 8)
    out = np.zeros((nmb, 128), np.int16)
    ru = np.zeros((cch, ccw), np.uint8) if rec else None
    rv = np.zeros((cch, ccw), np.uint8) if rec else None
    c = [np.ascontiguousarray(a) for a in (src_u, src_v, ref_u, ref_v)]
    lib().or_mc_tq_chroma_frame(ptr(c[0]), ptr(c[1]), ptr(c[2]), ptr(c[3]), 2 * ccw, 2 * cch,
                                ptr(np.ascontiguousarray(picks), i32p), int(qp), ptr(out, i16p),
                                ptr(ru) if rec else None, ptr(rv) if rec else None)
    return out, ru, rv


def deblock_frame(y, u, v, picks, coeffs, qp, offset_a=0, offset_b=0, chroma_qp_offset=0):
    """In-loop deblocking of a plain-ME picture: returns filtered copies of
    (y, u, v); u and v may be None."""
    ch, cw = y.shape
    yo = np.array(y, np.uint8, copy=True)
    uo = None if u is None else np.array(u, np.uint8, copy=True)
    vo = None if v is None else np.array(v, np.uint8, copy=True)
    lib().or_deblock_frame_plain(ptr(yo), None if uo is None else ptr(uo), None if vo is None else ptr(vo), cw, ch,
                                 ptr(np.ascontiguousarray(picks), i32p),
                                 ptr(np.ascontiguousarray(coeffs, np.int16), i16p), int(qp), int(offset_a),
                                 int(offset_b), int(chroma_qp_offset))
    return yo, uo, vo


def deblock_tables():
    a = np.zeros(52, np.int32)
    b = np.zeros(52, np.int32)
    t = np.zeros((52, 3), np.int32)
    lib().or_deblock_tables(ptr(a, i32p), ptr(b, i32p), ptr(t, i32p))
    return a, b, t


def mc_chroma(ref: np.ndarray, x0, y0, bw, bh, mvx, mvy) -> np.ndarray:
    ch, cw = ref.shape
    out = np.zeros((bh, bw), np.uint8)
    lib().or_mc_chroma(ptr(np.ascontiguousarray(ref)), cw, ch, x0, y0, bw, bh, mvx, mvy, ptr(out))
    return out


def chroma_qp(qp) -> int:
    return lib().or_chroma_qp(int(qp))


def chroma_dc_quant(dc, qp, intra=False):
    """(levels, reconstructed DCs) of a 2x2 chroma DC block."""
    d = np.ascontiguousarray(dc, np.int32)
    lv = np.zeros(4, np.int32)
    rd = np.zeros(4, np.int32)
    lib().or_forward_quant_chroma_dc(ptr(d, i32p), int(qp), int(intra), ptr(lv, i32p))
    lib().or_inverse_quant_chroma_dc(ptr(lv, i32p), int(qp), ptr(rd, i32p))
    return lv, rd


def dequant4x4(levels, qp) -> np.ndarray:
    lv = np.ascontiguousarray(levels, np.int32)
    out = np.zeros(16, np.int32)
    lib().or_dequant4x4(ptr(lv, i32p), int(qp), ptr(out, i32p))
    return out


def inverse_core4(coeffs) -> np.ndarray:
    m = np.array(coeffs, np.int32)
    lib().or_inverse_core4(ptr(m, i32p))
    return m


def idct_four_t4_rec(pred8: np.ndarray, dct64: np.ndarray) -> np.ndarray:
    """idct_four_t4_rec over an 8x8 region: pred 8x8 u8 (stride 8), 64 i16."""
    rec = np.zeros((8, 8), np.uint8)
    lib().or_idct_four_t4_rec(ptr(rec), 8, ptr(np.ascontiguousarray(pred8)), 8,
                              ptr(np.ascontiguousarray(dct64, np.int16), i16p))
    return rec


def downsample2x(y):
    ch, cw = y.shape
    out = np.empty((ch // 2, cw // 2), np.uint8)
    lib().or_downsample2x(ptr(np.ascontiguousarray(y)), cw, ch, ptr(out))
    return out


def lookahead_clip(frames: np.ndarray, mode=2, nthreads=1):
    n, ch, cw = frames.shape
    nmb = (cw // 16) * (ch // 16)
    intra = np.zeros((n, nmb), np.int32)
    inter = np.zeros((n, nmb), np.int32)
    mvs = np.zeros((n, nmb, 2), np.int32)
    lib().or_lookahead_clip(ptr(np.ascontiguousarray(frames)), n, cw, ch, mode, ptr(intra, i32p), ptr(inter, i32p),
                            ptr(mvs, i32p), nthreads)
    return intra, inter, mvs


def pixel_path_clip(frames: np.ndarray, params, lambda_me, split_gate, qp, dz_div=6, pad=32, nthreads=1, tab=None):
    n, ch, cw = frames.shape
    nmb = (cw // 16) * (ch // 16)
    picks = np.zeros((n, nmb, 6), np.int32)
    costs = np.zeros((n, nmb, 2), np.int64)
    coeffs = np.zeros((n, nmb, 256), np.int16)
    intra = np.zeros((n, nmb), np.int32)
    inter = np.zeros((n, nmb), np.int32)
    mvs = np.zeros((n, nmb, 2), np.int32)
    tab = mv_cost_table() if tab is None else tab
    lib().or_pixel_path_clip(ptr(np.ascontiguousarray(frames)), n, cw, ch, pad, C.byref(params), ptr(tab, u16p),
                             float(lambda_me), int(split_gate), qp, dz_div, ptr(picks, i32p), ptr(costs, i64p),
                             ptr(coeffs, i16p), ptr(intra, i32p), ptr(inter, i32p), ptr(mvs, i32p), nthreads)
    return dict(picks=picks, costs=costs, coeffs=coeffs, la_intra=intra, la_inter=inter, la_mvs=mvs)


def closed_loop_clip(y, u, v, params, lambda_me, split_gate, qp, dz_div=6, pad=32, props=None, prop_t=0, tab=None):
    """The closed reconstruction loop (or_closed_loop_clip) over luma y (n, ch,
    cw) and chroma u, v (n, ch/2, cw/2): per frame picks, costs, luma and
    chroma levels, the deblocked reconstruction and fallback flags."""
    n, ch, cw = y.shape
    nmb = (cw // 16) * (ch // 16)
    out = dict(picks=np.zeros((n, nmb, 6), np.int32), costs=np.zeros((n, nmb, 2), np.int64),
               coeffs=np.zeros((n, nmb, 256), np.int16), ccoeffs=np.zeros((n, nmb, 128), np.int16),
               rec_y=np.zeros_like(y), rec_u=np.zeros_like(u), rec_v=np.zeros_like(v),
               fallback=np.zeros((n, nmb), np.int32))
    tab = mv_cost_table() if tab is None else tab
    pr = None if props is None else np.ascontiguousarray(props, np.int32)
    yc, uc, vc = (np.ascontiguousarray(a) for a in (y, u, v))
    lib().or_closed_loop_clip(ptr(yc), ptr(uc), ptr(vc), n, cw, ch, pad, C.byref(params), ptr(tab, u16p),
                              float(lambda_me), int(split_gate), qp, dz_div, None if pr is None else ptr(pr, i32p),
                              int(prop_t), ptr(out["picks"], i32p), ptr(out["costs"], i64p), ptr(out["coeffs"], i16p),
                              ptr(out["ccoeffs"], i16p), ptr(out["rec_y"]), ptr(out["rec_u"]), ptr(out["rec_v"]),
                              ptr(out["fallback"], i32p))
    return out


class CavlcTables(C.Structure):
    """or_cavlc_tables of h264_decoder.c."""
    _fields_ = [("ct_len", (C.c_uint8 * 68) * 4), ("ct_bits", (C.c_uint8 * 68) * 4), ("cdc_len", C.c_uint8 * 20),
                ("cdc_bits", C.c_uint8 * 20), ("tz_len", (C.c_uint8 * 16) * 15), ("tz_bits", (C.c_uint8 * 16) * 15),
                ("ctz_len", (C.c_uint8 * 4) * 3), ("ctz_bits", (C.c_uint8 * 4) * 3), ("run_len", (C.c_uint8 * 15) * 7),
                ("run_bits", (C.c_uint8 * 15) * 7), ("cbp_inter", C.c_uint8 * 48)]


def reference_cavlc_tables():
    """The decoder's VLC tables, as parsed from the reference's cavlc.rs
    (tests/golden/reference_cavlc_tables.json)."""
    import json
    import os

    here = os.path.dirname(os.path.abspath(__file__))
    j = json.load(open(os.path.join(here, "..", "tests", "golden", "reference_cavlc_tables.json")))
    t = CavlcTables()
    flat = lambda a: [int(x) for row in (a if isinstance(a[0], list) else [a]) for x in row]
    for field, key in (("ct_len", "COEFF_TOKEN_LEN"), ("ct_bits", "COEFF_TOKEN_BITS"),
                       ("cdc_len", "CHROMA_DC_COEFF_TOKEN_LEN"), ("cdc_bits", "CHROMA_DC_COEFF_TOKEN_BITS"),
                       ("tz_len", "TOTAL_ZEROS_LEN"), ("tz_bits", "TOTAL_ZEROS_BITS"),
                       ("ctz_len", "CHROMA_DC_TOTAL_ZEROS_LEN"), ("ctz_bits", "CHROMA_DC_TOTAL_ZEROS_BITS"),
                       ("run_len", "RUN_LEN"), ("run_bits", "RUN_BITS"), ("cbp_inter", "CBP_INTER")):
        vals = flat(j[key])
        dst = getattr(t, field)
        C.memmove(C.addressof(dst), (C.c_uint8 * len(vals))(*vals), len(vals))
    return t


def decode_stream(data: bytes, cw: int, ch: int, max_frames: int):
    """Frames (y, u, v) and the parsed picks / levels of a stream of the
    library's subset (or_decode_stream); raises on a malformed stream."""
    L = lib()
    if not getattr(L, "_dec_ready", False):
        L.or_decode_stream.argtypes = [u8p, C.c_size_t, C.POINTER(CavlcTables), C.c_int, C.c_int, C.c_int, u8p, u8p,
                                       u8p, i32p, i16p, i16p]
        L._dec_ready = True
    nmb = (cw // 16) * (ch // 16)
    y = np.zeros((max_frames, ch, cw), np.uint8)
    u = np.zeros((max_frames, ch // 2, cw // 2), np.uint8)
    v = np.zeros_like(u)
    picks = np.zeros((max_frames, nmb, 6), np.int32)
    coeffs = np.zeros((max_frames, nmb, 256), np.int16)
    ccoeffs = np.zeros((max_frames, nmb, 128), np.int16)
    buf = np.frombuffer(data, np.uint8).copy()
    t = reference_cavlc_tables()
    n = L.or_decode_stream(ptr(buf), len(buf), C.byref(t), cw, ch, max_frames, ptr(y), ptr(u), ptr(v),
                           ptr(picks, i32p), ptr(coeffs, i16p), ptr(ccoeffs, i16p))
    if n < 0:
        raise ValueError(f"or_decode_stream: {n}")
    return dict(y=y[:n], u=u[:n], v=v[:n], picks=picks[:n], coeffs=coeffs[:n], ccoeffs=ccoeffs[:n])
