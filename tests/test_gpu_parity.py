"""GPU parity: every CUDA entry point against the CPU oracle, bit-exact.

All calls go through the C ABI (rusty_h264_b200.accel -> libh264accel_cuda.so).
Inputs are seeded synthetic clips (rusty_h264_b200.synth) and the reference
tests' LCG streams; the oracle is oracle/liboracle.so.  Integer work, so the
tolerance is zero everywhere.
"""
import ctypes as C
import zlib

import numpy as np
import pytest

from oracle import oracle as O
from rusty_h264_b200 import accel as A
from rusty_h264_b200 import synth
from tests._lcg import Lcg64

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    a = A.Accel(0)
    yield a
    a.close()


@pytest.fixture(scope="module")
def cif():
    y, _, _ = synth.cif_clip(5, 0)
    return synth.coded_luma(y)


def dev(acc, a):
    return acc.to_dev(np.ascontiguousarray(a))


# ---------------------------------------------------------------------------
# a1/a2 planes
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("cw,ch,pad", [(64, 48, 16), (80, 64, 12), (176, 144, 32), (352, 288, 32), (48, 32, 3),
                                       (16, 16, 32)])
def test_hpel_planes_match_oracle(acc, cw, ch, pad):
    st = Lcg64(0x5EED_F00D_DEAD_BEEF + cw)
    frames = st.bytes(2 * cw * ch).reshape(2, ch, cw).copy()
    got = acc.hpel_build(dev(acc, frames), pad=pad)
    acc.sync()
    got = got.cpu().numpy()
    for i in range(2):
        want = O.build_planes4(frames[i], pad)
        assert np.array_equal(got[i], want), (cw, ch, pad, i)


def test_hpel_planes_1080p(acc):
    y, _, _ = synth.hd_clip(2, 7)
    f = synth.coded_luma(y)
    got = acc.hpel_build(dev(acc, f), pad=32)
    acc.sync()
    got = got.cpu().numpy()
    for i in range(2):
        assert np.array_equal(got[i], O.build_planes4(f[i], 32))


# ---------------------------------------------------------------------------
# a6/a7/a8 block metrics (encoder tests/satd_avg_compare.rs streams)
# ---------------------------------------------------------------------------

def test_block_metrics_match_oracle(acc):
    st = Lcg64(0x0DD0_C0DE_1234_5678)
    L = O.lib()
    ss, rs = 40, 56
    src_rows, pl_rows = 64, 96
    src = st.bytes(src_rows * ss)
    planes = st.bytes(pl_rows * rs)
    d_src, d_pl = dev(acc, src), dev(acc, planes)
    for (w, h) in [(16, 16), (16, 8), (8, 16), (8, 8), (8, 4), (4, 8), (4, 4)]:
        n = 96
        rnd = lambda m: int(st.next()) % m
        a_off = np.array([rnd(src_rows - h) * ss + rnd(ss - w + 1) for _ in range(n)], np.int64)
        b_off = np.array([rnd(pl_rows - h) * rs + rnd(rs - w + 1) for _ in range(n)], np.int64)
        c_off = np.array([rnd(pl_rows - h) * rs + rnd(rs - w + 1) for _ in range(n)], np.int64)
        da, db, dc = dev(acc, a_off), dev(acc, b_off), dev(acc, c_off)
        for metric in (A.METRIC_SATD_WELS, A.METRIC_SATD, A.METRIC_SAD, A.METRIC_SATD_AVG, A.METRIC_SAD_AVG):
            avg = metric in (A.METRIC_SATD_AVG, A.METRIC_SAD_AVG)
            got = acc.block_metric(metric, w, h, d_src, da, ss, d_pl, db, rs, d_pl if avg else None,
                                   dc if avg else None)
            acc.sync()
            got = got.cpu().numpy()
            for i in range(n):
                a = np.ascontiguousarray(src[a_off[i]:])
                b = np.ascontiguousarray(planes[b_off[i]:])
                c = np.ascontiguousarray(planes[c_off[i]:])
                if metric == A.METRIC_SATD_WELS:
                    want = L.or_satd_region_wels(O.ptr(a), ss, O.ptr(b), rs, w, h)
                elif metric == A.METRIC_SATD:
                    want = L.or_satd_px(O.ptr(a), ss, O.ptr(b), rs, w, h)
                elif metric == A.METRIC_SAD:
                    want = L.or_sad(O.ptr(a), ss, O.ptr(b), rs, w, h)
                elif metric == A.METRIC_SATD_AVG:
                    want = L.or_satd_avg(O.ptr(a), ss, O.ptr(b), O.ptr(c), rs, w, h)
                else:
                    want = L.or_sad_avg(O.ptr(a), ss, O.ptr(b), O.ptr(c), rs, w, h)
                assert got[i] == want, (w, h, metric, i)


# ---------------------------------------------------------------------------
# a3/a4/a5/a9 candidate distortion
# ---------------------------------------------------------------------------

SHAPES = [(16, 16), (16, 8), (8, 16), (8, 8), (8, 4), (4, 8), (4, 4)]


def test_candidate_dist_matches_oracle_everywhere(acc, cif):
    src, ref = cif[1], cif[0]
    planes = O.build_planes4(ref, 32)
    d_src, d_pl = dev(acc, src), dev(acc, planes)
    d_pics, _ = acc.pictures([d_src], [d_pl])
    rng = np.random.default_rng(11)
    ch, cw = src.shape
    cands = []
    for _ in range(1500):
        w, h = SHAPES[rng.integers(len(SHAPES))]
        x = int(rng.integers(0, cw - w + 1))
        y = int(rng.integers(0, ch - h + 1))
        r = int(rng.choice([16, 200, 2000]))  # interior, beyond the pad, far off the planes
        cands.append(A.Candidate(0, x, y, w, h, int(rng.integers(-r, r + 1)), int(rng.integers(-r, r + 1))))
    for metric, kind in ((A.METRIC_SATD, 0), (A.METRIC_SAD, 1)):
        got = acc.candidate_dist(d_pics, 1, cands, metric)
        acc.sync()
        got = got.cpu().numpy()
        for i, c in enumerate(cands):
            want = O.candidate_dist(src, ref, planes, kind, c.x, c.y, c.w, c.h, c.mvx, c.mvy)
            assert got[i] == want, (metric, c.x, c.y, c.w, c.h, c.mvx, c.mvy)


def test_candidate_dist_rejects_out_of_range(acc, cif):
    d_src, d_pl = dev(acc, cif[1]), dev(acc, O.build_planes4(cif[0], 32))
    d_pics, _ = acc.pictures([d_src], [d_pl])
    bad = [A.Candidate(1, 0, 0, 16, 16, 0, 0), A.Candidate(0, 340, 0, 16, 16, 0, 0), A.Candidate(0, 0, 0, 32, 16, 0, 0),
           A.Candidate(0, -4, 0, 8, 8, 0, 0)]
    got = acc.candidate_dist(d_pics, 1, bad, A.METRIC_SATD)
    acc.sync()
    assert (got.cpu().numpy() == -1).all()


# ---------------------------------------------------------------------------
# a10/a11/a12 motion search
# ---------------------------------------------------------------------------

def me_variants():
    tab_smooth = O.mv_cost_table()
    rng = np.random.default_rng(5)
    tab_true = np.sort(rng.integers(4, 300, 4096)).astype(np.uint16)  # stand-in measured table
    tab_true[0] = 4
    return [
        ("balanced", {}, None),
        ("sadfp", {"sadfp": 1}, None),
        ("smooth_cost", {"mv_cost_kind": 1}, tab_smooth),
        ("sadfp_smooth", {"sadfp": 1, "mv_cost_kind": 1}, tab_smooth),
        ("true_cost", {"mv_cost_kind": 2}, tab_true),
        ("fast", {"fast": 1, "subpel": 0, "sp_single_pass": 0}, None),
        ("fast_subpel", {"fast": 1, "sp_single_pass": 0}, None),
        ("fast_satd", {"fast": 1, "mb_use_satd": 1, "subpel": 0, "sp_single_pass": 0}, None),
        ("sp_fc", {"sp_fc": 1}, None),
        ("sp_fc_walk", {"sp_fc": 1, "sp_single_pass": 0}, None),
        ("walk_to_convergence", {"sp_single_pass": 0}, None),
        ("ring4_walk", {"subpel_pat": 1}, None),
        ("ring4_single", {"subpel_pat": 3}, None),
        ("cascade_diamond", {"me_fc": 0}, None),
        ("no_snap", {"me_snap": 0}, None),
        ("sp_maxit1", {"sp_single_pass": 0, "sp_maxit": 1}, None),
        ("full_ladder", {"dia_mask": 0x1F, "dia_sub_mask": 0x1C}, None),
    ]


def oracle_params(ov):
    p = O.balanced_params()
    for k, v in ov.items():
        setattr(p, k, v)
    return p


def make_jobs(rng, cw, ch, n, refine_frac=0.1):
    jobs = []
    for _ in range(n):
        w, h = SHAPES[rng.integers(len(SHAPES))]
        x = int(rng.integers(0, cw // w)) * w
        y = int(rng.integers(0, ch // h)) * h
        npred = int(rng.integers(1, 5))
        preds = [int(v) for v in rng.integers(-40, 41, 2 * npred)]
        if rng.random() < 0.3:
            preds[0] = (preds[0] >> 2) * 4
            preds[1] = (preds[1] >> 2) * 4
        qp = int(rng.integers(22, 38))
        lam = np.sqrt(A.frame_lambda(qp)) * float(rng.choice([1.0, 1.25, 1.6]))
        j = A.MeJob()
        j.pic, j.x, j.y, j.w, j.h, j.npred = 0, x, y, w, h, npred
        for k, v in enumerate(preds):
            j.preds[k] = v
        if rng.random() < refine_frac:
            j.has_start = 1
            j.start[0], j.start[1] = int(rng.integers(-30, 31)), int(rng.integers(-30, 31))
        j.lambda_me = lam
        jobs.append(j)
    return jobs


@pytest.mark.parametrize("name,ov,tab", me_variants(), ids=[v[0] for v in me_variants()])
def test_me_search_matches_oracle(acc, cif, name, ov, tab):
    src, ref = cif[2], cif[1]
    planes = O.build_planes4(ref, 32)
    d_src, d_pl = dev(acc, src), dev(acc, planes)
    d_pics, _ = acc.pictures([d_src], [d_pl])
    d_tab = dev(acc, tab) if tab is not None else None
    params = A.default_me_params(**ov)
    if d_tab is not None:
        params.d_mv_cost_tab = d_tab.data_ptr()
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    ch, cw = src.shape
    jobs = make_jobs(rng, cw, ch, 300)
    raw = acc.me_search(d_pics, 1, params, jobs)
    acc.sync()
    got = acc.me_results(raw)
    op = oracle_params(ov)
    for i, j in enumerate(jobs):
        preds = list(j.preds)[:2 * j.npred]
        start = (j.start[0], j.start[1]) if j.has_start else None
        (mx, my), cost, _ = O.motion_search(src, ref, planes, op, j.x, j.y, j.w, j.h, preds, j.lambda_me, start=start,
                                            tab=tab if tab is not None else O.mv_cost_table())
        assert got[i, 4] == 0
        assert (got[i, 0], got[i, 1], got[i, 2]) == (mx, my, cost), (name, i, j.x, j.y, j.w, j.h, preds, start)


def test_me_search_known_answers(acc):
    """The hand-traced cases of test_search_known_answers (the fixed arm's
    lam_fp, the snap, the seed restore, the mid-ring centre move) through
    h264a_me_search: the same vectors, costs and evaluation counts."""
    import test_search_known_answers as K

    n = 64
    xx, yy = np.arange(n)[None, :], np.arange(n)[:, None]
    ref2 = (10 + 2 * xx + yy).astype(np.uint8)
    src2 = (ref2 + 3).astype(np.uint8)
    cases = [  # (src, ref, x, y, preds, lambda, knobs, expected)
        (K.ramp_src(6), K.REF, 32, [0, 0], 40.0, {"mv_cost_kind": 1}, ((0, 0), 1596, 6)),
        (K.ramp_src(6), K.REF, 32, [0, 0], 40.0, {}, ((12, 0), 400, 18)),
        (K.ramp_src(6), K.REF, 32, [0, 0], 10.0, {"mv_cost_kind": 1}, ((12, 0), 390, 18)),
        (K.ramp_src(4), K.REF, 32, [6, 0], 40.0, {}, ((8, 0), 240, 7)),
        (K.ramp_src(4), K.REF, 32, [6, 0], 40.0, {"me_snap": 0}, ((6, 0), 336, 6)),
        (K.ramp_src(1), K.REF, 32, [2, 0], 40.0, {}, ((2, 0), 80, 7)),
        (src2, ref2, 16, [0, 0], 4.0, {"me_fc": 0}, ((4, 4), 56, 10)),
        (src2, ref2, 16, [0, 0], 4.0, {}, ((4, 4), 56, 14)),
    ]
    d_tab = dev(acc, O.mv_cost_table())
    for src, ref, xy, preds, lam, kn, want in cases:
        d_src, d_pl = dev(acc, src), dev(acc, O.build_planes4(ref, 32))
        d_pics, _ = acc.pictures([d_src], [d_pl])
        params = A.default_me_params(dia_mask=0b10000, subpel=0, **kn)
        params.d_mv_cost_tab = d_tab.data_ptr()
        j = A.MeJob()
        j.pic, j.x, j.y, j.w, j.h, j.npred = 0, xy, xy, 16, 16, 1
        j.preds[0], j.preds[1] = preds
        j.lambda_me = lam
        raw = acc.me_search(d_pics, 1, params, [j])
        acc.sync()
        got = acc.me_results(raw)[0]
        assert got[4] == 0
        assert ((int(got[0]), int(got[1])), int(got[2]), int(got[3])) == want, (kn, want)


def test_me_search_rejects_bad_jobs(acc, cif):
    d_src, d_pl = dev(acc, cif[1]), dev(acc, O.build_planes4(cif[0], 32))
    d_pics, _ = acc.pictures([d_src], [d_pl])
    bad = []
    for (pic, x, w, npred) in [(3, 0, 16, 1), (0, 344, 16, 1), (0, 0, 12, 1), (0, 0, 16, 0), (0, 0, 16, 5)]:
        j = A.MeJob()
        j.pic, j.x, j.y, j.w, j.h, j.npred, j.lambda_me = pic, x, 0, w, 16, npred, 4.0
        bad.append(j)
    raw = acc.me_search(d_pics, 1, A.default_me_params(), bad)
    acc.sync()
    assert (acc.me_results(raw)[:, 4] == -1).all()


def run_me_frames(acc, pairs, params, lam, split_gate, tab=None, pad=32):
    """pairs: list of (src, ref) luma frames; returns [(picks, costs)] from the GPU."""
    frames, keep, outs = [], [], []
    for src, ref in pairs:
        ch, cw = src.shape
        nmb = (cw // 16) * (ch // 16)
        d_src, d_pl = dev(acc, src), acc.hpel_build(dev(acc, ref[None]), pad)[0]
        picks = acc.zeros((nmb, 6), acc.torch.int32)
        costs = acc.zeros((nmb, 2), acc.torch.int64)
        keep += [d_src, d_pl]
        outs.append((picks, costs))
        frames.append(A.MeFrame(A.Picture(d_src.data_ptr(), d_pl.data_ptr(), cw, ch, pad), lam, split_gate,
                                picks.data_ptr(), costs.data_ptr()))
    acc.me_frames(frames, params)
    acc.sync()
    return [(p.cpu().numpy(), c.cpu().numpy()) for p, c in outs]


@pytest.mark.parametrize("split", [False, True])
@pytest.mark.parametrize("variant", ["balanced", "sadfp_smooth"])
def test_me_frames_matches_oracle(acc, cif, split, variant):
    ov = {} if variant == "balanced" else {"sadfp": 1, "mv_cost_kind": 1}
    tab = O.mv_cost_table()
    params = A.default_me_params(**ov)
    d_tab = dev(acc, tab)
    params.d_mv_cost_tab = d_tab.data_ptr()
    qp = 26
    lam = float(np.sqrt(A.frame_lambda(qp)))
    gate = A.split_gate_for_qp(qp) if split else -1
    # a mixed-resolution batch: four CIF frame pairs plus a small 160x96 pair
    small = np.ascontiguousarray(cif[:, 32:128, 48:208])
    pairs = [(cif[f], cif[f - 1]) for f in range(1, 5)] + [(small[1], small[0])]
    got = run_me_frames(acc, pairs, params, lam, gate)
    op = oracle_params(ov)
    for (src, ref), (picks, costs) in zip(pairs, got):
        wp, wc = O.me_frame(src, ref, O.build_planes4(ref, 32), op, lam, gate, tab=tab)
        assert np.array_equal(picks[:, :5], wp[:, :5]), variant
        assert np.array_equal(costs, wc), variant


@pytest.mark.parametrize("prop_t", [0, 300, 1 << 30])
def test_me_frames_learned_matches_oracle(acc, prop_t):
    """The learned-proposal search (h264a_me_frames_learned) against the
    oracle's or_me_frame_learned on 4 CIF P frames in one launch: proposals
    scattered around each MB's plain pick (exact, a few pixels off, far off),
    the split gate on, at thresholds where every MB, some and none fall back."""
    torch = acc.torch
    y, _, _ = synth.cif_clip(5, 2)
    clip = synth.coded_luma(y)
    n, ch, cw = clip.shape
    nmb = (cw // 16) * (ch // 16)
    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    params = A.default_me_params()
    d = dev(acc, clip)
    planes = acc.hpel_build(d[: n - 1], 32)
    rng = np.random.default_rng(17)
    pl_np = planes.cpu().numpy()
    frames, outs, want = [], [], []
    for f in range(1, n):
        plain, _ = O.me_frame(clip[f], clip[f - 1], pl_np[f - 1], O.balanced_params(), lam, gate)
        props = np.zeros((nmb, 16), np.int32)
        for i in range(8):
            k = rng.integers(0, 3, nmb)
            off = np.where(k[:, None] == 0, 0, np.where(k[:, None] == 1, rng.integers(-3, 4, (nmb, 2)),
                                                         rng.integers(-8, 9, (nmb, 2))))
            props[:, 2 * i:2 * i + 2] = ((plain[:, 1:3] + 2) // 4 + off) * 4
        want.append(O.me_frame_learned(clip[f], clip[f - 1], pl_np[f - 1], O.balanced_params(), lam, props, prop_t,
                                       gate))
        d_props = dev(acc, props)
        pk = acc.zeros((nmb, 6), torch.int32)
        co = acc.zeros((nmb, 2), torch.int64)
        fb = torch.full((nmb,), -1, dtype=torch.int32, device="cuda:0")
        outs.append((d_props, pk, co, fb))
        frames.append(A.MeLearnedFrame(A.MeFrame(A.Picture(d[f].data_ptr(), planes[f - 1].data_ptr(), cw, ch, 32), lam,
                                                 gate, pk.data_ptr(), co.data_ptr()), d_props.data_ptr(), prop_t,
                                       fb.data_ptr()))
    acc.me_frames_learned(frames, params)
    acc.sync()
    fell_total = 0
    for (_, pk, co, fb), (wp, wc, wf) in zip(outs, want):
        assert np.array_equal(fb.cpu().numpy(), wf)
        assert np.array_equal(pk.cpu().numpy()[:, :5], wp[:, :5])
        assert np.array_equal(co.cpu().numpy(), wc)
        fell_total += int(wf.sum())
    if prop_t >= 1 << 30:
        assert fell_total == 0
    elif prop_t == 0:
        assert fell_total > 0


def _mr_case(acc, frames, srcs, refs_of, lam, gate, params):
    """GPU multi-reference picks for sources srcs (indices into frames) with
    reference lists refs_of[i] (nearest first), and the oracle's."""
    torch = acc.torch
    n, ch, cw = frames.shape
    nmb = (cw // 16) * (ch // 16)
    d = dev(acc, frames)
    planes = acc.hpel_build(d, 32)
    pk = acc.zeros((len(srcs), nmb, 8), torch.int32)
    co = acc.zeros((len(srcs), nmb, 2), torch.int64)
    fr = []
    for i, (sidx, refs) in enumerate(zip(srcs, refs_of)):
        f = A.MeMrFrame()
        f.d_src = d[sidx].data_ptr()
        for r, ri in enumerate(refs):
            f.d_planes[r] = planes[ri].data_ptr()
        f.nref, f.cw, f.ch, f.pad = len(refs), cw, ch, 32
        f.lambda_me, f.split_gate = lam, gate
        f.d_picks, f.d_costs = pk[i].data_ptr(), co[i].data_ptr()
        fr.append(f)
    acc.me_frames_multiref(fr, params)
    acc.sync()
    got_p, got_c = pk.cpu().numpy(), co.cpu().numpy()
    for i, (sidx, refs) in enumerate(zip(srcs, refs_of)):
        ro = np.stack([frames[r] for r in refs])
        po = np.stack([O.build_planes4(frames[r], 32) for r in refs])
        wp, wc = O.me_frame_multiref(frames[sidx], ro, po, O.balanced_params(), lam, gate)
        assert np.array_equal(got_p[i, :, :7], wp[:, :7]), (i, np.argwhere(got_p[i, :, :7] != wp[:, :7])[:4])
        assert np.array_equal(got_c[i], wc), i
    return got_p, got_c


def test_me_frames_multiref_matches_oracle(acc):
    """best_part over 3, 2 and 1 references (mb16.rs:4921-4960) in one
    launch: the reference indices, MVs and costs of every pick equal the
    oracle's, the picks use every reference, and with one reference the
    picks and costs are those of h264a_me_frames."""
    torch = acc.torch
    y, _, _ = synth.cif_clip(6, 13)
    clip = synth.coded_luma(y)
    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    params = A.default_me_params()
    got_p, got_c = _mr_case(acc, clip, [5, 4, 3, 2], [[4, 3, 2], [3, 2], [2], [1, 0]], lam, gate, params)
    assert set(np.unique(got_p[0, :, 1])) == {0, 1, 2}
    assert (got_p[:, :, 0] > 0).any()
    # one reference: the single-reference frame kernel's picks and costs
    n, ch, cw = clip.shape
    nmb = (cw // 16) * (ch // 16)
    d = dev(acc, clip)
    planes = acc.hpel_build(d, 32)
    pk = acc.zeros((nmb, 6), torch.int32)
    co = acc.zeros((nmb, 2), torch.int64)
    acc.me_frames([A.MeFrame(A.Picture(d[3].data_ptr(), planes[2].data_ptr(), cw, ch, 32), lam, gate,
                             pk.data_ptr(), co.data_ptr())], params)
    acc.sync()
    p1 = pk.cpu().numpy()
    assert np.array_equal(got_p[2][:, [0, 2, 3, 5, 6]], p1[:, :5]) and np.array_equal(got_c[2], co.cpu().numpy())
    assert np.array_equal(got_p[2][:, 7], p1[:, 5])  # the same evaluation counts


def oracle_mc_tq_multiref(src, refs, picks8, qp, dz_div=6):
    """MC + luma T/Q of multi-reference picks from the single-reference
    oracle: each 4x4 block's levels depend only on its source, its reference
    picture and its MV, so every MB is priced once per reference and each
    block taken from the reference of its half."""
    nmb = picks8.shape[0]
    p6 = np.zeros((nmb, 6), np.int32)
    p6[:, 0] = picks8[:, 0]
    p6[:, 1:3] = picks8[:, 2:4]
    p6[:, 3:5] = picks8[:, 5:7]
    out = np.zeros((nmb, 256), np.int16)
    shape = picks8[:, 0]
    for r, ref in enumerate(refs):
        c = O.mc_tq_frame(src, ref, p6, qp, dz_div)
        for by in range(0, 16, 4):
            for bx in range(0, 16, 4):
                part = np.where(shape == 1, by >= 8, np.where(shape == 2, bx >= 8, 0)).astype(int)
                ref_of = picks8[np.arange(nmb), 1 + 3 * part]
                off = ((2 if by >= 8 else 0) + (1 if bx >= 8 else 0)) * 64 + ((2 if by & 4 else 0) + (1 if bx & 4 else 0)) * 16
                sel = ref_of == r
                out[sel, off:off + 16] = c[sel, off:off + 16]
    return out


def test_mc_tq_frames_multiref_matches_oracle(acc):
    """MC + luma T/Q of multi-reference picks (each half from its own
    reference, the picks of a three-reference search) equals the
    single-reference oracle block by block."""
    torch = acc.torch
    y, _, _ = synth.cif_clip(6, 17)
    clip = synth.coded_luma(y)
    qp = 26
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    got_p, _ = _mr_case(acc, clip, [5, 3], [[4, 3, 2], [2, 1]], lam, A.split_gate_for_qp(qp), A.default_me_params())
    n, ch, cw = clip.shape
    nmb = (cw // 16) * (ch // 16)
    d = dev(acc, clip)
    planes = acc.hpel_build(d, 32)
    pk = dev(acc, got_p)
    co = acc.zeros((2, nmb, 256), torch.int16)
    fr = []
    for i, (sidx, refs) in enumerate(zip([5, 3], [[4, 3, 2], [2, 1]])):
        f = A.McTqMrFrame()
        f.d_src = d[sidx].data_ptr()
        for r, ri in enumerate(refs):
            f.d_planes[r] = planes[ri].data_ptr()
        f.nref, f.cw, f.ch, f.pad = len(refs), cw, ch, 32
        f.d_picks, f.qp, f.dz_div, f.d_coeffs = pk[i].data_ptr(), qp, 6, co[i].data_ptr()
        fr.append(f)
    acc.mc_tq_frames_multiref(fr)
    acc.sync()
    got = co.cpu().numpy()
    for i, (sidx, refs) in enumerate(zip([5, 3], [[4, 3, 2], [2, 1]])):
        want = oracle_mc_tq_multiref(clip[sidx], [clip[r] for r in refs], got_p[i], qp)
        assert np.array_equal(got[i], want), i
    assert (got != 0).any()


def test_me_frames_multiref_720p_three_references(acc):
    """A 1280x720 frame of the textured generator searched over its three
    previous frames equals the oracle."""
    y = synth.coded_luma(synth.hd_clip(5, 21, 1280, 720)[0])
    qp = 30
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    _mr_case(acc, y, [4], [[3, 2, 1]], lam, A.split_gate_for_qp(qp), A.default_me_params())


def test_me_frames_single_mb_and_flat(acc):
    flat = np.full((2, 16, 16), 90, np.uint8)
    rng = np.random.default_rng(3)
    tiny = rng.integers(0, 256, (2, 32, 48)).astype(np.uint8)
    params = A.default_me_params()
    pairs = [(flat[1], flat[0]), (tiny[1], tiny[0])]
    got = run_me_frames(acc, pairs, params, 5.0, 0)
    op = O.balanced_params()
    for (src, ref), (picks, costs) in zip(pairs, got):
        wp, wc = O.me_frame(src, ref, O.build_planes4(ref, 32), op, 5.0, 0)
        assert np.array_equal(picks[:, :5], wp[:, :5]) and np.array_equal(costs, wc)


@pytest.mark.parametrize("variant", ["balanced", "sadfp"])
def test_me_frames_more_than_96_frames_in_one_launch(acc, variant):
    """137 frames of three sizes in one call: more than a launch's parameters
    hold, so the frame table goes to device memory and one wavefront launch
    deals them all. Bit-exact with the oracle frame by frame, for the
    Balanced instance and the generic one."""
    params = A.default_me_params() if variant == "balanced" else A.default_me_params(sadfp=1)
    op = O.balanced_params() if variant == "balanced" else oracle_params({"sadfp": 1})
    lam = float(np.sqrt(A.frame_lambda(30)))
    gate = A.split_gate_for_qp(30)
    pairs = []
    for i, (w, h) in enumerate([(160, 96)] * 100 + [(352, 288)] * 7 + [(64, 48)] * 30):
        y, _, _ = synth.cif_clip(2, 50 + i, w, h)
        f = synth.coded_luma(y)
        pairs.append((f[1], f[0]))
    got = run_me_frames(acc, pairs, params, lam, gate)
    for k, ((src, ref), (picks, costs)) in enumerate(zip(pairs, got)):
        wp, wc = O.me_frame(src, ref, O.build_planes4(ref, 32), op, lam, gate)
        assert np.array_equal(picks[:, :5], wp[:, :5]) and np.array_equal(costs, wc), (k, src.shape)


def test_me_frames_2160p_720p_cif_in_one_launch(acc):
    """The resolutions of the multi-stream workload (CIF, 720p, 2160p) in one
    wavefront launch, frames of different sizes interleaving in the queue,
    bit-exact with the oracle (the 2160p pair alone is 32,400 MBs)."""
    params = A.default_me_params()
    lam = float(np.sqrt(A.frame_lambda(27)) * 1.25)
    gate = A.split_gate_for_qp(27)
    pairs = []
    for seed, (w, h) in ((1, (3840, 2160)), (2, (1280, 720)), (3, (352, 288))):
        y, _, _ = synth.cif_clip(2, seed, w, h)
        f = synth.coded_luma(y)
        pairs.append((f[1], f[0]))
    got = run_me_frames(acc, pairs, params, lam, gate)
    op = O.balanced_params()
    for (src, ref), (picks, costs) in zip(pairs, got):
        wp, wc = O.me_frame(src, ref, O.build_planes4(ref, 32), op, lam, gate)
        assert np.array_equal(picks[:, :5], wp[:, :5]) and np.array_equal(costs, wc), src.shape


@pytest.mark.parametrize("pad", [32, 35, 16])
def test_me_frames_window_edges(acc, cif, pad):
    """The per-MB shared-memory window and the plane path it falls back to:
    a large global shift puts seeds and ring points outside the window, a pad
    of 35 leaves plane rows off the 16-byte grid (no window at all), and a pad
    of 16 on a 16x16 frame makes the planes narrower than the window."""
    shifted = np.ascontiguousarray(np.roll(cif[2], (-17, 21), (0, 1)))
    tiny = np.ascontiguousarray(cif[2, 100:116, 200:216])
    tiny_ref = np.ascontiguousarray(cif[1, 100:116, 200:216])
    pairs = [(shifted, cif[2]), (cif[3], cif[2]), (tiny, tiny_ref)]
    lam = float(np.sqrt(A.frame_lambda(30)))
    gate = A.split_gate_for_qp(30)
    got = run_me_frames(acc, pairs, A.default_me_params(), lam, gate, pad=pad)
    op = O.balanced_params()
    for (src, ref), (picks, costs) in zip(pairs, got):
        wp, wc = O.me_frame(src, ref, O.build_planes4(ref, pad), op, lam, gate, pad=pad)
        assert np.array_equal(picks[:, :5], wp[:, :5]) and np.array_equal(costs, wc), pad


@pytest.mark.parametrize("R,stride", [(8, 7), (16, 29), (32, 53)])
def test_fullpel_grid_matches_oracle(acc, cif, R, stride):
    """SAD and SATD grids and both argmins against the oracle on a strided
    subset of MBs (and the last one): R = 8, 16 and 32, whose SAD launches
    take different numbers of MBs per CTA."""
    src, ref = cif[3], cif[2]
    planes = O.build_planes4(ref, 32)
    d_src, d_pl = dev(acc, src), dev(acc, planes)
    pic = A.Picture(d_src.data_ptr(), d_pl.data_ptr(), 352, 288, 32)
    nmb = 22 * 18
    rng = np.random.default_rng(9)
    centers = rng.integers(-64, 65, (nmb, 2)).astype(np.int32)
    pmv = rng.integers(-64, 65, (nmb, 2)).astype(np.int32)
    tab = O.mv_cost_table()
    lam = 6.5
    n = 2 * R + 1
    checked = list(range(0, nmb, stride)) + [nmb - 1]
    oracle_grids = {}
    for m in checked:
        mbx, mby = m % 22, m // 22
        cx, cy = (centers[m] + 2) >> 2
        ws = np.zeros(n * n, np.int32)
        wt = np.zeros(n * n, np.int32)
        for dy in range(-R, R + 1):
            for dx in range(-R, R + 1):
                i = (dy + R) * n + dx + R
                mvx, mvy = int(cx + dx) * 4, int(cy + dy) * 4
                ws[i] = O.candidate_dist(src, ref, planes, 1, mbx * 16, mby * 16, 16, 16, mvx, mvy)
                wt[i] = O.candidate_dist(src, ref, planes, 0, mbx * 16, mby * 16, 16, 16, mvx, mvy)
        oracle_grids[m] = (ws, wt)
    for metric in (0, 1):
        for kind in (0, 1):
            sad, satd, best = acc.fullpel_grid(pic, R, dev(acc, centers), dev(acc, pmv), metric, kind, dev(acc, tab),
                                               lam)
            acc.sync()
            sad, satd, best = sad.cpu().numpy(), satd.cpu().numpy(), best.cpu().numpy()
            for m in checked:
                cx, cy = (centers[m] + 2) >> 2
                ws, wt = oracle_grids[m]
                assert np.array_equal(sad[m], ws) and np.array_equal(satd[m], wt), m
                dist = ws if metric == 0 else wt
                bc, bi = None, None
                for i in range(n * n):  # raster order, strict <
                    dy, dx = i // n - R, i % n - R
                    mvx, mvy = int(cx + dx) * 4, int(cy + dy) * 4
                    rate = O.lib().or_mvbits(kind, O.ptr(tab, O.u16p), mvx - int(pmv[m, 0])) + \
                        O.lib().or_mvbits(kind, O.ptr(tab, O.u16p), mvy - int(pmv[m, 1]))
                    c = int(dist[i]) + int(lam * rate)
                    if bc is None or c < bc:
                        bc, bi = c, i
                dy, dx = bi // n - R, bi % n - R
                assert best[m].tolist() == [int(cx + dx) * 4, int(cy + dy) * 4, bc, int(dist[bi])], (m, metric, kind)


# ---------------------------------------------------------------------------
# a13/a14/a15 transform + quant
# ---------------------------------------------------------------------------

def test_dct_quant_4x4_matches_oracle(acc):
    rng = np.random.default_rng(21)
    src = rng.integers(0, 256, (64, 96)).astype(np.uint8)
    pred = rng.integers(0, 256, (64, 96)).astype(np.uint8)
    pred[:8, :8] = 0
    src[:8, :8] = 255
    n = 200
    xy = np.stack([rng.integers(0, 96 - 8, n), rng.integers(0, 64 - 8, n)], 1).astype(np.int32)
    xy[0] = (0, 0)
    qp = rng.integers(0, 52, n).astype(np.uint8)
    for dz in (6, 3, 2):
        got = acc.dct_quant_4x4(dev(acc, src), 96, dev(acc, pred), 96, dev(acc, xy), dev(acc, qp), dz)
        acc.sync()
        got = got.cpu().numpy()
        L = O.lib()
        for i in range(n):
            x, y = xy[i]
            d = np.zeros(64, np.int16)
            s = src.reshape(-1)[y * 96 + x:]
            p = pred.reshape(-1)[y * 96 + x:]
            L.or_dct_four_t4(O.ptr(d, O.i16p), O.ptr(s), 96, O.ptr(p), 96)
            ff, mf = np.zeros(8, np.int16), np.zeros(8, np.int16)
            L.or_quant_dz_ff(int(qp[i]), dz, O.ptr(ff, O.i16p))
            L.or_quant_mf_oh(int(qp[i]), O.ptr(mf, O.i16p))
            L.or_quant_four_4x4(O.ptr(d, O.i16p), O.ptr(ff, O.i16p), O.ptr(mf, O.i16p))
            assert np.array_equal(got[i], d), (i, dz)


def test_dct_quant_8x8_matches_oracle(acc):
    rng = np.random.default_rng(22)
    src = rng.integers(0, 256, (64, 96)).astype(np.uint8)
    pred = rng.integers(0, 256, (64, 96)).astype(np.uint8)
    n = 100
    xy = np.stack([rng.integers(0, 96 - 8, n), rng.integers(0, 64 - 8, n)], 1).astype(np.int32)
    qp = rng.integers(0, 52, n).astype(np.uint8)
    weights = [None, rng.integers(6, 40, 64).astype(np.int32)]
    L = O.lib()
    for wgt in weights:
        got = acc.dct_quant_8x8(dev(acc, src), 96, dev(acc, pred), 96, dev(acc, xy), dev(acc, qp), wgt, 6)
        acc.sync()
        got = got.cpu().numpy()
        w = np.full(64, 16, np.int32) if wgt is None else wgt
        for i in range(n):
            x, y = xy[i]
            res = (src[y:y + 8, x:x + 8].astype(np.int32) - pred[y:y + 8, x:x + 8]).reshape(-1).copy()
            c = np.zeros(64, np.int32)
            lv = np.zeros(64, np.int32)
            L.or_forward_core_8x8(O.ptr(res, O.i32p), O.ptr(c, O.i32p))
            L.or_quantize_8x8(O.ptr(c, O.i32p), int(qp[i]), O.ptr(w, O.i32p), 6, O.ptr(lv, O.i32p))
            assert np.array_equal(got[i], lv), i


def test_mc_tq_frames_matches_oracle(acc, cif):
    params = O.balanced_params()
    qp = 26
    lam = float(np.sqrt(A.frame_lambda(qp)))
    frames, keep, outs = [], [], []
    for f in (1, 2, 3):
        src, ref = cif[f], cif[f - 1]
        picks, _ = O.me_frame(src, ref, O.build_planes4(ref, 32), params, lam, A.split_gate_for_qp(qp))
        d_src, d_pl = dev(acc, src), acc.hpel_build(dev(acc, ref[None]), 32)[0]
        d_pk = dev(acc, picks)
        co = acc.zeros((picks.shape[0], 256), acc.torch.int16)
        keep += [d_src, d_pl, d_pk]
        outs.append((co, src, ref, picks, qp + f))
        frames.append(A.TqFrame(A.Picture(d_src.data_ptr(), d_pl.data_ptr(), 352, 288, 32), d_pk.data_ptr(), qp + f, 6,
                                co.data_ptr()))
    acc.mc_tq_frames(frames)
    acc.sync()
    for co, src, ref, picks, q in outs:
        assert np.array_equal(co.cpu().numpy(), O.mc_tq_frame(src, ref, picks, q, 6))


@pytest.mark.parametrize("split", [False, True])
def test_me_tq_frames_matches_oracle(acc, cif, split):
    """Plain-ME with each MB's MC + luma T/Q in the same launch: picks, costs
    and coefficients bit-exact with the oracle's me_frame + mc_tq_frame.  The
    batch mixes CIF pairs at three QPs, a 160x96 pair, and a pair whose
    reference is the source moved by (21, 9) pixels, so that early MBs' final
    MVs lie outside the staged window and their prediction comes from the
    planes."""
    params = A.default_me_params()
    lam = float(np.sqrt(A.frame_lambda(26)))
    gate = A.split_gate_for_qp(26) if split else -1
    moved = np.ascontiguousarray(np.roll(cif[2], (9, 21), (0, 1)))
    small = np.ascontiguousarray(cif[:, 32:128, 48:208])
    pairs = [(cif[1], cif[0], 22), (cif[2], cif[1], 30), (cif[3], cif[2], 40), (small[1], small[0], 27),
             (cif[2], moved, 26)]
    frames, keep, outs = [], [], []
    for src, ref, q in pairs:
        ch, cw = src.shape
        nmb = (cw // 16) * (ch // 16)
        d_src, d_pl = dev(acc, src), acc.hpel_build(dev(acc, ref[None]), 32)[0]
        picks = acc.zeros((nmb, 6), acc.torch.int32)
        costs = acc.zeros((nmb, 2), acc.torch.int64)
        co = acc.zeros((nmb, 256), acc.torch.int16)
        keep += [d_src, d_pl]
        outs.append((picks, costs, co, src, ref, q))
        me = A.MeFrame(A.Picture(d_src.data_ptr(), d_pl.data_ptr(), cw, ch, 32), lam, gate, picks.data_ptr(),
                       costs.data_ptr())
        frames.append(A.MeTqFrame(me, q, 6, co.data_ptr()))
    acc.me_tq_frames(frames, params)
    acc.sync()
    for picks, costs, co, src, ref, q in outs:
        wp, wc = O.me_frame(src, ref, O.build_planes4(ref, 32), O.balanced_params(), lam, gate)
        assert np.array_equal(picks.cpu().numpy()[:, :5], wp[:, :5]) and np.array_equal(costs.cpu().numpy(), wc), q
        assert np.array_equal(co.cpu().numpy(), O.mc_tq_frame(src, ref, wp, q, 6)), q


@pytest.mark.parametrize("qp", [0, 10, 24, 30, 51])
def test_mc_tq_rec_frames_matches_oracle(acc, cif, qp):
    """MC + T/Q with the luma reconstruction (mb16.rs:3575-3605): coefficients
    and reconstructed frames bit-exact with the oracle, across the qp < 24 and
    qp >= 24 dequant arms."""
    params = O.balanced_params()
    lam = float(np.sqrt(A.frame_lambda(max(qp, 12))))
    frames, keep, outs = [], [], []
    for f in (1, 2):
        src, ref = cif[f], cif[f - 1]
        picks, _ = O.me_frame(src, ref, O.build_planes4(ref, 32), params, lam, A.split_gate_for_qp(max(qp, 12)))
        d_src, d_pl = dev(acc, src), acc.hpel_build(dev(acc, ref[None]), 32)[0]
        d_pk = dev(acc, picks)
        co = acc.zeros((picks.shape[0], 256), acc.torch.int16)
        rec = acc.torch.full((288, 352), 7, dtype=acc.torch.uint8, device="cuda:0")
        keep += [d_src, d_pl, d_pk]
        outs.append((co, rec, src, ref, picks))
        tq = A.TqFrame(A.Picture(d_src.data_ptr(), d_pl.data_ptr(), 352, 288, 32), d_pk.data_ptr(), qp, 6,
                       co.data_ptr())
        frames.append(A.TqRecFrame(tq, rec.data_ptr()))
    acc.mc_tq_rec_frames(frames)
    acc.sync()
    for co, rec, src, ref, picks in outs:
        wc, wr = O.mc_tq_rec_frame(src, ref, picks, qp, 6)
        assert np.array_equal(co.cpu().numpy(), wc)
        assert np.array_equal(rec.cpu().numpy(), wr)
    # the reconstruction is the prediction plus a bounded error
    assert np.abs(outs[0][1].cpu().numpy().astype(int) - cif[1].astype(int)).mean() < (40 if qp > 40 else 12)


@pytest.mark.parametrize("qp", [0, 20, 29, 30, 36, 51])
def test_mc_tq_chroma_frames_matches_oracle(acc, qp):
    """The inter MB's chroma MC + T/Q (with the 2x2 DC) and reconstruction,
    bit-exact with the oracle for every pick shape, across the chroma-QP map
    and both dequant arms; one frame without reconstruction."""
    y, _, _ = synth.cif_clip(4, 1)
    luma = synth.coded_luma(y)
    # textured chroma: the half-res luma, and its negative shifted by a few pixels
    u = np.stack([O.downsample2x(a) for a in luma])
    v = np.ascontiguousarray(255 - np.roll(u, (3, -5), (1, 2)))
    lam = float(np.sqrt(A.frame_lambda(max(qp, 12))))
    frames, keep, outs = [], [], []
    for f in (1, 2, 3):
        src, ref = luma[f], luma[f - 1]
        picks, _ = O.me_frame(src, ref, O.build_planes4(ref, 32), O.balanced_params(), lam, 0)
        # force every shape: the search's picks, then 16x8 and 8x16 with distinct MVs
        if f == 2:
            picks[::3, 0] = 1
            picks[1::3, 0] = 2
            picks[:, 3] = picks[:, 1] + 5
            picks[:, 4] = picks[:, 2] - 3
        d = [dev(acc, a) for a in (u[f], v[f], u[f - 1], v[f - 1], picks)]
        co = acc.zeros((picks.shape[0], 128), acc.torch.int16)
        want_rec = f != 3
        ru = acc.torch.full((144, 176), 3, dtype=acc.torch.uint8, device="cuda:0") if want_rec else None
        rv = acc.torch.full((144, 176), 3, dtype=acc.torch.uint8, device="cuda:0") if want_rec else None
        keep += d + [co, ru, rv]
        outs.append((co, ru, rv, f, picks))
        frames.append(A.TqChromaFrame(d[0].data_ptr(), d[1].data_ptr(), d[2].data_ptr(), d[3].data_ptr(), 352, 288,
                                      d[4].data_ptr(), qp, co.data_ptr(), ru.data_ptr() if want_rec else None,
                                      rv.data_ptr() if want_rec else None))
    acc.mc_tq_chroma_frames(frames)
    acc.sync()
    for co, ru, rv, f, picks in outs:
        wc, wu, wv = O.mc_tq_chroma_frame(u[f], v[f], u[f - 1], v[f - 1], picks, qp)
        assert np.array_equal(co.cpu().numpy(), wc), (qp, f)
        if ru is not None:
            assert np.array_equal(ru.cpu().numpy(), wu) and np.array_equal(rv.cpu().numpy(), wv), (qp, f)


@pytest.mark.parametrize("qp,offs", [(22, (0, 0, 0)), (30, (0, 0, 0)), (36, (2, -1, 3)), (45, (-2, 3, -4)), (51, (0, 0, 0))])
def test_deblock_frames_matches_oracle(acc, qp, offs):
    """In-loop deblocking of reconstructed plain-ME pictures, bit-exact with
    the oracle: three CIF pictures with chroma and a 160x96 one luma-only, in
    one wavefront launch; picks forced through every shape on one picture."""
    y, _, _ = synth.cif_clip(4, 2)
    luma = synth.coded_luma(y)
    half = np.stack([O.downsample2x(a) for a in luma])
    lam = float(np.sqrt(A.frame_lambda(qp)))
    frames, keep, cases = [], [], []
    for f in (1, 2, 3, 4):
        small = f == 4
        src, ref = (np.ascontiguousarray(luma[1, 64:160, 96:256]), np.ascontiguousarray(luma[0, 64:160, 96:256])) \
            if small else (luma[f], luma[f - 1])
        picks, _ = O.me_frame(src, ref, O.build_planes4(ref, 32), O.balanced_params(), lam, A.split_gate_for_qp(qp))
        if f == 2:
            picks[::3, 0] = 1
            picks[1::3, 0] = 2
            picks[:, 3] = picks[:, 1] + 5
            picks[:, 4] = picks[:, 2] - 3
        coeffs, rec = O.mc_tq_rec_frame(src, ref, picks, qp, 6)
        ch, cw = src.shape
        if small:
            ru = rv = None
        else:
            _, ru, rv = O.mc_tq_chroma_frame(half[f], 255 - half[f], half[f - 1], 255 - half[f - 1], picks, qp)
        dy = dev(acc, rec)
        du, dv = (dev(acc, ru), dev(acc, rv)) if ru is not None else (None, None)
        dp, dc = dev(acc, picks), dev(acc, coeffs)
        keep += [dy, du, dv, dp, dc]
        cases.append((dy, du, dv, rec, ru, rv, picks, coeffs))
        frames.append(A.DeblockFrame(dy.data_ptr(), du.data_ptr() if du is not None else None,
                                     dv.data_ptr() if dv is not None else None, cw, ch, dp.data_ptr(), dc.data_ptr(),
                                     qp, *offs))
    acc.deblock_frames(frames)
    acc.sync()
    changed = 0
    for dy, du, dv, rec, ru, rv, picks, coeffs in cases:
        wy, wu, wv = O.deblock_frame(rec, ru, rv, picks, coeffs, qp, *offs)
        got = dy.cpu().numpy()
        assert np.array_equal(got, wy), qp
        changed += int((wy != rec).sum())
        if du is not None:
            assert np.array_equal(du.cpu().numpy(), wu) and np.array_equal(dv.cpu().numpy(), wv), qp
    assert changed > 0  # the filter did something on these pictures


def test_deblock_frames_1080p_wavefront(acc):
    """Six 1920x1088 pictures with chroma in one wavefront launch, so that
    thousands of MB tickets are in flight at once, bit-exact with the oracle.
    Picks are seeded synthetic ones (every shape, MVs around the clip's
    background motion, some far off) and the pictures are the oracle's
    reconstruction from them, so bS 0, 1 and 2 all occur."""
    qp, w, h = 34, 1920, 1088
    y, _, _ = synth.hd_clip(7, 3, w, h)
    luma = synth.coded_luma(y)
    half = np.stack([O.downsample2x(a) for a in luma])
    rng = np.random.default_rng(11)
    nmb = (w // 16) * (h // 16)
    frames, keep, cases = [], [], []
    for f in range(1, 7):
        picks = np.zeros((nmb, 6), np.int32)
        picks[:, 0] = rng.integers(0, 3, nmb)
        jit = rng.integers(-8, 9, (nmb, 2)) * (rng.random((nmb, 1)) < 0.4)
        picks[:, 1:3] = np.array([-5, 2]) + jit
        jit1 = rng.integers(-6, 7, (nmb, 2)) * (rng.random((nmb, 1)) < 0.5)
        picks[:, 3:5] = np.where(picks[:, :1] == 0, picks[:, 1:3], picks[:, 1:3] + jit1)
        coeffs, rec = O.mc_tq_rec_frame(luma[f], luma[f - 1], picks, qp, 6)
        _, ru, rv = O.mc_tq_chroma_frame(half[f], 255 - half[f], half[f - 1], 255 - half[f - 1], picks, qp)
        dy, du, dv, dp, dc = (dev(acc, a) for a in (rec, ru, rv, picks, coeffs))
        keep += [dy, du, dv, dp, dc]
        cases.append((dy, du, dv, rec, ru, rv, picks, coeffs))
        frames.append(A.DeblockFrame(dy.data_ptr(), du.data_ptr(), dv.data_ptr(), w, h, dp.data_ptr(), dc.data_ptr(),
                                     qp, 0, 0, 0))
    acc.deblock_frames(frames)
    acc.sync()
    for k, (dy, du, dv, rec, ru, rv, picks, coeffs) in enumerate(cases):
        wy, wu, wv = O.deblock_frame(rec, ru, rv, picks, coeffs, qp)
        assert (wy != rec).sum() > 1000
        assert np.array_equal(dy.cpu().numpy(), wy), k
        assert np.array_equal(du.cpu().numpy(), wu) and np.array_equal(dv.cpu().numpy(), wv), k


def test_deblock_frames_mixed_sizes_wavefront(acc):
    """A 1920x1088 picture, a CIF one and a 160x96 one in one wavefront
    launch: the 1080p picture alone has more MBs (8,160) than the kernel keeps
    resident, so its tail tickets must be dealt after the segments that hold
    every picture's first MBs. Bit-exact with the oracle."""
    qp = 31
    rng = np.random.default_rng(5)
    frames, keep, cases = [], [], []
    for seed, (w, h) in ((4, (160, 96)), (5, (1920, 1088)), (6, (352, 288))):
        y, _, _ = synth.cif_clip(2, seed, w, h)
        luma = synth.coded_luma(y)
        half = np.stack([O.downsample2x(a) for a in luma])
        nmb = (w // 16) * (h // 16)
        picks = np.zeros((nmb, 6), np.int32)
        picks[:, 0] = rng.integers(0, 3, nmb)
        picks[:, 1:3] = rng.integers(-9, 10, (nmb, 2))
        picks[:, 3:5] = np.where(picks[:, :1] == 0, picks[:, 1:3], picks[:, 1:3] + rng.integers(-4, 5, (nmb, 2)))
        coeffs, rec = O.mc_tq_rec_frame(luma[1], luma[0], picks, qp, 6)
        _, ru, rv = O.mc_tq_chroma_frame(half[1], 255 - half[1], half[0], 255 - half[0], picks, qp)
        dy, du, dv, dp, dc = (dev(acc, a) for a in (rec, ru, rv, picks, coeffs))
        keep += [dy, du, dv, dp, dc]
        cases.append((dy, du, dv, rec, ru, rv, picks, coeffs))
        frames.append(A.DeblockFrame(dy.data_ptr(), du.data_ptr(), dv.data_ptr(), w, h, dp.data_ptr(), dc.data_ptr(),
                                     qp, 0, 0, 0))
    acc.deblock_frames(frames)
    acc.sync()
    for k, (dy, du, dv, rec, ru, rv, picks, coeffs) in enumerate(cases):
        wy, wu, wv = O.deblock_frame(rec, ru, rv, picks, coeffs, qp)
        assert (wy != rec).sum() > 0
        assert np.array_equal(dy.cpu().numpy(), wy), k
        assert np.array_equal(du.cpu().numpy(), wu) and np.array_equal(dv.cpu().numpy(), wv), k


# ---------------------------------------------------------------------------
# a16-a19 lookahead
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("mode", [2, 1, 0])
def test_lookahead_matches_oracle(acc, cif, mode):
    full = dev(acc, cif)
    half = acc.downsample2x(full)
    acc.sync()
    assert np.array_equal(half.cpu().numpy(), np.stack([O.downsample2x(f) for f in cif]))
    intra, inter, mvs = acc.lookahead_costs(full, half, mode)
    acc.sync()
    wi, wn, wm = O.lookahead_clip(cif, mode)
    assert np.array_equal(intra.cpu().numpy(), wi)
    assert np.array_equal(inter.cpu().numpy(), wn)
    assert np.array_equal(mvs.cpu().numpy(), wm)


@pytest.mark.parametrize("cw,ch,pan", [(352, 288, (44, 26)), (208, 144, (6, -4))])
def test_lookahead_window_misses_and_no_window(acc, cw, ch, pan):
    """HalfRes searches on a panning texture: a 44x26-pixel pan per frame
    walks candidates out of the block's shared-memory window (they read the
    clamped picture instead), and a 208-pixel clip has 104-byte half-res rows,
    which no tensor map can describe, so it searches without windows. All
    three outputs bit-exact with the oracle."""
    rng = np.random.default_rng(cw)
    H, W = ch + 4 * abs(pan[1]) + 16, cw + 4 * abs(pan[0]) + 16
    tex = rng.random((H, W))
    for _ in range(3):  # smooth it, so that the diamond can follow the pan
        tex = (tex + np.roll(tex, 1, 0) + np.roll(tex, 1, 1) + np.roll(tex, (1, 1), (0, 1))) / 4
    tex = (255 * (tex - tex.min()) / (tex.max() - tex.min())).astype(np.uint8)
    oy, ox = 2 * abs(pan[1]) + 8, 2 * abs(pan[0]) + 8
    clip = np.stack([tex[oy + k * pan[1]:oy + k * pan[1] + ch, ox + k * pan[0]:ox + k * pan[0] + cw] for k in range(3)])
    clip = np.ascontiguousarray(clip)
    full = dev(acc, clip)
    half = acc.downsample2x(full)
    intra, inter, mvs = acc.lookahead_costs(full, half, 2)
    acc.sync()
    wi, wn, wm = O.lookahead_clip(clip, 2)
    assert np.array_equal(intra.cpu().numpy(), wi)
    assert np.array_equal(inter.cpu().numpy(), wn)
    assert np.array_equal(mvs.cpu().numpy(), wm)
    if pan[0] > 16:
        assert (np.abs(wm[1:, :, 0]) >= 32).mean() > 0.25  # the search follows the pan past the window


@pytest.mark.parametrize("mode", [2, 0])
def test_lookahead_streams_one_launch(acc, mode):
    """h264a_lookahead_streams over four clips of three sizes and lengths
    (CIF x 5, 208x144 x 3 without windows, 384x272 x 6, and a one-frame clip,
    intra only) gives, stream by stream, what h264a_lookahead_costs gives each
    alone, and the CIF stream equals the oracle."""
    torch = acc.torch
    cif = synth.coded_luma(synth.cif_clip(5, 3)[0])
    hd = synth.coded_luma(synth.hd_clip(6, 4, 384, 272)[0])
    rng = np.random.default_rng(9)
    small = rng.integers(0, 256, (3, 144, 208)).astype(np.uint8)
    one = rng.integers(0, 256, (1, 64, 96)).astype(np.uint8)
    clips, keep, streams, alone = [cif, small, hd, one], [], [], []
    for c in clips:
        n, ch, cw = c.shape
        nmb = (cw // 16) * (ch // 16)
        full = dev(acc, c)
        half = acc.downsample2x(full)
        outs = [acc.zeros((n, nmb), torch.int32), acc.zeros((n, nmb), torch.int32), acc.zeros((n, nmb, 2), torch.int32)]
        keep.append((full, half, outs))
        streams.append(A.LaStream(full.data_ptr(), half.data_ptr(), cw, ch, n, outs[0].data_ptr(), outs[1].data_ptr(),
                                  outs[2].data_ptr()))
        i1, n1, m1 = acc.lookahead_costs(full, half, mode)
        acc.sync()
        alone.append((i1.cpu().numpy(), n1.cpu().numpy(), m1.cpu().numpy()))
    acc.lookahead_streams(streams, mode)
    acc.sync()
    for k, (_, _, outs) in enumerate(keep):
        got = [o.cpu().numpy() for o in outs]
        for g, a in zip(got, alone[k]):
            assert np.array_equal(g, a), (mode, k)
    wi, wn, wm = O.lookahead_clip(cif, mode)
    assert np.array_equal(alone[0][0], wi) and np.array_equal(alone[0][1], wn) and np.array_equal(alone[0][2], wm)


def test_lookahead_streams_more_than_one_launch(acc):
    """26 small clips (more than the 24 streams one launch takes) of 2 to 4
    frames: two chains launches, each stream equal to the oracle."""
    torch = acc.torch
    rng = np.random.default_rng(21)
    keep, streams, clips = [], [], []
    for k in range(26):
        n, ch, cw = 2 + k % 3, 32 + 16 * (k % 2), 48 + 16 * (k % 3)
        base = rng.integers(0, 256, (ch + 8, cw + 8)).astype(np.uint8)
        c = np.ascontiguousarray(np.stack([base[f % 3: f % 3 + ch, f: f + cw] for f in range(n)]))
        nmb = (cw // 16) * (ch // 16)
        full = dev(acc, c)
        half = acc.downsample2x(full)
        outs = [acc.zeros((n, nmb), torch.int32), acc.zeros((n, nmb), torch.int32), acc.zeros((n, nmb, 2), torch.int32)]
        keep.append(outs)
        keep.append((full, half))
        clips.append((c, outs))
        streams.append(A.LaStream(full.data_ptr(), half.data_ptr(), cw, ch, n, outs[0].data_ptr(), outs[1].data_ptr(),
                                  outs[2].data_ptr()))
    acc.lookahead_streams(streams, 2)
    acc.sync()
    for k, (c, outs) in enumerate(clips):
        wi, wn, wm = O.lookahead_clip(c, 2)
        got = [o.cpu().numpy() for o in outs]
        assert np.array_equal(got[0], wi) and np.array_equal(got[1], wn) and np.array_equal(got[2], wm), k


def test_lookahead_flat_and_static(acc):
    flat = np.full((3, 32, 32), 77, np.uint8)
    full = dev(acc, flat)
    half = acc.downsample2x(full)
    intra, inter, mvs = acc.lookahead_costs(full, half, 2)
    acc.sync()
    wi, wn, wm = O.lookahead_clip(flat, 2)
    assert np.array_equal(intra.cpu().numpy(), wi) and (wi == 1).all()
    assert np.array_equal(inter.cpu().numpy(), wn) and np.array_equal(mvs.cpu().numpy(), wm)


def test_lookahead_beside_me_in_one_context(acc):
    """The lookahead has a work queue of its own in a context, so it may run
    on a second stream while plain-ME runs on the first; both give the
    results of the same calls made one after the other, on ten 1080p
    frames."""
    torch = acc.torch
    y, _, _ = synth.hd_clip(10, 2)
    f = synth.coded_luma(y)
    n, ch, cw = f.shape
    nmb = (cw // 16) * (ch // 16)
    d = dev(acc, f)
    planes = acc.hpel_build(d[: n - 1], 32)
    half = acc.downsample2x(d)
    acc.sync()
    params = A.default_me_params()
    lam = float(np.sqrt(A.frame_lambda(27)) * 1.25)
    gate = A.split_gate_for_qp(27)
    runs = []
    for concurrent in (False, True):
        picks = acc.zeros((n, nmb, 6), torch.int32)
        costs = acc.zeros((n, nmb, 2), torch.int64)
        frames = [A.MeFrame(A.Picture(d[i].data_ptr(), planes[i - 1].data_ptr(), cw, ch, 32), lam, gate,
                            picks[i].data_ptr(), costs[i].data_ptr()) for i in range(1, n)]
        main, side = torch.cuda.current_stream(), torch.cuda.Stream()
        side.wait_stream(main)
        if concurrent:
            with torch.cuda.stream(side):
                la = acc.lookahead_costs(d, half, 2)
            acc.me_frames(frames, params)
        else:
            acc.me_frames(frames, params)
            la = acc.lookahead_costs(d, half, 2)
        main.wait_stream(side)
        torch.cuda.synchronize()
        acc.sync()
        runs.append([picks, costs, *la])
    for a, b in zip(*runs):
        assert torch.equal(a, b)


# ---------------------------------------------------------------------------
# The whole path through the host-buffer entry point
# ---------------------------------------------------------------------------

def compare_pixel_path(got, want):
    for k in ("picks", "costs", "coeffs", "la_intra", "la_inter", "la_mvs"):
        g, w = got[k], want[k]
        if k == "picks":
            g, w = g[..., :5], w[..., :5]
        assert np.array_equal(g, w), k


def test_pixel_path_host_cif_matches_oracle(acc, cif):
    params = A.default_me_params()
    qp = 26
    lam = float(np.sqrt(A.frame_lambda(qp)))
    gate = A.split_gate_for_qp(qp)
    got = acc.pixel_path_host(cif, params, lam, gate, qp)
    want = O.pixel_path_clip(cif, O.balanced_params(), lam, gate, qp, nthreads=4)
    compare_pixel_path(got, want)


def test_pixel_path_host_40_frames_matches_oracle(acc):
    """40 CIF frames through the host-buffer entry point (39 P frames in one
    wavefront launch)."""
    y, _, _ = synth.cif_clip(40, 5)
    frames = synth.coded_luma(y)
    params = A.default_me_params()
    qp = 30
    lam = float(np.sqrt(A.frame_lambda(qp)))
    gate = A.split_gate_for_qp(qp)
    got = acc.pixel_path_host(frames, params, lam, gate, qp)
    want = O.pixel_path_clip(frames, O.balanced_params(), lam, gate, qp, nthreads=8)
    compare_pixel_path(got, want)


def test_pixel_path_host_pinned_outputs_matches_oracle(acc):
    """Outputs in pinned host memory, where the bands of finished MB rows
    come down while the launch still runs: the results equal the oracle's,
    frame 0's rows are zero, and a second call into the same buffers (filled
    with -1 at first) gives the same."""
    torch = acc.torch
    y, _, _ = synth.cif_clip(12, 9)
    frames = synth.coded_luma(y)
    n, ch, cw = frames.shape
    nmb = (cw // 16) * (ch // 16)
    params = A.default_me_params()
    qp = 28
    lam = float(np.sqrt(A.frame_lambda(qp)))
    gate = A.split_gate_for_qp(qp)
    out = {k: torch.full(shape, -1, dtype=dt).pin_memory().numpy() for k, shape, dt in (
        ("picks", (n, nmb, 6), torch.int32), ("costs", (n, nmb, 2), torch.int64),
        ("coeffs", (n, nmb, 256), torch.int16), ("la_intra", (n, nmb), torch.int32),
        ("la_inter", (n, nmb), torch.int32), ("la_mvs", (n, nmb, 2), torch.int32))}
    for _ in range(2):  # a second call into the same buffers
        got = acc.pixel_path_host(frames, params, lam, gate, qp, out=out)
        want = O.pixel_path_clip(frames, O.balanced_params(), lam, gate, qp, nthreads=8)
        compare_pixel_path(got, want)
        assert (got["picks"][0] == 0).all() and (got["coeffs"][0] == 0).all() and (got["costs"][0] == 0).all()


def test_pixel_path_prefetch_matches_oracle(acc):
    """Batches uploaded ahead of their calls by pixel_path_prefetch (pinned
    host frames): every call equals the oracle. Covered: two pending
    prefetches, a third refused, a call whose frames match none of them (it
    uploads them itself and gives up the newer prefetch), a prefetch of another
    geometry, and the streaming loop on one buffer (prefetch k+1, then call k)."""
    torch = acc.torch
    params, qp = A.default_me_params(), 28
    lam = float(np.sqrt(A.frame_lambda(qp)))
    gate = A.split_gate_for_qp(qp)
    clips = [synth.coded_luma(synth.cif_clip(5, seed)[0]) for seed in (3, 4, 5)]
    clips.append(synth.coded_luma(synth.cif_clip(4, 6, 176, 144)[0]))
    a, b, c, s = (torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy() for x in clips)
    want = [O.pixel_path_clip(x, O.balanced_params(), lam, gate, qp, nthreads=8) for x in (a, b, c, s)]
    run = lambda x: acc.pixel_path_host(x, params, lam, gate, qp)
    acc.pixel_path_prefetch(a)
    acc.pixel_path_prefetch(b)
    with pytest.raises(A.AccelError):
        acc.pixel_path_prefetch(c)  # two uploads are already pending
    compare_pixel_path(run(c), want[2])
    compare_pixel_path(run(a), want[0])
    acc.pixel_path_prefetch(s)
    compare_pixel_path(run(b), want[1])
    compare_pixel_path(run(s), want[3])
    acc.pixel_path_prefetch(a)
    for k in range(3):
        if k < 2:
            acc.pixel_path_prefetch(a)
        compare_pixel_path(run(a), want[0])
    assert acc._prefetched == []


def test_pixel_path_host_1080p_matches_oracle(acc):
    y, _, _ = synth.hd_clip(3, 1)
    frames = synth.coded_luma(y)
    params = A.default_me_params()
    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    got = acc.pixel_path_host(frames, params, lam, gate, qp)
    want = O.pixel_path_clip(frames, O.balanced_params(), lam, gate, qp, nthreads=8)
    compare_pixel_path(got, want)
    # size-independent properties of the full-size output
    assert (got["picks"][1:, :, 0] <= 2).all()
    assert (got["la_inter"] <= got["la_intra"]).all() and (got["la_intra"] >= 1).all()


def test_bench_workload_matches_oracle(acc):
    """The benchmarked workload itself: the seed-1 1080p clip of 60 frames, QP
    27, lme = sqrt(lambda)*1.25, partitions on, Balanced preset, through
    h264a_pixel_path_host as bench.py's e2e leg runs it.  In this frame model
    P frame f depends only on source frames f and f-1, so the oracle run on
    the pair (f-1, f) is an exact check of frame f: P frames 1, 2, 30, 58 and
    59 are checked that way, and the lookahead of all 60 frames in full."""
    y, _, _ = synth.hd_clip(60, 1)
    frames = synth.coded_luma(y)
    params = A.default_me_params()
    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    got = acc.pixel_path_host(frames, params, lam, gate, qp)
    for f in (1, 2, 30, 58, 59):
        want = O.pixel_path_clip(np.ascontiguousarray(frames[f - 1:f + 1]), O.balanced_params(), lam, gate, qp,
                                 nthreads=8)
        assert np.array_equal(got["picks"][f][:, :5], want["picks"][1][:, :5]), f
        assert np.array_equal(got["costs"][f], want["costs"][1]), f
        assert np.array_equal(got["coeffs"][f], want["coeffs"][1]), f
    intra, inter, mvs = O.lookahead_clip(frames, mode=2, nthreads=8)
    assert np.array_equal(got["la_intra"], intra)
    assert np.array_equal(got["la_inter"], inter)
    assert np.array_equal(got["la_mvs"], mvs)
    # the partition searches ran on this clip (the gate opens for many MBs)
    assert (got["picks"][1:, :, 0] > 0).mean() > 0.05


def test_cif_workload_whole_path_matches_oracle(acc):
    """The CPU-runnable workload verbatim: the CIF clip (gradient + moving
    noise box) of 30 frames at QP 26 through the whole path, every frame
    against the oracle."""
    y, _, _ = synth.cif_clip(30, 0)
    frames = synth.coded_luma(y)
    params = A.default_me_params()
    qp = 26
    lam = float(np.sqrt(A.frame_lambda(qp)))
    gate = A.split_gate_for_qp(qp)
    got = acc.pixel_path_host(frames, params, lam, gate, qp)
    want = O.pixel_path_clip(frames, O.balanced_params(), lam, gate, qp, nthreads=8)
    compare_pixel_path(got, want)


# ---------------------------------------------------------------------------
# Failure handling
# ---------------------------------------------------------------------------

def test_bounded_wait_times_out_and_context_survives(acc, cif):
    assert acc.selftest_bounded_wait(2000) == A.H264A_E_TIMEOUT
    msg = acc.L.h264a_last_error()
    assert b"bounded wait" in msg and b"self-test" in msg and b"status 2" in msg
    # the context and device still work afterwards
    got = acc.hpel_build(dev(acc, cif[:1]), 32)
    acc.sync()
    assert np.array_equal(got.cpu().numpy()[0], O.build_planes4(cif[0], 32))


def test_invalid_arguments_rejected_before_launch(acc, cif):
    d = dev(acc, cif[:1])
    out = acc.empty((1, 4, 288 + 4, 352 + 4), acc.torch.uint8)
    rc = acc.L.h264a_hpel_build(acc.ctx, d.data_ptr(), 352, 288, 2, 1, 352 * 288, out.data_ptr(), None)
    assert rc == -1 and b"pad" in acc.L.h264a_last_error()
    rc = acc.L.h264a_fullpel_grid(acc.ctx, C.byref(A.Picture(d.data_ptr(), out.data_ptr(), 352, 288, 32)), 65, None,
                                  None, 0, 0, None, 1.0, None, None, None, None)
    assert rc == -1
    rc = acc.L.h264a_block_metric(acc.ctx, 0, 12, 16, d.data_ptr(), d.data_ptr(), 16, d.data_ptr(), d.data_ptr(),
                                  None, None, 16, 1, d.data_ptr(), None)
    assert rc == -1


# ---------------------------------------------------------------------------
# The closed reconstruction loop (h264a_pixel_path_closed)
# ---------------------------------------------------------------------------

def _coded_yuv(y, u, v):
    return synth.coded_luma(y), synth.coded_chroma(u), synth.coded_chroma(v)


def _compare_closed(got, want, keys=("picks", "costs", "coeffs", "ccoeffs", "rec_y", "rec_u", "rec_v")):
    for k in keys:
        g, w = got[k], want[k]
        if k == "picks":
            g, w = g[..., :5], w[..., :5]
        assert np.array_equal(g, w), (k, np.argwhere(g != w)[:3])


def test_closed_loop_cif_30_frames_matches_oracle(acc):
    """The CPU-runnable workload (CIF, 30 frames, QP 26) through the closed
    loop: every frame's search runs on the deblocked reconstruction of the
    frame before it; picks, costs, luma and chroma levels and every
    reconstruction equal the oracle's."""
    Y, U, V = _coded_yuv(*synth.cif_clip(30, 0))
    qp = 26
    lam = float(np.sqrt(A.frame_lambda(qp)))
    gate = A.split_gate_for_qp(qp)
    got = acc.pixel_path_closed(Y, U, V, A.default_me_params(), lam, gate, qp)
    want = O.closed_loop_clip(Y, U, V, O.balanced_params(), lam, gate, qp)
    _compare_closed(got, want)
    assert (got["picks"][1:, :, 0] > 0).any()
    # the reconstruction is not the source: the loop really closes
    assert not np.array_equal(got["rec_y"][1:], Y[1:])


def test_closed_loop_1080p_8_frames_matches_oracle(acc):
    Y, U, V = _coded_yuv(*synth.hd_clip(8, 1, with_chroma=True))
    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    got = acc.pixel_path_closed(Y, U, V, A.default_me_params(), lam, gate, qp)
    want = O.closed_loop_clip(Y, U, V, O.balanced_params(), lam, gate, qp)
    _compare_closed(got, want)


def test_closed_loop_learned_matches_oracle(acc):
    """The learned search inside the closed loop: the proposals the network
    made for each frame (from the source pairs, before the loop) fed to the
    oracle's closed loop give the same picks, levels and reconstructions,
    with the same fallback flags."""
    from rusty_h264_b200 import mvnet

    Y, U, V = _coded_yuv(*synth.cif_clip(6, 4))
    qp = 30
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    net = mvnet.MvNet(acc, seed=21)
    got = acc.pixel_path_closed(Y, U, V, A.default_me_params(), lam, gate, qp, net=net, fallback_t=100)
    want = O.closed_loop_clip(Y, U, V, O.balanced_params(), lam, gate, qp, props=got["props"], prop_t=100)
    _compare_closed(got, want)
    assert np.array_equal(got["fallback"], want["fallback"])
    assert (got["props"][1:] != 0).any()
    net.close()


def test_closed_loop_into_pinned_outputs_matches_oracle(acc):
    """The host entry writing into caller-provided pinned arrays (each frame's
    downloads queued as the kernel reports it final) gives the oracle's
    outputs, twice in a row into the same arrays."""
    torch = acc.torch
    Y, U, V = _coded_yuv(*synth.cif_clip(12, 8))
    n, ch, cw = Y.shape
    nmb = (cw // 16) * (ch // 16)
    qp = 25
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    pinned = lambda shp, dt: torch.zeros(shp, dtype=dt).pin_memory().numpy()
    out = dict(picks=pinned((n, nmb, 6), torch.int32), costs=pinned((n, nmb, 2), torch.int64),
               coeffs=pinned((n, nmb, 256), torch.int16), ccoeffs=pinned((n, nmb, 128), torch.int16),
               rec_y=pinned(Y.shape, torch.uint8), rec_u=pinned(U.shape, torch.uint8), rec_v=pinned(V.shape, torch.uint8))
    want = O.closed_loop_clip(Y, U, V, O.balanced_params(), lam, gate, qp)
    for _ in range(2):
        got = acc.pixel_path_closed(Y, U, V, A.default_me_params(), lam, gate, qp, out=out)
        assert got is out
        _compare_closed(got, want)
    with pytest.raises(ValueError):
        acc.pixel_path_closed(Y, U, V, A.default_me_params(), lam, gate, qp, out=dict(out, picks=out["costs"]))


def test_closed_frames_device_path_equals_host_path(acc):
    """h264a_closed_frames on device buffers gives what the host-buffer entry
    gives (which the tests above pin to the oracle)."""
    torch = acc.torch
    Y, U, V = _coded_yuv(*synth.cif_clip(5, 6))
    n, ch, cw = Y.shape
    nmb = (cw // 16) * (ch // 16)
    qp = 28
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    params = A.default_me_params()
    want = acc.pixel_path_closed(Y, U, V, params, lam, gate, qp)
    dy, du, dv = dev(acc, Y), dev(acc, U), dev(acc, V)
    ry, ru, rv = torch.empty_like(dy), torch.empty_like(du), torch.empty_like(dv)
    planes = acc.empty((A.closed_plane_bytes(n, cw, ch),), torch.uint8)
    pk = acc.empty((n, nmb, 6), torch.int32)
    co = acc.empty((n, nmb, 2), torch.int64)
    lv = acc.empty((n, nmb, 256), torch.int16)
    cl = acc.empty((n, nmb, 128), torch.int16)
    job = A.ClosedDev(dy.data_ptr(), du.data_ptr(), dv.data_ptr(), ry.data_ptr(), ru.data_ptr(), rv.data_ptr(),
                      planes.data_ptr(), n, cw, ch, lam, gate, qp, 6, None, 0, None, pk.data_ptr(), co.data_ptr(),
                      lv.data_ptr(), cl.data_ptr(), None, None)
    for _ in range(2):  # twice into the same buffers
        acc.closed_frames(job, params)
        acc.sync()
        got = dict(picks=pk.cpu().numpy(), costs=co.cpu().numpy(), coeffs=lv.cpu().numpy(), ccoeffs=cl.cpu().numpy(),
                   rec_y=ry.cpu().numpy(), rec_u=ru.cpu().numpy(), rec_v=rv.cpu().numpy())
        _compare_closed(got, want)


def _closed_buffers(acc, Y, U, V):
    torch = acc.torch
    n, ch, cw = Y.shape
    nmb = (cw // 16) * (ch // 16)
    b = dict(y=dev(acc, Y), u=dev(acc, U), v=dev(acc, V))
    b["ry"], b["ru"], b["rv"] = b["y"].clone(), b["u"].clone(), b["v"].clone()  # frame 0: lossless
    b["planes"] = acc.empty((4 * (cw + 64) * (ch + 64),), torch.uint8)
    b["picks"] = acc.zeros((n, nmb, 6), torch.int32)
    b["costs"] = acc.zeros((n, nmb, 2), torch.int64)
    b["coeffs"] = acc.zeros((n, nmb, 256), torch.int16)
    b["ccoeffs"] = acc.zeros((n, nmb, 128), torch.int16)
    return b


def _closed_result(b):
    return dict(picks=b["picks"].cpu().numpy(), costs=b["costs"].cpu().numpy(), coeffs=b["coeffs"].cpu().numpy(),
                ccoeffs=b["ccoeffs"].cpu().numpy(), rec_y=b["ry"].cpu().numpy(), rec_u=b["ru"].cpu().numpy(),
                rec_v=b["rv"].cpu().numpy())


def test_closed_step_frame_and_unfused_launches_equal_the_loop(acc):
    """The loop frame by frame through h264a_closed_step_frame (planes, then
    the search with each MB's reconstruction and deblocking fused in), and the
    same frames through the separate launches (plain-ME, MC + luma T/Q +
    reconstruction, chroma, deblocking), both give what h264a_pixel_path_closed
    gives."""
    Y, U, V = _coded_yuv(*synth.cif_clip(5, 9))
    n, ch, cw = Y.shape
    fs = cw * ch
    qp = 29
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    params = A.default_me_params()
    want = acc.pixel_path_closed(Y, U, V, params, lam, gate, qp)
    for fused in (True, False):
        b = _closed_buffers(acc, Y, U, V)
        for f in range(1, n):
            acc._check(acc.L.h264a_hpel_build(acc.ctx, b["ry"][f - 1].data_ptr(), cw, ch, 32, 1, fs,
                                              b["planes"].data_ptr(), acc._stream()))
            pic = A.Picture(b["y"][f].data_ptr(), b["planes"].data_ptr(), cw, ch, 32)
            me = A.MeFrame(pic, lam, gate, b["picks"][f].data_ptr(), b["costs"][f].data_ptr())
            if fused:
                acc.closed_step(A.ClosedStep(me, b["u"][f].data_ptr(), b["v"][f].data_ptr(), b["ru"][f - 1].data_ptr(),
                                             b["rv"][f - 1].data_ptr(), b["ry"][f].data_ptr(), b["ru"][f].data_ptr(),
                                             b["rv"][f].data_ptr(), b["coeffs"][f].data_ptr(),
                                             b["ccoeffs"][f].data_ptr(), qp, 6, None, None, 0), params)
                continue
            acc.me_frames([me], params)
            acc.mc_tq_rec_frames([A.TqRecFrame(A.TqFrame(pic, b["picks"][f].data_ptr(), qp, 6,
                                                         b["coeffs"][f].data_ptr()), b["ry"][f].data_ptr())])
            acc.mc_tq_chroma_frames([A.TqChromaFrame(b["u"][f].data_ptr(), b["v"][f].data_ptr(),
                                                     b["ru"][f - 1].data_ptr(), b["rv"][f - 1].data_ptr(), cw, ch,
                                                     b["picks"][f].data_ptr(), qp, b["ccoeffs"][f].data_ptr(),
                                                     b["ru"][f].data_ptr(), b["rv"][f].data_ptr())])
            acc.deblock_frames([A.DeblockFrame(b["ry"][f].data_ptr(), b["ru"][f].data_ptr(), b["rv"][f].data_ptr(), cw,
                                               ch, b["picks"][f].data_ptr(), b["coeffs"][f].data_ptr(), qp, 0, 0, 0)])
        acc.sync()
        _compare_closed(_closed_result(b), want)


@pytest.mark.parametrize("h,w,qp", [(16, 16, 20), (32, 48, 36), (288, 32, 24), (48, 352, 44), (144, 176, 14)])
def test_closed_loop_small_and_narrow_frames_match_oracle(acc, h, w, qp):
    """Frames of one MB, one MB column or two MB rows (no top-right
    neighbour, or none above) and QPs from 14 to 44 (every deblocking
    threshold row, bS 0/1/2) through the fused loop equal the oracle."""
    y, u, v = synth.cif_clip(4, 17 + h)
    oy, ox = min(40, 288 - h), min(64, 352 - w)  # even: chroma at half the offsets
    Y = np.ascontiguousarray(y[:, oy:oy + h, ox:ox + w])
    U = np.ascontiguousarray(u[:, oy // 2:(oy + h) // 2, ox // 2:(ox + w) // 2])
    V = np.ascontiguousarray(v[:, oy // 2:(oy + h) // 2, ox // 2:(ox + w) // 2])
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    got = acc.pixel_path_closed(Y, U, V, A.default_me_params(), lam, gate, qp)
    want = O.closed_loop_clip(Y, U, V, O.balanced_params(), lam, gate, qp)
    _compare_closed(got, want)


@pytest.mark.parametrize("learned", [False, True])
def test_me_frames_wide_kernel_equals_batched(acc, learned):
    """Frames run one at a time take the wide kernel (a CTA per MB, the four
    partitions one warp each); the same frames in one call take the narrow
    kernel (a warp per MB).  Picks, costs and fallback flags are identical,
    and both equal the oracle (first frame)."""
    torch = acc.torch
    y, _, _ = synth.hd_clip(5, 12, 352, 288)
    clip = synth.coded_luma(y)
    n, ch, cw = clip.shape
    nmb = (cw // 16) * (ch // 16)
    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    params = A.default_me_params()
    d = dev(acc, clip)
    planes = acc.hpel_build(d[: n - 1], 32)
    rng = np.random.default_rng(3)
    props = dev(acc, rng.integers(-8, 9, (n, nmb, 16)).astype(np.int32) * 4)
    outs = []
    for batched in (True, False):
        pk = acc.zeros((n, nmb, 6), torch.int32)
        co = acc.zeros((n, nmb, 2), torch.int64)
        fb = acc.zeros((n, nmb), torch.int32)
        fr = [A.MeFrame(A.Picture(d[i].data_ptr(), planes[i - 1].data_ptr(), cw, ch, 32), lam, gate,
                        pk[i].data_ptr(), co[i].data_ptr()) for i in range(1, n)]
        lf = [A.MeLearnedFrame(fr[i - 1], props[i].data_ptr(), 200, fb[i].data_ptr()) for i in range(1, n)]
        calls = [lf] if batched else [[x] for x in lf]
        for c in calls:
            if learned:
                acc.me_frames_learned(c, params)
            else:
                acc.me_frames([x.me for x in c], params)
        acc.sync()
        outs.append((pk.cpu().numpy(), co.cpu().numpy(), fb.cpu().numpy()))
    (pa, ca, fa), (pb, cb_, fb_) = outs
    assert np.array_equal(pa[..., :5], pb[..., :5]) and np.array_equal(ca, cb_)
    assert np.array_equal(pa[..., 5], pb[..., 5])
    if learned:
        assert np.array_equal(fa, fb_)
    else:
        wp, wc = O.me_frame(clip[1], clip[0], O.build_planes4(clip[0], 32), O.balanced_params(), lam, gate)
        assert np.array_equal(pb[1, :, :5], wp[:, :5]) and np.array_equal(cb_[1], wc)
    assert (pb[1:, :, 0] > 0).any()  # the partition searches ran
