"""Python binding of libh264accel_cuda.so (include/h264accel.h).

The library is the product: C++/CUDA kernels for sm_100a behind a C ABI.  This
module only marshals arguments: device buffers are torch CUDA tensors (torch
is plumbing here), structs are ctypes mirrors of the header.  There is no CPU
fallback: constructing :class:`Accel` without the built library or without a
B200 raises.

Names follow the reference crate `rusty_h264-accel` and the encoder functions
each entry replaces (see the header for file:line).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libh264accel_cuda.so")

# metric ids (include/h264accel.h)
METRIC_SATD_WELS = 0
METRIC_SATD = 1
METRIC_SAD = 2
METRIC_SATD_AVG = 3
METRIC_SAD_AVG = 4

H264A_OK = 0
H264A_E_TIMEOUT = -3


class Picture(C.Structure):
    _fields_ = [("d_src", C.c_void_p), ("d_planes", C.c_void_p), ("cw", C.c_int32), ("ch", C.c_int32),
                ("pad", C.c_int32)]


class Candidate(C.Structure):
    _fields_ = [("pic", C.c_int32), ("x", C.c_int32), ("y", C.c_int32), ("w", C.c_int32), ("h", C.c_int32),
                ("mvx", C.c_int32), ("mvy", C.c_int32)]


class MeParams(C.Structure):
    _fields_ = [
        ("fast", C.c_int32), ("mb_use_satd", C.c_int32), ("sadfp", C.c_int32), ("mv_cost_kind", C.c_int32),
        ("d_mv_cost_tab", C.c_void_p), ("sadfp_lambda", C.c_double),
        ("me_snap", C.c_int32), ("me_fc", C.c_int32), ("dia_mask", C.c_uint32), ("dia_sub_mask", C.c_uint32),
        ("subpel", C.c_int32), ("subpel_pat", C.c_int32), ("sp_single_pass", C.c_int32), ("sub_pat", C.c_int32),
        ("me_subpel_iter", C.c_int32), ("sp_maxit", C.c_int32), ("sp_fc", C.c_int32),
    ]


class MeJob(C.Structure):
    _fields_ = [("pic", C.c_int32), ("x", C.c_int32), ("y", C.c_int32), ("w", C.c_int32), ("h", C.c_int32),
                ("npred", C.c_int32), ("preds", C.c_int32 * 8), ("has_start", C.c_int32), ("start", C.c_int32 * 2),
                ("lambda_me", C.c_double)]


class MeResult(C.Structure):
    _fields_ = [("mvx", C.c_int32), ("mvy", C.c_int32), ("cost", C.c_int64), ("evals", C.c_int32),
                ("status", C.c_int32)]


class MeFrame(C.Structure):
    _fields_ = [("pic", Picture), ("lambda_me", C.c_double), ("split_gate", C.c_int64), ("d_picks", C.c_void_p),
                ("d_costs", C.c_void_p)]


class MeLearnedFrame(C.Structure):
    _fields_ = [("me", MeFrame), ("d_props", C.c_void_p), ("fallback_t", C.c_int32), ("d_fallback", C.c_void_p)]


class MeTqFrame(C.Structure):
    _fields_ = [("me", MeFrame), ("qp", C.c_int32), ("dz_div", C.c_int32), ("d_coeffs", C.c_void_p)]


class TqFrame(C.Structure):
    _fields_ = [("pic", Picture), ("d_picks", C.c_void_p), ("qp", C.c_int32), ("dz_div", C.c_int32),
                ("d_coeffs", C.c_void_p)]


class TqRecFrame(C.Structure):
    _fields_ = [("tq", TqFrame), ("d_rec", C.c_void_p)]


class DeblockFrame(C.Structure):
    _fields_ = [("d_y", C.c_void_p), ("d_u", C.c_void_p), ("d_v", C.c_void_p), ("cw", C.c_int32), ("ch", C.c_int32),
                ("d_picks", C.c_void_p), ("d_coeffs", C.c_void_p), ("qp", C.c_int32), ("offset_a", C.c_int32),
                ("offset_b", C.c_int32), ("chroma_qp_offset", C.c_int32)]


class TqChromaFrame(C.Structure):
    _fields_ = [("d_src_u", C.c_void_p), ("d_src_v", C.c_void_p), ("d_ref_u", C.c_void_p), ("d_ref_v", C.c_void_p),
                ("cw", C.c_int32), ("ch", C.c_int32), ("d_picks", C.c_void_p), ("qp", C.c_int32),
                ("d_coeffs", C.c_void_p), ("d_rec_u", C.c_void_p), ("d_rec_v", C.c_void_p)]


class ClosedJob(C.Structure):
    _fields_ = [("h_y", C.c_void_p), ("h_u", C.c_void_p), ("h_v", C.c_void_p), ("n", C.c_int32), ("cw", C.c_int32),
                ("ch", C.c_int32), ("lambda_me", C.c_double), ("split_gate", C.c_int64), ("qp", C.c_int32),
                ("dz_div", C.c_int32), ("net", C.c_void_p), ("fallback_t", C.c_int32), ("h_picks", C.c_void_p),
                ("h_costs", C.c_void_p), ("h_coeffs", C.c_void_p), ("h_ccoeffs", C.c_void_p), ("h_rec_y", C.c_void_p),
                ("h_rec_u", C.c_void_p), ("h_rec_v", C.c_void_p), ("h_props", C.c_void_p),
                ("h_fallback", C.c_void_p)]


class StreamFrames(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("cw", C.c_int32), ("ch", C.c_int32), ("n", C.c_int32),
                ("qp", C.c_int32), ("h_y0", C.c_void_p), ("h_u0", C.c_void_p), ("h_v0", C.c_void_p),
                ("h_picks", C.c_void_p), ("h_coeffs", C.c_void_p), ("h_ccoeffs", C.c_void_p)]


class ClosedDev(C.Structure):
    _fields_ = [("d_y", C.c_void_p), ("d_u", C.c_void_p), ("d_v", C.c_void_p), ("d_rec_y", C.c_void_p),
                ("d_rec_u", C.c_void_p), ("d_rec_v", C.c_void_p), ("d_planes", C.c_void_p), ("n", C.c_int32),
                ("cw", C.c_int32), ("ch", C.c_int32), ("lambda_me", C.c_double), ("split_gate", C.c_int64),
                ("qp", C.c_int32), ("dz_div", C.c_int32), ("net", C.c_void_p), ("fallback_t", C.c_int32),
                ("d_guide_mvs", C.c_void_p), ("d_picks", C.c_void_p), ("d_costs", C.c_void_p),
                ("d_coeffs", C.c_void_p), ("d_ccoeffs", C.c_void_p), ("d_props", C.c_void_p),
                ("d_fallback", C.c_void_p)]


class ClosedStep(C.Structure):
    _fields_ = [("me", MeFrame), ("d_u", C.c_void_p), ("d_v", C.c_void_p), ("d_ref_u", C.c_void_p),
                ("d_ref_v", C.c_void_p), ("d_rec_y", C.c_void_p), ("d_rec_u", C.c_void_p), ("d_rec_v", C.c_void_p),
                ("d_coeffs", C.c_void_p), ("d_ccoeffs", C.c_void_p), ("qp", C.c_int32), ("dz_div", C.c_int32),
                ("d_props", C.c_void_p), ("d_fallback", C.c_void_p), ("fallback_t", C.c_int32)]


class MeMrFrame(C.Structure):
    _fields_ = [("d_src", C.c_void_p), ("d_planes", C.c_void_p * 4), ("nref", C.c_int32), ("cw", C.c_int32),
                ("ch", C.c_int32), ("pad", C.c_int32), ("lambda_me", C.c_double), ("split_gate", C.c_int64),
                ("d_picks", C.c_void_p), ("d_costs", C.c_void_p)]


class LaStream(C.Structure):
    _fields_ = [("d_full", C.c_void_p), ("d_half", C.c_void_p), ("cw", C.c_int32), ("ch", C.c_int32),
                ("n", C.c_int32), ("d_intra", C.c_void_p), ("d_inter", C.c_void_p), ("d_mvs", C.c_void_p)]


BATCH_VARIANTS = 6  # H264A_BATCH_VARIANTS
CLOSED_PLANE_PICTURES = 16  # H264A_CLOSED_PLANE_PICTURES


def closed_plane_bytes(n: int, cw: int, ch: int, pad: int = 32) -> int:
    """Plane scratch of h264a_closed_frames: min(n, 16) pictures' F|H|V|C planes."""
    return 4 * min(n, CLOSED_PLANE_PICTURES) * (cw + 2 * pad) * (ch + 2 * pad)


class BatchStream(C.Structure):
    _fields_ = [("cw", C.c_int32), ("ch", C.c_int32), ("pad", C.c_int32), ("d_src", C.c_void_p),
                ("d_planes", C.c_void_p), ("d_picks", C.c_void_p), ("d_costs", C.c_void_p),
                ("lambda_me", C.c_double), ("split_gate", C.c_int64), ("d_coeffs", C.c_void_p),
                ("qp", C.c_int32), ("dz_div", C.c_int32)]


class McTqMrFrame(C.Structure):
    _fields_ = [("d_src", C.c_void_p), ("d_planes", C.c_void_p * 4), ("nref", C.c_int32), ("cw", C.c_int32),
                ("ch", C.c_int32), ("pad", C.c_int32), ("d_picks", C.c_void_p), ("qp", C.c_int32),
                ("dz_div", C.c_int32), ("d_coeffs", C.c_void_p)]


class BatchConfig(C.Structure):
    _fields_ = [("gop_step", C.c_int32), ("nslots", C.c_int32), ("nref", C.c_int32), ("autotune", C.c_int32),
                ("variant", C.c_int32)]


class BatchInfo(C.Structure):
    _fields_ = [("variant", C.c_int32), ("tuned", C.c_int32), ("ms", C.c_float * BATCH_VARIANTS),
                ("graphs", C.c_int32), ("steps", C.c_int64)]


# Every entry point the header declares (checked by tests/test_capi_symbols.py).
EXPORTS = (
    "h264a_version", "h264a_last_error", "h264a_ctx_create", "h264a_ctx_destroy", "h264a_sync",
    "h264a_dev_alloc", "h264a_dev_free", "h264a_memcpy_h2d", "h264a_memcpy_d2h", "h264a_hpel_build",
    "h264a_block_metric", "h264a_candidate_dist", "h264a_me_params_default", "h264a_build_mv_cost_table",
    "h264a_me_search", "h264a_me_frames", "h264a_fullpel_grid", "h264a_dct_quant_4x4", "h264a_dct_quant_8x8",
    "h264a_mc_tq_frames", "h264a_downsample2x", "h264a_lookahead_costs", "h264a_pixel_path_host",
    "h264a_pixel_path_prefetch",
    "h264a_selftest_bounded_wait", "h264a_measure_int32_peak", "h264a_me_frames_noalloc",
    "h264a_mc_tq_rec_frames", "h264a_mc_tq_chroma_frames", "h264a_deblock_frames", "h264a_me_tq_frames",
    "h264a_mvnet_create", "h264a_mvnet_destroy", "h264a_mvnet_set_params", "h264a_mvnet_get_params",
    "h264a_mvnet_forward", "h264a_mvnet_grads", "h264a_mvnet_train_step", "h264a_mvnet_propose",
    "h264a_me_frames_learned", "h264a_pixel_path_closed", "h264a_write_stream_cavlc", "h264a_cavlc_table_code",
    "h264a_closed_frames", "h264a_closed_step_frame", "h264a_me_frames_multiref",
    "h264a_batch_create", "h264a_batch_step", "h264a_batch_get_info", "h264a_batch_destroy",
    "h264a_batch_variant_shape", "h264a_lookahead_streams", "h264a_mc_tq_frames_multiref",
)

_lib = None


def load_library() -> C.CDLL:
    """Loads the in-tree library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C rusty_h264_b200/csrc`")
    L = C.CDLL(LIB_PATH)
    L.h264a_version.restype = C.c_char_p
    L.h264a_last_error.restype = C.c_char_p
    vp, i32, i64, f64, sz = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_size_t
    L.h264a_ctx_create.argtypes = [i32, C.POINTER(vp)]
    L.h264a_ctx_destroy.argtypes = [vp]
    L.h264a_sync.argtypes = [vp, vp]
    L.h264a_hpel_build.argtypes = [vp, vp, i32, i32, i32, i32, sz, vp, vp]
    L.h264a_block_metric.argtypes = [vp, i32, i32, i32, vp, vp, i32, vp, vp, vp, vp, i32, i32, vp, vp]
    L.h264a_candidate_dist.argtypes = [vp, vp, i32, vp, i32, i32, vp, vp]
    L.h264a_me_params_default.argtypes = [C.POINTER(MeParams)]
    L.h264a_me_params_default.restype = None
    L.h264a_build_mv_cost_table.argtypes = [vp]
    L.h264a_build_mv_cost_table.restype = None
    L.h264a_me_search.argtypes = [vp, vp, i32, C.POINTER(MeParams), vp, i32, vp, vp]
    L.h264a_me_frames.argtypes = [vp, vp, i32, C.POINTER(MeParams), vp]
    L.h264a_me_tq_frames.argtypes = [vp, vp, i32, C.POINTER(MeParams), vp]
    L.h264a_fullpel_grid.argtypes = [vp, C.POINTER(Picture), i32, vp, vp, i32, i32, vp, f64, vp, vp, vp, vp]
    L.h264a_dct_quant_4x4.argtypes = [vp, vp, i32, vp, i32, vp, vp, i32, i32, vp, vp]
    L.h264a_dct_quant_8x8.argtypes = [vp, vp, i32, vp, i32, vp, vp, vp, i32, i32, vp, vp]
    L.h264a_mc_tq_frames.argtypes = [vp, vp, i32, vp]
    L.h264a_mc_tq_rec_frames.argtypes = [vp, vp, i32, vp]
    L.h264a_mc_tq_chroma_frames.argtypes = [vp, vp, i32, vp]
    L.h264a_deblock_frames.argtypes = [vp, vp, i32, vp]
    L.h264a_downsample2x.argtypes = [vp, vp, i32, i32, i32, sz, vp, vp]
    L.h264a_lookahead_costs.argtypes = [vp, vp, vp, i32, i32, i32, i32, vp, vp, vp, vp]
    L.h264a_pixel_path_prefetch.argtypes = [vp, vp, i32, i32, i32]
    L.h264a_pixel_path_host.argtypes = [vp, vp, i32, i32, i32, C.POINTER(MeParams), vp, f64, i64, i32, i32, vp, vp, vp,
                                        vp, vp, vp]
    L.h264a_selftest_bounded_wait.argtypes = [vp, i32, vp]
    L.h264a_measure_int32_peak.argtypes = [vp, C.POINTER(C.c_double)]
    L.h264a_me_frames_noalloc.argtypes = [vp, i32, C.POINTER(MeParams), vp, vp]
    L.h264a_me_frames_learned.argtypes = [vp, vp, i32, C.POINTER(MeParams), vp]
    L.h264a_pixel_path_closed.argtypes = [vp, C.POINTER(ClosedJob), C.POINTER(MeParams), vp]
    L.h264a_closed_frames.argtypes = [vp, C.POINTER(ClosedDev), C.POINTER(MeParams), vp]
    L.h264a_closed_step_frame.argtypes = [vp, C.POINTER(ClosedStep), C.POINTER(MeParams), vp]
    L.h264a_me_frames_multiref.argtypes = [vp, vp, C.c_int, C.POINTER(MeParams), vp]
    L.h264a_lookahead_streams.argtypes = [vp, vp, i32, i32, vp]
    L.h264a_mc_tq_frames_multiref.argtypes = [vp, vp, i32, vp]
    L.h264a_batch_create.argtypes = [vp, vp, i32, C.POINTER(BatchConfig), C.POINTER(MeParams), C.POINTER(vp)]
    L.h264a_batch_step.argtypes = [vp, i64, i32, vp]
    L.h264a_batch_get_info.argtypes = [vp, C.POINTER(BatchInfo)]
    L.h264a_batch_destroy.argtypes = [vp]
    L.h264a_batch_variant_shape.argtypes = [i32, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.h264a_write_stream_cavlc.argtypes = [C.POINTER(StreamFrames), vp, sz, C.POINTER(sz), vp]
    L.h264a_cavlc_table_code.argtypes = [i32, i32, i32, i32, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.h264a_mvnet_create.argtypes = [i32, C.c_uint64, C.POINTER(vp)]
    L.h264a_mvnet_destroy.argtypes = [vp]
    L.h264a_mvnet_set_params.argtypes = [vp, vp]
    L.h264a_mvnet_get_params.argtypes = [vp, vp]
    L.h264a_mvnet_forward.argtypes = [vp, vp, i32, i32, i32, vp, vp, vp]
    L.h264a_mvnet_grads.argtypes = [vp, vp, i32, i32, i32, vp, vp, vp, vp, vp]
    L.h264a_mvnet_train_step.argtypes = [vp, vp, i32, i32, i32, vp, vp, C.c_float, vp, vp]
    L.h264a_mvnet_propose.argtypes = [vp, vp, i32, vp]
    _lib = L
    return L


def default_me_params(**overrides) -> MeParams:
    p = MeParams()
    load_library().h264a_me_params_default(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def mv_cost_table() -> np.ndarray:
    """The smooth mvd-cost table (mv cost kind 1), built by the library."""
    t = np.zeros(4096, np.uint16)
    load_library().h264a_build_mv_cost_table(t.ctypes.data_as(C.c_void_p))
    return t


def write_stream_cavlc(y0, u0, v0, picks, coeffs, ccoeffs, qp: int, width: int = None, height: int = None):
    """Annex-B bytes of the frame model's stream (h264a_write_stream_cavlc, host
    only) and the bytes of each frame.  y0/u0/v0: frame 0; picks (n, nmb, 6),
    coeffs (n, nmb, 256), ccoeffs (n, nmb, 128)."""
    L = load_library()
    ch, cw = y0.shape
    n = picks.shape[0]
    arrs = [np.ascontiguousarray(a) for a in (y0, u0, v0)] + [np.ascontiguousarray(picks, np.int32),
                                                               np.ascontiguousarray(coeffs, np.int16),
                                                               np.ascontiguousarray(ccoeffs, np.int16)]
    sf = StreamFrames(width or cw, height or ch, cw, ch, n, qp, *[a.ctypes.data for a in arrs])
    ln = C.c_size_t()
    fb = np.zeros(n, np.int64)
    rc = L.h264a_write_stream_cavlc(C.byref(sf), None, 0, C.byref(ln), None)
    if rc != H264A_OK:
        raise AccelError(rc, L.h264a_last_error().decode())
    out = np.zeros(ln.value, np.uint8)
    rc = L.h264a_write_stream_cavlc(C.byref(sf), out.ctypes.data_as(C.c_void_p), out.size, C.byref(ln),
                                    fb.ctypes.data_as(C.c_void_p))
    if rc != H264A_OK:
        raise AccelError(rc, L.h264a_last_error().decode())
    return out.tobytes(), fb


def split_gate_for_qp(qp: int) -> int:
    """The 16x16 J above which the partition searches run (mb16.rs:8885-8887)."""
    qstep16 = (10, 11, 13, 14, 16, 18)[qp % 6] << (qp // 6)
    return ((30 * (qstep16 + 160)) >> 3) * 2


def frame_lambda(qp: int, scale: float = 1.0) -> float:
    """Slice λ (mb16.rs:8642): 0.85·scale·2^((qp−12)/3)."""
    return 0.85 * scale * 2.0 ** ((qp - 12.0) / 3.0)


def _dptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


class AccelError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"h264accel error {code}: {msg}")
        self.code = code


class Accel:
    """One library context on one CUDA device."""

    def __init__(self, device: int = 0):
        import torch

        self.torch = torch
        if not torch.cuda.is_available():
            raise RuntimeError("rusty_h264_b200 needs a CUDA device (sm_100a); none is visible")
        self.L = load_library()
        self.device = device
        self._prefetched = []  # (address, array) of frames whose upload may still be pending
        torch.cuda.set_device(device)
        ctx = C.c_void_p()
        self._check(self.L.h264a_ctx_create(device, C.byref(ctx)))
        self.ctx = ctx

    def close(self):
        if getattr(self, "ctx", None):
            self.L.h264a_ctx_destroy(self.ctx)  # waits for pending prefetch uploads
            self.ctx = None
            self._prefetched = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- plumbing ---------------------------------------------------------
    def _check(self, rc: int):
        if rc != H264A_OK:
            raise AccelError(rc, self.L.h264a_last_error().decode())

    def _stream(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def sync(self):
        self._check(self.L.h264a_sync(self.ctx, self._stream()))

    def to_dev(self, arr) -> "torch.Tensor":
        t = self.torch.from_numpy(np.ascontiguousarray(arr))
        return t.to(f"cuda:{self.device}")

    def struct_array_dev(self, items: Sequence[C.Structure]):
        """Copies a list of ctypes structs into a device byte tensor."""
        n = len(items)
        if n == 0:
            return self.torch.zeros(1, dtype=self.torch.uint8, device=f"cuda:{self.device}")
        T = type(items[0])
        arr = (T * n)(*items)
        raw = np.frombuffer(bytes(arr), np.uint8)
        return self.to_dev(raw)

    def empty(self, shape, dtype):
        return self.torch.empty(shape, dtype=dtype, device=f"cuda:{self.device}")

    def zeros(self, shape, dtype):
        return self.torch.zeros(shape, dtype=dtype, device=f"cuda:{self.device}")

    # ---- a1/a2 ------------------------------------------------------------
    def hpel_build(self, frames, pad: int = 32, out=None):
        """Planes (n, 4, ph, pw) u8 of n luma frames (n, ch, cw) u8 (device)."""
        n, ch, cw = frames.shape
        pw, ph = cw + 2 * pad, ch + 2 * pad
        if out is None:
            out = self.empty((n, 4, ph, pw), self.torch.uint8)
        self._check(self.L.h264a_hpel_build(self.ctx, _dptr(frames), cw, ch, pad, n, cw * ch, _dptr(out),
                                             self._stream()))
        return out

    # ---- a6/a7/a8 -----------------------------------------------------------
    def block_metric(self, metric, w, h, a, a_off, sa, b, b_off, sb, c=None, c_off=None):
        n = int(a_off.numel())
        out = self.empty((n,), self.torch.int32)
        self._check(self.L.h264a_block_metric(self.ctx, metric, w, h, _dptr(a), _dptr(a_off), sa, _dptr(b),
                                              _dptr(b_off), _dptr(c), _dptr(c_off), sb, n, _dptr(out), self._stream()))
        return out

    # ---- a3/a4/a5/a9 ----------------------------------------------------------
    def pictures(self, srcs, planes, pad: int = 32):
        """Device array of h264a_picture for (src frame, planes) pairs."""
        pics = []
        for s, p in zip(srcs, planes):
            ch, cw = s.shape[-2:]
            pics.append(Picture(_dptr(s), _dptr(p), cw, ch, pad))
        return self.struct_array_dev(pics), pics

    def candidate_dist(self, d_pics, npics, cands: Sequence[Candidate], metric=METRIC_SATD):
        d_c = self.struct_array_dev(cands)
        out = self.empty((len(cands),), self.torch.int32)
        self._check(self.L.h264a_candidate_dist(self.ctx, _dptr(d_pics), npics, _dptr(d_c), len(cands), metric,
                                                _dptr(out), self._stream()))
        return out

    # ---- a10/a11/a12 ----------------------------------------------------------
    def me_search(self, d_pics, npics, params: MeParams, jobs: Sequence[MeJob]):
        d_j = self.struct_array_dev(jobs)
        out = self.zeros((len(jobs) * C.sizeof(MeResult),), self.torch.uint8)
        self._check(self.L.h264a_me_search(self.ctx, _dptr(d_pics), npics, C.byref(params), _dptr(d_j), len(jobs),
                                           _dptr(out), self._stream()))
        return out

    @staticmethod
    def me_results(raw) -> np.ndarray:
        b = raw.cpu().numpy().tobytes()
        res = (MeResult * (len(b) // C.sizeof(MeResult))).from_buffer_copy(b)
        return np.array([(r.mvx, r.mvy, r.cost, r.evals, r.status) for r in res], np.int64).reshape(-1, 5)

    def me_frames(self, frames: Sequence[MeFrame], params: MeParams):
        arr = (MeFrame * len(frames))(*frames)
        self._check(self.L.h264a_me_frames(self.ctx, C.cast(arr, C.c_void_p), len(frames), C.byref(params),
                                           self._stream()))

    def me_frames_multiref(self, frames: Sequence[MeMrFrame], params: MeParams):
        """Plain-ME of frames over up to 4 reference pictures each
        (h264a_me_frames_multiref), enqueued on the current stream."""
        arr = (MeMrFrame * len(frames))(*frames)
        self._check(self.L.h264a_me_frames_multiref(self.ctx, C.cast(arr, C.c_void_p), len(frames), C.byref(params),
                                                    self._stream()))

    def mc_tq_frames_multiref(self, frames: Sequence[McTqMrFrame]):
        """MC + luma T/Q of multi-reference picks (h264a_mc_tq_frames_multiref)."""
        arr = (McTqMrFrame * len(frames))(*frames)
        self._check(self.L.h264a_mc_tq_frames_multiref(self.ctx, C.cast(arr, C.c_void_p), len(frames),
                                                       self._stream()))

    def lookahead_streams(self, streams: Sequence[LaStream], mode: int = 2):
        """h264a_lookahead_costs of several streams in one launch (h264a_lookahead_streams)."""
        arr = (LaStream * len(streams))(*streams)
        self._check(self.L.h264a_lookahead_streams(self.ctx, C.cast(arr, C.c_void_p), len(streams), int(mode),
                                                   self._stream()))

    def batch_create(self, streams: Sequence[BatchStream], cfg: BatchConfig, params: MeParams) -> "Batch":
        """A batch of streams stepping G P frames per graph launch (h264a_batch_create)."""
        arr = (BatchStream * len(streams))(*streams)
        h = C.c_void_p()
        self._check(self.L.h264a_batch_create(self.ctx, C.cast(arr, C.c_void_p), len(streams), C.byref(cfg),
                                              C.byref(params), C.byref(h)))
        return Batch(self, h)

    def me_frames_learned(self, frames: Sequence[MeLearnedFrame], params: MeParams):
        """me_frames with the learned proposals in each MB's 16x16 search."""
        arr = (MeLearnedFrame * len(frames))(*frames)
        self._check(self.L.h264a_me_frames_learned(self.ctx, C.cast(arr, C.c_void_p), len(frames), C.byref(params),
                                                   self._stream()))

    def me_tq_frames(self, frames: Sequence[MeTqFrame], params: MeParams):
        """me_frames with each MB's MC + luma T/Q fused into the same launch."""
        arr = (MeTqFrame * len(frames))(*frames)
        self._check(self.L.h264a_me_tq_frames(self.ctx, C.cast(arr, C.c_void_p), len(frames), C.byref(params),
                                              self._stream()))

    def fullpel_grid(self, pic: Picture, R: int, centers=None, pmv=None, metric=0, kind=0, tab=None, lam=0.0,
                     want_grids=True):
        nmb = (pic.cw // 16) * (pic.ch // 16)
        n = 2 * R + 1
        sad = self.empty((nmb, n * n), self.torch.int32) if want_grids else None
        satd = self.empty((nmb, n * n), self.torch.int32) if want_grids else None
        best = self.empty((nmb, 4), self.torch.int32)
        self._check(self.L.h264a_fullpel_grid(self.ctx, C.byref(pic), R, _dptr(centers), _dptr(pmv), metric, kind,
                                              _dptr(tab), float(lam), _dptr(sad), _dptr(satd), _dptr(best),
                                              self._stream()))
        return sad, satd, best

    # ---- a13/a14/a15 ----------------------------------------------------------
    def dct_quant_4x4(self, src, ss, pred, ps, xy, qp, dz_div=6):
        n = int(xy.shape[0])
        out = self.empty((n, 64), self.torch.int16)
        self._check(self.L.h264a_dct_quant_4x4(self.ctx, _dptr(src), ss, _dptr(pred), ps, _dptr(xy), _dptr(qp),
                                               dz_div, n, _dptr(out), self._stream()))
        return out

    def dct_quant_8x8(self, src, ss, pred, ps, xy, qp, weight: Optional[np.ndarray] = None, dz_div=6):
        n = int(xy.shape[0])
        out = self.empty((n, 64), self.torch.int32)
        w = None if weight is None else np.ascontiguousarray(weight, np.int32)
        self._check(self.L.h264a_dct_quant_8x8(self.ctx, _dptr(src), ss, _dptr(pred), ps, _dptr(xy), _dptr(qp),
                                               None if w is None else w.ctypes.data_as(C.c_void_p), dz_div, n,
                                               _dptr(out), self._stream()))
        return out

    def mc_tq_frames(self, frames: Sequence[TqFrame]):
        arr = (TqFrame * len(frames))(*frames)
        self._check(self.L.h264a_mc_tq_frames(self.ctx, C.cast(arr, C.c_void_p), len(frames), self._stream()))

    def deblock_frames(self, frames: Sequence[DeblockFrame]):
        arr = (DeblockFrame * len(frames))(*frames)
        self._check(self.L.h264a_deblock_frames(self.ctx, C.cast(arr, C.c_void_p), len(frames), self._stream()))

    def mc_tq_chroma_frames(self, frames: Sequence[TqChromaFrame]):
        arr = (TqChromaFrame * len(frames))(*frames)
        self._check(self.L.h264a_mc_tq_chroma_frames(self.ctx, C.cast(arr, C.c_void_p), len(frames), self._stream()))

    def mc_tq_rec_frames(self, frames: Sequence[TqRecFrame]):
        arr = (TqRecFrame * len(frames))(*frames)
        self._check(self.L.h264a_mc_tq_rec_frames(self.ctx, C.cast(arr, C.c_void_p), len(frames), self._stream()))

    # ---- a16-a19 ------------------------------------------------------------------
    def downsample2x(self, frames):
        n, ch, cw = frames.shape
        out = self.empty((n, ch // 2, cw // 2), self.torch.uint8)
        self._check(self.L.h264a_downsample2x(self.ctx, _dptr(frames), cw, ch, n, cw * ch, _dptr(out),
                                              self._stream()))
        return out

    def lookahead_costs(self, full, half, mode=2):
        n, ch, cw = full.shape
        nmb = (cw // 16) * (ch // 16)
        intra = self.empty((n, nmb), self.torch.int32)
        inter = self.empty((n, nmb), self.torch.int32)
        mvs = self.empty((n, nmb, 2), self.torch.int32)
        self._check(self.L.h264a_lookahead_costs(self.ctx, _dptr(full), _dptr(half), cw, ch, n, mode, _dptr(intra),
                                                 _dptr(inter), _dptr(mvs), self._stream()))
        return intra, inter, mvs

    def selftest_bounded_wait(self, spin_limit: int):
        """Runs a bounded wait that must time out; returns h264a_sync's code."""
        self._check(self.L.h264a_selftest_bounded_wait(self.ctx, spin_limit, self._stream()))
        return self.L.h264a_sync(self.ctx, self._stream())

    def measure_int32_peak(self) -> float:
        """INT32 lane-instruction rate of this device, Gop/s."""
        v = C.c_double()
        self._check(self.L.h264a_measure_int32_peak(self.ctx, C.byref(v)))
        return v.value

    # ---- the closed reconstruction loop -------------------------------------------
    def pixel_path_closed(self, y: np.ndarray, u: np.ndarray, v: np.ndarray, params: MeParams, lambda_me: float,
                          split_gate: int, qp: int, dz_div: int = 6, net=None, fallback_t: int = 0,
                          tab: Optional[np.ndarray] = None, out: Optional[dict] = None):
        """Luma y (n, ch, cw) and chroma u, v (n, ch/2, cw/2) u8 through the
        closed loop; returns picks, costs, coeffs, ccoeffs, rec_y/u/v (and
        props, fallback with a net).  `out`: preallocated C-contiguous output
        arrays of those names, shapes and dtypes (pinned ones make the
        per-frame downloads asynchronous)."""
        n, ch, cw = y.shape
        nmb = (cw // 16) * (ch // 16)
        ins = [np.ascontiguousarray(a, np.uint8) for a in (y, u, v)]
        want = dict(picks=((n, nmb, 6), np.int32), costs=((n, nmb, 2), np.int64),
                    coeffs=((n, nmb, 256), np.int16), ccoeffs=((n, nmb, 128), np.int16),
                    rec_y=(ins[0].shape, np.uint8), rec_u=(ins[1].shape, np.uint8), rec_v=(ins[2].shape, np.uint8))
        if net is not None:
            want["props"] = ((n, nmb, 16), np.int32)
            want["fallback"] = ((n, nmb), np.int32)
        if out is None:
            out = {k: np.zeros(shp, dt) for k, (shp, dt) in want.items()}
        for k, (shp, dt) in want.items():
            a = out.get(k)
            if a is None or a.shape != tuple(shp) or a.dtype != dt or not a.flags.c_contiguous:
                raise ValueError(f"pixel_path_closed: out[{k!r}] must be a C-contiguous {dt.__name__} array {shp}")
        p = lambda k: out[k].ctypes.data if k in out else None
        job = ClosedJob(ins[0].ctypes.data, ins[1].ctypes.data, ins[2].ctypes.data, n, cw, ch, float(lambda_me),
                        int(split_gate), qp, dz_div, None if net is None else net.h.value, int(fallback_t),
                        p("picks"), p("costs"), p("coeffs"), p("ccoeffs"), p("rec_y"), p("rec_u"), p("rec_v"),
                        p("props"), p("fallback"))
        self._check(self.L.h264a_pixel_path_closed(self.ctx, C.byref(job), C.byref(params),
                                                   None if tab is None else tab.ctypes.data_as(C.c_void_p)))
        return out

    def closed_frames(self, job: ClosedDev, params: MeParams):
        """The closed loop on device buffers (h264a_closed_frames), enqueued on
        the current stream."""
        self._check(self.L.h264a_closed_frames(self.ctx, C.byref(job), C.byref(params), self._stream()))

    def closed_step(self, step: ClosedStep, params: MeParams):
        """One P frame of the closed loop (h264a_closed_step_frame): the search
        with each MB's reconstruction and deblocking fused in, enqueued on the
        current stream."""
        self._check(self.L.h264a_closed_step_frame(self.ctx, C.byref(step), C.byref(params), self._stream()))

    # ---- end to end from host memory --------------------------------------------
    def pixel_path_prefetch(self, frames: np.ndarray):
        """Queues the upload of frames (n, ch, cw) u8, C-contiguous (pinned for
        an asynchronous copy), for the next pixel_path_host call on them.  The
        array is kept alive here until then; do not change it meanwhile."""
        if not frames.flags.c_contiguous or frames.dtype != np.uint8 or frames.ndim != 3:
            raise ValueError("pixel_path_prefetch needs a C-contiguous (n, ch, cw) uint8 array")
        n, ch, cw = frames.shape
        self._check(self.L.h264a_pixel_path_prefetch(self.ctx, frames.ctypes.data_as(C.c_void_p), n, cw, ch))
        self._prefetched.append((frames.ctypes.data, frames))  # released by the call that takes it

    def pixel_path_host(self, frames: np.ndarray, params: MeParams, lambda_me: float, split_gate: int, qp: int,
                        dz_div: int = 6, tab: Optional[np.ndarray] = None, out=None):
        n, ch, cw = frames.shape
        nmb = (cw // 16) * (ch // 16)
        if out is None:
            out = dict(picks=np.zeros((n, nmb, 6), np.int32), costs=np.zeros((n, nmb, 2), np.int64),
                       coeffs=np.zeros((n, nmb, 256), np.int16), la_intra=np.zeros((n, nmb), np.int32),
                       la_inter=np.zeros((n, nmb), np.int32), la_mvs=np.zeros((n, nmb, 2), np.int32))
        fr = np.ascontiguousarray(frames)
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        self._check(self.L.h264a_pixel_path_host(
            self.ctx, ptr(fr), n, cw, ch, C.byref(params), None if tab is None else ptr(tab), float(lambda_me),
            int(split_gate), qp, dz_div, ptr(out["picks"]), ptr(out["costs"]), ptr(out["coeffs"]),
            ptr(out["la_intra"]), ptr(out["la_inter"]), ptr(out["la_mvs"])))
        for i, (addr, _) in enumerate(self._prefetched):  # the oldest prefetch of these frames is used up
            if addr == fr.ctypes.data:
                del self._prefetched[i]
                break
        return out


class Batch:
    """A batch of streams on the device (h264a_batch_*): step(k, count)
    enqueues step k on the current stream as one graph launch; info() reports
    the launch shape and the tuner's timings."""

    def __init__(self, acc: Accel, handle: C.c_void_p):
        self.acc, self.h = acc, handle

    def step(self, k: int, count: int):
        self.acc._check(self.acc.L.h264a_batch_step(self.h, int(k), int(count), self.acc._stream()))

    def info(self) -> dict:
        bi = BatchInfo()
        self.acc._check(self.acc.L.h264a_batch_get_info(self.h, C.byref(bi)))
        return {"variant": bi.variant, "tuned": bool(bi.tuned), "ms": [round(float(x), 4) for x in bi.ms],
                "graphs": bi.graphs, "steps": bi.steps}

    def close(self):
        if self.h:
            self.acc.L.h264a_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_variant_shape(variant: int):
    """(MBs per CTA, staged window) of launch shape `variant` (host-only)."""
    L = load_library()
    n, st = C.c_int(), C.c_int()
    rc = L.h264a_batch_variant_shape(int(variant), C.byref(n), C.byref(st))
    if rc != H264A_OK:
        raise AccelError(rc, L.h264a_last_error().decode())
    return n.value, bool(st.value)
