"""h264a_me_frames_noalloc: the plain-ME entry point for callers that cannot
allocate device memory while they encode (an encoder thread that must not
block on the CUDA allocator, or a host that owns every buffer under a fixed
budget).  Through the C ABI it must give exactly what h264a_me_frames gives
(integer work: zero tolerance), on two calls in a row sharing its fixed
scratch array, and refuse a request larger than that array.

This file is collected last, so a run that stops at the first failure has run
every other test before it.  The comparison runs here, after the rest of the
suite in the same process, and once more in a fresh Python process of its own
(test_noalloc_in_a_fresh_process), where the entry point's first call on the
device is the one that looks up its scratch array.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from rusty_h264_b200 import accel as A
from rusty_h264_b200 import synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    a = A.Accel(0)
    yield a
    a.close()


def frames_for(acc, clip, lam, gate):
    """(frames for the existing entry, frames for the no-alloc entry) over the
    same sources/planes but separate output buffers."""
    n, ch, cw = clip.shape
    nmb = (cw // 16) * (ch // 16)
    d = acc.to_dev(clip)
    planes = acc.hpel_build(d[: n - 1], 32)
    keep = [d, planes]
    ref_frames, new_frames, outs = [], [], []
    for i in range(1, n):
        pic = A.Picture(d[i].data_ptr(), planes[i - 1].data_ptr(), cw, ch, 32)
        pk_a = acc.zeros((nmb, 6), acc.torch.int32)
        co_a = acc.zeros((nmb, 2), acc.torch.int64)
        pk_b = acc.torch.full((nmb, 6), -7, dtype=acc.torch.int32, device="cuda:0")
        co_b = acc.torch.full((nmb, 2), -7, dtype=acc.torch.int64, device="cuda:0")
        keep += [pk_a, co_a, pk_b, co_b]
        outs.append((pk_a, co_a, pk_b, co_b))
        ref_frames.append(A.MeFrame(pic, lam, gate, pk_a.data_ptr(), co_a.data_ptr()))
        new_frames.append(A.MeFrame(pic, lam, gate, pk_b.data_ptr(), co_b.data_ptr()))
    return ref_frames, new_frames, outs, keep


def call_noalloc(acc, frames, params, status):
    arr = (A.MeFrame * len(frames))(*frames)
    return acc.L.h264a_me_frames_noalloc(C.cast(arr, C.c_void_p), len(frames), C.byref(params), status.data_ptr(),
                                         C.c_void_p(acc.torch.cuda.current_stream().cuda_stream))


@pytest.mark.parametrize("case", [0, 1])
def test_noalloc_matches_me_frames_on_two_consecutive_calls(acc, case):
    y, _, _ = synth.cif_clip(6, 3)
    clip = synth.coded_luma(y)
    status = acc.torch.full((1,), 99, dtype=acc.torch.int32, device="cuda:0")
    # two calls in a row: a 5-frame CIF batch with splits, then a different
    # mixed-size batch with other parameters; each against h264a_me_frames
    runs = [
        (clip, A.default_me_params(), float(np.sqrt(A.frame_lambda(26))), A.split_gate_for_qp(26)),
        (np.ascontiguousarray(clip[:3, 16:144, 32:240]), A.default_me_params(sadfp=1),
         float(np.sqrt(A.frame_lambda(32)) * 1.25), A.split_gate_for_qp(32)),
    ]
    if case == 1:
        runs.reverse()
    for clip_i, params, lam, gate in runs:
        ref_frames, new_frames, outs, keep = frames_for(acc, clip_i, lam, gate)
        acc.me_frames(ref_frames, params)
        rc = call_noalloc(acc, new_frames, params, status)
        assert rc == 0, acc.L.h264a_last_error()
        acc.sync()
        assert int(status.item()) == 0
        for pk_a, co_a, pk_b, co_b in outs:
            assert np.array_equal(pk_a.cpu().numpy(), pk_b.cpu().numpy())
            assert np.array_equal(co_a.cpu().numpy(), co_b.cpu().numpy())
        del keep


def test_noalloc_rejects_requests_beyond_its_scratch(acc):
    buf = acc.zeros((64,), acc.torch.uint8)
    p = buf.data_ptr()
    # nine 1080p frames are 73,440 macroblocks, more than H264A_NOALLOC_MAX_MBS
    frames = [A.MeFrame(A.Picture(p, p, 1920, 1088, 32), 5.0, -1, p, p) for _ in range(9)]
    status = acc.zeros((1,), acc.torch.int32)
    rc = call_noalloc(acc, frames, A.default_me_params(), status)
    assert rc == -1
    assert b"exceed" in acc.L.h264a_last_error()


def test_noalloc_in_a_fresh_process():
    """The two-call comparison again, alone in a new interpreter: there the
    no-alloc entry's set-up (the per-device address lookup) runs on a device
    that nothing else in the process has touched through it before."""
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    node = os.path.abspath(__file__) + "::test_noalloc_matches_me_frames_on_two_consecutive_calls"
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider", node],
                       cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "2 passed" in r.stdout, r.stdout[-3000:]
