"""The C ABI library loads and exports exactly what include/h264accel.h declares
(CPU only: no kernel is launched)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from rusty_h264_b200 import accel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "h264accel.h")).read()
    return sorted(set(re.findall(r"H264A_API\s+[\w\s\*]*?\b(h264a_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(accel.LIB_PATH):
        pytest.skip("libh264accel_cuda.so not built (run __graft_entry__.build())")
    return accel.load_library()


def test_header_and_binding_agree():
    assert header_functions() == sorted(accel.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    for name in header_functions():
        assert hasattr(lib, name), name


def test_exported_surface_is_only_the_abi():
    if not os.path.exists(accel.LIB_PATH):
        pytest.skip("library not built")
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", accel.LIB_PATH], capture_output=True, text=True).stdout
    ours = sorted({ln.split()[-1] for ln in out.splitlines() if " T h264a_" in ln})
    assert ours == header_functions()


def test_version_and_defaults(lib):
    assert b"sm_100a" in lib.h264a_version()
    p = accel.default_me_params()
    assert (p.fast, p.sadfp, p.mv_cost_kind, p.me_snap, p.me_fc) == (0, 0, 0, 1, 1)
    assert (p.dia_mask, p.dia_sub_mask, p.subpel, p.sp_single_pass, p.sub_pat) == (0x1C, 0x10, 1, 1, 2)
    assert p.sadfp_lambda == 0.5 and p.subpel_pat == -1


def test_mv_cost_table_matches_oracle(lib):
    from oracle import oracle as O

    assert np.array_equal(accel.mv_cost_table(), O.mv_cost_table())


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror has the size and field offsets the C compiler gives the header's struct."""
    import subprocess

    from rusty_h264_b200.mvnet import MvnetFrame

    mirrors = {"h264a_picture": accel.Picture, "h264a_candidate": accel.Candidate, "h264a_me_params": accel.MeParams,
               "h264a_me_job": accel.MeJob, "h264a_me_result": accel.MeResult, "h264a_me_frame": accel.MeFrame,
               "h264a_me_tq_frame": accel.MeTqFrame,
               "h264a_tq_frame": accel.TqFrame, "h264a_tq_rec_frame": accel.TqRecFrame,
               "h264a_tq_chroma_frame": accel.TqChromaFrame, "h264a_deblock_frame": accel.DeblockFrame,
               "h264a_me_learned_frame": accel.MeLearnedFrame, "h264a_closed_job": accel.ClosedJob,
               "h264a_closed_dev": accel.ClosedDev, "h264a_closed_step": accel.ClosedStep,
               "h264a_stream_frames": accel.StreamFrames, "h264a_mvnet_frame": MvnetFrame,
               "h264a_me_mr_frame": accel.MeMrFrame, "h264a_batch_stream": accel.BatchStream,
               "h264a_batch_config": accel.BatchConfig, "h264a_batch_info": accel.BatchInfo,
               "h264a_la_stream": accel.LaStream, "h264a_mc_tq_mr_frame": accel.McTqMrFrame}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "h264accel.h"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(ln.rsplit(" ", 1) for ln in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split("\n") if ln)
    for cname, py in mirrors.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)


def test_context_without_device_fails_cleanly(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    ctx = C.c_void_p()
    rc = lib.h264a_ctx_create(0, C.byref(ctx))
    assert rc == -5 and not ctx.value  # H264A_E_NODEV
    assert b"no CUDA device" in lib.h264a_last_error()
    with pytest.raises(RuntimeError):
        accel.Accel()


def test_split_gate_and_lambda_helpers():
    # mb16.rs:8885-8887 and :8642
    assert accel.split_gate_for_qp(27) == ((30 * ((14 << 4) + 160)) >> 3) * 2
    assert abs(accel.frame_lambda(12) - 0.85) < 1e-12


def test_batch_launch_shapes(lib):
    """The autotuner's launch shapes: 2, 4 and 8 MBs per CTA, each with the
    window staged by TMA and read from L2; variant 0 is the default shape."""
    shapes = [accel.batch_variant_shape(v) for v in range(accel.BATCH_VARIANTS)]
    assert shapes[0] == (4, True)
    assert sorted(shapes) == sorted((n, st) for n in (2, 4, 8) for st in (False, True))
    with pytest.raises(accel.AccelError):
        accel.batch_variant_shape(accel.BATCH_VARIANTS)
