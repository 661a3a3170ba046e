"""The Annex-B output of the frame model (h264a_write_stream_cavlc, host code
of the library) against the reference: its VLC tables equal the ones the
reference's cavlc.rs holds (parsed into tests/golden/reference_cavlc_tables.json),
and its streams decode, with the oracle's restatement of the reference
decoder's CAVLC path (oracle/h264_decoder.c, driven by those same parsed
tables), to exactly the encoder's reconstruction and syntax.  No GPU: the
frames come from the oracle's closed loop."""
import ctypes as C
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from rusty_h264_b200 import accel as A
from rusty_h264_b200 import synth

HERE = os.path.dirname(os.path.abspath(__file__))


def _code(L, tab, i, j, k):
    ln, bits = C.c_int(), C.c_int()
    assert L.h264a_cavlc_table_code(tab, i, j, k, C.byref(ln), C.byref(bits)) == 0
    return ln.value, bits.value


def test_writer_vlc_tables_equal_the_reference_tables():
    L = A.load_library()
    t = json.load(open(os.path.join(HERE, "golden", "reference_cavlc_tables.json")))
    for cls in range(3):
        for tc in range(17):
            for t1 in range(4):
                want = (t["COEFF_TOKEN_LEN"][cls][tc * 4 + t1], t["COEFF_TOKEN_BITS"][cls][tc * 4 + t1])
                assert _code(L, 0, cls, tc, t1) == want, (cls, tc, t1)
    for tc in range(5):
        for t1 in range(4):
            want = (t["CHROMA_DC_COEFF_TOKEN_LEN"][tc * 4 + t1], t["CHROMA_DC_COEFF_TOKEN_BITS"][tc * 4 + t1])
            assert _code(L, 1, 0, tc, t1) == want
    for tc in range(1, 16):
        for z in range(16):
            assert _code(L, 2, 0, tc, z) == (t["TOTAL_ZEROS_LEN"][tc - 1][z], t["TOTAL_ZEROS_BITS"][tc - 1][z])
    for tc in range(1, 4):
        for z in range(4):
            want = (t["CHROMA_DC_TOTAL_ZEROS_LEN"][tc - 1][z], t["CHROMA_DC_TOTAL_ZEROS_BITS"][tc - 1][z])
            assert _code(L, 3, 0, tc, z) == want
    for zl in range(1, 8):
        for r in range(15):
            assert _code(L, 4, 0, zl, r) == (t["RUN_LEN"][zl - 1][r], t["RUN_BITS"][zl - 1][r])
    for code_num, cbp in enumerate(t["CBP_INTER"]):
        assert _code(L, 5, 0, cbp, 0)[1] == code_num


def _round_trip(Y, U, V, qp, width=None, height=None):
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    r = O.closed_loop_clip(Y, U, V, O.balanced_params(), lam, A.split_gate_for_qp(qp), qp)
    data, fb = A.write_stream_cavlc(Y[0], U[0], V[0], r["picks"], r["coeffs"], r["ccoeffs"], qp, width, height)
    n, ch, cw = Y.shape
    d = O.decode_stream(data, cw, ch, n + 1)
    assert len(d["y"]) == n
    for k, g in (("y", "rec_y"), ("u", "rec_u"), ("v", "rec_v")):
        assert np.array_equal(d[k], r[g]), k
    assert np.array_equal(d["picks"][1:, :, :5], r["picks"][1:, :, :5])
    assert np.array_equal(d["coeffs"], r["coeffs"]) and np.array_equal(d["ccoeffs"], r["ccoeffs"])
    assert fb.sum() == len(data)
    return r, data, fb


@pytest.mark.parametrize("qp", [22, 37])
def test_cif_stream_decodes_to_the_reconstruction(qp):
    Y = synth.coded_luma(synth.cif_clip(6, 1)[0])
    _, U, V = synth.cif_clip(6, 1)
    r, data, fb = _round_trip(Y, U, V, qp)
    # frame 0 is I_PCM: 384 bytes per MB plus headers
    assert fb[0] >= 396 * 384
    assert (r["picks"][1:, :, 0] > 0).any() or qp == 37


def test_cropped_textured_stream_decodes_to_the_reconstruction():
    """A 300x264 clip (coded 304x272, display cropped in the SPS) of the
    textured generator with partitions and large motion."""
    y, u, v = synth.hd_clip(4, 3, 300, 264, with_chroma=True)
    Y, U, V = synth.coded_luma(y), synth.coded_chroma(u), synth.coded_chroma(v)
    assert Y.shape[1:] == (272, 304)
    r, _, _ = _round_trip(Y, U, V, 24, 300, 264)
    assert (r["picks"][1:, :, 0] > 0).any()


def test_large_levels_and_every_pick_shape_round_trip():
    """Levels up to +-3000 (the escape codes of level_prefix 15 and beyond),
    trailing-one runs, every pick shape and MVs far from their predictors:
    the decoder parses back exactly the syntax written."""
    rng = np.random.default_rng(8)
    cw, ch, n = 64, 48, 3
    nmb = (cw // 16) * (ch // 16)
    Y = rng.integers(0, 256, (n, ch, cw)).astype(np.uint8)
    U = rng.integers(0, 256, (n, ch // 2, cw // 2)).astype(np.uint8)
    V = rng.integers(0, 256, (n, ch // 2, cw // 2)).astype(np.uint8)
    picks = np.zeros((n, nmb, 6), np.int32)
    picks[1:, :, 0] = rng.integers(0, 3, (n - 1, nmb))
    picks[1:, :, 1:5] = rng.integers(-300, 300, (n - 1, nmb, 4))
    picks[1:, :, 3:5] = np.where(picks[1:, :, :1] == 0, picks[1:, :, 1:3], picks[1:, :, 3:5])
    coeffs = np.zeros((n, nmb, 256), np.int16)
    ccoeffs = np.zeros((n, nmb, 128), np.int16)
    mag = rng.choice([1, 1, 1, 2, 5, 40, 3000], (n - 1, nmb, 256))
    keep = rng.random((n - 1, nmb, 256)) < 0.3
    coeffs[1:] = (mag * rng.choice([-1, 1], mag.shape) * keep).astype(np.int16)
    coeffs[1:, 1, :] = 0  # an MB without luma levels
    cm = rng.choice([1, 1, 2, 9, 700], (n - 1, nmb, 128))
    ccoeffs[1:] = (cm * rng.choice([-1, 1], cm.shape) * (rng.random(cm.shape) < 0.4)).astype(np.int16)
    ccoeffs[1:, 2, :] = 0
    ccoeffs[1:, 3, :] = 0
    ccoeffs[1:, 3, 0] = 5  # chroma DC only
    data, _ = A.write_stream_cavlc(Y[0], U[0], V[0], picks, coeffs, ccoeffs, 10)
    d = O.decode_stream(data, cw, ch, n)
    assert np.array_equal(d["y"][0], Y[0]) and np.array_equal(d["u"][0], U[0])
    assert np.array_equal(d["picks"][1:, :, :5], picks[1:, :, :5])
    assert np.array_equal(d["coeffs"], coeffs) and np.array_equal(d["ccoeffs"], ccoeffs)


def test_writer_rejects_bad_input():
    y = np.zeros((48, 64), np.uint8)
    c = np.zeros((24, 32), np.uint8)
    picks = np.zeros((2, 12, 6), np.int32)
    picks[1, 0, 0] = 3
    with pytest.raises(A.AccelError):
        A.write_stream_cavlc(y, c, c, picks, np.zeros((2, 12, 256), np.int16), np.zeros((2, 12, 128), np.int16), 26)
    with pytest.raises(A.AccelError):  # display size more than a MB below the coded size
        A.write_stream_cavlc(y, c, c, np.zeros((1, 12, 6), np.int32), np.zeros((1, 12, 256), np.int16),
                             np.zeros((1, 12, 128), np.int16), 26, 40, 48)
