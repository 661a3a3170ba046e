"""GPU: the batched plain-ME runtime (h264a_batch_*) against the oracle.

Streams of three sizes step G P frames per graph launch over three
references; every frame's picks and costs equal the oracle's best_part over
the same references (oracle/h264_oracle.c, or_me_frame_multiref), through
graph captures, replays, the warm-up frames with fewer references and a
short last step, for the autotuned launch shape and for every shape forced.
"""
import numpy as np
import pytest

from oracle import oracle as O
from rusty_h264_b200 import accel as A
from rusty_h264_b200 import synth

pytestmark = pytest.mark.gpu

NREF, G, NSLOTS, PAD = 3, 2, 8, 32


@pytest.fixture(scope="module")
def acc():
    a = A.Accel(0)
    yield a
    a.close()


def _clips(nframes: int):
    """CIF (the CIF generator), 384x272 (the textured 1080p generator at that
    size) and 48x32 (seeded noise panning (+1, -1) px per frame)."""
    cif = synth.coded_luma(synth.cif_clip(nframes, 7)[0])
    hd = synth.coded_luma(synth.hd_clip(nframes, 11, 384, 272)[0])
    rng = np.random.default_rng(5)
    big = rng.integers(0, 256, (32 + nframes + 8, 48 + nframes + 8)).astype(np.uint8)
    tiny = np.stack([big[8 + f: 8 + f + 32, 8 + nframes - f: 8 + nframes - f + 48] for f in range(nframes)])
    return [cif, hd, tiny]


class _Rings:
    """Each stream's device rings (sources, planes, picks, costs)."""

    def __init__(self, acc, clips, lam, gate, qp=None):
        torch = acc.torch
        self.clips, self.rings, self.streams, self.coeffs = clips, [], [], []
        for c in clips:
            _, ch, cw = c.shape
            nmb = (cw // 16) * (ch // 16)
            pb = 4 * (cw + 2 * PAD) * (ch + 2 * PAD)
            src = acc.zeros((NSLOTS, ch, cw), torch.uint8)
            planes = acc.zeros((NSLOTS, pb), torch.uint8)
            picks = acc.zeros((NSLOTS, nmb, 8), torch.int32)
            costs = acc.zeros((NSLOTS, nmb, 2), torch.int64)
            co = acc.zeros((NSLOTS, nmb, 256), torch.int16) if qp is not None else None
            self.rings.append((src, planes, picks, costs))
            self.coeffs.append(co)
            self.streams.append(A.BatchStream(cw, ch, PAD, src.data_ptr(), planes.data_ptr(), picks.data_ptr(),
                                              costs.data_ptr(), lam, gate, 0 if co is None else co.data_ptr(),
                                              qp or 0, 6))

    def upload(self, acc, frames):
        for c, (src, _, _, _) in zip(self.clips, self.rings):
            for f in frames:
                src[f % NSLOTS].copy_(acc.torch.from_numpy(np.ascontiguousarray(c[f])))

    def results(self, f):
        return [(r[2][f % NSLOTS].cpu().numpy(), r[3][f % NSLOTS].cpu().numpy()) for r in self.rings]

    def levels(self, f):
        return [co[f % NSLOTS].cpu().numpy() for co in self.coeffs]


def _run(acc, clips, lam, gate, params, autotune=1, variant=0, qp=None, levels=None):
    """Steps the batch over every P frame; returns {frame: [(picks, costs) per stream]} and the batch info
    (with qp, the luma levels of every frame go to levels[frame] too)."""
    n = clips[0].shape[0]
    rings = _Rings(acc, clips, lam, gate, qp)
    b = acc.batch_create(rings.streams, A.BatchConfig(G, NSLOTS, NREF, autotune, variant), params)
    out, k = {}, 0
    while k * G + 1 < n:
        count = min(G, n - 1 - k * G)
        rings.upload(acc, range(k * G, k * G + count + 1))
        b.step(k, count)
        acc.sync()
        for f in range(k * G + 1, k * G + count + 1):
            out[f] = rings.results(f)
            if qp is not None:
                levels[f] = rings.levels(f)
        k += 1
    info = b.info()
    b.close()
    return out, info


def _oracle(clip, f, lam, gate):
    refs = [f - 1 - r for r in range(min(NREF, f))]
    ro = np.stack([clip[r] for r in refs])
    po = np.stack([O.build_planes4(clip[r], PAD) for r in refs])
    return O.me_frame_multiref(clip[f], ro, po, O.balanced_params(), lam, gate)


def _setup(qp=27):
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    return lam, A.split_gate_for_qp(qp), A.default_me_params()


def test_batch_steps_match_oracle(acc):
    """18 frames of three streams: steps 0..8 (the last one frame), graphs
    captured for the 7 slot layouts and replayed for the others; every frame
    of every stream equals the oracle; the tuner timed all six shapes."""
    clips = _clips(18)
    lam, gate, params = _setup()
    out, info = _run(acc, clips, lam, gate, params)
    for f, res in sorted(out.items()):
        for s, (clip, (gp, gc)) in enumerate(zip(clips, res)):
            wp, wc = _oracle(clip, f, lam, gate)
            assert np.array_equal(gp[:, :7], wp[:, :7]), (f, s, np.argwhere(gp[:, :7] != wp[:, :7])[:4])
            assert np.array_equal(gc, wc), (f, s)
    assert info["tuned"] and all(m > 0 for m in info["ms"]) and 0 <= info["variant"] < A.BATCH_VARIANTS
    # layouts (slot of kG, warm-up, count): (0,0,2) (2,2,2) (4,3,2) (6,3,2) (0,3,2) (2,3,2), replays, (0,3,1)
    assert info["graphs"] == 7 and info["steps"] == 9
    picks = np.stack([out[f][0][0] for f in sorted(out)])
    assert set(np.unique(picks[2:, :, 1])) == {0, 1, 2}  # CIF picks use every reference


@pytest.mark.parametrize("variant", range(A.BATCH_VARIANTS))
def test_batch_every_launch_shape_matches(acc, variant):
    """Each launch shape forced (2, 4, 8 MBs per CTA; window staged or read
    from L2) gives the oracle's picks and costs on the first 6 frames."""
    clips = _clips(6)
    lam, gate, params = _setup(32)
    out, info = _run(acc, clips, lam, gate, params, autotune=0, variant=variant)
    assert info["variant"] == variant and not info["tuned"]
    for f, res in sorted(out.items()):
        for s, (clip, (gp, gc)) in enumerate(zip(clips, res)):
            wp, wc = _oracle(clip, f, lam, gate)
            assert np.array_equal(gp[:, :7], wp[:, :7]) and np.array_equal(gc, wc), (variant, f, s)


def test_batch_tuning_cached_per_signature(acc):
    """A batch whose signature was tuned before in the context takes the
    cached shape without timing again; invalid configurations are refused."""
    clips = _clips(4)
    lam, gate, params = _setup()
    _, first = _run(acc, clips, lam, gate, params)
    _, second = _run(acc, clips, lam, gate, params)
    assert second["tuned"] and second["variant"] == first["variant"] and all(m == 0 for m in second["ms"])
    rings = _Rings(acc, clips, lam, gate)
    for cfg in (A.BatchConfig(G, 7, NREF, 1, 0), A.BatchConfig(G, 4, NREF, 1, 0), A.BatchConfig(0, 8, NREF, 1, 0),
                A.BatchConfig(G, NSLOTS, 5, 1, 0), A.BatchConfig(G, NSLOTS, NREF, 0, A.BATCH_VARIANTS)):
        with pytest.raises(A.AccelError):
            acc.batch_create(rings.streams, cfg, params)
    b = acc.batch_create(rings.streams, A.BatchConfig(G, NSLOTS, NREF, 1, 0), params)
    with pytest.raises(A.AccelError):
        b.step(0, G + 1)
    b.close()


def test_batch_one_reference_one_frame_steps(acc):
    """G = 1, one reference, the smallest ring (3 slots): every step is one
    frame of each stream and equals h264a_me_frames_multiref's one-reference
    search (the oracle) frame by frame, across ring wrap-arounds."""
    global NREF, G, NSLOTS
    saved = (NREF, G, NSLOTS)
    NREF, G, NSLOTS = 1, 1, 3
    try:
        clips = _clips(7)
        lam, gate, params = _setup(30)
        out, info = _run(acc, clips, lam, gate, params, autotune=0, variant=3)
        assert info["steps"] == 6 and info["graphs"] == 4  # slots 0, 1, 2 (+ the warm-up layout of step 0)
        for f, res in sorted(out.items()):
            for s, (clip, (gp, gc)) in enumerate(zip(clips, res)):
                wp, wc = _oracle(clip, f, lam, gate)
                assert np.array_equal(gp[:, :7], wp[:, :7]) and np.array_equal(gc, wc), (f, s)
                assert (gp[:, 1] == 0).all() and (gp[:, 4] == 0).all()  # one reference: index 0 throughout
    finally:
        NREF, G, NSLOTS = saved


def _oracle_levels(src, refs, picks8, qp):
    """MC + luma T/Q of multi-reference picks from the single-reference
    oracle, each 4x4 block from the reference of its half."""
    nmb = picks8.shape[0]
    p6 = np.zeros((nmb, 6), np.int32)
    p6[:, 0], p6[:, 1:3], p6[:, 3:5] = picks8[:, 0], picks8[:, 2:4], picks8[:, 5:7]
    out = np.zeros((nmb, 256), np.int16)
    for r, ref in enumerate(refs):
        c = O.mc_tq_frame(src, ref, p6, qp)
        for by in range(0, 16, 4):
            for bx in range(0, 16, 4):
                part = np.where(picks8[:, 0] == 1, by >= 8, np.where(picks8[:, 0] == 2, bx >= 8, 0)).astype(int)
                sel = picks8[np.arange(nmb), 1 + 3 * part] == r
                off = ((2 if by >= 8 else 0) + (1 if bx >= 8 else 0)) * 64 + ((2 if by & 4 else 0) + (1 if bx & 4 else 0)) * 16
                out[sel, off:off + 16] = c[sel, off:off + 16]
    return out


def test_batch_steps_with_mc_tq(acc):
    """Streams with coefficient rings: each step's graph also runs the MC +
    luma T/Q of the step's frames from the picks, each half from its own
    reference; every frame's levels equal the oracle's and the picks still
    equal the oracle's search."""
    clips = _clips(8)
    qp = 28
    lam, gate, params = _setup(qp)
    levels = {}
    out, info = _run(acc, clips, lam, gate, params, qp=qp, levels=levels)
    assert info["graphs"] >= 3
    for f, res in sorted(out.items()):
        refs_idx = [f - 1 - r for r in range(min(NREF, f))]
        for s, (clip, (gp, gc)) in enumerate(zip(clips, res)):
            wp, wc = _oracle(clip, f, lam, gate)
            assert np.array_equal(gp[:, :7], wp[:, :7]) and np.array_equal(gc, wc), (f, s)
            want = _oracle_levels(clip[f], [clip[r] for r in refs_idx], gp, qp)
            assert np.array_equal(levels[f][s], want), (f, s)
    assert any((lv != 0).any() for lvs in levels.values() for lv in lvs)
