"""Known-answer cases of motion_search and of the lookahead's inter_cost on
tiny constructed cost surfaces, each traced by hand through the reference's
code.  They pin the oracle (and, in test_gpu_parity's mirror, the GPU search)
to the reference's control flow independently of the restatements.

The surfaces are ramps: the reference row is 40 + 2x, the source the same
ramp offset by 2s, so at a full- or half-pel MV mx (quarter-pel) the residual
is the constant 2s - mx/2 and every 16x16 distortion is 256 |2s - mx/2| (the
6-tap filter reproduces a linear ramp exactly; SATD and SAD of a constant
block agree).  The searches run one diamond rung (step 4, 1 px: dia_mask
0b10000) without sub-pel refinement, so every evaluation can be listed.
mvbits (mb16.rs:2478-2480): 1 + 2 floor(log2(codenum + 1)), codenum 2d - 1
for d > 0 and -2d otherwise: bits(0) = 1, bits(+-2) = 5, bits(4) = 7,
bits(-6) = 7, bits(8) = 9, bits(12) = 9, bits(16) = 11.
"""
import numpy as np
import pytest

from oracle import oracle as O

W = H = 96
X = np.arange(W)
REF = np.tile((40 + 2 * X).astype(np.uint8), (H, 1))
PLANES = O.build_planes4(REF, 32)


def ramp_src(two_s):
    """The reference ramp offset by two_s (= 2 x the shift in pixels)."""
    return np.tile((40 + 2 * X + two_s).astype(np.uint8), (H, 1))


def search(src, preds, lam, **kw):
    pr = O.balanced_params(dia_mask=0b10000, subpel=0, **kw)
    return O.motion_search(src, REF, PLANES, pr, 32, 32, 16, 16, preds, lam)


def test_ramp_distortions_are_linear():
    """The surfaces the cases below rely on: D(mx) = 128 |4s - mx|."""
    src = ramp_src(6)  # s = 3 px: zero at mx = 12
    for mx in range(-4, 21, 2):
        assert O.candidate_dist(src, REF, PLANES, 0, 32, 32, 16, 16, mx, 0) == 128 * abs(12 - mx)
        assert O.candidate_dist(src, REF, PLANES, 0, 32, 32, 16, 16, mx, 4) == 128 * abs(12 - mx)


def test_fixed_centre_arm_prices_16_wide_rates_with_lam_fp():
    """mb16.rs:2686-2690: the fixed-centre batch arm of a 16-wide block adds
    (lam_fp * rate) with lam_fp = lambda (no B2), while `cost` (the seeds and
    every other arm) uses lam_r = lambda / 4 under the table rate models
    (mv_cost_kind 1).  lambda = 40, the smooth table (tab[0] = 3, tab[4] = 25):
      seeds: (0,0) and the predictor (0,0): 1536 + floor(10 * 6) = 1596;
      rung 4, fixed arm around (0,0): (4,0) 1024 + 40 * 28 = 2144,
      (-4,0) 2048 + 1120, (0,+-4) 1536 + 1120: none below 1596, the rung ends.
    Result (0,0) at 1596 after 6 evaluations.  Priced with lam_r instead,
    (4,0) would cost 1024 + 280 and the walk would reach (12,0).
    With the Exp-Golomb model (kind 0) lam_r = lam_fp and the walk goes
    (4,0) 1344 -> (8,0) 912 -> (12,0) 400, the zero of the ramp."""
    tab = O.mv_cost_table()
    assert (tab[0], tab[4]) == (3, 25)
    src = ramp_src(6)
    assert search(src, [(0, 0)], 40.0, mv_cost_kind=1) == ((0, 0), 1596, 6)
    assert search(src, [(0, 0)], 40.0, mv_cost_kind=0) == ((12, 0), 400, 18)
    # with lambda = 10 the quirk no longer blocks the first step, and the cost
    # the walk returns is the fixed arm's: 0 + 10 * (tab[12] + tab[0]) = 390,
    # not floor(2.5 * 39)
    assert tab[12] == 36
    assert search(src, [(0, 0)], 10.0, mv_cost_kind=1) == ((12, 0), 390, 18)


def test_fractional_seed_snaps_to_full_pel():
    """mb16.rs:2597-2607: a fractional winning seed is snapped to the nearest
    full-pel vector ((v + 2) div_euclid 4 * 4), priced, and the diamond starts
    there.  Source shift 2 px (zero at mx = 8), predictor (6,0), lambda 40:
      seeds: (0,0) 1024 + 40 * (bits(-6) + 1) = 1344, (6,0) 256 + 80 = 336;
      snap: (8,0) 0 + 40 * (bits(2) + 1) = 240 (7th evaluation);
      rung 4 around (8,0): (12,0) and (4,0) 512 + ..., (8,+-4) 480: no move.
    Result (8,0) at 240 (below the seed's 336, so no restore).  Without the
    snap (me_snap 0) the diamond runs the cascade arm around (6,0) and finds
    nothing below 336: (6,0)."""
    src = ramp_src(4)
    assert search(src, [(6, 0)], 40.0) == ((8, 0), 240, 7)
    assert search(src, [(6, 0)], 40.0, me_snap=0) == ((6, 0), 336, 6)


def test_seed_restore_returns_the_pre_snap_seed():
    """mb16.rs:3297-3300: after refinement, a snapped search whose result
    costs more than the pre-snap seed returns the seed.  Source shift 0.5 px
    (zero at mx = 2), predictor (2,0), lambda 40:
      seeds: (0,0) 256 + 40 * 6 = 496, (2,0) 0 + 80 = 80 (the seed);
      snap: (4,0) 256 + 40 * (bits(2) + 1) = 496;
      rung 4 around (4,0): (0,0) 496 (not below), (8,0) 768 + ...,
      (4,+-4) 256 + 480: no move, best 496.
    seed_c 80 < 496: the search returns (2,0) at 80."""
    src = ramp_src(1)
    assert search(src, [(2, 0)], 40.0) == ((2, 0), 80, 7)


def test_cascade_moves_the_ring_centre_mid_ring():
    """mb16.rs:2708-2727: the cascade arm (me_fc 0) walks the four points in
    the order (+s,0), (-s,0), (0,+s), (0,-s), each relative to the CURRENT
    best, so an improvement moves the centre of the rest of the ring.
    Reference 10 + 2x + y (64x64), source = reference + 3, so
    D(dx, dy px) = 256 |3 - 2dx - dy|; predictor (0,0), lambda 4:
      seeds (0,0) and (0,0): 768 + 8;
      ring 1: (4,0) 256 + 32 = 288 moves; (-4,0) from (4,0) is (0,0): 776;
              (0,4) from (4,0) is (4,4): 0 + 4 * 14 = 56 moves;
              (0,-4) from (4,4) is (4,0): 288;
      ring 2 around (4,4): (8,4) 512 + ..., (0,4) 512 + ..., (4,8) 256 + ...,
              (4,0) 288: no move.
    Result (4,4) at 56 after 2 + 4 + 4 = 10 evaluations.  Around a fixed
    centre the same surface takes three rings (14 evaluations): (4,0), then
    (4,4), then a ring without a move."""
    n = 64
    xx, yy = np.arange(n)[None, :], np.arange(n)[:, None]
    ref = (10 + 2 * xx + yy).astype(np.uint8)
    src = (ref + 3).astype(np.uint8)
    planes = O.build_planes4(ref, 32)
    for mx, my in ((0, 0), (4, 0), (4, 4), (0, 4), (8, 4)):
        assert O.candidate_dist(src, ref, planes, 0, 16, 16, 16, 16, mx, my) == 256 * abs(3 - 2 * (mx // 4) - my // 4)
    pr = O.balanced_params(dia_mask=0b10000, subpel=0, me_fc=0)
    assert O.motion_search(src, ref, planes, pr, 16, 16, 16, 16, [(0, 0)], 4.0) == ((4, 4), 56, 10)
    pr = O.balanced_params(dia_mask=0b10000, subpel=0, me_fc=1)
    assert O.motion_search(src, ref, planes, pr, 16, 16, 16, 16, [(0, 0)], 4.0) == ((4, 4), 56, 14)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_lookahead_zero_residual_exits_with_zero_mv(mode):
    """mbtree.rs:165-167 (inter_cost): a block whose (0,0) residual SATD is 0
    returns (0, (0,0)) at once, whatever its neighbour seed.  Frame 1 moves
    its left MB column (content shifted 4 px, so those MBs find a non-zero
    MV) and keeps the rest static: the static MBs right of a moving one are
    seeded with its MV and still return inter cost 0 and MV (0,0)."""
    rng = np.random.default_rng(11)
    f0 = rng.integers(0, 256, (64, 96)).astype(np.uint8)
    f1 = f0.copy()
    f1[:, :16] = np.roll(f0, 4, axis=1)[:, :16]
    _, inter, mvs = O.lookahead_clip(np.stack([f0, f1]), mode=mode)
    mb_w = 96 // 16
    moving = mvs[1].reshape(-1, mb_w, 2)[:, 0]
    assert (moving != 0).any()
    static_inter = inter[1].reshape(-1, mb_w)[:, 2:]
    static_mvs = mvs[1].reshape(-1, mb_w, 2)[:, 2:]
    assert (static_inter == 0).all() and (static_mvs == 0).all()
