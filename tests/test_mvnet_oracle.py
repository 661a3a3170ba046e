"""The learned-proposal network's CPU oracle (oracle/mvnet_ref.py) checked
against itself by finite differences (float64, no bf16 rounding), and the
label mapping shared by the oracle and the host code."""
import numpy as np

from oracle import mvnet_ref as M
from rusty_h264_b200 import mvnet


def _params(rng):
    p = {}
    for n, s in M.SHAPES:
        fan = np.prod(s[1:]) if len(s) > 1 else 1
        p[n] = rng.normal(0, np.sqrt(2 / fan), s) if len(s) > 1 else rng.normal(0, 0.1, s)
    return M.flatten(p, np.float64)


def test_oracle_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    flat = _params(rng)
    P, ch, cw = 2, 48, 64  # two frame pairs of 4 x 3 MBs
    x0 = rng.integers(-128, 128, (P, ch, cw, 2)) / 64.0
    B = P * (ch // 16) * (cw // 16)
    nmv = rng.integers(-40, 40, (B, 6))
    lab = rng.integers(0, M.NCLS, B)
    _, g, _ = M.loss_and_grads(flat, x0, nmv, lab, round_bf16=False)
    o = 0
    for name, shp in M.SHAPES:
        k = int(np.prod(shp))
        for i in rng.integers(o, o + k, 3):
            e = 1e-6
            fp, fm = flat.copy(), flat.copy()
            fp[i] += e
            fm[i] -= e
            fd = (M.loss_and_grads(fp, x0, nmv, lab, False)[0] - M.loss_and_grads(fm, x0, nmv, lab, False)[0]) / (2 * e)
            assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (name, i, fd, g[i])
        o += k
    assert o == M.NPARAMS == mvnet.NPARAMS


def test_label_classes():
    mv = np.array([[0, 0], [1, 1], [2, -2], [-2, 2], [4, 0], [-6, 7], [33, -40], [1000, -1000], [30, 34]])
    got = mvnet.class_of_mv(mv)
    want = [M.class_of_mv(int(x), int(y)) for x, y in mv]
    assert list(got) == want
    assert M.class_of_mv(0, 0) == 8 * 17 + 8
    assert M.mv_of_class(M.class_of_mv(8, -12)) == (8, -12)
    assert M.mv_of_class(M.class_of_mv(1000, -1000)) == (32, -32)


def test_neighbour_mvs_rule():
    mvs = np.arange(2 * 12).reshape(12, 2)  # 4 x 3 MBs
    nb = mvnet.neighbour_mvs(mvs, 4, 3)
    g = mvs.reshape(3, 4, 2)
    assert (nb[0] == 0).all()
    assert list(nb[5]) == list(g[1, 0]) + list(g[0, 1]) + list(g[0, 2])
    assert list(nb[7][4:]) == [0, 0]  # right column: no top-right
    assert list(nb[4][:2]) == [0, 0]  # left column: no left

