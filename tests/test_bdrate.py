"""The BD-rate restatement (rusty_h264_b200/bdrate.py, after the reference's
bench/examples/bdrate.rs) on curves with known answers."""
import numpy as np

from rusty_h264_b200 import bdrate


def test_polyfit3_recovers_a_cubic():
    x = np.array([30.0, 33.0, 36.5, 40.0, 42.0])
    c = np.array([0.5, -0.25, 0.01, -0.0002])
    y = c[0] + c[1] * x + c[2] * x ** 2 + c[3] * x ** 3
    assert np.allclose(bdrate.polyfit3(x, y), c, rtol=1e-6, atol=1e-9)


def test_bd_rate_known_answers():
    anchor = [(1000.0, 32.0), (1800.0, 35.0), (3200.0, 38.0), (6000.0, 41.0)]
    assert abs(bdrate.bd_rate(anchor, anchor)) < 1e-9
    # the same curve at 10% more rate everywhere: +10%
    assert abs(bdrate.bd_rate(anchor, [(r * 1.1, d) for r, d in anchor]) - 10.0) < 1e-6
    # 5% less rate: -5%
    assert abs(bdrate.bd_rate(anchor, [(r * 0.95, d) for r, d in anchor]) + 5.0) < 1e-6


def test_psnr():
    a = np.full((2, 4, 4), 100, np.uint8)
    assert bdrate.psnr(a, a) == 99.0
    b = a.copy()
    b[0, 0, 0] = 110  # mse = 100 / 32
    assert abs(bdrate.psnr(a, b) - 10 * np.log10(255 ** 2 / (100 / 32))) < 1e-9
