"""Bjontegaard-delta rate and PSNR, as the reference's BD-rate tool computes
them (bench/examples/bdrate.rs): PSNR from the luma squared error summed over
every frame of a decoded stream against its source (bdrate.rs:164-179), and
the BD-rate of a test curve against an anchor from least-squares cubic fits
of log10(rate) over PSNR, integrated over the PSNRs both curves cover
(polyfit3 bdrate.rs:189-228, bd_rate :232-250)."""
from __future__ import annotations

import numpy as np


def psnr(src: np.ndarray, dec: np.ndarray) -> float:
    """PSNR (dB) of decoded luma frames against their source, from the
    squared error summed over all frames (99 for a lossless match)."""
    d = src.astype(np.float64) - dec.astype(np.float64)
    mse = float((d * d).mean())
    return 99.0 if mse <= 0.0 else 10.0 * np.log10(255.0 * 255.0 / mse)


def polyfit3(x, y) -> np.ndarray:
    """Coefficients c0..c3 of the least-squares cubic through (x, y): the
    normal equations A[j][k] = sum x^(j+k), b[j] = sum y x^j, solved by
    Gauss-Jordan elimination with partial pivoting."""
    a = np.zeros((4, 4))
    b = np.zeros(4)
    for xi, yi in zip(x, y):
        xp = xi ** np.arange(7)
        for j in range(4):
            a[j] += xp[j:j + 4]
            b[j] += yi * xp[j]
    for c in range(4):
        piv = c + int(np.argmax(np.abs(a[c:, c])))
        a[[c, piv]] = a[[piv, c]]
        b[[c, piv]] = b[[piv, c]]
        for r in range(4):
            if r != c:
                f = a[r, c] / a[c, c]
                a[r, c:] -= f * a[c, c:]
                b[r] -= f * b[c]
    return b / np.diag(a)


def bd_rate(anchor, test) -> float:
    """BD-rate (%) of `test` against `anchor`, each a list of (rate, psnr)
    points: negative means the test curve spends fewer bits at equal PSNR."""
    def prep(p):
        v = sorted((d, np.log10(r)) for r, d in p)
        return [q[0] for q in v], [q[1] for q in v]

    da, la = prep(anchor)
    dt, lt = prep(test)
    ca, ct = polyfit3(da, la), polyfit3(dt, lt)
    lo, hi = max(da[0], dt[0]), min(da[-1], dt[-1])
    integ = lambda c, x: c[0] * x + c[1] * x * x / 2 + c[2] * x ** 3 / 3 + c[3] * x ** 4 / 4
    avg = (integ(ct, hi) - integ(ct, lo) - (integ(ca, hi) - integ(ca, lo))) / (hi - lo)
    return (10.0 ** avg - 1.0) * 100.0
