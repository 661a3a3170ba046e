"""The reference tests' pseudo-random streams, reproduced bit-for-bit.

`lcg64` is the 64-bit LCG the accel and encoder tests use
(`state = state*6364136223846793005 + 1442695040888963407`, output
`state >> 33`; e.g. crates/rusty_h264-accel/src/satd_sad.rs:422-425).
`lcg32` is the 32-bit LCG of the common/inter.rs and transform.rs tests
(`state*1664525 + 1013904223`).  Bulk generation uses the closed form
state_k = A^k*s0 + c*(1 + A + ... + A^(k-1)) mod 2^64 in numpy.
"""
import numpy as np

A64 = np.uint64(6364136223846793005)
C64 = np.uint64(1442695040888963407)


class Lcg64:
    def __init__(self, seed: int):
        self.state = seed & 0xFFFFFFFFFFFFFFFF

    def next(self) -> int:
        self.state = (self.state * 6364136223846793005 + 1442695040888963407) & 0xFFFFFFFFFFFFFFFF
        return self.state >> 33

    def bulk(self, n: int) -> np.ndarray:
        """Next n outputs (state >> 33, as uint64)."""
        if n == 0:
            return np.zeros(0, np.uint64)
        with np.errstate(over="ignore"):
            ak = np.cumprod(np.full(n, A64, np.uint64), dtype=np.uint64)  # A^1..A^n
            pw = np.concatenate([np.ones(1, np.uint64), ak[:-1]])         # A^0..A^(n-1)
            ck = np.cumsum(pw, dtype=np.uint64) * C64                      # c*(A^0+..+A^(k-1))
            st = ak * np.uint64(self.state) + ck
        self.state = int(st[-1])
        return st >> np.uint64(33)

    def bytes(self, n: int) -> np.ndarray:
        return (self.bulk(n) & np.uint64(0xFF)).astype(np.uint8)


class Lcg32:
    def __init__(self, seed: int, a: int = 1664525, c: int = 1013904223):
        self.state = seed & 0xFFFFFFFF
        self.a, self.c = a, c

    def next(self) -> int:
        self.state = (self.state * self.a + self.c) & 0xFFFFFFFF
        return self.state
