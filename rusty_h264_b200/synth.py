"""Seeded synthetic YUV 4:2:0 clips for the benchmark and parity workloads.

The reference benchmarks on the Derf corpus, which is not available here;
these generators stand in for it with the shapes and statistics of the two
single-GPU workloads:

* ``cif_clip``: 352x288, horizontal gradient 0->235 scrolling 2 px/frame, a
  64x64 box of seeded uniform noise moving (+3,-1) px/frame, Gaussian noise
  sigma 2; chroma flat 128 plus sigma 1.
* ``hd_clip``: 1920x1080, 4-octave seeded value noise translated by
  (1.25,-0.5) px/frame (a 4x-upsampled texture decimated at the frame's
  quarter-pel phase), eight textured rectangles with sides U[32,256] and
  quarter-pel velocities U[-6,6] px/frame, Gaussian noise sigma 1.5.

``coded_luma`` edge-clamps a frame to the macroblock grid the way the encoder
prepares its source (crates/rusty_h264-encoder/src/mbtree.rs:45-56).
"""
from __future__ import annotations

import numpy as np


def coded_luma(y: np.ndarray) -> np.ndarray:
    h, w = y.shape[-2:]
    ch, cw = (h + 15) // 16 * 16, (w + 15) // 16 * 16
    rows = np.minimum(np.arange(ch), h - 1)
    cols = np.minimum(np.arange(cw), w - 1)
    return np.ascontiguousarray(y[..., rows[:, None], cols[None, :]])


def coded_chroma(c: np.ndarray) -> np.ndarray:
    """4:2:0 chroma edge-clamped to half the coded luma size (the luma
    rounded up to whole MBs), as the encoder prepares it
    (crates/rusty_h264-encoder/src/mb16.rs:1504-1506)."""
    h, w = c.shape[-2:]
    ch, cw = (2 * h + 15) // 16 * 8, (2 * w + 15) // 16 * 8
    rows = np.minimum(np.arange(ch), h - 1)
    cols = np.minimum(np.arange(cw), w - 1)
    return np.ascontiguousarray(c[..., rows[:, None], cols[None, :]])


def _to_u8(x: np.ndarray) -> np.ndarray:
    return np.clip(np.rint(x), 0, 255).astype(np.uint8)


def cif_clip(frames: int = 30, seed: int = 0, w: int = 352, h: int = 288):
    rng = np.random.default_rng(seed)
    box = rng.integers(0, 256, (64, 64)).astype(np.float32)
    x = np.arange(w, dtype=np.float32)
    ys, us, vs = [], [], []
    bx0, by0 = 40, 150
    for t in range(frames):
        grad = 235.0 * ((x + 2 * t) % w) / (w - 1)
        y = np.broadcast_to(grad, (h, w)).copy()
        bx, by = bx0 + 3 * t, by0 - t
        x0, y0 = max(bx, 0), max(by, 0)
        x1, y1 = min(bx + 64, w), min(by + 64, h)
        if x1 > x0 and y1 > y0:
            y[y0:y1, x0:x1] = box[y0 - by:y1 - by, x0 - bx:x1 - bx]
        y += rng.normal(0.0, 2.0, (h, w)).astype(np.float32)
        ys.append(_to_u8(y))
        us.append(_to_u8(128 + rng.normal(0.0, 1.0, (h // 2, w // 2))))
        vs.append(_to_u8(128 + rng.normal(0.0, 1.0, (h // 2, w // 2))))
    return np.stack(ys), np.stack(us), np.stack(vs)


def _value_noise(rng, H: int, W: int, octaves: int = 4, base: int = 128) -> np.ndarray:
    """Sum of bilinearly interpolated random lattices (cell base, base/2, ...)."""
    out = np.zeros((H, W), np.float32)
    amp, tot = 1.0, 0.0
    cell = base
    for _ in range(octaves):
        gh, gw = H // cell + 2, W // cell + 2
        g = rng.random((gh, gw), dtype=np.float32)
        yy = np.arange(H, dtype=np.float32) / cell
        xx = np.arange(W, dtype=np.float32) / cell
        y0 = yy.astype(np.int32)
        x0 = xx.astype(np.int32)
        fy = (yy - y0)[:, None]
        fx = (xx - x0)[None, :]
        a = g[y0][:, x0]
        b = g[y0][:, x0 + 1]
        c = g[y0 + 1][:, x0]
        d = g[y0 + 1][:, x0 + 1]
        out += amp * ((a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy)
        tot += amp
        amp *= 0.5
        cell = max(cell // 2, 1)
    return out / tot


def _decimate_phases(tex4: np.ndarray) -> dict:
    """4x4 box decimation of a 4x texture at each of the 16 sub-sample phases."""
    H4, W4 = tex4.shape
    c = np.zeros((H4 + 1, W4 + 1), np.float64)
    c[1:, 1:] = np.cumsum(np.cumsum(tex4, 0), 1)
    out = {}
    for py in range(4):
        for px in range(4):
            hh, ww = (H4 - py) // 4, (W4 - px) // 4
            ys = py + 4 * np.arange(hh + 1)
            xs = px + 4 * np.arange(ww + 1)
            blk = c[ys[1:]][:, xs[1:]] - c[ys[:-1]][:, xs[1:]] - c[ys[1:]][:, xs[:-1]] + c[ys[:-1]][:, xs[:-1]]
            out[(py, px)] = (blk / 16.0).astype(np.float32)
    return out


def hd_clip(frames: int = 60, seed: int = 1, w: int = 1920, h: int = 1080, with_chroma: bool = False):
    """Luma (and optionally chroma) of the 1080p synthetic workload, uint8.
    Chroma (flat 128 plus sigma 1) comes from its own seeded stream, so the
    luma is the same with or without it."""
    rng = np.random.default_rng(seed)
    crng = np.random.default_rng([seed, 0xC4])
    # background texture at 4x, with margin for the whole clip's motion
    vx4, vy4 = 5, -2  # (1.25, -0.5) px/frame in quarter-pel units
    mx = abs(vx4) * frames // 4 + 8
    my = abs(vy4) * frames // 4 + 8
    Hb, Wb = (h + 2 * my) * 4, (w + 2 * mx) * 4
    tex = 20.0 + 215.0 * _value_noise(rng, Hb // 4, Wb // 4, 4, 64)
    tex4 = np.repeat(np.repeat(tex, 4, 0), 4, 1)
    tex4 += rng.normal(0.0, 6.0, tex4.shape).astype(np.float32)  # sub-pixel detail
    bg = _decimate_phases(tex4)
    rects = []
    for _ in range(8):
        rw, rh = (int(v) for v in rng.integers(32, 257, 2))
        t4 = 255.0 * _value_noise(rng, rh, rw, 4, 16)
        t4 = np.repeat(np.repeat(t4, 4, 0), 4, 1) + rng.normal(0.0, 12.0, (rh * 4, rw * 4)).astype(np.float32)
        ph = _decimate_phases(np.pad(t4, ((0, 4), (0, 4)), mode="edge"))
        x4 = int(rng.integers(0, (w - rw) * 4))
        y4 = int(rng.integers(0, (h - rh) * 4))
        vx = int(np.round(rng.uniform(-6, 6) * 4))
        vy = int(np.round(rng.uniform(-6, 6) * 4))
        rects.append((rw, rh, ph, x4, y4, vx, vy))
    ys = np.empty((frames, h, w), np.uint8)
    us = np.empty((frames, h // 2, w // 2), np.uint8) if with_chroma else None
    vs = np.empty((frames, h // 2, w // 2), np.uint8) if with_chroma else None
    for t in range(frames):
        ox4 = mx * 4 + vx4 * t
        oy4 = my * 4 + vy4 * t
        img = bg[(oy4 % 4, ox4 % 4)][oy4 // 4:oy4 // 4 + h, ox4 // 4:ox4 // 4 + w].copy()
        for rw, rh, ph, x4, y4, vx, vy in rects:
            px4, py4 = x4 + vx * t, y4 + vy * t
            src = ph[(py4 % 4, px4 % 4)][:rh, :rw]
            X, Y = px4 // 4, py4 // 4
            x0, y0, x1, y1 = max(X, 0), max(Y, 0), min(X + rw, w), min(Y + rh, h)
            if x1 > x0 and y1 > y0:
                img[y0:y1, x0:x1] = src[y0 - Y:y1 - Y, x0 - X:x1 - X]
        img += rng.normal(0.0, 1.5, (h, w)).astype(np.float32)
        ys[t] = _to_u8(img)
        if with_chroma:
            us[t] = _to_u8(128 + crng.normal(0.0, 1.0, (h // 2, w // 2)))
            vs[t] = _to_u8(128 + crng.normal(0.0, 1.0, (h // 2, w // 2)))
    return ys, us, vs
