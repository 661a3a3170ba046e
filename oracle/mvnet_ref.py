"""CPU restatement of the learned motion-vector proposal network (float64 numpy).

TEST INFRASTRUCTURE ONLY: tests/ use it to check the GPU kernels' forward
pass, loss and gradients.  Nothing in the product imports it.

The network has no counterpart in the reference encoder (rusty_h264 searches
every MB with motion_search, crates/rusty_h264-encoder/src/mb16.rs:2433); it
proposes candidate MVs for that search.  Its definition, which the CUDA kernels
(rusty_h264_b200/csrc/mvnet.cu) implement:

* input, per frame pair (current frame f, reference frame f-1, both cw x ch
  luma with cw, ch multiples of 16): a 2-channel image, channel 0 the
  reference and channel 1 the current frame, as (u8 - 128) / 64 (exact in
  bf16);
* trunk, over the whole image: conv1 2->16, conv2 16->32, conv3 32->32, each
  3x3, stride 2, zero padding 1 at the frame edges, bias, ReLU: a map of
  (ch/8) x (cw/8) cells of 32 features, one cell per 8x8 pixels;
* per MB (mbx, mby): the 6x6 cells whose pixels are the MB's co-located 48x48
  region (cells 2*mby-2 .. 2*mby+3, 2*mbx-2 .. 2*mbx+3; zero outside the map),
  1152 features in (cell y, cell x, channel) order, then the quarter-pel MVs
  of 3 neighbour MBs (left, top, top-right; each component clamped to +-128,
  divided by 64), zero-padded to 1168;
* FC1 1168 -> 256, bias, ReLU; head 256 -> 296 logits, of which the first 289
  are classes: class c = (dy + 8) * 17 + (dx + 8) is the full-pel MV
  (4*dx, 4*dy) quarter-pel, |dx|, |dy| <= 8 (the +-32 quarter-pel grid);
* loss: mean softmax cross-entropy over the 289 classes and every MB of the
  batch's frame pairs.

Numerics: weights and activations are bf16 (round to nearest even) at every
layer boundary and every product is accumulated in float32 on the GPU (float64
here).  Backward: dL = (softmax - onehot) / B in bf16; dH, the per-MB feature
gradient dF, the conv3 map gradient (the sum of the dF entries of the up to 9
MBs whose crops hold the cell), dA2 and dA1 are each rounded to bf16 after
their ReLU mask; weight and bias gradients are float32 sums.  This file
applies the same roundings, so what remains between the two is accumulation
order.
"""
from __future__ import annotations

import numpy as np

NCLS = 289      # 17 x 17 full-pel offsets
HEAD_N = 296    # head rows (the last 7 are padding, never a class)
FEAT = 1168     # 1152 trunk features + 6 MV features + 10 zeros
MV_CLAMP = 128

# parameter tensors in the order of the flat float32 vector of the C ABI
SHAPES = (
    ("w1", (16, 3, 3, 2)), ("b1", (16,)),
    ("w2", (32, 3, 3, 16)), ("b2", (32,)),
    ("w3", (32, 3, 3, 32)), ("b3", (32,)),
    ("w4", (256, FEAT)), ("b4", (256,)),
    ("w5", (HEAD_N, 256)), ("b5", (HEAD_N,)),
)
NPARAMS = int(sum(np.prod(s) for _, s in SHAPES))


def bf16(x) -> np.ndarray:
    """Round to the nearest bf16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float64).astype(np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unflatten(flat: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shp in SHAPES:
        k = int(np.prod(shp))
        out[name] = np.asarray(flat[o:o + k], np.float64).reshape(shp)
        o += k
    return out


def flatten(p: dict, dtype=np.float32) -> np.ndarray:
    return np.concatenate([np.asarray(p[n], np.float64).ravel() for n, _ in SHAPES]).astype(dtype)


def class_of_mv(mvx: int, mvy: int) -> int:
    """Label class of a quarter-pel MV: its nearest full-pel offset (halves
    away from zero), clamped to the +-8 pixel grid."""
    def q(v):
        a = (abs(int(v)) + 2) >> 2
        return max(-8, min(8, a if v >= 0 else -a))
    return (q(mvy) + 8) * 17 + (q(mvx) + 8)


def mv_of_class(c: int):
    return (4 * (c % 17 - 8), 4 * (c // 17 - 8))


def image(cur: np.ndarray, ref: np.ndarray) -> np.ndarray:
    """(ch, cw, 2) network input of a frame pair."""
    return np.stack([(ref.astype(np.float64) - 128.0) / 64.0, (cur.astype(np.float64) - 128.0) / 64.0], axis=-1)


def mv_features(nmv: np.ndarray) -> np.ndarray:
    return np.clip(np.asarray(nmv, np.float64), -MV_CLAMP, MV_CLAMP) / 64.0


def _patches(x: np.ndarray) -> np.ndarray:
    """im2col of a 3x3 stride-2 pad-1 conv: (B, H, W, C) -> (B, H/2, W/2, 9*C),
    tap-major (ky, kx) then channel."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C))
    xp[:, 1:H + 1, 1:W + 1] = x
    oh, ow = H // 2, W // 2
    cols = []
    for ky in range(3):
        for kx in range(3):
            cols.append(xp[:, ky:ky + 2 * oh:2, kx:kx + 2 * ow:2, :])
    return np.concatenate(cols, axis=-1)


def _conv(x, w, b):
    co = w.shape[0]
    return _patches(x) @ w.reshape(co, -1).T + b


def _conv_back_data(dy: np.ndarray, w: np.ndarray, in_shape) -> np.ndarray:
    """Gradient of a 3x3 stride-2 pad-1 conv with respect to its input."""
    B, H, W, C = in_shape
    co = w.shape[0]
    dp = dy @ w.reshape(co, -1)  # (B, oh, ow, 9*C)
    oh, ow = H // 2, W // 2
    dxp = np.zeros((B, H + 2, W + 2, C))
    t = 0
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + 2 * oh:2, kx:kx + 2 * ow:2, :] += dp[..., t * C:(t + 1) * C]
            t += 1
    return dxp[:, 1:H + 1, 1:W + 1]


def _crops(a3: np.ndarray) -> np.ndarray:
    """(B, H3, W3, 32) map -> (B * mb_h * mb_w, 1152) per-MB crops."""
    B, H3, W3, C = a3.shape
    mb_h, mb_w = H3 // 2, W3 // 2
    ap = np.zeros((B, H3 + 4, W3 + 4, C))
    ap[:, 2:H3 + 2, 2:W3 + 2] = a3
    out = np.zeros((B, mb_h, mb_w, 6, 6, C))
    for cy in range(6):
        for cx in range(6):
            out[:, :, :, cy, cx] = ap[:, cy:cy + 2 * mb_h:2, cx:cx + 2 * mb_w:2]
    return out.reshape(B * mb_h * mb_w, 6 * 6 * C)


def _uncrop(df: np.ndarray, shape) -> np.ndarray:
    """Adjoint of _crops: per-MB crop gradients summed back onto the map."""
    B, H3, W3, C = shape
    mb_h, mb_w = H3 // 2, W3 // 2
    d = df.reshape(B, mb_h, mb_w, 6, 6, C)
    ap = np.zeros((B, H3 + 4, W3 + 4, C))
    for cy in range(6):
        for cx in range(6):
            ap[:, cy:cy + 2 * mb_h:2, cx:cx + 2 * mb_w:2] += d[:, :, :, cy, cx]
    return ap[:, 2:H3 + 2, 2:W3 + 2]


def forward(params: dict, x0: np.ndarray, nmv: np.ndarray, round_bf16: bool = True) -> dict:
    """Activations and logits for images x0 (P, ch, cw, 2) and nmv (P*nmb, 6),
    MBs pair-major, raster order within a pair."""
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, np.float64))
    p = {k: r(v) for k, v in params.items()} if round_bf16 else params
    a1 = r(np.maximum(_conv(x0, p["w1"], p["b1"]), 0.0))
    a2 = r(np.maximum(_conv(a1, p["w2"], p["b2"]), 0.0))
    a3 = r(np.maximum(_conv(a2, p["w3"], p["b3"]), 0.0))
    crops = _crops(a3)
    f = np.zeros((crops.shape[0], FEAT))
    f[:, :1152] = crops
    f[:, 1152:1158] = mv_features(nmv)
    h = r(np.maximum(f @ p["w4"].T + p["b4"], 0.0))
    logits = h @ p["w5"].T + p["b5"]
    return dict(p=p, x0=x0, a1=a1, a2=a2, a3=a3, f=f, h=h, logits=logits)


def loss_and_dlogits(logits: np.ndarray, labels: np.ndarray):
    z = logits[:, :NCLS]
    z = z - z.max(axis=1, keepdims=True)
    e = np.exp(z)
    prob = e / e.sum(axis=1, keepdims=True)
    B = logits.shape[0]
    loss = float(-np.log(prob[np.arange(B), labels]).mean())
    d = np.zeros_like(logits)
    d[:, :NCLS] = prob
    d[np.arange(B), labels] -= 1.0
    return loss, d / B


def backward(act: dict, dlogits: np.ndarray, round_bf16: bool = True) -> dict:
    r = bf16 if round_bf16 else (lambda v: np.asarray(v, np.float64))
    p = act["p"]
    g = {}
    dl = r(dlogits)
    g["w5"] = dl.T @ act["h"]
    g["b5"] = dl.sum(0)
    dh = r((dl @ p["w5"]) * (act["h"] > 0))
    g["w4"] = dh.T @ act["f"]
    g["b4"] = dh.sum(0)
    df = r((dh @ p["w4"])[:, :1152])
    da3 = r(_uncrop(df, act["a3"].shape) * (act["a3"] > 0))
    g["w3"] = np.einsum("bhwo,bhwk->ok", da3, _patches(act["a2"])).reshape(p["w3"].shape)
    g["b3"] = da3.sum((0, 1, 2))
    da2 = r(_conv_back_data(da3, p["w3"], act["a2"].shape) * (act["a2"] > 0))
    g["w2"] = np.einsum("bhwo,bhwk->ok", da2, _patches(act["a1"])).reshape(p["w2"].shape)
    g["b2"] = da2.sum((0, 1, 2))
    da1 = r(_conv_back_data(da2, p["w2"], act["a1"].shape) * (act["a1"] > 0))
    g["w1"] = np.einsum("bhwo,bhwk->ok", da1, _patches(act["x0"])).reshape(p["w1"].shape)
    g["b1"] = da1.sum((0, 1, 2))
    return g


def loss_and_grads(flat_params: np.ndarray, x0, nmv, labels, round_bf16: bool = True):
    act = forward(unflatten(flat_params), x0, nmv, round_bf16)
    loss, dl = loss_and_dlogits(act["logits"], labels)
    g = backward(act, dl, round_bf16)
    return loss, flatten(g, np.float64), act["logits"]
