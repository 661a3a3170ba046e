"""Host side of the learned motion-vector proposals.

* :class:`MvNet` binds the ``h264a_mvnet_*`` entry points of
  libh264accel_cuda.so (include/h264accel.h): the network's parameters,
  optimiser state and batch workspace live on the GPU, and its forward,
  backward and Adam steps are the library's own tensor-core kernels.
* :func:`harvest` turns clips into training samples: the inputs are the MB's
  co-located regions of frames f and f-1 and the HalfRes lookahead MVs of its
  left, top and top-right neighbours; the label is the plain search's 16x16
  MV (h264a_me_frames, Balanced preset) at a given QP.
* :func:`train` runs the training loop over a sample set resident on the GPU.

The network has no counterpart in the reference encoder, which runs
motion_search (crates/rusty_h264-encoder/src/mb16.rs:2433) on every MB.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import accel as A

NPARAMS = 389528
MAX_PIXELS = 8388608
NCLS = 289
HEAD_N = 296


class MvnetFrame(C.Structure):
    _fields_ = [("d_cur", C.c_void_p), ("d_ref", C.c_void_p), ("cw", C.c_int32), ("ch", C.c_int32),
                ("d_guide_mvs", C.c_void_p), ("d_props", C.c_void_p)]


def class_of_mv(mv: np.ndarray) -> np.ndarray:
    """Label class of quarter-pel MVs (..., 2): the nearest full-pel offset
    (halves away from zero), clamped to +-8 pixels; (dy+8)*17 + dx+8."""
    mv = np.asarray(mv, np.int64)
    q = np.sign(mv) * ((np.abs(mv) + 2) >> 2)
    q = np.clip(q, -8, 8)
    return ((q[..., 1] + 8) * 17 + (q[..., 0] + 8)).astype(np.int16)


def neighbour_mvs(mvs: np.ndarray, mb_w: int, mb_h: int) -> np.ndarray:
    """(nmb, 6) MVs of each MB's left, top and top-right neighbours (zero
    where the neighbour is outside the frame), the rule h264a_mvnet_propose
    applies to its guide MVs."""
    g = np.asarray(mvs, np.int64).reshape(mb_h, mb_w, 2)
    out = np.zeros((mb_h, mb_w, 6), np.int64)
    out[:, 1:, 0:2] = g[:, :-1]
    out[1:, :, 2:4] = g[:-1, :]
    out[1:, :-1, 4:6] = g[:-1, 1:]
    return np.clip(out, -32768, 32767).reshape(-1, 6).astype(np.int16)


class MvNet:
    """One network on one device (parameters, Adam state, a batch workspace)."""

    def __init__(self, acc: "A.Accel", seed: int = 1):
        self.acc = acc
        self.L = acc.L
        h = C.c_void_p()
        acc._check(self.L.h264a_mvnet_create(acc.device, seed, C.byref(h)))
        self.h = h
        self.loss_buf = acc.zeros((1,), acc.torch.float32)

    def close(self):
        if getattr(self, "h", None):
            self.L.h264a_mvnet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(NPARAMS, np.float32)
        self.acc._check(self.L.h264a_mvnet_get_params(self.h, p.ctypes.data_as(C.c_void_p)))
        return p

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == NPARAMS
        self.acc._check(self.L.h264a_mvnet_set_params(self.h, p.ctypes.data_as(C.c_void_p)))

    def forward(self, pairs_ptr: int, npairs: int, cw: int, ch: int, nmv_ptr: int):
        nmb = (cw // 16) * (ch // 16)
        out = self.acc.empty((npairs * nmb, HEAD_N), self.acc.torch.float32)
        self.acc._check(self.L.h264a_mvnet_forward(self.h, pairs_ptr, npairs, cw, ch, nmv_ptr, A._dptr(out),
                                                   self.acc._stream()))
        return out

    def grads(self, pairs_ptr: int, npairs: int, cw: int, ch: int, nmv_ptr: int, labels_ptr: int):
        g = self.acc.empty((NPARAMS,), self.acc.torch.float32)
        loss = self.acc.empty((1,), self.acc.torch.float32)
        self.acc._check(self.L.h264a_mvnet_grads(self.h, pairs_ptr, npairs, cw, ch, nmv_ptr, labels_ptr, A._dptr(g),
                                                 A._dptr(loss), self.acc._stream()))
        return g, loss

    def train_step(self, pairs_ptr: int, npairs: int, cw: int, ch: int, nmv_ptr: int, labels_ptr: int, lr: float):
        self.acc._check(self.L.h264a_mvnet_train_step(self.h, pairs_ptr, npairs, cw, ch, nmv_ptr, labels_ptr,
                                                      float(lr), A._dptr(self.loss_buf), self.acc._stream()))

    def propose(self, frames):
        """frames: MvnetFrame structs (device pointers); fills their d_props."""
        arr = (MvnetFrame * len(frames))(*frames)
        self.acc._check(self.L.h264a_mvnet_propose(self.h, C.cast(arr, C.c_void_p), len(frames),
                                                   self.acc._stream()))


class TrainSet:
    """Training items of one frame geometry, resident on the device: item i
    is a frame pair (pointers in pairs[i] = (current, reference)) with the
    neighbour features nmv[i] (nmb x 6 i16) and labels labels[i] (nmb i16)
    of one QP."""

    def __init__(self, acc, cw, ch):
        self.acc, self.cw, self.ch = acc, cw, ch
        self.pairs, self.nmv, self.labels, self.keep, self.qps = [], [], [], [], []

    def finish(self):
        t = self.acc.torch
        dev = f"cuda:{self.acc.device}"
        self.d_pairs = t.tensor(np.array(self.pairs, np.int64), device=dev)
        self.d_nmv = t.from_numpy(np.stack(self.nmv)).to(dev)
        self.d_labels = t.from_numpy(np.stack(self.labels)).to(dev)
        return self

    def __len__(self):
        return len(self.pairs)


def harvest(acc, clips, qps, lam_scale: float = 1.25, ts: "TrainSet" = None) -> TrainSet:
    """Training items of clips (n, ch, cw) u8 of one geometry: every frame
    pair (f, f-1), f >= 1, at every QP in `qps`, labelled with the plain
    search's 16x16 MVs (no partitions) against frame f-1, with the HalfRes
    lookahead MVs of each MB's neighbours as features.  Call ts.finish()
    after the last clip."""
    torch = acc.torch
    for clip in clips:
        n, ch, cw = clip.shape
        if ts is None:
            ts = TrainSet(acc, cw, ch)
        assert (cw, ch) == (ts.cw, ts.ch)
        mb_w, mb_h = cw // 16, ch // 16
        nmb = mb_w * mb_h
        d = acc.to_dev(clip)
        planes = acc.hpel_build(d[: n - 1], 32)
        half = acc.downsample2x(d)
        _, _, la_mvs = acc.lookahead_costs(d, half, 2)
        la = la_mvs.cpu().numpy()
        params = A.default_me_params()
        ts.keep.append(d)
        for qp in qps:
            lam = float(np.sqrt(A.frame_lambda(qp)) * lam_scale)
            picks = torch.zeros((n, nmb, 6), dtype=torch.int32, device=d.device)
            costs = torch.zeros((n, nmb, 2), dtype=torch.int64, device=d.device)
            fr = [A.MeFrame(A.Picture(d[f].data_ptr(), planes[f - 1].data_ptr(), cw, ch, 32), lam, -1,
                            picks[f].data_ptr(), costs[f].data_ptr()) for f in range(1, n)]
            acc.me_frames(fr, params)
            acc.sync()
            pk = picks.cpu().numpy()
            for f in range(1, n):
                ts.pairs.append((d[f].data_ptr(), d[f - 1].data_ptr()))
                ts.nmv.append(neighbour_mvs(la[f], mb_w, mb_h))
                ts.labels.append(class_of_mv(pk[f, :, 1:3]))
                ts.qps.append(qp)
        del planes, half
    return ts


def train(net: MvNet, ts: TrainSet, epochs: float = 2.0, lr: float = 2e-3, pairs_per_step: int = 4, seed: int = 0,
          log_every: int = 0):
    """Adam over shuffled batches of `pairs_per_step` items, the learning
    rate decayed along a cosine to 5% of `lr`.  Returns (loss log, seconds,
    steps)."""
    acc = net.acc
    torch = acc.torch
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    n = len(ts)
    P = max(1, min(pairs_per_step, n, MAX_PIXELS // (ts.cw * ts.ch)))
    per_epoch = max(1, n // P)
    steps = max(1, int(round(epochs * per_epoch)))
    losses = []
    acc.sync()
    t0 = time.perf_counter()
    for k in range(steps):
        if k % per_epoch == 0:
            perm = torch.randperm(n, generator=g).to(ts.d_pairs.device)
            pp = ts.d_pairs.index_select(0, perm).contiguous()
            nm = ts.d_nmv.index_select(0, perm).contiguous()
            lb = ts.d_labels.index_select(0, perm).contiguous()
        o = (k % per_epoch) * P
        frac = k / max(1, steps - 1)
        cur_lr = lr * (0.05 + 0.95 * 0.5 * (1.0 + np.cos(np.pi * frac)))
        net.train_step(pp[o].data_ptr(), P, ts.cw, ts.ch, nm[o].data_ptr(), lb[o].data_ptr(), cur_lr)
        if log_every and (k % log_every == 0 or k == steps - 1):
            losses.append((k, float(net.loss_buf.item())))
    acc.sync()
    return losses, time.perf_counter() - t0, steps


def evaluate_topk(net: MvNet, ts: TrainSet, ks=(1, 8)):
    """Fraction of MBs whose label is among the network's top-k classes."""
    hits = {k: 0 for k in ks}
    total = 0
    P = max(1, MAX_PIXELS // (ts.cw * ts.ch))
    for o in range(0, len(ts), P):
        cnt = min(P, len(ts) - o)
        lg = net.forward(ts.d_pairs[o].data_ptr(), cnt, ts.cw, ts.ch, ts.d_nmv[o].data_ptr()).cpu().numpy()[:, :NCLS]
        lab = ts.d_labels[o:o + cnt].cpu().numpy().reshape(-1)
        order = np.argsort(-lg, axis=1, kind="stable")
        for k in ks:
            hits[k] += int((order[:, :k] == lab[:, None]).any(axis=1).sum())
        total += len(lab)
    return {k: hits[k] / max(1, total) for k in ks}
