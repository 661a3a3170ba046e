"""Benchmark of the encoder pixel hot path on B200.

Workload (one step): the 1080p synthetic clip (1920x1080 coded as 1920x1088,
60 frames, the seeded generator in rusty_h264_b200/synth.py) through the whole
path: half-pel planes of the 59 reference pictures, plain-ME of the 59 P
frames (best_part 16x16 + 16x8/8x16 per MB, Balanced preset, QP 27, lme =
sqrt(lambda)*1.25), MC + luma T/Q of every chosen MB, and the HalfRes mb-tree
lookahead (downsample + frame costs) of all 60 frames.

* value: Mpx/s of displayed luma (60 x 1920 x 1080 per step) with the clip
  resident in HBM, CUDA-event timed on the launching stream.  The clip, planes
  and coefficients (~1 GB) exceed the 126 MB L2, so no flush is needed.
* e2e: the same work through h264a_pixel_path_host from pinned host memory,
  host->device copy of the frames and device->host copy of every result
  inside the timed region, over K steps streamed the way an encoder feeds
  consecutive batches: each step's upload is queued (h264a_pixel_path_prefetch)
  before the previous step's call, so it overlaps that call's compute
  (wall-clock timed from the first upload to the last result).  The line also
  gives one synchronous call on its own (upload inside the call).
* roofline: the dominant kernel (the persistent ME kernel) against the INT32
  issue rate measured on this device by h264a_measure_int32_peak; the
  algorithmic work is 112 integer ops per 4x4 Hadamard-SATD evaluation the
  reference performs (the kernel reports the count per MB).
* cpu_baseline: the C restatement of the reference path (oracle/) on one host
  core over an 8-frame sample of the same clip.

--impl reference times that CPU restatement with all host threads over the
whole 60-frame clip instead.
With --gpus N (torchrun) every rank runs an independent replica on its own
clip (distinct seed): replicas only, no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "1080p encode Mpx/s: plain GPU ME vs learned-proposal ME at ≤0.5% BD-rate"
W, H, FRAMES, QP = 1920, 1080, 60, 27
SATD_OPS_PER_4X4 = 112


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=FRAMES)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mixed", action="store_true",
                    help="also time plain-ME over the 16-stream mixed-resolution batch (not part of value)")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-proposal arm")
    ap.add_argument("--learned-epochs", type=float, default=6.0)
    ap.add_argument("--no-closed", action="store_true", help="skip the closed-loop and BD-rate records")
    ap.add_argument("--bd-frames", type=int, default=16)
    ap.add_argument("--gop-step", type=int, default=29,
                    help="P frames of every stream per batched step (--mixed; 29: the clip's whole GOP)")
    ap.add_argument("--bd-4k", action="store_true",
                    help="also the BD-rate record on a 3840x2160 clip of the same generator (seed 2)")
    return ap.parse_args()


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        # NCCL for the GPU ranks; the reference arm's ranks need no GPU (gloo)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def clip(seed: int, frames: int):
    from rusty_h264_b200 import synth

    cache = os.path.join("/tmp", f"h264a_hd_clip_s{seed}_f{frames}.npy")
    if os.path.exists(cache):
        return np.load(cache)
    y, _, _ = synth.hd_clip(frames, seed)
    f = synth.coded_luma(y)
    try:
        np.save(cache, f)
    except OSError:
        pass
    return f


# The mixed-resolution batch: (width, height, streams), 16 streams of 30 frames.
MIXED = ((352, 288, 4), (1280, 720, 6), (1920, 1080, 4), (3840, 2160, 2))
MIXED_FRAMES = 30


def mixed_stream(args):
    """Coded luma of one stream of the mixed batch (the 1080p generator at w x h)."""
    seed, w, h = args
    from rusty_h264_b200 import synth

    cache = os.path.join("/tmp", f"h264a_mixed_s{seed}_{w}x{h}_f{MIXED_FRAMES}.npy")
    if os.path.exists(cache):
        return np.load(cache)
    y, _, _ = synth.hd_clip(MIXED_FRAMES, seed, w, h)
    f = synth.coded_luma(y)
    try:
        np.save(cache, f)
    except OSError:
        pass
    return f


def mixed_inputs():
    """The 16 streams, generated in a spawn-started process pool."""
    import concurrent.futures as cf
    import multiprocessing as mp

    jobs = []
    for w, h, k in MIXED:
        jobs += [(1000 + len(jobs), w, h) for _ in range(k)]
    with cf.ProcessPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(mixed_stream, jobs))


def mixed_batch(acc, torch, streams, params, lam: float, gate: int, gop_step: int = 29):
    """Plain-ME (one reference) of every P frame of the mixed batch in one
    h264a_me_frames call: one persistent wavefront launch over all 464 frames,
    largest first (the frame table in device memory).  Every stream's
    picks and costs must equal the same stream run on its own; then the
    batched call is timed with CUDA events (3 warm-up, 5 timed)."""
    from rusty_h264_b200 import accel as A

    bufs, frames_all, per_stream = [], [], []
    for f in streams:
        n, ch, cw = f.shape
        nmb = (cw // 16) * (ch // 16)
        d = torch.from_numpy(f).cuda()
        planes = acc.hpel_build(d[: n - 1], 32)
        picks = torch.zeros((n, nmb, 6), dtype=torch.int32, device="cuda")
        costs = torch.zeros((n, nmb, 2), dtype=torch.int64, device="cuda")
        fr = [A.MeFrame(A.Picture(d[i].data_ptr(), planes[i - 1].data_ptr(), cw, ch, 32), lam, gate,
                        picks[i].data_ptr(), costs[i].data_ptr()) for i in range(1, n)]
        bufs.append((d, planes, picks, costs))
        frames_all += fr
        per_stream.append(fr)
    acc.sync()
    alone = []
    for s, fr in enumerate(per_stream):
        acc.me_frames(fr, params)
        acc.sync()
        alone.append((bufs[s][2].clone(), bufs[s][3].clone()))
    for b in bufs:
        b[2].zero_()
        b[3].zero_()
    acc.me_frames(frames_all, params)
    acc.sync()
    for s, b in enumerate(bufs):
        assert torch.equal(b[2], alone[s][0]) and torch.equal(b[3], alone[s][1]), f"stream {s}: batched != alone"
    ts = []
    for it in range(8):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        acc.me_frames(frames_all, params)
        e1.record()
        torch.cuda.synchronize()
        if it >= 3:
            ts.append(e0.elapsed_time(e1))
    acc.sync()
    ms = float(np.median(ts))
    px = sum((f.shape[0] - 1) * f.shape[1] * f.shape[2] for f in streams)
    mbs = sum((f.shape[0] - 1) * (f.shape[1] // 16) * (f.shape[2] // 16) for f in streams)
    three = mixed_batch_3ref(acc, torch, bufs, params, lam, gate, gop_step)
    return bufs, {"streams": "4 x 352x288, 6 x 1280x720, 4 x 1920x1080, 2 x 3840x2160; 30 frames each, 1080p generator",
            "p_frames": len(frames_all), "macroblocks": int(mbs), "me_ms": round(ms, 3),
            "me_mpx_s": round(px / (ms * 1e-3) / 1e6, 1), "launches": 1,
            **three,
            "batched_equals_alone": True,
            "note": "plain-ME of all P frames (one reference, and up to three: the previous three pictures); "
                    "not part of value"}


def mixed_batch_3ref(acc, torch, bufs, params, lam: float, gate: int, gop_step: int = 29) -> dict:
    """The mixed batch through the batched runtime (h264a_batch_*), search and
    MC + luma T/Q at QP 27: gop_step P frames of every stream per step (29 by default: each stream's whole GOP,
    one step) over up to three references (the previous three source
    pictures, nearest first), each step one graph launch (the planes of the
    step's frames, then one persistent launch over all 16 streams), in the
    launch shape the autotuner picked.  Every stream's picks, costs and levels
    must equal h264a_me_frames_multiref + h264a_mc_tq_frames_multiref of that
    stream alone; the steps of the 29 P
    frames are timed with CUDA events (3 warm-up passes, median of 5).  The
    tuner also runs on each resolution alone, to report the shape it picks
    per resolution."""
    import ctypes as C

    from rusty_h264_b200 import accel as A

    NREF, PAD, QP = 3, 32, 27
    G = gop_step
    NSLOTS = -(-max(32, G + NREF + 1) // G) * G  # a multiple of G with room for a step and its references
    rings, streams, alone = [], [], []
    for d, _, _, _ in bufs:
        n, ch, cw = d.shape
        nmb = (cw // 16) * (ch // 16)
        pb = 4 * (cw + 2 * PAD) * (ch + 2 * PAD)
        src = torch.zeros((NSLOTS, ch, cw), dtype=torch.uint8, device="cuda")
        src[:n].copy_(d)
        planes = torch.zeros((NSLOTS, pb), dtype=torch.uint8, device="cuda")
        picks = torch.zeros((NSLOTS, nmb, 8), dtype=torch.int32, device="cuda")
        costs = torch.zeros((NSLOTS, nmb, 2), dtype=torch.int64, device="cuda")
        levels = torch.zeros((NSLOTS, nmb, 256), dtype=torch.int16, device="cuda")
        rings.append((src, planes, picks, costs, n, levels))
        streams.append(A.BatchStream(cw, ch, PAD, src.data_ptr(), planes.data_ptr(), picks.data_ptr(),
                                     costs.data_ptr(), lam, gate, levels.data_ptr(), QP, 6))
    # the unbatched path: each stream's P frames in one h264a_me_frames_multiref call
    for src, planes, picks, costs, n, levels in rings:
        ch, cw = src.shape[1], src.shape[2]
        acc.hpel_build(src[: n - 1], PAD, out=planes[: n - 1])
        fr = []
        for f in range(1, n):
            nref = min(NREF, f)
            refs = [planes[f - 1 - r].data_ptr() for r in range(nref)] + [0] * (4 - nref)
            fr.append(A.MeMrFrame(src[f].data_ptr(), (C.c_void_p * 4)(*refs), nref, cw, ch, PAD, lam, gate,
                                  picks[f].data_ptr(), costs[f].data_ptr()))
        acc.me_frames_multiref(fr, params)
        tq = [A.McTqMrFrame(m.d_src, m.d_planes, m.nref, cw, ch, PAD, m.d_picks, QP, 6, levels[f].data_ptr())
              for f, m in zip(range(1, n), fr)]
        acc.mc_tq_frames_multiref(tq)
        acc.sync()
        alone.append((picks[1:n].clone(), costs[1:n].clone(), levels[1:n].clone()))
        picks.zero_()
        levels.zero_()
        costs.zero_()
        planes.zero_()
    nmax = max(r[4] for r in rings)
    steps = [(k, min(G, nmax - 1 - k * G)) for k in range((nmax - 2) // G + 1)]
    b = acc.batch_create(streams, A.BatchConfig(G, NSLOTS, NREF, 1, 0), params)
    for k, count in steps:
        b.step(k, count)
    acc.sync()
    for s, (src, planes, picks, costs, n, levels) in enumerate(rings):
        assert torch.equal(levels[1:n], alone[s][2]), f"stream {s}: batched levels != alone"
        assert torch.equal(picks[1:n], alone[s][0]) and torch.equal(costs[1:n], alone[s][1]), \
            f"stream {s}: batched steps != alone"
    ts = []
    for it in range(8):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k, count in steps:
            b.step(k, count)
        e1.record()
        torch.cuda.synchronize()
        if it >= 3:
            ts.append(e0.elapsed_time(e1))
    info = b.info()
    b.close()
    # the tuner on each resolution alone (its own signature, so it times again)
    per_res = {}
    for w, h, _ in MIXED:
        sub = [st for st in streams if (st.cw, st.ch) == (w, -(-h // 16) * 16)]
        bs = acc.batch_create(sub, A.BatchConfig(G, NSLOTS, NREF, 1, 0), params)
        bs.step(0, min(G, nmax - 1))
        acc.sync()
        inf = bs.info()
        bs.close()
        shape = A.batch_variant_shape(inf["variant"])
        per_res[f"{w}x{h}"] = {"variant": inf["variant"], "mbs_per_cta": shape[0], "staged_window": shape[1],
                               "ms": inf["ms"]}
    shape = A.batch_variant_shape(info["variant"])
    ms = float(np.median(ts))
    px = sum((r[4] - 1) * r[0].shape[1] * r[0].shape[2] for r in rings)
    return {"me_3ref_ms": round(ms, 3), "me_3ref_mpx_s": round(px / (ms * 1e-3) / 1e6, 1),
            "gop_step": G, "graph_launches": len(steps), "batched_equals_alone_3ref": True,
            "with_mc_tq": "each step also runs the MC + luma T/Q (QP 27) of its frames, levels checked too",
            "autotune": {"variant": info["variant"], "mbs_per_cta": shape[0], "staged_window": shape[1],
                         "ms_per_variant": info["ms"], "graphs": info["graphs"], "per_resolution": per_res}}


def mixed_learned(acc, torch, bufs, net, params, lam: float, gate: int, plain_ms: float) -> dict:
    """Learned-proposal ME over the mixed batch (one reference, the source
    model of mixed_batch): the HalfRes lookahead of all 16 streams in one
    h264a_lookahead_streams launch (the proposals' guide MVs), the proposals of all 464 P frames in one h264a_mvnet_propose
    call, then one h264a_me_frames_learned launch over all of them.  Timed
    with CUDA events (median of 5 after 2 warm-ups), against the plain-ME
    launch of the same frames; J of the picks against plain-ME's."""
    from rusty_h264_b200 import accel as A
    from rusty_h264_b200 import mvnet

    T = LEARNED_FALLBACK_T
    per, pfr, lfr = [], [], []
    for d, planes, ppicks, pcosts in bufs:
        n, ch, cw = d.shape
        nmb = (cw // 16) * (ch // 16)
        half = torch.empty((n, ch // 2, cw // 2), dtype=torch.uint8, device="cuda")
        la = torch.zeros((3, n, nmb, 2), dtype=torch.int32, device="cuda")
        props = torch.zeros((n, nmb, 16), dtype=torch.int32, device="cuda")
        picks = torch.zeros((n, nmb, 6), dtype=torch.int32, device="cuda")
        costs = torch.zeros((n, nmb, 2), dtype=torch.int64, device="cuda")
        fb = torch.zeros((n, nmb), dtype=torch.int32, device="cuda")
        per.append((d, half, la, props, picks, costs, fb, pcosts))
        pfr += [mvnet.MvnetFrame(d[i].data_ptr(), d[i - 1].data_ptr(), cw, ch, la[2][i].data_ptr(),
                                 props[i].data_ptr()) for i in range(1, n)]
        lfr += [A.MeLearnedFrame(A.MeFrame(A.Picture(d[i].data_ptr(), planes[i - 1].data_ptr(), cw, ch, 32), lam,
                                           gate, picks[i].data_ptr(), costs[i].data_ptr()), props[i].data_ptr(), T,
                                 fb[i].data_ptr()) for i in range(1, n)]

    las = [A.LaStream(d.data_ptr(), half.data_ptr(), d.shape[2], d.shape[1], d.shape[0], la[0].data_ptr(),
                      la[1].data_ptr(), la[2].data_ptr()) for d, half, la, *_ in per]

    def lookahead():  # each stream's half-res frames, then all 16 lookaheads in one launch
        for d, half, la, *_ in per:
            n, ch, cw = d.shape
            acc._check(acc.L.h264a_downsample2x(acc.ctx, d.data_ptr(), cw, ch, n, cw * ch, half.data_ptr(),
                                                acc._stream()))
        acc.lookahead_streams(las, 2)

    def step():
        lookahead()
        net.propose(pfr)
        acc.me_frames_learned(lfr, params)

    step_ms = events_ms(torch, step)
    stage = {"lookahead": events_ms(torch, lookahead), "propose": events_ms(torch, lambda: net.propose(pfr)),
             "learned_me": events_ms(torch, lambda: acc.me_frames_learned(lfr, params))}
    acc.sync()
    px = sum((p[0].shape[0] - 1) * p[0].shape[1] * p[0].shape[2] for p in per)
    jl = sum(float(p[5][1:, :, 0].sum().item()) for p in per)
    jp = sum(float(p[7][1:, :, 0].sum().item()) for p in per)
    fbr = sum(float(p[6][1:].float().sum().item()) for p in per) / sum(p[6][1:].numel() for p in per)
    return {"value": round(px / (step_ms * 1e-3) / 1e6, 1), "unit": "Mpx/s", "ms_per_step": round(step_ms, 3),
            "stage_ms": {k: round(v, 3) for k, v in stage.items()},
            "learned_me_mpx_s": round(px / (stage["learned_me"] * 1e-3) / 1e6, 1),
            "plain_me_ms": round(plain_ms, 3), "fallback_t": T, "fallback_rate": round(fbr, 4),
            "J_pick_vs_plain": round(jl / jp - 1, 5),
            "note": "the mixed batch's 464 P frames, one reference: lookahead + proposals + learned ME per step"}


# Training clips of the learned proposals: the 1080p generator with seeds the
# benchmarked clip (seed 1) does not use, at the four QPs of the BD-rate points.
TRAIN_SEEDS = (100, 101, 102, 103)
TRAIN_FRAMES = 16
BD_QPS = (22, 27, 32, 37)
# The learned search's fallback threshold (SATD of the best proposal above the
# predictor's): at 4096 about 0.6% of the benchmarked clip's MBs fall back.
# A sweep of 256 / 1024 / 4096 / never on the 60-frame closed loop gave
# 174 / 156 / 130 / 129 ms per step against plain's 188 ms, at BD-rates of
# -3.1 / -3.7 / -3.8 / -3.8 % against plain (16 frames, QP 22-37).
LEARNED_FALLBACK_T = 4096


def train_clip(seed):
    from rusty_h264_b200 import synth

    cache = os.path.join("/tmp", f"h264a_train_s{seed}_f{TRAIN_FRAMES}.npy")
    if os.path.exists(cache):
        return np.load(cache)
    f = synth.coded_luma(synth.hd_clip(TRAIN_FRAMES, seed)[0])
    try:
        np.save(cache, f)
    except OSError:
        pass
    return f


def events_ms(torch, fn, reps=5, warm=2):
    """Median CUDA-event time of fn() on the current stream."""
    ts = []
    for r in range(reps + warm):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        if r >= warm:
            ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def learned_arm(acc, torch, f, U, V, d_frames, planes, params, lam, gate, qp, plain_src, epochs, train_clips, steps):
    """The learned-proposal arm.  The network is trained here by the library's
    kernels on clips of other seeds (labels: plain-ME's 16x16 MVs at QP
    22/27/32/37), its held-out accuracy measured on the benchmarked clip, and
    then the headline workload -- the closed loop over the 60-frame clip --
    runs with the learned search: the lookahead first (its MVs feed the
    proposals), then per frame planes, proposals, learned ME, reconstruction
    and deblocking, CUDA-event timed like the plain arm.  A second record runs
    the source-reference model with proposals against plain-ME on the same
    references, where the J of the picks compares directly."""
    from rusty_h264_b200 import accel as A
    from rusty_h264_b200 import mvnet

    n, ch, cw = f.shape
    nmb = (cw // 16) * (ch // 16)
    t0 = time.perf_counter()
    ts = mvnet.harvest(acc, train_clips, BD_QPS).finish()
    harvest_s = time.perf_counter() - t0
    net = mvnet.MvNet(acc, seed=1)
    losses, train_s, tsteps = mvnet.train(net, ts, epochs=epochs, lr=2e-3, pairs_per_step=4, log_every=10)
    n_items = len(ts)
    del ts
    held = mvnet.harvest(acc, [f[:9]], (qp,)).finish()
    topk = mvnet.evaluate_topk(net, held, (1, 8))
    del held
    T = LEARNED_FALLBACK_T
    # ---- the closed loop with the learned search ----
    cb = ClosedBufs(acc, torch, f, U, V, learned=True)
    job = cb.job(A, lam, gate, qp, net=net, fallback_t=T)

    def closed_step():
        cb.lookahead(acc)
        acc.closed_frames(job, params)

    closed_ms = events_ms(torch, closed_step, reps=steps, warm=2)
    acc.sync()
    closed = {"value": round(n * W * H / (closed_ms * 1e-3) / 1e6, 2), "unit": "Mpx/s",
              "ms_per_step": round(closed_ms, 3), "fallback_t": T,
              "fallback_rate": round(float(cb.fb[1:].float().mean().item()), 4),
              "timing": f"median of {steps} CUDA-event timed steps (lookahead, then the learned closed loop)"}
    rec_y = cb.ry.cpu().numpy()
    del cb
    # ---- the source-reference model with proposals, against plain-ME ----
    half = torch.empty((n, ch // 2, cw // 2), dtype=torch.uint8, device=d_frames.device)
    la = torch.empty((3, n, nmb, 2), dtype=torch.int32, device=d_frames.device)
    props = torch.zeros((n, nmb, 16), dtype=torch.int32, device=d_frames.device)
    picks = torch.zeros((n, nmb, 6), dtype=torch.int32, device=d_frames.device)
    costs = torch.zeros((n, nmb, 2), dtype=torch.int64, device=d_frames.device)
    coeffs = torch.zeros((n, nmb, 256), dtype=torch.int16, device=d_frames.device)
    fb = torch.zeros((n, nmb), dtype=torch.int32, device=d_frames.device)
    la_mvs = la[2]
    pfr = [mvnet.MvnetFrame(d_frames[i].data_ptr(), d_frames[i - 1].data_ptr(), cw, ch, la_mvs[i].data_ptr(),
                            props[i].data_ptr()) for i in range(1, n)]
    lfr = [A.MeLearnedFrame(A.MeFrame(A.Picture(d_frames[i].data_ptr(), planes[i - 1].data_ptr(), cw, ch, 32), lam,
                                      gate, picks[i].data_ptr(), costs[i].data_ptr()), props[i].data_ptr(), T,
                            fb[i].data_ptr()) for i in range(1, n)]
    tqf = [A.TqFrame(A.Picture(d_frames[i].data_ptr(), planes[i - 1].data_ptr(), cw, ch, 32), picks[i].data_ptr(),
                     qp, 6, coeffs[i].data_ptr()) for i in range(1, n)]

    def lookahead():
        acc._check(acc.L.h264a_downsample2x(acc.ctx, d_frames.data_ptr(), cw, ch, n, cw * ch, half.data_ptr(),
                                            acc._stream()))
        acc._check(acc.L.h264a_lookahead_costs(acc.ctx, d_frames.data_ptr(), half.data_ptr(), cw, ch, n, 2,
                                               la[0].data_ptr(), la[1].data_ptr(), la_mvs.data_ptr(), acc._stream()))

    def step():
        acc.hpel_build(d_frames[: n - 1], 32, out=planes)
        lookahead()
        net.propose(pfr)
        acc.me_frames_learned(lfr, params)
        acc.mc_tq_frames(tqf)

    step_ms = events_ms(torch, step)
    stage = {"lookahead": events_ms(torch, lookahead), "propose": events_ms(torch, lambda: net.propose(pfr)),
             "learned_me": events_ms(torch, lambda: acc.me_frames_learned(lfr, params))}
    acc.sync()
    c = costs.cpu().numpy()[1:]
    pc = plain_src["costs"][1:]
    src_model = {
        "value": round(n * W * H / (step_ms * 1e-3) / 1e6, 2), "unit": "Mpx/s", "ms_per_step": round(step_ms, 3),
        "stage_ms": {k: round(v, 3) for k, v in stage.items()}, "plain_me_ms": round(plain_src["me_ms"], 3),
        "fallback_rate": round(float(fb.cpu().numpy()[1:].mean()), 4),
        "J_pick_vs_plain": round(float(c[:, :, 0].sum() / pc[:, :, 0].sum() - 1), 5),
        "J16_vs_plain": round(float(c[:, :, 1].sum() / pc[:, :, 1].sum() - 1), 5),
    }
    out = {
        "workload": "the benchmarked closed loop with proposals + the learned 16x16 search (partitions as plain-ME)",
        "closed_loop": closed,
        "training": {"items": n_items, "mbs": int(n_items * nmb), "qps": list(BD_QPS),
                     "clips": f"{len(train_clips)} x {TRAIN_FRAMES} frames, 1080p generator seeds {list(TRAIN_SEEDS)}",
                     "steps": tsteps, "batch_mbs": int(4 * nmb), "seconds": round(train_s, 2),
                     "harvest_seconds": round(harvest_s, 2), "loss_first": round(losses[0][1], 4),
                     "loss_last": round(losses[-1][1], 4)},
        "heldout_topk": {"top1": round(topk[1], 4), "top8": round(topk[8], 4),
                         "note": "the benchmarked clip (not trained on), frames 1-8, plain 16x16 MVs as labels"},
        "source_reference_model": src_model,
    }
    return out, net, rec_y


def bd_rate_record(acc, f, U, V, params, lam_scale, net, bd_frames, width=W, height=H):
    """BD-rate of the learned search against plain-ME through the closed loop
    at QP 22/27/32/37 on the clip's first bd_frames frames: rate = the
    Annex-B bytes of the P frames (h264a_write_stream_cavlc), PSNR = luma of
    the P frames' reconstruction against the source (the tests check that the
    decoder reproduces the reconstruction exactly)."""
    from rusty_h264_b200 import accel as A
    from rusty_h264_b200 import bdrate

    m = bd_frames
    curves = {"plain": [], "learned": []}
    for q in BD_QPS:
        lq = float(np.sqrt(A.frame_lambda(q)) * lam_scale)
        gq = A.split_gate_for_qp(q)
        for name, nt in (("plain", None), ("learned", net)):
            r = acc.pixel_path_closed(f[:m], U[:m], V[:m], params, lq, gq, q, net=nt, fallback_t=LEARNED_FALLBACK_T)
            data, fbytes = A.write_stream_cavlc(f[0], U[0], V[0], r["picks"], r["coeffs"], r["ccoeffs"], q, width,
                                                height)
            curves[name].append((float(fbytes[1:].sum()), bdrate.psnr(f[1:m, :height], r["rec_y"][1:m, :height])))
    return {
        "size": f"{width}x{height}", "qps": list(BD_QPS), "frames": m,
        "plain": [(round(r), round(d, 3)) for r, d in curves["plain"]],
        "learned": [(round(r), round(d, 3)) for r, d in curves["learned"]],
        "bd_rate_pct_learned_vs_plain": round(bdrate.bd_rate(curves["plain"], curves["learned"]), 3),
        "rate": "bytes of the P frames' NAL units (CAVLC, Baseline); PSNR of the P frames' luma (display area)",
    }


class ClosedBufs:
    """Device buffers of the closed loop over a clip with chroma (and, for the
    learned search, proposals, fallback flags and the lookahead's outputs)."""

    def __init__(self, acc, torch, f, U, V, learned=False):
        n, ch, cw = f.shape
        nmb = (cw // 16) * (ch // 16)
        dev = f"cuda:{acc.device}"
        self.n, self.cw, self.ch, self.nmb = n, cw, ch, nmb
        self.y = torch.from_numpy(f).to(dev)
        self.u = torch.from_numpy(np.ascontiguousarray(U)).to(dev)
        self.v = torch.from_numpy(np.ascontiguousarray(V)).to(dev)
        self.ry, self.ru, self.rv = torch.empty_like(self.y), torch.empty_like(self.u), torch.empty_like(self.v)
        from rusty_h264_b200 import accel as A

        self.planes = torch.empty((A.closed_plane_bytes(n, cw, ch),), dtype=torch.uint8, device=dev)
        self.picks = torch.zeros((n, nmb, 6), dtype=torch.int32, device=dev)
        self.costs = torch.zeros((n, nmb, 2), dtype=torch.int64, device=dev)
        self.coeffs = torch.zeros((n, nmb, 256), dtype=torch.int16, device=dev)
        self.ccoeffs = torch.zeros((n, nmb, 128), dtype=torch.int16, device=dev)
        self.half = torch.empty((n, ch // 2, cw // 2), dtype=torch.uint8, device=dev)
        self.la = torch.empty((4, n, nmb), dtype=torch.int32, device=dev)  # intra, inter, mv x / y pairs
        self.props = torch.zeros((n, nmb, 16), dtype=torch.int32, device=dev) if learned else None
        self.fb = torch.zeros((n, nmb), dtype=torch.int32, device=dev) if learned else None

    def job(self, A, lam, gate, qp, net=None, fallback_t=256):
        p = lambda t: None if t is None else t.data_ptr()
        return A.ClosedDev(p(self.y), p(self.u), p(self.v), p(self.ry), p(self.ru), p(self.rv), p(self.planes), self.n,
                           self.cw, self.ch, lam, gate, qp, 6, None if net is None else net.h.value, fallback_t,
                           p(self.la[2]) if net is not None else None, p(self.picks), p(self.costs), p(self.coeffs),
                           p(self.ccoeffs), p(self.props) if net is not None else None,
                           p(self.fb) if net is not None else None)

    def lookahead(self, acc):
        """downsample2x + the HalfRes lookahead of every frame (the mb-tree
        input, and the guide MVs of the proposals)."""
        n, cw, ch = self.n, self.cw, self.ch
        acc._check(acc.L.h264a_downsample2x(acc.ctx, self.y.data_ptr(), cw, ch, n, cw * ch, self.half.data_ptr(),
                                            acc._stream()))
        acc._check(acc.L.h264a_lookahead_costs(acc.ctx, self.y.data_ptr(), self.half.data_ptr(), cw, ch, n, 2,
                                               self.la[0].data_ptr(), self.la[1].data_ptr(), self.la[2].data_ptr(),
                                               acc._stream()))


def closed_stage_ms(acc, torch, A, cb, params, lam, gate, qp, reps=2):
    """The closed loop frame by frame, with events between the launches (the
    planes of rec(f-1), then h264a_closed_step_frame: the search with each
    MB's reconstruction and deblocking fused in, one frame per launch), for
    comparison with the pipelined launch, which overlaps consecutive frames."""
    n, cw, ch = cb.n, cb.cw, cb.ch
    fs = cw * ch
    acc._check(acc.L.h264a_closed_frames(acc.ctx, C_byref(cb.job(A, lam, gate, qp)), C_byref(params), acc._stream()))
    tot = {"hpel": 0.0, "me_rec_deblock": 0.0}
    for _ in range(reps):
        for f in range(1, n):
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            ev[0].record()
            acc._check(acc.L.h264a_hpel_build(acc.ctx, cb.ry[f - 1].data_ptr(), cw, ch, 32, 1, fs, cb.planes.data_ptr(),
                                              acc._stream()))
            ev[1].record()
            pic = A.Picture(cb.y[f].data_ptr(), cb.planes.data_ptr(), cw, ch, 32)
            me = A.MeFrame(pic, lam, gate, cb.picks[f].data_ptr(), cb.costs[f].data_ptr())
            acc.closed_step(A.ClosedStep(me, cb.u[f].data_ptr(), cb.v[f].data_ptr(), cb.ru[f - 1].data_ptr(),
                                         cb.rv[f - 1].data_ptr(), cb.ry[f].data_ptr(), cb.ru[f].data_ptr(),
                                         cb.rv[f].data_ptr(), cb.coeffs[f].data_ptr(), cb.ccoeffs[f].data_ptr(), qp,
                                         6, None, None, 0), params)
            ev[2].record()
            torch.cuda.synchronize()
            for k, (a, b) in zip(tot, zip(ev[:-1], ev[1:])):
                tot[k] += a.elapsed_time(b) / reps
    acc.sync()
    return tot


def C_byref(x):
    import ctypes

    return ctypes.byref(x)


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 5 ms from a thread (reads only), or nvidia-smi
    at 100 ms where NVML cannot be loaded.  The device is found by its PCI bus
    id, so a remapped CUDA_VISIBLE_DEVICES still samples the right GPU."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.nv = None
        self.samples = []
        self.busid = None
        try:
            import torch

            pr = torch.cuda.get_device_properties(device)
            self.busid = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
        except Exception:
            pass

    def _nvml_sample(self):
        nv, h = self.nv
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        return (nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM),
                int(get_reasons(h)))

    def _poll(self):
        while not self.done.is_set():
            try:
                self.samples.append(self._nvml_sample())
            except Exception:
                pass
            self.done.wait(0.005)

    def start(self):
        try:
            import pynvml as nv

            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByPciBusId(self.busid) if self.busid else nv.nvmlDeviceGetHandleByIndex(self.device)
            self.nv = (nv, h)
            self._nvml_sample()
            self.done = threading.Event()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nv = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.busid or str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.nv is not None:
            self.done.set()
            self.t.join(timeout=5)
            if not self.samples:
                try:
                    self.samples.append(self._nvml_sample())
                except Exception:
                    pass
            sm = [x[0] for x in self.samples]
            reasons = {nm for nm, bit in self.REASONS.items() if any(x[2] & bit for x in self.samples)}
            return {"sm_mhz": float(np.median(sm)) if sm else None,
                    "sm_max_mhz": max(x[1] for x in self.samples) if self.samples else None,
                    "reasons": sorted(reasons), "samples": len(sm), "source": "nvml, 5 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 100 ms"}


def workload_config(frames: int, ws: int) -> dict:
    """The `config` both arms print: the same workload, so their lines compare."""
    return {"workload": "1080p 60-frame clip with chroma, closed-loop pixel path: per P frame the planes of the "
                        "deblocked reconstruction of the previous frame, plain-ME, MC + T/Q + reconstruction of luma "
                        "and chroma, deblocking; HalfRes lookahead of every frame; frame 0 lossless",
            "frames_per_step": frames, "qp": QP, "preset": "balanced", "split_partitions": True,
            "l2": "inputs and outputs (~1 GB) exceed L2; no flush", "parallelism": f"replicas x{ws}"}


def cpu_closed(y, u, v, lam: float, gate: int, nthreads: int):
    """The CPU restatement of the headline workload: the closed loop (serial
    over frames and, as in the reference, over MBs in raster order) plus the
    HalfRes lookahead (frames split over nthreads).  Returns (Mpx/s, s)."""
    from oracle import oracle as O

    t0 = time.perf_counter()
    O.closed_loop_clip(y, u, v, O.balanced_params(), lam, gate, QP)
    O.lookahead_clip(y, mode=2, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return y.shape[0] * W * H / dt / 1e6, dt


def cpu_baseline(frames: np.ndarray, nthreads: int, lam: float, gate: int):
    """The CPU restatement of the reference path on a bounded sample."""
    from oracle import oracle as O

    t0 = time.perf_counter()
    O.pixel_path_clip(frames, O.balanced_params(), lam, gate, QP, nthreads=nthreads)
    dt = time.perf_counter() - t0
    return frames.shape[0] * W * H / dt / 1e6, dt


def _grid_roofline(nmb: int, R: int, grid_ms: dict, int32_peak: float) -> dict:
    """INT32 roofline of the exhaustive grid on one frame: SAD is 2 lane-ops
    per 4 pixels (__vsadu4 + accumulate), SATD 112 per 4x4 block."""
    cands = nmb * (2 * R + 1) ** 2
    ops = {"sad": cands * 256 // 2, "satd": cands * 16 * SATD_OPS_PER_4X4}
    out = {"kernels": {"sad": "fullpel_sad_kernel", "satd": "fullpel_satd_kernel"}, "bound": "int32", "R": R,
           "unit": "Gop/s", "peak": round(int32_peak, 1), "frame": "one 1920x1088 frame"}
    for k, ms in grid_ms.items():
        g = ops[k] / (ms * 1e-3) / 1e9
        out[k] = {"ms": round(ms, 4), "ops": ops[k], "achieved": round(g, 1), "frac": round(g / int32_peak, 4)}
    return out


def cpu_model() -> dict:
    """Host CPU model name and online core count (stated with every CPU number)."""
    model = "unknown"
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                model = ln.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count()}


def cpu_stages(frames: np.ndarray, lam: float, gate: int) -> dict:
    """Per-stage time of the CPU restatement on one thread over `frames`
    (planes of the n-1 references, plain-ME and MC+T/Q of the n-1 P frames,
    HalfRes lookahead of all n), in ms per frame and Mpx/s."""
    from oracle import oracle as O

    n = frames.shape[0]
    params = O.balanced_params()
    t = {}
    t0 = time.perf_counter()
    planes = [O.build_planes4(frames[i], 32) for i in range(n - 1)]
    t["planes"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    picks = [O.me_frame(frames[i], frames[i - 1], planes[i - 1], params, lam, gate)[0] for i in range(1, n)]
    t["me"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    for i in range(1, n):
        O.mc_tq_frame(frames[i], frames[i - 1], picks[i - 1], QP)
    t["tq"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.lookahead_clip(frames, mode=2, nthreads=1)
    t["la"] = time.perf_counter() - t0
    out = {k: {"ms_per_frame": round(v * 1e3 / n, 3), "mpx_s": round(n * W * H / v / 1e6, 3)} for k, v in t.items()}
    tot = sum(t.values())
    out["total"] = {"ms_per_frame": round(tot * 1e3 / n, 3), "mpx_s": round(n * W * H / tot / 1e6, 3)}
    return out


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from oracle import oracle as O
    from rusty_h264_b200.accel import frame_lambda, split_gate_for_qp

    from rusty_h264_b200 import synth

    nthreads = O.lib().or_num_threads()
    lam = float(np.sqrt(frame_lambda(QP)) * 1.25)
    gate = split_gate_for_qp(QP)
    f = clip(1, args.frames)
    sample = args.frames  # the whole clip: the same workload as the GPU arm
    frames = np.ascontiguousarray(f[:sample])
    _, u_src, v_src = synth.hd_clip(args.frames, 1, with_chroma=True)
    U, V = synth.coded_chroma(u_src), synth.coded_chroma(v_src)
    for _ in range(args.warmup):  # short warm-ups: a full step is ~20 s of single-core work
        cpu_closed(np.ascontiguousarray(frames[:3]), np.ascontiguousarray(U[:3]), np.ascontiguousarray(V[:3]), lam,
                   gate, nthreads)
    times = []
    for _ in range(args.steps):
        _, dt = cpu_closed(frames, U, V, lam, gate, nthreads)
        times.append(dt)
    ms = float(np.mean(times)) * 1e3
    value = sample * W * H / (ms * 1e-3) / 1e6
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": "Mpx/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/i32", "data": "synthetic (seeded 1080p generator)", "impl": "reference",
        "config": workload_config(sample, ws),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mpx/s", "cores": nthreads, "kind": "port",
                         "sample": f"all {sample} frames of the 1080p clip per step; the closed loop is serial "
                                   f"(frame f needs rec(f-1), MBs in raster order) on one core, the lookahead "
                                   f"split over {nthreads} threads",
                         "cpu": cpu_model()},
        "e2e": {"value": round(value, 3), "unit": "Mpx/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, ws, rank, local):
    import torch

    from rusty_h264_b200 import accel as A

    mixed_streams = mixed_inputs() if args.mixed and rank == 0 else None  # host work, before any GPU call
    train_clips = [train_clip(s) for s in TRAIN_SEEDS] if not args.no_learned and rank == 0 else None
    torch.cuda.set_device(local)
    acc = A.Accel(local)
    n = args.frames
    f = clip(1 + rank, n)
    ch, cw = f.shape[1:]
    pad = 32
    pw, ph = cw + 2 * pad, ch + 2 * pad
    nmb = (cw // 16) * (ch // 16)
    qp = QP
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    params = A.default_me_params()
    dev = f"cuda:{local}"
    d_frames = torch.from_numpy(f).to(dev)
    planes = torch.empty((n - 1, 4, ph, pw), dtype=torch.uint8, device=dev)
    picks = torch.zeros((n, nmb, 6), dtype=torch.int32, device=dev)
    costs = torch.zeros((n, nmb, 2), dtype=torch.int64, device=dev)
    coeffs = torch.zeros((n, nmb, 256), dtype=torch.int16, device=dev)
    half = torch.empty((n, ch // 2, cw // 2), dtype=torch.uint8, device=dev)
    la_intra = torch.empty((n, nmb), dtype=torch.int32, device=dev)
    la_inter = torch.empty((n, nmb), dtype=torch.int32, device=dev)
    la_mvs = torch.empty((n, nmb, 2), dtype=torch.int32, device=dev)
    me_frames, tq_frames = [], []
    for i in range(1, n):
        pic = A.Picture(d_frames[i].data_ptr(), planes[i - 1].data_ptr(), cw, ch, pad)
        me_frames.append(A.MeFrame(pic, lam, gate, picks[i].data_ptr(), costs[i].data_ptr()))
        tq_frames.append(A.TqFrame(pic, picks[i].data_ptr(), qp, 6, coeffs[i].data_ptr()))
    stream = torch.cuda.current_stream()
    ev = {k: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for k in ("hpel", "me", "tq", "la")}
    stage_ms = {k: [] for k in ev}

    side = torch.cuda.Stream(device=dev)

    def lookahead():
        h = acc.L.h264a_downsample2x(acc.ctx, d_frames.data_ptr(), cw, ch, n, cw * ch, half.data_ptr(),
                                     acc._stream())
        acc._check(h)
        acc._check(acc.L.h264a_lookahead_costs(acc.ctx, d_frames.data_ptr(), half.data_ptr(), cw, ch, n, 2,
                                               la_intra.data_ptr(), la_inter.data_ptr(), la_mvs.data_ptr(),
                                               acc._stream()))

    def step(record=False):
        """One pass of the path.  Timed steps run the lookahead (its own work
        queue in the context) on a side stream beside planes, ME and T/Q, so
        that it fills the SMs the ME wavefront leaves idle while it ramps up
        and down; record=True runs the stages one after another on one
        stream, with events between them, for the per-stage times."""
        e = ev
        if not record:
            side.wait_stream(stream)
            with torch.cuda.stream(side):
                lookahead()
        if record:
            e["hpel"][0].record(stream)
        acc.hpel_build(d_frames[: n - 1], pad, out=planes)
        if record:
            e["hpel"][1].record(stream)
            e["me"][0].record(stream)
        acc.me_frames(me_frames, params)
        if record:
            e["me"][1].record(stream)
            e["tq"][0].record(stream)
        acc.mc_tq_frames(tq_frames)
        if record:
            e["tq"][1].record(stream)
            e["la"][0].record(stream)
            lookahead()
            e["la"][1].record(stream)
        else:
            stream.wait_stream(side)

    # hpel_build, one me_frames launch, mc_tq_frames per 96 frames, downsample2x, la_intra, la_chains
    kernels_per_step = 1 + 1 + (n - 1 + 95) // 96 + 1 + 2

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()

    for _ in range(args.warmup):
        step()
    acc.sync()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    acc.sync()
    clk = clocks.stop()
    barrier()
    ms = t0.elapsed_time(t1) / args.steps
    if ws > 1:
        import torch.distributed as dist

        tt = torch.tensor([ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    value = ws * n * W * H / (ms * 1e-3) / 1e6

    # per-stage device times (a separate pass with events between the stages)
    for _ in range(max(3, args.steps // 2)):
        step(record=True)
        torch.cuda.synchronize()
        for k, (a, b) in ev.items():
            stage_ms[k].append(a.elapsed_time(b))
    acc.sync()
    stage = {k: float(np.mean(v)) for k, v in stage_ms.items()}

    # The reconstruction side (not part of `value`): MC + T/Q with the luma
    # reconstruction, the chroma MC + T/Q + reconstruction, and the in-loop
    # deblocking of the reconstructed pictures, over the same 59 P frames.  The half-res luma planes of the lookahead stand in for the
    # chroma planes (960x544, textured).
    rec = torch.empty((n, ch, cw), dtype=torch.uint8, device=dev)
    ccoef = torch.empty((n, nmb, 128), dtype=torch.int16, device=dev)
    crec = torch.empty((2, n, ch // 2, cw // 2), dtype=torch.uint8, device=dev)
    rec_frames = [A.TqRecFrame(tq_frames[i - 1], rec[i].data_ptr()) for i in range(1, n)]
    chroma_frames = [A.TqChromaFrame(half[i].data_ptr(), half[i].data_ptr(), half[i - 1].data_ptr(),
                                     half[i - 1].data_ptr(), cw, ch, picks[i].data_ptr(), qp, ccoef[i].data_ptr(),
                                     crec[0, i].data_ptr(), crec[1, i].data_ptr()) for i in range(1, n)]
    db_frames = [A.DeblockFrame(rec[i].data_ptr(), crec[0, i].data_ptr(), crec[1, i].data_ptr(), cw, ch,
                                picks[i].data_ptr(), coeffs[i].data_ptr(), qp, 0, 0, 0) for i in range(1, n)]
    extra = {"mc_tq_rec": [], "chroma_mc_tq_rec": [], "deblock": []}
    for _ in range(max(3, args.steps // 2) + 1):
        a, b, c2, d2 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        a.record(stream)
        acc.mc_tq_rec_frames(rec_frames)
        b.record(stream)
        acc.mc_tq_chroma_frames(chroma_frames)
        c2.record(stream)
        acc.deblock_frames(db_frames)
        d2.record(stream)
        torch.cuda.synchronize()
        extra["mc_tq_rec"].append(a.elapsed_time(b))
        extra["chroma_mc_tq_rec"].append(b.elapsed_time(c2))
        extra["deblock"].append(c2.elapsed_time(d2))
    acc.sync()
    extra_ms = {k: round(float(np.mean(v[1:])), 4) for k, v in extra.items()}

    # The exhaustive full-pel probe as cost grids (h264a_fullpel_grid, not part
    # of value): one frame at R = 32, the SAD and the SATD argmin timed apart.
    grid_r = 32
    pic1 = A.Picture(d_frames[1].data_ptr(), planes[0].data_ptr(), cw, ch, pad)
    grid_ms = {}
    for metric, key in ((0, "sad"), (1, "satd")):
        ts = []
        for rep in range(4):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            acc.fullpel_grid(pic1, grid_r, metric=metric, want_grids=False)
            b.record(stream)
            torch.cuda.synchronize()
            if rep:
                ts.append(a.elapsed_time(b))
        grid_ms[key] = float(np.mean(ts))
    acc.sync()
    work4x4 = int(picks[1:, :, 5].sum().item())
    int32_peak = acc.measure_int32_peak()
    # The same ME over the first third of the P frames: a launch's time is set
    # by the wavefront's critical path (254 anti-diagonals per 1080p frame),
    # so a third of the work takes most of the time.
    sub_n = max(1, (n - 1) // 3)
    sub_ms = []
    for rep in range(4):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        acc.me_frames(me_frames[:sub_n], params)
        b.record(stream)
        torch.cuda.synchronize()
        if rep:
            sub_ms.append(a.elapsed_time(b))
    acc.sync()
    me_ops = work4x4 * SATD_OPS_PER_4X4
    achieved = me_ops / (stage["me"] * 1e-3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    hpel_bytes = (n - 1) * (cw * ch + 4 * pw * ph)
    roofline = {
        "kernel": "me_frames_kernel (persistent plain-ME)", "bound": "int32", "achieved": round(achieved, 1),
        "peak": round(int32_peak, 1), "unit": "Gop/s", "frac": round(achieved / int32_peak, 4),
        "peak_source": "measured live by h264a_measure_int32_peak (INT32 is not in MEASURED_PEAKS.json)",
        # dram__bytes_read.sum + dram__bytes_write.sum of one launch (ncu --set full of the
        # 60-frame step: 481,440 MBs, 1374.5 MB + 42.6 MB), scaled by MBs to this launch
        "traffic": int(1415.2e6 / 481440 * (n - 1) * nmb),
        "traffic_source": "ncu capture of the 60-frame 1080p launch, scaled by macroblocks",
        "work": {"satd_4x4_evals_per_step": work4x4, "ops_per_4x4": SATD_OPS_PER_4X4},
        "critical_path": {"me_ms_all_frames": round(stage["me"], 3), "frames": n - 1,
                          "me_ms_third_of_frames": round(float(np.mean(sub_ms)), 3), "frames_in_third": sub_n,
                          "note": "a third of the frames takes most of the launch time: the wavefront's critical "
                                  "path, not INT32 throughput, bounds the kernel"},
        "fullpel_grid": _grid_roofline(nmb, grid_r, grid_ms, int32_peak),
        "hpel_kernel": {"bound": "hbm", "achieved_gbs": round(hpel_bytes / (stage["hpel"] * 1e-3) / 1e9, 1),
                        "peak_gbs": hbm_peak, "frac": round(hpel_bytes / (stage["hpel"] * 1e-3) / 1e9 / hbm_peak, 4),
                        "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650"},
    }
    source_model = {
        "workload": "the same clip with every P frame searched against the previous SOURCE frame (the frames are "
                    "then independent and interleave in one ME launch): planes, plain-ME, MC+T/Q, HalfRes lookahead",
        "value": round(value, 2), "unit": "Mpx/s", "ms_per_step": round(ms, 4),
        "stage_ms": {k: round(v, 4) for k, v in stage.items()},
        "reconstruction_ms": dict(extra_ms, note="timed separately over the same 59 P frames"),
        "roofline": roofline, "clocks": clk, "gpu_launches_per_step": kernels_per_step,
    }

    # ---- the headline: the closed reconstruction loop, device-resident ----
    from rusty_h264_b200 import synth

    _, u_src, v_src = synth.hd_clip(n, 1 + rank, with_chroma=True)
    U, V = synth.coded_chroma(u_src), synth.coded_chroma(v_src)
    cb = ClosedBufs(acc, torch, f, U, V)
    cjob = cb.job(A, lam, gate, qp)
    side2 = torch.cuda.Stream(device=dev)

    def closed_step():
        # the lookahead (mb-tree input) beside the loop, on its own queue
        side2.wait_stream(stream)
        with torch.cuda.stream(side2):
            cb.lookahead(acc)
        acc.closed_frames(cjob, params)
        stream.wait_stream(side2)

    for _ in range(args.warmup):
        closed_step()
    acc.sync()
    barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(args.steps):
        closed_step()
    t1.record(stream)
    torch.cuda.synchronize()
    acc.sync()
    clk = clocks.stop()
    barrier()
    cms = t0.elapsed_time(t1) / args.steps
    if ws > 1:
        import torch.distributed as dist

        tt = torch.tensor([cms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        cms = float(tt.item())
    cvalue = ws * n * W * H / (cms * 1e-3) / 1e6
    # the loop's own launch (planes of rec(0), then the pipelined kernel over
    # every P frame) timed alone on its stream, and the frame-by-frame path
    loop_ms = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        acc.closed_frames(cjob, params)
        e1.record(stream)
        torch.cuda.synchronize()
        loop_ms.append(e0.elapsed_time(e1))
    acc.sync()
    pipe_ms = float(np.median(loop_ms))
    cstage = closed_stage_ms(acc, torch, A, cb, params, lam, gate, qp)
    cwork = int(cb.picks[1:, :, 5].sum().item())
    c_achieved = cwork * SATD_OPS_PER_4X4 / (pipe_ms * 1e-3) / 1e9
    croof = {
        "kernel": "closed_pipe_kernel (one launch over every P frame: a CTA per MB, its search, MC + T/Q, "
                  "reconstruction and deblocking, each reconstruction's planes built band by band; consecutive "
                  "frames overlap)", "bound": "int32",
        "achieved": round(c_achieved, 1), "peak": round(int32_peak, 1), "unit": "Gop/s",
        "frac": round(c_achieved / int32_peak, 4),
        "peak_source": "measured live by h264a_measure_int32_peak (INT32 is not in MEASURED_PEAKS.json)",
        "traffic": int(1415.2e6 / 481440 * nmb * (n - 1)),
        "traffic_source": "ncu capture of the 60-frame source-model launch (1415.2 MB over 481,440 MBs), scaled "
                          "by macroblocks to the launch's 59 P frames",
        "work": {"satd_4x4_evals_per_step": cwork, "ops_per_4x4": SATD_OPS_PER_4X4,
                 "launch_ms": round(pipe_ms, 3), "launches": 1,
                 "timing": "CUDA events around h264a_closed_frames alone (memsets, the planes of rec(0), the "
                           "pipelined kernel), median of 3"},
        "note": "each frame is a wavefront of 254 anti-diagonals bound by its critical path; the pipelined launch "
                "overlaps a frame with the rows of the previous one its searches do not read",
    }
    closed_launches = 2 + 3  # the planes of rec(0) and the pipelined kernel; lookahead 3
    line = {
        "metric": METRIC, "value": round(cvalue, 2), "unit": "Mpx/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(cms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8/i32", "data": "synthetic (seeded 1080p generator with chroma, per-rank seed)",
        "config": workload_config(n, ws),
        "stage_ms": {"closed_frames_launch": round(pipe_ms, 4),
                     "frame_by_frame": {k: round(v, 4) for k, v in cstage.items()},
                     "note": "frame_by_frame: the same loop as h264a_closed_step_frame launches, one frame "
                             "after another (planes, then the fused kernel), for comparison"},
        "roofline": croof,
        "clocks": clk,
        "gpu_launches": closed_launches * args.steps,
        "source_reference_model": source_model,
    }
    if not args.no_e2e:
        host_frames = torch.from_numpy(f).pin_memory()
        outs = dict(picks=torch.zeros((n, nmb, 6), dtype=torch.int32).pin_memory(),
                    costs=torch.zeros((n, nmb, 2), dtype=torch.int64).pin_memory(),
                    coeffs=torch.zeros((n, nmb, 256), dtype=torch.int16).pin_memory(),
                    la_intra=torch.zeros((n, nmb), dtype=torch.int32).pin_memory(),
                    la_inter=torch.zeros((n, nmb), dtype=torch.int32).pin_memory(),
                    la_mvs=torch.zeros((n, nmb, 2), dtype=torch.int32).pin_memory())
        outs_np = {k: v.numpy() for k, v in outs.items()}
        fr_np = host_frames.numpy()
        def stream(steps):
            # every step's frames go up inside the loop; step k+1's upload is
            # queued before step k's call and overlaps its compute
            acc.pixel_path_prefetch(fr_np)
            for k in range(steps):
                if k + 1 < steps:
                    acc.pixel_path_prefetch(fr_np)
                acc.pixel_path_host(fr_np, params, lam, gate, qp, out=outs_np)

        stream(args.warmup)
        barrier()
        s0 = time.perf_counter()
        stream(args.steps)
        e2e_ms = (time.perf_counter() - s0) * 1e3 / args.steps
        s0 = time.perf_counter()  # one synchronous call on its own, for comparison
        acc.pixel_path_host(fr_np, params, lam, gate, qp, out=outs_np)
        single_ms = (time.perf_counter() - s0) * 1e3
        if ws > 1:
            import torch.distributed as dist

            tt = torch.tensor([e2e_ms, single_ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_ms, single_ms = (float(v) for v in tt.tolist())
        d2h = sum(v.numel() * v.element_size() for v in outs.values())
        source_model["e2e"] = {"value": round(ws * n * W * H / (e2e_ms * 1e-3) / 1e6, 2), "unit": "Mpx/s",
                       "h2d_bytes_per_step": int(f.nbytes), "d2h_bytes_per_step": int(d2h),
                       "ms_per_step": round(e2e_ms, 3),
                       "timing": "wall clock over the streamed steps (each upload queued before the previous "
                                 "step's call, h264a_pixel_path_prefetch)",
                       "single_call_ms": round(single_ms, 3)}
        # the host path and the device-resident path must agree
        for k, t in (("picks", picks), ("coeffs", coeffs), ("la_intra", la_intra), ("la_inter", la_inter),
                     ("la_mvs", la_mvs)):
            assert np.array_equal(outs_np[k], t.cpu().numpy()), k
        # the closed loop through the host-buffer entry: every step uploads the
        # clip (luma + chroma) and downloads picks, costs, levels and the
        # reconstruction
        hy, hu, hv = (torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy() for a in (f, U, V))
        pinned = lambda shp, dt: torch.zeros(shp, dtype=dt).pin_memory().numpy()
        r_host = dict(picks=pinned((n, nmb, 6), torch.int32), costs=pinned((n, nmb, 2), torch.int64),
                      coeffs=pinned((n, nmb, 256), torch.int16), ccoeffs=pinned((n, nmb, 128), torch.int16),
                      rec_y=pinned(hy.shape, torch.uint8), rec_u=pinned(hu.shape, torch.uint8),
                      rec_v=pinned(hv.shape, torch.uint8))
        for _ in range(max(1, args.warmup)):
            acc.pixel_path_closed(hy, hu, hv, params, lam, gate, qp, out=r_host)
        barrier()
        s0 = time.perf_counter()
        for _ in range(args.steps):
            acc.pixel_path_closed(hy, hu, hv, params, lam, gate, qp, out=r_host)
        ce2e_ms = (time.perf_counter() - s0) * 1e3 / args.steps
        if ws > 1:
            import torch.distributed as dist

            tt = torch.tensor([ce2e_ms], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ce2e_ms = float(tt.item())
        line["e2e"] = {"value": round(ws * n * W * H / (ce2e_ms * 1e-3) / 1e6, 2), "unit": "Mpx/s",
                       "h2d_bytes_per_step": int(hy.nbytes + hu.nbytes + hv.nbytes),
                       "d2h_bytes_per_step": int(sum(r_host[k].nbytes for k in ("picks", "costs", "coeffs", "ccoeffs",
                                                                                 "rec_y", "rec_u", "rec_v"))),
                       "ms_per_step": round(ce2e_ms, 3),
                       "timing": "wall clock over synchronous h264a_pixel_path_closed calls from pinned host "
                                 "buffers (uploads, the loop, downloads of picks, costs, levels and reconstruction; "
                                 "each frame's downloads start when the kernel reports it final)"}
        # the host entry and the device-resident loop agree
        assert np.array_equal(r_host["rec_y"], cb.ry.cpu().numpy())
        assert np.array_equal(r_host["coeffs"], cb.coeffs.cpu().numpy())
    if rank == 0 and ws == 1 and not args.no_cpu:
        sample = np.ascontiguousarray(f[:8])
        v, dt = cpu_closed(sample, np.ascontiguousarray(U[:8]), np.ascontiguousarray(V[:8]), lam, gate, 1)
        line["cpu_baseline"] = {"value": round(v, 3), "unit": "Mpx/s", "cores": 1, "kind": "port",
                                "sample": "8 frames of the 1080p clip with chroma through the closed loop "
                                          "(7 P frames) + lookahead, one thread",
                                "cpu": cpu_model(), "stages": cpu_stages(sample, lam, gate)}
    if args.mixed and rank == 0:
        mixed_bufs, line["mixed_batch"] = mixed_batch(acc, torch, mixed_streams, params, lam, gate, args.gop_step)
    if not args.no_learned and rank == 0:
        from rusty_h264_b200 import bdrate

        plain_src = {"costs": costs.cpu().numpy(), "me_ms": stage["me"]}
        line["learned"], net, lrec = learned_arm(acc, torch, f, U, V, d_frames, planes, params, lam, gate, qp,
                                                 plain_src, args.learned_epochs, train_clips, args.steps)
        line["learned"]["closed_loop"]["psnr_p_frames"] = round(bdrate.psnr(f[1:, :H], lrec[1:, :H]), 3)
        line["learned"]["closed_loop"]["plain_psnr_p_frames"] = round(
            bdrate.psnr(f[1:, :H], cb.ry.cpu().numpy()[1:, :H]), 3)
        if not args.no_closed:
            line["bd_rate"] = bd_rate_record(acc, f, U, V, params, 1.25, net, args.bd_frames)
            if args.bd_4k:
                y4, u4, v4 = synth.hd_clip(args.bd_frames, 2, 3840, 2160, with_chroma=True)
                line["bd_rate_4k"] = bd_rate_record(acc, synth.coded_luma(y4), synth.coded_chroma(u4),
                                                    synth.coded_chroma(v4), params, 1.25, net, args.bd_frames,
                                                    3840, 2160)
        if args.mixed:
            line["mixed_batch"]["learned"] = mixed_learned(acc, torch, mixed_bufs, net, params, lam, gate,
                                                           line["mixed_batch"]["me_ms"])
        net.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    acc.close()


def main():
    args = parse()
    ws, rank, local = dist_init()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_ours(args, ws, rank, local)
    if ws > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
