"""Runs the closed reconstruction loop (h264a_pixel_path_closed) over the
seeded synthetic 1080p clip with chroma, and prints one JSON line: frames,
QP, the share of MBs that picked a 16x8 / 8x16 shape, and the luma PSNR of
the P frames' reconstruction.  The command the closed-loop profiles under
profiles/ were taken with:

    python -m rusty_h264_b200.closed_clip --frames 60 [--learned]

--learned runs the learned search with an untrained proposal net (seeded):
the launches and their shapes are those of a trained one.
"""
import argparse
import json

import numpy as np

from . import accel as A
from . import bdrate, synth


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", type=int, default=60)
    ap.add_argument("--qp", type=int, default=27)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--learned", action="store_true")
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    y, u, v = synth.hd_clip(a.frames, a.seed, with_chroma=True)
    Y, U, V = synth.coded_luma(y), synth.coded_chroma(u), synth.coded_chroma(v)
    acc = A.Accel(a.device)
    net = None
    if a.learned:
        from . import mvnet

        net = mvnet.MvNet(acc, seed=a.seed)
    lam = float(np.sqrt(A.frame_lambda(a.qp)) * 1.25)
    r = acc.pixel_path_closed(Y, U, V, A.default_me_params(), lam, A.split_gate_for_qp(a.qp), a.qp, net=net,
                              fallback_t=256)
    h = y.shape[1]
    print(json.dumps({"frames": a.frames, "qp": a.qp, "learned": a.learned,
                      "split_share": round(float((r["picks"][1:, :, 0] > 0).mean()), 4),
                      "psnr_p_frames": round(bdrate.psnr(y[1:], r["rec_y"][1:, :h]), 3)}))
    if net is not None:
        net.close()
    acc.close()


if __name__ == "__main__":
    main()
