"""The learned-proposal network's GPU kernels through the C ABI, against the
float64 CPU oracle (oracle/mvnet_ref.py), which applies the same bf16
roundings at the layer boundaries.  What remains between the two is fp32
accumulation order and the rare activation whose bf16 rounding flips with it,
so the tolerances are normwise: logits within 1% of their largest magnitude,
every gradient tensor within 2% (relative L2) with cosine > 0.999, the loss
within 0.1%."""
import numpy as np
import pytest

from oracle import mvnet_ref as M
from rusty_h264_b200 import accel as A
from rusty_h264_b200 import mvnet, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def acc():
    a = A.Accel(0)
    yield a
    a.close()


def small_batch(acc, P=3, cw=96, ch=64, seed=1):
    """P frame pairs of a textured clip, random neighbour MVs and labels."""
    # a crop of the textured generator's CIF-size frames (its rectangles need
    # frames wider and taller than 256 pixels)
    y, _, _ = synth.hd_clip(P + 1, 7 + seed, 352, 288)
    clip = np.ascontiguousarray(synth.coded_luma(y)[:, 16:16 + ch, 32:32 + cw])
    d = acc.to_dev(clip)
    pairs = acc.torch.tensor([[d[f].data_ptr(), d[f - 1].data_ptr()] for f in range(1, P + 1)], dtype=acc.torch.int64,
                             device="cuda:0")
    nmb = (cw // 16) * (ch // 16)
    rng = np.random.default_rng(seed)
    nmv = rng.integers(-150, 150, (P * nmb, 6)).astype(np.int16)
    lab = rng.integers(0, M.NCLS, P * nmb).astype(np.int16)
    x0 = np.stack([M.image(clip[f], clip[f - 1]) for f in range(1, P + 1)])
    return dict(clip=clip, d=d, pairs=pairs, nmv=nmv, lab=lab, d_nmv=acc.to_dev(nmv), d_lab=acc.to_dev(lab), x0=x0,
                P=P, cw=cw, ch=ch)


def test_forward_matches_oracle(acc):
    net = mvnet.MvNet(acc, seed=3)
    b = small_batch(acc)
    got = net.forward(b["pairs"].data_ptr(), b["P"], b["cw"], b["ch"], b["d_nmv"].data_ptr()).cpu().numpy()
    want = M.forward(M.unflatten(net.params()), b["x0"], b["nmv"].astype(np.int64))["logits"]
    assert got.shape == want.shape
    assert np.abs(got - want).max() <= 1e-2 * np.abs(want).max() + 1e-3
    net.close()


@pytest.mark.parametrize("P,cw,ch", [(3, 96, 64), (1, 176, 144), (2, 48, 32)])
def test_gradients_match_oracle(acc, P, cw, ch):
    net = mvnet.MvNet(acc, seed=5 + P)
    b = small_batch(acc, P, cw, ch, seed=2 + P)
    g, loss = net.grads(b["pairs"].data_ptr(), P, cw, ch, b["d_nmv"].data_ptr(), b["d_lab"].data_ptr())
    g = g.cpu().numpy().astype(np.float64)
    wl, wg, _ = M.loss_and_grads(net.params(), b["x0"], b["nmv"].astype(np.int64), b["lab"].astype(np.int64))
    assert abs(float(loss.item()) - wl) <= 1e-3 * abs(wl)
    o = 0
    for name, shp in M.SHAPES:
        k = int(np.prod(shp))
        a, w = g[o:o + k], wg[o:o + k]
        nw = np.linalg.norm(w)
        if nw > 0:
            assert np.linalg.norm(a - w) <= 2e-2 * nw, name
            assert a @ w / (np.linalg.norm(a) * nw) > 0.999, name
        else:
            assert np.abs(a).max() == 0, name
        o += k
    net.close()


def test_training_reduces_loss_and_propose_is_top8(acc):
    """A few hundred Adam steps on one CIF clip's items cut the loss; then
    h264a_mvnet_propose over whole frames equals the top-8 of the forward
    logits of the same MBs (neighbour features from the guide MVs)."""
    y, _, _ = synth.cif_clip(4, 3)
    clip = synth.coded_luma(y)
    n, ch, cw = clip.shape
    ts = mvnet.harvest(acc, [clip], (27,)).finish()
    net = mvnet.MvNet(acc, seed=9)
    losses, _, steps = mvnet.train(net, ts, epochs=150, lr=2e-3, pairs_per_step=1, log_every=1)
    first = np.mean([v for _, v in losses[:5]])
    last = np.mean([v for _, v in losses[-5:]])
    assert last < 0.6 * first, (first, last)
    mb_w, mb_h = cw // 16, ch // 16
    nmb = mb_w * mb_h
    rng = np.random.default_rng(4)
    guide = rng.integers(-60, 60, (2, nmb, 2)).astype(np.int32)
    d_guide = acc.to_dev(guide)
    d = ts.keep[0]
    props = acc.zeros((2, nmb, 16), acc.torch.int32)
    net.propose([mvnet.MvnetFrame(d[f + 1].data_ptr(), d[f].data_ptr(), cw, ch, d_guide[f].data_ptr(),
                                  props[f].data_ptr()) for f in range(2)])
    got = props.cpu().numpy().reshape(2, nmb, 8, 2)
    pairs = acc.torch.tensor([[d[f + 1].data_ptr(), d[f].data_ptr()] for f in range(2)], dtype=acc.torch.int64,
                             device="cuda:0")
    nmv = np.concatenate([mvnet.neighbour_mvs(guide[f], mb_w, mb_h) for f in range(2)])
    lg = net.forward(pairs.data_ptr(), 2, cw, ch, acc.to_dev(nmv).data_ptr()).cpu().numpy()[:, :M.NCLS]
    top = np.argsort(-lg, axis=1, kind="stable")[:, :8]
    want = np.stack([4 * (top % 17 - 8), 4 * (top // 17 - 8)], -1).reshape(2, nmb, 8, 2)
    assert np.array_equal(got, want)
    net.close()
