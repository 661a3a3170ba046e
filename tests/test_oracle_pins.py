"""Pins the CPU oracle to the reference's own tests (CPU only, no GPU).

Each test ports one reference test (file:line in its docstring) with the same
corpus or LCG stream, checking the oracle against either the reference's
literal expected values (tests/golden/reference_known_answers.json) or an
independent numpy restatement of the formula that reference test spells out.
Where the reference loops tens of thousands of times, the first part of the
identical stream is used so the CPU suite stays fast.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests._lcg import Lcg32, Lcg64

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_known_answers.json")))

H4 = np.array([[1, 1, 1, 1], [1, 1, -1, -1], [1, -1, -1, 1], [1, -1, 1, -1]], np.int64)
CF = np.array([[1, 1, 1, 1], [2, 1, -1, -2], [1, -1, -1, 1], [1, -2, 2, -1]], np.int64)


def np_satd_sum(src, pred):
    """Σ|H·d·Hᵀ| over the 4x4 blocks of (src - pred): the scalar satd_px."""
    d = src.astype(np.int64) - pred.astype(np.int64)
    h, w = d.shape
    tot = 0
    for by in range(0, h, 4):
        for bx in range(0, w, 4):
            tot += int(np.abs(H4 @ d[by:by + 4, bx:bx + 4] @ H4.T).sum())
    return tot


def np_wels(src, pred):
    """openh264's region SATD: Σ_4x4 ((Σ|H·d|+1)>>1) (x86_asm.rs satd_region_ref)."""
    d = src.astype(np.int64) - pred.astype(np.int64)
    h, w = d.shape
    tot = 0
    for by in range(0, h, 4):
        for bx in range(0, w, 4):
            tot += (int(np.abs(H4 @ d[by:by + 4, bx:bx + 4] @ H4.T).sum()) + 1) >> 1
    return tot


def corpus(seed):
    """satd_sad.rs:389-400 / x86_asm.rs:306-314 structured corpus."""
    i = np.arange(16)[:, None]
    j = np.arange(16)[None, :]
    a = ((i * 37 + j * 101 + seed * 3) & 0xFF).astype(np.uint8)
    b = ((i * 53 + j * 17 + seed * 29 + 7) & 0xFF).astype(np.uint8)
    return np.ascontiguousarray(a), np.ascontiguousarray(b)


def test_satd_sad_family_matches_openh264_formula():
    """satd_sad.rs:403-427, x86_asm.rs:303-323: every shape vs the openh264-C formula."""
    L = O.lib()
    for seed in range(96):
        a, b = corpus(seed)
        for w, h in [(16, 16), (16, 8), (8, 16), (8, 8), (4, 4)]:
            got = L.or_satd_region_wels(O.ptr(a), 16, O.ptr(b), 16, w, h)
            assert got == np_wels(a[:h, :w], b[:h, :w]), (seed, w, h)
        for w, h in [(16, 16), (16, 8), (8, 16)]:
            got = L.or_sad(O.ptr(a), 16, O.ptr(b), 16, w, h)
            assert got == int(np.abs(a[:h, :w].astype(int) - b[:h, :w].astype(int)).sum())


def test_satd_extremes():
    """satd_sad.rs:430-452: saturated and alternating blocks."""
    L = O.lib()
    for va, vb in [(0, 255), (255, 0), (0, 0), (255, 255)]:
        a = np.full((16, 16), va, np.uint8)
        b = np.full((16, 16), vb, np.uint8)
        assert L.or_satd_region_wels(O.ptr(a), 16, O.ptr(b), 16, 16, 16) == np_wels(a, b)
    i = np.arange(16)[:, None]
    j = np.arange(16)[None, :]
    a = np.ascontiguousarray(np.where((i + j) % 2 == 0, 255, 0).astype(np.uint8))
    b = np.ascontiguousarray(np.broadcast_to(np.where(i % 2 == 0, 0, 255), (16, 16)).astype(np.uint8))
    assert L.or_satd_region_wels(O.ptr(a), 16, O.ptr(b), 16, 16, 16) == np_wels(a, b)
    assert L.or_satd_region_wels(O.ptr(a), 16, O.ptr(b), 16, 8, 8) == np_wels(a[:8, :8], b[:8, :8])


def test_satd_px_is_exactly_twice_wels():
    """encoder tests/satd_asm_compare.rs:38-75: 2·Wels == Σ|H·d| (seed 0x1234_5678_9abc_def0)."""
    st = Lcg64(0x1234_5678_9ABC_DEF0)
    L = O.lib()
    for n in (4, 8, 16):
        for _ in range(600):
            src = st.bytes(n * n).reshape(n, n).copy()
            pred = st.bytes(n * n).reshape(n, n).copy()
            rust = np_satd_sum(src, pred)
            wels = L.or_satd_region_wels(O.ptr(src), n, O.ptr(pred), n, n, n)
            assert 2 * wels == rust
            assert O.satd_px(src, n, pred, n, n, n) == rust


def test_satd_avg_matches_materialized():
    """encoder tests/satd_avg_compare.rs:129-170 (seed 0xabcd_ef01_2345_6789), every x4 shape."""
    st = Lcg64(0xABCD_EF01_2345_6789)
    L = O.lib()
    for _ in range(150):
        ss = 16 + int(st.next()) % 32
        rs = 16 + int(st.next()) % 32
        src = st.bytes(15 * ss + 16 + 8)
        planes = [st.bytes(15 * rs + 16 + 4 * rs + 64) for _ in range(3)]
        idx = [(int(st.next()) % 3, (int(st.next()) % 4) * rs + int(st.next()) % 32,
                int(st.next()) % 3, (int(st.next()) % 4) * rs + int(st.next()) % 32) for _ in range(4)]
        for (pa, oa, pb, ob) in idx:
            for w, h in [(16, 16), (16, 8), (8, 16), (8, 8)]:
                A = planes[pa][oa:]
                B = planes[pb][ob:]
                got = L.or_satd_avg(O.ptr(src), ss, O.ptr(np.ascontiguousarray(A)), O.ptr(np.ascontiguousarray(B)),
                                    rs, w, h)
                s2 = np.lib.stride_tricks.as_strided(src, (h, w), (ss, 1))
                a2 = np.lib.stride_tricks.as_strided(A, (h, w), (rs, 1)).astype(np.int32)
                b2 = np.lib.stride_tricks.as_strided(B, (h, w), (rs, 1)).astype(np.int32)
                avg = ((a2 + b2 + 1) >> 1).astype(np.uint8)
                assert got == np_satd_sum(s2, avg)


def test_quant_mf_oh_table_matches_reference_rows():
    """transform.rs:1447-1500: derived MF table == the reference's literal 52 rows."""
    L = O.lib()
    rows = GOLD["quant_mf_oh"]["rows"]
    for qp in range(52):
        mf = np.zeros(8, np.int16)
        L.or_quant_mf_oh(qp, O.ptr(mf, O.i16p))
        assert mf.tolist() == rows[qp], qp


def test_quant_four_matches_wels_new_quant():
    """transform_quant.rs:199-222 and x86_asm.rs:325-352 with the fixed FF/MF vectors."""
    g = GOLD["quant_four_fixed"]
    ff = np.array(g["ff"], np.int16)
    mf = np.array(g["mf"], np.int16)
    L = O.lib()
    for seed in range(64):
        k = np.arange(64)
        inp = (((k * 37 + seed * 53) % 2000) - 1000).astype(np.int16)
        got = inp.copy()
        L.or_quant_four_4x4(O.ptr(got, O.i16p), O.ptr(ff, O.i16p), O.ptr(mf, O.i16p))
        row = (k % 16) // 4
        col = k % 4
        pos = (row & 1) * 4 + col
        c = inp.astype(np.int64)
        lvl = ((np.abs(c) + ff[pos]) * mf[pos]) >> 16
        want = np.where(c < 0, -lvl, lvl).astype(np.int16)
        assert np.array_equal(got, want), seed


def test_quant_four_full_range_lcg():
    """transform_quant.rs:591-617 (seed 0x1234): full i16 range incl. i16::MIN."""
    st = Lcg64(0x1234)
    L = O.lib()
    for rnd in range(300):
        ffmf = (st.bulk(16) % np.uint64(32768)).astype(np.int16)
        ff = np.ascontiguousarray(ffmf[0::2])
        mf = np.ascontiguousarray(ffmf[1::2])
        inp = (st.bulk(64) & np.uint64(0xFFFF)).astype(np.uint16).view(np.int16).copy()
        if rnd == 0:
            inp[0], inp[1], inp[2] = -32768, 32767, 0
        got = inp.copy()
        L.or_quant_four_4x4(O.ptr(got, O.i16p), O.ptr(ff, O.i16p), O.ptr(mf, O.i16p))
        k = np.arange(64)
        pos = (((k % 16) // 4) & 1) * 4 + k % 4
        c = inp.astype(np.int64)
        lvl = (((np.abs(c) + ff[pos].astype(np.int64)) * mf[pos].astype(np.int64)) >> 16).astype(np.int64)
        want = np.where(c < 0, -lvl, lvl).astype(np.int64).astype(np.int16)
        assert np.array_equal(got, want), rnd


def test_dct_four_t4_matches_forward_core_formula():
    """transform_quant.rs:141-166: dct_four_t4 == Cf·X·Cfᵀ per sub-block, openh264 order."""
    L = O.lib()
    y = np.arange(8)[:, None]
    x = np.arange(8)[None, :]
    for seed in range(128):
        src = np.ascontiguousarray(((y * 31 + x * 17 + seed * 7) & 0xFF).astype(np.uint8))
        pred = np.ascontiguousarray(((y * 13 + x * 41 + seed * 5 + 9) & 0xFF).astype(np.uint8))
        dct = np.zeros(64, np.int16)
        L.or_dct_four_t4(O.ptr(dct, O.i16p), O.ptr(src), 8, O.ptr(pred), 8)
        for k, (ox, oy) in enumerate([(0, 0), (4, 0), (0, 4), (4, 4)]):
            d = src[oy:oy + 4, ox:ox + 4].astype(np.int64) - pred[oy:oy + 4, ox:ox + 4]
            want = (CF @ d @ CF.T).reshape(-1)
            assert np.array_equal(dct[k * 16:(k + 1) * 16], want.astype(np.int16)), (seed, k)


def test_dct_lcg_stream_and_saturated_round():
    """transform_quant.rs:620-640 (seed 0xbeef): random src/pred incl. the 255-vs-0 round."""
    st = Lcg64(0xBEEF)
    L = O.lib()
    for rnd in range(300):
        sp = st.bytes(128)
        src = np.ascontiguousarray(sp[0::2].reshape(8, 8))
        pred = np.ascontiguousarray(sp[1::2].reshape(8, 8))
        if rnd == 0:
            src[:] = 255
            pred[:] = 0
        dct = np.zeros(64, np.int16)
        L.or_dct_four_t4(O.ptr(dct, O.i16p), O.ptr(src), 8, O.ptr(pred), 8)
        for k, (ox, oy) in enumerate([(0, 0), (4, 0), (0, 4), (4, 4)]):
            d = src[oy:oy + 4, ox:ox + 4].astype(np.int64) - pred[oy:oy + 4, ox:ox + 4]
            assert np.array_equal(dct[k * 16:(k + 1) * 16], (CF @ d @ CF.T).reshape(-1).astype(np.int16))


def test_forward_transforms_flat_known_answers():
    """transform.rs:1167-1188: flat 4x4 -> DC 64, flat 8x8 -> DC 256, AC zero."""
    L = O.lib()
    g4 = GOLD["forward_core_flat"]
    out = np.zeros(16, np.int32)
    L.or_forward_core(O.ptr(np.array(g4["input"], np.int32), O.i32p), O.ptr(out, O.i32p))
    assert out[0] == g4["dc"] and not out[1:].any()
    g8 = GOLD["forward_core_8x8_flat"]
    out8 = np.zeros(64, np.int32)
    L.or_forward_core_8x8(O.ptr(np.array(g8["input"], np.int32), O.i32p), O.ptr(out8, O.i32p))
    assert out8[0] == g8["dc"] and not out8[1:].any()


def test_quantize_structure_matches_quant_four():
    """transform.rs:121-139: quantize == quant_four_4x4 with quant_dz_ff + QUANT_MF_OH."""
    L = O.lib()
    rng = np.random.default_rng(7)
    for qp in range(52):
        c = rng.integers(-4080, 4081, 16).astype(np.int32)
        out = np.zeros(16, np.int32)
        L.or_quantize(O.ptr(c, O.i32p), qp, 6, O.ptr(out, O.i32p))
        ff = np.zeros(8, np.int16)
        mf = np.zeros(8, np.int16)
        L.or_quant_dz_ff(qp, 6, O.ptr(ff, O.i16p))
        L.or_quant_mf_oh(qp, O.ptr(mf, O.i16p))
        d = np.zeros(64, np.int16)
        d[:16] = c
        L.or_quant_four_4x4(O.ptr(d, O.i16p), O.ptr(ff, O.i16p), O.ptr(mf, O.i16p))
        assert np.array_equal(out, d[:16].astype(np.int32))


def test_median_and_mv_prediction_known_answers():
    """inter.rs:1994-2034."""
    L = O.lib()
    for a, b, c, want in GOLD["median3"]["cases"]:
        assert L.or_median3(a, b, c) == want
    for case in GOLD["predict_mv"]["cases"]:
        arrs = [np.array(case[k], np.int32) for k in ("a", "b", "c")]
        out = np.zeros(2, np.int32)
        L.or_predict_mv(*[O.ptr(x, O.i32p) for x in arrs], case["cur_ref"], O.ptr(out, O.i32p))
        assert out.tolist() == case["want"], case


def test_mc_luma_known_answers():
    """inter.rs:2037-2063: zero-MV copy, edge clamp, flat stays flat."""
    for case in GOLD["mc_luma"]["cases"]:
        ref = np.array(case["ref"], np.uint8).reshape(case["ch"], case["cw"])
        got = O.mc_luma(ref, case["x0"], case["y0"], case["bw"], case["bh"], case["mvx"], case["mvy"])
        assert got.reshape(-1).tolist() == case["want"]
    fl = GOLD["mc_luma"]["flat"]
    ref = np.full((fl["ch"], fl["cw"]), fl["value"], np.uint8)
    for fx, fy in fl["phases"]:
        got = O.mc_luma(ref, fl["x0"], fl["y0"], fl["bw"], fl["bh"], fx, fy)
        assert (got == fl["value"]).all()


def np_luma_sample_block(ref, x0, y0, bw, bh, mvx, mvy):
    """luma_sample (inter.rs:134-176) vectorised over a block: the spec §8.4.2.2.1 oracle."""
    ch, cw = ref.shape
    ix0, iy0 = x0 + (mvx >> 2), y0 + (mvy >> 2)
    fx, fy = mvx & 3, mvy & 3
    yy = iy0 + np.arange(bh)[:, None]
    xx = ix0 + np.arange(bw)[None, :]
    R = ref.astype(np.int64)

    def g(dx, dy):
        return R[np.clip(yy + dy, 0, ch - 1), np.clip(xx + dx, 0, cw - 1)]

    def hor6(dy):
        return g(-2, dy) - 5 * g(-1, dy) + 20 * g(0, dy) + 20 * g(1, dy) - 5 * g(2, dy) + g(3, dy)

    def ver6(dx):
        return g(dx, -2) - 5 * g(dx, -1) + 20 * g(dx, 0) + 20 * g(dx, 1) - 5 * g(dx, 2) + g(dx, 3)

    clip = lambda v: np.clip(v, 0, 255)
    if fx == 0 and fy == 0:
        return g(0, 0)
    b = clip((hor6(0) + 16) >> 5)
    h = clip((ver6(0) + 16) >> 5)
    m = clip((ver6(1) + 16) >> 5)
    s = clip((hor6(1) + 16) >> 5)
    j = clip((hor6(-2) - 5 * hor6(-1) + 20 * hor6(0) + 20 * hor6(1) - 5 * hor6(2) + hor6(3) + 512) >> 10)
    av = lambda p, q: (p + q + 1) >> 1
    return {
        (1, 0): av(g(0, 0), b), (2, 0): b, (3, 0): av(g(1, 0), b),
        (0, 1): av(g(0, 0), h), (1, 1): av(b, h), (2, 1): av(b, j), (3, 1): av(b, m),
        (0, 2): h, (1, 2): av(h, j), (2, 2): j, (3, 2): av(j, m),
        (0, 3): av(g(0, 1), h), (1, 3): av(h, s), (2, 3): av(j, s), (3, 3): av(m, s),
    }[(fx, fy)]


def test_mc_luma_block_kernels_match_per_pixel_spec():
    """inter.rs:1914-1947 (40x32, LCG32 0x1357_9bdf): mc_luma == luma_sample, interior and edge."""
    st = Lcg32(0x1357_9BDF)
    cw, ch = 40, 32
    ref = np.array([(st.next() >> 24) & 0xFF for _ in range(cw * ch)], np.uint8).reshape(ch, cw)
    for bw, bh in [(16, 16), (8, 8), (4, 4), (8, 16), (16, 8)]:
        for x0, y0 in [(8, 8), (0, 0), (cw - bw, ch - bh)]:
            for mvx in range(-9, 10):
                for mvy in range(-9, 10):
                    got = O.mc_luma(ref, x0, y0, bw, bh, mvx, mvy)
                    want = np_luma_sample_block(ref, x0, y0, bw, bh, mvx, mvy)
                    assert np.array_equal(got, want), (bw, bh, x0, y0, mvx, mvy)


def test_luma_sample_oracle_matches_numpy_spec():
    """The C luma_sample restatement agrees with the vectorised spec form."""
    rng = np.random.default_rng(3)
    ref = rng.integers(0, 256, (24, 20), dtype=np.uint8)
    for fx in range(4):
        for fy in range(4):
            for ix, iy in [(-5, -5), (0, 0), (7, 9), (19, 23), (25, 30)]:
                want = np_luma_sample_block(ref, ix, iy, 1, 1, fx, fy)[0, 0]
                assert O.luma_sample(ref, ix, iy, fx, fy) == want


def np_hpel_planes(f):
    """H/V/C from the padded plane with taps clamped to the plane (inter.rs:908-991)."""
    ph, pw = f.shape
    F = f.astype(np.int64)
    ys = np.arange(ph)[:, None]
    xs = np.arange(pw)[None, :]
    tap = [1, -5, 20, 20, -5, 1]

    def at(dy, dx):
        return F[np.clip(ys + dy, 0, ph - 1), np.clip(xs + dx, 0, pw - 1)]

    Hs = sum(t * at(0, k - 2) for k, t in enumerate(tap))
    Vs = sum(t * at(k - 2, 0) for k, t in enumerate(tap))
    # centre: horizontal 6-tap over the clamped-column vertical intermediates
    vt = sum(t * F[np.clip(np.arange(ph) + k - 2, 0, ph - 1)] for k, t in enumerate(tap))  # ph x pw
    Cs = sum(t * vt[:, np.clip(np.arange(pw) + k - 2, 0, pw - 1)] for k, t in enumerate(tap))
    clip = lambda v: np.clip(v, 0, 255).astype(np.uint8)
    return clip((Hs + 16) >> 5), clip((Vs + 16) >> 5), clip((Cs + 512) >> 10)


def test_fused_hpel_builder_matches_tiles():
    """inter.rs:1824-1868 (LCG64 0x5eed_f00d_dead_beef): fused == tiles == spec, 3 geometries."""
    st = Lcg64(0x5EED_F00D_DEAD_BEEF)
    for cw, ch, pad in [(64, 48, 16), (80, 64, 12), (176, 144, 32)]:
        ref = st.bytes(cw * ch).reshape(ch, cw).copy()
        f = O.pad_plane(ref, pad)
        h1, v1, c1 = O.hpel_tiles(f)
        h2, v2, c2 = O.hpel_fused(f)
        assert np.array_equal(h1, h2) and np.array_equal(v1, v2) and np.array_equal(c1, c2)
        h3, v3, c3 = np_hpel_planes(f)
        assert np.array_equal(h2, h3) and np.array_equal(v2, v3) and np.array_equal(c2, c3)


def test_hpel_block_matches_mc_luma():
    """inter.rs:1871-1911 (96x64, LCG32 0x9E37_79B9): plane reads == mc_luma (strided sample)."""
    st = Lcg32(0x9E37_79B9)
    cw, ch = 96, 64
    ref = np.array([(st.next() >> 24) & 0xFF for _ in range(cw * ch)], np.uint8).reshape(ch, cw)
    planes = O.build_planes4(ref, 32)
    src = ref.copy()
    checked = 0
    for bw, bh in [(16, 16), (16, 8), (8, 16), (8, 8), (8, 4), (4, 8), (4, 4)]:
        for fy in range(4):
            for fx in range(4):
                if fx == 0 and fy == 0:
                    continue
                for y0 in range(0, ch - bh, 21):
                    for x0 in range(0, cw - bw, 25):
                        for dx, dy in [(0, 0), (4, 0), (-4, -4), (8, 8), (-64, -64), (96, 40), (40, -96)]:
                            mvx, mvy = dx + fx, dy + fy
                            # mc_satd_hp takes the plane arms where they apply and mc_luma
                            # elsewhere; its SATD must equal SATD against mc_luma's block.
                            want = O.mc_luma(ref, x0, y0, bw, bh, mvx, mvy)
                            d = O.candidate_dist(src, ref, planes, 0, x0, y0, bw, bh, mvx, mvy)
                            assert d == np_satd_sum(src[y0:y0 + bh, x0:x0 + bw], want)
                            checked += 1
    assert checked > 2000


# ---------------------------------------------------------------------------
# reconstruction: dequantize + inverse 4x4 + add (transform.rs:233, 381;
# accel/src/transform_quant.rs:56-119)
# ---------------------------------------------------------------------------

NORM_ADJUST = [[10, 16, 13], [11, 18, 14], [13, 20, 16], [14, 23, 18], [16, 25, 20], [18, 29, 23]]
POS_GROUP_FLAT = [0, 2, 0, 2, 2, 1, 2, 1, 0, 2, 0, 2, 2, 1, 2, 1]


def np_dequant(levels, qp):
    """dequantize spelled out as transform.rs:233-284 writes it."""
    m, shift = qp % 6, qp // 6
    out = []
    for i, lv in enumerate(levels):
        ls = 16 * NORM_ADJUST[m][POS_GROUP_FLAT[i]]
        out.append((lv * ls) << (shift - 4) if qp >= 24 else (lv * ls + (1 << (3 - shift))) >> (4 - shift))
    return out


def np_inv_1d(d0, d1, d2, d3):
    e0, e1, e2, e3 = d0 + d2, d0 - d2, (d1 >> 1) - d3, d1 + (d3 >> 1)
    return [e0 + e3, e1 + e2, e1 - e2, e0 - e3]


def np_inverse(coeffs, rows_first=True, norm=True):
    m = [list(coeffs[r * 4:r * 4 + 4]) for r in range(4)]
    def rows(m):
        return [np_inv_1d(*m[r]) for r in range(4)]
    def cols(m):
        t = [np_inv_1d(m[0][c], m[1][c], m[2][c], m[3][c]) for c in range(4)]
        return [[t[c][r] for c in range(4)] for r in range(4)]
    m = cols(rows(m)) if rows_first else rows(cols(m))
    flat = [v for row in m for v in row]
    return [(v + 32) >> 6 for v in flat] if norm else flat


def test_dequant_matches_the_reference_formula():
    """transform.rs:1064-1125 (dequant_4x4_matches_scalar): the xorshift32
    stream from 0x2f6e_1c37, 64 cases per qp with magnitudes 3, 11 and 15 bits
    and zero, every qp 0..51."""
    st = 0x2F6E1C37

    def rnd():
        nonlocal st
        st ^= (st << 13) & 0xFFFFFFFF
        st ^= st >> 17
        st ^= (st << 5) & 0xFFFFFFFF
        return st

    for qp in range(52):
        for case in range(64):
            lv = []
            for _ in range(16):
                r = rnd()
                mag = [r & 0x7, r & 0x7FF, r & 0x7FFF, 0][case % 4]
                lv.append(-mag if r & 0x80000000 else mag)
            assert list(O.dequant4x4(lv, qp)) == np_dequant(lv, qp), (qp, case)


def test_inverse_core_is_row_first():
    """transform.rs:1268-1331: this block tells the two orders apart, and the
    inverse transform is rows first."""
    coeffs = [9, 2, -1, 2, -2, 2, -2, 1, -1, -2, 3, 5, -1, -1, -5, 3]
    assert np_inverse(coeffs, True, False) != np_inverse(coeffs, False, False)
    assert list(O.inverse_core4(coeffs)) == np_inverse(coeffs, True)
    # scaled up, the order shows in the normalized output too
    rng = np.random.default_rng(5)
    differ = 0
    for _ in range(500):
        c = [int(v) for v in rng.integers(-3000, 3000, 16)]
        want = np_inverse(c, True)
        assert list(O.inverse_core4(c)) == want
        differ += want != np_inverse(c, False)
    assert differ > 0


def test_dc_only_inverse_is_flat():
    """transform.rs:341-356 (dequantize_dc4): a DC-only block inverts to the
    flat (f + 32) >> 6 at every position."""
    for f in (-4096, -65, 0, 31, 32, 64, 1000, 20000):
        assert list(O.inverse_core4([f] + [0] * 15)) == [(f + 32) >> 6] * 16


def test_idct_rec_matches_reference():
    """accel/src/transform_quant.rs:169-195 (idct_rec_matches_reference): the
    pred/dct patterns of 128 seeds through idct_four_t4_rec."""
    sub = [(0, 0), (4, 0), (0, 4), (4, 4)]
    for seed in range(128):
        pred = np.array([(i * 7 + seed * 3) & 0xFF for i in range(64)], np.uint8).reshape(8, 8)
        dct = np.array([((i * 53 + seed * 29) % 4096) - 2048 for i in range(64)], np.int16)
        got = O.idct_four_t4_rec(pred, dct)
        for k, (ox, oy) in enumerate(sub):
            m = np_inverse([int(v) for v in dct[k * 16:k * 16 + 16]], True)
            for dy in range(4):
                for dx in range(4):
                    want = min(255, max(0, int(pred[oy + dy, ox + dx]) + m[dy * 4 + dx]))
                    assert got[oy + dy, ox + dx] == want, (seed, k)


# ---------------------------------------------------------------------------
# chroma: mc_chroma (inter.rs:1268), chroma_qp (predict.rs:64), the 2x2 DC
# (transform.rs:1017-1050)
# ---------------------------------------------------------------------------

def test_chroma_known_answers():
    """predict.rs:868-872 (chroma_qp_mapping), inter.rs:2066-2080
    (mc_chroma_zero_mv_copies, mc_chroma_bilinear_midpoint)."""
    assert (O.chroma_qp(20), O.chroma_qp(30), O.chroma_qp(51)) == (20, 29, 39)
    r = np.array([0, 1, 2, 3, 10, 11, 12, 13, 20, 21, 22, 23, 30, 31, 32, 33], np.uint8).reshape(4, 4)
    assert list(O.mc_chroma(r, 1, 1, 2, 2, 0, 0).ravel()) == [11, 12, 21, 22]
    assert int(O.mc_chroma(np.array([[0, 8], [0, 8]], np.uint8), 0, 0, 1, 1, 4, 0)[0, 0]) == 4


def test_mc_chroma_matches_per_pixel():
    """inter.rs:1952-1990 (mc_chroma_block_matches_per_pixel): the LCG
    reference picture (state 0xabcd_1234, x·1664525 + 1013904223, top byte),
    four block sizes at three positions, every MV in -12..12."""
    cw, ch = 24, 20
    st = 0xABCD1234
    ref = []
    for _ in range(cw * ch):
        st = (st * 1664525 + 1013904223) & 0xFFFFFFFF
        ref.append(st >> 24)
    ref = np.array(ref, np.uint8).reshape(ch, cw)

    def at(x, y):
        return int(ref[min(max(y, 0), ch - 1), min(max(x, 0), cw - 1)])

    for bw, bh in [(8, 8), (4, 4), (8, 4), (4, 8)]:
        for x0, y0 in [(4, 4), (0, 0), (cw - bw, ch - bh)]:
            for mvx in range(-12, 13):
                for mvy in range(-12, 13, 5):
                    got = O.mc_chroma(ref, x0, y0, bw, bh, mvx, mvy)
                    ix0, iy0, fx, fy = x0 + (mvx >> 3), y0 + (mvy >> 3), mvx & 7, mvy & 7
                    for dy in range(bh):
                        for dx in range(bw):
                            x, y = ix0 + dx, iy0 + dy
                            v = ((8 - fx) * (8 - fy) * at(x, y) + fx * (8 - fy) * at(x + 1, y) +
                                 (8 - fx) * fy * at(x, y + 1) + fx * fy * at(x + 1, y + 1) + 32) >> 6
                            assert got[dy, dx] == v, (bw, bh, x0, y0, mvx, mvy)


def test_chroma_dc_end_to_end_flat_block():
    """transform.rs:1402-1420: a flat chroma DC block survives the 2x2 forward
    quant, the inverse and the 4x4 inverse within 1 + 2^(qp/6)."""
    for r in (4, -6, 11):
        for qp in (0, 18, 30):
            lv, rd = O.chroma_dc_quant([16 * r] * 4, qp, intra=True)
            tol = 1 + (1 << (qp // 6))
            for d in rd:
                for v in O.inverse_core4([int(d)] + [0] * 15):
                    assert abs(int(v) - r) <= tol, (r, qp)


# ---------------------------------------------------------------------------
# in-loop deblocking (deblock.rs) of plain-ME pictures
# ---------------------------------------------------------------------------

def test_deblock_tables_match_reference():
    """ALPHA, BETA and TC0 as extracted from the reference's deblock.rs."""
    g = GOLD["deblock"]
    a, b, t = O.deblock_tables()
    assert list(a) == g["alpha"]["values"] and list(b) == g["beta"]["values"] and t.tolist() == g["tc0"]["rows"]


def _plain_picks(nmb, mv=(0, 0)):
    p = np.zeros((nmb, 6), np.int32)
    p[:, 1], p[:, 2], p[:, 3], p[:, 4] = mv[0], mv[1], mv[0], mv[1]
    return p


def test_deblock_leaves_flat_and_unfiltered_pictures():
    """A flat picture has nothing to smooth; a picture with no coefficients
    and one MV everywhere has bS 0 on every edge."""
    rng = np.random.default_rng(2)
    nmb = 6 * 4
    flat = np.full((64, 96), 77, np.uint8)
    co = np.zeros((nmb, 256), np.int16)
    co[::3, 5] = 7
    y, u, v = O.deblock_frame(flat, flat[:32, :48], flat[:32, :48], _plain_picks(nmb), co, 30)
    assert (y == 77).all() and (u == 77).all() and (v == 77).all()
    tex = rng.integers(0, 256, (64, 96)).astype(np.uint8)
    y, _, _ = O.deblock_frame(tex, None, None, _plain_picks(nmb, (8, -4)), np.zeros((nmb, 256), np.int16), 40)
    assert np.array_equal(y, tex)


def np_luma_line(line, bs, alpha, beta, tc0):
    """filter_luma_line (deblock.rs:67-115) on p3 p2 p1 p0 q0 q1 q2 q3."""
    p3, p2, p1, p0, q0, q1, q2, q3 = (int(v) for v in line)
    out = list(line)
    clip1 = lambda v: min(255, max(0, v))
    clip3 = lambda lo, hi, v: min(hi, max(lo, v))
    if abs(p0 - q0) >= alpha or abs(p1 - p0) >= beta or abs(q1 - q0) >= beta:
        return out
    ap, aq = abs(p2 - p0), abs(q2 - q0)
    tc = tc0 + (ap < beta) + (aq < beta)
    delta = clip3(-tc, tc, (((q0 - p0) << 2) + (p1 - q1) + 4) >> 3)
    out[3], out[4] = clip1(p0 + delta), clip1(q0 - delta)
    if ap < beta:
        out[2] = clip1(p1 + clip3(-tc0, tc0, (p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1))
    if aq < beta:
        out[5] = clip1(q1 + clip3(-tc0, tc0, (q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1))
    return out


def test_deblock_single_mb_edge_matches_line_filter():
    """Two MBs side by side, coefficients only in the right MB's first block
    column: bS 2 on the MB edge's rows of that block and on its internal edge,
    0 elsewhere.  Each filtered line equals filter_luma_line restated here."""
    rng = np.random.default_rng(8)
    base = rng.integers(90, 110, (16, 32)).astype(np.int32)
    base[:, 16:] += 12  # a step at the MB edge
    y = base.astype(np.uint8)
    co = np.zeros((2, 256), np.int16)
    co[1, 0] = 3  # MB 1, region 0, sub-block 0: block (0, 0)
    qp = 36
    a, b, t = O.deblock_tables()
    got, _, _ = O.deblock_frame(y, None, None, _plain_picks(2), co, qp)
    want = y.astype(np.int32).copy()
    # vertical MB edge x=16, rows 0..3 (block row 0) bS 2; internal edge x=20 rows 0..3 bS 2
    for x in (16, 20):
        for r in range(4):
            want[r, x - 4:x + 4] = np_luma_line(want[r, x - 4:x + 4], 2, a[qp], b[qp], t[qp][1])
    # horizontal internal edge y=4 at columns 16..19 (block (0,0) above block (0,1)) bS 2
    for c in range(16, 20):
        want[0:8, c] = np_luma_line(want[0:8, c], 2, a[qp], b[qp], t[qp][1])
    assert np.array_equal(got.astype(np.int32), want)


def _lcg32_bytes(seed: int, n: int) -> np.ndarray:
    """n draws (s >> 24) of the LCG s <- s*1664525 + 1013904223 mod 2^32,
    computed 4096 at a time from the jump-ahead multipliers (same stream as
    stepping Lcg32 n times)."""
    a, c, blk = 1664525, 1013904223, 4096
    mul = np.empty(blk, np.uint64)
    add = np.empty(blk, np.uint64)
    m, k = 1, 0
    for i in range(blk):  # state_{i+1} = mul[i] * state_0 + add[i]
        m, k = (m * a) & 0xFFFFFFFF, (k * a + c) & 0xFFFFFFFF
        mul[i], add[i] = m, k
    out = np.empty(n, np.uint8)
    st = seed & 0xFFFFFFFF
    for o in range(0, n, blk):
        v = (mul * np.uint64(st) + add) & np.uint64(0xFFFFFFFF)
        take = min(blk, n - o)
        out[o:o + take] = (v[:take] >> np.uint64(24)).astype(np.uint8)
        st = int(v[-1])
    return out


def test_lcg32_jump_ahead_matches_stepping():
    st = Lcg32(0xDEAD_BEEF)
    want = np.array([st.next() >> 24 for _ in range(5000)], np.uint8)
    assert np.array_equal(_lcg32_bytes(0xDEAD_BEEF, 5000), want)


def test_coded_plane_extension_matches_per_pixel():
    """mb16.rs:1552-1584 (clamp_plane_matches_per_pixel_oracle, its LCG
    0xDEAD_BEEF stream and seven geometries): the coded-size edge extension the
    tests and the benchmark apply to every frame (rusty_h264_b200.synth.
    coded_luma, restating clamp_plane mb16.rs:1523) equals the per-pixel
    definition out[y][x] = plane[min(y, h-1)][min(x, w-1)]."""
    from rusty_h264_b200 import synth

    cases = [(1920, 1080, 1920, 1088), (960, 540, 960, 544), (352, 288, 352, 288), (100, 100, 112, 112),
             (37, 5, 48, 16), (16, 1, 16, 16), (1, 1, 16, 16)]
    stream = _lcg32_bytes(0xDEAD_BEEF, sum(w * h for w, h, _, _ in cases))
    o = 0
    for w, h, ow, oh in cases:
        plane = stream[o:o + w * h].reshape(h, w)
        o += w * h
        got = synth.coded_luma(plane)
        want = plane[np.minimum(np.arange(oh), h - 1)[:, None], np.minimum(np.arange(ow), w - 1)[None, :]]
        assert got.shape == (oh, ow) and np.array_equal(got, want), (w, h, ow, oh)


# ---------------------------------------------------------------------------
# mb-tree lookahead (mbtree.rs:61-263), restated independently of the C oracle
# ---------------------------------------------------------------------------

def np_downsample2x(y):
    """downsample2x (mbtree.rs:61-74): (sum of each 2x2 + 2) / 4."""
    s = y[0::2, 0::2].astype(np.int64) + y[0::2, 1::2] + y[1::2, 0::2] + y[1::2, 1::2]
    return ((s + 2) // 4).astype(np.uint8)


def np_intra_cost(pic, bx0, by0, bs):
    """intra_cost (mbtree.rs:78-93): the 4x4 Hadamard magnitudes of the block
    without each DC term (the block sum), at least 1."""
    tot = 0
    for by in range(by0, by0 + bs, 4):
        for bx in range(bx0, bx0 + bs, 4):
            h = H4 @ pic[by:by + 4, bx:bx + 4].astype(np.int64) @ H4.T
            tot += int(np.abs(h).sum() - abs(h[0, 0]))
    return max(min(tot, 2**31 - 1), 1)


def np_mc_satd(cur, ref, bx0, by0, bs, mv):
    """mc_satd (mbtree.rs:102-147): SATD of the block against the reference at
    a quarter-pel MV, every read clamped (the in-place and mc_luma arms agree)."""
    pred = np_luma_sample_block(ref, bx0, by0, bs, bs, mv[0], mv[1])
    return np_satd_sum(cur[by0:by0 + bs, bx0:bx0 + bs], pred)


def np_inter_cost(cur, ref, bx0, by0, bs, seed, max_step):
    """inter_cost (mbtree.rs:154-197): (0,0), the seed when nonzero, then the
    four-point diamond (+x, -x, +y, -y, each around the centre as it moves) at
    steps max_step .. 1, a step repeated while it moves; 0 at (0,0) ends it."""
    best_mv = (0, 0)
    best = np_mc_satd(cur, ref, bx0, by0, bs, best_mv)
    if best == 0:
        return 0, best_mv
    if seed != (0, 0):
        c = np_mc_satd(cur, ref, bx0, by0, bs, seed)
        if c < best:
            best, best_mv = c, seed
    step = max_step
    while step >= 1:
        while True:
            moved = False
            for dx, dy in ((step, 0), (-step, 0), (0, step), (0, -step)):
                mv = (best_mv[0] + dx * 4, best_mv[1] + dy * 4)
                c = np_mc_satd(cur, ref, bx0, by0, bs, mv)
                if c < best:
                    best, best_mv, moved = c, mv, True
            if not moved:
                break
        step >>= 1
    return min(best, 2**31 - 1), best_mv


def np_lookahead_clip(frames, mode):
    """frame_costs (mbtree.rs:208-263) of every frame against the previous one
    (frame 0 intra only): raster order, seed = left MV, else top MV; HalfRes
    searches and scores at half resolution, Hybrid refines at full resolution
    from the half-res MV.  Halving the seed truncates toward zero, as Rust's /."""
    n, ch, cw = frames.shape
    mb_w, mb_h = cw // 16, ch // 16
    half = np.stack([np_downsample2x(f) for f in frames])
    halve = lambda v: int(v / 2)
    intra = np.zeros((n, mb_w * mb_h), np.int32)
    inter = np.zeros_like(intra)
    mvs = np.zeros((n, mb_w * mb_h, 2), np.int32)
    for f in range(n):
        for m in range(mb_w * mb_h):
            mbx, mby = m % mb_w, m // mb_w
            seed = tuple(mvs[f, m - 1]) if mbx > 0 else (tuple(mvs[f, m - mb_w]) if mby > 0 else (0, 0))
            seed = (int(seed[0]), int(seed[1]))
            ic = np_intra_cost(half[f], mbx * 8, mby * 8, 8) if mode == 2 else np_intra_cost(frames[f], mbx * 16, mby * 16, 16)
            if f == 0:
                cost, mv = ic, (0, 0)
            elif mode == 0:
                c, mv = np_inter_cost(frames[f], frames[f - 1], mbx * 16, mby * 16, 16, seed, 8)
                cost = min(c, ic)
            elif mode == 2:
                c, mvp = np_inter_cost(half[f], half[f - 1], mbx * 8, mby * 8, 8, (halve(seed[0]), halve(seed[1])), 8)
                cost, mv = min(c, ic), (mvp[0] * 2, mvp[1] * 2)
            else:
                _, mvp = np_inter_cost(half[f], half[f - 1], mbx * 8, mby * 8, 8, (halve(seed[0]), halve(seed[1])), 8)
                c, mv = np_inter_cost(frames[f], frames[f - 1], mbx * 16, mby * 16, 16, (mvp[0] * 2, mvp[1] * 2), 2)
                cost = min(c, ic)
            intra[f, m], inter[f, m], mvs[f, m] = ic, cost, mv
    return intra, inter, mvs


def _panning_clip(n, cw, ch, pan, seed):
    rng = np.random.default_rng(seed)
    H, W = ch + abs(pan[1]) * n + 16, cw + abs(pan[0]) * n + 16
    tex = rng.random((H, W))
    for _ in range(3):
        tex = (tex + np.roll(tex, 1, 0) + np.roll(tex, 1, 1) + np.roll(tex, (1, 1), (0, 1))) / 4
    tex = (255 * (tex - tex.min()) / (tex.max() - tex.min())).astype(np.uint8)
    oy, ox = abs(pan[1]) * n // 2 + 8, abs(pan[0]) * n // 2 + 8
    return np.ascontiguousarray(np.stack([tex[oy + k * pan[1]:oy + k * pan[1] + ch, ox + k * pan[0]:ox + k * pan[0] + cw]
                                          for k in range(n)]))


def test_downsample2x_matches_numpy():
    rng = np.random.default_rng(1)
    for cw, ch in ((32, 16), (96, 48), (352, 288)):
        y = rng.integers(0, 256, (ch, cw)).astype(np.uint8)
        assert np.array_equal(O.downsample2x(y), np_downsample2x(y))


@pytest.mark.parametrize("mode", [2, 1, 0])
def test_lookahead_oracle_matches_numpy_restatement(mode):
    """The C oracle's frame_costs against the independent numpy/Python
    restatement above, on a synthetic clip (moving boxes over noise) and a
    panning texture that moves the diamond several steps, in all three modes."""
    from rusty_h264_b200 import synth

    y, _, _ = synth.cif_clip(3, 11, 96, 64)
    for clip in (synth.coded_luma(y), _panning_clip(3, 96, 64, (7, -3), 5)):
        got = O.lookahead_clip(clip, mode)
        want = np_lookahead_clip(clip, mode)
        for g, w, name in zip(got, want, ("intra", "inter", "mvs")):
            assert np.array_equal(g, w), (mode, name)


# ---------------------------------------------------------------------------
# plain-ME of a frame (motion_search + best_part + the split decision), Balanced
# preset, restated independently of the C oracle from mb16.rs / inter.rs
# ---------------------------------------------------------------------------

def np_mvbits(d):
    """mvbits kind 0 (mb16.rs:2454-2482): the se(v) Exp-Golomb length of d."""
    code = 2 * d - 1 if d > 0 else -2 * d
    return 1 + 2 * ((code + 1).bit_length() - 1)


def np_motion_search(src, ref, lx, ly, rw, rh, preds, lam, start=None):
    """motion_search (mb16.rs:2433-3302) under the Balanced preset: seeds (0,0)
    then the predictors, the centre snapped to full-pel, the ladder of 4-point
    diamonds at 16, 8, 4 quarter-pel (fixed-centre argmin where the +-step box
    is inside the picture, first-improvement cascade otherwise, a rung walked
    while it moves), one pass of the 8-point half-pel then quarter-pel rings
    (each point around the centre as it moves), and the pre-snap seed kept if
    cheaper.  Distortion: the exact 4x4 Hadamard SATD against the clamped
    luma_sample prediction; rate: (lambda * bits) truncated.  With a start
    vector (mb16.rs:2445) the search prices only it, skips the snap and the
    diamond ladder, and refines it with the sub-pel rings."""
    ch, cw = src.shape
    center = preds[0]
    memo = {}

    def cost(mv):
        if mv not in memo:
            pred = np_luma_sample_block(ref, lx, ly, rw, rh, mv[0], mv[1])
            rate = np_mvbits(mv[0] - center[0]) + np_mvbits(mv[1] - center[1])
            memo[mv] = np_satd_sum(src[ly:ly + rh, lx:lx + rw], pred) + int(lam * rate)
        return memo[mv]

    if start is not None:
        best, best_c = start, cost(start)
    else:
        best, best_c = (0, 0), cost((0, 0))
        for p in preds:
            if cost(p) < best_c:
                best, best_c = p, cost(p)
    seed_mv, seed_c = best, best_c
    if start is None and (best[0] & 3 or best[1] & 3):
        best = (((best[0] + 2) // 4) * 4, ((best[1] + 2) // 4) * 4)
        best_c = cost(best)
    for step in ((16, 8, 4) if start is None else ()):
        ring = ((step, 0), (-step, 0), (0, step), (0, -step))
        while True:
            s = step >> 2
            bx, by = lx + (best[0] >> 2), ly + (best[1] >> 2)
            if (best[0] & 3) == 0 and (best[1] & 3) == 0 and bx - s >= 0 and by - s >= 0 and \
                    bx + s + rw <= cw and by + s + rh <= ch:
                bi, bc = None, best_c
                for d in ring:
                    c = cost((best[0] + d[0], best[1] + d[1]))
                    if c < bc:
                        bi, bc = d, c
                if bi is None:
                    break
                best, best_c = (best[0] + bi[0], best[1] + bi[1]), bc
                continue
            moved = False
            for d in ring:
                mv = (best[0] + d[0], best[1] + d[1])
                if cost(mv) < best_c:
                    best, best_c, moved = mv, cost(mv), True
            if not moved:
                break
    for step in (2, 1):
        for d in ((step, 0), (-step, 0), (0, step), (0, -step), (step, step), (-step, -step), (step, -step),
                  (-step, step)):
            mv = (best[0] + d[0], best[1] + d[1])
            if cost(mv) < best_c:
                best, best_c = mv, cost(mv)
    if seed_c < best_c:
        best, best_c = seed_mv, seed_c
    return best, best_c


def np_predict_mv(a, b, c):
    """predict_mv (inter.rs:36-69) for ref 0 with neighbours None (unavailable)
    or their MVs (every coded neighbour refers to ref 0)."""
    (mva, ra), (mvb, rb), (mvc, rc) = ((n, 0) if n is not None else ((0, 0), -1) for n in (a, b, c))
    if b is None and c is None and a is not None:
        mvb, rb, mvc, rc = mva, ra, mva, ra
    if (ra == 0) + (rb == 0) + (rc == 0) == 1:
        return mva if ra == 0 else (mvb if rb == 0 else mvc)
    med = lambda x, y, z: sorted((x, y, z))[1]
    return (med(mva[0], mvb[0], mvc[0]), med(mva[1], mvb[1], mvc[1]))


def np_learned_16x16(src, ref, lx, ly, pmv, props, prop_t, lam):
    """The learned-proposal 16x16 search (no counterpart in the reference):
    the predictor and the 8 proposals priced with the search's cost; if the
    cheapest proposal's SATD exceeds the predictor's by more than prop_t, the
    plain search, else motion_search from the cheapest of the nine (the
    predictor first on ties).  Returns (mv, J, fell back)."""
    cands = [tuple(pmv)] + [(int(props[2 * i]), int(props[2 * i + 1])) for i in range(8)]
    dist, cost = [], []
    for mv in cands:
        pred = np_luma_sample_block(ref, lx, ly, 16, 16, mv[0], mv[1])
        d = np_satd_sum(src[ly:ly + 16, lx:lx + 16], pred)
        dist.append(d)
        cost.append(d + int(lam * (np_mvbits(mv[0] - pmv[0]) + np_mvbits(mv[1] - pmv[1]))))
    bp = 1 + int(np.argmin(cost[1:]))
    if dist[bp] > dist[0] + prop_t:
        mv, c = np_motion_search(src, ref, lx, ly, 16, 16, [tuple(pmv)], lam)
        return mv, c, True
    mv, c = np_motion_search(src, ref, lx, ly, 16, 16, [tuple(pmv)], lam, start=cands[int(np.argmin(cost))])
    return mv, c, False


def np_me_frame(src, ref, lam, gate, props=None, prop_t=0):
    """The plain-ME frame model: every MB in raster order coded inter with ref
    0; the neighbours of its top-left 4x4 block (mv_neighbors_block,
    mb16.rs:1871: left, top, top-right else top-left) give predict_mv;
    best_part 16x16 seeded [pmv], and when its J exceeds the gate the 16x8 and
    8x16 halves seeded [pmv, mv16], the shape taken on strictly lower summed J
    (mb16.rs:8869-8913).  With props (16 i32 per MB) the 16x16 search is
    np_learned_16x16, and the halves of an MB that took a proposal search
    refine-only from mv16; the fallback flags are returned as a third array."""
    ch, cw = src.shape
    mb_w, mb_h = cw // 16, ch // 16
    picks = np.zeros((mb_w * mb_h, 6), np.int32)
    costs = np.zeros((mb_w * mb_h, 2), np.int64)
    blk = {}  # (bx4, by4) -> MV of coded 4x4 blocks
    fell = np.zeros(mb_w * mb_h, np.int32)

    def get(bx, by):
        return blk.get((bx, by)) if 0 <= bx < mb_w * 4 and 0 <= by < mb_h * 4 else None

    for m in range(mb_w * mb_h):
        mbx, mby = m % mb_w, m // mb_w
        lx, ly, bx, by = mbx * 16, mby * 16, mbx * 4, mby * 4
        c = get(bx + 4, by - 1)
        pmv = np_predict_mv(get(bx - 1, by), get(bx, by - 1), c if c is not None else get(bx - 1, by - 1))
        if props is None:
            mv16, c16 = np_motion_search(src, ref, lx, ly, 16, 16, [pmv], lam)
        else:
            mv16, c16, fb = np_learned_16x16(src, ref, lx, ly, pmv, props[m], prop_t, lam)
            fell[m] = fb
        shape, mv0, mv1, best = 0, mv16, mv16, c16
        if gate >= 0 and c16 > gate:
            seeds = [pmv, mv16]
            # the learned search's partitions, when its 16x16 search took a
            # proposal: refine-only from the 16x16 MV
            st = mv16 if props is not None and not fell[m] else None
            (mt, ct), (mb_, cb) = (np_motion_search(src, ref, lx, ly + o, 16, 8, seeds, lam, start=st) for o in (0, 8))
            (ml, cl), (mr, cr) = (np_motion_search(src, ref, lx + o, ly, 8, 16, seeds, lam, start=st) for o in (0, 8))
            if ct + cb < best:
                shape, mv0, mv1, best = 1, mt, mb_, ct + cb
            if cl + cr < best:
                shape, mv0, mv1, best = 2, ml, mr, cl + cr
        picks[m, :5] = (shape, mv0[0], mv0[1], mv1[0], mv1[1])
        costs[m] = (best, c16)
        for j in range(4):
            for i in range(4):
                part = (j >= 2) if shape == 1 else ((i >= 2) if shape == 2 else 0)
                blk[(bx + i, by + j)] = mv1 if part else mv0
    return (picks, costs) if props is None else (picks, costs, fell)


@pytest.mark.parametrize("gate_on", [False, True])
def test_me_frame_oracle_matches_numpy_restatement(gate_on):
    """The C oracle's plain-ME frame (or_me_frame_plain) against the
    independent restatement above, Balanced preset, on a 96x64 crop of the
    CIF clip and on a panning texture, with and without the partition split."""
    from rusty_h264_b200 import synth
    from rusty_h264_b200 import accel as A

    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    qstep16 = (10, 11, 13, 14, 16, 18)[qp % 6] << (qp // 6)
    gate = ((30 * (qstep16 + 160)) >> 3) * 2 if gate_on else -1
    assert not gate_on or gate == A.split_gate_for_qp(qp)
    y, _, _ = synth.cif_clip(3, 7)
    crop = np.ascontiguousarray(synth.coded_luma(y)[:, 96:160, 128:224])
    for frames in (crop, _panning_clip(2, 96, 64, (5, -3), 9)):
        src, ref = frames[1], frames[0]
        wp, wc = O.me_frame(src, ref, O.build_planes4(ref, 32), O.balanced_params(), lam, gate)
        gp, gc = np_me_frame(src, ref, lam, gate)
        assert np.array_equal(wp[:, :5], gp[:, :5]), np.argwhere(wp[:, :5] != gp[:, :5])[:4]
        assert np.array_equal(wc, gc)


@pytest.mark.parametrize("prop_t", [0, 40, 1 << 30])
def test_learned_me_frame_oracle_matches_numpy_restatement(prop_t):
    """The C oracle's learned-proposal frame (or_me_frame_learned) against the
    restatement above: proposals scattered around the true motion of a
    panning texture (some exact, some off by a few pixels, some far), with
    the split gate on, at thresholds that make every MB, some MBs and no MB
    fall back."""
    from rusty_h264_b200 import accel as A

    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    frames = _panning_clip(2, 96, 64, (5, -3), 11)
    src, ref = frames[1], frames[0]
    nmb = 6 * 4
    rng = np.random.default_rng(prop_t % 997)
    props = np.zeros((nmb, 16), np.int32)
    for m in range(nmb):
        for i in range(8):
            k = rng.integers(0, 3)
            off = (0, 0) if k == 0 else (tuple(rng.integers(-3, 4, 2)) if k == 1 else tuple(rng.integers(-8, 9, 2)))
            props[m, 2 * i] = 4 * (-5 + off[0])
            props[m, 2 * i + 1] = 4 * (3 + off[1])
    wp, wc, wf = O.me_frame_learned(src, ref, O.build_planes4(ref, 32), O.balanced_params(), lam, props, prop_t, gate)
    gp, gc, gf = np_me_frame(src, ref, lam, gate, props, prop_t)
    assert np.array_equal(wf, gf)
    assert np.array_equal(wp[:, :5], gp[:, :5]), np.argwhere(wp[:, :5] != gp[:, :5])[:4]
    assert np.array_equal(wc, gc)
    if prop_t >= 1 << 30:
        assert not wf.any()


# ---------------------------------------------------------------------------
# MC + luma T/Q of picked MBs (mb16.rs:3436-3450), restated independently
# ---------------------------------------------------------------------------

# H.264 forward quantization multipliers per qp % 6 for the (even,even),
# (odd,odd) and mixed positions (transform.rs QUANT_MF).
QUANT_MF_STD = [[13107, 5243, 8066], [11916, 4660, 7490], [10082, 4194, 6554], [9362, 3647, 5825],
                [8192, 3355, 5243], [7282, 2893, 4559]]


def np_quant_dz_ff(qp, dz):
    """quant_dz_ff (transform.rs:144-156): round(F / MF) per openh264 slot, with
    F = 2^(15 + qp/6) / dz and slots in groups (0,2,0,2,2,1,2,1)."""
    f = (1 << (15 + qp // 6)) // dz
    return [(f + QUANT_MF_STD[qp % 6][g] // 2) // QUANT_MF_STD[qp % 6][g] for g in (0, 2, 0, 2, 2, 1, 2, 1)]


def np_mc_tq_frame(src, ref, picks, qp, dz=6):
    """Per MB: the prediction of each 4x4 block under its partition's MV
    (luma_sample), the 4x4 forward core Cf.d.Cf^T of each sub-block in the
    dct[256] order (quadrants (0,0),(8,0),(0,8),(8,8), sub-blocks
    (0,0),(4,0),(0,4),(4,4)), then ((|c| + FF[pos]) * MF[pos]) >> 16 with the
    sign, pos = (row & 1) * 4 + col, MF = QUANT_MF_OH[qp]."""
    ch, cw = src.shape
    mb_w = cw // 16
    ff = np.array(np_quant_dz_ff(qp, dz), np.int64)
    mf = np.array(GOLD["quant_mf_oh"]["rows"][qp], np.int64)
    pos = np.array([((i // 4) & 1) * 4 + i % 4 for i in range(16)])
    out = np.zeros((len(picks), 256), np.int16)
    for m, (shape, m0x, m0y, m1x, m1y) in enumerate(picks[:, :5]):
        lx, ly = (m % mb_w) * 16, (m // mb_w) * 16
        pred = np.zeros((16, 16), np.int64)
        for by in range(0, 16, 4):
            for bx in range(0, 16, 4):
                part = (by >= 8) if shape == 1 else ((bx >= 8) if shape == 2 else False)
                mvx, mvy = (m1x, m1y) if part else (m0x, m0y)
                pred[by:by + 4, bx:bx + 4] = np_luma_sample_block(ref, lx + bx, ly + by, 4, 4, int(mvx), int(mvy))
        d = src[ly:ly + 16, lx:lx + 16].astype(np.int64) - pred
        for qi, (qx, qy) in enumerate(((0, 0), (8, 0), (0, 8), (8, 8))):
            for k, (ox, oy) in enumerate(((0, 0), (4, 0), (0, 4), (4, 4))):
                c = (CF @ d[qy + oy:qy + oy + 4, qx + ox:qx + ox + 4] @ CF.T).reshape(16)
                lvl = ((np.abs(c) + ff[pos]) * mf[pos]) >> 16
                out[m, qi * 64 + k * 16:qi * 64 + k * 16 + 16] = np.where(c < 0, -lvl, lvl)
    return out


@pytest.mark.parametrize("qp", [0, 20, 27, 51])
def test_mc_tq_oracle_matches_numpy_restatement(qp):
    """The C oracle's MC + luma T/Q of picked MBs against the restatement above,
    on the panning texture's plain-ME picks (16x16, 16x8 and 8x16, sub-pel MVs)
    and on picks forced through every shape with far and fractional MVs."""
    from rusty_h264_b200 import accel as A

    frames = _panning_clip(2, 96, 64, (5, -3), 9)
    src, ref = frames[1], frames[0]
    lam = float(np.sqrt(A.frame_lambda(27)) * 1.25)
    picks, _ = O.me_frame(src, ref, O.build_planes4(ref, 32), O.balanced_params(), lam, A.split_gate_for_qp(27))
    rng = np.random.default_rng(qp)
    forced = picks.copy()
    forced[:, 0] = np.arange(len(forced)) % 3
    forced[:, 1:5] = rng.integers(-160, 161, (len(forced), 4))
    for p in (picks, forced):
        assert np.array_equal(O.mc_tq_frame(src, ref, p, qp, 6), np_mc_tq_frame(src, ref, p, qp)), qp


# ---------------------------------------------------------------------------
# best_part over several references (mb16.rs:4921-4960)
# ---------------------------------------------------------------------------

def test_multiref_oracle_one_reference_is_plain_me():
    """With one reference the multi-reference frame model is plain-ME: the
    same shapes, MVs and costs, every reference index 0."""
    from rusty_h264_b200 import accel as A
    from rusty_h264_b200 import synth

    y, _, _ = synth.cif_clip(3, 5)
    c = synth.coded_luma(y)
    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    gate = A.split_gate_for_qp(qp)
    pl = O.build_planes4(c[1], 32)
    mp, mc = O.me_frame_multiref(c[2], c[1:2], pl[None], O.balanced_params(), lam, gate)
    wp, wc = O.me_frame(c[2], c[1], pl, O.balanced_params(), lam, gate)
    assert np.array_equal(mp[:, [0, 2, 3, 5, 6]], wp[:, :5]) and np.array_equal(mc, wc)
    assert not mp[:, [1, 4]].any()


def test_multiref_oracle_identical_references_keep_the_nearest():
    """Three copies of one reference: every search finds the same MV on each,
    and ref_bits (te(v): ue(r) = 1, 3, 3 bits for r = 0, 1, 2, mb16.rs:5967)
    makes reference 0 the strictly cheapest, so every pick uses reference 0
    and its 16x16 cost is the single-reference one plus floor(lambda * 1)."""
    from rusty_h264_b200 import accel as A
    from rusty_h264_b200 import synth

    y, _, _ = synth.cif_clip(3, 6)
    c = synth.coded_luma(y)
    qp = 27
    lam = float(np.sqrt(A.frame_lambda(qp)) * 1.25)
    pl = O.build_planes4(c[1], 32)
    mp, mc = O.me_frame_multiref(c[2], np.stack([c[1]] * 3), np.stack([pl] * 3), O.balanced_params(), lam, -1)
    wp, wc = O.me_frame(c[2], c[1], pl, O.balanced_params(), lam, -1)
    assert not mp[:, [1, 4]].any()
    assert np.array_equal(mp[:, [2, 3]], wp[:, [1, 2]])
    assert np.array_equal(mc[:, 1], wc[:, 1] + int(lam * 1))
