// tq_device.cuh -- the forward 4x4 transform + quantisation of one block
// (dct_four_t4 + quant_four_4x4, crates/rusty_h264-accel/src/
// transform_quant.rs:71-135) and its quant tables, shared by the T/Q kernels
// and by the plain-ME kernel, which can run an MB's MC + T/Q right after its
// pick.
#pragma once

#include <climits>

#include "h264a_device.cuh"

namespace h264a {

struct QuantTables4 {
    int16_t ff[52][8];
    int16_t mf[52][8];
};

// QUANT_MF (transform.rs:25-32) and openh264's slot -> position group map.
static const int kQuantMf[6][3] = {{13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
                                   {9362, 3647, 5825},  {8192, 3355, 5243},  {7282, 2893, 4559}};
static const int kGroup8[8] = {0, 2, 0, 2, 2, 1, 2, 1};

// quant_dz_ff (transform.rs:145-159) and QUANT_MF_OH[qp] (transform.rs:1447):
// the openh264 table is round-half-up(MF << 16 >> qbits), qbits = 15 + qp/6.
// One QP's row: ff and mf by position slot (row & 1) * 4 + column.
static inline void make_quant_row4(int qp, int dz_div, int16_t ff[8], int16_t mf[8]) {
    const int m = qp % 6;
    const long long qbits = 15 + qp / 6;
    const long long f = (1LL << qbits) / dz_div;
    for (int i = 0; i < 8; i++) {
        const long long mfg = kQuantMf[m][kGroup8[i]];
        ff[i] = int16_t((f + mfg / 2) / mfg);
        const int sh = int(qbits) - 16;
        const long long r = sh < 0 ? mfg << 1 : (sh == 0 ? mfg : (mfg + (1LL << (sh - 1))) >> sh);
        mf[i] = int16_t(r);
    }
}

static inline QuantTables4 make_tables4(int dz_div) {
    QuantTables4 t;
    for (int qp = 0; qp < 52; qp++) make_quant_row4(qp, dz_div, t.ff[qp], t.mf[qp]);
    return t;
}

// fwd_1d + forward_core (transform.rs:72-119), rows then columns, in place.
__device__ __forceinline__ void forward_core4(int m[16]) {
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int x0 = m[r * 4], x1 = m[r * 4 + 1], x2 = m[r * 4 + 2], x3 = m[r * 4 + 3];
        const int t0 = x0 + x3, t1 = x1 + x2, t2 = x1 - x2, t3 = x0 - x3;
        m[r * 4] = t0 + t1; m[r * 4 + 1] = 2 * t3 + t2; m[r * 4 + 2] = t0 - t1; m[r * 4 + 3] = t3 - 2 * t2;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int x0 = m[c], x1 = m[4 + c], x2 = m[8 + c], x3 = m[12 + c];
        const int t0 = x0 + x3, t1 = x1 + x2, t2 = x1 - x2, t3 = x0 - x3;
        m[c] = t0 + t1; m[4 + c] = 2 * t3 + t2; m[8 + c] = t0 - t1; m[12 + c] = t3 - 2 * t2;
    }
}

// Residual -> dct_four_t4's i16 cast -> quant_four_4x4 (pos = (row&1)*4+col),
// written as 16 consecutive i16 (two 16-byte stores).
__device__ __forceinline__ void tq4x4_store(const uint32_t s[4], const uint32_t p[4], const int16_t* ff,
                                            const int16_t* mf, int16_t* out, int lv[16] = nullptr) {
    int m[16];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) m[r * 4 + c] = byte_of(s[r], c) - byte_of(p[r], c);
    forward_core4(m);
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 16; i += 2) {
        int v2[2];
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int idx = i + k;
            const int pos = ((idx >> 2) & 1) * 4 + (idx & 3);
            const int c = int(int16_t(m[idx]));
            const int lvl = ((abs(c) + int(ff[pos])) * int(mf[pos])) >> 16;
            v2[k] = int(int16_t(c < 0 ? -lvl : lvl));
            if (lv) lv[idx] = v2[k];
        }
        w[i >> 1] = (uint32_t(uint16_t(v2[0]))) | (uint32_t(uint16_t(v2[1])) << 16);
    }
    uint4* o = reinterpret_cast<uint4*>(out);
    o[0] = make_uint4(w[0], w[1], w[2], w[3]);
    o[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

// ---- reconstruction ------------------------------------------------------------

// 16 * NORM_ADJUST (transform.rs:15-22) by qp % 6 and position group (both
// even 0, both odd 1, else 2: POS_GROUP_FLAT, transform.rs:48-52).
static __constant__ int kLevelScale[6][3] = {{160, 256, 208}, {176, 288, 224}, {208, 320, 256},
                                      {224, 368, 288}, {256, 400, 320}, {288, 464, 368}};

// The inter MB's luma reconstruction of one 4x4 block (mb16.rs:3575-3605):
// dequantize (transform.rs:233-284, flat scaling) each level, cast it to i16
// as the reference does, inverse core transform rows then columns with
// (x + 32) >> 6 (transform_quant.rs:30-35, 56-69), add the prediction and
// clamp (idct_four_t4_rec, transform_quant.rs:96-119).  Four packed rows out.
// dc_override (the chroma DC from inverse_quant_chroma_dc) replaces the
// dequantized coefficient 0 when given.
__device__ __forceinline__ void rec4x4(const int lv[16], const uint32_t p[4], int qp, uint32_t out[4],
                                       int dc_override = INT_MIN) {
    const int m6 = qp % 6, shift = qp / 6;
    int m[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const int g = ((i >> 2) & 1) == (i & 1) ? ((i & 1) ? 1 : 0) : 2;
        const int ls = kLevelScale[m6][g];
        const int d = qp >= 24 ? int(uint32_t(lv[i] * ls) << (shift - 4)) : (lv[i] * ls + (1 << (3 - shift))) >> (4 - shift);
        m[i] = int(int16_t(d));
    }
    if (dc_override != INT_MIN) m[0] = int(int16_t(dc_override));
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int d0 = m[r * 4], d1 = m[r * 4 + 1], d2 = m[r * 4 + 2], d3 = m[r * 4 + 3];
        const int e0 = d0 + d2, e1 = d0 - d2, e2 = (d1 >> 1) - d3, e3 = d1 + (d3 >> 1);
        m[r * 4] = e0 + e3; m[r * 4 + 1] = e1 + e2; m[r * 4 + 2] = e1 - e2; m[r * 4 + 3] = e0 - e3;
    }
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int d0 = m[c], d1 = m[4 + c], d2 = m[8 + c], d3 = m[12 + c];
        const int e0 = d0 + d2, e1 = d0 - d2, e2 = (d1 >> 1) - d3, e3 = d1 + (d3 >> 1);
        m[c] = e0 + e3; m[4 + c] = e1 + e2; m[8 + c] = e1 - e2; m[12 + c] = e0 - e3;
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
        uint32_t w = 0;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int v = byte_of(p[r], c) + ((m[r * 4 + c] + 32) >> 6);
            w |= uint32_t(v < 0 ? 0 : (v > 255 ? 255 : v)) << (8 * c);
        }
        out[r] = w;
    }
}

// ---- the inter MB's chroma block --------------------------------------------

// QUANT_MF[m][0] (transform.rs:25-32), the chroma DC multiplier.
static __constant__ int kQuantMfDc[6] = {13107, 11916, 10082, 9362, 8192, 7282};

// Packed 4 pixels of one output row of mc_chroma (inter.rs:1268-1361):
// (wa·a + wb·b + wc·c + wd·d + 32) >> 6 over rows y, y+1 of the clamped
// reference, columns x..x+4.
__device__ __forceinline__ uint32_t chroma_row(const uint8_t* ref, int w, int h, int x, int y, int wa, int wb, int wc,
                                               int wd, bool cg = false) {
    const int ya = clampi(y, 0, h - 1), yb = clampi(y + 1, 0, h - 1);
    const uint8_t* ra = ref + (long long)ya * w;
    const uint8_t* rb = ref + (long long)yb * w;
    int a[5], b[5];
    if (x >= 0 && x + 5 <= w) {
        const uint32_t a0 = cg ? ld4u_cg(ra + x) : ld4u(ra + x), b0 = cg ? ld4u_cg(rb + x) : ld4u(rb + x);
#pragma unroll
        for (int k = 0; k < 4; k++) { a[k] = byte_of(a0, k); b[k] = byte_of(b0, k); }
        a[4] = ldb(ra + x + 4, cg);
        b[4] = ldb(rb + x + 4, cg);
    } else {
#pragma unroll
        for (int k = 0; k < 5; k++) {
            const int xx = clampi(x + k, 0, w - 1);
            a[k] = ldb(ra + xx, cg);
            b[k] = ldb(rb + xx, cg);
        }
    }
    uint32_t o = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) o |= uint32_t((wa * a[k] + wb * a[k + 1] + wc * b[k] + wd * b[k + 1] + 32) >> 6) << (8 * k);
    return o;
}

// Chroma 4x4 block k (SUBBLOCKS order (0,0),(4,0),(0,4),(4,4)) of one plane
// of an inter MB, at chroma sample (x, y), predicted with the partition's
// luma MV: mb16.rs:3408-3428 (chroma MC), 3465-3500 (dct_four_t4,
// quant_four_4x4 at the chroma QP q, forward_quant_chroma_dc,
// transform.rs:1023), 3606-3628 (dequantize with the DC from
// inverse_quant_chroma_dc, transform.rs:1038, idct_four_t4_rec).  The four
// blocks of a plane are four consecutive lanes of an aligned quad, which trade
// their DC coefficients for the 2x2 transform, so every lane of the warp calls
// this (shuffles over the full warp).  Levels go to co (16 i16, 16-byte
// aligned) unless it is null; the reconstructed rows to r4.
__device__ __forceinline__ void chroma_tq_rec(const uint8_t* src, const uint8_t* ref, int ccw, int cch, int x, int y,
                                              int mvx, int mvy, int k, int q, const int16_t* ff, const int16_t* mf,
                                              int16_t* co, uint32_t r4[4], bool ref_cg = false) {
    const int fx = mvx & 7, fy = mvy & 7;
    const int wa = (8 - fx) * (8 - fy), wb = fx * (8 - fy), wc = (8 - fx) * fy, wd = fx * fy;
    uint32_t s[4], p[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        s[r] = *reinterpret_cast<const uint32_t*>(src + (long long)(y + r) * ccw + x);
        p[r] = chroma_row(ref, ccw, cch, x + (mvx >> 3), y + r + (mvy >> 3), wa, wb, wc, wd, ref_cg);
    }
    int mm[16];
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int c = 0; c < 4; c++) mm[r * 4 + c] = byte_of(s[r], c) - byte_of(p[r], c);
    forward_core4(mm);
    const int dc = int(int16_t(mm[0]));
    // AC levels (quant_four_4x4); slot 0 carries the DC level below
    int lv[16];
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const int pos = ((i >> 2) & 1) * 4 + (i & 3);
        const int cc = int(int16_t(mm[i]));
        const int l = ((abs(cc) + int(ff[pos])) * int(mf[pos])) >> 16;
        lv[i] = int(int16_t(cc < 0 ? -l : l));
    }
    // 2x2 DC: hadamard_2x2 of the four blocks' DCs, then quant (inter dead-zone)
    const int base = int(threadIdx.x & 31) & ~3;
    const int d0 = __shfl_sync(0xffffffffu, dc, base + 0), d1 = __shfl_sync(0xffffffffu, dc, base + 1);
    const int d2 = __shfl_sync(0xffffffffu, dc, base + 2), d3 = __shfl_sync(0xffffffffu, dc, base + 3);
    const int sb = k & 1 ? -1 : 1, sc = k & 2 ? -1 : 1;
    const int f = d0 + sb * d1 + sc * d2 + sb * sc * d3;  // row k of the 2x2 Hadamard
    const int m6 = q % 6, qbits = 15 + q / 6;
    const long long off = (1LL << qbits) / 6;
    const long long la = (long long)(f < 0 ? -f : f) * kQuantMfDc[m6] + 2 * off;
    const int dl = int(f < 0 ? -(la >> (qbits + 1)) : (la >> (qbits + 1)));
    if (co != nullptr) {
        uint32_t w[8];
#pragma unroll
        for (int i = 0; i < 16; i += 2)
            w[i >> 1] = uint32_t(uint16_t(i == 0 ? dl : lv[i])) | (uint32_t(uint16_t(lv[i + 1])) << 16);
        uint4* o = reinterpret_cast<uint4*>(co);
        o[0] = make_uint4(w[0], w[1], w[2], w[3]);
        o[1] = make_uint4(w[4], w[5], w[6], w[7]);
    }
    // reconstruction: inverse_quant_chroma_dc of the DC levels, dequantize of
    // the AC levels, both cast to i16, then the inverse 4x4 and the add
    const int l0 = __shfl_sync(0xffffffffu, dl, base + 0), l1 = __shfl_sync(0xffffffffu, dl, base + 1);
    const int l2 = __shfl_sync(0xffffffffu, dl, base + 2), l3 = __shfl_sync(0xffffffffu, dl, base + 3);
    const int gk = l0 + sb * l1 + sc * l2 + sb * sc * l3;
    const int rdc = int(uint32_t(gk * kLevelScale[m6][0]) << (q / 6)) >> 5;
    lv[0] = 0;
    rec4x4(lv, p, q, r4, rdc);
}

}  // namespace h264a
