/*
 * h264_oracle.c -- CPU restatement of rusty_h264's encoder pixel hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for the CUDA path; never shipped).
 * Each function names the reference function and file:line it restates; paths
 * are relative to the Remade-With-Rust/rusty_h264 project root.
 */
#include "h264_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline int32_t iabs32(int32_t v) { return v < 0 ? -v : v; }
static inline int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int32_t clip_u8(int32_t v) { return clampi(v, 0, 255); }

/* ======================================================================== */
/* SATD / SAD  (crates/rusty_h264-accel/src/satd_sad.rs)                      */
/* ======================================================================== */

/* satd4x4_scalar, satd_sad.rs:39-58: (Σ|H·d| + 1) >> 1 with the openh264
 * butterfly order (rows then columns). */
int32_t or_satd4x4_wels(const uint8_t *a, int sa, const uint8_t *b, int sb) {
    int32_t m[4][4];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) m[i][j] = (int32_t)a[i * sa + j] - (int32_t)b[i * sb + j];
    for (int i = 0; i < 4; i++) {
        int32_t s0 = m[i][0] + m[i][2], s1 = m[i][1] + m[i][3];
        int32_t s2 = m[i][0] - m[i][2], s3 = m[i][1] - m[i][3];
        m[i][0] = s0 + s1; m[i][1] = s2 + s3; m[i][2] = s2 - s3; m[i][3] = s0 - s1;
    }
    int32_t sum = 0;
    for (int j = 0; j < 4; j++) {
        int32_t s0 = m[0][j] + m[2][j], s1 = m[1][j] + m[3][j];
        int32_t s2 = m[0][j] - m[2][j], s3 = m[1][j] - m[3][j];
        sum += iabs32(s0 + s1) + iabs32(s2 + s3) + iabs32(s2 - s3) + iabs32(s0 - s1);
    }
    return (sum + 1) >> 1;
}

/* satd_region_scalar, satd_sad.rs:60-72 (rounding per 4x4 block). */
int32_t or_satd_region_wels(const uint8_t *a, int sa, const uint8_t *b, int sb, int w, int h) {
    int32_t s = 0;
    for (int by = 0; by < h; by += 4)
        for (int bx = 0; bx < w; bx += 4) s += or_satd4x4_wels(a + by * sa + bx, sa, b + by * sb + bx, sb);
    return s;
}

/* sad_scalar, satd_sad.rs:74-82. */
int32_t or_sad(const uint8_t *a, int sa, const uint8_t *b, int sb, int w, int h) {
    int32_t s = 0;
    for (int i = 0; i < h; i++)
        for (int j = 0; j < w; j++) s += iabs32((int32_t)a[i * sa + j] - (int32_t)b[i * sb + j]);
    return s;
}

/* hadamard_1d / hadamard_4x4, transform.rs:631-657 (rows then columns). */
void or_hadamard_4x4(const int32_t in[16], int32_t out[16]) {
    int32_t m[16];
    memcpy(m, in, sizeof m);
    for (int r = 0; r < 4; r++) {
        int32_t a = m[r * 4], b = m[r * 4 + 1], c = m[r * 4 + 2], d = m[r * 4 + 3];
        m[r * 4] = a + b + c + d; m[r * 4 + 1] = a + b - c - d;
        m[r * 4 + 2] = a - b - c + d; m[r * 4 + 3] = a - b + c - d;
    }
    for (int c = 0; c < 4; c++) {
        int32_t a = m[c], b = m[4 + c], cc = m[8 + c], d = m[12 + c];
        m[c] = a + b + cc + d; m[4 + c] = a + b - cc - d;
        m[8 + c] = a - b - cc + d; m[12 + c] = a - b + cc - d;
    }
    memcpy(out, m, sizeof m);
}

/* Scalar Σ|hadamard_4x4(res)| over the 4x4 blocks (transform.rs:701 satd_4x4_sum). */
static int64_t satd_px_scalar(const uint8_t *src, int ss, const uint8_t *pred, int ps, int w, int h) {
    int64_t total = 0;
    for (int by = 0; by < h / 4; by++)
        for (int bx = 0; bx < w / 4; bx++) {
            int32_t blk[16], hh[16];
            for (int dy = 0; dy < 4; dy++)
                for (int dx = 0; dx < 4; dx++)
                    blk[dy * 4 + dx] = (int32_t)src[(by * 4 + dy) * ss + bx * 4 + dx] -
                                       (int32_t)pred[(by * 4 + dy) * ps + bx * 4 + dx];
            or_hadamard_4x4(blk, hh);
            for (int k = 0; k < 16; k++) total += iabs32(hh[k]);
        }
    return total;
}

/* satd_px, mb16.rs:6027-6079.  The accel build serves 16x16/16x8/8x16/8x8/4x4
 * and 8x4/4x8 as 2·Wels-SATD (exact: every 4x4 Hadamard sum is even); the
 * scalar arm covers the rest.  Both are kept so tests can pin their equality. */
int64_t or_satd_px(const uint8_t *src, int ss, const uint8_t *pred, int ps, int w, int h) {
    if ((w == 16 && (h == 16 || h == 8)) || (w == 8 && (h == 16 || h == 8)) || (w == 4 && h == 4) ||
        (w == 8 && h == 4) || (w == 4 && h == 8))
        return 2 * (int64_t)or_satd_region_wels(src, ss, pred, ps, w, h);
    return satd_px_scalar(src, ss, pred, ps, w, h);
}

/* satd_avg, accel/src/satd_avg.rs:579-602: Σ|H·(src − (a+b+1)>>1)| -- the value
 * satd_px computes on the materialised average (encoder tests/satd_avg_compare.rs). */
uint32_t or_satd_avg(const uint8_t *src, int ss, const uint8_t *a, const uint8_t *b, int stride, int w, int h) {
    uint8_t avg[256];
    for (int r = 0; r < h; r++)
        for (int i = 0; i < w; i++)
            avg[r * w + i] = (uint8_t)(((uint32_t)a[r * stride + i] + b[r * stride + i] + 1) >> 1);
    return (uint32_t)satd_px_scalar(src, ss, avg, w, w, h);
}

/* sad_avg_strided, mb16.rs:6104-6116. */
int64_t or_sad_avg(const uint8_t *src, int ss, const uint8_t *a, const uint8_t *b, int stride, int w, int h) {
    int64_t s = 0;
    for (int r = 0; r < h; r++)
        for (int i = 0; i < w; i++) {
            int32_t p = (int32_t)(((uint32_t)a[r * stride + i] + b[r * stride + i] + 1) >> 1);
            s += iabs32((int32_t)src[r * ss + i] - p);
        }
    return s;
}

/* ======================================================================== */
/* Transform / quant (crates/rusty_h264-common/src/transform.rs)             */
/* ======================================================================== */

/* QUANT_MF, transform.rs:25-32 (H.264 forward quant multipliers). */
static const int32_t QUANT_MF[6][3] = {
    {13107, 5243, 8066}, {11916, 4660, 7490}, {10082, 4194, 6554},
    {9362, 3647, 5825},  {8192, 3355, 5243},  {7282, 2893, 4559},
};
/* openh264's 8 quant slots map onto position groups (transform.rs:152). */
static const int GROUP8[8] = {0, 2, 0, 2, 2, 1, 2, 1};

/* fwd_1d + forward_core, transform.rs:72-119 (rows then columns). */
void or_forward_core(const int32_t in[16], int32_t out[16]) {
    int32_t m[16];
    memcpy(m, in, sizeof m);
    for (int r = 0; r < 4; r++) {
        int32_t x0 = m[r * 4], x1 = m[r * 4 + 1], x2 = m[r * 4 + 2], x3 = m[r * 4 + 3];
        int32_t t0 = x0 + x3, t1 = x1 + x2, t2 = x1 - x2, t3 = x0 - x3;
        m[r * 4] = t0 + t1; m[r * 4 + 1] = 2 * t3 + t2; m[r * 4 + 2] = t0 - t1; m[r * 4 + 3] = t3 - 2 * t2;
    }
    for (int c = 0; c < 4; c++) {
        int32_t x0 = m[c], x1 = m[4 + c], x2 = m[8 + c], x3 = m[12 + c];
        int32_t t0 = x0 + x3, t1 = x1 + x2, t2 = x1 - x2, t3 = x0 - x3;
        m[c] = t0 + t1; m[4 + c] = 2 * t3 + t2; m[8 + c] = t0 - t1; m[12 + c] = t3 - 2 * t2;
    }
    memcpy(out, m, sizeof m);
}

/* quant_dz_ff, transform.rs:145-159. */
void or_quant_dz_ff(int qp, int64_t dz_div, int16_t ff[8]) {
    int m = qp % 6;
    int64_t qbits = 15 + qp / 6;
    int64_t f = ((int64_t)1 << qbits) / dz_div;
    for (int i = 0; i < 8; i++) {
        int64_t mfg = QUANT_MF[m][GROUP8[i]];
        ff[i] = (int16_t)((f + mfg / 2) / mfg);
    }
}

/* QUANT_MF_OH[qp], transform.rs:1446-1500 (openh264 g_kiQuantMF): the table
 * equals round-half-up(MF · 2^(16 − qbits)), qbits = 15 + qp/6, which is how it
 * is produced here; tests pin every row against the reference's literal rows. */
void or_quant_mf_oh(int qp, int16_t mf[8]) {
    int m = qp % 6;
    int qbits = 15 + qp / 6;
    for (int i = 0; i < 8; i++) {
        int64_t v = QUANT_MF[m][GROUP8[i]];
        int sh = qbits - 16; /* >= -1 */
        int64_t r = sh < 0 ? v << 1 : (sh == 0 ? v : (v + ((int64_t)1 << (sh - 1))) >> sh);
        mf[i] = (int16_t)r;
    }
}

/* quantize, transform.rs:121-139. */
void or_quantize(const int32_t c[16], int qp, int64_t dz_div, int32_t out[16]) {
    int16_t mf[8], ff[8];
    or_quant_mf_oh(qp, mf);
    or_quant_dz_ff(qp, dz_div, ff);
    for (int idx = 0; idx < 16; idx++) {
        int p = idx & 7;
        int32_t a = iabs32(c[idx]);
        int32_t lvl = ((a + (int32_t)ff[p]) * (int32_t)mf[p]) >> 16;
        out[idx] = c[idx] < 0 ? -lvl : lvl;
    }
}

/* fwd_1d_8x8, transform.rs:492-524. */
static void fwd_1d_8x8(const int32_t s[8], int32_t y[8]) {
    int32_t a0 = s[0] + s[7], a1 = s[1] + s[6], a2 = s[2] + s[5], a3 = s[3] + s[4];
    int32_t a4 = s[0] - s[7], a5 = s[1] - s[6], a6 = s[2] - s[5], a7 = s[3] - s[4];
    int32_t b0 = a0 + a3, b1 = a1 + a2, b2 = a0 - a3, b3 = a1 - a2;
    y[0] = b0 + b1;
    y[2] = b2 + (b3 >> 1);
    y[4] = b0 - b1;
    y[6] = (b2 >> 1) - b3;
    int32_t b4 = a5 + a6 + ((a4 >> 1) + a4);
    int32_t b5 = a4 - a7 - ((a6 >> 1) + a6);
    int32_t b6 = a4 + a7 - ((a5 >> 1) + a5);
    int32_t b7 = a5 - a6 + ((a7 >> 1) + a7);
    y[1] = b4 + (b7 >> 2);
    y[3] = b5 + (b6 >> 2);
    y[5] = b6 - (b5 >> 2);
    y[7] = (b4 >> 2) - b7;
}

/* forward_core_8x8, transform.rs:548-566. */
void or_forward_core_8x8(const int32_t in[64], int32_t out[64]) {
    int32_t m[64], t[8], o[8];
    memcpy(m, in, sizeof m);
    for (int r = 0; r < 8; r++) {
        for (int k = 0; k < 8; k++) t[k] = m[r * 8 + k];
        fwd_1d_8x8(t, o);
        for (int k = 0; k < 8; k++) m[r * 8 + k] = o[k];
    }
    for (int c = 0; c < 8; c++) {
        for (int k = 0; k < 8; k++) t[k] = m[k * 8 + c];
        fwd_1d_8x8(t, o);
        for (int k = 0; k < 8; k++) m[k * 8 + c] = o[k];
    }
    memcpy(out, m, sizeof m);
}

/* QUANT_MF_8X8, transform.rs:595-602, and pos_group_8x8, transform.rs:434-449. */
static const int32_t QUANT_MF_8X8[6][6] = {
    {13107, 14564, 8192, 13797, 10486, 10923}, {11916, 13797, 7490, 12483, 9362, 10083},
    {10083, 11398, 6242, 10923, 7944, 8456},   {9362, 10486, 5825, 10083, 7490, 7944},
    {8192, 9362, 5140, 8738, 6554, 6899},      {7282, 8192, 4520, 7710, 5699, 6096},
};
static int pos_group_8x8(int i, int j) {
    int i4 = i % 4, j4 = j % 4;
    if (i4 == 0 && j4 == 0) return 0;
    if (i % 2 == 1 && j % 2 == 1) return 1;
    if (i4 == 2 && j4 == 2) return 2;
    if ((i4 == 0 && j % 2 == 1) || (i % 2 == 1 && j4 == 0)) return 3;
    if ((i4 == 0 && j4 == 2) || (i4 == 2 && j4 == 0)) return 4;
    return 5;
}

/* quantize_8x8, transform.rs:613-629. */
void or_quantize_8x8(const int32_t c[64], int qp, const int32_t weight[64], int64_t dz_div, int32_t out[64]) {
    int m = qp % 6;
    int64_t qbits = 16 + qp / 6;
    int64_t ff = ((int64_t)1 << qbits) / dz_div;
    for (int idx = 0; idx < 64; idx++) {
        int64_t mf = (int64_t)QUANT_MF_8X8[m][pos_group_8x8(idx / 8, idx % 8)] * 16 / weight[idx];
        int64_t a = c[idx] < 0 ? -(int64_t)c[idx] : (int64_t)c[idx];
        int32_t lvl = (int32_t)((a * mf + ff) >> qbits);
        out[idx] = c[idx] < 0 ? -lvl : lvl;
    }
}

/* dct_four_t4_scalar, accel/src/transform_quant.rs:71-92: sub-blocks in order
 * (0,0),(4,0),(0,4),(4,4); coefficients cast to i16. */
void or_dct_four_t4(int16_t dct[64], const uint8_t *src, int ss, const uint8_t *pred, int ps) {
    static const int SUB[4][2] = {{0, 0}, {4, 0}, {0, 4}, {4, 4}};
    for (int k = 0; k < 4; k++) {
        int ox = SUB[k][0], oy = SUB[k][1];
        int32_t m[16], o[16];
        for (int dy = 0; dy < 4; dy++)
            for (int dx = 0; dx < 4; dx++)
                m[dy * 4 + dx] = (int32_t)src[(oy + dy) * ss + ox + dx] - (int32_t)pred[(oy + dy) * ps + ox + dx];
        or_forward_core(m, o);
        for (int i = 0; i < 16; i++) dct[k * 16 + i] = (int16_t)o[i];
    }
}

/* quant_four_4x4_scalar, accel/src/transform_quant.rs:122-135. */
void or_quant_four_4x4(int16_t dct[64], const int16_t ff[8], const int16_t mf[8]) {
    for (int blk = 0; blk < 4; blk++)
        for (int row = 0; row < 4; row++)
            for (int col = 0; col < 4; col++) {
                int idx = blk * 16 + row * 4 + col;
                int pos = (row & 1) * 4 + col;
                int32_t c = dct[idx];
                int32_t lvl = ((iabs32(c) + (int32_t)ff[pos]) * (int32_t)mf[pos]) >> 16;
                dct[idx] = (int16_t)(c < 0 ? -lvl : lvl);
            }
}

/* The encoder's luma T/Q of one MB (mb16.rs:3436-3450): four 8x8 regions in
 * order (0,0),(8,0),(0,8),(8,8), each dct_four_t4 then quant_four_4x4 with
 * quant_dz_ff(qp, dz) and QUANT_MF_OH[qp].  pred16 has stride 16. */
void or_mb_luma_tq(const uint8_t *src, int ss, const uint8_t *pred16, int qp, int dz_div, int16_t out[256]) {
    static const int Q[4][2] = {{0, 0}, {8, 0}, {0, 8}, {8, 8}};
    int16_t ff[8], mf[8];
    or_quant_dz_ff(qp, dz_div, ff);
    or_quant_mf_oh(qp, mf);
    for (int qi = 0; qi < 4; qi++)
        or_dct_four_t4(out + qi * 64, src + Q[qi][1] * ss + Q[qi][0], ss, pred16 + Q[qi][1] * 16 + Q[qi][0], 16);
    for (int qi = 0; qi < 4; qi++) or_quant_four_4x4(out + qi * 64, ff, mf);
}

/* ---- reconstruction: dequant + inverse 4x4 + add ---------------------------- */

/* NORM_ADJUST (transform.rs:15-22) by qp % 6 and position group; the group of
 * raster position idx is POS_GROUP_FLAT (transform.rs:48-52): (row, col) both
 * even -> 0, both odd -> 1, else 2. */
static const int32_t OR_NORM_ADJUST[6][3] = {{10, 16, 13}, {11, 18, 14}, {13, 20, 16},
                                             {14, 23, 18}, {16, 25, 20}, {18, 29, 23}};
static int or_pos_group4(int idx) {
    int r = (idx >> 2) & 1, c = idx & 1;
    return (r == 0 && c == 0) ? 0 : ((r == 1 && c == 1) ? 1 : 2);
}

/* dequantize (transform.rs:233-284), flat scaling list: LevelScale =
 * 16 * NORM_ADJUST; qp >= 24: (l * ls) << (qp/6 - 4), else
 * (l * ls + 2^(3 - qp/6)) >> (4 - qp/6). */
void or_dequant4x4(const int32_t lv[16], int qp, int32_t out[16]) {
    int m = qp % 6, shift = qp / 6;
    for (int i = 0; i < 16; i++) {
        int32_t ls = 16 * OR_NORM_ADJUST[m][or_pos_group4(i)];
        if (qp >= 24)
            out[i] = (int32_t)((uint32_t)(lv[i] * ls) << (shift - 4));
        else
            out[i] = (lv[i] * ls + (1 << (3 - shift))) >> (4 - shift);
    }
}

/* inv_1d + inverse_core (transform_quant.rs:30-35, 56-69): rows first, then
 * columns, then (x + 32) >> 6. */
static void or_inv_1d(int32_t d0, int32_t d1, int32_t d2, int32_t d3, int32_t o[4]) {
    int32_t e0 = d0 + d2, e1 = d0 - d2, e2 = (d1 >> 1) - d3, e3 = d1 + (d3 >> 1);
    o[0] = e0 + e3; o[1] = e1 + e2; o[2] = e1 - e2; o[3] = e0 - e3;
}
void or_inverse_core4(int32_t m[16]) {
    int32_t o[4];
    for (int r = 0; r < 4; r++) {
        or_inv_1d(m[r * 4], m[r * 4 + 1], m[r * 4 + 2], m[r * 4 + 3], o);
        for (int k = 0; k < 4; k++) m[r * 4 + k] = o[k];
    }
    for (int c = 0; c < 4; c++) {
        or_inv_1d(m[c], m[4 + c], m[8 + c], m[12 + c], o);
        for (int k = 0; k < 4; k++) m[k * 4 + c] = o[k];
    }
    for (int i = 0; i < 16; i++) m[i] = (m[i] + 32) >> 6;
}

/* idct_four_t4_rec_scalar (transform_quant.rs:96-119): four coefficient
 * blocks in SUBBLOCKS order, each inverse-transformed and added to pred with
 * clamping into rec. */
void or_idct_four_t4_rec(uint8_t *rec, int srec, const uint8_t *pred, int spred, const int16_t dct[64]) {
    static const int SB[4][2] = {{0, 0}, {4, 0}, {0, 4}, {4, 4}};
    for (int k = 0; k < 4; k++) {
        int32_t m[16];
        for (int i = 0; i < 16; i++) m[i] = dct[k * 16 + i];
        or_inverse_core4(m);
        for (int dy = 0; dy < 4; dy++)
            for (int dx = 0; dx < 4; dx++) {
                int v = pred[(SB[k][1] + dy) * spred + SB[k][0] + dx] + m[dy * 4 + dx];
                rec[(SB[k][1] + dy) * srec + SB[k][0] + dx] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
            }
    }
}

/* The inter MB's luma reconstruction (mb16.rs:3575-3605): per 8x8 quad the
 * levels of its four blocks are dequantized, cast to i16 (the reference's
 * `deq[i] as i16`), inverse-transformed and added to the 16x16 prediction.
 * (A quad with no coded block copies the prediction, which is the same bytes:
 * the inverse of all-zero levels is zero.) */
void or_mb_luma_rec(uint8_t *rec, int srec, const uint8_t *pred16, const int16_t levels[256], int qp) {
    static const int Q[4][2] = {{0, 0}, {8, 0}, {0, 8}, {8, 8}};
    for (int qi = 0; qi < 4; qi++) {
        int16_t dct_in[64];
        for (int k = 0; k < 4; k++) {
            int32_t lv[16], dq[16];
            for (int i = 0; i < 16; i++) lv[i] = levels[(qi * 4 + k) * 16 + i];
            or_dequant4x4(lv, qp, dq);
            for (int i = 0; i < 16; i++) dct_in[k * 16 + i] = (int16_t)dq[i];
        }
        or_idct_four_t4_rec(rec + Q[qi][1] * srec + Q[qi][0], srec, pred16 + Q[qi][1] * 16 + Q[qi][0], 16, dct_in);
    }
}

/* ---- chroma: QP map, 2x2 DC transform and quant ------------------------- */

/* chroma_qp (predict.rs:64-73): identity below 30, then the QPC table. */
int or_chroma_qp(int qp) {
    static const int QPC[22] = {29, 30, 31, 32, 32, 33, 34, 34, 35, 35, 36, 36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39};
    return qp < 30 ? qp : QPC[qp - 30];
}

/* hadamard_2x2 (transform.rs:1017-1021). */
static void or_hadamard2x2(const int32_t d[4], int32_t o[4]) {
    o[0] = d[0] + d[1] + d[2] + d[3];
    o[1] = d[0] - d[1] + d[2] - d[3];
    o[2] = d[0] + d[1] - d[2] - d[3];
    o[3] = d[0] - d[1] - d[2] + d[3];
}

/* forward_quant_chroma_dc (transform.rs:1023-1035). */
void or_forward_quant_chroma_dc(const int32_t dc[4], int qp, int intra, int32_t out[4]) {
    int32_t f[4];
    or_hadamard2x2(dc, f);
    int m = qp % 6;
    int qbits = 15 + qp / 6;
    int64_t off = intra ? ((int64_t)1 << qbits) / 3 : ((int64_t)1 << qbits) / 6;
    int64_t mf = QUANT_MF[m][0];
    for (int i = 0; i < 4; i++) {
        int64_t a = f[i] < 0 ? -(int64_t)f[i] : f[i];
        int64_t level = (a * mf + 2 * off) >> (qbits + 1);
        out[i] = (int32_t)(f[i] < 0 ? -level : level);
    }
}

/* inverse_quant_chroma_dc (transform.rs:1038-1050). */
void or_inverse_quant_chroma_dc(const int32_t levels[4], int qp, int32_t out[4]) {
    int32_t g[4];
    or_hadamard2x2(levels, g);
    int m = qp % 6, shift = qp / 6;
    int32_t ls = 16 * OR_NORM_ADJUST[m][0];
    for (int i = 0; i < 4; i++) out[i] = (int32_t)((uint32_t)(g[i] * ls) << shift) >> 5;
}

/* ======================================================================== */
/* Inter prediction (crates/rusty_h264-common/src/inter.rs)                 */
/* ======================================================================== */

/* median3, inter.rs:9-11. */
int32_t or_median3(int32_t a, int32_t b, int32_t c) {
    int32_t mn = a < b ? a : b; mn = mn < c ? mn : c;
    int32_t mx = a > b ? a : b; mx = mx > c ? mx : c;
    return a + b + c - mn - mx;
}

/* predict_mv, inter.rs:36-69. */
void or_predict_mv(const or_mv_neighbor *a, const or_mv_neighbor *b, const or_mv_neighbor *c, int cur_ref,
                   int32_t out[2]) {
    int32_t mva[2] = {0, 0}, mvb[2] = {0, 0}, mvc[2] = {0, 0};
    int32_t ra = -1, rb = -1, rc = -1;
    if (a->available && a->ref_idx >= 0) { mva[0] = a->mvx; mva[1] = a->mvy; ra = a->ref_idx; }
    if (b->available && b->ref_idx >= 0) { mvb[0] = b->mvx; mvb[1] = b->mvy; rb = b->ref_idx; }
    if (c->available && c->ref_idx >= 0) { mvc[0] = c->mvx; mvc[1] = c->mvy; rc = c->ref_idx; }
    if (!b->available && !c->available && a->available) {
        mvb[0] = mva[0]; mvb[1] = mva[1]; rb = ra;
        mvc[0] = mva[0]; mvc[1] = mva[1]; rc = ra;
    }
    int matches = (ra == cur_ref) + (rb == cur_ref) + (rc == cur_ref);
    if (matches == 1) {
        const int32_t *p = ra == cur_ref ? mva : (rb == cur_ref ? mvb : mvc);
        out[0] = p[0]; out[1] = p[1];
    } else {
        out[0] = or_median3(mva[0], mvb[0], mvc[0]);
        out[1] = or_median3(mva[1], mvb[1], mvc[1]);
    }
}

/* predict_partition_mv, inter.rs:76-98. */
void or_predict_partition_mv(int mode, int part, const or_mv_neighbor *a, const or_mv_neighbor *b,
                             const or_mv_neighbor *c, int cur_ref, int32_t out[2]) {
    if (mode == 0) { or_predict_mv(a, b, c, cur_ref, out); return; }
#define M(n) ((n)->available && (n)->ref_idx == cur_ref)
    if (mode == 1 && part == 0 && M(b)) { out[0] = b->mvx; out[1] = b->mvy; return; }
    if (mode == 1 && part == 1 && M(a)) { out[0] = a->mvx; out[1] = a->mvy; return; }
    if (mode == 2 && part == 0 && M(a)) { out[0] = a->mvx; out[1] = a->mvy; return; }
    if (mode == 2 && part == 1 && M(c)) { out[0] = c->mvx; out[1] = c->mvy; return; }
#undef M
    or_predict_mv(a, b, c, cur_ref, out);
}

/* at(), inter.rs:124-128: edge-clamped reference read. */
static inline int32_t at(const uint8_t *ref, int cw, int ch, int x, int y) {
    return ref[clampi(y, 0, ch - 1) * cw + clampi(x, 0, cw - 1)];
}

/* luma_sample, inter.rs:134-176 -- the per-pixel spec oracle (§8.4.2.2.1). */
int32_t or_luma_sample(const uint8_t *ref, int cw, int ch, int ix, int iy, int fx, int fy) {
#define G(dx, dy) at(ref, cw, ch, ix + (dx), iy + (dy))
#define HOR6(dy) (G(-2, dy) - 5 * G(-1, dy) + 20 * G(0, dy) + 20 * G(1, dy) - 5 * G(2, dy) + G(3, dy))
#define VER6(dx) (G(dx, -2) - 5 * G(dx, -1) + 20 * G(dx, 0) + 20 * G(dx, 1) - 5 * G(dx, 2) + G(dx, 3))
    if (fx == 0 && fy == 0) return G(0, 0);
    int32_t b = clip_u8((HOR6(0) + 16) >> 5);
    int32_t h = clip_u8((VER6(0) + 16) >> 5);
    int32_t m = clip_u8((VER6(1) + 16) >> 5);
    int32_t s = clip_u8((HOR6(1) + 16) >> 5);
    int32_t j1 = HOR6(-2) - 5 * HOR6(-1) + 20 * HOR6(0) + 20 * HOR6(1) - 5 * HOR6(2) + HOR6(3);
    int32_t j = clip_u8((j1 + 512) >> 10);
    switch (fx * 4 + fy) {
    case 1 * 4 + 0: return (G(0, 0) + b + 1) >> 1;
    case 2 * 4 + 0: return b;
    case 3 * 4 + 0: return (G(1, 0) + b + 1) >> 1;
    case 0 * 4 + 1: return (G(0, 0) + h + 1) >> 1;
    case 1 * 4 + 1: return (b + h + 1) >> 1;
    case 2 * 4 + 1: return (b + j + 1) >> 1;
    case 3 * 4 + 1: return (b + m + 1) >> 1;
    case 0 * 4 + 2: return h;
    case 1 * 4 + 2: return (h + j + 1) >> 1;
    case 2 * 4 + 2: return j;
    case 3 * 4 + 2: return (j + m + 1) >> 1;
    case 0 * 4 + 3: return (G(0, 1) + h + 1) >> 1;
    case 1 * 4 + 3: return (h + s + 1) >> 1;
    case 2 * 4 + 3: return (j + s + 1) >> 1;
    default: return (m + s + 1) >> 1;
    }
#undef G
#undef HOR6
#undef VER6
}

/* luma_tile_into, inter.rs:365-400: clamped (bw+5)×(bh+5) halo, block at (2,2). */
static int luma_tile_into(uint8_t *t, const uint8_t *ref, int cw, int ch, int ix0, int iy0, int bw, int bh) {
    int ts = bw + 5;
    for (int ty = 0; ty < bh + 5; ty++) {
        int ry = clampi(iy0 - 2 + ty, 0, ch - 1);
        for (int tx = 0; tx < ts; tx++) t[ty * ts + tx] = ref[ry * cw + clampi(ix0 - 2 + tx, 0, cw - 1)];
    }
    return ts;
}

/* luma_h, inter.rs:404-430 (scalar arm). */
static void luma_h(const uint8_t *t, int ts, int bw, int bh, int dr, int dc, uint8_t *dst) {
    for (int r = 0; r < bh; r++) {
        const uint8_t *w = t + (2 + r + dr) * ts + 2 + dc - 2;
        for (int c = 0; c < bw; c++) {
            int32_t f = w[c] - 5 * w[c + 1] + 20 * w[c + 2] + 20 * w[c + 3] - 5 * w[c + 4] + w[c + 5];
            dst[r * bw + c] = (uint8_t)clip_u8((f + 16) >> 5);
        }
    }
}

/* luma_v, inter.rs:433-452 (scalar arm). */
static void luma_v(const uint8_t *t, int ts, int bw, int bh, int dr, int dc, uint8_t *dst) {
    for (int r = 0; r < bh; r++)
        for (int c = 0; c < bw; c++) {
            int p = (2 + r + dr) * ts + 2 + dc + c;
            int32_t f = t[p - 2 * ts] - 5 * t[p - ts] + 20 * t[p] + 20 * t[p + ts] - 5 * t[p + 2 * ts] + t[p + 3 * ts];
            dst[r * bw + c] = (uint8_t)clip_u8((f + 16) >> 5);
        }
}

/* luma_centre, inter.rs:456-484 (scalar arm): vertical i32 intermediates then horizontal. */
static void luma_centre(const uint8_t *t, int ts, int bw, int bh, uint8_t *dst) {
    int32_t itmp[21];
    for (int r = 0; r < bh; r++) {
        for (int j = 0; j < bw + 5; j++) {
            int p = (2 + r) * ts + j;
            itmp[j] = t[p - 2 * ts] - 5 * t[p - ts] + 20 * t[p] + 20 * t[p + ts] - 5 * t[p + 2 * ts] + t[p + 3 * ts];
        }
        for (int c = 0; c < bw; c++) {
            const int32_t *w = itmp + c;
            int32_t f = w[0] - 5 * w[1] + 20 * w[2] + 20 * w[3] - 5 * w[4] + w[5];
            dst[r * bw + c] = (uint8_t)clip_u8((f + 512) >> 10);
        }
    }
}

/* pixel_avg, inter.rs:487-516 (scalar arm). */
static void pixel_avg(const uint8_t *a, const uint8_t *b, int n, uint8_t *dst) {
    for (int i = 0; i < n; i++) dst[i] = (uint8_t)(((int32_t)a[i] + b[i] + 1) >> 1);
}

/* avg_full, inter.rs:519-540 (scalar arm). */
static void avg_full(const uint8_t *t, int ts, int bw, int bh, int dr, int dc, const uint8_t *half, uint8_t *dst) {
    for (int r = 0; r < bh; r++)
        for (int x = 0; x < bw; x++)
            dst[r * bw + x] = (uint8_t)(((int32_t)t[(2 + r + dr) * ts + 2 + dc + x] + half[r * bw + x] + 1) >> 1);
}

/* mc_luma_subpel, inter.rs:668-697, through the compose arms of
 * qpel_one_filter :553, qpel_hv :589, qpel_centre_adj :619. */
static void mc_luma_subpel(const uint8_t *t, int ts, int bw, int bh, int fx, int fy, uint8_t *out) {
    uint8_t a[256], b[256];
    int n = bw * bh;
    switch (fx * 4 + fy) {
    case 2 * 4 + 0: luma_h(t, ts, bw, bh, 0, 0, out); break;
    case 0 * 4 + 2: luma_v(t, ts, bw, bh, 0, 0, out); break;
    case 2 * 4 + 2: luma_centre(t, ts, bw, bh, out); break;
    case 1 * 4 + 0: luma_h(t, ts, bw, bh, 0, 0, a); avg_full(t, ts, bw, bh, 0, 0, a, out); break;
    case 3 * 4 + 0: luma_h(t, ts, bw, bh, 0, 0, a); avg_full(t, ts, bw, bh, 0, 1, a, out); break;
    case 0 * 4 + 1: luma_v(t, ts, bw, bh, 0, 0, a); avg_full(t, ts, bw, bh, 0, 0, a, out); break;
    case 0 * 4 + 3: luma_v(t, ts, bw, bh, 0, 0, a); avg_full(t, ts, bw, bh, 1, 0, a, out); break;
    case 1 * 4 + 1: luma_h(t, ts, bw, bh, 0, 0, a); luma_v(t, ts, bw, bh, 0, 0, b); pixel_avg(a, b, n, out); break;
    case 3 * 4 + 1: luma_h(t, ts, bw, bh, 0, 0, a); luma_v(t, ts, bw, bh, 0, 1, b); pixel_avg(a, b, n, out); break;
    case 1 * 4 + 3: luma_h(t, ts, bw, bh, 1, 0, a); luma_v(t, ts, bw, bh, 0, 0, b); pixel_avg(a, b, n, out); break;
    case 3 * 4 + 3: luma_h(t, ts, bw, bh, 1, 0, a); luma_v(t, ts, bw, bh, 0, 1, b); pixel_avg(a, b, n, out); break;
    case 2 * 4 + 1: luma_h(t, ts, bw, bh, 0, 0, a); luma_centre(t, ts, bw, bh, b); pixel_avg(a, b, n, out); break;
    case 2 * 4 + 3: luma_h(t, ts, bw, bh, 1, 0, a); luma_centre(t, ts, bw, bh, b); pixel_avg(a, b, n, out); break;
    case 1 * 4 + 2: luma_v(t, ts, bw, bh, 0, 0, a); luma_centre(t, ts, bw, bh, b); pixel_avg(a, b, n, out); break;
    default: /* (3,2) */ luma_v(t, ts, bw, bh, 0, 1, a); luma_centre(t, ts, bw, bh, b); pixel_avg(a, b, n, out); break;
    }
}

/* mc_luma, inter.rs:1193-1262. */
void or_mc_luma(const uint8_t *ref, int cw, int ch, int x0, int y0, int bw, int bh, int mvx, int mvy, uint8_t *out) {
    int ix0 = x0 + (mvx >> 2), iy0 = y0 + (mvy >> 2);
    int fx = mvx & 3, fy = mvy & 3;
    if (fx == 0 && fy == 0) {
        for (int dy = 0; dy < bh; dy++)
            for (int dx = 0; dx < bw; dx++) out[dy * bw + dx] = (uint8_t)at(ref, cw, ch, ix0 + dx, iy0 + dy);
        return;
    }
    uint8_t tile[21 * 21];
    int ts = luma_tile_into(tile, ref, cw, ch, ix0, iy0, bw, bh);
    mc_luma_subpel(tile, ts, bw, bh, fx, fy, out);
}

/* pad_plane_into, inter.rs:798-813 (edge replication). */
void or_pad_plane(const uint8_t *src, int w, int h, int pad, uint8_t *f) {
    int pw = w + 2 * pad, ph = h + 2 * pad;
    for (int y = 0; y < ph; y++) {
        int sy = clampi(y - pad, 0, h - 1);
        const uint8_t *row = src + (size_t)sy * w;
        uint8_t *d = f + (size_t)y * pw;
        memset(d, row[0], pad);
        memcpy(d + pad, row, w);
        memset(d + pad + w, row[w - 1], pad);
    }
}

/* build_hpel_fused, inter.rs:908-991: one pass per row, vertical 6-tap
 * intermediates (i32, unrounded) over clamped columns, then H, V, C. */
void or_hpel_fused(const uint8_t *f, int pw, int ph, uint8_t *h, uint8_t *v, uint8_t *c) {
    int32_t *vt = (int32_t *)malloc(sizeof(int32_t) * (pw + 5));
    uint8_t *hb = (uint8_t *)malloc(pw + 5);
    for (int y = 0; y < ph; y++) {
        const uint8_t *rows[6];
        for (int k = 0; k < 6; k++) rows[k] = f + (size_t)clampi(y - 2 + k, 0, ph - 1) * pw;
#define TAP(x) (rows[0][x] - 5 * rows[1][x] + 20 * rows[2][x] + 20 * rows[3][x] - 5 * rows[4][x] + rows[5][x])
        for (int j = 0; j < pw + 5; j++) {
            int x = clampi(j - 2, 0, pw - 1);
            vt[j] = TAP(x);
            hb[j] = rows[2][x];
        }
#undef TAP
        uint8_t *hrow = h + (size_t)y * pw, *vrow = v + (size_t)y * pw, *crow = c + (size_t)y * pw;
        for (int x = 0; x < pw; x++) {
            vrow[x] = (uint8_t)clip_u8((vt[x + 2] + 16) >> 5);
            const int32_t *w = vt + x;
            int32_t s = w[0] - 5 * w[1] + 20 * w[2] + 20 * w[3] - 5 * w[4] + w[5];
            crow[x] = (uint8_t)clip_u8((s + 512) >> 10);
            const uint8_t *b = hb + x;
            int32_t sh = b[0] - 5 * b[1] + 20 * b[2] + 20 * b[3] - 5 * b[4] + b[5];
            hrow[x] = (uint8_t)clip_u8((sh + 16) >> 5);
        }
    }
    free(vt);
    free(hb);
}

/* build_hpel_tiles, inter.rs:868-899: 16x16 tile walk through the clamped tile
 * and the block kernels -- the fused builder's oracle in the reference. */
void or_hpel_tiles(const uint8_t *f, int pw, int ph, uint8_t *h, uint8_t *v, uint8_t *c) {
    uint8_t tile[21 * 21], blk[256];
    for (int by = 0; by < ph; by += 16)
        for (int bx = 0; bx < pw; bx += 16) {
            int bh = ph - by < 16 ? ph - by : 16;
            int bw = pw - bx < 16 ? pw - bx : 16;
            int ts = luma_tile_into(tile, f, pw, ph, bx, by, bw, bh);
            for (int kind = 0; kind < 3; kind++) {
                uint8_t *plane = kind == 0 ? h : (kind == 1 ? v : c);
                if (kind == 0) luma_h(tile, ts, bw, bh, 0, 0, blk);
                else if (kind == 1) luma_v(tile, ts, bw, bh, 0, 0, blk);
                else luma_centre(tile, ts, bw, bh, blk);
                for (int r = 0; r < bh; r++) memcpy(plane + (size_t)(by + r) * pw + bx, blk + r * bw, bw);
            }
        }
}

/* build_hpel_planes, inter.rs:816-849 (pad then the fused builder). */
void or_build_hpel_planes(const uint8_t *ref, int cw, int ch, int pad, uint8_t *f, uint8_t *h, uint8_t *v, uint8_t *c) {
    int pw = cw + 2 * pad, ph = ch + 2 * pad;
    or_pad_plane(ref, cw, ch, pad, f);
    or_hpel_fused(f, pw, ph, h, v, c);
}

static const uint8_t *plane_ptr(const or_hpel_planes *p, int idx) {
    return idx == 0 ? p->f : idx == 1 ? p->h : idx == 2 ? p->v : p->c;
}

/* hpel_ref, inter.rs:1015-1051 (planes 0=f 1=h 2=v 3=c). */
int or_hpel_ref(const or_hpel_planes *p, int x0, int y0, int bw, int bh, int mvx, int mvy, int *plane, int64_t *base) {
    int fx = mvx & 3, fy = mvy & 3;
    int pl;
    if (fx == 2 && fy == 0) pl = 1;
    else if (fx == 0 && fy == 2) pl = 2;
    else if (fx == 2 && fy == 2) pl = 3;
    else if (fx == 0 && fy == 0) pl = 0;
    else return 0;
    int px = x0 + (mvx >> 2) + p->pad, py = y0 + (mvy >> 2) + p->pad;
    if (px < 0 || py < 0 || px + bw + 1 > p->pw || py + bh + 1 > p->ph) return 0;
    int64_t b = (int64_t)py * p->pw + px;
    if (b + (int64_t)(bh - 1) * p->pw + bw > (int64_t)p->pw * p->ph) return 0;
    *plane = pl;
    *base = b;
    return 1;
}

/* hpel_qpel_refs, inter.rs:1060-1105. */
int or_hpel_qpel_refs(const or_hpel_planes *p, int x0, int y0, int bw, int bh, int mvx, int mvy, int *pa, int64_t *oa,
                      int *pb, int64_t *ob) {
    int fx = mvx & 3, fy = mvy & 3;
    if ((fx & 1) == 0 && (fy & 1) == 0) return 0;
    int px = x0 + (mvx >> 2) + p->pad, py = y0 + (mvy >> 2) + p->pad;
    if (px < 0 || py < 0 || px + bw + 1 > p->pw || py + bh + 1 > p->ph) return 0;
    int64_t st = p->pw, base = (int64_t)py * st + px;
    int a, b;
    int64_t da, db;
    switch (fx * 4 + fy) {
    case 1 * 4 + 0: a = 0; da = 0; b = 1; db = 0; break;
    case 3 * 4 + 0: a = 0; da = 1; b = 1; db = 0; break;
    case 0 * 4 + 1: a = 0; da = 0; b = 2; db = 0; break;
    case 0 * 4 + 3: a = 0; da = st; b = 2; db = 0; break;
    case 1 * 4 + 1: a = 1; da = 0; b = 2; db = 0; break;
    case 3 * 4 + 1: a = 1; da = 0; b = 2; db = 1; break;
    case 1 * 4 + 3: a = 1; da = st; b = 2; db = 0; break;
    case 3 * 4 + 3: a = 1; da = st; b = 2; db = 1; break;
    case 2 * 4 + 1: a = 1; da = 0; b = 3; db = 0; break;
    case 2 * 4 + 3: a = 1; da = st; b = 3; db = 0; break;
    case 1 * 4 + 2: a = 2; da = 0; b = 3; db = 0; break;
    default: /* (3,2) */ a = 2; da = 1; b = 3; db = 0; break;
    }
    int64_t len = (int64_t)p->pw * p->ph;
    if (base + da + (int64_t)(bh - 1) * st + bw > len || base + db + (int64_t)(bh - 1) * st + bw > len) return 0;
    *pa = a; *oa = base + da; *pb = b; *ob = base + db;
    return 1;
}

/* hpel_block, inter.rs:1107-1162. */
int or_hpel_block(const or_hpel_planes *p, int x0, int y0, int bw, int bh, int mvx, int mvy, uint8_t *out) {
    int fx = mvx & 3, fy = mvy & 3;
    if (fx == 0 && fy == 0) return 0;
    int px = x0 + (mvx >> 2) + p->pad, py = y0 + (mvy >> 2) + p->pad;
    if (px < 0 || py < 0 || px + bw + 1 > p->pw || py + bh + 1 > p->ph) return 0;
    int64_t base = (int64_t)py * p->pw + px;
    const uint8_t *single = NULL;
    if (fx == 2 && fy == 0) single = p->h;
    else if (fx == 0 && fy == 2) single = p->v;
    else if (fx == 2 && fy == 2) single = p->c;
    if (single) {
        for (int r = 0; r < bh; r++) memcpy(out + r * bw, single + base + (int64_t)r * p->pw, bw);
        return 1;
    }
    int pa, pb;
    int64_t oa, ob;
    if (!or_hpel_qpel_refs(p, x0, y0, bw, bh, mvx, mvy, &pa, &oa, &pb, &ob)) return 0;
    if (bw != 16 && bw != 8 && bw != 4) return 0;
    const uint8_t *A = plane_ptr(p, pa), *B = plane_ptr(p, pb);
    for (int r = 0; r < bh; r++)
        for (int i = 0; i < bw; i++)
            out[r * bw + i] = (uint8_t)(((int32_t)A[oa + (int64_t)r * p->pw + i] + B[ob + (int64_t)r * p->pw + i] + 1) >> 1);
    return 1;
}

/* ======================================================================== */
/* Motion search (crates/rusty_h264-encoder/src/mb16.rs)                     */
/* ======================================================================== */

/* mvbits closure, mb16.rs:2454-2482. */
uint32_t or_mvbits(int kind, const uint16_t *tab, int32_t d) {
    if (kind == 1 || kind == 2) {
        uint32_t a = (uint32_t)(d < 0 ? -(int64_t)d : d);
        if (a > 4095) a = 4095;
        return tab[a];
    }
    uint32_t codenum = d > 0 ? (uint32_t)(2 * d - 1) : (uint32_t)(-2 * d);
    uint32_t x = codenum + 1;
    return 1 + 2 * (31 - (uint32_t)__builtin_clz(x));
}

/* build_mv_cost, mb16.rs:508-519 (f64 log2, round half away from zero). */
void or_build_mv_cost(uint16_t out[4096]) {
    for (uint32_t a = 0; a < 4096; a++) {
        double c = 2.0 * log2((double)(a + 1)) + 0.718 + (a != 0 ? 1.0 : 0.0);
        out[a] = (uint16_t)round(c * 4.0);
    }
}

/* mc_satd_hp, mb16.rs:1930-2010 (hr_on and sa_on as in the accel build). */
int64_t or_mc_satd_hp(const or_me_frame *fr, int use_planes, int lx, int ly, int rw, int rh, int mvx, int mvy) {
    int cw = fr->cw, ch = fr->ch;
    const uint8_t *src = fr->src + (int64_t)ly * cw + lx;
    int ix0 = lx + (mvx >> 2), iy0 = ly + (mvy >> 2);
    if ((mvx & 3) == 0 && (mvy & 3) == 0 && ix0 >= 0 && iy0 >= 0 && ix0 + rw <= cw && iy0 + rh <= ch)
        return or_satd_px(src, cw, fr->ref + (int64_t)iy0 * cw + ix0, cw, rw, rh);
    uint8_t pred[256];
    if (use_planes) {
        const or_hpel_planes *p = &fr->planes;
        int pl;
        int64_t base;
        if (or_hpel_ref(p, lx, ly, rw, rh, mvx, mvy, &pl, &base))
            return or_satd_px(src, cw, plane_ptr(p, pl) + base, p->pw, rw, rh);
        int pa, pb;
        int64_t oa, ob;
        if (((rw == 16 || rw == 8) && (rh == 16 || rh == 8)) &&
            or_hpel_qpel_refs(p, lx, ly, rw, rh, mvx, mvy, &pa, &oa, &pb, &ob))
            return or_satd_avg(src, cw, plane_ptr(p, pa) + oa, plane_ptr(p, pb) + ob, p->pw, rw, rh);
        if (or_hpel_block(p, lx, ly, rw, rh, mvx, mvy, pred)) return or_satd_px(src, cw, pred, rw, rw, rh);
    }
    or_mc_luma(fr->ref, cw, ch, lx, ly, rw, rh, mvx, mvy, pred);
    return or_satd_px(src, cw, pred, rw, rw, rh);
}

/* mc_sad_hp, mb16.rs:2018-2074 (also the value mc_sad :2090 returns). */
int64_t or_mc_sad_hp(const or_me_frame *fr, int use_planes, int lx, int ly, int rw, int rh, int mvx, int mvy) {
    int cw = fr->cw, ch = fr->ch;
    const uint8_t *src = fr->src + (int64_t)ly * cw + lx;
    int ix0 = lx + (mvx >> 2), iy0 = ly + (mvy >> 2);
    if ((mvx & 3) == 0 && (mvy & 3) == 0 && ix0 >= 0 && iy0 >= 0 && ix0 + rw <= cw && iy0 + rh <= ch)
        return or_sad(src, cw, fr->ref + (int64_t)iy0 * cw + ix0, cw, rw, rh);
    uint8_t pred[256];
    if (use_planes) {
        const or_hpel_planes *p = &fr->planes;
        int pl;
        int64_t base;
        if (or_hpel_ref(p, lx, ly, rw, rh, mvx, mvy, &pl, &base))
            return or_sad(src, cw, plane_ptr(p, pl) + base, p->pw, rw, rh);
        int pa, pb;
        int64_t oa, ob;
        if (or_hpel_qpel_refs(p, lx, ly, rw, rh, mvx, mvy, &pa, &oa, &pb, &ob))
            return or_sad_avg(src, cw, plane_ptr(p, pa) + oa, plane_ptr(p, pb) + ob, p->pw, rw, rh);
        if (or_hpel_block(p, lx, ly, rw, rh, mvx, mvy, pred)) return or_sad(src, cw, pred, rw, rw, rh);
    }
    or_mc_luma(fr->ref, cw, ch, lx, ly, rw, rh, mvx, mvy, pred);
    return or_sad(src, cw, pred, rw, rw, rh);
}

typedef struct {
    const or_me_frame *fr;
    const or_me_params *pr;
    int lx, ly, rw, rh;
    int32_t cx, cy;
    double lam_r, lam_fp, lambda_me;
    int sadfp, use_sad, use_planes;
    int32_t evals;
} ms_ctx;

static uint32_t ms_rate(const ms_ctx *m, int32_t mvx, int32_t mvy) {
    return or_mvbits(m->pr->mv_cost_kind, m->pr->mv_cost_tab, mvx - m->cx) +
           or_mvbits(m->pr->mv_cost_kind, m->pr->mv_cost_tab, mvy - m->cy);
}

/* the `cost` closure, mb16.rs:2540-2566 */
static int64_t ms_cost(ms_ctx *m, int32_t mvx, int32_t mvy) {
    uint32_t rate = ms_rate(m, mvx, mvy);
    m->evals++;
    int64_t dist = m->use_sad ? or_mc_sad_hp(m->fr, m->use_planes, m->lx, m->ly, m->rw, m->rh, mvx, mvy)
                              : or_mc_satd_hp(m->fr, m->use_planes, m->lx, m->ly, m->rw, m->rh, mvx, mvy);
    return dist + (int64_t)(m->lam_r * (double)rate);
}

/* the `cost_fp` closure, mb16.rs:2569-2578 */
static int64_t ms_cost_fp(ms_ctx *m, int32_t mvx, int32_t mvy) {
    if (!m->sadfp) return ms_cost(m, mvx, mvy);
    uint32_t rate = ms_rate(m, mvx, mvy);
    m->evals++;
    return or_mc_sad_hp(m->fr, m->use_planes, m->lx, m->ly, m->rw, m->rh, mvx, mvy) +
           (int64_t)(m->lam_fp * (double)rate);
}

static const int32_t DIA_RUNGS[5] = {64, 32, 16, 8, 4};

/* motion_search, mb16.rs:2433-3302, for the accel (x86-64 default) build:
 * seeds, integer snap, fixed-centre/cascade diamond ladder, B2 reprice,
 * half/quarter rings (with the optional batched sp_fc arms), seed restore.
 * The me_wide rescue grid (Quality preset only) is not part of this path. */
void or_motion_search(const or_me_frame *fr, const or_me_params *pr, int lx, int ly, int rw, int rh,
                      const int32_t *preds, int npred, double lambda_me, const int32_t *start, or_me_result *out) {
    ms_ctx m;
    m.fr = fr; m.pr = pr; m.lx = lx; m.ly = ly; m.rw = rw; m.rh = rh;
    m.cx = preds[0]; m.cy = preds[1];
    m.lambda_me = lambda_me;
    m.lam_r = pr->mv_cost_kind != 0 ? lambda_me * 0.25 : lambda_me;
    int refine_only = start != NULL;
    m.sadfp = !pr->fast && !refine_only && pr->sadfp;
    m.lam_fp = lambda_me * (m.sadfp ? pr->sadfp_lambda : 1.0);
    m.use_sad = pr->fast && !pr->mb_use_satd;
    m.use_planes = !pr->fast;
    m.evals = 0;
    int cw = fr->cw, ch = fr->ch;
    const uint8_t *src = fr->src + (int64_t)ly * cw + lx;

    int32_t bx_ = 0, by_ = 0;
    int64_t best_c;
    if (refine_only) {
        bx_ = start[0]; by_ = start[1];
        best_c = ms_cost(&m, bx_, by_);
    } else {
        best_c = ms_cost_fp(&m, 0, 0);
        for (int i = 0; i < npred; i++) {
            int64_t pc = ms_cost_fp(&m, preds[2 * i], preds[2 * i + 1]);
            if (pc < best_c) { best_c = pc; bx_ = preds[2 * i]; by_ = preds[2 * i + 1]; }
        }
    }
    int32_t seed_x = bx_, seed_y = by_;
    int64_t seed_c = best_c;
    if (!refine_only && pr->me_snap && ((bx_ & 3) != 0 || (by_ & 3) != 0)) {
        int32_t sx = ((bx_ + 2) >> 2) * 4, sy = ((by_ + 2) >> 2) * 4; /* div_euclid by 4 */
        best_c = ms_cost_fp(&m, sx, sy);
        bx_ = sx; by_ = sy;
    }
    /* ladder */
    int32_t steps[5];
    int nsteps = 0;
    if (pr->fast) {
        steps[0] = 16; steps[1] = 4; nsteps = 2;
    } else {
        uint32_t mask = (rw < 8 || rh < 8) ? pr->dia_sub_mask : pr->dia_mask;
        for (int i = 0; i < 5; i++)
            if (mask & (1u << i)) steps[nsteps++] = DIA_RUNGS[i];
    }
    int x4shape = (rw == 16 || rw == 8) && (rh == 16 || rh == 8);
    int fc = !pr->fast && pr->me_fc && x4shape;
    for (int si = 0; si < nsteps && !refine_only; si++) {
        int32_t step = steps[si];
        for (;;) {
            if (fc && (bx_ & 3) == 0 && (by_ & 3) == 0) {
                int s = step >> 2;
                int bx = lx + (bx_ >> 2), by = ly + (by_ >> 2);
                if (bx - s >= 0 && by - s >= 0 && bx + s + rw <= cw && by + s + rh <= ch) {
                    static const int RX[4] = {1, -1, 0, 0}, RY[4] = {0, 0, 1, -1};
                    int bi = -1;
                    int64_t bc = best_c;
                    for (int i = 0; i < 4; i++) {
                        int32_t mx = bx_ + RX[i] * step, my = by_ + RY[i] * step;
                        int64_t cc;
                        if (rw == 16) { /* sad_x4 / satd_x4 batch, priced with lam_fp */
                            const uint8_t *r = fr->ref + (int64_t)(by + RY[i] * s) * cw + bx + RX[i] * s;
                            int64_t d = m.sadfp ? (int64_t)or_sad(src, cw, r, cw, rw, rh) : or_satd_px(src, cw, r, cw, rw, rh);
                            m.evals++;
                            cc = d + (int64_t)(m.lam_fp * (double)ms_rate(&m, mx, my));
                        } else {
                            cc = ms_cost_fp(&m, mx, my);
                        }
                        if (cc < bc) { bc = cc; bi = i; }
                    }
                    if (bi < 0) break;
                    best_c = bc;
                    bx_ += RX[bi] * step; by_ += RY[bi] * step;
                    continue;
                }
            }
            int improved = 0;
            const int32_t rx[4] = {step, -step, 0, 0}, ry[4] = {0, 0, step, -step};
            for (int i = 0; i < 4; i++) {
                int32_t cx = bx_ + rx[i], cy = by_ + ry[i];
                int64_t cc = ms_cost_fp(&m, cx, cy);
                if (cc < best_c) { best_c = cc; bx_ = cx; by_ = cy; improved = 1; }
            }
            if (!improved) break;
        }
    }
    if (m.sadfp) {
        best_c = ms_cost(&m, bx_, by_);
        seed_c = ms_cost(&m, seed_x, seed_y);
    }
    /* sub-pel (mb16.rs:2956-3283) */
    if (pr->subpel) {
        int sub_shape = rw < 8 || rh < 8;
        int pat = pr->subpel_pat >= 0 ? pr->subpel_pat : (sub_shape ? pr->sub_pat : (pr->sp_single_pass ? 2 : 0));
        int sp_fc = pr->sp_fc && !pr->fast && x4shape;
        static const int32_t SPSTEPS[2] = {2, 1};
        for (int k = 0; k < 2; k++) {
            int32_t step = SPSTEPS[k];
            const int32_t r8x[8] = {step, -step, 0, 0, step, -step, step, -step};
            const int32_t r8y[8] = {0, 0, step, -step, step, -step, -step, step};
            int nring = (pat & 1) ? 4 : 8;
            int iter = 0;
            for (;;) {
                if (sp_fc && (pat & 1) == 0 &&
                    (step == 1 || ((bx_ & 3) == 0 && (by_ & 3) == 0))) {
                    iter++;
                    int all = 1;
                    int pa[8], pb[8];
                    int64_t oa[8], ob[8];
                    for (int i = 0; i < 8 && all; i++) {
                        if (step == 1)
                            all = or_hpel_qpel_refs(&fr->planes, lx, ly, rw, rh, bx_ + r8x[i], by_ + r8y[i], &pa[i], &oa[i], &pb[i], &ob[i]);
                        else
                            all = or_hpel_ref(&fr->planes, lx, ly, rw, rh, bx_ + r8x[i], by_ + r8y[i], &pa[i], &oa[i]);
                    }
                    if (all) {
                        int bi = -1;
                        int64_t bc = best_c;
                        for (int i = 0; i < 8; i++) {
                            int32_t mx = bx_ + r8x[i], my = by_ + r8y[i];
                            int64_t cc;
                            if (rw == 16) { /* satd_avg_x4 / satd_x4p batch, priced with lambda_me */
                                int64_t d = step == 1
                                    ? (int64_t)or_satd_avg(src, cw, plane_ptr(&fr->planes, pa[i]) + oa[i],
                                                           plane_ptr(&fr->planes, pb[i]) + ob[i], fr->planes.pw, rw, rh)
                                    : or_satd_px(src, cw, plane_ptr(&fr->planes, pa[i]) + oa[i], fr->planes.pw, rw, rh);
                                m.evals++;
                                cc = d + (int64_t)(m.lambda_me * (double)ms_rate(&m, mx, my));
                            } else {
                                cc = ms_cost(&m, mx, my);
                            }
                            if (cc < bc) { bc = cc; bi = i; }
                        }
                        if (bi < 0 || !pr->me_subpel_iter || (pat & 2) || (pr->sp_maxit != 0 && iter >= pr->sp_maxit)) {
                            if (bi >= 0) { best_c = bc; bx_ += r8x[bi]; by_ += r8y[bi]; }
                            break;
                        }
                        best_c = bc; bx_ += r8x[bi]; by_ += r8y[bi];
                        continue;
                    }
                    iter--;
                }
                int improved = 0;
                iter++;
                for (int i = 0; i < nring; i++) {
                    int32_t cx = bx_ + r8x[i], cy = by_ + r8y[i];
                    int64_t cc = ms_cost(&m, cx, cy);
                    if (cc < best_c) { best_c = cc; bx_ = cx; by_ = cy; improved = 1; }
                }
                if (!improved || !pr->me_subpel_iter || (pat & 2) || (pr->sp_maxit != 0 && iter >= pr->sp_maxit)) break;
            }
        }
    }
    if (pr->me_snap && seed_c < best_c) { bx_ = seed_x; by_ = seed_y; best_c = seed_c; }
    out->mvx = bx_; out->mvy = by_; out->cost = best_c; out->evals = m.evals;
}

/* mc_chroma (inter.rs:1268-1361): eighth-pel bilinear of a bw x bh chroma
 * block, every tap read with clamped coordinates; the copy and tile fast
 * paths of the reference give the same values. */
void or_mc_chroma(const uint8_t *ref, int cw, int ch, int x0, int y0, int bw, int bh, int32_t mvx, int32_t mvy,
                  uint8_t *out) {
    int ix0 = x0 + (mvx >> 3), iy0 = y0 + (mvy >> 3);
    int fx = mvx & 7, fy = mvy & 7;
    int wa = (8 - fx) * (8 - fy), wb = fx * (8 - fy), wc = (8 - fx) * fy, wd = fx * fy;
    for (int dy = 0; dy < bh; dy++)
        for (int dx = 0; dx < bw; dx++) {
            int x = ix0 + dx, y = iy0 + dy;
            int xa = x < 0 ? 0 : (x > cw - 1 ? cw - 1 : x), xb = x + 1 < 0 ? 0 : (x + 1 > cw - 1 ? cw - 1 : x + 1);
            int ya = y < 0 ? 0 : (y > ch - 1 ? ch - 1 : y), yb = y + 1 < 0 ? 0 : (y + 1 > ch - 1 ? ch - 1 : y + 1);
            int v = wa * ref[ya * cw + xa] + wb * ref[ya * cw + xb] + wc * ref[yb * cw + xa] + wd * ref[yb * cw + xb];
            out[dy * bw + dx] = (uint8_t)((v + 32) >> 6);
        }
}

/* ---- plain-ME frame model --------------------------------------------------- */

typedef struct { int32_t mvx, mvy, ref_idx, coded; } blk4;

static or_mv_neighbor nb_get(const blk4 *g, int w4, int h4, int bx, int by) {
    or_mv_neighbor n = {0, 0, 0, -1};
    if (bx < 0 || by < 0 || bx >= w4 || by >= h4 || !g[by * w4 + bx].coded) return n;
    const blk4 *b = &g[by * w4 + bx];
    n.available = 1; n.mvx = b->mvx; n.mvy = b->mvy; n.ref_idx = b->ref_idx;
    return n;
}

/* mv_neighbors_block, mb16.rs:1871-1890. */
static void mv_neighbors_block(const blk4 *g, int w4, int h4, int pbx, int pby, int pwb, or_mv_neighbor nb[3]) {
    nb[0] = nb_get(g, w4, h4, pbx - 1, pby);
    nb[1] = nb_get(g, w4, h4, pbx, pby - 1);
    nb[2] = nb_get(g, w4, h4, pbx + pwb, pby - 1);
    if (!nb[2].available) nb[2] = nb_get(g, w4, h4, pbx - 1, pby - 1);
}

/* best_part, mb16.rs:4921-4960, single reference (ref_bits 0); start non-NULL:
 * a refine-only search from it (the learned search's partitions). */
static void best_part1s(const or_me_frame *fr, const or_me_params *pr, const or_mv_neighbor nb[3], int rx, int ry,
                        int rw, int rh, const int32_t *extra, int nextra, double lme, const int32_t *start,
                        or_me_result *res) {
    int32_t seeds[8];
    or_predict_mv(&nb[0], &nb[1], &nb[2], 0, seeds);
    for (int i = 0; i < nextra; i++) { seeds[2 + 2 * i] = extra[2 * i]; seeds[3 + 2 * i] = extra[2 * i + 1]; }
    or_motion_search(fr, pr, rx, ry, rw, rh, seeds, 1 + nextra, lme, start, res);
}
static void best_part1(const or_me_frame *fr, const or_me_params *pr, const or_mv_neighbor nb[3], int rx, int ry, int rw,
                       int rh, const int32_t *extra, int nextra, double lme, or_me_result *res) {
    best_part1s(fr, pr, nb, rx, ry, rw, rh, extra, nextra, lme, NULL, res);
}

/* The learned-proposal 16x16 search (no counterpart in the reference): price
 * the median predictor and the MB's 8 proposals with motion_search's `cost`
 * closure (mb16.rs:2540-2566, mvd centre = the predictor); if the cheapest
 * proposal's distortion exceeds the predictor's by more than prop_t, run the
 * plain search (*fell = 1), else motion_search with the cheapest of the nine
 * (first wins, the predictor first) as its start vector (mb16.rs:2445). */
static void learned_16x16(const or_me_frame *fr, const or_me_params *pr, const or_mv_neighbor nb[3], int lx, int ly,
                          double lme, const int32_t *props, int32_t prop_t, or_me_result *res, int32_t *fell) {
    int32_t pmv[2];
    or_predict_mv(&nb[0], &nb[1], &nb[2], 0, pmv);
    const double lam_r = pr->mv_cost_kind != 0 ? lme * 0.25 : lme;
    int32_t cand[9][2];
    cand[0][0] = pmv[0]; cand[0][1] = pmv[1];
    for (int i = 0; i < 8; i++) { cand[i + 1][0] = props[2 * i]; cand[i + 1][1] = props[2 * i + 1]; }
    int bi = 0, bp = 1;
    int64_t cbest = 0, cprop = 0, dist[9];
    for (int i = 0; i < 9; i++) {
        uint32_t rate = or_mvbits(pr->mv_cost_kind, pr->mv_cost_tab, cand[i][0] - pmv[0]) +
                        or_mvbits(pr->mv_cost_kind, pr->mv_cost_tab, cand[i][1] - pmv[1]);
        dist[i] = or_mc_satd_hp(fr, 1, lx, ly, 16, 16, cand[i][0], cand[i][1]);
        int64_t c = dist[i] + (int64_t)(lam_r * (double)rate);
        if (i == 0 || c < cbest) { cbest = c; bi = i; }
        if (i == 1 || (i > 1 && c < cprop)) { cprop = c; bp = i; }
    }
    *fell = dist[bp] > dist[0] + prop_t;
    if (*fell) or_motion_search(fr, pr, lx, ly, 16, 16, pmv, 1, lme, NULL, res);
    else or_motion_search(fr, pr, lx, ly, 16, 16, pmv, 1, lme, cand[bi], res);
}

void or_me_frame_learned(const or_me_frame *fr, const or_me_params *pr, double lambda_me, int64_t split_gate,
                         const int32_t *props, int32_t prop_t, or_mb_pick *out, int32_t *fell);

void or_me_frame_plain(const or_me_frame *fr, const or_me_params *pr, double lambda_me, int64_t split_gate,
                       or_mb_pick *out) {
    or_me_frame_learned(fr, pr, lambda_me, split_gate, NULL, 0, out, NULL);
}

/* or_me_frame_plain, with the learned 16x16 search when props (16 i32 per MB)
 * is given; fell (optional) receives each MB's fallback flag. */
void or_me_frame_learned(const or_me_frame *fr, const or_me_params *pr, double lambda_me, int64_t split_gate,
                         const int32_t *props, int32_t prop_t, or_mb_pick *out, int32_t *fell) {
    int mb_w = fr->cw / 16, mb_h = fr->ch / 16;
    int w4 = mb_w * 4, h4 = mb_h * 4;
    blk4 *g = (blk4 *)calloc((size_t)w4 * h4, sizeof(blk4));
    for (int mby = 0; mby < mb_h; mby++)
        for (int mbx = 0; mbx < mb_w; mbx++) {
            int lx = mbx * 16, ly = mby * 16;
            or_mv_neighbor nb[3];
            mv_neighbors_block(g, w4, h4, mbx * 4, mby * 4, 4, nb);
            or_me_result r16;
            int32_t f = 1;
            if (props) {
                learned_16x16(fr, pr, nb, lx, ly, lambda_me, props + 16 * (mby * mb_w + mbx), prop_t, &r16, &f);
                if (fell) fell[mby * mb_w + mbx] = f;
            } else {
                best_part1(fr, pr, nb, lx, ly, 16, 16, NULL, 0, lambda_me, &r16);
            }
            or_mb_pick *pk = &out[mby * mb_w + mbx];
            pk->shape = 0;
            pk->mv[0][0] = pk->mv[1][0] = r16.mvx;
            pk->mv[0][1] = pk->mv[1][1] = r16.mvy;
            pk->cost = r16.cost;
            pk->cost16 = r16.cost;
            pk->mv16[0] = r16.mvx; pk->mv16[1] = r16.mvy;
            if (split_gate >= 0 && r16.cost > split_gate) {
                int32_t e[2] = {r16.mvx, r16.mvy};
                /* the learned search, when its 16x16 search took a proposal:
                 * the partitions refine-only from the 16x16 MV */
                const int32_t *st = props && !f ? e : NULL;
                or_me_result rt, rb, rl, rr;
                best_part1s(fr, pr, nb, lx, ly, 16, 8, e, 1, lambda_me, st, &rt);
                best_part1s(fr, pr, nb, lx, ly + 8, 16, 8, e, 1, lambda_me, st, &rb);
                best_part1s(fr, pr, nb, lx, ly, 8, 16, e, 1, lambda_me, st, &rl);
                best_part1s(fr, pr, nb, lx + 8, ly, 8, 16, e, 1, lambda_me, st, &rr);
                int64_t best_c = r16.cost;
                if (rt.cost + rb.cost < best_c) {
                    best_c = rt.cost + rb.cost;
                    pk->shape = 1;
                    pk->mv[0][0] = rt.mvx; pk->mv[0][1] = rt.mvy; pk->mv[1][0] = rb.mvx; pk->mv[1][1] = rb.mvy;
                }
                if (rl.cost + rr.cost < best_c) {
                    best_c = rl.cost + rr.cost;
                    pk->shape = 2;
                    pk->mv[0][0] = rl.mvx; pk->mv[0][1] = rl.mvy; pk->mv[1][0] = rr.mvx; pk->mv[1][1] = rr.mvy;
                }
                pk->cost = best_c;
            }
            /* commit the pick onto the 4x4 grid (mb16.rs:1850-1866 shape) */
            for (int dy = 0; dy < 4; dy++)
                for (int dx = 0; dx < 4; dx++) {
                    int part = pk->shape == 1 ? (dy >= 2) : (pk->shape == 2 ? (dx >= 2) : 0);
                    blk4 *b = &g[(mby * 4 + dy) * w4 + mbx * 4 + dx];
                    b->mvx = pk->mv[part][0]; b->mvy = pk->mv[part][1]; b->ref_idx = 0; b->coded = 1;
                }
        }
    free(g);
}

/* ref_bits (mb16.rs:5967-5981): the bits of ref_idx r among nref references,
 * te(v): none for one reference, one bit for two, ue(r) beyond. */
static uint32_t ref_bits(int r, int nref) {
    if (nref <= 1) return 0;
    if (nref == 2) return 1;
    uint32_t n = (uint32_t)r + 1, len = 1;
    while (n > 1) { n >>= 1; len += 2; }
    return len;
}

/* best_part (mb16.rs:4921-4960) over nref references: per reference r the
 * seeds [predict_mv(a, b, c, r), extra...], motion_search on that reference,
 * the cost plus (lme * ref_bits) truncated to i64, the lowest cost kept
 * (strictly lower; references in order). */
static void best_part_mr(const or_me_frame *frs, int nref, const or_me_params *pr, const or_mv_neighbor nb[3],
                         int rx, int ry, int rw, int rh, const int32_t *extra, int nextra, double lme, int32_t *ref,
                         or_me_result *res) {
    int64_t bc = INT64_MAX;
    for (int r = 0; r < nref; r++) {
        int32_t seeds[8];
        or_predict_mv(&nb[0], &nb[1], &nb[2], r, seeds);
        for (int i = 0; i < nextra; i++) { seeds[2 + 2 * i] = extra[2 * i]; seeds[3 + 2 * i] = extra[2 * i + 1]; }
        or_me_result o;
        or_motion_search(&frs[r], pr, rx, ry, rw, rh, seeds, 1 + nextra, lme, NULL, &o);
        const int64_t c = o.cost + (int64_t)(lme * (double)ref_bits(r, nref));
        if (c < bc) {
            bc = c;
            *ref = r;
            *res = o;
            res->cost = c;
        }
    }
}

/* The plain-ME frame model over nref references (the frame's frs[0..nref),
 * reference 0 the nearest): as or_me_frame_plain, each partition's search
 * best_part over the references, the neighbours' reference indices feeding
 * predict_mv (an MV predicts only from neighbours of the same reference,
 * inter.rs:36-69).  Picks: shape, ref_idx and MV of each half, costs. */
void or_me_frame_multiref(const or_me_frame *frs, int nref, const or_me_params *pr, double lambda_me,
                          int64_t split_gate, or_mb_pick_mr *out) {
    const or_me_frame *fr = &frs[0];
    int mb_w = fr->cw / 16, mb_h = fr->ch / 16;
    int w4 = mb_w * 4, h4 = mb_h * 4;
    blk4 *g = (blk4 *)calloc((size_t)w4 * h4, sizeof(blk4));
    for (int mby = 0; mby < mb_h; mby++)
        for (int mbx = 0; mbx < mb_w; mbx++) {
            int lx = mbx * 16, ly = mby * 16;
            or_mv_neighbor nb[3];
            mv_neighbors_block(g, w4, h4, mbx * 4, mby * 4, 4, nb);
            or_me_result r16 = {0, 0, 0, 0};
            int32_t ref16 = 0;
            best_part_mr(frs, nref, pr, nb, lx, ly, 16, 16, NULL, 0, lambda_me, &ref16, &r16);
            or_mb_pick_mr *pk = &out[mby * mb_w + mbx];
            pk->shape = 0;
            pk->ref[0] = pk->ref[1] = ref16;
            pk->mv[0][0] = pk->mv[1][0] = r16.mvx;
            pk->mv[0][1] = pk->mv[1][1] = r16.mvy;
            pk->cost = pk->cost16 = r16.cost;
            if (split_gate >= 0 && r16.cost > split_gate) {
                int32_t e[2] = {r16.mvx, r16.mvy}, rf[4] = {0, 0, 0, 0};
                or_me_result rp[4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}};
                best_part_mr(frs, nref, pr, nb, lx, ly, 16, 8, e, 1, lambda_me, &rf[0], &rp[0]);
                best_part_mr(frs, nref, pr, nb, lx, ly + 8, 16, 8, e, 1, lambda_me, &rf[1], &rp[1]);
                best_part_mr(frs, nref, pr, nb, lx, ly, 8, 16, e, 1, lambda_me, &rf[2], &rp[2]);
                best_part_mr(frs, nref, pr, nb, lx + 8, ly, 8, 16, e, 1, lambda_me, &rf[3], &rp[3]);
                int64_t best_c = r16.cost;
                for (int sh = 1; sh <= 2; sh++) {
                    const int a = sh == 1 ? 0 : 2;
                    if (rp[a].cost + rp[a + 1].cost < best_c) {
                        best_c = rp[a].cost + rp[a + 1].cost;
                        pk->shape = sh;
                        for (int k = 0; k < 2; k++) {
                            pk->ref[k] = rf[a + k];
                            pk->mv[k][0] = rp[a + k].mvx;
                            pk->mv[k][1] = rp[a + k].mvy;
                        }
                    }
                }
                pk->cost = best_c;
            }
            for (int dy = 0; dy < 4; dy++)
                for (int dx = 0; dx < 4; dx++) {
                    int part = pk->shape == 1 ? (dy >= 2) : (pk->shape == 2 ? (dx >= 2) : 0);
                    blk4 *b = &g[(mby * 4 + dy) * w4 + mbx * 4 + dx];
                    b->mvx = pk->mv[part][0]; b->mvy = pk->mv[part][1]; b->ref_idx = pk->ref[part]; b->coded = 1;
                }
        }
    free(g);
}

/* Exhaustive full-pel SAD and SATD over ±R of MB (mbx,mby), values as the ME
 * cost functions return them (mc_sad_hp / mc_satd_hp at full-pel MVs: edge reads
 * clamp).  Grid layout: (dy+R)*(2R+1) + (dx+R). */
void or_fullpel_grid_mb(const or_me_frame *fr, int mbx, int mby, int R, int32_t *sad_grid, int32_t *satd_grid) {
    int n = 2 * R + 1;
    for (int dy = -R; dy <= R; dy++)
        for (int dx = -R; dx <= R; dx++) {
            int idx = (dy + R) * n + (dx + R);
            if (sad_grid) sad_grid[idx] = (int32_t)or_mc_sad_hp(fr, 1, mbx * 16, mby * 16, 16, 16, dx * 4, dy * 4);
            if (satd_grid) satd_grid[idx] = (int32_t)or_mc_satd_hp(fr, 1, mbx * 16, mby * 16, 16, 16, dx * 4, dy * 4);
        }
}

/* ======================================================================== */
/* mb-tree lookahead (crates/rusty_h264-encoder/src/mbtree.rs)               */
/* ======================================================================== */

/* downsample2x, mbtree.rs:61-74. */
void or_downsample2x(const uint8_t *y, int cw, int ch, uint8_t *out) {
    int hw = cw / 2, hh = ch / 2;
    for (int j = 0; j < hh; j++)
        for (int i = 0; i < hw; i++) {
            uint32_t s = (uint32_t)y[2 * j * cw + 2 * i] + y[2 * j * cw + 2 * i + 1] + y[(2 * j + 1) * cw + 2 * i] +
                         y[(2 * j + 1) * cw + 2 * i + 1];
            out[j * hw + i] = (uint8_t)((s + 2) / 4);
        }
}

/* intra_cost, mbtree.rs:78-93: Σ|Hadamard AC| (DC excluded), at least 1. */
int32_t or_intra_cost(const uint8_t *sy, int cw, int bx0, int by0, int bs) {
    int64_t s = 0;
    for (int by = 0; by < bs / 4; by++)
        for (int bx = 0; bx < bs / 4; bx++) {
            int32_t blk[16], h[16];
            for (int dy = 0; dy < 4; dy++)
                for (int dx = 0; dx < 4; dx++) blk[dy * 4 + dx] = sy[(by0 + by * 4 + dy) * cw + bx0 + bx * 4 + dx];
            or_hadamard_4x4(blk, h);
            for (int k = 1; k < 16; k++) s += iabs32(h[k]);
        }
    if (s > INT32_MAX) s = INT32_MAX;
    return s < 1 ? 1 : (int32_t)s;
}

/* mc_satd, mbtree.rs:102-152. */
int64_t or_la_mc_satd(const uint8_t *sy, int cw, int ch, const uint8_t *ref, int bx0, int by0, int bs, int mvx, int mvy) {
    int ix = bx0 + (mvx >> 2), iy = by0 + (mvy >> 2);
    if ((mvx & 3) == 0 && (mvy & 3) == 0 && ix >= 0 && iy >= 0 && ix + bs <= cw && iy + bs <= ch && by0 + bs <= ch &&
        bx0 + bs <= cw)
        return or_satd_px(sy + (int64_t)by0 * cw + bx0, cw, ref + (int64_t)iy * cw + ix, cw, bs, bs);
    uint8_t pred[256];
    or_mc_luma(ref, cw, ch, bx0, by0, bs, bs, mvx, mvy, pred);
    return satd_px_scalar(sy + (int64_t)by0 * cw + bx0, cw, pred, bs, bs, bs);
}

/* inter_cost, mbtree.rs:154-197. */
void or_inter_cost(const uint8_t *sy, int cw, int ch, const uint8_t *ref, int bx0, int by0, int bs, int seedx, int seedy,
                   int max_step, int32_t *cost, int32_t mv[2], int32_t *evals) {
    int32_t bmx = 0, bmy = 0;
    int32_t ev = 1;
    int64_t best = or_la_mc_satd(sy, cw, ch, ref, bx0, by0, bs, 0, 0);
    if (best != 0) {
        if (seedx != 0 || seedy != 0) {
            int64_t s = or_la_mc_satd(sy, cw, ch, ref, bx0, by0, bs, seedx, seedy);
            ev++;
            if (s < best) { best = s; bmx = seedx; bmy = seedy; }
        }
        for (int step = max_step; step >= 1; step >>= 1) {
            for (;;) {
                int moved = 0;
                const int dxs[4] = {step, -step, 0, 0}, dys[4] = {0, 0, step, -step};
                for (int i = 0; i < 4; i++) {
                    int32_t mx = bmx + dxs[i] * 4, my = bmy + dys[i] * 4;
                    int64_t s = or_la_mc_satd(sy, cw, ch, ref, bx0, by0, bs, mx, my);
                    ev++;
                    if (s < best) { best = s; bmx = mx; bmy = my; moved = 1; }
                }
                if (!moved) break;
            }
        }
    }
    if (best > INT32_MAX) best = INT32_MAX;
    *cost = (int32_t)best;
    mv[0] = bmx; mv[1] = bmy;
    if (evals) *evals = ev;
}

/* frame_costs, mbtree.rs:208-263. */
void or_frame_costs(const uint8_t *full, int cwf, int chf, const uint8_t *half, int cwh, int chh, int mb_w, int mb_h,
                    const uint8_t *ref_full, const uint8_t *ref_half, int mode, int32_t *intra, int32_t *inter,
                    int32_t *mvs) {
    for (int mby = 0; mby < mb_h; mby++)
        for (int mbx = 0; mbx < mb_w; mbx++) {
            int m = mby * mb_w + mbx;
            int32_t sfx = 0, sfy = 0;
            if (mbx > 0) { sfx = mvs[2 * (m - 1)]; sfy = mvs[2 * (m - 1) + 1]; }
            else if (mby > 0) { sfx = mvs[2 * (m - mb_w)]; sfy = mvs[2 * (m - mb_w) + 1]; }
            int32_t ic = mode == 2 ? or_intra_cost(half, cwh, mbx * 8, mby * 8, 8)
                                   : or_intra_cost(full, cwf, mbx * 16, mby * 16, 16);
            int32_t cost, mv[2] = {0, 0};
            if (mode == 0 && ref_full) {
                or_inter_cost(full, cwf, chf, ref_full, mbx * 16, mby * 16, 16, sfx, sfy, 8, &cost, mv, NULL);
            } else if (mode == 2 && ref_half) {
                int32_t mvp[2];
                or_inter_cost(half, cwh, chh, ref_half, mbx * 8, mby * 8, 8, sfx / 2, sfy / 2, 8, &cost, mvp, NULL);
                mv[0] = mvp[0] * 2; mv[1] = mvp[1] * 2;
            } else if (mode == 1 && ref_full && ref_half) {
                int32_t mvp[2];
                or_inter_cost(half, cwh, chh, ref_half, mbx * 8, mby * 8, 8, sfx / 2, sfy / 2, 8, &cost, mvp, NULL);
                or_inter_cost(full, cwf, chf, ref_full, mbx * 16, mby * 16, 16, mvp[0] * 2, mvp[1] * 2, 2, &cost, mv, NULL);
            } else {
                cost = ic;
            }
            intra[m] = ic;
            inter[m] = cost < ic ? cost : ic;
            mvs[2 * m] = mv[0];
            mvs[2 * m + 1] = mv[1];
        }
}
