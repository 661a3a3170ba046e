// tq_device.cuh -- the forward 4x4 transform + quantisation of one block
// (dct_four_t4 + quant_four_4x4, crates/rusty_h264-accel/src/
// transform_quant.rs:71-135) and its quant tables, shared by the T/Q kernels
// and by the plain-ME kernel, which can run an MB's MC + T/Q right after its
// pick.
#pragma once

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

}  // namespace h264a
