// deblock_device.cuh -- the in-loop deblocking filter of one MB
// (crates/rusty_h264-common/src/deblock.rs) on shared-memory tiles, shared by
// the deblocking kernel and the closed loop's fused motion-search kernel, and
// the per-picture thresholds the host derives for it.
//
// Pictures of this path: every MB inter with reference 0, 4x4 transforms, one
// QP per picture.  bS (bs_inter and the single-list arm of bs1_tile,
// deblock.rs:328-333, 396-404) is 2 with coefficients on either side, else 1
// when the two blocks' MVs differ by 4 quarter-pels in x or y, else 0.
#pragma once

#include <algorithm>

#include "h264a_device.cuh"

namespace h264a {

// Spec Tables 8-16/8-17 as deblock.rs:11-41 holds them: alpha and beta by
// indexA / indexB, tc0 by [indexA][bS-1].
static const int kAlpha[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,   0,   0,   0,   0,   0,   0,   4,   4,
                               5,  6,  7,  8,  9,  10, 12, 13, 15, 17,  20,  22,  25,  28,  32,  36,  40,  45,
                               50, 56, 63, 71, 80, 90, 101, 113, 127, 144, 162, 182, 203, 226, 255, 255};
static const int kBeta[52] = {0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  0,  0,  0,  2,  2,  2,  3,  3,  3,  3,  4,  4,  4,
                              6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18};
static const int kTc0[52][3] = {
    {0, 0, 0},  {0, 0, 0},  {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},
    {0, 0, 0},  {0, 0, 0},  {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},
    {0, 0, 0},  {0, 0, 1},  {0, 0, 1},   {0, 0, 1},   {0, 0, 1},   {0, 1, 1},   {0, 1, 1},   {1, 1, 1},
    {1, 1, 1},  {1, 1, 1},  {1, 1, 1},   {1, 1, 2},   {1, 1, 2},   {1, 1, 2},   {1, 1, 2},   {1, 2, 3},
    {1, 2, 3},  {2, 2, 3},  {2, 2, 4},   {2, 3, 4},   {2, 3, 4},   {3, 3, 5},   {3, 4, 6},   {3, 4, 6},
    {4, 5, 7},  {4, 5, 8},  {4, 6, 9},   {5, 7, 10},  {6, 8, 11},  {6, 8, 13},  {7, 10, 14}, {8, 11, 16},
    {9, 12, 18}, {10, 13, 20}, {11, 15, 23}, {13, 17, 25}};

// Alpha, beta and tc0 of one picture (deblock.rs:1921-1929; MB edges average
// two equal QPs, so the picture QP indexes the tables).
struct DbThresh {
    int alpha_y, beta_y, alpha_c, beta_c;
    int tc_y[3], tc_c[3];
};

// chroma_qp (predict.rs:64-73).
static inline int chroma_qp_of(int qp) {
    static const int kQpc[22] = {29, 30, 31, 32, 32, 33, 34, 34, 35, 35, 36, 36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39};
    return qp < 30 ? qp : kQpc[qp - 30];
}

static inline DbThresh db_thresholds(int qp, int offset_a, int offset_b, int chroma_qp_offset) {
    DbThresh d;
    const int ia = std::min(std::max(qp + offset_a, 0), 51), ib = std::min(std::max(qp + offset_b, 0), 51);
    const int qpc = chroma_qp_of(std::min(std::max(qp + chroma_qp_offset, 0), 51));
    const int ica = std::min(std::max(qpc + offset_a, 0), 51), icb = std::min(std::max(qpc + offset_b, 0), 51);
    d.alpha_y = kAlpha[ia];
    d.beta_y = kBeta[ib];
    d.alpha_c = kAlpha[ica];
    d.beta_c = kBeta[icb];
    for (int q = 0; q < 3; q++) {
        d.tc_y[q] = kTc0[ia][q];
        d.tc_c[q] = kTc0[ica][q];
    }
    return d;
}

constexpr int LT = 20;            // luma tile: 20 x 20 (stride 20), the MB at (4, 4)
constexpr int CT = 12, CR = 10;   // chroma tile: 10 rows x 12 (stride 12), the MB at (2, 4)

__device__ __forceinline__ int clip1(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
__device__ __forceinline__ int clip3(int lo, int hi, int v) { return v < lo ? lo : (v > hi ? hi : v); }

// filter_luma_line (deblock.rs:67-115) on shared bytes: q0 at q, samples
// `step` apart.
__device__ __forceinline__ void luma_line(uint8_t* q, int step, int bs, int alpha, int beta, int tc0) {
    const int p0 = q[-step], p1 = q[-2 * step], p2 = q[-3 * step], p3 = q[-4 * step];
    const int q0 = q[0], q1 = q[step], q2 = q[2 * step], q3 = q[3 * step];
    if (abs(p0 - q0) >= alpha || abs(p1 - p0) >= beta || abs(q1 - q0) >= beta) return;
    const int ap = abs(p2 - p0), aq = abs(q2 - q0);
    if (bs < 4) {
        const int tc = tc0 + (ap < beta) + (aq < beta);
        const int delta = clip3(-tc, tc, (((q0 - p0) << 2) + (p1 - q1) + 4) >> 3);
        q[-step] = uint8_t(clip1(p0 + delta));
        q[0] = uint8_t(clip1(q0 - delta));
        if (ap < beta) q[-2 * step] = uint8_t(clip1(p1 + clip3(-tc0, tc0, (p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1)));
        if (aq < beta) q[step] = uint8_t(clip1(q1 + clip3(-tc0, tc0, (q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1)));
    } else {
        const bool strong = abs(p0 - q0) < (alpha >> 2) + 2;
        if (strong && ap < beta) {
            q[-step] = uint8_t(clip1((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3));
            q[-2 * step] = uint8_t(clip1((p2 + p1 + p0 + q0 + 2) >> 2));
            q[-3 * step] = uint8_t(clip1((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3));
        } else {
            q[-step] = uint8_t(clip1((2 * p1 + p0 + q1 + 2) >> 2));
        }
        if (strong && aq < beta) {
            q[0] = uint8_t(clip1((q2 + 2 * q1 + 2 * q0 + 2 * p0 + p1 + 4) >> 3));
            q[step] = uint8_t(clip1((q2 + q1 + q0 + p0 + 2) >> 2));
            q[2 * step] = uint8_t(clip1((2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3));
        } else {
            q[0] = uint8_t(clip1((2 * q1 + q0 + p1 + 2) >> 2));
        }
    }
}

// filter_chroma_line (deblock.rs:117-137).
__device__ __forceinline__ void chroma_line(uint8_t* q, int step, int bs, int alpha, int beta, int tc0) {
    const int p0 = q[-step], p1 = q[-2 * step], q0 = q[0], q1 = q[step];
    if (abs(p0 - q0) >= alpha || abs(p1 - p0) >= beta || abs(q1 - q0) >= beta) return;
    if (bs < 4) {
        const int tc = tc0 + 1;
        const int delta = clip3(-tc, tc, (((q0 - p0) << 2) + (p1 - q1) + 4) >> 3);
        q[-step] = uint8_t(clip1(p0 + delta));
        q[0] = uint8_t(clip1(q0 - delta));
    } else {
        q[-step] = uint8_t(clip1((2 * p1 + p0 + q1 + 2) >> 2));
        q[0] = uint8_t(clip1((2 * q1 + q0 + p1 + 2) >> 2));
    }
}

// MV and coefficient flag of 4x4 block (bx, by) of MB m (coefficients in the
// reference's dct[256] order: 8x8 region, then 4x4 sub-block), read through L2
// (the MB may have been written by another CTA of the same launch).
__device__ __forceinline__ void block_state_at(const int32_t* picks, const int16_t* coeffs, int m, int bx, int by,
                                               int& mvx, int& mvy, bool& nz) {
    const int32_t* pk = picks + 6 * m;
    const int shape = __ldcg(pk);
    const int part = shape == 1 ? (by >= 2) : (shape == 2 ? (bx >= 2) : 0);
    mvx = __ldcg(pk + 1 + 2 * part);
    mvy = __ldcg(pk + 2 + 2 * part);
    const int qi = (by >= 2 ? 2 : 0) + (bx >= 2 ? 1 : 0), k = (by & 1) * 2 + (bx & 1);
    const uint4* c = reinterpret_cast<const uint4*>(coeffs + (long long)m * 256 + (qi * 4 + k) * 16);
    const uint4 a = __ldcg(c), b = __ldcg(c + 1);
    nz = (a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w) != 0u;
}

// The bS of one MB's 32 edge segments from the two blocks' MVs and
// coefficient flags; e == 0 segments on the picture border have none.
__device__ __forceinline__ int bs_of(bool pnz, bool qnz, int pmx, int pmy, int qmx, int qmy) {
    return (pnz || qnz) ? 2 : ((abs(pmx - qmx) >= 4 || abs(pmy - qmy) >= 4) ? 1 : 0);
}

// Filters one MB held in shared tiles (the MB's samples and the left/top
// strips its edges reach), one warp: lanes 0..15 luma row / column `lane`
// through all four edges of a direction, lanes 16..31 chroma row / column
// lane & 7 of plane (lane >> 3) & 1 (luma edges 0 and 2).  bs[0..15] are the
// vertical edges (edge e = i / 4, block row i % 4), bs[16..31] the horizontal
// ones.  Vertical edges first, then horizontal (deblock.rs's per-MB order).
__device__ __forceinline__ void deblock_mb_tiles(int lane, uint8_t* lt, uint8_t* ct0, uint8_t* ct1, const int* bsw,
                                                 bool left, bool top, bool has_c, const DbThresh& th) {
    const int pl = (lane >> 3) & 1, li = lane & 7;
    uint8_t* ct = pl ? ct1 : ct0;
    if (lane < 16) {
        uint8_t* row = lt + (4 + lane) * LT + 4;
        for (int e = left ? 0 : 1; e < 4; e++) {
            const int bs = bsw[e * 4 + (lane >> 2)];
            if (bs) luma_line(row + 4 * e, 1, bs, th.alpha_y, th.beta_y, th.tc_y[bs - 1]);
        }
    } else if (has_c) {
        uint8_t* row = ct + (2 + li) * CT + 4;
        for (int ce = left ? 0 : 2; ce < 4; ce += 2) {
            const int bs = bsw[ce * 4 + (li >> 1)];
            if (bs) chroma_line(row + 2 * ce, 1, bs, th.alpha_c, th.beta_c, th.tc_c[bs - 1]);
        }
    }
    __syncwarp();
    if (lane < 16) {
        uint8_t* col = lt + 4 * LT + 4 + lane;
        for (int e = top ? 0 : 1; e < 4; e++) {
            const int bs = bsw[16 + e * 4 + (lane >> 2)];
            if (bs) luma_line(col + 4 * e * LT, LT, bs, th.alpha_y, th.beta_y, th.tc_y[bs - 1]);
        }
    } else if (has_c) {
        uint8_t* col = ct + 2 * CT + 4 + li;
        for (int ce = top ? 0 : 2; ce < 4; ce += 2) {
            const int bs = bsw[16 + ce * 4 + (li >> 1)];
            if (bs) chroma_line(col + 2 * ce * CT, CT, bs, th.alpha_c, th.beta_c, th.tc_c[bs - 1]);
        }
    }
    __syncwarp();
}

// One lane's word of an MB's left and top strips (the neighbours' samples its
// edges reach): luma left strip (lanes 0..15, row `lane`, columns -4..-1) and
// top strip (lanes 16..31, rows -4..-1); chroma left strips (lanes 0..15) and
// top strips (lanes 16..23).  Each word moves between the picture (through L2)
// and its place in the tiles.
struct DbStrips {
    unsigned int* lg;
    uint32_t* ls;
    unsigned int* cg;
    uint32_t* cs;
    bool lok, cok;
    __device__ __forceinline__ DbStrips(int lane, uint8_t* y, int cw, int x0, int y0, uint8_t* const uv[2], int cx0,
                                        int cy0, uint8_t* lt, uint8_t* ct0, uint8_t* ct1, bool left, bool top,
                                        bool has_c) {
        const int ccw = cw / 2;
        lok = lane < 16 ? left : top;
        const int lr = lane < 16 ? lane : ((lane - 16) >> 2) - 4, lc = lane < 16 ? -4 : (lane & 3) * 4;
        lg = reinterpret_cast<unsigned int*>(y + (long long)(y0 + lr) * cw + x0 + lc);
        ls = reinterpret_cast<uint32_t*>(lt + (4 + lr) * LT + 4 + lc);
        cok = has_c && lane < 24 && (lane < 16 ? left : top);
        const int cpl = lane < 16 ? lane >> 3 : (lane >> 2) & 1;
        const int cr = lane < 16 ? lane & 7 : ((lane >> 1) & 1) - 2, cc = lane < 16 ? -4 : (lane & 1) * 4;
        cg = cok ? reinterpret_cast<unsigned int*>(uv[cpl] + (long long)(cy0 + cr) * ccw + cx0 + cc) : nullptr;
        cs = reinterpret_cast<uint32_t*>((cpl ? ct1 : ct0) + (2 + cr) * CT + 4 + cc);
    }
    __device__ __forceinline__ void load() const {
        if (lok) *ls = __ldcg(lg);
        if (cok) *cs = __ldcg(cg);
    }
    __device__ __forceinline__ void store() const {
        if (lok) __stcg(lg, *ls);
        if (cok) __stcg(cg, *cs);
    }
};

// Writes an MB's filtered samples from its tiles back to the picture, one warp.
__device__ __forceinline__ void db_store_mb(int lane, const uint8_t* lt, const uint8_t* ct0, const uint8_t* ct1,
                                            uint8_t* y, int cw, int x0, int y0, uint8_t* const uv[2], int cx0, int cy0,
                                            bool has_c) {
    for (int i = lane; i < 64; i += 32) {
        const int r = i >> 2, c4 = (i & 3) * 4;
        __stcg(reinterpret_cast<unsigned int*>(y + (long long)(y0 + r) * cw + x0 + c4),
               *reinterpret_cast<const uint32_t*>(lt + (4 + r) * LT + 4 + c4));
    }
    if (has_c) {
        const int p = lane >> 4, r = (lane >> 1) & 7, c4 = (lane & 1) * 4;
        __stcg(reinterpret_cast<unsigned int*>(uv[p] + (long long)(cy0 + r) * (cw / 2) + cx0 + c4),
               *reinterpret_cast<const uint32_t*>((p ? ct1 : ct0) + (2 + r) * CT + 4 + c4));
    }
}

}  // namespace h264a
