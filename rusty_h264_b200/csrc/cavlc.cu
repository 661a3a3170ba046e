// cavlc.cu -- Annex-B H.264 Baseline stream of the frame model (host code).
//
// The pixel path's outputs become a decodable stream: frame 0 is an IDR
// picture of I_PCM macroblocks (the frame model codes it losslessly, so its
// reconstruction is the source), frames 1..n-1 are P pictures whose every MB
// is P_L0_16x16, P_L0_L0_16x8 or P_L0_L0_8x16 (reference 0) with its MVs
// coded against the spec's MV predictor and its luma/chroma levels coded with
// CAVLC.  The syntax follows the reference's writer: slice data and MB layer
// (crates/rusty_h264-encoder/src/mb16.rs:5266-5845, CAVLC P slices),
// residual blocks (crates/rusty_h264-common/src/cavlc.rs:485,
// encode_residual_block), coded_block_pattern (cavlc.rs:136), parameter sets
// and NAL framing (crates/rusty_h264-common/src/nal.rs).  The VLC tables are
// the standard's Tables 9-4, 9-5, 9-7, 9-8, 9-9 and 9-10.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "h264accel_internal.h"

namespace h264a {
namespace cavlc {

// ---- bit writer ---------------------------------------------------------------
struct Bits {
    std::vector<uint8_t> b;
    uint32_t cur = 0;
    int n = 0;  // bits in cur
    void put(uint32_t v, int len) {  // len <= 32
        for (int i = len - 1; i >= 0; i--) {
            cur = (cur << 1) | ((v >> i) & 1u);
            if (++n == 8) {
                b.push_back(uint8_t(cur));
                cur = 0;
                n = 0;
            }
        }
    }
    void ue(uint32_t v) {
        const uint64_t x = uint64_t(v) + 1;
        int len = 0;
        while ((x >> (len + 1)) != 0) len++;
        put(0, len);
        put(uint32_t(x), len + 1);
    }
    void se(int32_t v) { ue(v > 0 ? uint32_t(2 * int64_t(v) - 1) : uint32_t(-2 * int64_t(v))); }
    bool aligned() const { return n == 0; }
    void trailing() {  // rbsp_trailing_bits
        put(1, 1);
        while (n) put(0, 1);
    }
};

// NAL unit: start code, header, the RBSP with emulation prevention
void nal(std::vector<uint8_t>& out, int ref_idc, int type, const std::vector<uint8_t>& rbsp) {
    static const uint8_t sc[4] = {0, 0, 0, 1};
    out.insert(out.end(), sc, sc + 4);
    out.push_back(uint8_t((ref_idc << 5) | type));
    int zeros = 0;
    for (uint8_t c : rbsp) {
        if (zeros >= 2 && c <= 3) {
            out.push_back(3);
            zeros = 0;
        }
        out.push_back(c);
        zeros = c == 0 ? zeros + 1 : 0;
    }
}

// ---- tables -------------------------------------------------------------------
// Table 9-4 (4:2:0, inter column): codeNum of each coded_block_pattern.
const uint8_t CBP_INTER_CODE[48] = {
    0, 2, 3, 7, 4, 8, 17, 13, 5, 18, 9, 14, 10, 15, 16, 11, 1, 32, 33, 36, 34, 37, 44, 40,
    35, 45, 38, 41, 39, 42, 43, 19, 6, 24, 25, 20, 26, 21, 46, 28, 27, 47, 22, 29, 23, 30, 31, 12};

struct Code {
    uint8_t len, bits;
};
// Table 9-5, coeff_token: [nC class][TotalCoeff][TrailingOnes]; classes
// 0 <= nC < 2, 2 <= nC < 4, 4 <= nC < 8 (8 <= nC: 6-bit fixed length).
const Code COEFF_TOKEN[3][17][4] = {
    {{{1, 1}, {0, 0}, {0, 0}, {0, 0}},
     {{6, 5}, {2, 1}, {0, 0}, {0, 0}},
     {{8, 7}, {6, 4}, {3, 1}, {0, 0}},
     {{9, 7}, {8, 6}, {7, 5}, {5, 3}},
     {{10, 7}, {9, 6}, {8, 5}, {6, 3}},
     {{11, 7}, {10, 6}, {9, 5}, {7, 4}},
     {{13, 15}, {11, 6}, {10, 5}, {8, 4}},
     {{13, 11}, {13, 14}, {11, 5}, {9, 4}},
     {{13, 8}, {13, 10}, {13, 13}, {10, 4}},
     {{14, 15}, {14, 14}, {13, 9}, {11, 4}},
     {{14, 11}, {14, 10}, {14, 13}, {13, 12}},
     {{15, 15}, {15, 14}, {14, 9}, {14, 12}},
     {{15, 11}, {15, 10}, {15, 13}, {14, 8}},
     {{16, 15}, {15, 1}, {15, 9}, {15, 12}},
     {{16, 11}, {16, 14}, {16, 13}, {15, 8}},
     {{16, 7}, {16, 10}, {16, 9}, {16, 12}},
     {{16, 4}, {16, 6}, {16, 5}, {16, 8}}},
    {{{2, 3}, {0, 0}, {0, 0}, {0, 0}},
     {{6, 11}, {2, 2}, {0, 0}, {0, 0}},
     {{6, 7}, {5, 7}, {3, 3}, {0, 0}},
     {{7, 7}, {6, 10}, {6, 9}, {4, 5}},
     {{8, 7}, {6, 6}, {6, 5}, {4, 4}},
     {{8, 4}, {7, 6}, {7, 5}, {5, 6}},
     {{9, 7}, {8, 6}, {8, 5}, {6, 8}},
     {{11, 15}, {9, 6}, {9, 5}, {6, 4}},
     {{11, 11}, {11, 14}, {11, 13}, {7, 4}},
     {{12, 15}, {11, 10}, {11, 9}, {9, 4}},
     {{12, 11}, {12, 14}, {12, 13}, {11, 12}},
     {{12, 8}, {12, 10}, {12, 9}, {11, 8}},
     {{13, 15}, {13, 14}, {13, 13}, {12, 12}},
     {{13, 11}, {13, 10}, {13, 9}, {13, 12}},
     {{13, 7}, {14, 11}, {13, 6}, {13, 8}},
     {{14, 9}, {14, 8}, {14, 10}, {13, 1}},
     {{14, 7}, {14, 6}, {14, 5}, {14, 4}}},
    {{{4, 15}, {0, 0}, {0, 0}, {0, 0}},
     {{6, 15}, {4, 14}, {0, 0}, {0, 0}},
     {{6, 11}, {5, 15}, {4, 13}, {0, 0}},
     {{6, 8}, {5, 12}, {5, 14}, {4, 12}},
     {{7, 15}, {5, 10}, {5, 11}, {4, 11}},
     {{7, 11}, {5, 8}, {5, 9}, {4, 10}},
     {{7, 9}, {6, 14}, {6, 13}, {4, 9}},
     {{7, 8}, {6, 10}, {6, 9}, {4, 8}},
     {{8, 15}, {7, 14}, {7, 13}, {5, 13}},
     {{8, 11}, {8, 14}, {7, 10}, {6, 12}},
     {{9, 15}, {8, 10}, {8, 13}, {7, 12}},
     {{9, 11}, {9, 14}, {8, 9}, {8, 12}},
     {{9, 8}, {9, 10}, {9, 13}, {8, 8}},
     {{10, 13}, {9, 7}, {9, 9}, {9, 12}},
     {{10, 9}, {10, 12}, {10, 11}, {10, 10}},
     {{10, 5}, {10, 8}, {10, 7}, {10, 6}},
     {{10, 1}, {10, 4}, {10, 3}, {10, 2}}},
};
// chroma DC (nC == -1) coeff_token, [TotalCoeff 0..4][TrailingOnes]
const Code COEFF_TOKEN_CDC[5][4] = {{{2, 1}, {0, 0}, {0, 0}, {0, 0}},
                                    {{6, 7}, {1, 1}, {0, 0}, {0, 0}},
                                    {{6, 4}, {6, 6}, {3, 1}, {0, 0}},
                                    {{6, 3}, {7, 3}, {7, 2}, {6, 5}},
                                    {{6, 2}, {8, 3}, {8, 2}, {7, 0}}};
// Tables 9-7 and 9-8, total_zeros of 4x4 blocks: [TotalCoeff-1][total_zeros]
const Code TOTAL_ZEROS[15][16] = {
    {{1, 1}, {3, 3}, {3, 2}, {4, 3}, {4, 2}, {5, 3}, {5, 2}, {6, 3}, {6, 2}, {7, 3}, {7, 2}, {8, 3}, {8, 2}, {9, 3}, {9, 2}, {9, 1}},
    {{3, 7}, {3, 6}, {3, 5}, {3, 4}, {3, 3}, {4, 5}, {4, 4}, {4, 3}, {4, 2}, {5, 3}, {5, 2}, {6, 3}, {6, 2}, {6, 1}, {6, 0}},
    {{4, 5}, {3, 7}, {3, 6}, {3, 5}, {4, 4}, {4, 3}, {3, 4}, {3, 3}, {4, 2}, {5, 3}, {5, 2}, {6, 1}, {5, 1}, {6, 0}},
    {{5, 3}, {3, 7}, {4, 5}, {4, 4}, {3, 6}, {3, 5}, {3, 4}, {4, 3}, {3, 3}, {4, 2}, {5, 2}, {5, 1}, {5, 0}},
    {{4, 5}, {4, 4}, {4, 3}, {3, 7}, {3, 6}, {3, 5}, {3, 4}, {3, 3}, {4, 2}, {5, 1}, {4, 1}, {5, 0}},
    {{6, 1}, {5, 1}, {3, 7}, {3, 6}, {3, 5}, {3, 4}, {3, 3}, {3, 2}, {4, 1}, {3, 1}, {6, 0}},
    {{6, 1}, {5, 1}, {3, 5}, {3, 4}, {3, 3}, {2, 3}, {3, 2}, {4, 1}, {3, 1}, {6, 0}},
    {{6, 1}, {4, 1}, {5, 1}, {3, 3}, {2, 3}, {2, 2}, {3, 2}, {3, 1}, {6, 0}},
    {{6, 1}, {6, 0}, {4, 1}, {2, 3}, {2, 2}, {3, 1}, {2, 1}, {5, 1}},
    {{5, 1}, {5, 0}, {3, 1}, {2, 3}, {2, 2}, {2, 1}, {4, 1}},
    {{4, 0}, {4, 1}, {3, 1}, {3, 2}, {1, 1}, {3, 3}},
    {{4, 0}, {4, 1}, {2, 1}, {1, 1}, {3, 1}},
    {{3, 0}, {3, 1}, {1, 1}, {2, 1}},
    {{2, 0}, {2, 1}, {1, 1}},
    {{1, 0}, {1, 1}},
};
// Table 9-9a, chroma DC total_zeros: [TotalCoeff-1][total_zeros]
const Code TOTAL_ZEROS_CDC[3][4] = {{{1, 1}, {2, 1}, {3, 1}, {3, 0}}, {{1, 1}, {2, 1}, {2, 0}}, {{1, 1}, {1, 0}}};
// Table 9-10, run_before: [min(zerosLeft, 7) - 1][run_before]
const Code RUN_BEFORE[7][15] = {
    {{1, 1}, {1, 0}},
    {{1, 1}, {2, 1}, {2, 0}},
    {{2, 3}, {2, 2}, {2, 1}, {2, 0}},
    {{2, 3}, {2, 2}, {2, 1}, {3, 1}, {3, 0}},
    {{2, 3}, {2, 2}, {3, 3}, {3, 2}, {3, 1}, {3, 0}},
    {{2, 3}, {3, 0}, {3, 1}, {3, 3}, {3, 2}, {3, 5}, {3, 4}},
    {{3, 7}, {3, 6}, {3, 5}, {3, 4}, {3, 3}, {3, 2}, {3, 1}, {4, 1}, {5, 1}, {6, 1}, {7, 1}, {8, 1}, {9, 1}, {10, 1},
     {11, 1}},
};
// frame zigzag scan of a 4x4 block: raster index of scan position i
const uint8_t ZIGZAG[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};

// level_prefix >= 15 with its escape suffix: code is levelCode minus the
// (15 << suffixLength) (+15 when suffixLength is 0) that prefix 15 starts at
void put_escape(Bits& w, int64_t rem) {
    int prefix = 15;
    while (rem >= (1LL << (prefix - 3))) {  // prefixes beyond 15 lie outside Baseline conformance
        rem -= (1LL << (prefix - 3));
        prefix++;
    }
    w.put(0, prefix);
    w.put(1, 1);
    w.put(uint32_t(rem), prefix - 3);
}

// ---- residual_block (CAVLC) -----------------------------------------------------
// coeffs: maxc levels in scan order; nc: the coeff_token context (-1 chroma
// DC).  Returns TotalCoeff.
int residual_block(Bits& w, const int* coeffs, int maxc, int nc) {
    int nz[16], tc = 0;
    for (int i = 0; i < maxc; i++)
        if (coeffs[i]) nz[tc++] = i;
    int t1 = 0;
    for (int k = tc - 1; k >= 0 && t1 < 3; k--) {
        const int v = coeffs[nz[k]];
        if (v == 1 || v == -1) t1++;
        else break;
    }
    Code ct;
    if (nc == -1) ct = COEFF_TOKEN_CDC[tc][t1];
    else if (nc >= 8) ct = Code{6, uint8_t(tc == 0 ? 3 : (((tc - 1) << 2) | t1))};
    else ct = COEFF_TOKEN[nc < 2 ? 0 : (nc < 4 ? 1 : 2)][tc][t1];
    w.put(ct.bits, ct.len);
    if (tc == 0) return 0;
    // levels, highest frequency first
    int suffix = (tc > 10 && t1 < 3) ? 1 : 0;
    for (int k = tc - 1, i = 0; k >= 0; k--, i++) {
        const int level = coeffs[nz[k]];
        if (i < t1) {
            w.put(level < 0 ? 1 : 0, 1);
            continue;
        }
        int64_t code = level > 0 ? 2LL * level - 2 : -2LL * level - 1;
        if (i == t1 && t1 < 3) code -= 2;
        if (suffix == 0) {
            if (code < 14) {
                w.put(1, int(code) + 1);  // level_prefix = code, no suffix
            } else if (code < 30) {
                w.put(1, 15);  // level_prefix 14, 4-bit suffix
                w.put(uint32_t(code - 14), 4);
            } else {
                put_escape(w, code - 30);
            }
        } else {
            if (code < (15LL << suffix)) {
                w.put(1, int(code >> suffix) + 1);
                w.put(uint32_t(code & ((1 << suffix) - 1)), suffix);
            } else {
                put_escape(w, code - (15LL << suffix));
            }
        }
        if (suffix == 0) suffix = 1;
        const int a = level < 0 ? -level : level;
        if (a > (3 << (suffix - 1)) && suffix < 6) suffix++;
    }
    // total_zeros and run_before
    const int tz = nz[tc - 1] + 1 - tc;
    if (tc < maxc) {
        const Code c = nc == -1 ? TOTAL_ZEROS_CDC[tc - 1][tz] : TOTAL_ZEROS[tc - 1][tz];
        w.put(c.bits, c.len);
    }
    int left = tz;
    for (int k = tc - 1; k > 0 && left > 0; k--) {
        const int run = nz[k] - nz[k - 1] - 1;
        const Code c = RUN_BEFORE[(left < 7 ? left : 7) - 1][run];
        w.put(c.bits, c.len);
        left -= run;
    }
    return tc;
}

// ---- MV prediction (8.4.1.3), every neighbour inter with reference 0 ---------
struct Nb {
    bool av;
    int x, y;
};
int med3(int a, int b, int c) { return a + b + c - std::min(std::min(a, b), c) - std::max(std::max(a, b), c); }
// the median rule with a, b, c (c already replaced by d when absent)
void median_pred(const Nb& a, const Nb& b, const Nb& c, int& px, int& py) {
    Nb A = a, B = b, C = c;
    if (!B.av && !C.av && A.av) { B = A; C = A; }
    const int m = int(A.av) + int(B.av) + int(C.av);
    if (m == 1) {  // exactly one neighbour refers to reference 0
        const Nb& o = A.av ? A : (B.av ? B : C);
        px = o.x; py = o.y;
        return;
    }
    px = med3(A.av ? A.x : 0, B.av ? B.x : 0, C.av ? C.x : 0);
    py = med3(A.av ? A.y : 0, B.av ? B.y : 0, C.av ? C.y : 0);
}

struct Frame {
    int mb_w, mb_h;
    std::vector<int32_t> mv;  // 2 per 4x4 block of coded MBs
    std::vector<uint8_t> done;
    Nb at(int bx, int by) const {  // 4x4 block (bx, by), available if its MB is coded
        if (bx < 0 || by < 0 || bx >= 4 * mb_w || by >= 4 * mb_h || !done[(by >> 2) * mb_w + (bx >> 2)])
            return Nb{false, 0, 0};
        const size_t i = 2 * (size_t(by) * 4 * mb_w + bx);
        return Nb{true, mv[i], mv[i + 1]};
    }
};

// mvp of partition `part` of MB (mbx, mby) under shape s (8.4.1.3.1: the
// directional rules of 16x8 and 8x16, else the median)
void predict(const Frame& F, int mbx, int mby, int shape, int part, const int32_t* cur_mv, int& mx, int& my) {
    int x0 = 0, y0 = 0, w4 = 4;
    if (shape == 1) y0 = part ? 2 : 0;
    if (shape == 2) { x0 = part ? 2 : 0; w4 = 2; }
    const int bx = 4 * mbx + x0, by = 4 * mby + y0;
    // neighbours inside the current MB that are already coded (16x8 lower:
    // the upper partition is B; 8x16 right: the left partition is A)
    auto get = [&](int x, int y) -> Nb {
        if (x >= 4 * mbx && x < 4 * mbx + 4 && y >= 4 * mby && y < 4 * mby + 4) {
            const int lx = x - 4 * mbx, ly = y - 4 * mby;
            const int p = shape == 1 ? (ly >= 2) : (shape == 2 ? (lx >= 2) : 0);
            if (p < part) return Nb{true, cur_mv[2 * p], cur_mv[2 * p + 1]};
            return Nb{false, 0, 0};
        }
        return F.at(x, y);
    };
    const Nb a = get(bx - 1, by), b = get(bx, by - 1);
    Nb c = get(bx + w4, by - 1);
    if (!c.av) c = get(bx - 1, by - 1);
    if (shape == 1 && part == 0 && b.av) { mx = b.x; my = b.y; return; }
    if (shape == 1 && part == 1 && a.av) { mx = a.x; my = a.y; return; }
    if (shape == 2 && part == 0 && a.av) { mx = a.x; my = a.y; return; }
    if (shape == 2 && part == 1 && c.av) { mx = c.x; my = c.y; return; }
    median_pred(a, b, c, mx, my);
}

struct Params {
    int width, height, cw, ch, n, qp;
};

void write_sps(std::vector<uint8_t>& out, const Params& p) {
    Bits w;
    w.put(66, 8);    // profile_idc: Baseline
    w.put(0xC0, 8);  // constraint_set0/1 (constrained baseline), reserved zeros
    const int mbs = (p.cw / 16) * (p.ch / 16);
    w.put(mbs <= 8192 ? 40 : 51, 8);  // level_idc
    w.ue(0);      // seq_parameter_set_id
    w.ue(12);     // log2_max_frame_num_minus4: frame_num is 16 bits
    w.ue(2);      // pic_order_cnt_type 2 (output order = decoding order)
    w.ue(1);      // max_num_ref_frames
    w.put(0, 1);  // gaps_in_frame_num_value_allowed_flag
    w.ue(p.cw / 16 - 1);
    w.ue(p.ch / 16 - 1);
    w.put(1, 1);  // frame_mbs_only_flag
    w.put(1, 1);  // direct_8x8_inference_flag
    const bool crop = p.width != p.cw || p.height != p.ch;
    w.put(crop, 1);
    if (crop) {  // in chroma sample units (4:2:0)
        w.ue(0);
        w.ue((p.cw - p.width) / 2);
        w.ue(0);
        w.ue((p.ch - p.height) / 2);
    }
    w.put(0, 1);  // vui_parameters_present_flag
    w.trailing();
    nal(out, 3, 7, w.b);
}

void write_pps(std::vector<uint8_t>& out, const Params& p) {
    Bits w;
    w.ue(0);          // pic_parameter_set_id
    w.ue(0);          // seq_parameter_set_id
    w.put(0, 1);      // entropy_coding_mode_flag: CAVLC
    w.put(0, 1);      // bottom_field_pic_order_in_frame_present_flag
    w.ue(0);          // num_slice_groups_minus1
    w.ue(0);          // num_ref_idx_l0_default_active_minus1
    w.ue(0);          // num_ref_idx_l1_default_active_minus1
    w.put(0, 1);      // weighted_pred_flag
    w.put(0, 2);      // weighted_bipred_idc
    w.se(p.qp - 26);  // pic_init_qp_minus26
    w.se(0);          // pic_init_qs_minus26
    w.se(0);          // chroma_qp_index_offset
    w.put(0, 1);      // deblocking_filter_control_present_flag: filter on, offsets 0
    w.put(0, 1);      // constrained_intra_pred_flag
    w.put(0, 1);      // redundant_pic_cnt_present_flag
    w.trailing();
    nal(out, 3, 8, w.b);
}

void write_idr(std::vector<uint8_t>& out, const Params& p, const uint8_t* y, const uint8_t* u, const uint8_t* v) {
    Bits w;
    w.ue(0);       // first_mb_in_slice
    w.ue(7);       // slice_type: I (all slices)
    w.ue(0);       // pic_parameter_set_id
    w.put(0, 16);  // frame_num
    w.ue(0);       // idr_pic_id
    w.put(0, 1);   // no_output_of_prior_pics_flag
    w.put(0, 1);   // long_term_reference_flag
    w.se(0);       // slice_qp_delta
    const int mb_w = p.cw / 16, mb_h = p.ch / 16, ccw = p.cw / 2;
    for (int mby = 0; mby < mb_h; mby++)
        for (int mbx = 0; mbx < mb_w; mbx++) {
            w.ue(25);  // mb_type I_PCM
            while (!w.aligned()) w.put(0, 1);  // pcm_alignment_zero_bit
            for (int r = 0; r < 16; r++)
                for (int c = 0; c < 16; c++) w.put(y[size_t(mby * 16 + r) * p.cw + mbx * 16 + c], 8);
            for (const uint8_t* pl : {u, v})
                for (int r = 0; r < 8; r++)
                    for (int c = 0; c < 8; c++) w.put(pl[size_t(mby * 8 + r) * ccw + mbx * 8 + c], 8);
        }
    w.trailing();
    nal(out, 3, 5, w.b);
}

void write_p(std::vector<uint8_t>& out, const Params& p, int frame_num, const int32_t* picks, const int16_t* coeffs,
             const int16_t* ccoeffs) {
    Bits w;
    w.ue(0);  // first_mb_in_slice
    w.ue(5);  // slice_type: P (all slices)
    w.ue(0);  // pic_parameter_set_id
    w.put(uint32_t(frame_num & 0xffff), 16);
    w.put(0, 1);  // num_ref_idx_active_override_flag
    w.put(0, 1);  // ref_pic_list_modification_flag_l0
    w.put(0, 1);  // adaptive_ref_pic_marking_mode_flag
    w.se(0);      // slice_qp_delta
    Frame F;
    F.mb_w = p.cw / 16;
    F.mb_h = p.ch / 16;
    F.mv.assign(size_t(2) * 16 * F.mb_w * F.mb_h, 0);
    F.done.assign(size_t(F.mb_w) * F.mb_h, 0);
    // TotalCoeff of every luma 4x4 block and chroma 4x4 AC block (nC contexts)
    std::vector<uint8_t> tc_y(size_t(16) * F.mb_w * F.mb_h, 0), tc_c[2];
    tc_c[0].assign(size_t(4) * F.mb_w * F.mb_h, 0);
    tc_c[1].assign(size_t(4) * F.mb_w * F.mb_h, 0);
    const int W4 = 4 * F.mb_w, W2 = 2 * F.mb_w;
    // nC of a block (9.2.1): its left and top blocks are available whenever
    // they are inside the picture (one slice, MBs in raster order, and a
    // block's left and top blocks inside its own MB come earlier in the
    // block scan)
    auto nc_of = [&](const std::vector<uint8_t>& tc, int stride, int bx, int by) {
        const bool ha = bx > 0, hb = by > 0;
        const int na = ha ? tc[size_t(by) * stride + bx - 1] : 0, nb = hb ? tc[size_t(by - 1) * stride + bx] : 0;
        return ha && hb ? (na + nb + 1) >> 1 : (ha ? na : (hb ? nb : 0));
    };
    for (int mby = 0; mby < F.mb_h; mby++)
        for (int mbx = 0; mbx < F.mb_w; mbx++) {
            const int m = mby * F.mb_w + mbx;
            const int32_t* pk = picks + 6 * m;
            const int shape = pk[0];
            const int np = shape == 0 ? 1 : 2;
            const int32_t cur[4] = {pk[1], pk[2], pk[3], pk[4]};
            w.ue(0);      // mb_skip_run
            w.ue(shape);  // mb_type P_L0_16x16 / P_L0_L0_16x8 / P_L0_L0_8x16
            for (int part = 0; part < np; part++) {
                int mx, my;
                predict(F, mbx, mby, shape, part, cur, mx, my);
                w.se(cur[2 * part] - mx);
                w.se(cur[2 * part + 1] - my);
            }
            // the coded_block_pattern from the MB's levels
            const int16_t* L = coeffs + size_t(256) * m;
            const int16_t* Cc = ccoeffs + size_t(128) * m;
            int cbp = 0;
            for (int b8 = 0; b8 < 4; b8++)
                for (int i = 0; i < 64; i++)
                    if (L[b8 * 64 + i]) {
                        cbp |= 1 << b8;
                        break;
                    }
            bool dc = false, ac = false;
            for (int c = 0; c < 2; c++)
                for (int b = 0; b < 4; b++) {
                    dc = dc || Cc[c * 64 + b * 16] != 0;
                    for (int i = 1; i < 16; i++) ac = ac || Cc[c * 64 + b * 16 + i] != 0;
                }
            cbp |= (ac ? 2 : (dc ? 1 : 0)) << 4;
            w.ue(CBP_INTER_CODE[cbp]);
            if (cbp) w.se(0);  // mb_qp_delta
            for (int b8 = 0; b8 < 4; b8++)
                for (int b4 = 0; b4 < 4; b4++) {
                    const int bx = 4 * mbx + (b8 & 1) * 2 + (b4 & 1), by = 4 * mby + (b8 >> 1) * 2 + (b4 >> 1);
                    int tcnt = 0;
                    if (cbp & (1 << b8)) {
                        int sc[16];
                        for (int i = 0; i < 16; i++) sc[i] = L[b8 * 64 + b4 * 16 + ZIGZAG[i]];
                        tcnt = residual_block(w, sc, 16, nc_of(tc_y, W4, bx, by));
                    }
                    tc_y[size_t(by) * W4 + bx] = uint8_t(tcnt);
                }
            if (cbp >> 4)
                for (int c = 0; c < 2; c++) {
                    int d[4];
                    for (int b = 0; b < 4; b++) d[b] = Cc[c * 64 + b * 16];
                    residual_block(w, d, 4, -1);
                }
            for (int c = 0; c < 2; c++)
                for (int b = 0; b < 4; b++) {
                    const int bx = 2 * mbx + (b & 1), by = 2 * mby + (b >> 1);
                    int tcnt = 0;
                    if ((cbp >> 4) == 2) {
                        int sc[15];
                        for (int i = 1; i < 16; i++) sc[i - 1] = Cc[c * 64 + b * 16 + ZIGZAG[i]];
                        tcnt = residual_block(w, sc, 15, nc_of(tc_c[c], W2, bx, by));
                    }
                    tc_c[c][size_t(by) * W2 + bx] = uint8_t(tcnt);
                }
            // commit the MB's MVs to the 4x4 grid
            for (int r = 0; r < 4; r++)
                for (int q = 0; q < 4; q++) {
                    const int part = shape == 1 ? (r >= 2) : (shape == 2 ? (q >= 2) : 0);
                    const size_t i = 2 * (size_t(4 * mby + r) * W4 + 4 * mbx + q);
                    F.mv[i] = cur[2 * part];
                    F.mv[i + 1] = cur[2 * part + 1];
                }
            F.done[m] = 1;
        }
    w.trailing();
    nal(out, 2, 1, w.b);
}

}  // namespace cavlc
}  // namespace h264a

extern "C" int h264a_write_stream_cavlc(const h264a_stream_frames* in, uint8_t* h_out, size_t cap, size_t* out_len,
                                        int64_t* h_frame_bytes) {
    using namespace h264a;
    if (!in || !out_len) return fail(H264A_E_ARG, "write_stream_cavlc: null pointer");
    const int n = in->n, cw = in->cw, ch = in->ch;
    if (n < 1 || cw < 16 || ch < 16 || cw % 16 || ch % 16 || in->width < 1 || in->height < 1 || in->width > cw ||
        in->height > ch || cw - in->width >= 16 || ch - in->height >= 16 || ((in->width | in->height) & 1))
        return fail(H264A_E_ARG, "write_stream_cavlc: bad geometry (coded size the MB-aligned even display size)");
    if (in->qp < 0 || in->qp > 51) return fail(H264A_E_ARG, "write_stream_cavlc: qp out of 0..51");
    if (!in->h_y0 || !in->h_u0 || !in->h_v0 || (n > 1 && (!in->h_picks || !in->h_coeffs || !in->h_ccoeffs)))
        return fail(H264A_E_ARG, "write_stream_cavlc: null frame data");
    const size_t nmb = size_t(cw / 16) * (ch / 16);
    for (int f = 1; f < n; f++)
        for (size_t m = 0; m < nmb; m++)
            if (uint32_t(in->h_picks[(f * nmb + m) * 6]) > 2u)
                return fail(H264A_E_ARG, "write_stream_cavlc: pick shape out of 0..2");
    cavlc::Params p{in->width, in->height, cw, ch, n, in->qp};
    std::vector<uint8_t> out;
    cavlc::write_sps(out, p);
    cavlc::write_pps(out, p);
    cavlc::write_idr(out, p, in->h_y0, in->h_u0, in->h_v0);
    if (h_frame_bytes) h_frame_bytes[0] = int64_t(out.size());  // with the parameter sets
    for (int f = 1; f < n; f++) {
        const size_t prev = out.size();
        cavlc::write_p(out, p, f, in->h_picks + f * nmb * 6, in->h_coeffs + f * nmb * 256, in->h_ccoeffs + f * nmb * 128);
        if (h_frame_bytes) h_frame_bytes[f] = int64_t(out.size() - prev);
    }
    *out_len = out.size();
    if (h_out) {
        if (cap < out.size()) return fail(H264A_E_ARG, "write_stream_cavlc: output buffer too small");
        memcpy(h_out, out.data(), out.size());
    }
    return H264A_OK;
}

extern "C" int h264a_cavlc_table_code(int table, int i, int j, int k, int* len, int* bits) {
    using namespace h264a::cavlc;
    if (!len || !bits) return h264a::fail(H264A_E_ARG, "cavlc_table_code: null pointer");
    Code c{0, 0};
    switch (table) {
        case 0:  // coeff_token, nC class i (0..2), TotalCoeff j, TrailingOnes k
            if (i < 0 || i > 2 || j < 0 || j > 16 || k < 0 || k > 3) return H264A_E_ARG;
            c = COEFF_TOKEN[i][j][k];
            break;
        case 1:  // chroma DC coeff_token, TotalCoeff j, TrailingOnes k
            if (j < 0 || j > 4 || k < 0 || k > 3) return H264A_E_ARG;
            c = COEFF_TOKEN_CDC[j][k];
            break;
        case 2:  // total_zeros, TotalCoeff j (1..15), total_zeros k
            if (j < 1 || j > 15 || k < 0 || k > 15) return H264A_E_ARG;
            c = TOTAL_ZEROS[j - 1][k];
            break;
        case 3:  // chroma DC total_zeros
            if (j < 1 || j > 3 || k < 0 || k > 3) return H264A_E_ARG;
            c = TOTAL_ZEROS_CDC[j - 1][k];
            break;
        case 4:  // run_before, min(zerosLeft,7) j (1..7), run k
            if (j < 1 || j > 7 || k < 0 || k > 14) return H264A_E_ARG;
            c = RUN_BEFORE[j - 1][k];
            break;
        case 5:  // inter coded_block_pattern j -> codeNum
            if (j < 0 || j > 47) return H264A_E_ARG;
            *len = 0;
            *bits = CBP_INTER_CODE[j];
            return H264A_OK;
        default:
            return H264A_E_ARG;
    }
    *len = c.len;
    *bits = c.bits;
    return H264A_OK;
}
