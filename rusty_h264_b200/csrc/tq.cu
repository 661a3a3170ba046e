// tq.cu -- a13/a14/a15: forward integer transforms and quantisation.
//
//  * dct_four_t4 + quant_four_4x4 (crates/rusty_h264-accel/src/transform_quant.rs:
//    71-135) with FF = quant_dz_ff(qp, dz) and MF = QUANT_MF_OH[qp]
//    (crates/rusty_h264-common/src/transform.rs:145-159, 1447-1500);
//  * forward_core_8x8 + quantize_8x8 (transform.rs:492-629);
//  * the fused MC + luma T/Q of chosen MBs (mb16.rs:3436-3450).
// All in registers, one thread per 4x4 block (one row/column per thread for
// 8x8); HBM traffic is the source and prediction bytes in and the
// coefficients out.
#include <climits>
#include <cstring>
#include <vector>

#include "tq_device.cuh"

namespace h264a {


__global__ void dct_quant_4x4_kernel(const uint8_t* __restrict__ src, int ss, const uint8_t* __restrict__ pred, int ps,
                                     const int32_t* __restrict__ xy, const uint8_t* __restrict__ qp, QuantTables4 qt,
                                     int n, int16_t* __restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long r = t >> 2;
    if (r >= n) return;
    const int k = int(t & 3);
    const int ox = (k & 1) * 4, oy = (k >> 1) * 4;  // sub-block order (0,0),(4,0),(0,4),(4,4)
    const int x = xy[2 * r] + ox, y = xy[2 * r + 1] + oy;
    uint32_t s[4], p[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        s[i] = ld4u(src + (long long)(y + i) * ss + x);
        p[i] = ld4u(pred + (long long)(y + i) * ps + x);
    }
    const int q = qp[r] > 51 ? 51 : qp[r];
    tq4x4_store(s, p, qt.ff[q], qt.mf[q], out + r * 64 + k * 16);
}

// ---- 8x8 -------------------------------------------------------------------

struct QuantTables8 {
    int32_t mf[6][64];   // QUANT_MF_8X8[qp%6][group] * 16 / weight
    long long ff[52];    // (1 << (16 + qp/6)) / dz
};

static const int kQuantMf8[6][6] = {
    {13107, 14564, 8192, 13797, 10486, 10923}, {11916, 13797, 7490, 12483, 9362, 10083},
    {10083, 11398, 6242, 10923, 7944, 8456},   {9362, 10486, 5825, 10083, 7490, 7944},
    {8192, 9362, 5140, 8738, 6554, 6899},      {7282, 8192, 4520, 7710, 5699, 6096},
};

static int pos_group_8x8(int i, int j) {
    const int i4 = i % 4, j4 = j % 4;
    if (i4 == 0 && j4 == 0) return 0;
    if (i % 2 == 1 && j % 2 == 1) return 1;
    if (i4 == 2 && j4 == 2) return 2;
    if ((i4 == 0 && j % 2 == 1) || (i % 2 == 1 && j4 == 0)) return 3;
    if ((i4 == 0 && j4 == 2) || (i4 == 2 && j4 == 0)) return 4;
    return 5;
}

// fwd_1d_8x8 (transform.rs:492-524).
__device__ __forceinline__ void fwd8(const int s[8], int y[8]) {
    const int a0 = s[0] + s[7], a1 = s[1] + s[6], a2 = s[2] + s[5], a3 = s[3] + s[4];
    const int a4 = s[0] - s[7], a5 = s[1] - s[6], a6 = s[2] - s[5], a7 = s[3] - s[4];
    const int b0 = a0 + a3, b1 = a1 + a2, b2 = a0 - a3, b3 = a1 - a2;
    y[0] = b0 + b1;
    y[2] = b2 + (b3 >> 1);
    y[4] = b0 - b1;
    y[6] = (b2 >> 1) - b3;
    const int b4 = a5 + a6 + ((a4 >> 1) + a4);
    const int b5 = a4 - a7 - ((a6 >> 1) + a6);
    const int b6 = a4 + a7 - ((a5 >> 1) + a5);
    const int b7 = a5 - a6 + ((a7 >> 1) + a7);
    y[1] = b4 + (b7 >> 2);
    y[3] = b5 + (b6 >> 2);
    y[5] = b6 - (b5 >> 2);
    y[7] = (b4 >> 2) - b7;
}

// 8 threads per region: thread r transforms row r, then column r (through
// shared memory), then quantises that column.
__global__ void __launch_bounds__(256) dct_quant_8x8_kernel(const uint8_t* __restrict__ src, int ss,
                                                           const uint8_t* __restrict__ pred, int ps,
                                                           const int32_t* __restrict__ xy,
                                                           const uint8_t* __restrict__ qp, QuantTables8 qt, int n,
                                                           int32_t* __restrict__ out) {
    __shared__ int tile[32][65];
    const int local = threadIdx.x >> 3;  // region within the block
    const int row = threadIdx.x & 7;
    const long long r = (long long)blockIdx.x * 32 + local;
    const bool live = r < n;
    if (live) {
        const int x = xy[2 * r], y = xy[2 * r + 1] + row;
        const uint32_t s0 = ld4u(src + (long long)y * ss + x), s1 = ld4u(src + (long long)y * ss + x + 4);
        const uint32_t p0 = ld4u(pred + (long long)y * ps + x), p1 = ld4u(pred + (long long)y * ps + x + 4);
        int v[8], o[8];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            v[c] = byte_of(s0, c) - byte_of(p0, c);
            v[c + 4] = byte_of(s1, c) - byte_of(p1, c);
        }
        fwd8(v, o);
#pragma unroll
        for (int c = 0; c < 8; c++) tile[local][row * 8 + c] = o[c];
    }
    __syncthreads();
    if (!live) return;
    int v[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = tile[local][k * 8 + row];
    fwd8(v, o);
    const int q = qp[r] > 51 ? 51 : qp[r];
    const int m = q % 6;
    const int qbits = 16 + q / 6;
    const long long ff = qt.ff[q];
#pragma unroll
    for (int k = 0; k < 8; k++) {
        const int idx = k * 8 + row;
        const long long a = o[k] < 0 ? -(long long)o[k] : (long long)o[k];
        const int lvl = int((a * qt.mf[m][idx] + ff) >> qbits);
        out[r * 64 + idx] = o[k] < 0 ? -lvl : lvl;
    }
}

// ---- fused MC + luma T/Q of whole frames ---------------------------------------

struct TqFrameDesc {
    h264a_picture pic;
    const int32_t* picks;
    int qp;
    int16_t* coeffs;
    int mb_w;
    int nmb;
    uint8_t* rec;  // cw x ch luma reconstruction, or nullptr
    // multi-reference picks (8 i32 per MB: shape, then reference index and
    // MV of each half) predict each half from rplanes[its reference];
    // stride 6: single-reference picks, pic.d_planes
    const uint8_t* rplanes[4];
    int stride;
};

constexpr int TQ_MAXF = 96;
struct TqBatch {
    TqFrameDesc f[TQ_MAXF];
    int mb_base[TQ_MAXF];
    int n;
};

__global__ void mc_tq_frames_kernel(const __grid_constant__ TqBatch batch, long long total_mb, QuantTables4 qt) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long g = t >> 4;  // MB index across the batch
    if (g >= total_mb) return;
    int lo = 0, hi = batch.n - 1;  // last frame whose base <= g
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (batch.mb_base[mid] <= g) lo = mid; else hi = mid - 1;
    }
    const TqFrameDesc& fd = batch.f[lo];
    const int m = int(g - batch.mb_base[lo]);
    const int blk = int(t & 15);
    const int bx = (blk & 3) * 4, by = (blk >> 2) * 4;  // 4x4 block inside the MB
    const int mbx = m % fd.mb_w, mby = m / fd.mb_w;
    const int32_t* pk = fd.picks + fd.stride * m;
    const int shape = pk[0];
    const int part = shape == 1 ? (by >= 8) : (shape == 2 ? (bx >= 8) : 0);
    int mvx, mvy;
    const uint8_t* planes = fd.pic.d_planes;
    if (fd.stride == 8) {
        planes = fd.rplanes[pk[1 + 3 * part] & 3];
        mvx = pk[2 + 3 * part];
        mvy = pk[3 + 3 * part];
    } else {
        mvx = pk[1 + 2 * part];
        mvy = pk[2 + 2 * part];
    }
    Planes P{planes, fd.pic.cw + 2 * fd.pic.pad, fd.pic.ch + 2 * fd.pic.pad, fd.pic.pad, 0};
    P.ps = (long long)P.pw * P.ph;
    const int x = mbx * 16 + bx, y = mby * 16 + by;
    uint32_t s[4], p[4];
#pragma unroll
    for (int i = 0; i < 4; i++) s[i] = ld4u(fd.pic.d_src + (long long)(y + i) * fd.pic.cw + x);
    pred_rows(P, x + (mvx >> 2), y + (mvy >> 2), mvx & 3, mvy & 3, p);
    // reference layout: region qi (0,0),(8,0),(0,8),(8,8); sub-block k (0,0),(4,0),(0,4),(4,4)
    const int qi = (by >= 8 ? 2 : 0) + (bx >= 8 ? 1 : 0);
    const int k = ((by & 4) ? 2 : 0) + ((bx & 4) ? 1 : 0);
    const int q = fd.qp > 51 ? 51 : (fd.qp < 0 ? 0 : fd.qp);
    if (fd.rec == nullptr) {
        tq4x4_store(s, p, qt.ff[q], qt.mf[q], fd.coeffs + (long long)m * 256 + qi * 64 + k * 16);
        return;
    }
    int lv[16];
    tq4x4_store(s, p, qt.ff[q], qt.mf[q], fd.coeffs + (long long)m * 256 + qi * 64 + k * 16, lv);
    uint32_t r4[4];
    rec4x4(lv, p, q, r4);
    // x is a multiple of 4 and cw of 16, so each row is one aligned word
#pragma unroll
    for (int i = 0; i < 4; i++) *reinterpret_cast<uint32_t*>(fd.rec + (long long)(y + i) * fd.pic.cw + x) = r4[i];
}

}  // namespace h264a

using namespace h264a;

extern "C" int h264a_dct_quant_4x4(h264a_ctx* ctx, const uint8_t* d_src, int ss, const uint8_t* d_pred, int ps,
                                   const int32_t* d_xy, const uint8_t* d_qp, int dz_div, int n, int16_t* d_out,
                                   void* stream) {
    if (!ctx || !d_src || !d_pred || !d_xy || !d_qp || !d_out) return fail(H264A_E_ARG, "dct_quant_4x4: null pointer");
    if (n < 0 || dz_div < 1 || ss < 8 || ps < 8) return fail(H264A_E_ARG, "dct_quant_4x4: bad count, stride or dz");
    if ((reinterpret_cast<uintptr_t>(d_out) & 15) != 0) return fail(H264A_E_ARG, "dct_quant_4x4: out must be 16-byte aligned");
    if (n == 0) return H264A_OK;
    const QuantTables4 qt = make_tables4(dz_div);
    const long long threads = (long long)n * 4;
    dct_quant_4x4_kernel<<<unsigned((threads + 255) / 256), 256, 0, pick_stream(ctx, stream)>>>(d_src, ss, d_pred, ps,
                                                                                                d_xy, d_qp, qt, n, d_out);
    return check_launch("dct_quant_4x4_kernel");
}

extern "C" int h264a_dct_quant_8x8(h264a_ctx* ctx, const uint8_t* d_src, int ss, const uint8_t* d_pred, int ps,
                                   const int32_t* d_xy, const uint8_t* d_qp, const int32_t* h_weight, int dz_div,
                                   int n, int32_t* d_out, void* stream) {
    if (!ctx || !d_src || !d_pred || !d_xy || !d_qp || !d_out) return fail(H264A_E_ARG, "dct_quant_8x8: null pointer");
    if (n < 0 || dz_div < 1 || ss < 8 || ps < 8) return fail(H264A_E_ARG, "dct_quant_8x8: bad count, stride or dz");
    if (n == 0) return H264A_OK;
    QuantTables8 qt;
    for (int m = 0; m < 6; m++)
        for (int idx = 0; idx < 64; idx++) {
            const int w = h_weight ? h_weight[idx] : 16;
            if (w <= 0) return fail(H264A_E_ARG, "dct_quant_8x8: weights must be positive");
            qt.mf[m][idx] = int32_t((long long)kQuantMf8[m][pos_group_8x8(idx / 8, idx % 8)] * 16 / w);
        }
    for (int q = 0; q < 52; q++) qt.ff[q] = (1LL << (16 + q / 6)) / dz_div;
    dct_quant_8x8_kernel<<<unsigned((n + 31) / 32), 256, 0, pick_stream(ctx, stream)>>>(d_src, ss, d_pred, ps, d_xy,
                                                                                        d_qp, qt, n, d_out);
    return check_launch("dct_quant_8x8_kernel");
}

// ---- the inter MB's chroma: MC, T/Q with the 2x2 DC, reconstruction -------------

struct TqcFrameDesc {
    const uint8_t* src[2];
    const uint8_t* ref[2];
    const int32_t* picks;
    int16_t* coeffs;
    uint8_t* rec[2];
    int ccw, cch, mb_w, nmb, qpc;
};
constexpr int TQC_MAXF = 64;
struct TqcBatch {
    TqcFrameDesc f[TQC_MAXF];
    int mb_base[TQC_MAXF];
    int n;
};

// One thread per (MB, plane, 4x4 block k in SUBBLOCKS order), eight
// consecutive lanes per MB: chroma_tq_rec with the MB's partition MV.
__global__ void mc_tq_chroma_kernel(const __grid_constant__ TqcBatch batch, long long total_mb, QuantTables4 qt) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long g = t >> 3;
    const bool live = g < total_mb;
    const long long gg = live ? g : total_mb - 1;  // dead lanes shadow the last MB so the shuffles stay full-warp
    int lo = 0, hi = batch.n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (batch.mb_base[mid] <= gg) lo = mid; else hi = mid - 1;
    }
    const TqcFrameDesc& fd = batch.f[lo];
    const int m = int(gg - batch.mb_base[lo]);
    const int c = int((t >> 2) & 1), k = int(t & 3);
    const int bx = (k & 1) * 4, by = (k >> 1) * 4;
    const int mbx = m % fd.mb_w, mby = m / fd.mb_w;
    const int32_t* pk = fd.picks + 6 * m;
    const int shape = pk[0];
    const int part = shape == 1 ? (by >= 4) : (shape == 2 ? (bx >= 4) : 0);
    const int mvx = pk[1 + 2 * part], mvy = pk[2 + 2 * part];
    const int x = mbx * 8 + bx, y = mby * 8 + by;
    uint32_t r4[4];
    chroma_tq_rec(fd.src[c], fd.ref[c], fd.ccw, fd.cch, x, y, mvx, mvy, k, fd.qpc, qt.ff[fd.qpc], qt.mf[fd.qpc],
                  live ? fd.coeffs + (long long)m * 128 + c * 64 + k * 16 : nullptr, r4);
    if (!live || fd.rec[c] == nullptr) return;
#pragma unroll
    for (int r = 0; r < 4; r++) *reinterpret_cast<uint32_t*>(fd.rec[c] + (long long)(y + r) * fd.ccw + x) = r4[r];
}

// Shared by h264a_mc_tq_frames and h264a_mc_tq_rec_frames: frame i's T/Q
// input is frames[i], its reconstruction target recs[i] (recs may be null).
static int mc_tq_launch(h264a_ctx* ctx, const h264a_tq_frame* h_frames, uint8_t* const* recs, int nframes,
                        void* stream) {
    if (!ctx || !h_frames || nframes < 1) return fail(H264A_E_ARG, "mc_tq_frames: bad arguments");
    const int dz = h_frames[0].dz_div;
    for (int i = 0; i < nframes; i++) {
        const h264a_tq_frame& f = h_frames[i];
        if (recs && (!recs[i] || (reinterpret_cast<uintptr_t>(recs[i]) & 3) != 0))
            return fail(H264A_E_ARG, "mc_tq_rec_frames: reconstruction buffers must be non-null and 4-byte aligned");
        if (!f.pic.d_src || !f.pic.d_planes || !f.d_picks || !f.d_coeffs)
            return fail(H264A_E_ARG, "mc_tq_frames: null frame pointer");
        if (f.pic.cw < 16 || f.pic.ch < 16 || f.pic.cw % 16 || f.pic.ch % 16 || f.pic.pad < 3 || f.pic.pad > 128)
            return fail(H264A_E_ARG, "mc_tq_frames: frames must be MB-aligned with 3 <= pad <= 128");
        if (f.dz_div != dz || dz < 1) return fail(H264A_E_ARG, "mc_tq_frames: one dz_div >= 1 per call");
        if ((reinterpret_cast<uintptr_t>(f.d_coeffs) & 15) != 0)
            return fail(H264A_E_ARG, "mc_tq_frames: coefficients must be 16-byte aligned");
        if ((long long)(f.pic.cw / 16) * (f.pic.ch / 16) > (1 << 24))
            return fail(H264A_E_ARG, "mc_tq_frames: frame too large");
    }
    cudaStream_t st = pick_stream(ctx, stream);
    const QuantTables4 qt = make_tables4(dz);
    for (int g0 = 0; g0 < nframes; g0 += TQ_MAXF) {
        const int gn = nframes - g0 < TQ_MAXF ? nframes - g0 : TQ_MAXF;
        TqBatch b;
        memset(&b, 0, sizeof b);
        b.n = gn;
        long long total = 0;
        for (int k = 0; k < gn; k++) {
            const h264a_tq_frame& f = h_frames[g0 + k];
            b.f[k] = {f.pic, f.d_picks, f.qp, f.d_coeffs, f.pic.cw / 16, (f.pic.cw / 16) * (f.pic.ch / 16),
                      recs ? recs[g0 + k] : nullptr, {nullptr, nullptr, nullptr, nullptr}, 6};
            b.mb_base[k] = int(total);
            total += b.f[k].nmb;
        }
        const long long threads = total * 16;
        mc_tq_frames_kernel<<<unsigned((threads + 255) / 256), 256, 0, st>>>(b, total, qt);
        const int rc = check_launch("mc_tq_frames_kernel");
        if (rc) return rc;
    }
    return H264A_OK;
}

int h264a::mc_tq_mr_run(h264a_ctx* ctx, const h264a_mc_tq_mr_frame* h_frames, int nframes, cudaStream_t st) {
    if (!ctx || !h_frames || nframes < 1) return fail(H264A_E_ARG, "mc_tq_frames_multiref: bad arguments");
    const int dz = h_frames[0].dz_div;
    for (int i = 0; i < nframes; i++) {
        const h264a_mc_tq_mr_frame& f = h_frames[i];
        if (!f.d_src || !f.d_picks || !f.d_coeffs) return fail(H264A_E_ARG, "mc_tq_frames_multiref: null frame pointer");
        if (f.nref < 1 || f.nref > 4) return fail(H264A_E_ARG, "mc_tq_frames_multiref: 1 to 4 references per frame");
        for (int r = 0; r < f.nref; r++)
            if (!f.d_planes[r]) return fail(H264A_E_ARG, "mc_tq_frames_multiref: null reference planes");
        if (f.cw < 16 || f.ch < 16 || f.cw % 16 || f.ch % 16 || f.pad < 3 || f.pad > 128)
            return fail(H264A_E_ARG, "mc_tq_frames_multiref: frames must be MB-aligned with 3 <= pad <= 128");
        if (f.dz_div != dz || dz < 1) return fail(H264A_E_ARG, "mc_tq_frames_multiref: one dz_div >= 1 per call");
        if (((reinterpret_cast<uintptr_t>(f.d_coeffs) & 15) | (reinterpret_cast<uintptr_t>(f.d_src) & 3)) != 0)
            return fail(H264A_E_ARG, "mc_tq_frames_multiref: coefficients 16-byte and sources 4-byte aligned");
        if ((long long)(f.cw / 16) * (f.ch / 16) > (1 << 24)) return fail(H264A_E_ARG, "mc_tq_frames_multiref: frame too large");
    }
    const QuantTables4 qt = make_tables4(dz);
    for (int g0 = 0; g0 < nframes; g0 += TQ_MAXF) {
        const int gn = nframes - g0 < TQ_MAXF ? nframes - g0 : TQ_MAXF;
        TqBatch b;
        memset(&b, 0, sizeof b);
        b.n = gn;
        long long total = 0;
        for (int k = 0; k < gn; k++) {
            const h264a_mc_tq_mr_frame& f = h_frames[g0 + k];
            TqFrameDesc& d = b.f[k];
            d.pic = h264a_picture{f.d_src, f.d_planes[0], f.cw, f.ch, f.pad};
            d.picks = f.d_picks;
            d.qp = f.qp;
            d.coeffs = f.d_coeffs;
            d.mb_w = f.cw / 16;
            d.nmb = (f.cw / 16) * (f.ch / 16);
            d.rec = nullptr;
            for (int r = 0; r < 4; r++) d.rplanes[r] = f.d_planes[r < f.nref ? r : 0];
            d.stride = 8;
            b.mb_base[k] = int(total);
            total += d.nmb;
        }
        if (total >= (1LL << 31)) return fail(H264A_E_ARG, "mc_tq_frames_multiref: too many macroblocks in one call");
        const long long threads = total * 16;
        mc_tq_frames_kernel<<<unsigned((threads + 255) / 256), 256, 0, st>>>(b, total, qt);
        const int rc = check_launch("mc_tq_frames_kernel");
        if (rc) return rc;
    }
    return H264A_OK;
}

extern "C" int h264a_mc_tq_frames_multiref(h264a_ctx* ctx, const h264a_mc_tq_mr_frame* h_frames, int nframes,
                                           void* stream) {
    return mc_tq_mr_run(ctx, h_frames, nframes, pick_stream(ctx, stream));
}

extern "C" int h264a_mc_tq_frames(h264a_ctx* ctx, const h264a_tq_frame* h_frames, int nframes, void* stream) {
    return mc_tq_launch(ctx, h_frames, nullptr, nframes, stream);
}

extern "C" int h264a_mc_tq_rec_frames(h264a_ctx* ctx, const h264a_tq_rec_frame* h_frames, int nframes,
                                      void* stream) {
    if (!h_frames || nframes < 1) return fail(H264A_E_ARG, "mc_tq_rec_frames: bad arguments");
    std::vector<h264a_tq_frame> tq(nframes);
    std::vector<uint8_t*> rec(nframes);
    for (int i = 0; i < nframes; i++) {
        tq[i] = h_frames[i].tq;
        rec[i] = h_frames[i].d_rec;
    }
    return mc_tq_launch(ctx, tq.data(), rec.data(), nframes, stream);
}

extern "C" int h264a_mc_tq_chroma_frames(h264a_ctx* ctx, const h264a_tq_chroma_frame* h_frames, int nframes,
                                         void* stream) {
    if (!ctx || !h_frames || nframes < 1) return fail(H264A_E_ARG, "mc_tq_chroma_frames: bad arguments");
    for (int i = 0; i < nframes; i++) {
        const h264a_tq_chroma_frame& f = h_frames[i];
        if (!f.d_src_u || !f.d_src_v || !f.d_ref_u || !f.d_ref_v || !f.d_picks || !f.d_coeffs)
            return fail(H264A_E_ARG, "mc_tq_chroma_frames: null frame pointer");
        if (f.cw < 16 || f.ch < 16 || f.cw % 16 || f.ch % 16 || (long long)(f.cw / 16) * (f.ch / 16) > (1 << 24))
            return fail(H264A_E_ARG, "mc_tq_chroma_frames: frames must be MB-aligned");
        const uintptr_t a4 = reinterpret_cast<uintptr_t>(f.d_src_u) | reinterpret_cast<uintptr_t>(f.d_src_v) |
                             reinterpret_cast<uintptr_t>(f.d_ref_u) | reinterpret_cast<uintptr_t>(f.d_ref_v) |
                             reinterpret_cast<uintptr_t>(f.d_rec_u) | reinterpret_cast<uintptr_t>(f.d_rec_v);
        if ((a4 & 3) != 0 || (reinterpret_cast<uintptr_t>(f.d_coeffs) & 15) != 0)
            return fail(H264A_E_ARG, "mc_tq_chroma_frames: planes must be 4-byte and coefficients 16-byte aligned");
        if ((f.d_rec_u == nullptr) != (f.d_rec_v == nullptr))
            return fail(H264A_E_ARG, "mc_tq_chroma_frames: give both reconstruction planes or neither");
        if (f.qp < 0 || f.qp > 51) return fail(H264A_E_ARG, "mc_tq_chroma_frames: qp out of 0..51");
    }
    static const int kQpc[22] = {29, 30, 31, 32, 32, 33, 34, 34, 35, 35, 36, 36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39};
    cudaStream_t st = pick_stream(ctx, stream);
    const QuantTables4 qt = make_tables4(6);
    for (int g0 = 0; g0 < nframes; g0 += TQC_MAXF) {
        const int gn = nframes - g0 < TQC_MAXF ? nframes - g0 : TQC_MAXF;
        TqcBatch b;
        memset(&b, 0, sizeof b);
        b.n = gn;
        long long total = 0;
        for (int k = 0; k < gn; k++) {
            const h264a_tq_chroma_frame& f = h_frames[g0 + k];
            TqcFrameDesc& d = b.f[k];
            d.src[0] = f.d_src_u; d.src[1] = f.d_src_v;
            d.ref[0] = f.d_ref_u; d.ref[1] = f.d_ref_v;
            d.picks = f.d_picks;
            d.coeffs = f.d_coeffs;
            d.rec[0] = f.d_rec_u; d.rec[1] = f.d_rec_v;
            d.ccw = f.cw / 2; d.cch = f.ch / 2;
            d.mb_w = f.cw / 16;
            d.nmb = (f.cw / 16) * (f.ch / 16);
            d.qpc = f.qp < 30 ? f.qp : kQpc[f.qp - 30];  // chroma_qp (predict.rs:64-73)
            b.mb_base[k] = int(total);
            total += d.nmb;
        }
        const long long threads = total * 8;
        mc_tq_chroma_kernel<<<unsigned((threads + 255) / 256), 256, 0, st>>>(b, total, qt);
        const int rc = check_launch("mc_tq_chroma_kernel");
        if (rc) return rc;
    }
    return H264A_OK;
}

