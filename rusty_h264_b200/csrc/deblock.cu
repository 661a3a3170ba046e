// deblock.cu -- §8f row 3: in-loop deblocking of the plain-ME P pictures
// (crates/rusty_h264-common/src/deblock.rs).
//
// The reference filters MBs in raster order, in place: per MB the luma
// vertical edges, the luma horizontal edges, then per chroma plane its
// vertical and horizontal edges.  An MB's filtering reads and writes three
// samples into its left and top neighbours, and the top edge reads samples
// that the top-right MB's left edge wrote, so an MB is ready once its left
// and top-right neighbours are done: the same wavefront as motion-vector
// prediction.  One persistent kernel deals MB tickets in that order (frames
// interleaved, bounded waits on the neighbours' flags); a warp filters its MB
// on shared-memory tiles (20x20 luma and 10x12 per chroma plane, the MB plus
// the samples its edges reach) and writes them back through L2.  No MB
// earlier in the order writes an MB's own samples, so they and bS are loaded
// before the wait; after it only the neighbours' strips are fetched, and luma
// (lanes 0..15) and chroma (lanes 16..31) are filtered side by side, one line
// per lane through all edges of a direction.
//
// Pictures of this path: every MB inter with reference 0, 4x4 transforms,
// one QP per picture.  bS (bs_inter and the single-list arm of bs1_tile,
// deblock.rs:328-333, 396-404) is 2 with coefficients on either side, else 1
// when the two blocks' MVs differ by 4 quarter-pels in x or y, else 0.
#include <algorithm>
#include <cstring>
#include <vector>

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

struct DbFrameDesc {
    uint8_t* y;
    uint8_t* uv[2];
    const int32_t* picks;
    const int16_t* coeffs;
    int cw, ch, mb_w, mb_h, flag_base;
    int alpha_y, beta_y, alpha_c, beta_c;
    int tc_y[3], tc_c[3];
};
constexpr int DB_MAXF = 64;
struct DbBatch {
    DbFrameDesc f[DB_MAXF];
    long long seg_start[DB_MAXF + 1];
    int n;
};

constexpr int DB_WARPS = 4;
// Resident CTAs per SM: 8 x 4 warps hold about two and a half wavefront steps
// of a 59-picture 1080p batch; more only adds warps polling flags.
constexpr int DB_BLOCKS_PER_SM = 8;
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
// reference's dct[256] order: 8x8 region, then 4x4 sub-block).
__device__ __forceinline__ void block_state(const DbFrameDesc& fd, int m, int bx, int by, int& mvx, int& mvy,
                                            bool& nz) {
    const int32_t* pk = fd.picks + 6 * m;
    const int shape = pk[0];
    const int part = shape == 1 ? (by >= 2) : (shape == 2 ? (bx >= 2) : 0);
    mvx = pk[1 + 2 * part];
    mvy = pk[2 + 2 * part];
    const int qi = (by >= 2 ? 2 : 0) + (bx >= 2 ? 1 : 0), k = (by & 1) * 2 + (bx & 1);
    const uint4* c = reinterpret_cast<const uint4*>(fd.coeffs + (long long)m * 256 + (qi * 4 + k) * 16);
    const uint4 a = c[0], b = c[1];
    nz = (a.x | a.y | a.z | a.w | b.x | b.y | b.z | b.w) != 0u;
}

__global__ void __launch_bounds__(32 * DB_WARPS) deblock_frames_kernel(const __grid_constant__ DbBatch batch,
                                                                       long long total, int* __restrict__ counter,
                                                                       int* __restrict__ flags, int epoch,
                                                                       int* __restrict__ status, int spin_limit) {
    __shared__ __align__(16) uint8_t ltile[DB_WARPS][LT * LT];
    __shared__ __align__(16) uint8_t ctile[DB_WARPS][2][CR * CT];
    __shared__ int bsw[DB_WARPS][32];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    uint8_t* lt = ltile[w];
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(counter, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) return;
        // segments are dealt from s = 0 (every frame, j = n - 1) on
        int s = 0;
        while (s + 1 < batch.n && batch.seg_start[s + 1] <= t) s++;
        const int j = batch.n - 1 - s;
        const long long u = t - batch.seg_start[s];
        const int nxt = j + 1 < batch.n ? batch.f[j + 1].mb_w * batch.f[j + 1].mb_h : 0;
        const DbFrameDesc& fd = batch.f[int(u % (j + 1))];
        const int k = nxt + int(u / (j + 1));
        int mbx, mby;
        wave_mb(fd.mb_w, fd.mb_h, k, mbx, mby);
        const int m = mby * fd.mb_w + mbx;
        int* fl = flags + fd.flag_base;
        const int y0 = mby * 16, x0 = mbx * 16;
        const int cy0 = mby * 8, cx0 = mbx * 8, ccw = fd.cw / 2;
        const bool has_c = fd.uv[0] != nullptr;
        // ---- before the wait: the MB's own samples (no MB earlier in the
        // order writes them) and bS: lanes 0..15 the vertical edges (edge
        // e = lane / 4, block row lane % 4), lanes 16..31 the horizontal ones ----
        for (int i = lane; i < 64; i += 32) {
            const int r = i >> 2, c4 = (i & 3) * 4;
            *reinterpret_cast<uint32_t*>(lt + (4 + r) * LT + 4 + c4) =
                __ldcg(reinterpret_cast<const unsigned int*>(fd.y + (long long)(y0 + r) * fd.cw + x0 + c4));
        }
        if (has_c) {
            const int pl = lane >> 4, r = (lane >> 1) & 7, c4 = (lane & 1) * 4;
            *reinterpret_cast<uint32_t*>(&ctile[w][pl][(2 + r) * CT + 4 + c4]) =
                __ldcg(reinterpret_cast<const unsigned int*>(fd.uv[pl] + (long long)(cy0 + r) * ccw + cx0 + c4));
        }
        {
            const int hor = lane >> 4, e = (lane >> 2) & 3, sg = lane & 3;
            int bs = 0;
            if (e > 0 || (hor ? mby > 0 : mbx > 0)) {
                int pmx, pmy, qmx, qmy;
                bool pnz, qnz;
                if (hor) {
                    block_state(fd, e > 0 ? m : m - fd.mb_w, sg, e > 0 ? e - 1 : 3, pmx, pmy, pnz);
                    block_state(fd, m, sg, e, qmx, qmy, qnz);
                } else {
                    block_state(fd, e > 0 ? m : m - 1, e > 0 ? e - 1 : 3, sg, pmx, pmy, pnz);
                    block_state(fd, m, e, sg, qmx, qmy, qnz);
                }
                bs = (pnz || qnz) ? 2 : ((abs(pmx - qmx) >= 4 || abs(pmy - qmy) >= 4) ? 1 : 0);
            }
            bsw[w][lane] = bs;
        }
        // ---- wait for the left (lane 0) and top-right (lane 1) neighbours ----
        if (lane == 0 && mbx > 0) wait_flag(fl + m - 1, epoch, status, 1, spin_limit);
        if (lane == 1 && mby > 0)
            wait_flag(fl + m - fd.mb_w + (mbx < fd.mb_w - 1 ? 1 : 0), epoch, status, 1, spin_limit);
        __syncwarp();
        // ---- the neighbours' samples the edges reach, through L2: luma left
        // strip (lanes 0..15, row `lane`) and top strip (lanes 16..31); chroma
        // left strips (lanes 0..15) and top strips (lanes 16..23) ----
        const bool lok = lane < 16 ? mbx > 0 : mby > 0;
        const int lr = lane < 16 ? lane : ((lane - 16) >> 2) - 4, lc = lane < 16 ? -4 : (lane & 3) * 4;
        unsigned int* lg = reinterpret_cast<unsigned int*>(fd.y + (long long)(y0 + lr) * fd.cw + x0 + lc);
        uint32_t* ls = reinterpret_cast<uint32_t*>(lt + (4 + lr) * LT + 4 + lc);
        const bool cok = has_c && lane < 24 && (lane < 16 ? mbx > 0 : mby > 0);
        const int cpl = lane < 16 ? lane >> 3 : (lane >> 2) & 1;
        const int cr = lane < 16 ? lane & 7 : ((lane >> 1) & 1) - 2, cc = lane < 16 ? -4 : (lane & 1) * 4;
        unsigned int* cg = cok ? reinterpret_cast<unsigned int*>(fd.uv[cpl] + (long long)(cy0 + cr) * ccw + cx0 + cc)
                               : nullptr;
        uint32_t* cs = reinterpret_cast<uint32_t*>(&ctile[w][cpl][(2 + cr) * CT + 4 + cc]);
        if (lok) *ls = __ldcg(lg);
        if (cok) *cs = __ldcg(cg);
        __syncwarp();
        // ---- vertical edges: lanes 0..15 luma row `lane` (edges 0..3), lanes
        // 16..31 chroma row lane & 7 of plane (lane >> 3) & 1 (columns 0, 4) ----
        const int pl = (lane >> 3) & 1, li = lane & 7;
        if (lane < 16) {
            uint8_t* row = lt + (4 + lane) * LT + 4;
            for (int e = mbx > 0 ? 0 : 1; e < 4; e++) {
                const int bs = bsw[w][e * 4 + (lane >> 2)];
                if (bs) luma_line(row + 4 * e, 1, bs, fd.alpha_y, fd.beta_y, fd.tc_y[bs - 1]);
            }
        } else if (has_c) {
            uint8_t* row = &ctile[w][pl][(2 + li) * CT + 4];
            for (int ce = mbx > 0 ? 0 : 2; ce < 4; ce += 2) {  // luma edges 0 and 2
                const int bs = bsw[w][ce * 4 + (li >> 1)];
                if (bs) chroma_line(row + 2 * ce, 1, bs, fd.alpha_c, fd.beta_c, fd.tc_c[bs - 1]);
            }
        }
        __syncwarp();
        // ---- horizontal edges: luma column `lane`, chroma column lane & 7 ----
        if (lane < 16) {
            uint8_t* col = lt + 4 * LT + 4 + lane;
            for (int e = mby > 0 ? 0 : 1; e < 4; e++) {
                const int bs = bsw[w][16 + e * 4 + (lane >> 2)];
                if (bs) luma_line(col + 4 * e * LT, LT, bs, fd.alpha_y, fd.beta_y, fd.tc_y[bs - 1]);
            }
        } else if (has_c) {
            uint8_t* col = &ctile[w][pl][2 * CT + 4 + li];
            for (int ce = mby > 0 ? 0 : 2; ce < 4; ce += 2) {
                const int bs = bsw[w][16 + ce * 4 + (li >> 1)];
                if (bs) chroma_line(col + 2 * ce * CT, CT, bs, fd.alpha_c, fd.beta_c, fd.tc_c[bs - 1]);
            }
        }
        __syncwarp();
        // ---- write back: the MB and the strips ----
        for (int i = lane; i < 64; i += 32) {
            const int r = i >> 2, c4 = (i & 3) * 4;
            __stcg(reinterpret_cast<unsigned int*>(fd.y + (long long)(y0 + r) * fd.cw + x0 + c4),
                   *reinterpret_cast<const uint32_t*>(lt + (4 + r) * LT + 4 + c4));
        }
        if (lok) __stcg(lg, *ls);
        if (has_c) {
            const int p = lane >> 4, r = (lane >> 1) & 7, c4 = (lane & 1) * 4;
            __stcg(reinterpret_cast<unsigned int*>(fd.uv[p] + (long long)(cy0 + r) * ccw + cx0 + c4),
                   *reinterpret_cast<const uint32_t*>(&ctile[w][p][(2 + r) * CT + 4 + c4]));
        }
        if (cok) __stcg(cg, *cs);
        __syncwarp();  // every lane's stores ordered before lane 0's release
        if (lane == 0) st_release(fl + m, epoch);
        __syncwarp();
    }
}

}  // namespace h264a

using namespace h264a;

extern "C" int h264a_deblock_frames(h264a_ctx* ctx, const h264a_deblock_frame* h_frames, int nframes, void* stream) {
    if (!ctx || !h_frames || nframes < 1) return fail(H264A_E_ARG, "deblock_frames: bad arguments");
    for (int i = 0; i < nframes; i++) {
        const h264a_deblock_frame& f = h_frames[i];
        if (!f.d_y || !f.d_picks || !f.d_coeffs) return fail(H264A_E_ARG, "deblock_frames: null frame pointer");
        if ((f.d_u == nullptr) != (f.d_v == nullptr))
            return fail(H264A_E_ARG, "deblock_frames: give both chroma planes or neither");
        if (f.cw < 16 || f.ch < 16 || f.cw % 16 || f.ch % 16 || (long long)(f.cw / 16) * (f.ch / 16) > (1 << 24))
            return fail(H264A_E_ARG, "deblock_frames: frames must be MB-aligned");
        const uintptr_t a = reinterpret_cast<uintptr_t>(f.d_y) | reinterpret_cast<uintptr_t>(f.d_u) |
                            reinterpret_cast<uintptr_t>(f.d_v);
        if ((a & 3) != 0 || (reinterpret_cast<uintptr_t>(f.d_coeffs) & 15) != 0)
            return fail(H264A_E_ARG, "deblock_frames: planes must be 4-byte and coefficients 16-byte aligned");
        if (f.qp < 0 || f.qp > 51) return fail(H264A_E_ARG, "deblock_frames: qp out of 0..51");
    }
    static const int kQpc[22] = {29, 30, 31, 32, 32, 33, 34, 34, 35, 35, 36, 36, 37, 37, 37, 38, 38, 38, 39, 39, 39, 39};
    cudaStream_t st = pick_stream(ctx, stream);
    std::vector<int> order(nframes);
    for (int i = 0; i < nframes; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (long long)h_frames[a].cw * h_frames[a].ch > (long long)h_frames[b].cw * h_frames[b].ch;
    });
    for (int g0 = 0; g0 < nframes; g0 += DB_MAXF) {
        const int gn = nframes - g0 < DB_MAXF ? nframes - g0 : DB_MAXF;
        DbBatch b;
        memset(&b, 0, sizeof b);
        b.n = gn;
        long long total = 0;
        for (int k = 0; k < gn; k++) {
            const h264a_deblock_frame& f = h_frames[order[g0 + k]];
            DbFrameDesc& d = b.f[k];
            d.y = f.d_y;
            d.uv[0] = f.d_u;
            d.uv[1] = f.d_v;
            d.picks = f.d_picks;
            d.coeffs = f.d_coeffs;
            d.cw = f.cw;
            d.ch = f.ch;
            d.mb_w = f.cw / 16;
            d.mb_h = f.ch / 16;
            d.flag_base = int(total);
            // thresholds (deblock.rs:1921-1929); MB edges average two equal QPs
            const int ia = std::min(std::max(f.qp + f.offset_a, 0), 51), ib = std::min(std::max(f.qp + f.offset_b, 0), 51);
            const int qc0 = std::min(std::max(f.qp + f.chroma_qp_offset, 0), 51);
            const int qpc = qc0 < 30 ? qc0 : kQpc[qc0 - 30];  // chroma_qp (predict.rs:64-73)
            const int ica = std::min(std::max(qpc + f.offset_a, 0), 51), icb = std::min(std::max(qpc + f.offset_b, 0), 51);
            d.alpha_y = kAlpha[ia];
            d.beta_y = kBeta[ib];
            d.alpha_c = kAlpha[ica];
            d.beta_c = kBeta[icb];
            for (int q = 0; q < 3; q++) {
                d.tc_y[q] = kTc0[ia][q];
                d.tc_c[q] = kTc0[ica][q];
            }
            total += (long long)d.mb_w * d.mb_h;
        }
        long long acc = 0;
        for (int s = 0; s < gn; s++) {
            const int jj = gn - 1 - s;
            b.seg_start[s] = acc;
            const long long nj = (long long)b.f[jj].mb_w * b.f[jj].mb_h;
            const long long nn = jj + 1 < gn ? (long long)b.f[jj + 1].mb_w * b.f[jj + 1].mb_h : 0;
            acc += (nj - nn) * (jj + 1);
        }
        b.seg_start[gn] = acc;
        if (acc != total) return fail(H264A_E_ARG, "deblock_frames: internal queue layout error");
        int rc = ensure_me_scratch(ctx, size_t(total));
        if (rc) return rc;
        H264A_CUDA(cudaMemsetAsync(ctx->q[Q_MAIN].d_counter, 0, sizeof(int32_t), st));
        const int epoch = next_epoch(ctx, st);
        if (epoch < 0) return H264A_E_CUDA;
        int per_sm = 0;
        H264A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, deblock_frames_kernel, 32 * DB_WARPS, 0));
        if (per_sm > DB_BLOCKS_PER_SM) per_sm = DB_BLOCKS_PER_SM;
        long long blocks = (long long)ctx->num_sms * (per_sm > 0 ? per_sm : 1);
        const long long need = (total + DB_WARPS - 1) / DB_WARPS;
        if (blocks > need) blocks = need;
        deblock_frames_kernel<<<unsigned(blocks), 32 * DB_WARPS, 0, st>>>(b, total, ctx->q[Q_MAIN].d_counter, ctx->q[Q_MAIN].d_flags,
                                                                          epoch, ctx->d_status, SPIN_LIMIT);
        rc = check_launch("deblock_frames_kernel");
        if (rc) return rc;
    }
    return H264A_OK;
}
