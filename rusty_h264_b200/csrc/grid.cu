// grid.cu -- exhaustive full-pel cost grids: 16x16 SAD and SATD of every
// integer offset within ±R of each MB's centre, the distortions the ME cost
// functions return at full-pel MVs (mc_sad_hp / mc_satd_hp,
// crates/rusty_h264-encoder/src/mb16.rs:1930-2074), and the per-MB argmin of
// dist + (λ·bits(mv − pmv)) in raster order with first-wins ties, the order of
// the exhaustive probe in motion_search (mb16.rs:2889-2900).
//
// The (16+2R)² search window of an MB (edge reads clamped, i.e. read from the
// padded F plane with clamping) is staged once in shared memory.
//  * SAD (fullpel_sad_kernel): a work item is one column offset and a run of
//    GRID_K row offsets; every window row is loaded and byte-aligned once and
//    feeds the GRID_K candidates it overlaps with one packed __vsadu4 per 4
//    pixels, the source MB in registers.  A CTA takes `mbs` consecutive MBs,
//    chosen on the host so that their items fill whole rounds of its threads
//    (3 at R = 32: 975 items in four rounds of 256).  The argmin skips the
//    lambda*rate of a candidate whose distortion alone cannot beat the
//    thread's best (exact: a thread meets its candidates in scan order).
//  * SATD (fullpel_satd_kernel): one CTA per MB; a thread owns four
//    horizontally adjacent offsets, and two aligned words per window row
//    segment yield all four candidates' rows by funnel shifts.
#include "h264a_device.cuh"

namespace h264a {

constexpr int GRID_K = 13;      // row offsets per SAD work item
constexpr int GRID_THREADS = 256;

struct GridArgs {
    Planes P;
    const uint8_t* src;
    int cw, ch, mb_w, R;
    const int32_t* centers;
    const int32_t* pmv;
    int metric, kind;
    const uint16_t* tab;
    double lambda;
    int32_t* sad_grid;
    int32_t* satd_grid;
    int32_t* best;
};

__device__ __forceinline__ uint32_t win_word(const uint8_t* row, int x) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(row + (x & ~3));
    const uint32_t sh = uint32_t(x & 3) * 8u;
    return sh ? __funnelshift_r(w[0], w[1], sh) : w[0];
}

// Stages the clamped window of MB (lx, ly) with full-pel centre (cxf, cyf):
// window (x, y) = picture (lx+cxf-R+x, ly+cyf-R+y), rows `ws` .. `wrows`-1
// and columns past `ws` zero (the reads of the last partial chunk and the
// fifth word of an unaligned read land there).  Row per warp, lanes along it.
__device__ __forceinline__ void stage_grid_window(uint8_t* win, const Planes& P, int lx, int ly, int cxf, int cyf,
                                                  int R, int ws, int pitch, int wrows, int row0, int rstep) {
    const int ox = lx + cxf - R + P.pad, oy = ly + cyf - R + P.pad;
    for (int y = row0; y < wrows; y += rstep) {
        const uint8_t* prow = P.base + (long long)clampi(oy + y, 0, P.ph - 1) * P.pw;
        for (int x = threadIdx.x & 31; x < pitch; x += 32)
            win[y * pitch + x] = (y < ws && x < ws) ? __ldg(prow + clampi(ox + x, 0, P.pw - 1)) : uint8_t(0);
    }
}

__device__ __forceinline__ long long grid_cost(const GridArgs& a, int dist, int mvx, int mvy, int pmx, int pmy) {
    return dist + lam_cost(a.lambda, mvbits(a.kind, a.tab, mvx - pmx) + mvbits(a.kind, a.tab, mvy - pmy));
}

// The argmin record of MB mb from its best key (cost << 32 | scan index).
__device__ __forceinline__ void grid_store_best(const GridArgs& a, int mb, long long key, int cxf, int cyf, int pmx,
                                                int pmy) {
    const int n = 2 * a.R + 1;
    const int idx = int(key & 0xffffffffLL);
    const long long cost = key >> 32;
    const int dyi = idx / n, dxi = idx % n;
    const int mvx = (cxf + dxi - a.R) * 4, mvy = (cyf + dyi - a.R) * 4;
    const long long rc = lam_cost(a.lambda, mvbits(a.kind, a.tab, mvx - pmx) + mvbits(a.kind, a.tab, mvy - pmy));
    a.best[4 * mb + 0] = mvx;
    a.best[4 * mb + 1] = mvy;
    a.best[4 * mb + 2] = int32_t(cost > 0x7fffffffLL ? 0x7fffffffLL : cost);
    a.best[4 * mb + 3] = int32_t(cost - rc);
}

__device__ __forceinline__ void grid_center(const GridArgs& a, int mb, int& cxf, int& cyf, int& pmx, int& pmy) {
    cxf = cyf = 0;
    if (a.centers) {
        cxf = (a.centers[2 * mb] + 2) >> 2;  // snapped like motion_search's integer snap
        cyf = (a.centers[2 * mb + 1] + 2) >> 2;
    }
    pmx = a.pmv ? a.pmv[2 * mb] : 0;
    pmy = a.pmv ? a.pmv[2 * mb + 1] : 0;
}

constexpr int SAD_MAX_MBS = 8;

// SAD grid and argmin of MBs mbs*blockIdx.x .. +mbs-1 (of nmb); dynamic
// shared memory: mbs windows of win_bytes.
__global__ void __launch_bounds__(GRID_THREADS, 2) fullpel_sad_kernel(GridArgs a, int mbs, int nmb, int win_bytes) {
    extern __shared__ __align__(16) uint8_t wins[];
    __shared__ __align__(16) uint32_t src_s[SAD_MAX_MBS][16][4];
    __shared__ unsigned long long best_s[SAD_MAX_MBS];
    const int R = a.R, n = 2 * R + 1;
    const int ws = 16 + 2 * R, pitch = (ws + 4 + 3) & ~3, wrows = ws + GRID_K;
    const int mb0 = blockIdx.x * mbs;
    const int nm = nmb - mb0 < mbs ? nmb - mb0 : mbs;
    const int nwarps = blockDim.x >> 5;
    for (int q = 0; q < nm; q++) {
        const int mb = mb0 + q;
        int cxf, cyf, pmx, pmy;
        grid_center(a, mb, cxf, cyf, pmx, pmy);
        stage_grid_window(wins + q * win_bytes, a.P, (mb % a.mb_w) * 16, (mb / a.mb_w) * 16, cxf, cyf, R, ws, pitch,
                          wrows, threadIdx.x >> 5, nwarps);
    }
    for (int t = threadIdx.x; t < nm * 64; t += blockDim.x) {
        const int q = t >> 6, r = (t >> 2) & 15, c = t & 3, mb = mb0 + q;
        src_s[q][r][c] = ld4u(a.src + (long long)((mb / a.mb_w) * 16 + r) * a.cw + (mb % a.mb_w) * 16 + 4 * c);
    }
    if (threadIdx.x < SAD_MAX_MBS) best_s[threadIdx.x] = ULLONG_MAX;
    __syncthreads();
    const bool argmin = a.metric == 0;
    const int chunks = (n + GRID_K - 1) / GRID_K, per_mb = n * chunks;
    for (int item = threadIdx.x; item < nm * per_mb; item += blockDim.x) {
        const int q = item / per_mb, it = item - q * per_mb;
        const int mb = mb0 + q;
        const int dxi = it % n, dy0 = (it / n) * GRID_K;
        const uint32_t sh = uint32_t(dxi & 3) * 8u;
        const uint8_t* win = wins + q * win_bytes;
        uint32_t s[16][4];
#pragma unroll
        for (int r = 0; r < 16; r++) {
            const uint4 v = *reinterpret_cast<const uint4*>(&src_s[q][r][0]);
            s[r][0] = v.x; s[r][1] = v.y; s[r][2] = v.z; s[r][3] = v.w;
        }
        int acc[GRID_K];
#pragma unroll
        for (int k = 0; k < GRID_K; k++) acc[k] = 0;
#pragma unroll
        for (int i = 0; i < GRID_K + 15; i++) {
            // the row's 16 bytes at dxi: five aligned words and funnel shifts
            const uint32_t* rw = reinterpret_cast<const uint32_t*>(win + (dy0 + i) * pitch + (dxi & ~3));
            uint32_t a5[5];
#pragma unroll
            for (int c = 0; c < 5; c++) a5[c] = rw[c];
            uint32_t w[4];
#pragma unroll
            for (int c = 0; c < 4; c++) w[c] = __funnelshift_r(a5[c], a5[c + 1], sh);
#pragma unroll
            for (int k = 0; k < GRID_K; k++) {
                const int r = i - k;
                if (r >= 0 && r < 16)
                    acc[k] += int(__vsadu4(s[r][0], w[0]) + __vsadu4(s[r][1], w[1]) + __vsadu4(s[r][2], w[2]) +
                                  __vsadu4(s[r][3], w[3]));
            }
        }
        int cxf, cyf, pmx, pmy;
        grid_center(a, mb, cxf, cyf, pmx, pmy);
        long long best_key = LLONG_MAX;  // this item's (cost << 32 | scan index) minimum
#pragma unroll
        for (int k = 0; k < GRID_K; k++) {
            const int dyi = dy0 + k;
            if (dyi < n) {
                const int idx = dyi * n + dxi;
                if (a.sad_grid) a.sad_grid[(long long)mb * n * n + idx] = acc[k];
                if (argmin && acc[k] < int(best_key >> 32)) {  // lambda*rate >= 0: a larger distortion cannot win
                    const long long key = (grid_cost(a, acc[k], (cxf + dxi - R) * 4, (cyf + dyi - R) * 4, pmx, pmy)
                                           << 32) | (long long)idx;
                    best_key = key < best_key ? key : best_key;
                }
            }
        }
        if (argmin && best_key != LLONG_MAX) atomicMin(&best_s[q], (unsigned long long)best_key);
    }
    __syncthreads();
    if (argmin && a.best && threadIdx.x < nm) {
        const int mb = mb0 + threadIdx.x;
        int cxf, cyf, pmx, pmy;
        grid_center(a, mb, cxf, cyf, pmx, pmy);
        grid_store_best(a, mb, (long long)best_s[threadIdx.x], cxf, cyf, pmx, pmy);
    }
}

// SATD grid and argmin, one CTA per MB; dynamic shared memory: the window.
__global__ void __launch_bounds__(GRID_THREADS, 2) fullpel_satd_kernel(GridArgs a) {
    extern __shared__ __align__(16) uint8_t win[];
    __shared__ long long red_key[GRID_THREADS / 32];
    const int mb = blockIdx.x;
    const int lx = (mb % a.mb_w) * 16, ly = (mb / a.mb_w) * 16;
    const int R = a.R, n = 2 * R + 1;
    int cxf, cyf, pmx, pmy;
    grid_center(a, mb, cxf, cyf, pmx, pmy);
    const int ws = 16 + 2 * R, pitch = (ws + 4 + 3) & ~3, wrows = ws + GRID_K;
    stage_grid_window(win, a.P, lx, ly, cxf, cyf, R, ws, pitch, wrows, threadIdx.x >> 5, GRID_THREADS / 32);
    // the source MB in shared memory (the four candidates' rows need the registers)
    __shared__ uint32_t src_s[16][4];
    if (threadIdx.x < 64)
        src_s[threadIdx.x >> 2][threadIdx.x & 3] =
            ld4u(a.src + (long long)(ly + (threadIdx.x >> 2)) * a.cw + lx + 4 * (threadIdx.x & 3));
    __syncthreads();

    long long best_key = LLONG_MAX;  // (cost << 32) | scan index; min = first-wins argmin
    const long long grid_base = (long long)mb * n * n;
    const bool argmin = a.metric == 1;

    {
        const int gx = (n + 3) / 4;  // groups of four adjacent column offsets
        for (int item = threadIdx.x; item < gx * n; item += blockDim.x) {
            const int g = item % gx, dyi = item / gx;
            const int dx0 = g * 4;
            int acc[4] = {0, 0, 0, 0};
#pragma unroll
            for (int by = 0; by < 4; by++) {
#pragma unroll
                for (int bx = 0; bx < 4; bx++) {
                    uint32_t p[4][4];  // [candidate][row]
#pragma unroll
                    for (int r = 0; r < 4; r++) {
                        const uint8_t* row = win + (dyi + by * 4 + r) * pitch + dx0 + bx * 4;
                        const uint32_t lo = win_word(row, 0), hi = win_word(row, 4);
                        p[0][r] = lo;
                        p[1][r] = __funnelshift_r(lo, hi, 8);
                        p[2][r] = __funnelshift_r(lo, hi, 16);
                        p[3][r] = __funnelshift_r(lo, hi, 24);
                    }
                    const uint32_t sr[4] = {src_s[by * 4][bx], src_s[by * 4 + 1][bx], src_s[by * 4 + 2][bx],
                                            src_s[by * 4 + 3][bx]};
#pragma unroll
                    for (int q = 0; q < 4; q++) acc[q] += satd4x4_rows(sr, p[q]);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int dxi = dx0 + q;
                if (dxi < n) {
                    const int idx = dyi * n + dxi;
                    if (a.satd_grid) a.satd_grid[grid_base + idx] = acc[q];
                    if (argmin) {
                        const long long key =
                            (grid_cost(a, acc[q], (cxf + dxi - R) * 4, (cyf + dyi - R) * 4, pmx, pmy) << 32) |
                            (long long)idx;
                        best_key = key < best_key ? key : best_key;
                    }
                }
            }
        }
    }
    // ---- argmin over the CTA ----
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const long long other = __shfl_xor_sync(0xffffffffu, best_key, o);
        best_key = other < best_key ? other : best_key;
    }
    if ((threadIdx.x & 31) == 0) red_key[threadIdx.x >> 5] = best_key;
    __syncthreads();
    if (threadIdx.x == 0 && a.best && argmin) {
        long long k = red_key[0];
        for (int i = 1; i < GRID_THREADS / 32; i++) k = red_key[i] < k ? red_key[i] : k;
        grid_store_best(a, mb, k, cxf, cyf, pmx, pmy);
    }
}

}  // namespace h264a

using namespace h264a;

extern "C" int h264a_fullpel_grid(h264a_ctx* ctx, const h264a_picture* h_pic, int R, const int32_t* d_centers,
                                  const int32_t* d_pmv, int metric, int mv_cost_kind, const uint16_t* d_mv_cost_tab,
                                  double lambda, int32_t* d_sad_grid, int32_t* d_satd_grid, int32_t* d_best,
                                  void* stream) {
    if (!ctx || !h_pic || !h_pic->d_src || !h_pic->d_planes) return fail(H264A_E_ARG, "fullpel_grid: null pointer");
    if (R < 1 || R > 64) return fail(H264A_E_ARG, "fullpel_grid: 1 <= R <= 64");
    if (metric != 0 && metric != 1) return fail(H264A_E_ARG, "fullpel_grid: metric 0 (SAD) or 1 (SATD)");
    if ((mv_cost_kind == 1 || mv_cost_kind == 2) && !d_mv_cost_tab)
        return fail(H264A_E_ARG, "fullpel_grid: mv cost kinds 1 and 2 need a table");
    const h264a_picture& pc = *h_pic;
    if (pc.cw < 16 || pc.ch < 16 || pc.cw % 16 || pc.ch % 16 || pc.pad < 3 || pc.pad > 128)
        return fail(H264A_E_ARG, "fullpel_grid: MB-aligned picture with 3 <= pad <= 128");
    GridArgs a;
    a.P.base = pc.d_planes;
    a.P.pad = pc.pad;
    a.P.pw = pc.cw + 2 * pc.pad;
    a.P.ph = pc.ch + 2 * pc.pad;
    a.P.ps = (long long)a.P.pw * a.P.ph;
    a.src = pc.d_src;
    a.cw = pc.cw;
    a.ch = pc.ch;
    a.mb_w = pc.cw / 16;
    a.R = R;
    a.centers = d_centers;
    a.pmv = d_pmv;
    a.metric = metric;
    a.kind = mv_cost_kind;
    a.tab = d_mv_cost_tab;
    a.lambda = lambda;
    a.sad_grid = d_sad_grid;
    a.satd_grid = d_satd_grid;
    a.best = d_best;
    const int ws = 16 + 2 * R;
    const int pitch = (ws + 4 + 3) & ~3;
    const size_t smem = (size_t)(ws + GRID_K) * pitch;  // one window
    const int nmb = (pc.cw / 16) * (pc.ch / 16);
    cudaStream_t st = pick_stream(ctx, stream);
    // one launch per metric wanted (its grid, or the argmin's metric)
    if (d_sad_grid || metric == 0) {
        // MBs per CTA: the most even fill of whole rounds of GRID_THREADS
        // items, at most SAD_MAX_MBS windows and 100 KB (two CTAs per SM)
        const int n = 2 * R + 1, per_mb = n * ((n + GRID_K - 1) / GRID_K);
        const int win_bytes = int((smem + 15) & ~size_t(15));
        int mbs = 1;
        double best_fill = 0.0;
        for (int m = 1; m <= SAD_MAX_MBS && size_t(m) * win_bytes <= 100 * 1024; m++) {
            const int rounds = (m * per_mb + GRID_THREADS - 1) / GRID_THREADS;
            const double fill = double(m * per_mb) / double(rounds * GRID_THREADS);
            if (fill > best_fill + 1e-9) {
                best_fill = fill;
                mbs = m;
            }
        }
        const size_t sm = size_t(mbs) * win_bytes;
        if (sm > 48 * 1024)
            H264A_CUDA(cudaFuncSetAttribute(fullpel_sad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sm)));
        fullpel_sad_kernel<<<unsigned((nmb + mbs - 1) / mbs), GRID_THREADS, sm, st>>>(a, mbs, nmb, win_bytes);
        const int rc = check_launch("fullpel_sad_kernel");
        if (rc) return rc;
    }
    if (d_satd_grid || metric == 1) {
        if (smem > 48 * 1024)
            H264A_CUDA(cudaFuncSetAttribute(fullpel_satd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        fullpel_satd_kernel<<<nmb, GRID_THREADS, smem, st>>>(a);
        const int rc = check_launch("fullpel_satd_kernel");
        if (rc) return rc;
    }
    return H264A_OK;
}
