// grid.cu -- exhaustive full-pel cost grids: 16x16 SAD and SATD of every
// integer offset within ±R of each MB's centre, the distortions the ME cost
// functions return at full-pel MVs (mc_sad_hp / mc_satd_hp,
// crates/rusty_h264-encoder/src/mb16.rs:1930-2074), and the per-MB argmin of
// dist + (λ·bits(mv − pmv)) in raster order with first-wins ties, the order of
// the exhaustive probe in motion_search (mb16.rs:2889-2900).
//
// One CTA per MB and metric.  The (16+2R)² search window (edge reads clamped,
// i.e. read from the padded F plane with clamping) is staged once in shared
// memory and the source MB is held in registers.
//  * SAD: a thread owns one column offset and a run of K row offsets; every
//    window row is loaded and byte-aligned once and feeds the K candidates it
//    overlaps with one packed __vsadu4 per 4 pixels.
//  * SATD: a thread owns four horizontally adjacent offsets; two aligned words
//    per window row segment yield all four candidates' rows by funnel shifts.
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

// One metric per instance (METRIC 0 SAD, 1 SATD), so that each keeps the
// source MB in registers without spilling at two CTAs per SM; the instance
// whose metric is a.metric also forms the argmin.
template <int METRIC>
__global__ void __launch_bounds__(GRID_THREADS, 2) fullpel_grid_kernel(GridArgs a) {
    extern __shared__ __align__(16) uint8_t win[];
    __shared__ long long red_key[GRID_THREADS / 32];
    const int mb = blockIdx.x;
    const int mbx = mb % a.mb_w, mby = mb / a.mb_w;
    const int lx = mbx * 16, ly = mby * 16;
    const int R = a.R, n = 2 * R + 1;
    int cxf = 0, cyf = 0;
    if (a.centers) {
        cxf = (a.centers[2 * mb] + 2) >> 2;  // snapped like motion_search's integer snap
        cyf = (a.centers[2 * mb + 1] + 2) >> 2;
    }
    const int pmx = a.pmv ? a.pmv[2 * mb] : 0, pmy = a.pmv ? a.pmv[2 * mb + 1] : 0;
    const int ws = 16 + 2 * R;                     // window side
    const int pitch = (ws + 4 + 3) & ~3;           // room for the 5th word of an unaligned read
    const int wrows = ws + GRID_K;                 // spare rows for the last partial SAD chunk
    // stage the clamped window: picture coords (lx+cxf-R+x, ly+cyf-R+y)
    const int ox = lx + cxf - R + a.P.pad, oy = ly + cyf - R + a.P.pad;
    for (int y = threadIdx.x >> 5; y < wrows; y += GRID_THREADS / 32) {  // a row per warp, lanes along it
        const uint8_t* prow = a.P.base + (long long)clampi(oy + y, 0, a.P.ph - 1) * a.P.pw;
        for (int x = threadIdx.x & 31; x < pitch; x += 32)
            win[y * pitch + x] = (y < ws && x < ws) ? __ldg(prow + clampi(ox + x, 0, a.P.pw - 1)) : uint8_t(0);
    }
    // the source MB: in registers for SAD, in shared memory for SATD (whose
    // four candidates' rows need the registers)
    __shared__ uint32_t src_s[16][4];
    uint32_t s[16][4];
    if (METRIC == 0) {
#pragma unroll
        for (int r = 0; r < 16; r++)
#pragma unroll
            for (int c = 0; c < 4; c++) s[r][c] = ld4u(a.src + (long long)(ly + r) * a.cw + lx + 4 * c);
    } else if (threadIdx.x < 64) {
        src_s[threadIdx.x >> 2][threadIdx.x & 3] =
            ld4u(a.src + (long long)(ly + (threadIdx.x >> 2)) * a.cw + lx + 4 * (threadIdx.x & 3));
    }
    __syncthreads();

    long long best_key = LLONG_MAX;  // (cost << 32) | scan index; min = first-wins argmin
    const long long grid_base = (long long)mb * n * n;
    const bool argmin = a.metric == METRIC;

    // ---- SAD ----
    if (METRIC == 0) {
        const int chunks = (n + GRID_K - 1) / GRID_K;
        for (int item = threadIdx.x; item < n * chunks; item += blockDim.x) {
            const int dxi = item % n, ch = item / n;
            const int dy0 = ch * GRID_K;
            int acc[GRID_K];
#pragma unroll
            for (int k = 0; k < GRID_K; k++) acc[k] = 0;
#pragma unroll
            for (int i = 0; i < GRID_K + 15; i++) {
                const uint8_t* row = win + (dy0 + i) * pitch;
                uint32_t w[4];
#pragma unroll
                for (int c = 0; c < 4; c++) w[c] = win_word(row, dxi + 4 * c);
#pragma unroll
                for (int k = 0; k < GRID_K; k++) {
                    const int r = i - k;
                    if (r >= 0 && r < 16)
                        acc[k] += int(__vsadu4(s[r][0], w[0]) + __vsadu4(s[r][1], w[1]) + __vsadu4(s[r][2], w[2]) +
                                      __vsadu4(s[r][3], w[3]));
                }
            }
#pragma unroll
            for (int k = 0; k < GRID_K; k++) {
                const int dyi = dy0 + k;
                if (dyi < n) {
                    const int idx = dyi * n + dxi;
                    if (a.sad_grid) a.sad_grid[grid_base + idx] = acc[k];
                    if (argmin) {
                        const int mvx = (cxf + dxi - R) * 4, mvy = (cyf + dyi - R) * 4;
                        const long long cost =
                            acc[k] + lam_cost(a.lambda, mvbits(a.kind, a.tab, mvx - pmx) + mvbits(a.kind, a.tab, mvy - pmy));
                        const long long key = (cost << 32) | (long long)idx;
                        best_key = key < best_key ? key : best_key;
                    }
                }
            }
        }
    }
    // ---- SATD ----
    if (METRIC == 1) {
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
                        const int mvx = (cxf + dxi - R) * 4, mvy = (cyf + dyi - R) * 4;
                        const long long cost =
                            acc[q] + lam_cost(a.lambda, mvbits(a.kind, a.tab, mvx - pmx) + mvbits(a.kind, a.tab, mvy - pmy));
                        const long long key = (cost << 32) | (long long)idx;
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
        const int idx = int(k & 0xffffffffLL);
        const long long cost = k >> 32;
        const int dyi = idx / n, dxi = idx % n;
        const int mvx = (cxf + dxi - R) * 4, mvy = (cyf + dyi - R) * 4;
        const long long rc = lam_cost(a.lambda, mvbits(a.kind, a.tab, mvx - pmx) + mvbits(a.kind, a.tab, mvy - pmy));
        a.best[4 * mb + 0] = mvx;
        a.best[4 * mb + 1] = mvy;
        a.best[4 * mb + 2] = int32_t(cost > 0x7fffffffLL ? 0x7fffffffLL : cost);
        a.best[4 * mb + 3] = int32_t(cost - rc);
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
    const size_t smem = (size_t)(ws + GRID_K) * pitch;
    const int nmb = (pc.cw / 16) * (pc.ch / 16);
    cudaStream_t st = pick_stream(ctx, stream);
    // one launch per metric wanted (its grid, or the argmin's metric)
    if (d_sad_grid || metric == 0) {
        if (smem > 48 * 1024)
            H264A_CUDA(cudaFuncSetAttribute(fullpel_grid_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        fullpel_grid_kernel<0><<<nmb, GRID_THREADS, smem, st>>>(a);
        const int rc = check_launch("fullpel_grid_kernel<SAD>");
        if (rc) return rc;
    }
    if (d_satd_grid || metric == 1) {
        if (smem > 48 * 1024)
            H264A_CUDA(cudaFuncSetAttribute(fullpel_grid_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
        fullpel_grid_kernel<1><<<nmb, GRID_THREADS, smem, st>>>(a);
        const int rc = check_launch("fullpel_grid_kernel<SATD>");
        if (rc) return rc;
    }
    return H264A_OK;
}
