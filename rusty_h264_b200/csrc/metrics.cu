// metrics.cu -- a6/a7/a8 block metrics and a3/a4/a5/a9 candidate distortion.
//
// One thread per 4x4 sub-block; the sub-blocks of one block sit in an aligned
// group of nb = (w/4)(h/4) lanes and are summed with xor shuffles, so a warp
// finishes 32/nb blocks per pass.
#include "h264a_device.cuh"

namespace h264a {

__device__ __forceinline__ int nb_log2(int w, int h) { return (w == 16 ? 2 : (w == 8 ? 1 : 0)) + (h == 16 ? 2 : (h == 8 ? 1 : 0)); }

__global__ void block_metric_kernel(int metric, int w, int h, const uint8_t* __restrict__ A,
                                    const int64_t* __restrict__ a_off, int sa, const uint8_t* __restrict__ B,
                                    const int64_t* __restrict__ b_off, const uint8_t* __restrict__ Cc,
                                    const int64_t* __restrict__ c_off, int sb, int n, int32_t* __restrict__ out) {
    const int lg = nb_log2(w, h);
    const int nb = 1 << lg;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long pair = t >> lg;
    const int blk = int(t & (nb - 1));
    const int nbx = w >> 2;
    int v = 0;
    if (pair < n) {
        const int bx = (blk % nbx) * 4, by = (blk / nbx) * 4;
        const uint8_t* a = A + a_off[pair] + (long long)by * sa + bx;
        const uint8_t* b = B + b_off[pair] + (long long)by * sb + bx;
        uint32_t s[4], p[4];
#pragma unroll
        for (int r = 0; r < 4; r++) s[r] = ld4u(a + (long long)r * sa);
        if (metric == H264A_METRIC_SATD_AVG || metric == H264A_METRIC_SAD_AVG) {
            const uint8_t* c = Cc + c_off[pair] + (long long)by * sb + bx;
#pragma unroll
            for (int r = 0; r < 4; r++) p[r] = avg_up4(ld4u(b + (long long)r * sb), ld4u(c + (long long)r * sb));
        } else {
#pragma unroll
            for (int r = 0; r < 4; r++) p[r] = ld4u(b + (long long)r * sb);
        }
        if (metric == H264A_METRIC_SAD || metric == H264A_METRIC_SAD_AVG) {
            v = sad4x4_rows(s, p);
        } else {
            v = satd4x4_rows(s, p);
            if (metric == H264A_METRIC_SATD_WELS) v = (v + 1) >> 1;
        }
    }
    v = warp_seg_sum(v, nb);
    if (pair < n && blk == 0) out[pair] = v;
}

__device__ __forceinline__ bool dev_shape_ok(int w, int h) {
    return (w == 16 && (h == 16 || h == 8)) || (w == 8 && (h == 16 || h == 8 || h == 4)) ||
           (w == 4 && (h == 8 || h == 4));
}

// Out-of-range requests (bad picture index, shape, or a block outside its
// source picture) read nothing and report -1.
__global__ void candidate_dist_kernel(const h264a_picture* __restrict__ pics, int npics,
                                      const h264a_candidate* __restrict__ cands, int n, int metric,
                                      int32_t* __restrict__ out) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long ci = t >> 4;  // 16 lanes per candidate (the largest block)
    const int blk = int(t & 15);
    int v = 0;
    bool valid = false;
    if (ci < n) {
        const h264a_candidate c = cands[ci];
        valid = c.pic >= 0 && c.pic < npics && dev_shape_ok(c.w, c.h);
        h264a_picture pc{};
        if (valid) {
            pc = pics[c.pic];
            valid = c.x >= 0 && c.y >= 0 && c.x + c.w <= pc.cw && c.y + c.h <= pc.ch;
        }
        const int nbx = c.w >> 2, nb = valid ? nbx * (c.h >> 2) : 0;
        if (blk < nb) {
            Planes P{pc.d_planes, pc.cw + 2 * pc.pad, pc.ch + 2 * pc.pad, pc.pad, 0};
            P.ps = (long long)P.pw * P.ph;
            const int bx = (blk % nbx) * 4, by = (blk / nbx) * 4;
            uint32_t s[4], p[4];
#pragma unroll
            for (int r = 0; r < 4; r++) s[r] = ld4u(pc.d_src + (long long)(c.y + by + r) * pc.cw + c.x + bx);
            pred_rows(P, c.x + bx + (c.mvx >> 2), c.y + by + (c.mvy >> 2), c.mvx & 3, c.mvy & 3, p);
            v = metric == H264A_METRIC_SAD ? sad4x4_rows(s, p) : satd4x4_rows(s, p);
        }
    }
    v = warp_seg_sum(v, 16);
    if (ci < n && blk == 0) out[ci] = valid ? v : -1;
}

static bool shape_ok(int w, int h) {
    return (w == 16 && (h == 16 || h == 8)) || (w == 8 && (h == 16 || h == 8 || h == 4)) || (w == 4 && (h == 8 || h == 4));
}

}  // namespace h264a

using namespace h264a;

extern "C" int h264a_block_metric(h264a_ctx* ctx, int metric, int w, int h, const uint8_t* d_a, const int64_t* d_a_off,
                                  int sa, const uint8_t* d_b, const int64_t* d_b_off, const uint8_t* d_c,
                                  const int64_t* d_c_off, int sb, int n, int32_t* d_out, void* stream) {
    if (!ctx || !d_a || !d_a_off || !d_b || !d_b_off || !d_out) return fail(H264A_E_ARG, "block_metric: null pointer");
    if (metric < 0 || metric > 4) return fail(H264A_E_ARG, "block_metric: unknown metric");
    if (!shape_ok(w, h)) return fail(H264A_E_ARG, "block_metric: unsupported block shape");
    if ((metric == H264A_METRIC_SATD_AVG || metric == H264A_METRIC_SAD_AVG) && (!d_c || !d_c_off))
        return fail(H264A_E_ARG, "block_metric: averaging metric needs the third operand");
    if (n < 0 || sa < w || sb < w) return fail(H264A_E_ARG, "block_metric: bad count or stride");
    if (n == 0) return H264A_OK;
    const long long threads = (long long)n * (w / 4) * (h / 4);
    const int bs = 256;
    block_metric_kernel<<<unsigned((threads + bs - 1) / bs), bs, 0, pick_stream(ctx, stream)>>>(
        metric, w, h, d_a, d_a_off, sa, d_b, d_b_off, d_c, d_c_off, sb, n, d_out);
    return check_launch("block_metric_kernel");
}

extern "C" int h264a_candidate_dist(h264a_ctx* ctx, const h264a_picture* d_pics, int npics,
                                    const h264a_candidate* d_cands, int n, int metric, int32_t* d_out, void* stream) {
    if (!ctx || !d_pics || !d_cands || !d_out) return fail(H264A_E_ARG, "candidate_dist: null pointer");
    if (metric != H264A_METRIC_SATD && metric != H264A_METRIC_SAD)
        return fail(H264A_E_ARG, "candidate_dist: metric must be SATD or SAD");
    if (n < 0) return fail(H264A_E_ARG, "candidate_dist: negative count");
    if (n == 0) return H264A_OK;
    const long long threads = (long long)n * 16;
    const int bs = 256;
    candidate_dist_kernel<<<unsigned((threads + bs - 1) / bs), bs, 0, pick_stream(ctx, stream)>>>(
        d_pics, npics, d_cands, n, metric, d_out);
    return check_launch("candidate_dist_kernel");
}
