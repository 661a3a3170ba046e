// closed.cu -- the closed reconstruction loop: motion search against the
// deblocked reconstruction of the previous frame, as the reference encoder
// searches RefFrames built from its reconstructed planes
// (crates/rusty_h264-encoder/src/lib.rs:228-262).
//
// Per P frame f, on one stream, every step a kernel of this library:
//   planes of rec(f-1)                          h264a_hpel_build
//   [learned: proposals from (src f, rec f-1)]  h264a_mvnet_propose
//   motion search of src f on those planes      h264a_me_frames / _learned
//   MC + luma T/Q + luma reconstruction         h264a_mc_tq_rec_frames
//   chroma MC + T/Q + reconstruction            h264a_mc_tq_chroma_frames
//   in-loop deblocking of rec(f)                h264a_deblock_frames
// Frame f depends on all of rec(f-1) (a search may reach any row of the
// reference), so the frames run one after another and the parallelism is the
// MBs of one frame (the wavefront kernels).  Frame 0 reconstructs to itself
// (the frame model codes it losslessly).
#include <cstring>
#include <string>
#include <vector>

#include "h264accel_internal.h"

namespace {

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

int dev_alloc(DevBuf& b, size_t bytes) {
    if (cudaMalloc(&b.p, bytes) != cudaSuccess) {
        cudaGetLastError();
        return h264a::fail(H264A_E_NOMEM, "pixel_path_closed: cudaMalloc failed");
    }
    return H264A_OK;
}

}  // namespace

using namespace h264a;

extern "C" int h264a_pixel_path_closed(h264a_ctx* ctx, const h264a_closed_job* job, const h264a_me_params* params,
                                       const uint16_t* h_mv_cost_tab) {
    if (!ctx || !job || !params) return fail(H264A_E_ARG, "pixel_path_closed: null pointer");
    const int n = job->n, cw = job->cw, ch = job->ch;
    if (!job->h_y || !job->h_u || !job->h_v || !job->h_picks || !job->h_costs)
        return fail(H264A_E_ARG, "pixel_path_closed: null frame or output pointer");
    if (n < 1 || cw < 16 || ch < 16 || cw % 16 || ch % 16 || (long long)cw * ch > (1LL << 26))
        return fail(H264A_E_ARG, "pixel_path_closed: frames must be MB-aligned and at least one");
    if (job->qp < 0 || job->qp > 51 || job->dz_div < 1) return fail(H264A_E_ARG, "pixel_path_closed: bad qp/dz_div");
    if (job->net && job->fallback_t < 0) return fail(H264A_E_ARG, "pixel_path_closed: negative fallback threshold");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !h_mv_cost_tab)
        return fail(H264A_E_ARG, "pixel_path_closed: mv cost kinds 1 and 2 need the table");
    H264A_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int pad = 32, pw = cw + 2 * pad, ph = ch + 2 * pad;
    const int mb_w = cw / 16, mb_h = ch / 16, nmb = mb_w * mb_h;
    const size_t fs = size_t(cw) * ch, cs = fs / 4, ps4 = size_t(4) * pw * ph;
    // device layout: src Y|U|V, rec Y|U|V (n frames each), planes (one
    // picture), picks, costs, luma and chroma levels, proposals, lookahead
    DevBuf b_src, b_rec, b_planes, b_picks, b_costs, b_coef, b_ccoef, b_tab, b_props, b_fb, b_half, b_la;
    int rc = dev_alloc(b_src, n * (fs + 2 * cs));
    if (!rc) rc = dev_alloc(b_rec, n * (fs + 2 * cs));
    if (!rc) rc = dev_alloc(b_planes, ps4);
    if (!rc) rc = dev_alloc(b_picks, sizeof(int32_t) * 6 * nmb * n);
    if (!rc) rc = dev_alloc(b_costs, sizeof(int64_t) * 2 * nmb * n);
    if (!rc) rc = dev_alloc(b_coef, sizeof(int16_t) * 256 * nmb * n);
    if (!rc) rc = dev_alloc(b_ccoef, sizeof(int16_t) * 128 * nmb * n);
    if (!rc) rc = dev_alloc(b_tab, sizeof(uint16_t) * 4096);
    if (!rc && job->net) rc = dev_alloc(b_props, sizeof(int32_t) * 16 * nmb * n);
    if (!rc && job->net) rc = dev_alloc(b_fb, sizeof(int32_t) * nmb * n);
    if (!rc && job->net) rc = dev_alloc(b_half, n * fs / 4);
    if (!rc && job->net) rc = dev_alloc(b_la, sizeof(int32_t) * 4 * nmb * n);
    if (rc) return rc;
    uint8_t* sy = static_cast<uint8_t*>(b_src.p);
    uint8_t* su = sy + n * fs;
    uint8_t* sv = su + n * cs;
    uint8_t* ry = static_cast<uint8_t*>(b_rec.p);
    uint8_t* ru = ry + n * fs;
    uint8_t* rv = ru + n * cs;
    uint8_t* planes = static_cast<uint8_t*>(b_planes.p);
    int32_t* picks = static_cast<int32_t*>(b_picks.p);
    int64_t* costs = static_cast<int64_t*>(b_costs.p);
    int16_t* coef = static_cast<int16_t*>(b_coef.p);
    int16_t* ccoef = static_cast<int16_t*>(b_ccoef.p);
    int32_t* props = static_cast<int32_t*>(b_props.p);
    int32_t* fb = static_cast<int32_t*>(b_fb.p);
    H264A_CUDA(cudaMemcpyAsync(sy, job->h_y, n * fs, cudaMemcpyHostToDevice, st));
    H264A_CUDA(cudaMemcpyAsync(su, job->h_u, n * cs, cudaMemcpyHostToDevice, st));
    H264A_CUDA(cudaMemcpyAsync(sv, job->h_v, n * cs, cudaMemcpyHostToDevice, st));
    h264a_me_params prm = *params;
    if (h_mv_cost_tab) {
        H264A_CUDA(cudaMemcpyAsync(b_tab.p, h_mv_cost_tab, sizeof(uint16_t) * 4096, cudaMemcpyHostToDevice, st));
        prm.d_mv_cost_tab = static_cast<const uint16_t*>(b_tab.p);
    }
    H264A_CUDA(cudaMemsetAsync(picks, 0, sizeof(int32_t) * 6 * nmb, st));
    H264A_CUDA(cudaMemsetAsync(costs, 0, sizeof(int64_t) * 2 * nmb, st));
    H264A_CUDA(cudaMemsetAsync(coef, 0, sizeof(int16_t) * 256 * nmb, st));
    H264A_CUDA(cudaMemsetAsync(ccoef, 0, sizeof(int16_t) * 128 * nmb, st));
    // frame 0: coded losslessly, its reconstruction is the source
    H264A_CUDA(cudaMemcpyAsync(ry, sy, fs, cudaMemcpyDeviceToDevice, st));
    H264A_CUDA(cudaMemcpyAsync(ru, su, cs, cudaMemcpyDeviceToDevice, st));
    H264A_CUDA(cudaMemcpyAsync(rv, sv, cs, cudaMemcpyDeviceToDevice, st));
    int32_t* la_mvs = nullptr;
    if (job->net) {
        // guide MVs of the proposals: the HalfRes lookahead over the source
        // frames, known before any search runs
        H264A_CUDA(cudaMemsetAsync(props, 0, sizeof(int32_t) * 16 * nmb, st));
        H264A_CUDA(cudaMemsetAsync(fb, 0, sizeof(int32_t) * nmb, st));
        uint8_t* half = static_cast<uint8_t*>(b_half.p);
        int32_t* la = static_cast<int32_t*>(b_la.p);
        la_mvs = la + 2 * nmb * n;
        rc = h264a_downsample2x(ctx, sy, cw, ch, n, fs, half, st);
        if (!rc) rc = h264a_lookahead_costs(ctx, sy, half, cw, ch, n, 2, la, la + nmb * n, la_mvs, st);
        if (rc) return rc;
    }
    for (int f = 1; f < n && !rc; f++) {
        rc = h264a_hpel_build(ctx, ry + (f - 1) * fs, cw, ch, pad, 1, fs, planes, st);
        if (rc) break;
        h264a_me_frame mf;
        mf.pic = h264a_picture{sy + f * fs, planes, cw, ch, pad};
        mf.lambda_me = job->lambda_me;
        mf.split_gate = job->split_gate;
        mf.d_picks = picks + 6LL * nmb * f;
        mf.d_costs = costs + 2LL * nmb * f;
        if (job->net) {
            h264a_mvnet_frame nf{sy + f * fs, ry + (f - 1) * fs, cw, ch, la_mvs + 2LL * nmb * f, props + 16LL * nmb * f};
            rc = h264a_mvnet_propose(job->net, &nf, 1, st);
            if (rc) break;
            h264a_me_learned_frame lf{mf, props + 16LL * nmb * f, job->fallback_t, fb + (long long)nmb * f};
            rc = h264a_me_frames_learned(ctx, &lf, 1, &prm, st);
        } else {
            rc = h264a_me_frames(ctx, &mf, 1, &prm, st);
        }
        if (rc) break;
        h264a_tq_rec_frame tr;
        tr.tq = h264a_tq_frame{mf.pic, mf.d_picks, job->qp, job->dz_div, coef + 256LL * nmb * f};
        tr.d_rec = ry + f * fs;
        rc = h264a_mc_tq_rec_frames(ctx, &tr, 1, st);
        if (rc) break;
        h264a_tq_chroma_frame cf{su + f * cs, sv + f * cs, ru + (f - 1) * cs, rv + (f - 1) * cs, cw, ch, mf.d_picks,
                                 job->qp, ccoef + 128LL * nmb * f, ru + f * cs, rv + f * cs};
        rc = h264a_mc_tq_chroma_frames(ctx, &cf, 1, st);
        if (rc) break;
        h264a_deblock_frame df{ry + f * fs, ru + f * cs, rv + f * cs, cw, ch, mf.d_picks, coef + 256LL * nmb * f,
                               job->qp, 0, 0, 0};
        rc = h264a_deblock_frames(ctx, &df, 1, st);
    }
    if (rc) {
        cudaStreamSynchronize(st);
        return rc;
    }
    H264A_CUDA(cudaMemcpyAsync(job->h_picks, picks, sizeof(int32_t) * 6 * nmb * n, cudaMemcpyDeviceToHost, st));
    H264A_CUDA(cudaMemcpyAsync(job->h_costs, costs, sizeof(int64_t) * 2 * nmb * n, cudaMemcpyDeviceToHost, st));
    if (job->h_coeffs)
        H264A_CUDA(cudaMemcpyAsync(job->h_coeffs, coef, sizeof(int16_t) * 256 * nmb * n, cudaMemcpyDeviceToHost, st));
    if (job->h_ccoeffs)
        H264A_CUDA(cudaMemcpyAsync(job->h_ccoeffs, ccoef, sizeof(int16_t) * 128 * nmb * n, cudaMemcpyDeviceToHost, st));
    if (job->h_rec_y) H264A_CUDA(cudaMemcpyAsync(job->h_rec_y, ry, n * fs, cudaMemcpyDeviceToHost, st));
    if (job->h_rec_u) H264A_CUDA(cudaMemcpyAsync(job->h_rec_u, ru, n * cs, cudaMemcpyDeviceToHost, st));
    if (job->h_rec_v) H264A_CUDA(cudaMemcpyAsync(job->h_rec_v, rv, n * cs, cudaMemcpyDeviceToHost, st));
    if (job->net && job->h_props)
        H264A_CUDA(cudaMemcpyAsync(job->h_props, props, sizeof(int32_t) * 16 * nmb * n, cudaMemcpyDeviceToHost, st));
    if (job->net && job->h_fallback)
        H264A_CUDA(cudaMemcpyAsync(job->h_fallback, fb, sizeof(int32_t) * nmb * n, cudaMemcpyDeviceToHost, st));
    return h264a_sync(ctx, st);
}
