// closed.cu -- the closed reconstruction loop: motion search against the
// deblocked reconstruction of the previous frame, as the reference encoder
// searches RefFrames built from its reconstructed planes
// (crates/rusty_h264-encoder/src/lib.rs:228-262).
//
// The loop on the device: the planes of rec(0) (h264a_hpel_build), then
// every P frame in one launch of the pipelined kernel (closed_pipe_kernel,
// me.cu): each MB's search (the wide kernel's), its MC + T/Q and
// reconstruction of luma and chroma and its in-loop deblocking in the same
// CTA, and the planes of each reconstruction built segment by segment
// (16 picture rows by 16 MB columns) as its MBs are deblocked, so that about
// ten frames' wavefronts run at once, each a few MBs behind the one before.  With a proposal net the
// proposals of all frames come first, in one batched h264a_mvnet_propose pass
// over the source pairs (f, f-1).  One P frame alone is
// h264a_closed_step_frame (the planes of rec(f-1) are the caller's).
// Frame 0 reconstructs to itself (the frame model codes it losslessly).
#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "h264accel_internal.h"

using namespace h264a;

namespace {

constexpr int UPL_CHUNK = 4;  // frames per source upload of h264a_pixel_path_closed

int check_geometry(int n, int cw, int ch, int qp, int dz_div) {
    if (n < 1 || cw < 16 || ch < 16 || cw % 16 || ch % 16 || (long long)cw * ch > (1LL << 26))
        return fail(H264A_E_ARG, "closed loop: frames must be MB-aligned and at least one");
    if (qp < 0 || qp > 51 || dz_div < 1) return fail(H264A_E_ARG, "closed loop: qp out of 0..51 or dz_div < 1");
    return H264A_OK;
}

// One frame of the loop: the search with each MB's reconstruction and
// deblocking fused in (checked by the caller).
int step_run(h264a_ctx* ctx, const h264a_closed_step& s, const h264a_me_params& prm, cudaStream_t st) {
    const MeTqOut tq{s.d_coeffs, s.qp, s.dz_div, nullptr, nullptr, 0};
    const MeRecIn rec{s.d_u, s.d_v, s.d_ref_u, s.d_ref_v, s.d_rec_y, s.d_rec_u, s.d_rec_v, s.d_ccoeffs};
    if (s.d_props) {
        const MeLearnIn ln{s.d_props, s.d_fallback, s.fallback_t};
        return me_frames_run(ctx, &s.me, 1, &prm, &tq, st, &ln, &rec);
    }
    return me_frames_run(ctx, &s.me, 1, &prm, &tq, st, nullptr, &rec);
}

// The per-frame launches of the loop on device buffers (checked by the caller).
int closed_run(h264a_ctx* ctx, const h264a_closed_dev& j, const h264a_me_params& prm, cudaStream_t st,
               int32_t* frame_words = nullptr, int32_t token = 0, const int32_t* arrive = nullptr) {
    const int n = j.n, cw = j.cw, ch = j.ch, pad = 32;
    const int nmb = (cw / 16) * (ch / 16);
    const size_t fs = size_t(cw) * ch, cs = fs / 4;
    H264A_CUDA(cudaMemsetAsync(j.d_picks, 0, sizeof(int32_t) * 6 * nmb, st));
    H264A_CUDA(cudaMemsetAsync(j.d_costs, 0, sizeof(int64_t) * 2 * nmb, st));
    H264A_CUDA(cudaMemsetAsync(j.d_coeffs, 0, sizeof(int16_t) * 256 * nmb, st));
    H264A_CUDA(cudaMemsetAsync(j.d_ccoeffs, 0, sizeof(int16_t) * 128 * nmb, st));
    if (j.net) {
        H264A_CUDA(cudaMemsetAsync(j.d_props, 0, sizeof(int32_t) * 16 * nmb, st));
        if (j.d_fallback) H264A_CUDA(cudaMemsetAsync(j.d_fallback, 0, sizeof(int32_t) * nmb, st));
    }
    // frame 0: coded losslessly, its reconstruction is the source
    H264A_CUDA(cudaMemcpyAsync(j.d_rec_y, j.d_y, fs, cudaMemcpyDeviceToDevice, st));
    H264A_CUDA(cudaMemcpyAsync(j.d_rec_u, j.d_u, cs, cudaMemcpyDeviceToDevice, st));
    H264A_CUDA(cudaMemcpyAsync(j.d_rec_v, j.d_v, cs, cudaMemcpyDeviceToDevice, st));
    if (j.net && n > 1) {
        // the proposals of every P frame in one batched pass before the loop:
        // from the source pair (f, f-1), so none of them waits for a
        // reconstruction; the search prices them on rec(f-1)
        std::vector<h264a_mvnet_frame> nf(n - 1);
        for (int f = 1; f < n; f++)
            nf[f - 1] = h264a_mvnet_frame{j.d_y + f * fs, j.d_y + (f - 1) * fs, cw, ch,
                                          j.d_guide_mvs ? j.d_guide_mvs + 2LL * nmb * f : nullptr,
                                          j.d_props + 16LL * nmb * f};
        const int rc = h264a_mvnet_propose(j.net, nf.data(), n - 1, st);
        if (rc) return rc;
    }
    // the planes of rec(0) in the first plane buffer, then every P frame in
    // one pipelined launch
    int rc = h264a_hpel_build(ctx, j.d_rec_y, cw, ch, pad, 1, fs, j.d_planes, st);
    if (rc) return rc;
    ClosedPipeIn in;
    in.n = n; in.cw = cw; in.ch = ch; in.pad = pad;
    in.y = j.d_y; in.u = j.d_u; in.v = j.d_v;
    in.rec_y = j.d_rec_y; in.rec_u = j.d_rec_u; in.rec_v = j.d_rec_v;
    in.planes = j.d_planes;
    in.lambda_me = j.lambda_me;
    in.split_gate = j.split_gate;
    in.qp = j.qp; in.dz_div = j.dz_div;
    in.picks = j.d_picks; in.costs = j.d_costs; in.coeffs = j.d_coeffs; in.ccoeffs = j.d_ccoeffs;
    in.props = j.net ? j.d_props : nullptr;
    in.fallback = j.net ? j.d_fallback : nullptr;
    in.prop_t = j.fallback_t;
    in.arrive = arrive;
    in.atoken = token;
    rc = closed_pipe_run(ctx, in, &prm, st, frame_words, token);
    if (rc) return rc;
    return H264A_OK;
}

}  // namespace

extern "C" int h264a_closed_frames(h264a_ctx* ctx, const h264a_closed_dev* job, const h264a_me_params* params,
                                   void* stream) {
    if (!ctx || !job || !params) return fail(H264A_E_ARG, "closed_frames: null pointer");
    const h264a_closed_dev& j = *job;
    int rc = check_geometry(j.n, j.cw, j.ch, j.qp, j.dz_div);
    if (rc) return rc;
    if (!j.d_y || !j.d_u || !j.d_v || !j.d_rec_y || !j.d_rec_u || !j.d_rec_v || !j.d_planes || !j.d_picks ||
        !j.d_costs || !j.d_coeffs || !j.d_ccoeffs || (j.net && !j.d_props))
        return fail(H264A_E_ARG, "closed_frames: null device buffer");
    if (((reinterpret_cast<uintptr_t>(j.d_coeffs) | reinterpret_cast<uintptr_t>(j.d_ccoeffs)) & 15) ||
        ((reinterpret_cast<uintptr_t>(j.d_u) | reinterpret_cast<uintptr_t>(j.d_v) |
          reinterpret_cast<uintptr_t>(j.d_rec_u) | reinterpret_cast<uintptr_t>(j.d_rec_v)) & 3))
        return fail(H264A_E_ARG, "closed_frames: levels must be 16-byte and chroma 4-byte aligned");
    if (j.net && j.fallback_t < 0) return fail(H264A_E_ARG, "closed_frames: negative fallback threshold");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !params->d_mv_cost_tab)
        return fail(H264A_E_ARG, "closed_frames: mv cost kinds 1 and 2 need d_mv_cost_tab");
    return closed_run(ctx, j, *params, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int h264a_closed_step_frame(h264a_ctx* ctx, const h264a_closed_step* step, const h264a_me_params* params,
                                       void* stream) {
    if (!ctx || !step || !params) return fail(H264A_E_ARG, "closed_step_frame: null pointer");
    const h264a_closed_step& s = *step;
    if (s.qp < 0 || s.qp > 51 || s.dz_div < 1) return fail(H264A_E_ARG, "closed_step_frame: qp out of 0..51 or dz_div < 1");
    if (s.d_props && s.fallback_t < 0) return fail(H264A_E_ARG, "closed_step_frame: negative fallback threshold");
    return step_run(ctx, s, *params, reinterpret_cast<cudaStream_t>(stream));
}

extern "C" int h264a_pixel_path_closed(h264a_ctx* ctx, const h264a_closed_job* job, const h264a_me_params* params,
                                       const uint16_t* h_mv_cost_tab) {
    if (!ctx || !job || !params) return fail(H264A_E_ARG, "pixel_path_closed: null pointer");
    const int n = job->n, cw = job->cw, ch = job->ch;
    if (!job->h_y || !job->h_u || !job->h_v || !job->h_picks || !job->h_costs)
        return fail(H264A_E_ARG, "pixel_path_closed: null frame or output pointer");
    int rc = check_geometry(n, cw, ch, job->qp, job->dz_div);
    if (rc) return rc;
    if (job->net && job->fallback_t < 0) return fail(H264A_E_ARG, "pixel_path_closed: negative fallback threshold");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !h_mv_cost_tab)
        return fail(H264A_E_ARG, "pixel_path_closed: mv cost kinds 1 and 2 need the table");
    H264A_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const int pw = cw + 64, ph = ch + 64, nmb = (cw / 16) * (ch / 16);
    const size_t fs = size_t(cw) * ch, cs = fs / 4, cs_bytes = cs;
    // one cached device buffer, 256-byte aligned parts: src Y|U|V, rec Y|U|V,
    // planes, picks, costs, luma and chroma levels, mv-cost table, and with a
    // net the proposals, fallback flags, half-res frames and lookahead outputs
    size_t off = 0;
    auto part = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) & ~size_t(255);
        return o;
    };
    const size_t o_sy = part(n * fs), o_su = part(n * cs), o_sv = part(n * cs);
    const size_t o_ry = part(n * fs), o_ru = part(n * cs), o_rv = part(n * cs);
    const size_t o_pl = part(size_t(4) * std::min(n, H264A_CLOSED_PLANE_PICTURES) * pw * ph), o_pk = part(sizeof(int32_t) * 6 * nmb * n);
    const size_t o_co = part(sizeof(int64_t) * 2 * nmb * n), o_lv = part(sizeof(int16_t) * 256 * nmb * n);
    const size_t o_cl = part(sizeof(int16_t) * 128 * nmb * n), o_tab = part(sizeof(uint16_t) * 4096);
    const size_t o_arr = part(sizeof(int32_t) * n);
    size_t o_pr = 0, o_fb = 0, o_half = 0, o_la = 0;
    if (job->net) {
        o_pr = part(sizeof(int32_t) * 16 * nmb * n);
        o_fb = part(sizeof(int32_t) * nmb * n);
        o_half = part(n * fs / 4);
        o_la = part(sizeof(int32_t) * 4 * nmb * n);
    }
    if (off > ctx->cl_bytes) {
        if (ctx->cl_buf) cudaFree(ctx->cl_buf);
        ctx->cl_buf = nullptr;
        ctx->cl_bytes = 0;
        if (cudaMalloc(&ctx->cl_buf, off) != cudaSuccess) {
            cudaGetLastError();
            return fail(H264A_E_NOMEM, "pixel_path_closed: cudaMalloc failed");
        }
        ctx->cl_bytes = off;
    }
    char* b = static_cast<char*>(ctx->cl_buf);
    h264a_closed_dev j;
    memset(&j, 0, sizeof j);
    j.d_y = reinterpret_cast<uint8_t*>(b + o_sy);
    j.d_u = reinterpret_cast<uint8_t*>(b + o_su);
    j.d_v = reinterpret_cast<uint8_t*>(b + o_sv);
    j.d_rec_y = reinterpret_cast<uint8_t*>(b + o_ry);
    j.d_rec_u = reinterpret_cast<uint8_t*>(b + o_ru);
    j.d_rec_v = reinterpret_cast<uint8_t*>(b + o_rv);
    j.d_planes = reinterpret_cast<uint8_t*>(b + o_pl);
    j.n = n; j.cw = cw; j.ch = ch;
    j.lambda_me = job->lambda_me; j.split_gate = job->split_gate; j.qp = job->qp; j.dz_div = job->dz_div;
    j.net = job->net; j.fallback_t = job->fallback_t;
    j.d_picks = reinterpret_cast<int32_t*>(b + o_pk);
    j.d_costs = reinterpret_cast<int64_t*>(b + o_co);
    j.d_coeffs = reinterpret_cast<int16_t*>(b + o_lv);
    j.d_ccoeffs = reinterpret_cast<int16_t*>(b + o_cl);
    // The sources: with a net, all of them before anything runs (the
    // proposals of every frame come first); without, frame 0 before the
    // loop and the others on the upload stream beside it, in chunks of
    // UPL_CHUNK frames, each chunk followed by its frames' arrival words
    // (copied from pinned host words holding the call's token), which the
    // pipelined kernel waits for before it reads a frame's sources.
    const int up_n = job->net ? n : 1;
    H264A_CUDA(cudaMemcpyAsync(const_cast<uint8_t*>(j.d_y), job->h_y, up_n * fs, cudaMemcpyHostToDevice, st));
    H264A_CUDA(cudaMemcpyAsync(const_cast<uint8_t*>(j.d_u), job->h_u, up_n * cs, cudaMemcpyHostToDevice, st));
    H264A_CUDA(cudaMemcpyAsync(const_cast<uint8_t*>(j.d_v), job->h_v, up_n * cs, cudaMemcpyHostToDevice, st));
    h264a_me_params prm = *params;
    if (h_mv_cost_tab) {
        H264A_CUDA(cudaMemcpyAsync(b + o_tab, h_mv_cost_tab, sizeof(uint16_t) * 4096, cudaMemcpyHostToDevice, st));
        prm.d_mv_cost_tab = reinterpret_cast<const uint16_t*>(b + o_tab);
    }
    if (job->net) {
        // guide MVs of the proposals: the HalfRes lookahead over the source
        // frames, known before any search runs
        j.d_props = reinterpret_cast<int32_t*>(b + o_pr);
        j.d_fallback = reinterpret_cast<int32_t*>(b + o_fb);
        uint8_t* half = reinterpret_cast<uint8_t*>(b + o_half);
        int32_t* la = reinterpret_cast<int32_t*>(b + o_la);
        j.d_guide_mvs = la + 2 * nmb * n;
        rc = h264a_downsample2x(ctx, j.d_y, cw, ch, n, fs, half, st);
        if (!rc) rc = h264a_lookahead_costs(ctx, j.d_y, half, cw, ch, n, 2, la, la + nmb * n, la + 2 * nmb * n, st);
        if (rc) return rc;
    }
    // Each frame's outputs go down on the copy stream as soon as the pipelined
    // kernel reports the frame final (a mapped word per frame), while later
    // frames still run; the kernel's completion event covers the rest.
    rc = ensure_pp_rows(ctx, size_t(n));
    if (rc) {
        cudaStreamSynchronize(st);
        return rc;
    }
    const int32_t token = next_pp_token(ctx);
    int32_t* arrive = job->net || n < 2 ? nullptr : reinterpret_cast<int32_t*>(b + o_arr);
    cudaStream_t up = ctx->pf_stream;
    if (arrive) {
        if (ctx->upl_cap < size_t(n)) {
            if (ctx->upl_tok) cudaFreeHost(ctx->upl_tok);
            ctx->upl_tok = nullptr;
            ctx->upl_cap = 0;
            if (cudaHostAlloc(reinterpret_cast<void**>(&ctx->upl_tok), sizeof(int32_t) * n, cudaHostAllocDefault) !=
                cudaSuccess) {
                cudaGetLastError();
                cudaStreamSynchronize(st);
                return fail(H264A_E_NOMEM, "pixel_path_closed: cudaHostAlloc failed");
            }
            ctx->upl_cap = size_t(n);
        }
        for (int f = 0; f < n; f++) ctx->upl_tok[f] = token;  // the upload stream is idle: nothing reads them now
        for (int f0 = 1; f0 < n; f0 += UPL_CHUNK) {
            const int k = std::min(UPL_CHUNK, n - f0);
            cudaError_t e = cudaMemcpyAsync(const_cast<uint8_t*>(j.d_y) + fs * f0, job->h_y + fs * f0, fs * k,
                                            cudaMemcpyHostToDevice, up);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(const_cast<uint8_t*>(j.d_u) + cs * f0, job->h_u + cs * f0, cs * k,
                                    cudaMemcpyHostToDevice, up);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(const_cast<uint8_t*>(j.d_v) + cs * f0, job->h_v + cs * f0, cs * k,
                                    cudaMemcpyHostToDevice, up);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(arrive + f0, ctx->upl_tok + f0, sizeof(int32_t) * k, cudaMemcpyHostToDevice, up);
            if (e != cudaSuccess) {
                cudaStreamSynchronize(up);
                cudaStreamSynchronize(st);
                return cuda_fail(e, "pixel_path_closed: source uploads");
            }
        }
    }
    rc = closed_run(ctx, j, prm, st, ctx->pp_rows_dev, token, arrive);
    if (rc) {
        cudaStreamSynchronize(up);
        cudaStreamSynchronize(st);
        return rc;
    }
    cudaStream_t copy = ctx->copy_stream;
    cudaEvent_t done_ev = ctx->pp_ev[PP_EV_TQ];
    H264A_CUDA(cudaEventRecord(done_ev, st));
    auto down = [&](int f0, int f1) -> int {  // frames [f0, f1)
        const size_t k = size_t(f1 - f0), m0 = size_t(f0) * nmb;
        auto cp = [&](void* h, const void* d, size_t unit) {
            return cudaMemcpyAsync(static_cast<char*>(h) + unit * m0, static_cast<const char*>(d) + unit * m0,
                                   unit * k * nmb, cudaMemcpyDeviceToHost, copy);
        };
        auto cpf = [&](void* h, const void* d, size_t bytes) {  // per-frame planes
            return cudaMemcpyAsync(static_cast<char*>(h) + bytes * f0, static_cast<const char*>(d) + bytes * f0,
                                   bytes * k, cudaMemcpyDeviceToHost, copy);
        };
        cudaError_t e = cp(job->h_picks, j.d_picks, sizeof(int32_t) * 6);
        if (e == cudaSuccess) e = cp(job->h_costs, j.d_costs, sizeof(int64_t) * 2);
        if (e == cudaSuccess && job->h_coeffs) e = cp(job->h_coeffs, j.d_coeffs, sizeof(int16_t) * 256);
        if (e == cudaSuccess && job->h_ccoeffs) e = cp(job->h_ccoeffs, j.d_ccoeffs, sizeof(int16_t) * 128);
        if (e == cudaSuccess && job->h_rec_y) e = cpf(job->h_rec_y, j.d_rec_y, fs);
        if (e == cudaSuccess && job->h_rec_u) e = cpf(job->h_rec_u, j.d_rec_u, cs_bytes);
        if (e == cudaSuccess && job->h_rec_v) e = cpf(job->h_rec_v, j.d_rec_v, cs_bytes);
        return e == cudaSuccess ? H264A_OK : cuda_fail(e, "pixel_path_closed: result downloads");
    };
    auto drain = [&](int code) {
        cudaStreamSynchronize(copy);
        cudaStreamSynchronize(st);
        cudaStreamSynchronize(up);
        return code;
    };
    // frame 0 (final before the kernel starts) goes with frame 1
    const volatile int32_t* words = ctx->pp_rows_host;
    int sent = 0;
    while (sent < n) {
        const cudaError_t q = cudaEventQuery(done_ev);  // before the words: done means every frame is final
        if (q != cudaSuccess && q != cudaErrorNotReady) {
            cudaGetLastError();
            return drain(cuda_fail(q, "pixel_path_closed: the loop"));
        }
        int ready = sent;
        if (q == cudaSuccess) {
            ready = n;
        } else {
            while (ready < n && (ready == 0 || words[ready] == token)) ready++;
            if (ready == 1 && n > 1) ready = 0;  // frame 0 waits for frame 1
        }
        if (ready > sent) {
            rc = down(sent, ready);
            if (rc) return drain(rc);
            sent = ready;
        } else {
            std::this_thread::sleep_for(std::chrono::microseconds(50));
        }
    }
    if (job->net && job->h_props)
        H264A_CUDA(cudaMemcpyAsync(job->h_props, j.d_props, sizeof(int32_t) * 16 * nmb * n, cudaMemcpyDeviceToHost, copy));
    if (job->net && job->h_fallback)
        H264A_CUDA(cudaMemcpyAsync(job->h_fallback, j.d_fallback, sizeof(int32_t) * nmb * n, cudaMemcpyDeviceToHost,
                                   copy));
    const cudaError_t e_cs = cudaStreamSynchronize(copy);
    if (e_cs != cudaSuccess) return drain(cuda_fail(e_cs, "pixel_path_closed: result downloads"));
    const cudaError_t e_up = cudaStreamSynchronize(up);
    if (e_up != cudaSuccess) return drain(cuda_fail(e_up, "pixel_path_closed: source uploads"));
    return h264a_sync(ctx, st);
}
