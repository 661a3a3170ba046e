// capi.cu -- context, error reporting, parameter mirrors and the host-buffer
// pipeline entry of libh264accel_cuda.so.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <chrono>
#include <thread>
#include <vector>

#include "h264accel_internal.h"

namespace h264a {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

int fail(int code, const std::string& msg) {
    set_error(msg);
    return code;
}

int cuda_fail(cudaError_t e, const char* what) {
    return fail(H264A_E_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int check_launch(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, what);
    return H264A_OK;
}

MeParamsDev to_dev(const h264a_me_params& p) {
    MeParamsDev d;
    d.fast = p.fast;
    d.use_sad = p.fast && !p.mb_use_satd;
    d.sadfp = p.sadfp;
    d.kind = p.mv_cost_kind;
    d.tab = p.d_mv_cost_tab;
    d.sadfp_lambda = p.sadfp_lambda;
    d.me_snap = p.me_snap;
    d.fc = p.me_fc;
    d.dia_mask = p.dia_mask;
    d.dia_sub_mask = p.dia_sub_mask;
    d.subpel = p.subpel;
    d.subpel_pat = p.subpel_pat;
    d.sp_single_pass = p.sp_single_pass;
    d.sub_pat = p.sub_pat;
    d.me_subpel_iter = p.me_subpel_iter;
    d.sp_maxit = p.sp_maxit;
    d.sp_fc = p.sp_fc;
    return d;
}

int ensure_me_scratch(h264a_ctx* ctx, size_t n, int queue) {
    WorkQueue& q = ctx->q[queue];
    if (n <= q.flags_cap) return H264A_OK;
    if (q.d_flags) cudaFree(q.d_flags);
    q.d_flags = nullptr;
    q.flags_cap = 0;
    size_t cap = n < 4096 ? 4096 : n + n / 4;
    cap = (cap + 63) & ~size_t(63);
    const size_t bytes = cap * sizeof(int32_t);  // one done flag per MB
    if (cudaMalloc(&q.d_flags, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(H264A_E_NOMEM, "persistent-kernel scratch: cudaMalloc failed");
    }
    H264A_CUDA(cudaMemset(q.d_flags, 0, bytes));
    q.flags_cap = cap;
    q.epoch = 0;
    return H264A_OK;
}

int next_epoch(h264a_ctx* ctx, cudaStream_t st, int queue) {
    WorkQueue& q = ctx->q[queue];
    if (q.epoch >= 0x7ffffff0) {  // wrap: clear the flags so stale values never match
        if (cudaMemsetAsync(q.d_flags, 0, q.flags_cap * sizeof(int32_t), st) != cudaSuccess) {
            cudaGetLastError();
            set_error("persistent-kernel flags: reset failed");
            return -1;
        }
        q.epoch = 0;
    }
    return ++q.epoch;
}

}  // namespace h264a

using namespace h264a;

extern "C" const char* h264a_version(void) { return "h264accel_cuda 0.1.0 (sm_100a)"; }

extern "C" const char* h264a_last_error(void) { return g_last_error.c_str(); }

extern "C" int h264a_ctx_create(int device, h264a_ctx** out) {
    if (!out) return fail(H264A_E_ARG, "ctx_create: null out");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        return fail(H264A_E_NODEV, "ctx_create: no CUDA device");
    }
    if (device < 0 || device >= count) return fail(H264A_E_ARG, "ctx_create: device index out of range");
    cudaDeviceProp prop;
    H264A_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(H264A_E_NODEV, std::string("ctx_create: built for sm_100a, device is ") + prop.name);
    H264A_CUDA(cudaSetDevice(device));
    h264a_ctx* c = new h264a_ctx();
    c->device = device;
    c->num_sms = prop.multiProcessorCount;
    bool ev_ok = true;
    for (int i = 0; i < PP_EVENTS; i++)
        ev_ok = ev_ok && cudaEventCreateWithFlags(&c->pp_ev[i], cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < PP_SLOTS; i++)
        ev_ok = ev_ok && cudaEventCreateWithFlags(&c->pp_in[i].ev, cudaEventDisableTiming) == cudaSuccess;
    if (!ev_ok || cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->pf_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->la_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_counters, NUM_QUEUES * Q_COUNTER_STRIDE * sizeof(int32_t)) != cudaSuccess ||
        cudaMalloc(&c->d_status, sizeof(int32_t)) != cudaSuccess ||
        cudaMemset(c->d_status, 0, sizeof(int32_t)) != cudaSuccess) {
        const cudaError_t e = cudaGetLastError();
        h264a_ctx_destroy(c);
        return cuda_fail(e, "ctx_create");
    }
    for (int i = 0; i < NUM_QUEUES; i++) c->q[i].d_counter = c->d_counters + i * Q_COUNTER_STRIDE;
    *out = c;
    return H264A_OK;
}

extern "C" int h264a_ctx_destroy(h264a_ctx* ctx) {
    if (!ctx) return H264A_OK;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->la_stream) cudaStreamSynchronize(ctx->la_stream);
    if (ctx->pf_stream) cudaStreamSynchronize(ctx->pf_stream);
    if (ctx->d_counters) cudaFree(ctx->d_counters);
    if (ctx->d_status) cudaFree(ctx->d_status);
    for (int i = 0; i < NUM_QUEUES; i++)
        if (ctx->q[i].d_flags) cudaFree(ctx->q[i].d_flags);
    if (ctx->pp_buf) cudaFree(ctx->pp_buf);
    if (ctx->cl_buf) cudaFree(ctx->cl_buf);
    if (ctx->me_tab) cudaFree(ctx->me_tab);
    if (ctx->me_tab_host) cudaFreeHost(ctx->me_tab_host);
    if (ctx->me_tab_ev) cudaEventDestroy(ctx->me_tab_ev);
    if (ctx->pp_row_count) cudaFree(ctx->pp_row_count);
    if (ctx->pp_rows_host) cudaFreeHost(ctx->pp_rows_host);
    if (ctx->upl_tok) cudaFreeHost(ctx->upl_tok);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->la_stream) cudaStreamDestroy(ctx->la_stream);
    if (ctx->pf_stream) cudaStreamDestroy(ctx->pf_stream);
    for (int i = 0; i < PP_EVENTS; i++)
        if (ctx->pp_ev[i]) cudaEventDestroy(ctx->pp_ev[i]);
    for (int i = 0; i < PP_SLOTS; i++) {
        if (ctx->pp_in[i].d) cudaFree(ctx->pp_in[i].d);
        if (ctx->pp_in[i].ev) cudaEventDestroy(ctx->pp_in[i].ev);
    }
    delete ctx;
    return H264A_OK;
}

// Synchronises `stream` and reports a bounded-wait timeout recorded by a
// persistent kernel since the last sync (the status word is then cleared).
extern "C" int h264a_sync(h264a_ctx* ctx, void* stream) {
    if (!ctx) return fail(H264A_E_ARG, "sync: null ctx");
    cudaStream_t st = pick_stream(ctx, stream);
    H264A_CUDA(cudaStreamSynchronize(st));
    int32_t status = 0;
    H264A_CUDA(cudaMemcpy(&status, ctx->d_status, sizeof status, cudaMemcpyDeviceToHost));
    if (status != 0) {
        H264A_CUDA(cudaMemset(ctx->d_status, 0, sizeof(int32_t)));
        // the code a persistent kernel recorded when its wait gave up
        const char* what = status == 1   ? "for a neighbouring macroblock's flag"
                           : status == 2 ? "of the self-test, on a flag nothing sets"
                           : status == 3 ? "for a window copy into shared memory"
                                         : "";
        return fail(H264A_E_TIMEOUT, std::string("a bounded wait ") + what + " ran out (status " +
                                         std::to_string(status) + ")");
    }
    return H264A_OK;
}

extern "C" int h264a_dev_alloc(h264a_ctx* ctx, size_t bytes, void** d_out) {
    if (!ctx || !d_out) return fail(H264A_E_ARG, "dev_alloc: null pointer");
    if (cudaMalloc(d_out, bytes) != cudaSuccess) {
        cudaGetLastError();
        *d_out = nullptr;
        return fail(H264A_E_NOMEM, "dev_alloc: cudaMalloc failed");
    }
    return H264A_OK;
}

extern "C" int h264a_dev_free(h264a_ctx* ctx, void* d_ptr) {
    if (!ctx) return fail(H264A_E_ARG, "dev_free: null ctx");
    H264A_CUDA(cudaFree(d_ptr));
    return H264A_OK;
}

extern "C" int h264a_memcpy_h2d(h264a_ctx* ctx, void* d_dst, const void* h_src, size_t bytes, void* stream) {
    if (!ctx || (!d_dst && bytes) || (!h_src && bytes)) return fail(H264A_E_ARG, "memcpy_h2d: null pointer");
    H264A_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, pick_stream(ctx, stream)));
    return H264A_OK;
}

extern "C" int h264a_memcpy_d2h(h264a_ctx* ctx, void* h_dst, const void* d_src, size_t bytes, void* stream) {
    if (!ctx || (!d_src && bytes) || (!h_dst && bytes)) return fail(H264A_E_ARG, "memcpy_d2h: null pointer");
    H264A_CUDA(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, pick_stream(ctx, stream)));
    return H264A_OK;
}

extern "C" void h264a_me_params_default(h264a_me_params* p) {
    if (!p) return;
    memset(p, 0, sizeof *p);
    // Balanced preset (config.rs:8-38, mb16.rs:1620-1745 defaults)
    p->fast = 0;
    p->mb_use_satd = 0;
    p->sadfp = 0;
    p->mv_cost_kind = 0;
    p->d_mv_cost_tab = nullptr;
    p->sadfp_lambda = 0.5;
    p->me_snap = 1;
    p->me_fc = 1;
    p->dia_mask = 0x1c;      // [16,8,4] quarter-pel
    p->dia_sub_mask = 0x10;  // [4]
    p->subpel = 1;
    p->subpel_pat = -1;
    p->sp_single_pass = 1;
    p->sub_pat = 2;
    p->me_subpel_iter = 1;
    p->sp_maxit = 0;
    p->sp_fc = 0;
}

// build_mv_cost (mb16.rs:508-519): round(4·(2·log2(a+1) + 0.718 + [a≠0])).
extern "C" void h264a_build_mv_cost_table(uint16_t* h_out) {
    if (!h_out) return;
    for (uint32_t a = 0; a < 4096; a++) {
        const double c = 2.0 * std::log2(double(a + 1)) + 0.718 + (a != 0 ? 1.0 : 0.0);
        h_out[a] = uint16_t(std::round(c * 4.0));
    }
}

// ---------------------------------------------------------------------------
// The whole pixel path from host buffers
// ---------------------------------------------------------------------------

static size_t align256(size_t v) { return (v + 255) & ~size_t(255); }

// Grows the row-completion buffers of h264a_pixel_path_host to `rows` rows.
int h264a::ensure_pp_rows(h264a_ctx* ctx, size_t rows) {
    if (rows <= ctx->pp_rows_cap) return H264A_OK;
    if (ctx->pp_row_count) cudaFree(ctx->pp_row_count);
    if (ctx->pp_rows_host) cudaFreeHost(ctx->pp_rows_host);
    ctx->pp_row_count = ctx->pp_rows_host = ctx->pp_rows_dev = nullptr;
    ctx->pp_rows_cap = 0;
    const size_t bytes = rows * sizeof(int32_t);
    if (cudaMalloc(&ctx->pp_row_count, bytes) != cudaSuccess ||
        cudaHostAlloc(reinterpret_cast<void**>(&ctx->pp_rows_host), bytes, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->pp_rows_dev), ctx->pp_rows_host, 0) != cudaSuccess) {
        cudaGetLastError();
        return fail(H264A_E_NOMEM, "pixel_path_host: row-completion buffers");
    }
    memset(ctx->pp_rows_host, 0, bytes);
    ctx->pp_token = 0;
    ctx->pp_rows_cap = rows;
    return H264A_OK;
}

int32_t h264a::next_pp_token(h264a_ctx* ctx) {
    if (ctx->pp_token >= 0x7ffffff0) {  // stale words must never equal a new token
        memset(ctx->pp_rows_host, 0, ctx->pp_rows_cap * sizeof(int32_t));
        ctx->pp_token = 0;
    }
    return ++ctx->pp_token;
}

// Grows input slot `s` to `bytes`.  Only called for a slot that holds no
// pending upload and that no call is using, so nothing on the device reads it.
static int ensure_slot(PpInput& s, size_t bytes) {
    if (bytes <= s.cap) return H264A_OK;
    if (s.d) cudaFree(s.d);
    s.d = nullptr;
    s.cap = 0;
    if (cudaMalloc(&s.d, bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(H264A_E_NOMEM, "pixel_path: input slot allocation failed");
    }
    s.cap = bytes;
    return H264A_OK;
}

extern "C" int h264a_pixel_path_prefetch(h264a_ctx* ctx, const uint8_t* h_frames, int n, int cw, int ch) {
    if (!ctx || !h_frames) return fail(H264A_E_ARG, "pixel_path_prefetch: null pointer");
    if (n < 1 || cw < 16 || ch < 16 || cw % 16 || ch % 16) return fail(H264A_E_ARG, "pixel_path_prefetch: bad geometry");
    int k = -1;
    for (int i = 0; i < PP_SLOTS && k < 0; i++)
        if (!ctx->pp_in[i].pending) k = i;
    if (k < 0) return fail(H264A_E_ARG, "pixel_path_prefetch: two uploads are already pending");
    PpInput& in = ctx->pp_in[k];
    const size_t bytes = size_t(cw) * ch * n;
    const int rc = ensure_slot(in, bytes);
    if (rc) return rc;
    H264A_CUDA(cudaMemcpyAsync(in.d, h_frames, bytes, cudaMemcpyHostToDevice, ctx->pf_stream));
    H264A_CUDA(cudaEventRecord(in.ev, ctx->pf_stream));
    in.h = h_frames;
    in.n = n;
    in.cw = cw;
    in.ch = ch;
    in.pending = 1;
    in.seq = ++ctx->pp_seq;
    return H264A_OK;
}

extern "C" int h264a_pixel_path_host(h264a_ctx* ctx, const uint8_t* h_frames, int n, int cw, int ch,
                                     const h264a_me_params* params, const uint16_t* h_mv_cost_tab, double lambda_me,
                                     int64_t split_gate, int qp, int dz_div, int32_t* h_picks, int64_t* h_costs,
                                     int16_t* h_coeffs, int32_t* h_la_intra, int32_t* h_la_inter, int32_t* h_la_mvs) {
    if (!ctx || !h_frames || !params || !h_picks || !h_costs || !h_coeffs || !h_la_intra || !h_la_inter || !h_la_mvs)
        return fail(H264A_E_ARG, "pixel_path_host: null pointer");
    if (n < 1 || cw < 16 || ch < 16 || cw % 16 || ch % 16) return fail(H264A_E_ARG, "pixel_path_host: bad geometry");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !h_mv_cost_tab)
        return fail(H264A_E_ARG, "pixel_path_host: mv cost kinds 1 and 2 need a table");
    const int pad = 32;
    const int pw = cw + 2 * pad, ph = ch + 2 * pad;
    const size_t nmb = size_t(cw / 16) * (ch / 16);
    const size_t fs = size_t(cw) * ch, hs = fs / 4, p4 = size_t(4) * pw * ph;
    // one cached device arena
    size_t off = 0;
    const size_t o_planes = off; off = align256(off + p4 * (n > 1 ? n - 1 : 1));
    const size_t o_half = off; off = align256(off + hs * n);
    const size_t o_picks = off; off = align256(off + sizeof(int32_t) * 6 * nmb * n);
    const size_t o_costs = off; off = align256(off + sizeof(int64_t) * 2 * nmb * n);
    const size_t o_coeffs = off; off = align256(off + sizeof(int16_t) * 256 * nmb * n);
    const size_t o_intra = off; off = align256(off + sizeof(int32_t) * nmb * n);
    const size_t o_inter = off; off = align256(off + sizeof(int32_t) * nmb * n);
    const size_t o_mvs = off; off = align256(off + sizeof(int32_t) * 2 * nmb * n);
    const size_t o_tab = off; off = align256(off + sizeof(uint16_t) * 4096);
    if (off > ctx->pp_bytes) {
        if (ctx->pp_buf) cudaFree(ctx->pp_buf);
        ctx->pp_buf = nullptr;
        ctx->pp_bytes = 0;
        if (cudaMalloc(&ctx->pp_buf, off) != cudaSuccess) {
            cudaGetLastError();
            return fail(H264A_E_NOMEM, "pixel_path_host: device arena allocation failed");
        }
        ctx->pp_bytes = off;
    }
    char* base = reinterpret_cast<char*>(ctx->pp_buf);
    // the input slot: the oldest pending prefetch of these frames, else a
    // free slot the call uploads into (if both hold other prefetches, the
    // newest is given up: a later call of its frames uploads them again)
    int use = -1;
    for (int i = 0; i < PP_SLOTS; i++) {
        const PpInput& c = ctx->pp_in[i];
        if (c.pending && c.h == h_frames && c.n == n && c.cw == cw && c.ch == ch &&
            (use < 0 || c.seq < ctx->pp_in[use].seq))
            use = i;
    }
    const bool prefetched = use >= 0;
    if (!prefetched) {
        for (int i = 0; i < PP_SLOTS && use < 0; i++)
            if (!ctx->pp_in[i].pending) use = i;
        if (use < 0) {
            use = ctx->pp_in[0].seq > ctx->pp_in[1].seq ? 0 : 1;
            H264A_CUDA(cudaEventSynchronize(ctx->pp_in[use].ev));
        }
        ctx->pp_in[use].pending = 0;
        const int rs = ensure_slot(ctx->pp_in[use], fs * n);
        if (rs) return rs;
        ctx->pp_in[use].h = h_frames;
        ctx->pp_in[use].n = n;
        ctx->pp_in[use].cw = cw;
        ctx->pp_in[use].ch = ch;
    }
    PpInput& in = ctx->pp_in[use];
    in.pending = 0;
    uint8_t* d_frames = in.d;
    uint8_t* d_planes = reinterpret_cast<uint8_t*>(base + o_planes);
    uint8_t* d_half = reinterpret_cast<uint8_t*>(base + o_half);
    int32_t* d_picks = reinterpret_cast<int32_t*>(base + o_picks);
    int64_t* d_costs = reinterpret_cast<int64_t*>(base + o_costs);
    int16_t* d_coeffs = reinterpret_cast<int16_t*>(base + o_coeffs);
    int32_t* d_intra = reinterpret_cast<int32_t*>(base + o_intra);
    int32_t* d_inter = reinterpret_cast<int32_t*>(base + o_inter);
    int32_t* d_mvs = reinterpret_cast<int32_t*>(base + o_mvs);
    uint16_t* d_tab = reinterpret_cast<uint16_t*>(base + o_tab);
    // Three streams.  The frames go up in PP_CHUNKS chunks on the copy
    // stream while the compute stream builds each chunk's planes and half-res
    // frames (frames prefetched by h264a_pixel_path_prefetch are one chunk,
    // ready when its upload event fires).  Then the lookahead (its own work queue) runs on the lookahead
    // stream beside plain-ME with the fused MC + T/Q on the compute stream.
    // An MB row of every frame is final once all its MBs have stored their
    // coefficients (the kernel sets a host-visible word per row), and the
    // rows happen to finish from about half-way through the launch; this
    // thread polls those words and queues each band of finished rows, of all
    // frames at once, for download, so that little is left to copy when the
    // launch ends.
    cudaStream_t st = ctx->stream, cs = ctx->copy_stream, ls = ctx->la_stream;
    const int mb_w = cw / 16, mb_h = ch / 16;
    const int nk = prefetched ? 1 : (n < PP_CHUNKS ? n : PP_CHUNKS);
    for (int k = 0; k < nk && !prefetched; k++) {
        const int a = int((long long)k * n / nk), b = int((long long)(k + 1) * n / nk);
        H264A_CUDA(cudaMemcpyAsync(d_frames + fs * a, h_frames + fs * a, fs * (b - a), cudaMemcpyHostToDevice, cs));
        H264A_CUDA(cudaEventRecord(ctx->pp_ev[k], cs));
    }
    h264a_me_params prm = *params;
    if (prm.mv_cost_kind == 1 || prm.mv_cost_kind == 2) {
        H264A_CUDA(cudaMemcpyAsync(d_tab, h_mv_cost_tab, sizeof(uint16_t) * 4096, cudaMemcpyHostToDevice, st));
        prm.d_mv_cost_tab = d_tab;
    }
    int rc = ensure_pp_rows(ctx, size_t(n > 1 ? n - 1 : 1) * mb_h);
    if (rc) return rc;
    const int32_t token = next_pp_token(ctx);
    H264A_CUDA(cudaMemsetAsync(ctx->pp_row_count, 0, ctx->pp_rows_cap * sizeof(int32_t), st));
    for (int k = 0; k < nk; k++) {
        const int a = int((long long)k * n / nk), b = int((long long)(k + 1) * n / nk);
        H264A_CUDA(cudaStreamWaitEvent(st, prefetched ? in.ev : ctx->pp_ev[k], 0));
        const int refs = (b < n - 1 ? b : n - 1) - a;  // reference pictures 0..n-2 in this chunk
        if (refs > 0) {
            rc = h264a_hpel_build(ctx, d_frames + fs * a, cw, ch, pad, refs, fs, d_planes + p4 * a, st);
            if (rc) return rc;
        }
        rc = h264a_downsample2x(ctx, d_frames + fs * a, cw, ch, b - a, fs, d_half + hs * a, st);
        if (rc) return rc;
    }
    H264A_CUDA(cudaEventRecord(ctx->pp_ev[PP_EV_INPUTS], st));
    H264A_CUDA(cudaStreamWaitEvent(ls, ctx->pp_ev[PP_EV_INPUTS], 0));
    rc = h264a_lookahead_costs(ctx, d_frames, d_half, cw, ch, n, 2, d_intra, d_inter, d_mvs, ls);
    if (rc) return rc;
    // From here on copies into the caller's buffers may be in flight on the
    // copy and lookahead streams: every return drains both first.
    auto drain = [&](int code) {
        cudaStreamSynchronize(cs);
        cudaStreamSynchronize(ls);
        cudaGetLastError();
        return code;
    };
    auto check = [&](cudaError_t e, const char* what) { return e == cudaSuccess ? H264A_OK : drain(cuda_fail(e, what)); };
    // the lookahead ends long before ME: its results come down under ME
    if ((rc = check(cudaMemcpyAsync(h_la_intra, d_intra, sizeof(int32_t) * nmb * n, cudaMemcpyDeviceToHost, ls),
                    "pixel_path_host: lookahead download")) ||
        (rc = check(cudaMemcpyAsync(h_la_inter, d_inter, sizeof(int32_t) * nmb * n, cudaMemcpyDeviceToHost, ls),
                    "pixel_path_host: lookahead download")) ||
        (rc = check(cudaMemcpyAsync(h_la_mvs, d_mvs, sizeof(int32_t) * 2 * nmb * n, cudaMemcpyDeviceToHost, ls),
                    "pixel_path_host: lookahead download")) ||
        (rc = check(cudaEventRecord(ctx->pp_ev[PP_EV_LA], ls), "pixel_path_host: lookahead event")))
        return rc;
    if (n > 1) {
        std::vector<h264a_me_frame> mf(n - 1);
        std::vector<MeTqOut> tq(n - 1);
        for (int f = 1; f < n; f++) {
            h264a_picture pic{d_frames + fs * f, d_planes + p4 * (f - 1), cw, ch, pad};
            mf[f - 1] = {pic, lambda_me, split_gate, d_picks + 6 * nmb * f, d_costs + 2 * nmb * f};
            tq[f - 1] = MeTqOut{d_coeffs + 256 * nmb * f, qp, dz_div, ctx->pp_row_count + size_t(f - 1) * mb_h,
                                ctx->pp_rows_dev + size_t(f - 1) * mb_h, token};
        }
        rc = me_frames_run(ctx, mf.data(), n - 1, &prm, tq.data(), st);
        if (rc) return drain(rc);
    }
    if ((rc = check(cudaEventRecord(ctx->pp_ev[PP_EV_TQ], st), "pixel_path_host: ME + T/Q event"))) return rc;
    // frame 0 (the IDR) has no pick or coefficients: the kernels never write its rows
    memset(h_picks, 0, sizeof(int32_t) * 6 * nmb);
    memset(h_costs, 0, sizeof(int64_t) * 2 * nmb);
    memset(h_coeffs, 0, sizeof(int16_t) * 256 * nmb);
    // rows [r0, r1) of every P frame: one strided copy per output
    auto copy_rows = [&](int r0, int r1) -> int {
        const size_t m0 = nmb + size_t(r0) * mb_w, mc = size_t(r1 - r0) * mb_w;
        const size_t hgt = size_t(n - 1);
        H264A_CUDA(cudaMemcpy2DAsync(h_coeffs + 256 * m0, 512 * nmb, d_coeffs + 256 * m0, 512 * nmb, 512 * mc, hgt,
                                     cudaMemcpyDeviceToHost, cs));
        H264A_CUDA(cudaMemcpy2DAsync(h_picks + 6 * m0, 24 * nmb, d_picks + 6 * m0, 24 * nmb, 24 * mc, hgt,
                                     cudaMemcpyDeviceToHost, cs));
        H264A_CUDA(cudaMemcpy2DAsync(h_costs + 2 * m0, 16 * nmb, d_costs + 2 * m0, 16 * nmb, 16 * mc, hgt,
                                     cudaMemcpyDeviceToHost, cs));
        return H264A_OK;
    };
    if (n > 1) {
        const volatile int32_t* rows = ctx->pp_rows_host;
        std::vector<int> prefix(n - 1, 0);  // finished rows of each P frame, counted from the top
        int sent = 0;                       // rows of every P frame queued for download
        for (;;) {
            const cudaError_t q = cudaEventQuery(ctx->pp_ev[PP_EV_TQ]);  // before the words: done means all final
            if (q != cudaSuccess && q != cudaErrorNotReady) {
                cudaGetLastError();
                return drain(cuda_fail(q, "pixel_path_host: ME + T/Q"));  // no copy outlives the call
            }
            int ready = mb_h;
            if (q != cudaSuccess) {
                for (int f = 0; f < n - 1; f++) {
                    int r = prefix[f];
                    while (r < mb_h && rows[size_t(f) * mb_h + r] == token) r++;
                    prefix[f] = r;
                    ready = r < ready ? r : ready;
                }
            }
            if (ready > sent) {
                rc = copy_rows(sent, ready);
                if (rc) return drain(rc);
                sent = ready;
            }
            if (sent == mb_h) break;
            std::this_thread::sleep_for(std::chrono::microseconds(100));
        }
    }
    const cudaError_t e_cs = cudaStreamSynchronize(cs), e_ls = cudaStreamSynchronize(ls);
    if (e_cs != cudaSuccess || e_ls != cudaSuccess)
        return drain(cuda_fail(e_cs != cudaSuccess ? e_cs : e_ls, "pixel_path_host: result downloads"));
    return h264a_sync(ctx, st);
}
