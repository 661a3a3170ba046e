// batch.cu -- batched plain-ME over many streams of uneven resolution: one
// persistent launch per GOP step, replayed from captured CUDA graphs, in the
// launch shape a small autotuner found fastest for the batch.
//
// The reference parallelises a clip by GOPs on CPU threads, a fresh encoder
// per GOP (crates/rusty_h264-encoder/src/lib.rs:745-805).  On the GPU the
// streams advance together instead: step k of a batch is, for every stream,
// the planes of frames kG..kG+count-1 (h264a_hpel_build, one launch per
// stream) and then one launch of the multi-reference frame kernel (me.cu,
// me_frames_mr_kernel) over frames kG+1..kG+count of all streams, largest
// frames first in one work queue, so the small streams' MBs fill the SMs the
// large frames' wavefronts leave idle; for the streams that ask for it, the
// MC + luma T/Q of those frames follows in the same graph (one launch of
// tq.cu's MC kernel, each half predicted from its own reference).
//
// Every stream keeps its frames in a ring of nslots slots (frame f in slot
// f % nslots), so the frame table of a step depends only on the slot of
// frame kG, on how many of the step's frames still lack references (the
// first nref frames of a stream) and on count: each such layout is captured
// once (planes, queue reset, kernel) and replayed with one cudaGraphLaunch.
// The batch owns its queue (ticket counter and per-MB flags), cleared inside
// the graph, so a replay needs no host work.
//
// The autotuner times the H264A_BATCH_VARIANTS launch shapes of the kernel
// (MBs per CTA, window staged by TMA or read from L2) on the first step's
// real frames, keeps the fastest (median of 3 after a warm-up, CUDA events)
// and caches it in the context under the batch's signature.  Every shape
// computes the same picks and costs; only their speed differs.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "h264accel_internal.h"

using namespace h264a;

namespace {

constexpr int BQ_COUNTER_INTS = 32;  // the counter, then the flags 128 bytes on

struct StepGraph {
    MrTable table;
    void* d_table = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

}  // namespace

struct h264a_batch {
    h264a_ctx* ctx = nullptr;
    std::vector<h264a_batch_stream> s;
    h264a_batch_config cfg{};
    h264a_me_params params{};
    cudaStream_t cap = nullptr;  // the stream graphs are captured on
    int32_t* d_q = nullptr;      // counter, flags
    size_t flag_cap = 0;
    std::map<std::tuple<int, int, int>, StepGraph> graphs;
    std::string sig;
    int variant = 0, tuned = 0;
    float ms[H264A_BATCH_VARIANTS] = {};
    int64_t steps = 0;
};

namespace {

size_t plane_bytes(const h264a_batch_stream& s) {
    return size_t(4) * size_t(s.cw + 2 * s.pad) * size_t(s.ch + 2 * s.pad);
}

int nmb_of(const h264a_batch_stream& s) { return (s.cw / 16) * (s.ch / 16); }

// The frame table of step k (frames kG+1..kG+count of every stream).
int step_table(const h264a_batch* b, int64_t k, int count, MrTable& t) {
    const int G = b->cfg.gop_step, ns = b->cfg.nslots;
    std::vector<h264a_me_mr_frame> fr;
    fr.reserve(b->s.size() * size_t(count));
    for (const h264a_batch_stream& s : b->s) {
        const size_t fs = size_t(s.cw) * s.ch, pb = plane_bytes(s), nmb = size_t(nmb_of(s));
        for (int i = 1; i <= count; i++) {
            const int64_t f = k * G + i;
            h264a_me_mr_frame m;
            memset(&m, 0, sizeof m);
            const size_t slot = size_t(f % ns);
            m.d_src = s.d_src + slot * fs;
            m.nref = int(std::min<int64_t>(b->cfg.nref, f));
            for (int r = 0; r < m.nref; r++) m.d_planes[r] = s.d_planes + size_t((f - 1 - r) % ns) * pb;
            m.cw = s.cw;
            m.ch = s.ch;
            m.pad = s.pad;
            m.lambda_me = s.lambda_me;
            m.split_gate = s.split_gate;
            m.d_picks = s.d_picks + slot * 8 * nmb;
            m.d_costs = s.d_costs + slot * 2 * nmb;
            fr.push_back(m);
        }
    }
    return mr_table_build(fr.data(), int(fr.size()), t);
}

// The planes of frames kG..kG+count-1 of every stream (contiguous slots: the
// ring's size is a multiple of G).
int step_planes(h264a_batch* b, int64_t k, int count, cudaStream_t st) {
    const int G = b->cfg.gop_step, ns = b->cfg.nslots;
    const size_t slot = size_t((k * G) % ns);
    for (const h264a_batch_stream& s : b->s) {
        const size_t fs = size_t(s.cw) * s.ch, pb = plane_bytes(s);
        const int rc = h264a_hpel_build(b->ctx, s.d_src + slot * fs, s.cw, s.ch, s.pad, count, fs,
                                        s.d_planes + slot * pb, st);
        if (rc) return rc;
    }
    return H264A_OK;
}

// Queue reset and one kernel launch over table t (at d_table).
int step_search(h264a_batch* b, int variant, const MrTable& t, const void* d_table, cudaStream_t st) {
    H264A_CUDA(cudaMemsetAsync(b->d_q, 0, sizeof(int32_t) * (BQ_COUNTER_INTS + size_t(t.total)), st));
    const MeParamsDev prm = to_dev(b->params);
    return mr_launch(b->ctx, variant, prm, d_table, t, b->d_q, b->d_q + BQ_COUNTER_INTS, 1, st);
}

// The MC + luma T/Q of frames kG+1..kG+count of the streams with
// coefficient rings, from the picks the search just wrote.
int step_tq(h264a_batch* b, int64_t k, int count, cudaStream_t st) {
    const int G = b->cfg.gop_step, ns = b->cfg.nslots;
    std::vector<h264a_mc_tq_mr_frame> fr;
    for (const h264a_batch_stream& s : b->s) {
        if (!s.d_coeffs) continue;
        const size_t fs = size_t(s.cw) * s.ch, pb = plane_bytes(s), nmb = size_t(nmb_of(s));
        for (int i = 1; i <= count; i++) {
            const int64_t f = k * G + i;
            h264a_mc_tq_mr_frame m;
            memset(&m, 0, sizeof m);
            const size_t slot = size_t(f % ns);
            m.d_src = s.d_src + slot * fs;
            m.nref = int(std::min<int64_t>(b->cfg.nref, f));
            for (int r = 0; r < m.nref; r++) m.d_planes[r] = s.d_planes + size_t((f - 1 - r) % ns) * pb;
            m.cw = s.cw; m.ch = s.ch; m.pad = s.pad;
            m.d_picks = s.d_picks + slot * 8 * nmb;
            m.qp = s.qp;
            m.dz_div = s.dz_div;
            m.d_coeffs = s.d_coeffs + slot * 256 * nmb;
            fr.push_back(m);
        }
    }
    if (fr.empty()) return H264A_OK;
    return mc_tq_mr_run(b->ctx, fr.data(), int(fr.size()), st);
}

int upload_table(StepGraph& g) {
    if (cudaMalloc(&g.d_table, g.table.bytes.size()) != cudaSuccess) {
        cudaGetLastError();
        return fail(H264A_E_NOMEM, "batch: cudaMalloc of a step table failed");
    }
    H264A_CUDA(cudaMemcpy(g.d_table, g.table.bytes.data(), g.table.bytes.size(), cudaMemcpyHostToDevice));
    return H264A_OK;
}

// The autotuner: the step's planes, then every launch shape timed on the
// step's frames (one warm-up, the median of three).
int tune(h264a_batch* b, int64_t k, int count, const StepGraph& g, cudaStream_t st) {
    int rc = step_planes(b, k, count, st);
    if (rc) return rc;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    H264A_CUDA(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return cuda_fail(cudaGetLastError(), "batch: cudaEventCreate");
    }
    int best = 0;
    for (int v = 0; v < H264A_BATCH_VARIANTS && !rc; v++) {
        float t[3] = {};
        for (int it = 0; it < 4 && !rc; it++) {
            if (cudaEventRecord(e0, st) != cudaSuccess) {
                rc = cuda_fail(cudaGetLastError(), "batch: event");
                break;
            }
            rc = step_search(b, v, g.table, g.d_table, st);
            if (rc) break;
            if (cudaEventRecord(e1, st) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
                rc = cuda_fail(cudaGetLastError(), "batch: tuning run");
                break;
            }
            if (it > 0) cudaEventElapsedTime(&t[it - 1], e0, e1);
        }
        if (rc) break;
        std::sort(t, t + 3);
        b->ms[v] = t[1];
        if (b->ms[v] < b->ms[best]) best = v;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    // a bounded wait that ran out during tuning leaves its code in the status
    // word: report it rather than keep a shape measured on an aborted run
    int32_t status = 0;
    H264A_CUDA(cudaMemcpy(&status, b->ctx->d_status, sizeof status, cudaMemcpyDeviceToHost));
    if (status) return fail(H264A_E_TIMEOUT, "batch: a bounded wait ran out while tuning");
    b->variant = best;
    b->tuned = 1;
    b->ctx->tune_cache[b->sig] = best;
    return H264A_OK;
}

int capture(h264a_batch* b, int64_t k, int count, StepGraph& g) {
    H264A_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeRelaxed));
    int rc = step_planes(b, k, count, b->cap);
    if (!rc) rc = step_search(b, b->variant, g.table, g.d_table, b->cap);
    if (!rc) rc = step_tq(b, k, count, b->cap);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "batch: graph capture");
    g.graph = graph;
    H264A_CUDA(cudaGraphInstantiate(&g.exec, graph, 0));
    return H264A_OK;
}

void free_graph(StepGraph& g) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
    if (g.d_table) cudaFree(g.d_table);
    g = StepGraph();
}

}  // namespace

extern "C" int h264a_batch_create(h264a_ctx* ctx, const h264a_batch_stream* streams, int nstreams,
                                  const h264a_batch_config* cfg, const h264a_me_params* params, h264a_batch** out) {
    if (!ctx || !streams || !cfg || !params || !out) return fail(H264A_E_ARG, "batch_create: null pointer");
    *out = nullptr;
    if (nstreams < 1) return fail(H264A_E_ARG, "batch_create: need at least one stream");
    const int G = cfg->gop_step, ns = cfg->nslots, nref = cfg->nref;
    if (G < 1 || nref < 1 || nref > 4) return fail(H264A_E_ARG, "batch_create: need gop_step >= 1 and 1 <= nref <= 4");
    if (ns % G != 0 || ns < G + nref + 1)
        return fail(H264A_E_ARG, "batch_create: nslots must be a multiple of gop_step and at least gop_step + nref + 1");
    if (!cfg->autotune && (cfg->variant < 0 || cfg->variant >= H264A_BATCH_VARIANTS))
        return fail(H264A_E_ARG, "batch_create: no such variant");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !params->d_mv_cost_tab)
        return fail(H264A_E_ARG, "batch_create: mv cost kinds 1 and 2 need d_mv_cost_tab");
    long long total = 0;
    std::vector<std::string> sizes;
    for (int i = 0; i < nstreams; i++) {
        const h264a_batch_stream& s = streams[i];
        if (!s.d_src || !s.d_planes || !s.d_picks || !s.d_costs) return fail(H264A_E_ARG, "batch_create: null stream buffer");
        if (s.cw < 16 || s.ch < 16 || s.cw % 16 || s.ch % 16 || s.pad < 3 || s.pad > 128)
            return fail(H264A_E_ARG, "batch_create: streams must be MB-aligned with 3 <= pad <= 128");
        if (reinterpret_cast<uintptr_t>(s.d_src) & 3)
            return fail(H264A_E_ARG, "batch_create: source rings must be 4-byte aligned");
        if (s.d_coeffs && ((reinterpret_cast<uintptr_t>(s.d_coeffs) & 15) || s.qp < 0 || s.qp > 51 || s.dz_div < 1 ||
                           s.dz_div != streams[0].dz_div))
            return fail(H264A_E_ARG, "batch_create: coefficient rings 16-byte aligned, qp 0..51, one dz_div >= 1");
        total += (long long)nmb_of(s) * G;
        char buf[48];
        snprintf(buf, sizeof buf, "%dx%d", s.cw, s.ch);
        sizes.push_back(buf);
    }
    if (total >= (1LL << 31)) return fail(H264A_E_ARG, "batch_create: too many macroblocks per step");
    std::sort(sizes.begin(), sizes.end());
    h264a_batch* b = new h264a_batch();
    b->ctx = ctx;
    b->s.assign(streams, streams + nstreams);
    b->cfg = *cfg;
    b->params = *params;
    const MeParamsDev prm = to_dev(*params);
    char head[96];
    snprintf(head, sizeof head, "nref=%d;G=%d;fast=%d;kind=%d;sadfp=%d;", nref, G, prm.fast, prm.kind, prm.sadfp);
    b->sig = head;
    for (const std::string& z : sizes) b->sig += z + ",";
    if (!cfg->autotune) {
        b->variant = cfg->variant;
    } else {
        auto it = ctx->tune_cache.find(b->sig);
        if (it != ctx->tune_cache.end()) {
            b->variant = it->second;
            b->tuned = 1;
        }
    }
    b->flag_cap = size_t(total);
    int rc = H264A_OK;
    if (cudaMalloc(&b->d_q, sizeof(int32_t) * (BQ_COUNTER_INTS + b->flag_cap)) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(H264A_E_NOMEM, "batch_create: cudaMalloc of the queue failed");
    } else if (cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess) {
        rc = cuda_fail(cudaGetLastError(), "batch_create: capture stream");
    }
    if (rc) {
        h264a_batch_destroy(b);
        return rc;
    }
    *out = b;
    return H264A_OK;
}

extern "C" int h264a_batch_step(h264a_batch* b, int64_t k, int count, void* stream) {
    if (!b) return fail(H264A_E_ARG, "batch_step: null batch");
    if (k < 0 || count < 1 || count > b->cfg.gop_step)
        return fail(H264A_E_ARG, "batch_step: need k >= 0 and 1 <= count <= gop_step");
    if (k > (int64_t(1) << 40)) return fail(H264A_E_ARG, "batch_step: step index out of range");
    cudaStream_t st = pick_stream(b->ctx, stream);
    const int64_t kG = k * b->cfg.gop_step;
    const auto key = std::make_tuple(int(kG % b->cfg.nslots), int(std::min<int64_t>(kG, b->cfg.nref)), count);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
        StepGraph g;
        int rc = step_table(b, k, count, g.table);
        if (!rc) rc = upload_table(g);
        if (!rc && b->cfg.autotune && !b->tuned) rc = tune(b, k, count, g, st);
        if (!rc) rc = capture(b, k, count, g);
        if (rc) {
            free_graph(g);
            return rc;
        }
        it = b->graphs.emplace(key, g).first;
    }
    H264A_CUDA(cudaGraphLaunch(it->second.exec, st));
    b->steps++;
    return H264A_OK;
}

extern "C" int h264a_batch_get_info(const h264a_batch* b, h264a_batch_info* out) {
    if (!b || !out) return fail(H264A_E_ARG, "batch_get_info: null pointer");
    memset(out, 0, sizeof *out);
    out->variant = b->variant;
    out->tuned = b->tuned;
    for (int v = 0; v < H264A_BATCH_VARIANTS; v++) out->ms[v] = b->ms[v];
    out->graphs = int32_t(b->graphs.size());
    out->steps = b->steps;
    return H264A_OK;
}

extern "C" int h264a_batch_destroy(h264a_batch* b) {
    if (!b) return H264A_OK;
    cudaSetDevice(b->ctx->device);
    cudaDeviceSynchronize();  // no step of this batch still reads its tables
    for (auto& kv : b->graphs) free_graph(kv.second);
    if (b->d_q) cudaFree(b->d_q);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete b;
    return H264A_OK;
}
