// h264accel_internal.h -- host-side plumbing shared by the .cu files of
// libh264accel_cuda.so (context, error reporting, launch helpers).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "../../include/h264accel.h"

// The work queue of a persistent wavefront kernel: its ticket counter, one
// done flag per MB (flags_cap MBs) and the value a finished MB writes into
// its flag.
struct WorkQueue {
    int32_t *d_counter = nullptr;  // a word of h264a_ctx::d_counters
    int32_t *d_flags = nullptr;
    size_t flags_cap = 0;
    int32_t epoch = 0;
};
// Q_MAIN serves plain-ME, deblocking and the bounded-wait self-test (flags
// that only ever hold an epoch); Q_LOOKAHEAD the lookahead, which can
// therefore run on another stream beside them; Q_WIDE the wide and pipelined
// closed-loop kernels, whose flag space also holds MV words and counters and
// is cleared before each of their launches.  The counters sit 128 bytes apart.
constexpr int Q_MAIN = 0, Q_LOOKAHEAD = 1, Q_WIDE = 2, NUM_QUEUES = 3, Q_COUNTER_STRIDE = 32;
// h264a_pixel_path_host: PP_CHUNKS upload chunks; its events are the
// uploads, planes and half-res frames ready, ME + T/Q done, lookahead done.
constexpr int PP_CHUNKS = 4;
constexpr int PP_EV_INPUTS = PP_CHUNKS, PP_EV_TQ = PP_CHUNKS + 1, PP_EV_LA = PP_CHUNKS + 2, PP_EVENTS = PP_CHUNKS + 3;

// An input slot of h264a_pixel_path_host: a device copy of a batch of frames,
// uploaded by h264a_pixel_path_prefetch ahead of the call that uses it
// (pending until that call takes it) or by the call itself.
struct PpInput {
    uint8_t *d = nullptr;
    size_t cap = 0;
    const uint8_t *h = nullptr;  // the host frames it holds
    int n = 0, cw = 0, ch = 0;
    int pending = 0;             // prefetched, not yet used by a call
    long long seq = 0;           // prefetch order
    cudaEvent_t ev = nullptr;    // the upload is complete
};
constexpr int PP_SLOTS = 2;

struct h264a_ctx {
    int device = 0;
    int num_sms = 0;
    cudaStream_t stream = nullptr;
    // device scratch of the persistent kernels: the work queues and a status
    // word (the code of a bounded wait that ran out)
    int32_t *d_counters = nullptr;
    WorkQueue q[NUM_QUEUES];
    int32_t *d_status = nullptr;
    // cached buffers of h264a_pixel_path_host, its copy and lookahead streams
    // and events
    void *pp_buf = nullptr;
    size_t pp_bytes = 0;
    cudaStream_t copy_stream = nullptr;
    cudaStream_t la_stream = nullptr;
    cudaEvent_t pp_ev[PP_EVENTS] = {};
    // row completion of the fused ME + T/Q launch: device counters, and
    // mapped pinned words the host polls (pp_rows_cap rows), with the token
    // of the current call
    int32_t *pp_row_count = nullptr;
    int32_t *pp_rows_host = nullptr;
    int32_t *pp_rows_dev = nullptr;
    size_t pp_rows_cap = 0;
    int32_t pp_token = 0;
    // frame table of plain-ME launches over more than 96 frames: the device
    // copy, its pinned staging buffer (me_tab_cap bytes each) and the event
    // of the last upload from it
    void *me_tab = nullptr;
    void *me_tab_host = nullptr;
    size_t me_tab_cap = 0;
    cudaEvent_t me_tab_ev = nullptr;
    // cached device buffers of h264a_pixel_path_closed
    void *cl_buf = nullptr;
    size_t cl_bytes = 0;
    // input slots and the stream their prefetch uploads run on
    PpInput pp_in[PP_SLOTS];
    long long pp_seq = 0;
    cudaStream_t pf_stream = nullptr;
    // pinned host words holding the current token, the source of the arrival
    // words that h264a_pixel_path_closed's uploads write after each chunk
    int32_t *upl_tok = nullptr;
    size_t upl_cap = 0;
    // the batch runtime's autotuner: the launch shape found fastest for each
    // batch signature (resolutions, references, frames per step, preset)
    std::map<std::string, int> tune_cache;
};

namespace h264a {

void set_error(const std::string &msg);
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
// `stream` follows the CUDA convention: NULL is the device's default stream.
inline cudaStream_t pick_stream(h264a_ctx *, void *s) { return reinterpret_cast<cudaStream_t>(s); }
int check_launch(const char *what);
// grows the per-MB done flags of work queue `queue` to at least n entries
// (zeroed, epoch reset)
int ensure_me_scratch(h264a_ctx *ctx, size_t n, int queue = Q_MAIN);
// Per-frame outputs of the MC + luma T/Q fused into the plain-ME kernel:
// coefficients (256 i16 per MB, 16-byte aligned), the QP and dead-zone
// divisor, and optional row completion words (see FrameDesc in me.cu).
struct MeTqOut {
    int16_t *coeffs;
    int qp, dz_div;
    int32_t *row_count;  // optional: mb_h zeroed counters
    int32_t *row_done;   // with row_count: mb_h words the host can read
    int32_t row_token;
};
// Per-frame inputs of the learned-proposal search: 16 i32 of proposals per
// MB, an optional fallback flag per MB, and the fallback threshold.
struct MeLearnIn {
    const int32_t *props;
    int32_t *fallback;
    int32_t prop_t;
};
// Per-frame reconstruction fused into the wide plain-ME kernel (the closed
// loop): the frame's chroma source, the previous frame's chroma
// reconstruction, the frame's reconstruction planes (written, then deblocked
// in place) and chroma levels (128 i16 per MB, 16-byte aligned).  Luma levels
// and the QP come from the frame's MeTqOut.
struct MeRecIn {
    const uint8_t *src_u, *src_v;
    const uint8_t *ref_u, *ref_v;
    uint8_t *rec_y, *rec_u, *rec_v;
    int16_t *ccoeffs;
};
// The pipelined closed loop (closed_pipe_kernel in me.cu): frames 1..n-1 of
// a clip in one launch, each searched on the planes of the deblocked
// reconstruction of the frame before it.  planes: four picture-plane buffers
// (4 * (cw + 2 pad) * (ch + 2 pad) bytes each), buffer 0 holding the planes of
// rec[0] (built by the caller, as is rec[0] itself); outputs per frame as
// h264a_closed_dev's.  props non-null: the learned 16x16 search.
struct ClosedPipeIn {
    int n, cw, ch, pad;
    const uint8_t *y, *u, *v;
    uint8_t *rec_y, *rec_u, *rec_v;
    uint8_t *planes;
    double lambda_me;
    int64_t split_gate;
    int qp, dz_div;
    int32_t *picks;
    int64_t *costs;
    int16_t *coeffs, *ccoeffs;
    const int32_t *props;
    int32_t *fallback;
    int32_t prop_t;
    // arrival words (or null): frame h's sources are in device memory once
    // arrive[h] == atoken (written by the host's upload stream after them)
    const int32_t *arrive = nullptr;
    int32_t atoken = 0;
};
// frame_words (device view of mapped host words, or null): word h is set to
// `token` once every MB of frame h is final, for the host to start its
// downloads while later frames run.
int closed_pipe_run(h264a_ctx *ctx, const ClosedPipeIn &in, const h264a_me_params *params, cudaStream_t st,
                    int32_t *frame_words = nullptr, int32_t token = 0);
// grows the mapped completion words (and their device counters) of the
// host-buffer entry points to `rows` words
int ensure_pp_rows(h264a_ctx *ctx, size_t rows);
// the next token of those words (clearing them when the counter wraps)
int32_t next_pp_token(h264a_ctx *ctx);
// plain-ME of frames, with the fused T/Q when tq is given (one entry per
// frame), the learned-proposal 16x16 search when learn is given, and the
// fused reconstruction + deblocking when rec is given (tq required, at most
// two frames)
int me_frames_run(h264a_ctx *ctx, const h264a_me_frame *h_frames, int nframes, const h264a_me_params *params,
                  const MeTqOut *tq, void *stream, const MeLearnIn *learn = nullptr, const MeRecIn *rec = nullptr);
// A tiled TMA map of a dense 3D u8 tensor (w x h x d, rows of w bytes, planes
// of w*h), box bw x bh x bd, no multicast; 0 when the driver entry point is
// missing or the layout breaks the TMA rules (the caller then copies without).
int encode_u8_map_3d(CUtensorMap* map, const uint8_t* base, int w, int h, int d, int bw, int bh, int bd);
struct MeParamsDev;
// A multi-reference frame table laid out for the device: the frame
// descriptors (largest frames first, tensor maps encoded), the queue's
// segment starts and their frame counts.
struct MrTable {
    std::vector<char> bytes;
    int nframes = 0, nseg = 0;
    long long total = 0;  // MBs
    size_t b_desc = 0, b_seg = 0;
};
// h264a_mc_tq_frames_multiref on stream st (checks its arguments)
int mc_tq_mr_run(h264a_ctx *ctx, const h264a_mc_tq_mr_frame *h_frames, int nframes, cudaStream_t st);
// validates h_frames as h264a_me_frames_multiref does and lays out their table
int mr_table_build(const h264a_me_mr_frame *h_frames, int nframes, MrTable &t);
// one launch of the multi-reference kernel in launch shape `variant` over the
// table at d_table (t's bytes in device memory), on the queue counter/flags
// (flags of t.total MBs holding no `epoch`)
int mr_launch(h264a_ctx *ctx, int variant, const MeParamsDev &prm, const void *d_table, const MrTable &t,
              int32_t *counter, int32_t *flags, int epoch, cudaStream_t st);
// the flag value of the next persistent launch on `st`
int next_epoch(h264a_ctx *ctx, cudaStream_t st, int queue = Q_MAIN);

// Device-side mirror of h264a_me_params with only the fields the kernels read.
struct MeParamsDev {
    int32_t fast, use_sad, sadfp, kind;
    const uint16_t *tab;
    double sadfp_lambda;
    int32_t me_snap, fc;
    uint32_t dia_mask, dia_sub_mask;
    int32_t subpel, subpel_pat, sp_single_pass, sub_pat, me_subpel_iter, sp_maxit, sp_fc;
};
MeParamsDev to_dev(const h264a_me_params &p);

}  // namespace h264a

#define H264A_CUDA(call)                                              \
    do {                                                              \
        cudaError_t e_ = (call);                                      \
        if (e_ != cudaSuccess) return ::h264a::cuda_fail(e_, #call); \
    } while (0)
