/*
 * h264accel.h -- C ABI of libh264accel_cuda.so, the B200 (sm_100a) encoder
 * pixel hot path of rusty_h264.
 *
 * The reference's boundary is the free-function surface of the
 * `rusty_h264-accel` crate (crates/rusty_h264-accel/src/lib.rs:33-58), called
 * per block (~17 ns of work each).  A GPU launch costs ~100x that, so every
 * entry point here keeps the value contract of one reference function but
 * takes a whole batch (or a whole frame) per call.  Each declaration names the
 * reference function it replaces.
 *
 * Conventions
 *  - Every call returns H264A_OK (0) or a negative H264A_E_* code; the message
 *    is in h264a_last_error() (per thread).  Nothing aborts across the ABI.
 *  - Pointers named d_* are device pointers (CUDA global memory of the
 *    context's device); h_* are host pointers.  Callers own every buffer.
 *  - `stream` is a cudaStream_t (NULL = the device's default stream, as in the
 *    CUDA runtime).  Calls only enqueue work; results are ready when the
 *    stream is synchronised (h264a_sync).  The persistent wavefront kernels
 *    serialise on a context's work-queue scratch: h264a_me_frames (more than
 *    two frames) and h264a_deblock_frames share one queue,
 *    h264a_lookahead_costs has a second, and the one- and two-frame searches
 *    and the closed loop (h264a_me_frames with at most two frames,
 *    h264a_closed_step_frame, h264a_closed_frames, h264a_pixel_path_closed) a
 *    third, so within one context the lookahead may run on another stream
 *    beside any of them; otherwise use one context per concurrent stream.
 *  - Planes: a reference picture's cached planes are one buffer F|H|V|C, each
 *    pw*ph bytes with pw = cw + 2*pad, ph = ch + 2*pad, stride pw: the
 *    HpelPlanes layout of crates/rusty_h264-common/src/inter.rs:707-730.
 *  - Motion vectors are quarter-pel (i32, x then y), as in the reference.
 */
#ifndef H264ACCEL_H
#define H264ACCEL_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define H264A_API __attribute__((visibility("default")))
#else
#define H264A_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define H264A_OK 0
#define H264A_E_ARG (-1)       /* invalid argument (size, stride, pointer) */
#define H264A_E_CUDA (-2)      /* a CUDA runtime call failed */
#define H264A_E_TIMEOUT (-3)   /* a bounded device wait ran out (see h264a_last_error) */
#define H264A_E_NOMEM (-4)     /* device allocation failed */
#define H264A_E_NODEV (-5)     /* no usable sm_100 device */

typedef struct h264a_ctx h264a_ctx;

/* ---- context ----------------------------------------------------------- */
H264A_API const char *h264a_version(void);
H264A_API const char *h264a_last_error(void);
H264A_API int h264a_ctx_create(int device, h264a_ctx **out);
H264A_API int h264a_ctx_destroy(h264a_ctx *ctx);
H264A_API int h264a_sync(h264a_ctx *ctx, void *stream);
/* convenience device memory for callers without the CUDA runtime (FFI) */
H264A_API int h264a_dev_alloc(h264a_ctx *ctx, size_t bytes, void **d_out);
H264A_API int h264a_dev_free(h264a_ctx *ctx, void *d_ptr);
H264A_API int h264a_memcpy_h2d(h264a_ctx *ctx, void *d_dst, const void *h_src, size_t bytes, void *stream);
H264A_API int h264a_memcpy_d2h(h264a_ctx *ctx, void *h_dst, const void *d_src, size_t bytes, void *stream);

/* ---- a1/a2: half-pel planes -------------------------------------------- */
/* pad_plane_into + hpel_fused / build_hpel_planes
 * (common/src/inter.rs:798-849, accel/src/hpel.rs:34-203) for n pictures:
 * picture i is d_ref + i*ref_frame_stride (cw x ch, row stride cw), its planes
 * go to d_planes + i*4*pw*ph.  pad >= 3 (the reference default is 32). */
H264A_API int h264a_hpel_build(h264a_ctx *ctx, const uint8_t *d_ref, int cw, int ch, int pad, int n,
                     size_t ref_frame_stride, uint8_t *d_planes, void *stream);

/* ---- a6/a7/a8: block metrics -------------------------------------------- */
#define H264A_METRIC_SATD_WELS 0 /* Σ_4x4((Σ|H·d|+1)>>1): satd_16x16..satd_4x4 (satd_sad.rs:309-340) */
#define H264A_METRIC_SATD 1      /* Σ|H·d|: satd_x4 / satd_x4p (satd_avg.rs:350-420), satd_px (mb16.rs:6027) */
#define H264A_METRIC_SAD 2       /* Σ|a−b|: sad_16x16.. / sad_x4 (satd_sad.rs:342-363, satd_avg.rs:462) */
#define H264A_METRIC_SATD_AVG 3  /* Σ|H·(a−(b+c+1)>>1)|: satd_avg / satd_avg_x4 (satd_avg.rs:536-602) */
#define H264A_METRIC_SAD_AVG 4   /* Σ|a−(b+c+1)>>1|: sad_avg_strided (mb16.rs:6104) */
/* out[i] = metric of the w×h blocks at d_a+a_off[i] (stride sa) vs d_b+b_off[i]
 * (stride sb) [and d_c+c_off[i] for the *_AVG metrics, stride sb].
 * (w,h) in {16x16,16x8,8x16,8x8,8x4,4x8,4x4}.  The x4 calls are this with n=4k. */
H264A_API int h264a_block_metric(h264a_ctx *ctx, int metric, int w, int h, const uint8_t *d_a, const int64_t *d_a_off, int sa,
                       const uint8_t *d_b, const int64_t *d_b_off, const uint8_t *d_c, const int64_t *d_c_off, int sb,
                       int n, int32_t *d_out, void *stream);

/* ---- a3/a4/a5/a9: candidate distortion ---------------------------------- */
typedef struct {
    const uint8_t *d_src;    /* coded source luma, stride cw */
    const uint8_t *d_planes; /* the reference's F|H|V|C planes */
    int32_t cw, ch, pad;
} h264a_picture;

typedef struct {
    int32_t pic;             /* index into the picture array */
    int32_t x, y, w, h;      /* block in the source */
    int32_t mvx, mvy;        /* quarter-pel candidate */
} h264a_candidate;

/* Distortion of arbitrary candidates, exactly the values of MeCtx::eval
 * (accel/src/mectx.rs:112-166) / mc_satd_hp (metric SATD, mb16.rs:1930) and
 * mc_sad_hp (metric SAD, mb16.rs:2018), including candidates off the planes,
 * where the reference falls back to mc_luma (inter.rs:1193).  A candidate
 * whose picture index, shape or block position is out of range gets -1. */
H264A_API int h264a_candidate_dist(h264a_ctx *ctx, const h264a_picture *d_pics, int npics, const h264a_candidate *d_cands, int n,
                         int metric, int32_t *d_out, void *stream);

/* ---- a10/a11/a12: motion search ------------------------------------------ */
typedef struct {
    int32_t fast;            /* Preset::Fast: SAD cost, [16,4] ladder (config.rs:8-38) */
    int32_t mb_use_satd;     /* fast preset's SATD override (mb16.rs:2507) */
    int32_t sadfp;           /* B2: SAD-domain full-pel phase (mb16.rs:616-643) */
    int32_t mv_cost_kind;    /* 0 Exp-Golomb, 1 smooth table, 2 measured table (mb16.rs:563) */
    const uint16_t *d_mv_cost_tab; /* device, 4096 u16 (kinds 1, 2; see h264a_build_mv_cost_table) */
    double sadfp_lambda;     /* RFF_ME_SADL, 0.5 (mb16.rs:756) */
    int32_t me_snap;         /* tune_me_snap, 1 */
    int32_t me_fc;           /* fixed-centre diamond of the accel build, 1 (mb16.rs:700) */
    uint32_t dia_mask;       /* rungs of [64,32,16,8,4] qpel, 0b11100 (mb16.rs:828) */
    uint32_t dia_sub_mask;   /* sub-8x8 rungs, 0b10000 (mb16.rs:851) */
    int32_t subpel;          /* run the [2,1] sub-pel steps (mb16.rs:2956) */
    int32_t subpel_pat;      /* -1 = preset default, else RFF_SUBPEL_PAT 0..3 */
    int32_t sp_single_pass;  /* Balanced (mb16.rs:1664) */
    int32_t sub_pat;         /* RFF_SUBPEL_SUB, 2 */
    int32_t me_subpel_iter;  /* tune_me_subpel_iter, 1 */
    int32_t sp_maxit;        /* RFF_SP_MAXIT, 0 = unlimited */
    int32_t sp_fc;           /* RFF_SP_FC batched rings, 0 */
} h264a_me_params;

/* Fills *p with the Balanced-preset defaults the reference encoder runs. */
H264A_API void h264a_me_params_default(h264a_me_params *p);
/* The smooth mvd-cost table of mb16.rs:508-519 (kind 1), 4096 entries, host. */
H264A_API void h264a_build_mv_cost_table(uint16_t *h_out);

typedef struct {
    int32_t pic;
    int32_t x, y, w, h;      /* partition in the source, w,h in {16,8,4} */
    int32_t npred;           /* 1..4 seeds; preds[0] is the mvd centre */
    int32_t preds[8];
    int32_t has_start;       /* refine-only search from start (mb16.rs:2445) */
    int32_t start[2];
    double lambda_me;
} h264a_me_job;

typedef struct {
    int32_t mvx, mvy;
    int64_t cost;            /* J = D + (λ·bits) as i64, the search's own domain */
    int32_t evals;           /* distortion evaluations performed */
    int32_t status;          /* 0 ok */
} h264a_me_result;

/* n independent motion_search calls (mb16.rs:2433-3302), one warp each.  A
 * job with an out-of-range picture, shape, position or npred gets status -1. */
H264A_API int h264a_me_search(h264a_ctx *ctx, const h264a_picture *d_pics, int npics, const h264a_me_params *params,
                    const h264a_me_job *d_jobs, int n, h264a_me_result *d_out, void *stream);

/* Plain-ME frames: every MB of every frame runs best_part (mb16.rs:4921) for
 * 16x16 and, when its J exceeds split_gate (>= 0), the 16x8/8x16 partitions
 * with the MB's neighbours feeding predict_mv (inter.rs:36, mv_neighbors_block
 * mb16.rs:1871) in raster dependency order, every MB assumed coded inter with
 * ref 0.  One persistent launch drains a work queue over all frames (MBs of
 * different frames interleave); each MB waits (bounded) for its left and
 * top-right neighbours.  Picks: 6 i32 per MB {shape 0/1/2, mv0x, mv0y, mv1x,
 * mv1y, work} where work counts the 4x4-block distortion evaluations the
 * reference performs for the MB; costs: 2 i64 per MB {pick J, 16x16 J}.
 * Up to 96 frames the launch carries the frame table in its parameters; a
 * call of more frames uploads it through a staging buffer of the context and
 * waits for that buffer's previous upload, so such calls do not belong in a
 * stream capture. */
typedef struct {
    h264a_picture pic;
    double lambda_me;
    int64_t split_gate;
    int32_t *d_picks;
    int64_t *d_costs;
} h264a_me_frame;

H264A_API int h264a_me_frames(h264a_ctx *ctx, const h264a_me_frame *h_frames, int nframes, const h264a_me_params *params,
                    void *stream);

/* h264a_me_frames with the MC + luma T/Q of each MB's pick (as
 * h264a_mc_tq_frames, mb16.rs:3436-3450) in the same launch: the warp that
 * publishes an MB's pick then transforms and quantises the MB's 16 blocks, so
 * each MB's coefficients are written as soon as its pick is known and no
 * second pass reads the frames again.  d_coeffs: 256 i16 per MB, 16-byte
 * aligned, in any memory the device can write (device memory, or mapped
 * pinned host memory).  Outputs equal h264a_me_frames followed by
 * h264a_mc_tq_frames. */
typedef struct {
    h264a_me_frame me;
    int32_t qp, dz_div;
    int16_t *d_coeffs;
} h264a_me_tq_frame;

H264A_API int h264a_me_tq_frames(h264a_ctx *ctx, const h264a_me_tq_frame *h_frames, int nframes,
                                 const h264a_me_params *params, void *stream);

/* h264a_me_frames for callers that cannot allocate device memory when they
 * run motion estimation (an encoder thread that must not block on the CUDA
 * allocator, or a host that gives this library a fixed memory budget and owns
 * every buffer).  No counterpart in the reference.  It needs no context and
 * allocates nothing: the persistent kernel's scratch (queue counter and one
 * flag per macroblock) is a fixed device array inside the library, so one call
 * covers at most H264A_NOALLOC_MAX_MBS macroblocks (sum over its frames) and at
 * most 96 frames; larger requests return H264A_E_ARG.  The array is set up
 * (its device address looked up) on the first call on each device, so make
 * that first call before any stream capture; the address is kept for the
 * process, so do not call this entry point again on a device whose primary
 * context was reset (cudaDeviceReset).  Every call on a device shares the
 * array and clears the part it uses (queue counter and its macroblocks'
 * flags) on `stream` before its launch: calls that overlap on the GPU race
 * and must not be issued on concurrent streams.  The caller passes a device
 * int32 d_status, which the call zeroes and the kernel sets to non-zero if a
 * bounded wait ran out; read it after synchronising `stream`.  Outputs as
 * h264a_me_frames. */
#define H264A_NOALLOC_MAX_MBS 65536
H264A_API int h264a_me_frames_noalloc(const h264a_me_frame *h_frames, int nframes, const h264a_me_params *params,
                                      int32_t *d_status, void *stream);

/* Exhaustive full-pel 16x16 grid (±R around each MB's centre MV) with SAD and
 * SATD values as the ME cost functions return them (mc_sad_hp / mc_satd_hp at
 * full-pel MVs), and the per-MB argmin of dist + (λ·bits(mv − pmv)) in raster
 * order with first-wins ties (the exhaustive probe of mb16.rs:2889-2900).
 * d_centers/d_pmv: 2 i32 per MB (NULL = zero).  Grids (optional, NULL to
 * skip): (2R+1)^2 i32 per MB, row-major in dy.  d_best: 4 i32 per MB
 * {mvx, mvy, cost, dist} for metric (0 = SAD, 1 = SATD).  1 <= R <= 64. */
H264A_API int h264a_fullpel_grid(h264a_ctx *ctx, const h264a_picture *h_pic, int R, const int32_t *d_centers,
                       const int32_t *d_pmv, int metric, int mv_cost_kind, const uint16_t *d_mv_cost_tab,
                       double lambda, int32_t *d_sad_grid, int32_t *d_satd_grid, int32_t *d_best, void *stream);

/* ---- a13/a14/a15: forward transform + quant ------------------------------ */
/* dct_four_t4 + quant_four_4x4 (accel/src/transform_quant.rs:76, 122) over n
 * 8x8 regions: region i is at (xy[2i], xy[2i+1]) in both planes; 64 i16 out
 * per region in the reference's sub-block order; ff/mf from quant_dz_ff(qp,dz)
 * and QUANT_MF_OH[qp] (transform.rs:145, 1447), qp per region. */
H264A_API int h264a_dct_quant_4x4(h264a_ctx *ctx, const uint8_t *d_src, int ss, const uint8_t *d_pred, int ps,
                        const int32_t *d_xy, const uint8_t *d_qp, int dz_div, int n, int16_t *d_out, void *stream);
/* forward_core_8x8 + quantize_8x8 (transform.rs:548, 613), flat or given
 * scaling-list weights (host array of 64 i32, raster; NULL = flat 16):
 * 64 i32 levels per region, raster order. */
H264A_API int h264a_dct_quant_8x8(h264a_ctx *ctx, const uint8_t *d_src, int ss, const uint8_t *d_pred, int ps,
                        const int32_t *d_xy, const uint8_t *d_qp, const int32_t *h_weight, int dz_div, int n,
                        int32_t *d_out, void *stream);
/* MC of each MB's pick (the planes' quarter-pel prediction = mc_luma) then the
 * luma T/Q of mb16.rs:3436-3450: 256 i16 per MB, for n frames. */
typedef struct {
    h264a_picture pic;
    const int32_t *d_picks;  /* 6 i32 per MB, as h264a_me_frames writes */
    int32_t qp, dz_div;
    int16_t *d_coeffs;       /* 256 i16 per MB */
} h264a_tq_frame;
H264A_API int h264a_mc_tq_frames(h264a_ctx *ctx, const h264a_tq_frame *h_frames, int nframes, void *stream);
/* h264a_mc_tq_frames plus the inter MB's luma reconstruction of
 * mb16.rs:3575-3605 (dequantize, transform.rs:233; inverse 4x4 + add + clamp,
 * idct_four_t4_rec, accel/src/transform_quant.rs:96): d_rec receives the
 * cw x ch reconstructed luma (4-byte aligned), the next frame's reference
 * picture, without leaving the device. */
typedef struct {
    h264a_tq_frame tq;
    uint8_t *d_rec;
} h264a_tq_rec_frame;
H264A_API int h264a_mc_tq_rec_frames(h264a_ctx *ctx, const h264a_tq_rec_frame *h_frames, int nframes, void *stream);
/* The inter MB's chroma (mb16.rs:3408-3428, 3465-3500, 3606-3628): mc_chroma
 * (inter.rs:1268) of each partition with its luma MV, dct_four_t4 +
 * quant_four_4x4 at chroma_qp(qp) (predict.rs:64), the 2x2 DC through
 * forward_quant_chroma_dc (transform.rs:1023, inter dead-zone), and, when
 * d_rec_u/d_rec_v are given, the reconstruction (dequantize with the DC from
 * inverse_quant_chroma_dc, idct_four_t4_rec).  Out: 128 i16 per MB, U then V,
 * four 4x4 blocks each in the order (0,0),(4,0),(0,4),(4,4), 16 levels per
 * block in raster order with slot 0 holding the block's DC level (the
 * Hadamard output of that index). */
typedef struct {
    const uint8_t *d_src_u, *d_src_v; /* (cw/2) x (ch/2) source chroma, 4-byte aligned */
    const uint8_t *d_ref_u, *d_ref_v; /* the reference picture's chroma, 4-byte aligned */
    int32_t cw, ch;                   /* luma size, MB-aligned */
    const int32_t *d_picks;           /* 6 i32 per MB, as h264a_me_frames writes */
    int32_t qp;                       /* luma QP 0..51 */
    int16_t *d_coeffs;                /* 128 i16 per MB, 16-byte aligned */
    uint8_t *d_rec_u, *d_rec_v;       /* reconstruction planes, or both NULL */
} h264a_tq_chroma_frame;
H264A_API int h264a_mc_tq_chroma_frames(h264a_ctx *ctx, const h264a_tq_chroma_frame *h_frames, int nframes,
                                        void *stream);

/* In-loop deblocking (crates/rusty_h264-common/src/deblock.rs, filter_frame)
 * of reconstructed plain-ME P pictures: every MB inter with reference 0,
 * 4x4 transforms, one QP; bS from the picks and the luma levels (2 with
 * coefficients on either side, 1 for MVs 4 quarter-pels apart, else 0).  The
 * planes are filtered in place, MBs in the reference's raster order (as a
 * wavefront on the GPU); d_u / d_v may both be NULL (luma only). */
typedef struct {
    uint8_t *d_y, *d_u, *d_v;  /* cw x ch luma, (cw/2) x (ch/2) chroma, 4-byte aligned */
    int32_t cw, ch;            /* MB-aligned */
    const int32_t *d_picks;    /* 6 i32 per MB, as h264a_me_frames writes */
    const int16_t *d_coeffs;   /* 256 i16 luma levels per MB (h264a_mc_tq_frames), 16-byte aligned */
    int32_t qp;                /* the picture's QP, 0..51 */
    int32_t offset_a, offset_b, chroma_qp_offset; /* slice filter offsets and the chroma QP offset */
} h264a_deblock_frame;
H264A_API int h264a_deblock_frames(h264a_ctx *ctx, const h264a_deblock_frame *h_frames, int nframes, void *stream);

/* ---- a16-a19: mb-tree lookahead ------------------------------------------ */
/* downsample2x (encoder/src/mbtree.rs:61-74) of n frames cw x ch -> cw/2 x ch/2. */
H264A_API int h264a_downsample2x(h264a_ctx *ctx, const uint8_t *d_frames, int cw, int ch, int n, size_t frame_stride,
                       uint8_t *d_half, void *stream);
/* frame_costs (mbtree.rs:208-263) of n consecutive frames, frame f against
 * frame f-1 (frame 0 is the IDR: intra only).  mode 0 FullRes, 1 Hybrid,
 * 2 HalfRes (the default, config.rs:568).  d_full: n frames cw x ch;
 * d_half: their downsample2x (needed for modes 1, 2).  Out per MB: intra,
 * inter (i32) and the full-res quarter-pel MV (2 i32). */
H264A_API int h264a_lookahead_costs(h264a_ctx *ctx, const uint8_t *d_full, const uint8_t *d_half, int cw, int ch, int n,
                          int mode, int32_t *d_intra, int32_t *d_inter, int32_t *d_mvs, void *stream);
/* h264a_lookahead_costs of several streams (each its own clip of n
 * consecutive frames, any size) in one persistent launch of the chains (up
 * to 24 streams per launch), the per-GOP lookahead that encode_all runs for
 * each GOP (encoder/src/lib.rs:764-770, mbtree::gop_qp_offsets): outputs per
 * stream exactly as h264a_lookahead_costs gives them. */
typedef struct {
    const uint8_t *d_full, *d_half;
    int32_t cw, ch, n;
    int32_t *d_intra, *d_inter, *d_mvs;
} h264a_la_stream;
H264A_API int h264a_lookahead_streams(h264a_ctx *ctx, const h264a_la_stream *streams, int nstreams, int mode,
                                      void *stream);

/* ---- the whole pixel path from host memory -------------------------------- */
/* Copies n coded luma frames (cw x ch, contiguous) to the device, builds the
 * planes of frames 0..n-2, runs plain-ME + MC + T/Q for frames 1..n-1 (each
 * against the previous source frame) and the HalfRes lookahead for all n
 * frames, and copies the results back.  Output arrays are per frame (frame 0
 * rows are zero for picks/costs/coeffs): h_picks 6 i32/MB, h_costs 2 i64/MB,
 * h_coeffs 256 i16/MB, h_la_intra/h_la_inter 1 i32/MB, h_la_mvs 2 i32/MB.
 * ME runs with the MC + T/Q fused in, the lookahead beside it, and the rows
 * of MBs that are final come down while the launch still runs (pinned output
 * buffers make those copies asynchronous).  Device buffers are cached in the
 * context between calls of the same shape. */
H264A_API int h264a_pixel_path_host(h264a_ctx *ctx, const uint8_t *h_frames, int n, int cw, int ch, const h264a_me_params *params,
                          const uint16_t *h_mv_cost_tab, double lambda_me, int64_t split_gate, int qp, int dz_div,
                          int32_t *h_picks, int64_t *h_costs, int16_t *h_coeffs, int32_t *h_la_intra,
                          int32_t *h_la_inter, int32_t *h_la_mvs);
/* Queues the upload of n frames (cw x ch, contiguous; pinned memory makes it
 * asynchronous) into one of the context's two input slots, on a stream of its
 * own, and returns.  The next h264a_pixel_path_host call with the same
 * h_frames, n, cw and ch takes the frames from that slot instead of uploading
 * them, so a caller that prefetches batch k+1 before the call for batch k
 * overlaps each upload with the previous batch's compute.  The caller must not
 * change the frames until that call.  At most two prefetches may be pending
 * (H264A_E_ARG otherwise); a call whose frames match no pending prefetch
 * uploads them itself. */
H264A_API int h264a_pixel_path_prefetch(h264a_ctx *ctx, const uint8_t *h_frames, int n, int cw, int ch);

/* ---- learned motion-vector proposals ----------------------------------------- */
/* A small conv net that proposes the 8 most likely full-pel MVs of every
 * 16x16 MB of a frame; h264a_me_frames_learned then prices them with the
 * search's exact integer cost and refines the best with motion_search's
 * sub-pel refinement.  No counterpart in the reference, which runs
 * motion_search (mb16.rs:2433) on every MB.
 *   Input per frame pair (current frame, reference frame): a 2-channel image
 * (reference, current) as (u8 - 128) / 64.  Trunk over the whole image: three
 * 3x3 stride-2 convs (2->16->32->32 channels, zero padding at the frame
 * edges), a map of 32 features per 8x8 pixels.  Per MB: the 6x6 cells of its
 * co-located 48x48 region (zero outside the map) and the MVs of three
 * neighbour MBs (left, top, top-right) -> FC 1168->256 -> head 256->296
 * logits, of which the first 289 are the full-pel offsets (dx, dy) in
 * [-8, 8]^2, class (dy+8)*17 + dx+8.  bf16 weights and activations, fp32
 * accumulation on the tensor cores; trained with Adam on softmax
 * cross-entropy against the plain search's 16x16 MVs.
 *   A batch is npairs frame pairs of one geometry (cw x ch, at most
 * H264A_MVNET_MAX_PIXELS pixels in all) and its samples are every MB of
 * them, pair-major, raster order within a pair: d_nmv holds 6 i16 per MB
 * (the neighbour MVs, quarter-pel), d_labels 1 i16 per MB (class 0..288).
 * A net owns its parameters, optimiser state and the workspace of one batch;
 * calls on one net must not overlap. */
#define H264A_MVNET_NPARAMS 389528
#define H264A_MVNET_MAX_PIXELS 8388608
typedef struct h264a_mvnet h264a_mvnet;
typedef struct {
    const uint8_t *d_cur;    /* current frame luma, cw x ch, stride cw */
    const uint8_t *d_ref;    /* reference frame luma, same geometry */
} h264a_mvnet_pair;
/* seeded He-normal initialisation (zero biases) */
H264A_API int h264a_mvnet_create(int device, uint64_t seed, h264a_mvnet **out);
H264A_API int h264a_mvnet_destroy(h264a_mvnet *net);
/* flat fp32 parameter vector (w1 16x3x3x2, b1 16, w2 32x3x3x16, b2 32,
 * w3 32x3x3x32, b3 32, w4 256x1168, b4 256, w5 296x256, b5 296; conv weights
 * [out][ky][kx][in]); set_params also resets the optimiser state */
H264A_API int h264a_mvnet_set_params(h264a_mvnet *net, const float *h_params);
H264A_API int h264a_mvnet_get_params(h264a_mvnet *net, float *h_params);
/* logits of every MB of a batch (npairs * nmb x 296 fp32, device) */
H264A_API int h264a_mvnet_forward(h264a_mvnet *net, const h264a_mvnet_pair *d_pairs, int npairs, int cw, int ch,
                                  const int16_t *d_nmv, float *d_logits, void *stream);
/* mean cross-entropy loss (d_loss, 1 fp32) of a batch and its gradient
 * (d_grads, NPARAMS fp32), without updating the parameters */
H264A_API int h264a_mvnet_grads(h264a_mvnet *net, const h264a_mvnet_pair *d_pairs, int npairs, int cw, int ch,
                                const int16_t *d_nmv, const int16_t *d_labels, float *d_grads, float *d_loss,
                                void *stream);
/* one Adam step (beta 0.9 / 0.999, eps 1e-8) at learning rate lr on a batch;
 * d_loss (optional) receives the batch's loss before the step */
H264A_API int h264a_mvnet_train_step(h264a_mvnet *net, const h264a_mvnet_pair *d_pairs, int npairs, int cw, int ch,
                                     const int16_t *d_nmv, const int16_t *d_labels, float lr, float *d_loss,
                                     void *stream);
/* Proposals for every MB of whole frames: d_props receives 16 i32 per MB
 * (8 quarter-pel MVs, most likely first).  d_guide_mvs (optional, 2 i32 per
 * MB) are the MVs the neighbour features are read from -- the HalfRes
 * lookahead's MVs (h264a_lookahead_costs) are known before motion estimation
 * starts, so proposals for a whole batch of frames come from one pass. */
typedef struct {
    const uint8_t *d_cur, *d_ref;
    int32_t cw, ch;
    const int32_t *d_guide_mvs;
    int32_t *d_props;
} h264a_mvnet_frame;
H264A_API int h264a_mvnet_propose(h264a_mvnet *net, const h264a_mvnet_frame *h_frames, int nframes, void *stream);

/* h264a_me_frames with the learned proposals in each MB's 16x16 search: the
 * search prices the median predictor and the MB's 8 proposals (d_props, 16
 * i32 per MB, as h264a_mvnet_propose writes them) with its exact integer cost
 * J = SATD + (lambda*bits) as i64.  If the cheapest proposal's SATD exceeds
 * the predictor's by more than fallback_t, the MB runs the plain search
 * (motion_search from its predictors, mb16.rs:2433) and d_fallback[mb] = 1;
 * otherwise the search continues as motion_search with the cheapest of the
 * nine as its start vector (mb16.rs:2445: no full-pel phase, the sub-pel
 * refinement only) and d_fallback[mb] = 0 (d_fallback optional).  The
 * 16x8/8x16 partitions of an MB that took a proposal refine from its 16x16 MV
 * in the same way (start vector mv16, mvd centre the predictor); those of a
 * fallen-back MB, the neighbours, outputs and the queue are as
 * h264a_me_frames'.  No counterpart in the reference. */
typedef struct {
    h264a_me_frame me;
    const int32_t *d_props;
    int32_t fallback_t;
    int32_t *d_fallback;
} h264a_me_learned_frame;
H264A_API int h264a_me_frames_learned(h264a_ctx *ctx, const h264a_me_learned_frame *h_frames, int nframes,
                                      const h264a_me_params *params, void *stream);

/* ---- plain-ME over several reference pictures ----------------------------------- */
/* h264a_me_frames with best_part's loop over references (mb16.rs:4921-4960):
 * each search (16x16, and the 16x8/8x16 partitions when its J exceeds
 * split_gate) runs on every reference r = 0..nref-1 (d_planes[r]: its F|H|V|C
 * planes, reference 0 the nearest) seeded [predict_mv against r, extra], its
 * J plus (lambda_me * ref_bits(r, nref)) truncated to i64 (mb16.rs:5967), the
 * strictly cheapest reference kept; predictors take only neighbours of the
 * same reference (inter.rs:36-69).  Picks: 8 i32 per MB (shape, ref0, mv0x,
 * mv0y, ref1, mv1x, mv1y, 4x4-block evaluations); costs 2 i64 per MB (the
 * pick's J, the 16x16's).  1 <= nref <= 4.  Queue as h264a_me_frames. */
typedef struct {
    const uint8_t *d_src;
    const uint8_t *d_planes[4];
    int32_t nref, cw, ch, pad;
    double lambda_me;
    int64_t split_gate;
    int32_t *d_picks;
    int64_t *d_costs;
} h264a_me_mr_frame;
H264A_API int h264a_me_frames_multiref(h264a_ctx *ctx, const h264a_me_mr_frame *h_frames, int nframes,
                                       const h264a_me_params *params, void *stream);
/* h264a_mc_tq_frames for multi-reference picks (8 i32 per MB, as
 * h264a_me_frames_multiref writes them): each half of an MB is predicted
 * from the planes of its own reference (mb16.rs:3436-3450 with best_part's
 * reference, mb16.rs:4921-4960), then the luma T/Q; 256 i16 per MB. */
typedef struct {
    const uint8_t *d_src;
    const uint8_t *d_planes[4];
    int32_t nref, cw, ch, pad;
    const int32_t *d_picks;
    int32_t qp, dz_div;
    int16_t *d_coeffs;
} h264a_mc_tq_mr_frame;
H264A_API int h264a_mc_tq_frames_multiref(h264a_ctx *ctx, const h264a_mc_tq_mr_frame *h_frames, int nframes,
                                          void *stream);

/* ---- batched plain-ME over many streams, one launch per GOP step ----------------- */
/* Many streams of uneven resolution advance together, G P frames of every
 * stream per step, where the reference encodes GOPs on parallel CPU threads
 * with a fresh encoder each (encoder/src/lib.rs:745-805).  Step k builds the
 * planes of frames kG..kG+count-1 of every stream (h264a_hpel_build) and then
 * runs, in one persistent launch over all streams, h264a_me_frames_multiref
 * of frames kG+1..kG+count (count <= G, the last step may be short), frame f
 * against frames f-1, .., f-min(nref, f) (nearest first).  Each step runs as
 * a CUDA graph captured the first time its slot layout occurs and replayed
 * afterwards (one graph launch per step).  Picks and costs are those of
 * h264a_me_frames_multiref on the same frames (8 i32 and 2 i64 per MB).
 * Streams with d_coeffs (a ring of nslots x nmb x 256 i16, 16-byte aligned)
 * also get each frame's MC + luma T/Q at qp (h264a_mc_tq_frames_multiref,
 * one launch in the same graph after the search; one dz_div per batch).
 * Each stream owns a ring of nslots slots; frame f lives in slot f % nslots
 * of d_src (cw*ch bytes per slot, 4-byte aligned), d_planes (4*pw*ph bytes
 * per slot, pw = cw + 2*pad; 16-byte aligned with pw a multiple of 16 for the
 * TMA-staged shapes), d_picks (8*nmb i32) and d_costs (2*nmb i64).  nslots is
 * a multiple of G and at least G + nref + 1 (step k reads sources kG..kG+G
 * and planes from kG-nref+1 on); with 2G + nref + 1 slots the sources of
 * step k+1 can be uploaded while step k runs.  Launch shape: the autotuner
 * (autotune = 1) times every variant on the first step, keeps the fastest for
 * the batch's signature (resolutions, nref, G, preset; cached in the context)
 * and captures with it; autotune = 0 uses `variant`.  Steps of one batch run
 * one at a time in stream order (each batch has its own queue; the context's
 * queues are untouched).  No counterpart of the graphs or the tuner in the
 * reference. */
#define H264A_BATCH_VARIANTS 6
typedef struct {
    int32_t cw, ch, pad;
    uint8_t *d_src;
    uint8_t *d_planes;
    int32_t *d_picks;
    int64_t *d_costs;
    double lambda_me;
    int64_t split_gate;
    int16_t *d_coeffs; /* NULL: search only */
    int32_t qp, dz_div;
} h264a_batch_stream;
typedef struct {
    int32_t gop_step; /* G >= 1 */
    int32_t nslots;
    int32_t nref;     /* 1..4 */
    int32_t autotune;
    int32_t variant;  /* 0..H264A_BATCH_VARIANTS-1, used when autotune = 0 */
} h264a_batch_config;
typedef struct {
    int32_t variant;                      /* the launch shape the graphs use */
    int32_t tuned;                        /* 1 when the autotuner chose it (this batch or the cache) */
    float ms[H264A_BATCH_VARIANTS];       /* the tuner's median ME time per variant (0 if not timed) */
    int32_t graphs;                       /* graphs captured so far */
    int64_t steps;                        /* steps run */
} h264a_batch_info;
typedef struct h264a_batch h264a_batch;
H264A_API int h264a_batch_create(h264a_ctx *ctx, const h264a_batch_stream *streams, int nstreams,
                                 const h264a_batch_config *cfg, const h264a_me_params *params, h264a_batch **out);
H264A_API int h264a_batch_step(h264a_batch *b, int64_t k, int count, void *stream);
H264A_API int h264a_batch_get_info(const h264a_batch *b, h264a_batch_info *out);
H264A_API int h264a_batch_destroy(h264a_batch *b);
/* Variant v's shape: MBs a CTA holds at once (one warp each) and whether each
 * search's window is staged in shared memory by TMA (1) or read from L2 (0). */
H264A_API int h264a_batch_variant_shape(int variant, int *mbs_per_cta, int *staged);

/* ---- the closed reconstruction loop ------------------------------------------ */
/* The pixel path as the encoder runs it: every P frame searches, predicts
 * from and reconstructs against the deblocked reconstruction of the frame
 * before it, as the reference searches RefFrames built from its
 * reconstructed planes (encoder/src/lib.rs:228-262; luma reconstruction
 * mb16.rs:3575-3605, chroma mb16.rs:3606-3628, deblock.rs filter_frame with
 * zero offsets).  Frame 0 reconstructs to itself (coded losslessly in this
 * frame model); frames 1..n-1 run plain-ME (or, with a net, the learned
 * search: the proposals of every frame come first, in one batched pass over
 * the source pairs (f, f-1) with guide MVs from the HalfRes lookahead, and
 * the search prices them on the reconstruction),
 * MC + T/Q and reconstruction of luma and chroma, and deblocking.  Each
 * frame's MBs run as a wavefront, and consecutive frames overlap in one
 * launch: an MB of frame f waits only for the segments (16 rows by 16 MB
 * columns) of rec(f-1) its search reads, whose planes are built as those
 * MBs are deblocked, so about ten frames run at once.  From host buffers the
 * sources of frames 1.. are uploaded beside the launch and each frame's
 * outputs come down as it becomes final.
 * Inputs: n frames of luma
 * (cw x ch) and chroma (cw/2 x ch/2), contiguous, host memory.  Outputs per
 * frame (frame 0 rows zero): picks 6 i32/MB, costs 2 i64/MB, luma levels 256
 * i16/MB, chroma levels 128 i16/MB (as h264a_mc_tq_chroma_frames), the
 * reconstruction, and with a net its proposals (16 i32/MB) and fallback flags
 * (1 i32/MB); all but picks and costs optional.  Synchronous. */
typedef struct {
    const uint8_t *h_y, *h_u, *h_v;
    int32_t n, cw, ch;
    double lambda_me;
    int64_t split_gate;
    int32_t qp, dz_div;
    h264a_mvnet *net;            /* NULL: plain search */
    int32_t fallback_t;
    int32_t *h_picks;
    int64_t *h_costs;
    int16_t *h_coeffs, *h_ccoeffs;
    uint8_t *h_rec_y, *h_rec_u, *h_rec_v;
    int32_t *h_props, *h_fallback;
} h264a_closed_job;
H264A_API int h264a_pixel_path_closed(h264a_ctx *ctx, const h264a_closed_job *job, const h264a_me_params *params,
                                      const uint16_t *h_mv_cost_tab);
/* The same loop on device buffers, enqueued on `stream` (no allocation, no
 * host copy): the caller passes the n source frames, room for their
 * reconstruction (frame 0 is copied from the source), the planes of
 * min(n, H264A_CLOSED_PLANE_PICTURES) pictures as scratch (4*(cw+64)*(ch+64)
 * bytes each: the loop overlaps many consecutive frames, each building its
 * reconstruction's planes segment by segment while later frames search the
 * finished segments), the outputs (levels 16-byte aligned,
 * chroma 4-byte aligned), and with a net the proposals buffer (16 i32/MB per
 * frame), optional fallback flags and the guide MVs (2 i32/MB per frame, the
 * lookahead's, or NULL). */
#define H264A_CLOSED_PLANE_PICTURES 16
typedef struct {
    const uint8_t *d_y, *d_u, *d_v;
    uint8_t *d_rec_y, *d_rec_u, *d_rec_v;
    uint8_t *d_planes;
    int32_t n, cw, ch;
    double lambda_me;
    int64_t split_gate;
    int32_t qp, dz_div;
    h264a_mvnet *net;
    int32_t fallback_t;
    const int32_t *d_guide_mvs;
    int32_t *d_picks;
    int64_t *d_costs;
    int16_t *d_coeffs, *d_ccoeffs;
    int32_t *d_props, *d_fallback;
} h264a_closed_dev;
H264A_API int h264a_closed_frames(h264a_ctx *ctx, const h264a_closed_dev *job, const h264a_me_params *params,
                                  void *stream);
/* One P frame of that loop, the encoder's per-frame call (encode_frame's
 * motion search, mb16.rs inter MB coding and reconstruction, then
 * deblock.rs filter_frame on the picture): frame f's search on the planes
 * of rec(f-1) (me.pic: the source luma and those planes, built by
 * h264a_hpel_build), and in the same launch each MB's MC + T/Q and
 * reconstruction of luma and chroma and the in-loop deblocking of the
 * picture, written to d_rec_y/u/v.  d_ref_u/v: the chroma reconstruction of
 * frame f-1.  Levels as h264a_closed_frames' (16-byte aligned), planes 4-byte
 * aligned.  d_props non-NULL: the learned 16x16 search with those proposals
 * (16 i32/MB), fallback_t and optional d_fallback as h264a_me_frames_learned.
 * Enqueued on `stream`; one kernel launch. */
typedef struct {
    h264a_me_frame me;
    const uint8_t *d_u, *d_v;
    const uint8_t *d_ref_u, *d_ref_v;
    uint8_t *d_rec_y, *d_rec_u, *d_rec_v;
    int16_t *d_coeffs, *d_ccoeffs;
    int32_t qp, dz_div;
    const int32_t *d_props;
    int32_t *d_fallback;
    int32_t fallback_t;
} h264a_closed_step;
H264A_API int h264a_closed_step_frame(h264a_ctx *ctx, const h264a_closed_step *step, const h264a_me_params *params,
                                      void *stream);

/* ---- Annex-B output of the frame model (host) ---------------------------------- */
/* A decodable H.264 Baseline stream (CAVLC) of n frames of the frame model:
 * SPS, PPS, frame 0 as an IDR picture of I_PCM macroblocks (its lossless
 * reconstruction is the source frame), frames 1..n-1 as P pictures, one slice
 * each, every MB coded (mb_skip_run 0) as P_L0_16x16 / P_L0_L0_16x8 /
 * P_L0_L0_8x16 per its pick with reference 0, its MVs against the standard's
 * MV predictor, its levels (h264a_mc_tq_rec_frames' 256 luma levels and
 * h264a_mc_tq_chroma_frames' 128 chroma levels per MB) as CAVLC residual
 * blocks at the picture's QP.  Syntax after the reference's writer: CAVLC P
 * slices (encoder/src/mb16.rs:5266-5845), residual blocks
 * (common/src/cavlc.rs:485), parameter sets and NAL framing
 * (common/src/nal.rs).  width/height: display size (even, cropped from the
 * MB-aligned coded size).  With h_out NULL only *out_len is computed;
 * h_frame_bytes (optional, n entries) receives each frame's bytes (frame 0
 * with the parameter sets).  Host only, no GPU needed. */
typedef struct {
    int32_t width, height, cw, ch, n, qp;
    const uint8_t *h_y0, *h_u0, *h_v0;  /* frame 0 (cw x ch, cw/2 x ch/2) */
    const int32_t *h_picks;             /* n x nmb x 6 (frame 0 unused) */
    const int16_t *h_coeffs;            /* n x nmb x 256 */
    const int16_t *h_ccoeffs;           /* n x nmb x 128 */
} h264a_stream_frames;
H264A_API int h264a_write_stream_cavlc(const h264a_stream_frames *in, uint8_t *h_out, size_t cap, size_t *out_len,
                                       int64_t *h_frame_bytes);
/* The writer's VLC tables, for checking against the standard's: table 0
 * coeff_token (nC class i 0..2, TotalCoeff j, TrailingOnes k), 1 chroma-DC
 * coeff_token (j, k), 2 total_zeros (TotalCoeff j 1..15, total_zeros k),
 * 3 chroma-DC total_zeros, 4 run_before (min(zerosLeft,7) j, run k), 5 the
 * inter coded_block_pattern j -> codeNum (in *bits). */
H264A_API int h264a_cavlc_table_code(int table, int i, int j, int k, int *len, int *bits);

/* ---- diagnostics ----------------------------------------------------------- */
/* Failure-detection self-test: one warp runs the persistent kernel's bounded
 * wait on a flag that nothing sets, giving up after spin_limit polls.  The next
 * h264a_sync on `stream` then returns H264A_E_TIMEOUT and the context stays
 * usable.  No counterpart in the reference (it has no device waits). */
H264A_API int h264a_selftest_bounded_wait(h264a_ctx *ctx, int spin_limit, void *stream);
/* Measures the device's INT32 issue rate (three-input adds, lane instructions
 * per second / 1e9) with a short independent-chain kernel: the roofline
 * denominator of the SAD/SATD kernels.  Synchronous; no reference counterpart. */
H264A_API int h264a_measure_int32_peak(h264a_ctx *ctx, double *gops_out);

#ifdef __cplusplus
}
#endif
#endif /* H264ACCEL_H */
