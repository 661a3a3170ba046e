/*
 * h264_oracle.h -- CPU restatement of rusty_h264's encoder pixel hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * rusty_h264_b200: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg may load it.  The product never calls it.
 *
 * Every function restates one function of the Rust reference
 * (Remade-With-Rust/rusty_h264) and cites the file:line it follows.  Paths are
 * relative to the reference project root.
 *
 * Parity pin: the primitive functions are pinned by the known-answer and
 * differential tests the reference holds (ported in tests/test_oracle_*.py
 * and tests/golden/reference_known_answers.json).  motion_search and the
 * lookahead search have no golden vector in the reference; their restatement
 * is pinned only through the primitives they are built from.
 */
#ifndef H264_ORACLE_H
#define H264_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- SATD / SAD family (crates/rusty_h264-accel/src/satd_sad.rs) ---------- */
int32_t or_satd4x4_wels(const uint8_t *a, int sa, const uint8_t *b, int sb);
int32_t or_satd_region_wels(const uint8_t *a, int sa, const uint8_t *b, int sb, int w, int h);
int32_t or_sad(const uint8_t *a, int sa, const uint8_t *b, int sb, int w, int h);
/* Σ|H·d| over the 4x4 blocks of a w×h region (mb16.rs:6027 satd_px scalar arm) */
int64_t or_satd_px(const uint8_t *src, int ss, const uint8_t *pred, int ps, int w, int h);
/* fused (a+b+1)>>1 average + SATD (accel/src/satd_avg.rs:579) */
uint32_t or_satd_avg(const uint8_t *src, int ss, const uint8_t *a, const uint8_t *b, int stride, int w, int h);
/* fused average + SAD (encoder mb16.rs:6104 sad_avg_strided) */
int64_t or_sad_avg(const uint8_t *src, int ss, const uint8_t *a, const uint8_t *b, int stride, int w, int h);

/* ---- transform / quant (crates/rusty_h264-common/src/transform.rs) -------- */
void or_forward_core(const int32_t in[16], int32_t out[16]);
void or_hadamard_4x4(const int32_t in[16], int32_t out[16]);
void or_quant_dz_ff(int qp, int64_t dz_div, int16_t ff[8]);
void or_quant_mf_oh(int qp, int16_t mf[8]);
void or_quantize(const int32_t c[16], int qp, int64_t dz_div, int32_t out[16]);
void or_forward_core_8x8(const int32_t in[64], int32_t out[64]);
void or_quantize_8x8(const int32_t c[64], int qp, const int32_t weight[64], int64_t dz_div, int32_t out[64]);
/* accel/src/transform_quant.rs */
void or_dct_four_t4(int16_t dct[64], const uint8_t *src, int ss, const uint8_t *pred, int ps);
void or_quant_four_4x4(int16_t dct[64], const int16_t ff[8], const int16_t mf[8]);
/* one macroblock's luma T/Q exactly as mb16.rs:3436-3450 runs it */
void or_mb_luma_tq(const uint8_t *src, int ss, const uint8_t *pred16, int qp, int dz_div, int16_t out[256]);
void or_dequant4x4(const int32_t lv[16], int qp, int32_t out[16]);
void or_inverse_core4(int32_t m[16]);
void or_idct_four_t4_rec(uint8_t *rec, int srec, const uint8_t *pred, int spred, const int16_t dct[64]);
void or_mb_luma_rec(uint8_t *rec, int srec, const uint8_t *pred16, const int16_t levels[256], int qp);
int or_chroma_qp(int qp);
void or_forward_quant_chroma_dc(const int32_t dc[4], int qp, int intra, int32_t out[4]);
void or_inverse_quant_chroma_dc(const int32_t levels[4], int qp, int32_t out[4]);
void or_mc_chroma(const uint8_t *ref, int cw, int ch, int x0, int y0, int bw, int bh, int32_t mvx, int32_t mvy,
                  uint8_t *out);

/* ---- inter prediction (crates/rusty_h264-common/src/inter.rs) ------------- */
int32_t or_median3(int32_t a, int32_t b, int32_t c);
typedef struct { int32_t available; int32_t mvx, mvy; int32_t ref_idx; } or_mv_neighbor;
void or_predict_mv(const or_mv_neighbor *a, const or_mv_neighbor *b, const or_mv_neighbor *c, int cur_ref, int32_t out[2]);
void or_predict_partition_mv(int mode, int part, const or_mv_neighbor *a, const or_mv_neighbor *b,
                             const or_mv_neighbor *c, int cur_ref, int32_t out[2]);
int32_t or_luma_sample(const uint8_t *ref, int cw, int ch, int ix, int iy, int fx, int fy);
void or_mc_luma(const uint8_t *ref, int cw, int ch, int x0, int y0, int bw, int bh, int mvx, int mvy, uint8_t *out);
void or_pad_plane(const uint8_t *src, int w, int h, int pad, uint8_t *f);
void or_hpel_fused(const uint8_t *f, int pw, int ph, uint8_t *h, uint8_t *v, uint8_t *c);
void or_hpel_tiles(const uint8_t *f, int pw, int ph, uint8_t *h, uint8_t *v, uint8_t *c);

typedef struct {
    const uint8_t *f, *h, *v, *c; /* each pw×ph, stride pw */
    int pw, ph, pad, cw, ch;
} or_hpel_planes;
/* builds planes into caller buffers (each pw*ph bytes) -- inter.rs:816 */
void or_build_hpel_planes(const uint8_t *ref, int cw, int ch, int pad, uint8_t *f, uint8_t *h, uint8_t *v, uint8_t *c);
/* returns 1 and fills (plane index 0..3, base) or 0 -- inter.rs:1015 */
int or_hpel_ref(const or_hpel_planes *p, int x0, int y0, int bw, int bh, int mvx, int mvy, int *plane, int64_t *base);
int or_hpel_qpel_refs(const or_hpel_planes *p, int x0, int y0, int bw, int bh, int mvx, int mvy,
                      int *pa, int64_t *oa, int *pb, int64_t *ob);
int or_hpel_block(const or_hpel_planes *p, int x0, int y0, int bw, int bh, int mvx, int mvy, uint8_t *out);

/* ---- motion search (crates/rusty_h264-encoder/src/mb16.rs) ----------------- */
typedef struct {
    const uint8_t *src; /* coded source luma, stride cw */
    const uint8_t *ref; /* reference luma cw×ch */
    or_hpel_planes planes;
    int cw, ch;         /* ch = mb_h * 16 */
} or_me_frame;

typedef struct {
    int32_t fast;            /* Preset::Fast (SAD cost, no planes) */
    int32_t mb_use_satd;     /* fast-preset SATD override */
    int32_t sadfp;           /* B2: SAD-domain full-pel phase */
    int32_t mv_cost_kind;    /* 0 Exp-Golomb, 1 smooth table, 2 measured table */
    const uint16_t *mv_cost_tab; /* 4096 entries for kinds 1/2 */
    double sadfp_lambda;     /* RFF_ME_SADL (0.5) */
    int32_t me_snap;         /* tune_me_snap (1) */
    int32_t me_fc;           /* fixed-centre diamond (accel build default 1) */
    uint32_t dia_mask;       /* rungs of [64,32,16,8,4] (0b11100) */
    uint32_t dia_sub_mask;   /* sub-8x8 rungs (0b10000) */
    int32_t subpel;          /* run the [2,1] sub-pel steps */
    int32_t subpel_pat;      /* -1: preset default; 0..3 override */
    int32_t sp_single_pass;  /* Balanced */
    int32_t sub_pat;         /* RFF_SUBPEL_SUB (2) */
    int32_t me_subpel_iter;  /* tune_me_subpel_iter (1) */
    int32_t sp_maxit;        /* 0 = unlimited */
    int32_t sp_fc;           /* batched sub-pel rings (0) */
} or_me_params;

typedef struct { int32_t mvx, mvy; int64_t cost; int32_t evals; } or_me_result;

/* mvbits of one mvd component (mb16.rs:2454-2482) */
uint32_t or_mvbits(int kind, const uint16_t *tab, int32_t d);
/* smooth table (mb16.rs:508 build_mv_cost) */
void or_build_mv_cost(uint16_t out[4096]);
/* distortion of one candidate exactly as mc_satd_hp / mc_sad_hp / mc_sad dispatch */
int64_t or_mc_satd_hp(const or_me_frame *fr, int use_planes, int lx, int ly, int rw, int rh, int mvx, int mvy);
int64_t or_mc_sad_hp(const or_me_frame *fr, int use_planes, int lx, int ly, int rw, int rh, int mvx, int mvy);
/* motion_search (mb16.rs:2433-3302); start==NULL for a full search */
void or_motion_search(const or_me_frame *fr, const or_me_params *pr, int lx, int ly, int rw, int rh,
                      const int32_t *preds, int npred, double lambda_me, const int32_t *start, or_me_result *out);

/* Plain-ME frame model: every MB runs best_part(16x16) (and, when split_gate>=0,
 * the 16x8/8x16 partitions) in raster order, neighbours' picks feeding the
 * median predictor (mb16.rs:1871 mv_neighbors_block, inter.rs:36 predict_mv). */
typedef struct { int32_t shape; int32_t mv[2][2]; int64_t cost; int64_t cost16; int32_t mv16[2]; } or_mb_pick;
void or_me_frame_plain(const or_me_frame *fr, const or_me_params *pr, double lambda_me,
                       int64_t split_gate, or_mb_pick *out /* mb_w*mb_h */);
void or_me_frame_learned(const or_me_frame *fr, const or_me_params *pr, double lambda_me, int64_t split_gate,
                         const int32_t *props, int32_t prop_t, or_mb_pick *out, int32_t *fell);
/* the plain-ME frame model over nref references (frs[r]: the same source, the
 * planes of reference r; reference 0 the nearest) */
typedef struct { int32_t shape; int32_t ref[2]; int32_t mv[2][2]; int64_t cost; int64_t cost16; } or_mb_pick_mr;
void or_me_frame_multiref(const or_me_frame *frs, int nref, const or_me_params *pr, double lambda_me,
                          int64_t split_gate, or_mb_pick_mr *out);
/* in-loop deblocking of a plain-ME P picture (h264_oracle_par.c) */
void or_deblock_frame_plain(uint8_t *y, uint8_t *u, uint8_t *v, int cw, int ch, const int32_t *picks,
                            const int16_t *coeffs, int qp, int offset_a, int offset_b, int chroma_qp_offset);

/* Exhaustive full-pel grid over ±R around each MB (16x16 SAD and SATD), the
 * ME-oracle-probe order (mb16.rs:2889-2900: dy outer, dx inner, strict <). */
void or_fullpel_grid_mb(const or_me_frame *fr, int mbx, int mby, int R, int32_t *sad_grid, int32_t *satd_grid);

/* ---- mb-tree lookahead (crates/rusty_h264-encoder/src/mbtree.rs) ---------- */
void or_downsample2x(const uint8_t *y, int cw, int ch, uint8_t *out);
int32_t or_intra_cost(const uint8_t *sy, int cw, int bx0, int by0, int bs);
int64_t or_la_mc_satd(const uint8_t *sy, int cw, int ch, const uint8_t *ref, int bx0, int by0, int bs, int mvx, int mvy);
void or_inter_cost(const uint8_t *sy, int cw, int ch, const uint8_t *ref, int bx0, int by0, int bs,
                   int seedx, int seedy, int max_step, int32_t *cost, int32_t mv[2], int32_t *evals);
/* mode: 0 FullRes, 1 Hybrid, 2 HalfRes.  ref_* NULL for the IDR. */
void or_frame_costs(const uint8_t *full, int cwf, int chf, const uint8_t *half, int cwh, int chh,
                    int mb_w, int mb_h, const uint8_t *ref_full, const uint8_t *ref_half, int mode,
                    int32_t *intra, int32_t *inter, int32_t *mvs /* 2 per MB */);

#ifdef __cplusplus
}
#endif
#endif
