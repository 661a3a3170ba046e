/*
 * h264_oracle_par.c -- whole-clip driver of the CPU oracle (test
 * infrastructure and the timed CPU baseline only).
 *
 * It runs, per P frame f (reference = source frame f-1, the source-domain
 * reference the mb-tree lookahead also uses, mbtree.rs:431-434):
 *   planes  = build_hpel_planes(Y[f-1])                       inter.rs:816
 *   picks   = plain-ME frame model (best_part per MB)         mb16.rs:4921
 *   coeffs  = MC of each pick + luma T/Q at qp                mb16.rs:3436-3450
 * and, over the whole clip, the HalfRes lookahead
 *   half    = downsample2x(Y[f]);  costs = frame_costs(...)   mbtree.rs:61, 208
 * Frames are independent, so the driver shards them over threads the
 * way encode_all shards GOPs over std::thread (lib.rs:745-805), on POSIX
 * threads.
 */
#include "h264_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

/* A minimal dynamic parallel-for over [0, n) on POSIX threads. */
typedef struct {
    void (*fn)(void *arg, int i, int tid);
    void *arg;
    int n, tid;
    volatile int *next;
    pthread_mutex_t *mu;
} par_worker;

static void *par_main(void *p) {
    par_worker *w = (par_worker *)p;
    for (;;) {
        pthread_mutex_lock(w->mu);
        int i = (*w->next)++;
        pthread_mutex_unlock(w->mu);
        if (i >= w->n) break;
        w->fn(w->arg, i, w->tid);
    }
    return NULL;
}

static void par_for(int n, int nthreads, void (*fn)(void *, int, int), void *arg) {
    if (nthreads < 1) nthreads = 1;
    if (nthreads > n) nthreads = n > 0 ? n : 1;
    volatile int next = 0;
    pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
    pthread_t th[256];
    par_worker w[256];
    if (nthreads > 256) nthreads = 256;
    for (int t = 0; t < nthreads; t++) {
        w[t].fn = fn; w[t].arg = arg; w[t].n = n; w[t].tid = t; w[t].next = &next; w[t].mu = &mu;
    }
    for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, par_main, &w[t]);
    par_main(&w[0]);
    for (int t = 1; t < nthreads; t++) pthread_join(th[t], NULL);
}

typedef struct {
    int32_t fast, mb_use_satd, sadfp, mv_cost_kind;
    double sadfp_lambda;
    int32_t me_snap, me_fc;
    uint32_t dia_mask, dia_sub_mask;
    int32_t subpel, subpel_pat, sp_single_pass, sub_pat, me_subpel_iter, sp_maxit, sp_fc;
} or_me_params_flat;

static void unflatten(const or_me_params_flat *f, const uint16_t *tab, or_me_params *p) {
    p->fast = f->fast; p->mb_use_satd = f->mb_use_satd; p->sadfp = f->sadfp; p->mv_cost_kind = f->mv_cost_kind;
    p->mv_cost_tab = tab; p->sadfp_lambda = f->sadfp_lambda; p->me_snap = f->me_snap; p->me_fc = f->me_fc;
    p->dia_mask = f->dia_mask; p->dia_sub_mask = f->dia_sub_mask; p->subpel = f->subpel;
    p->subpel_pat = f->subpel_pat; p->sp_single_pass = f->sp_single_pass; p->sub_pat = f->sub_pat;
    p->me_subpel_iter = f->me_subpel_iter; p->sp_maxit = f->sp_maxit; p->sp_fc = f->sp_fc;
}

int or_num_threads(void) {
    long n = sysconf(_SC_NPROCESSORS_ONLN);
    return n > 0 ? (int)n : 1;
}

/* ctypes-friendly motion_search entry (the params struct passed flat). */
void or_motion_search_flat(const uint8_t *src, const uint8_t *ref, const uint8_t *planes4, int cw, int ch, int pad,
                           const or_me_params_flat *pf, const uint16_t *tab, int lx, int ly, int rw, int rh,
                           const int32_t *preds, int npred, double lambda_me, const int32_t *start, int32_t *out_mv,
                           int64_t *out_cost, int32_t *out_evals) {
    int pw = cw + 2 * pad, ph = ch + 2 * pad;
    size_t ps = (size_t)pw * ph;
    or_me_frame fr;
    fr.src = src; fr.ref = ref; fr.cw = cw; fr.ch = ch;
    fr.planes.f = planes4; fr.planes.h = planes4 + ps; fr.planes.v = planes4 + 2 * ps; fr.planes.c = planes4 + 3 * ps;
    fr.planes.pw = pw; fr.planes.ph = ph; fr.planes.pad = pad; fr.planes.cw = cw; fr.planes.ch = ch;
    or_me_params p;
    unflatten(pf, tab, &p);
    or_me_result r;
    or_motion_search(&fr, &p, lx, ly, rw, rh, preds, npred, lambda_me, start, &r);
    out_mv[0] = r.mvx; out_mv[1] = r.mvy;
    *out_cost = r.cost;
    if (out_evals) *out_evals = r.evals;
}

/* ctypes-friendly distortion of one candidate: kind 0 = SATD (mc_satd_hp), 1 = SAD. */
int64_t or_candidate_dist(const uint8_t *src, const uint8_t *ref, const uint8_t *planes4, int cw, int ch, int pad,
                          int kind, int lx, int ly, int rw, int rh, int mvx, int mvy) {
    int pw = cw + 2 * pad, ph = ch + 2 * pad;
    size_t ps = (size_t)pw * ph;
    or_me_frame fr;
    fr.src = src; fr.ref = ref; fr.cw = cw; fr.ch = ch;
    fr.planes.f = planes4; fr.planes.h = planes4 + ps; fr.planes.v = planes4 + 2 * ps; fr.planes.c = planes4 + 3 * ps;
    fr.planes.pw = pw; fr.planes.ph = ph; fr.planes.pad = pad; fr.planes.cw = cw; fr.planes.ch = ch;
    return kind == 0 ? or_mc_satd_hp(&fr, 1, lx, ly, rw, rh, mvx, mvy) : or_mc_sad_hp(&fr, 1, lx, ly, rw, rh, mvx, mvy);
}

/* Builds pad + H/V/C into one buffer laid out F|H|V|C (each pw*ph). */
void or_build_planes4(const uint8_t *ref, int cw, int ch, int pad, uint8_t *planes4) {
    int pw = cw + 2 * pad, ph = ch + 2 * pad;
    size_t ps = (size_t)pw * ph;
    or_build_hpel_planes(ref, cw, ch, pad, planes4, planes4 + ps, planes4 + 2 * ps, planes4 + 3 * ps);
}

/* Plain-ME frame model over one (src, ref) pair; picks written flat:
 * per MB {shape, mv0x, mv0y, mv1x, mv1y, cost_lo, cost_hi, evals-unused}. */
void or_me_frame_learned_flat(const uint8_t *src, const uint8_t *ref, const uint8_t *planes4, int cw, int ch, int pad,
                              const or_me_params_flat *pf, const uint16_t *tab, double lambda_me, int64_t split_gate,
                              const int32_t *props, int32_t prop_t, int32_t *picks, int64_t *costs, int32_t *fell);

void or_me_frame_flat(const uint8_t *src, const uint8_t *ref, const uint8_t *planes4, int cw, int ch, int pad,
                      const or_me_params_flat *pf, const uint16_t *tab, double lambda_me, int64_t split_gate,
                      int32_t *picks /* 6 per MB */, int64_t *costs /* 2 per MB: pick, 16x16 */) {
    or_me_frame_learned_flat(src, ref, planes4, cw, ch, pad, pf, tab, lambda_me, split_gate, NULL, 0, picks, costs,
                             NULL);
}

/* or_me_frame_multiref on flat buffers: nref reference pictures refs
 * (cw*ch each, contiguous) and their planes (4*pw*ph each); picks 8 i32 per
 * MB (shape, ref0, mv0x, mv0y, ref1, mv1x, mv1y, 0), costs 2 i64 per MB. */
void or_me_frame_multiref_flat(const uint8_t *src, const uint8_t *refs, const uint8_t *planes, int nref, int cw,
                               int ch, int pad, const or_me_params_flat *pf, const uint16_t *tab, double lambda_me,
                               int64_t split_gate, int32_t *picks, int64_t *costs) {
    int pw = cw + 2 * pad, ph = ch + 2 * pad;
    size_t ps = (size_t)pw * ph;
    or_me_frame frs[8];
    if (nref < 1 || nref > 8) return;
    for (int r = 0; r < nref; r++) {
        const uint8_t *pl = planes + 4 * ps * r;
        or_me_frame *fr = &frs[r];
        fr->src = src; fr->ref = refs + (size_t)cw * ch * r; fr->cw = cw; fr->ch = ch;
        fr->planes.f = pl; fr->planes.h = pl + ps; fr->planes.v = pl + 2 * ps; fr->planes.c = pl + 3 * ps;
        fr->planes.pw = pw; fr->planes.ph = ph; fr->planes.pad = pad; fr->planes.cw = cw; fr->planes.ch = ch;
    }
    or_me_params p;
    unflatten(pf, tab, &p);
    int nmb = (cw / 16) * (ch / 16);
    or_mb_pick_mr *pk = (or_mb_pick_mr *)malloc(sizeof(or_mb_pick_mr) * (size_t)nmb);
    or_me_frame_multiref(frs, nref, &p, lambda_me, split_gate, pk);
    for (int m = 0; m < nmb; m++) {
        int32_t *o = picks + 8 * m;
        o[0] = pk[m].shape;
        o[1] = pk[m].ref[0]; o[2] = pk[m].mv[0][0]; o[3] = pk[m].mv[0][1];
        o[4] = pk[m].ref[1]; o[5] = pk[m].mv[1][0]; o[6] = pk[m].mv[1][1];
        o[7] = 0;
        costs[2 * m] = pk[m].cost;
        costs[2 * m + 1] = pk[m].cost16;
    }
    free(pk);
}

/* or_me_frame_flat with the learned 16x16 search (props: 16 i32 per MB, NULL
 * for the plain search); fell (optional): the fallback flag per MB. */
void or_me_frame_learned_flat(const uint8_t *src, const uint8_t *ref, const uint8_t *planes4, int cw, int ch, int pad,
                              const or_me_params_flat *pf, const uint16_t *tab, double lambda_me, int64_t split_gate,
                              const int32_t *props, int32_t prop_t, int32_t *picks, int64_t *costs, int32_t *fell) {
    int pw = cw + 2 * pad, ph = ch + 2 * pad;
    size_t ps = (size_t)pw * ph;
    or_me_frame fr;
    fr.src = src; fr.ref = ref; fr.cw = cw; fr.ch = ch;
    fr.planes.f = planes4; fr.planes.h = planes4 + ps; fr.planes.v = planes4 + 2 * ps; fr.planes.c = planes4 + 3 * ps;
    fr.planes.pw = pw; fr.planes.ph = ph; fr.planes.pad = pad; fr.planes.cw = cw; fr.planes.ch = ch;
    or_me_params p;
    unflatten(pf, tab, &p);
    int nmb = (cw / 16) * (ch / 16);
    or_mb_pick *pk = (or_mb_pick *)malloc(sizeof(or_mb_pick) * nmb);
    or_me_frame_learned(&fr, &p, lambda_me, split_gate, props, prop_t, pk, fell);
    for (int i = 0; i < nmb; i++) {
        picks[6 * i + 0] = pk[i].shape;
        picks[6 * i + 1] = pk[i].mv[0][0];
        picks[6 * i + 2] = pk[i].mv[0][1];
        picks[6 * i + 3] = pk[i].mv[1][0];
        picks[6 * i + 4] = pk[i].mv[1][1];
        picks[6 * i + 5] = 0;
        costs[2 * i] = pk[i].cost;
        costs[2 * i + 1] = pk[i].cost16;
    }
    free(pk);
}

/* Motion-compensated luma prediction of one MB for a pick (16x16 or the two
 * 16x8 / 8x16 partitions), through mc_luma (inter.rs:1193). */
static void mb_pred_for_pick(const uint8_t *ref, int cw, int ch, int mbx, int mby, const int32_t *pick, uint8_t pred[256]) {
    int shape = pick[0];
    uint8_t part[256];
    if (shape == 0) {
        or_mc_luma(ref, cw, ch, mbx * 16, mby * 16, 16, 16, pick[1], pick[2], pred);
        return;
    }
    for (int k = 0; k < 2; k++) {
        int ox = shape == 2 ? 8 * k : 0, oy = shape == 1 ? 8 * k : 0;
        int bw = shape == 2 ? 8 : 16, bh = shape == 1 ? 8 : 16;
        or_mc_luma(ref, cw, ch, mbx * 16 + ox, mby * 16 + oy, bw, bh, pick[1 + 2 * k], pick[2 + 2 * k], part);
        for (int r = 0; r < bh; r++) memcpy(pred + (oy + r) * 16 + ox, part + r * bw, bw);
    }
}

/* MC + luma T/Q of every MB of one frame from its picks. */
void or_mc_tq_frame(const uint8_t *src, const uint8_t *ref, int cw, int ch, const int32_t *picks, int qp, int dz_div,
                    int16_t *coeffs /* 256 per MB */) {
    int mb_w = cw / 16, mb_h = ch / 16;
    for (int mby = 0; mby < mb_h; mby++)
        for (int mbx = 0; mbx < mb_w; mbx++) {
            int m = mby * mb_w + mbx;
            uint8_t pred[256];
            mb_pred_for_pick(ref, cw, ch, mbx, mby, picks + 6 * m, pred);
            or_mb_luma_tq(src + (int64_t)mby * 16 * cw + mbx * 16, cw, pred, qp, dz_div, coeffs + (int64_t)m * 256);
        }
}

/* MC + luma T/Q and the luma reconstruction of every MB of a frame
 * (mb16.rs:3436-3450 and 3575-3605): coeffs as or_mc_tq_frame, rec cw x ch. */
void or_mc_tq_rec_frame(const uint8_t *src, const uint8_t *ref, int cw, int ch, const int32_t *picks, int qp,
                        int dz_div, int16_t *coeffs, uint8_t *rec) {
    int mb_w = cw / 16, mb_h = ch / 16;
    for (int mby = 0; mby < mb_h; mby++)
        for (int mbx = 0; mbx < mb_w; mbx++) {
            int m = mby * mb_w + mbx;
            uint8_t pred[256];
            mb_pred_for_pick(ref, cw, ch, mbx, mby, picks + 6 * m, pred);
            or_mb_luma_tq(src + (int64_t)mby * 16 * cw + mbx * 16, cw, pred, qp, dz_div, coeffs + (int64_t)m * 256);
            or_mb_luma_rec(rec + (int64_t)mby * 16 * cw + mbx * 16, cw, pred, coeffs + (int64_t)m * 256, qp);
        }
}

/* The inter MB's chroma of mb16.rs:3408-3428, 3465-3500 and 3606-3628, per
 * MB: mc_chroma of each partition with the luma MV, per plane dct_four_t4 +
 * quant_four_4x4 at chroma_qp(qp) with the AC levels kept and slot 0 taken by
 * the block's DC (the 2x2 forward_quant_chroma_dc level, inter dead-zone);
 * reconstruction: dequantize of the AC levels, the DC replaced by
 * inverse_quant_chroma_dc (both cast to i16), idct_four_t4_rec onto the
 * prediction.  coeffs: 128 i16 per MB (U then V, SUBBLOCKS order, 16 each);
 * rec_u / rec_v may be NULL. */
void or_mc_tq_chroma_frame(const uint8_t *src_u, const uint8_t *src_v, const uint8_t *ref_u, const uint8_t *ref_v,
                           int cw, int ch, const int32_t *picks, int qp, int16_t *coeffs, uint8_t *rec_u,
                           uint8_t *rec_v) {
    int mb_w = cw / 16, mb_h = ch / 16, ccw = cw / 2, cch = ch / 2;
    int qpc = or_chroma_qp(qp);
    int16_t ff[8], mf[8];
    or_quant_dz_ff(qpc, 6, ff);
    or_quant_mf_oh(qpc, mf);
    for (int mby = 0; mby < mb_h; mby++)
        for (int mbx = 0; mbx < mb_w; mbx++) {
            int m = mby * mb_w + mbx;
            const int32_t *pk = picks + 6 * m;
            for (int c = 0; c < 2; c++) {
                const uint8_t *rf = c == 0 ? ref_u : ref_v, *sc = c == 0 ? src_u : src_v;
                uint8_t pred[64];
                int shape = pk[0];
                if (shape == 0) {
                    or_mc_chroma(rf, ccw, cch, mbx * 8, mby * 8, 8, 8, pk[1], pk[2], pred);
                } else {
                    for (int k = 0; k < 2; k++) {
                        int ox = shape == 2 ? 4 * k : 0, oy = shape == 1 ? 4 * k : 0;
                        int bw = shape == 2 ? 4 : 8, bh = shape == 1 ? 4 : 8;
                        uint8_t t[64];
                        or_mc_chroma(rf, ccw, cch, mbx * 8 + ox, mby * 8 + oy, bw, bh, pk[1 + 2 * k], pk[2 + 2 * k], t);
                        for (int r = 0; r < bh; r++) memcpy(pred + (oy + r) * 8 + ox, t + r * bw, bw);
                    }
                }
                int16_t cd[64];
                const uint8_t *s8 = sc + (int64_t)mby * 8 * ccw + mbx * 8;
                or_dct_four_t4(cd, s8, ccw, pred, 8);
                int32_t dc[4] = {cd[0], cd[16], cd[32], cd[48]};
                or_quant_four_4x4(cd, ff, mf);
                int32_t dl[4], rdc[4];
                or_forward_quant_chroma_dc(dc, qpc, 0, dl);
                or_inverse_quant_chroma_dc(dl, qpc, rdc);
                int16_t *out = coeffs + (int64_t)m * 128 + c * 64;
                for (int i = 0; i < 4; i++) {
                    out[i * 16] = (int16_t)dl[i];
                    for (int j = 1; j < 16; j++) out[i * 16 + j] = cd[i * 16 + j];
                }
                uint8_t *rp = c == 0 ? rec_u : rec_v;
                if (rp) {
                    int16_t d[64];
                    for (int i = 0; i < 4; i++) {
                        int32_t lv[16], dq[16];
                        lv[0] = 0;
                        for (int j = 1; j < 16; j++) lv[j] = cd[i * 16 + j];
                        or_dequant4x4(lv, qpc, dq);
                        for (int j = 0; j < 16; j++) d[i * 16 + j] = (int16_t)dq[j];
                        d[i * 16] = (int16_t)rdc[i];
                    }
                    or_idct_four_t4_rec(rp + (int64_t)mby * 8 * ccw + mbx * 8, ccw, pred, 8, d);
                }
            }
        }
}

/* ---- in-loop deblocking of a plain-ME P picture ---------------------------
 * crates/rusty_h264-common/src/deblock.rs, restated for the pictures this path
 * produces: every MB inter with reference 0, 4x4 transforms (no t8x8), one QP.
 * Spec Tables 8-16/8-17 (deblock.rs:11-41): alpha, beta by indexA/indexB,
 * tc0 by [indexA][bS-1]. */
static const int DB_ALPHA[52] = {0,  0,  0,  0,  0,  0,  0,  0,  0,  0,   0,   0,   0,   0,   0,   0,   4,   4,
                                 5,  6,  7,  8,  9,  10, 12, 13, 15, 17,  20,  22,  25,  28,  32,  36,  40,  45,
                                 50, 56, 63, 71, 80, 90, 101, 113, 127, 144, 162, 182, 203, 226, 255, 255};
static const int DB_BETA[52] = {0, 0, 0, 0, 0, 0, 0, 0,  0,  0,  0,  0,  0,  0,  0,  0,  2,  2,  2,  3,  3,  3,  3,  4,  4,  4,
                                6, 6, 7, 7, 8, 8, 9, 9, 10, 10, 11, 11, 12, 12, 13, 13, 14, 14, 15, 15, 16, 16, 17, 17, 18, 18};
static const int DB_TC0[52][3] = {
    {0, 0, 0},  {0, 0, 0},  {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},
    {0, 0, 0},  {0, 0, 0},  {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},   {0, 0, 0},
    {0, 0, 0},  {0, 0, 1},  {0, 0, 1},   {0, 0, 1},   {0, 0, 1},   {0, 1, 1},   {0, 1, 1},   {1, 1, 1},
    {1, 1, 1},  {1, 1, 1},  {1, 1, 1},   {1, 1, 2},   {1, 1, 2},   {1, 1, 2},   {1, 1, 2},   {1, 2, 3},
    {1, 2, 3},  {2, 2, 3},  {2, 2, 4},   {2, 3, 4},   {2, 3, 4},   {3, 3, 5},   {3, 4, 6},   {3, 4, 6},
    {4, 5, 7},  {4, 5, 8},  {4, 6, 9},   {5, 7, 10},  {6, 8, 11},  {6, 8, 13},  {7, 10, 14}, {8, 11, 16},
    {9, 12, 18}, {10, 13, 20}, {11, 15, 23}, {13, 17, 25}};

void or_deblock_tables(int32_t *alpha, int32_t *beta, int32_t *tc0) {
    for (int i = 0; i < 52; i++) {
        alpha[i] = DB_ALPHA[i];
        beta[i] = DB_BETA[i];
        for (int k = 0; k < 3; k++) tc0[3 * i + k] = DB_TC0[i][k];
    }
}

static int db_clip1(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
static int db_clip3(int lo, int hi, int v) { return v < lo ? lo : (v > hi ? hi : v); }
static int db_abs(int v) { return v < 0 ? -v : v; }

/* filter_luma_line (deblock.rs:67-115): one line across an edge, q0 at p[0],
 * samples `step` apart. */
static void db_luma_line(uint8_t *q, int64_t step, int bs, int alpha, int beta, int tc0) {
    int p0 = q[-step], p1 = q[-2 * step], p2 = q[-3 * step], p3 = q[-4 * step];
    int q0 = q[0], q1 = q[step], q2 = q[2 * step], q3 = q[3 * step];
    if (db_abs(p0 - q0) >= alpha || db_abs(p1 - p0) >= beta || db_abs(q1 - q0) >= beta) return;
    int ap = db_abs(p2 - p0), aq = db_abs(q2 - q0);
    if (bs < 4) {
        int tc = tc0 + (ap < beta) + (aq < beta);
        int delta = db_clip3(-tc, tc, (((q0 - p0) << 2) + (p1 - q1) + 4) >> 3);
        q[-step] = (uint8_t)db_clip1(p0 + delta);
        q[0] = (uint8_t)db_clip1(q0 - delta);
        if (ap < beta) q[-2 * step] = (uint8_t)db_clip1(p1 + db_clip3(-tc0, tc0, (p2 + ((p0 + q0 + 1) >> 1) - (p1 << 1)) >> 1));
        if (aq < beta) q[step] = (uint8_t)db_clip1(q1 + db_clip3(-tc0, tc0, (q2 + ((p0 + q0 + 1) >> 1) - (q1 << 1)) >> 1));
    } else {
        int strong = db_abs(p0 - q0) < (alpha >> 2) + 2;
        if (strong && ap < beta) {
            q[-step] = (uint8_t)db_clip1((p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3);
            q[-2 * step] = (uint8_t)db_clip1((p2 + p1 + p0 + q0 + 2) >> 2);
            q[-3 * step] = (uint8_t)db_clip1((2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3);
        } else {
            q[-step] = (uint8_t)db_clip1((2 * p1 + p0 + q1 + 2) >> 2);
        }
        if (strong && aq < beta) {
            q[0] = (uint8_t)db_clip1((q2 + 2 * q1 + 2 * q0 + 2 * p0 + p1 + 4) >> 3);
            q[step] = (uint8_t)db_clip1((q2 + q1 + q0 + p0 + 2) >> 2);
            q[2 * step] = (uint8_t)db_clip1((2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3);
        } else {
            q[0] = (uint8_t)db_clip1((2 * q1 + q0 + p1 + 2) >> 2);
        }
    }
}

/* filter_chroma_line (deblock.rs:117-137). */
static void db_chroma_line(uint8_t *q, int64_t step, int bs, int alpha, int beta, int tc0) {
    int p0 = q[-step], p1 = q[-2 * step], q0 = q[0], q1 = q[step];
    if (db_abs(p0 - q0) >= alpha || db_abs(p1 - p0) >= beta || db_abs(q1 - q0) >= beta) return;
    if (bs < 4) {
        int tc = tc0 + 1;
        int delta = db_clip3(-tc, tc, (((q0 - p0) << 2) + (p1 - q1) + 4) >> 3);
        q[-step] = (uint8_t)db_clip1(p0 + delta);
        q[0] = (uint8_t)db_clip1(q0 - delta);
    } else {
        q[-step] = (uint8_t)db_clip1((2 * p1 + p0 + q1 + 2) >> 2);
        q[0] = (uint8_t)db_clip1((2 * q1 + q0 + p1 + 2) >> 2);
    }
}

/* thresholds (deblock.rs:1921-1929). */
static void db_thresholds(int qpav, int oa, int ob, int *alpha, int *beta, const int **tc0) {
    int ia = db_clip3(0, 51, qpav + oa), ib = db_clip3(0, 51, qpav + ob);
    *alpha = DB_ALPHA[ia];
    *beta = DB_BETA[ib];
    *tc0 = DB_TC0[ia];
}

/* bS of an edge between two inter blocks, both ref 0 (bs_inter + bs1_tile's
 * single-list arm, deblock.rs:328-333, 396-404): 2 with coefficients on either
 * side, else 1 when the MVs differ by 4 quarter-pels in x or y, else 0. */
static int db_bs(int nzp, int nzq, int32_t pmx, int32_t pmy, int32_t qmx, int32_t qmy) {
    if (nzp || nzq) return 2;
    return (db_abs(pmx - qmx) >= 4 || db_abs(pmy - qmy) >= 4) ? 1 : 0;
}

/* The MV and coefficient flag of 4x4 block (bx, by) of MB m. */
static void db_block(const int32_t *picks, const int16_t *coeffs, int m, int bx, int by, int32_t mv[2], int *nz) {
    const int32_t *pk = picks + 6 * m;
    int part = pk[0] == 1 ? (by >= 2) : (pk[0] == 2 ? (bx >= 2) : 0);
    mv[0] = pk[1 + 2 * part];
    mv[1] = pk[2 + 2 * part];
    int qi = (by >= 2 ? 2 : 0) + (bx >= 2 ? 1 : 0), k = (by & 1) * 2 + (bx & 1);
    const int16_t *c = coeffs + (int64_t)m * 256 + (qi * 4 + k) * 16;
    *nz = 0;
    for (int i = 0; i < 16; i++) *nz |= c[i] != 0;
}

/* filter_frame_rows (deblock.rs:2135-2700) over the plain-ME picture: MBs in
 * raster order; per MB the luma vertical edges (block columns 0..3, the MB
 * edge skipped at the picture's left), then the horizontal ones, then per
 * chroma plane its vertical edges (chroma columns 0 and 4, bS of luma edges 0
 * and 2, one segment per two chroma lines) and horizontal edges; MB edges
 * average the two MBs' QPs (equal here), chroma uses chroma_qp(qp + offset).
 * u and v may be NULL (luma only). */
void or_deblock_frame_plain(uint8_t *y, uint8_t *u, uint8_t *v, int cw, int ch, const int32_t *picks,
                            const int16_t *coeffs, int qp, int offset_a, int offset_b, int chroma_qp_offset) {
    int mb_w = cw / 16, mb_h = ch / 16, ccw = cw / 2;
    int qpc = or_chroma_qp(db_clip3(0, 51, qp + chroma_qp_offset));
    int ay, by_, ac, bc;
    const int *ty, *tc;
    db_thresholds(qp, offset_a, offset_b, &ay, &by_, &ty);  /* (qp + qp + 1) >> 1 == qp on MB edges too */
    db_thresholds(qpc, offset_a, offset_b, &ac, &bc, &tc);
    for (int mby = 0; mby < mb_h; mby++)
        for (int mbx = 0; mbx < mb_w; mbx++) {
            int m = mby * mb_w + mbx;
            int bs_v[4][4], bs_h[4][4];
            for (int e = 0; e < 4; e++)
                for (int sg = 0; sg < 4; sg++) {
                    int32_t mp[2], mq[2];
                    int nzp, nzq;
                    /* vertical edge e, block row sg */
                    bs_v[e][sg] = 0;
                    if (e > 0 || mbx > 0) {
                        db_block(picks, coeffs, e > 0 ? m : m - 1, e > 0 ? e - 1 : 3, sg, mp, &nzp);
                        db_block(picks, coeffs, m, e, sg, mq, &nzq);
                        bs_v[e][sg] = db_bs(nzp, nzq, mp[0], mp[1], mq[0], mq[1]);
                    }
                    /* horizontal edge e, block column sg */
                    bs_h[e][sg] = 0;
                    if (e > 0 || mby > 0) {
                        db_block(picks, coeffs, e > 0 ? m : m - mb_w, sg, e > 0 ? e - 1 : 3, mp, &nzp);
                        db_block(picks, coeffs, m, sg, e, mq, &nzq);
                        bs_h[e][sg] = db_bs(nzp, nzq, mp[0], mp[1], mq[0], mq[1]);
                    }
                }
            for (int e = 0; e < 4; e++)
                for (int sg = 0; sg < 4; sg++) {
                    int bs = bs_v[e][sg];
                    if (!bs) continue;
                    for (int r = 0; r < 4; r++)
                        db_luma_line(y + (int64_t)(mby * 16 + sg * 4 + r) * cw + mbx * 16 + e * 4, 1, bs, ay, by_, ty[bs - 1]);
                }
            for (int e = 0; e < 4; e++)
                for (int sg = 0; sg < 4; sg++) {
                    int bs = bs_h[e][sg];
                    if (!bs) continue;
                    for (int c = 0; c < 4; c++)
                        db_luma_line(y + (int64_t)(mby * 16 + e * 4) * cw + mbx * 16 + sg * 4 + c, cw, bs, ay, by_, ty[bs - 1]);
                }
            for (int pl = 0; pl < 2; pl++) {
                uint8_t *cp = pl == 0 ? u : v;
                if (!cp) continue;
                for (int ce = 0; ce < 4; ce += 2)
                    for (int r = 0; r < 8; r++) {
                        int bs = bs_v[ce][(r * 2) / 4];
                        if (!bs) continue;
                        db_chroma_line(cp + (int64_t)(mby * 8 + r) * ccw + mbx * 8 + ce * 2, 1, bs, ac, bc, tc[bs - 1]);
                    }
                for (int ce = 0; ce < 4; ce += 2)
                    for (int c = 0; c < 8; c++) {
                        int bs = bs_h[ce][(c * 2) / 4];
                        if (!bs) continue;
                        db_chroma_line(cp + (int64_t)(mby * 8 + ce * 2) * ccw + mbx * 8 + c, ccw, bs, ac, bc, tc[bs - 1]);
                    }
            }
        }
}

typedef struct {
    const uint8_t *frames;
    uint8_t *half;
    int cw, ch, cwh, chh, mb_w, mb_h, nmb;
    size_t fs, hs;
    int mode;
    int32_t *intra, *inter, *mvs;
} la_args;

static void la_down(void *p, int f, int tid) {
    la_args *a = (la_args *)p;
    (void)tid;
    or_downsample2x(a->frames + a->fs * f, a->cw, a->ch, a->half + a->hs * f);
}

static void la_costs(void *p, int f, int tid) {
    la_args *a = (la_args *)p;
    (void)tid;
    or_frame_costs(a->frames + a->fs * f, a->cw, a->ch, a->half + a->hs * f, a->cwh, a->chh, a->mb_w, a->mb_h,
                   f > 0 ? a->frames + a->fs * (f - 1) : NULL, f > 0 ? a->half + a->hs * (f - 1) : NULL, a->mode,
                   a->intra + (size_t)a->nmb * f, a->inter + (size_t)a->nmb * f, a->mvs + (size_t)2 * a->nmb * f);
}

/* HalfRes lookahead of a whole clip (mbtree.rs:413-436 for mode HalfRes). */
void or_lookahead_clip(const uint8_t *frames, int nframes, int cw, int ch, int mode, int32_t *intra, int32_t *inter,
                       int32_t *mvs, int nthreads) {
    int mb_w = cw / 16, mb_h = ch / 16, nmb = mb_w * mb_h;
    int cwh = cw / 2, chh = ch / 2;
    size_t fs = (size_t)cw * ch, hs = (size_t)cwh * chh;
    uint8_t *half = (uint8_t *)malloc(hs * nframes);
    la_args a = {frames, half, cw, ch, cwh, chh, mb_w, mb_h, nmb, fs, hs, mode, intra, inter, mvs};
    par_for(nframes, nthreads, la_down, &a);
    par_for(nframes, nthreads, la_costs, &a);
    free(half);
}

typedef struct {
    const uint8_t *frames;
    int cw, ch, pad;
    const or_me_params_flat *pf;
    const uint16_t *tab;
    double lambda_me;
    int64_t split_gate;
    int qp, dz_div;
    int32_t *picks;
    int64_t *costs;
    int16_t *coeffs;
    int nmb;
    size_t fs, p4;
} pp_args;

static void pp_frame(void *p, int i, int tid) {
    pp_args *a = (pp_args *)p;
    (void)tid;
    int f = i + 1;
    uint8_t *planes = (uint8_t *)malloc(a->p4);
    const uint8_t *ref = a->frames + a->fs * (f - 1), *src = a->frames + a->fs * f;
    or_build_planes4(ref, a->cw, a->ch, a->pad, planes);
    or_me_frame_flat(src, ref, planes, a->cw, a->ch, a->pad, a->pf, a->tab, a->lambda_me, a->split_gate,
                     a->picks + (size_t)6 * a->nmb * f, a->costs + (size_t)2 * a->nmb * f);
    or_mc_tq_frame(src, ref, a->cw, a->ch, a->picks + (size_t)6 * a->nmb * f, a->qp, a->dz_div,
                   a->coeffs + (size_t)256 * a->nmb * f);
    free(planes);
}

/* The whole pixel path over a clip: planes, ME, MC+T/Q (frames 1..n-1) and the
 * lookahead (all frames).  Outputs are per frame; frame 0 rows are zero. */
void or_pixel_path_clip(const uint8_t *frames, int nframes, int cw, int ch, int pad, const or_me_params_flat *pf,
                        const uint16_t *tab, double lambda_me, int64_t split_gate, int qp, int dz_div,
                        int32_t *picks, int64_t *costs, int16_t *coeffs, int32_t *la_intra, int32_t *la_inter,
                        int32_t *la_mvs, int nthreads) {
    int nmb = (cw / 16) * (ch / 16);
    size_t fs = (size_t)cw * ch;
    int pw = cw + 2 * pad, ph = ch + 2 * pad;
    size_t p4 = (size_t)4 * pw * ph;
    memset(picks, 0, sizeof(int32_t) * 6 * nmb);
    memset(costs, 0, sizeof(int64_t) * 2 * nmb);
    memset(coeffs, 0, sizeof(int16_t) * 256 * nmb);
    pp_args a = {frames, cw, ch, pad, pf, tab, lambda_me, split_gate, qp, dz_div, picks, costs, coeffs, nmb, fs, p4};
    par_for(nframes - 1, nthreads, pp_frame, &a);
    or_lookahead_clip(frames, nframes, cw, ch, 2, la_intra, la_inter, la_mvs, nthreads);
}

/* The closed reconstruction loop over a clip of n frames (luma cw x ch,
 * chroma cw/2 x ch/2, each contiguous).  Frame 0 reconstructs to itself (the
 * frame model codes it losslessly).  P frame f runs the frame's motion search
 * against the planes of the deblocked reconstruction of frame f-1, as the
 * reference encoder searches RefFrames built from reconstructed planes
 * (encoder/src/lib.rs:228-262), predicts from that reconstruction, and its
 * luma (mb16.rs:3575-3605) and chroma (mb16.rs:3606-3628) reconstruction,
 * deblocked (deblock.rs filter_frame; offsets 0), is frame f+1's reference.
 * props (optional, 16 i32 per MB per frame) switch the 16x16 search to the
 * learned-proposal search with threshold prop_t.  Outputs per frame (frame 0
 * rows zero): picks 6 i32/MB, costs 2 i64/MB, luma levels 256 i16/MB, chroma
 * levels 128 i16/MB, the reconstruction, fallback flags (optional). */
void or_closed_loop_clip(const uint8_t *y, const uint8_t *u, const uint8_t *v, int n, int cw, int ch, int pad,
                         const or_me_params_flat *pf, const uint16_t *tab, double lambda_me, int64_t split_gate,
                         int qp, int dz_div, const int32_t *props, int32_t prop_t, int32_t *picks, int64_t *costs,
                         int16_t *coeffs, int16_t *ccoeffs, uint8_t *rec_y, uint8_t *rec_u, uint8_t *rec_v,
                         int32_t *fell) {
    int nmb = (cw / 16) * (ch / 16);
    size_t fs = (size_t)cw * ch, cs = fs / 4;
    int pw = cw + 2 * pad, ph = ch + 2 * pad;
    uint8_t *planes = (uint8_t *)malloc((size_t)4 * pw * ph);
    memset(picks, 0, sizeof(int32_t) * 6 * nmb);
    memset(costs, 0, sizeof(int64_t) * 2 * nmb);
    memset(coeffs, 0, sizeof(int16_t) * 256 * nmb);
    memset(ccoeffs, 0, sizeof(int16_t) * 128 * nmb);
    if (fell) memset(fell, 0, sizeof(int32_t) * nmb);
    memcpy(rec_y, y, fs);
    memcpy(rec_u, u, cs);
    memcpy(rec_v, v, cs);
    for (int f = 1; f < n; f++) {
        const uint8_t *ry = rec_y + fs * (f - 1), *ru = rec_u + cs * (f - 1), *rv = rec_v + cs * (f - 1);
        uint8_t *oy = rec_y + fs * f, *ou = rec_u + cs * f, *ov = rec_v + cs * f;
        int32_t *pk = picks + (size_t)6 * nmb * f;
        int16_t *co = coeffs + (size_t)256 * nmb * f;
        or_build_planes4(ry, cw, ch, pad, planes);
        or_me_frame_learned_flat(y + fs * f, ry, planes, cw, ch, pad, pf, tab, lambda_me, split_gate,
                                 props ? props + (size_t)16 * nmb * f : NULL, prop_t, pk,
                                 costs + (size_t)2 * nmb * f, fell ? fell + (size_t)nmb * f : NULL);
        or_mc_tq_rec_frame(y + fs * f, ry, cw, ch, pk, qp, dz_div, co, oy);
        or_mc_tq_chroma_frame(u + cs * f, v + cs * f, ru, rv, cw, ch, pk, qp, ccoeffs + (size_t)128 * nmb * f, ou, ov);
        or_deblock_frame_plain(oy, ou, ov, cw, ch, pk, co, qp, 0, 0, 0);
    }
    free(planes);
}
