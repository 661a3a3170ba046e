/* h264_decoder.c -- CPU restatement of the reference decoder's CAVLC path for
 * the stream subset the library writes (h264a_write_stream_cavlc).
 *
 * TEST INFRASTRUCTURE ONLY: tests/ decode the library's streams with it and
 * compare the pictures with the encoder's reconstruction.  Nothing in the
 * product links it.
 *
 * Follows crates/rusty_h264-decoder: decode_stream (src/lib.rs:838), the
 * slice header and decode_slice (src/lib.rs:893), the CAVLC slice data loop
 * (src/mb16.rs:3859 decode_slice_data, :3911 decode_slice_cavlc_inner), mb_type
 * mapping (src/mb16.rs:4079), residual blocks (common/src/cavlc.rs:608
 * decode_residual_block) and the standard's syntax (7.3) for the subset:
 * Baseline SPS/PPS, IDR I slices of I_PCM MBs, P slices of P_Skip,
 * P_L0_16x16, P_L0_L0_16x8 and P_L0_L0_8x16 MBs with reference 0, 4x4
 * transforms, deblocking on (slice offsets allowed) or off.  Reconstruction
 * uses the oracle's restated MC, dequantisation, inverse transform and
 * deblocking.  The VLC tables are passed in by the caller (the tests pass the
 * ones parsed from the reference's cavlc.rs), so this file holds none. */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "h264_oracle.h"

typedef struct {
    uint8_t ct_len[4][68], ct_bits[4][68];
    uint8_t cdc_len[20], cdc_bits[20];
    uint8_t tz_len[15][16], tz_bits[15][16];
    uint8_t ctz_len[3][4], ctz_bits[3][4];
    uint8_t run_len[7][15], run_bits[7][15];
    uint8_t cbp_inter[48]; /* codeNum -> coded_block_pattern */
} or_cavlc_tables;

typedef struct {
    const uint8_t *b;
    size_t n, pos; /* bytes, bit position */
    int err;
} br_t;

static uint32_t br_bit(br_t *r) {
    if (r->pos >= r->n * 8) { r->err = 1; return 0; }
    uint32_t v = (r->b[r->pos >> 3] >> (7 - (r->pos & 7))) & 1u;
    r->pos++;
    return v;
}
static uint32_t br_u(br_t *r, int len) {
    uint32_t v = 0;
    for (int i = 0; i < len; i++) v = (v << 1) | br_bit(r);
    return v;
}
static uint32_t br_peek(br_t *r, int len) {
    size_t p = r->pos;
    int e = r->err;
    uint32_t v = br_u(r, len);
    r->pos = p;
    r->err = e;
    return v;
}
static uint32_t br_ue(br_t *r) {
    int z = 0;
    while (!br_bit(r)) {
        if (r->err || ++z > 31) { r->err = 1; return 0; }
    }
    return z ? ((1u << z) - 1 + br_u(r, z)) : 0;
}
static int32_t br_se(br_t *r) {
    uint32_t k = br_ue(r);
    return (k & 1) ? (int32_t)((k + 1) / 2) : -(int32_t)(k / 2);
}
/* more_rbsp_data: anything before the trailing stop bit */
static int br_more(const br_t *r) {
    size_t last = r->n * 8; /* position just after the last 1 bit */
    while (last > 0 && !((r->b[(last - 1) >> 3] >> (7 - ((last - 1) & 7))) & 1)) last--;
    return r->pos + 1 < last;
}

/* residual_block: coeffs (maxc entries, scan order); nc -1 is chroma DC.
 * Returns TotalCoeff, or -1 on a malformed block. */
static int read_block(br_t *r, const or_cavlc_tables *t, int nc, int maxc, int *coeffs) {
    memset(coeffs, 0, sizeof(int) * maxc);
    int tc = -1, t1 = 0;
    if (nc == -1) {
        for (int i = 0; i < 20 && tc < 0; i++)
            if (t->cdc_len[i] && br_peek(r, t->cdc_len[i]) == t->cdc_bits[i]) {
                br_u(r, t->cdc_len[i]);
                tc = i / 4; t1 = i % 4;
            }
    } else {
        int cls = nc < 2 ? 0 : (nc < 4 ? 1 : (nc < 8 ? 2 : 3));
        for (int i = 0; i < 68 && tc < 0; i++)
            if (t->ct_len[cls][i] && br_peek(r, t->ct_len[cls][i]) == t->ct_bits[cls][i]) {
                br_u(r, t->ct_len[cls][i]);
                tc = i / 4; t1 = i % 4;
            }
    }
    if (tc < 0 || tc > maxc || r->err) return -1;
    if (tc == 0) return 0;
    int level[16];
    int suffix = (tc > 10 && t1 < 3) ? 1 : 0;
    for (int i = 0; i < tc; i++) {
        if (i < t1) { level[i] = br_bit(r) ? -1 : 1; continue; }
        int prefix = 0;
        while (!br_bit(r)) { if (r->err || ++prefix > 28) return -1; }
        int ssize = (prefix == 14 && suffix == 0) ? 4 : (prefix >= 15 ? prefix - 3 : suffix);
        int64_t code = ((int64_t)(prefix < 15 ? prefix : 15) << suffix) + (ssize ? br_u(r, ssize) : 0);
        if (prefix >= 15 && suffix == 0) code += 15;
        if (prefix >= 16) code += (1LL << (prefix - 3)) - 4096;
        if (i == t1 && t1 < 3) code += 2;
        level[i] = (code % 2 == 0) ? (int)((code + 2) >> 1) : (int)((-code - 1) >> 1);
        if (suffix == 0) suffix = 1;
        int a = level[i] < 0 ? -level[i] : level[i];
        if (a > (3 << (suffix - 1)) && suffix < 6) suffix++;
    }
    int tz = 0;
    if (tc < maxc) {
        int found = 0;
        if (nc == -1) {
            for (int z = 0; z < 4 && !found; z++)
                if (t->ctz_len[tc - 1][z] && br_peek(r, t->ctz_len[tc - 1][z]) == t->ctz_bits[tc - 1][z]) {
                    br_u(r, t->ctz_len[tc - 1][z]); tz = z; found = 1;
                }
        } else {
            for (int z = 0; z < 16 && !found; z++)
                if (t->tz_len[tc - 1][z] && br_peek(r, t->tz_len[tc - 1][z]) == t->tz_bits[tc - 1][z]) {
                    br_u(r, t->tz_len[tc - 1][z]); tz = z; found = 1;
                }
        }
        if (!found) return -1;
    }
    int run[16], left = tz;
    for (int i = 0; i < tc - 1; i++) {
        run[i] = 0;
        if (left > 0) {
            int zl = (left < 7 ? left : 7) - 1, found = 0;
            for (int k = 0; k < 15 && !found; k++)
                if (t->run_len[zl][k] && br_peek(r, t->run_len[zl][k]) == t->run_bits[zl][k]) {
                    br_u(r, t->run_len[zl][k]); run[i] = k; found = 1;
                }
            if (!found) return -1;
            left -= run[i];
        }
    }
    run[tc - 1] = left;
    int pos = tc + tz - 1;
    if (pos >= maxc || left < 0) return -1;
    for (int i = 0; i < tc; i++) {
        coeffs[pos] = level[i];
        pos -= 1 + run[i];
    }
    return r->err ? -1 : tc;
}

static const int ZZ[16] = {0, 1, 4, 8, 5, 2, 3, 6, 9, 12, 13, 10, 7, 11, 14, 15};

typedef struct {
    int cw, ch, width, height, qp_init, deblock_ctl, log2_fn;
} seq_t;

typedef struct { int av, mvx, mvy; } nb_t;

static nb_t grid_at(const int32_t *mv, const uint8_t *done, int mb_w, int mb_h, int bx, int by) {
    nb_t n = {0, 0, 0};
    if (bx < 0 || by < 0 || bx >= 4 * mb_w || by >= 4 * mb_h || !done[(by >> 2) * mb_w + (bx >> 2)]) return n;
    size_t i = 2 * ((size_t)by * 4 * mb_w + bx);
    n.av = 1; n.mvx = mv[i]; n.mvy = mv[i + 1];
    return n;
}
static or_mv_neighbor to_or(nb_t n) {
    or_mv_neighbor o;
    o.available = n.av; o.mvx = n.mvx; o.mvy = n.mvy; o.ref_idx = n.av ? 0 : -1;
    return o;
}

/* Luma and chroma prediction of an MB under its pick (shape, two MVs). */
static void mb_pred(const uint8_t *ry, const uint8_t *ru, const uint8_t *rv, int cw, int ch, int mbx, int mby,
                    const int32_t *pk, uint8_t py[256], uint8_t pu[64], uint8_t pv[64]) {
    int shape = pk[0];
    for (int k = 0; k < (shape ? 2 : 1); k++) {
        int ox = shape == 2 ? 8 * k : 0, oy = shape == 1 ? 8 * k : 0;
        int bw = shape == 2 ? 8 : 16, bh = shape == 1 ? 8 : 16;
        uint8_t t[256];
        or_mc_luma(ry, cw, ch, mbx * 16 + ox, mby * 16 + oy, bw, bh, pk[1 + 2 * k], pk[2 + 2 * k], t);
        for (int r = 0; r < bh; r++) memcpy(py + (oy + r) * 16 + ox, t + r * bw, bw);
        for (int c = 0; c < 2; c++) {
            uint8_t tc[64];
            or_mc_chroma(c ? rv : ru, cw / 2, ch / 2, mbx * 8 + ox / 2, mby * 8 + oy / 2, bw / 2, bh / 2, pk[1 + 2 * k],
                         pk[2 + 2 * k], tc);
            for (int r = 0; r < bh / 2; r++) memcpy((c ? pv : pu) + (oy / 2 + r) * 8 + ox / 2, tc + r * (bw / 2), bw / 2);
        }
    }
}

/* Chroma reconstruction of one MB's component from its levels (slot 0 of
 * each block the DC level), as mb16.rs:3606-3628. */
static void chroma_rec(uint8_t *rec, int stride, const uint8_t pred[64], const int16_t lv[64], int qp) {
    int qpc = or_chroma_qp(qp);
    int32_t dl[4] = {lv[0], lv[16], lv[32], lv[48]}, rdc[4];
    or_inverse_quant_chroma_dc(dl, qpc, rdc);
    int16_t d[64];
    for (int i = 0; i < 4; i++) {
        int32_t l[16], dq[16];
        l[0] = 0;
        for (int j = 1; j < 16; j++) l[j] = lv[i * 16 + j];
        or_dequant4x4(l, qpc, dq);
        for (int j = 0; j < 16; j++) d[i * 16 + j] = (int16_t)dq[j];
        d[i * 16] = (int16_t)rdc[i];
    }
    or_idct_four_t4_rec(rec, stride, pred, 8, d);
}

static void store_mb_mvs(int32_t *mv, int mb_w, int mbx, int mby, const int32_t *pk) {
    int shape = pk[0];
    for (int q = 0; q < 16; q++) {
        int part = shape == 1 ? (q / 4 >= 2) : (shape == 2 ? (q % 4 >= 2) : 0);
        size_t gi = 2 * ((size_t)(4 * mby + q / 4) * 4 * mb_w + 4 * mbx + q % 4);
        mv[gi] = pk[1 + 2 * part];
        mv[gi + 1] = pk[2 + 2 * part];
    }
}

/* nC of a block from its left / top neighbours' TotalCoeff (9.2.1): inside
 * the picture they are available (one slice, raster MB order, and inside an
 * MB the left and top blocks come earlier in the block scan). */
static int nc_of(const uint8_t *tc, int stride, int bx, int by) {
    int ha = bx > 0, hb = by > 0;
    int na = ha ? tc[(size_t)by * stride + bx - 1] : 0, nb = hb ? tc[(size_t)(by - 1) * stride + bx] : 0;
    return ha && hb ? (na + nb + 1) >> 1 : (ha ? na : (hb ? nb : 0));
}

/* Decodes an Annex-B stream of the subset into frames of the coded size
 * (cw x ch, chroma cw/2 x ch/2, max_frames of each).  picks (6 i32/MB),
 * coeffs (256 i16/MB) and ccoeffs (128 i16/MB) per frame receive the parsed
 * syntax (may be NULL).  Returns the number of frames, or -1 malformed /
 * unsupported, -2 geometry mismatch, -3 too many frames. */
int or_decode_stream(const uint8_t *data, size_t len, const or_cavlc_tables *t, int cw, int ch, int max_frames,
                     uint8_t *out_y, uint8_t *out_u, uint8_t *out_v, int32_t *picks, int16_t *coeffs,
                     int16_t *ccoeffs) {
    seq_t sq;
    memset(&sq, 0, sizeof sq);
    int have_sps = 0, have_pps = 0, nframes = 0;
    int mb_w = cw / 16, mb_h = ch / 16, nmb = mb_w * mb_h, W4 = 4 * mb_w, W2 = 2 * mb_w;
    size_t fs = (size_t)cw * ch, cs = fs / 4;
    uint8_t *rbsp = (uint8_t *)malloc(len + 1);
    int32_t *mv = (int32_t *)malloc(sizeof(int32_t) * 2 * 16 * nmb);
    uint8_t *done = (uint8_t *)malloc(nmb);
    uint8_t *tcy = (uint8_t *)malloc(16 * nmb), *tcc = (uint8_t *)malloc(2 * 4 * nmb);
    int32_t *fpk = (int32_t *)malloc(sizeof(int32_t) * 6 * nmb);
    int16_t *fco = (int16_t *)malloc(sizeof(int16_t) * 256 * nmb), *fcc = (int16_t *)malloc(sizeof(int16_t) * 128 * nmb);
    int ret = 0;
    size_t i = 0;
    while (i + 3 < len) {
        /* the next start code (00 00 01 or 00 00 00 01) */
        if (!(data[i] == 0 && data[i + 1] == 0 && (data[i + 2] == 1 || (data[i + 2] == 0 && data[i + 3] == 1)))) {
            i++;
            continue;
        }
        i += data[i + 2] == 1 ? 3 : 4;
        size_t j = i;
        while (j + 2 < len && !(data[j] == 0 && data[j + 1] == 0 && (data[j + 2] == 1 || data[j + 2] == 0))) j++;
        if (j + 2 >= len) j = len;
        /* NAL [i, j): header, then the RBSP without emulation prevention */
        int type = data[i] & 31;
        size_t n = 0;
        int zeros = 0;
        for (size_t k = i + 1; k < j; k++) {
            if (zeros >= 2 && data[k] == 3) { zeros = 0; continue; }
            rbsp[n++] = data[k];
            zeros = data[k] == 0 ? zeros + 1 : 0;
        }
        br_t r = {rbsp, n, 0, 0};
        i = j;
        if (type == 7) { /* SPS */
            if (br_u(&r, 8) != 66) { ret = -1; break; }
            br_u(&r, 16);
            br_ue(&r);
            sq.log2_fn = (int)br_ue(&r) + 4;
            if (br_ue(&r) != 2) { ret = -1; break; } /* pic_order_cnt_type */
            br_ue(&r);
            br_u(&r, 1);
            sq.cw = 16 * ((int)br_ue(&r) + 1);
            sq.ch = 16 * ((int)br_ue(&r) + 1);
            if (!br_u(&r, 1)) { ret = -1; break; } /* frame_mbs_only */
            br_u(&r, 1);
            sq.width = sq.cw; sq.height = sq.ch;
            if (br_u(&r, 1)) {
                int l = (int)br_ue(&r), rr = (int)br_ue(&r), tt = (int)br_ue(&r), bb = (int)br_ue(&r);
                sq.width = sq.cw - 2 * (l + rr);
                sq.height = sq.ch - 2 * (tt + bb);
            }
            if (sq.cw != cw || sq.ch != ch) { ret = -2; break; }
            have_sps = 1;
        } else if (type == 8) { /* PPS */
            br_ue(&r);
            br_ue(&r);
            if (br_u(&r, 1)) { ret = -1; break; } /* CABAC: not this subset */
            br_u(&r, 1);
            if (br_ue(&r) != 0) { ret = -1; break; }
            br_ue(&r);
            br_ue(&r);
            br_u(&r, 1);
            br_u(&r, 2);
            sq.qp_init = 26 + br_se(&r);
            br_se(&r);
            if (br_se(&r) != 0) { ret = -1; break; } /* chroma_qp_index_offset */
            sq.deblock_ctl = (int)br_u(&r, 1);
            have_pps = 1;
        } else if (type == 5 || type == 1) {
            if (!have_sps || !have_pps) { ret = -1; break; }
            if (nframes >= max_frames) { ret = -3; break; }
            br_ue(&r); /* first_mb_in_slice */
            int st = (int)br_ue(&r) % 5;
            br_ue(&r);
            br_u(&r, sq.log2_fn);
            if (type == 5) br_ue(&r); /* idr_pic_id */
            if (st == 0) { /* num_ref_idx_active_override, ref_pic_list_modification */
                if (br_u(&r, 1) || br_u(&r, 1)) { ret = -1; break; }
            }
            if (type == 5) { br_u(&r, 1); br_u(&r, 1); }
            else if (br_u(&r, 1)) { ret = -1; break; } /* adaptive marking: not this subset */
            int qp = sq.qp_init + br_se(&r);
            int dbf = 1, offa = 0, offb = 0;
            if (sq.deblock_ctl) {
                int idc = (int)br_ue(&r);
                if (idc > 1) { ret = -1; break; }
                if (idc != 1) { offa = 2 * br_se(&r); offb = 2 * br_se(&r); }
                dbf = idc != 1;
            }
            uint8_t *y = out_y + fs * nframes, *u = out_u + cs * nframes, *v = out_v + cs * nframes;
            memset(done, 0, nmb);
            memset(tcy, 0, 16 * nmb);
            memset(tcc, 0, 8 * nmb);
            memset(fpk, 0, sizeof(int32_t) * 6 * nmb);
            memset(fco, 0, sizeof(int16_t) * 256 * nmb);
            memset(fcc, 0, sizeof(int16_t) * 128 * nmb);
            const uint8_t *ry = nframes ? out_y + fs * (nframes - 1) : NULL;
            const uint8_t *ru = nframes ? out_u + cs * (nframes - 1) : NULL;
            const uint8_t *rv = nframes ? out_v + cs * (nframes - 1) : NULL;
            if (st == 0 && !ry) { ret = -1; break; }
            if (st != 0 && st != 2) { ret = -1; break; }
            int m = 0, bad = 0;
            while (m < nmb && !bad) {
                int skip = 0;
                if (st == 0) {
                    skip = (int)br_ue(&r);
                    if (skip > nmb - m) { bad = 1; break; }
                }
                for (int s = 0; s < skip; s++, m++) { /* P_Skip (8.4.1.1) */
                    int mbx = m % mb_w, mby = m / mb_w;
                    nb_t a = grid_at(mv, done, mb_w, mb_h, 4 * mbx - 1, 4 * mby);
                    nb_t b = grid_at(mv, done, mb_w, mb_h, 4 * mbx, 4 * mby - 1);
                    int32_t p[2] = {0, 0};
                    if (a.av && b.av && !(a.mvx == 0 && a.mvy == 0) && !(b.mvx == 0 && b.mvy == 0)) {
                        nb_t c = grid_at(mv, done, mb_w, mb_h, 4 * mbx + 4, 4 * mby - 1);
                        if (!c.av) c = grid_at(mv, done, mb_w, mb_h, 4 * mbx - 1, 4 * mby - 1);
                        or_mv_neighbor A = to_or(a), B = to_or(b), Cn = to_or(c);
                        or_predict_mv(&A, &B, &Cn, 0, p);
                    }
                    int32_t *pk = fpk + 6 * m;
                    pk[0] = 0; pk[1] = pk[3] = p[0]; pk[2] = pk[4] = p[1];
                    uint8_t py[256], pu[64], pv[64];
                    mb_pred(ry, ru, rv, cw, ch, mbx, mby, pk, py, pu, pv);
                    for (int rr = 0; rr < 16; rr++) memcpy(y + (size_t)(mby * 16 + rr) * cw + mbx * 16, py + rr * 16, 16);
                    for (int rr = 0; rr < 8; rr++) {
                        memcpy(u + (size_t)(mby * 8 + rr) * (cw / 2) + mbx * 8, pu + rr * 8, 8);
                        memcpy(v + (size_t)(mby * 8 + rr) * (cw / 2) + mbx * 8, pv + rr * 8, 8);
                    }
                    store_mb_mvs(mv, mb_w, mbx, mby, pk);
                    done[m] = 1;
                }
                if (m >= nmb) break;
                if (st == 0 && skip > 0 && !br_more(&r)) { bad = 1; break; }
                int mbx = m % mb_w, mby = m / mb_w;
                int mbt = (int)br_ue(&r);
                if (st == 2) { /* I slice: I_PCM only */
                    if (mbt != 25) { bad = 1; break; }
                    while (r.pos & 7) br_bit(&r);
                    for (int rr = 0; rr < 16; rr++)
                        for (int c = 0; c < 16; c++) y[(size_t)(mby * 16 + rr) * cw + mbx * 16 + c] = (uint8_t)br_u(&r, 8);
                    for (int pl = 0; pl < 2; pl++)
                        for (int rr = 0; rr < 8; rr++)
                            for (int c = 0; c < 8; c++)
                                (pl ? v : u)[(size_t)(mby * 8 + rr) * (cw / 2) + mbx * 8 + c] = (uint8_t)br_u(&r, 8);
                    done[m] = 1;
                    m++;
                    if (m < nmb && !br_more(&r)) { bad = 1; break; }
                    continue;
                }
                if (mbt > 2) { bad = 1; break; } /* P_8x8 and intra MBs: not this subset */
                int shape = mbt;
                int32_t *pk = fpk + 6 * m;
                pk[0] = shape;
                for (int part = 0; part < (shape ? 2 : 1); part++) {
                    int x0 = 0, y0 = 0, w4 = 4;
                    if (shape == 1) y0 = part ? 2 : 0;
                    if (shape == 2) { x0 = part ? 2 : 0; w4 = 2; }
                    int bx = 4 * mbx + x0, by = 4 * mby + y0;
                    nb_t nb[4];
                    int xs[4] = {bx - 1, bx, bx + w4, bx - 1}, ys[4] = {by, by - 1, by - 1, by - 1};
                    for (int q = 0; q < 4; q++) {
                        int lx = xs[q] - 4 * mbx, ly = ys[q] - 4 * mby;
                        if (lx >= 0 && lx < 4 && ly >= 0 && ly < 4) { /* inside this MB: earlier partitions */
                            int p = shape == 1 ? (ly >= 2) : (shape == 2 ? (lx >= 2) : 0);
                            nb[q].av = p < part;
                            nb[q].mvx = pk[1 + 2 * p];
                            nb[q].mvy = pk[2 + 2 * p];
                        } else {
                            nb[q] = grid_at(mv, done, mb_w, mb_h, xs[q], ys[q]);
                        }
                    }
                    if (!nb[2].av) nb[2] = nb[3];
                    or_mv_neighbor A = to_or(nb[0]), B = to_or(nb[1]), Cn = to_or(nb[2]);
                    int32_t p[2];
                    or_predict_partition_mv(shape, part, &A, &B, &Cn, 0, p);
                    pk[1 + 2 * part] = p[0] + br_se(&r);
                    pk[2 + 2 * part] = p[1] + br_se(&r);
                }
                if (!shape) { pk[3] = pk[1]; pk[4] = pk[2]; }
                uint32_t cn = br_ue(&r);
                if (cn > 47) { bad = 1; break; }
                int cbp = t->cbp_inter[cn];
                if (cbp) qp += br_se(&r);
                int16_t *L = fco + 256 * m, *Cc = fcc + 128 * m;
                for (int b8 = 0; b8 < 4 && !bad; b8++)
                    for (int b4 = 0; b4 < 4; b4++) {
                        int bx = 4 * mbx + (b8 & 1) * 2 + (b4 & 1), by = 4 * mby + (b8 >> 1) * 2 + (b4 >> 1);
                        int tcn = 0;
                        if (cbp & (1 << b8)) {
                            int sc[16];
                            tcn = read_block(&r, t, nc_of(tcy, W4, bx, by), 16, sc);
                            if (tcn < 0) { bad = 1; break; }
                            for (int q = 0; q < 16; q++) L[b8 * 64 + b4 * 16 + ZZ[q]] = (int16_t)sc[q];
                        }
                        tcy[(size_t)by * W4 + bx] = (uint8_t)tcn;
                    }
                if (bad) break;
                if (cbp >> 4)
                    for (int c = 0; c < 2 && !bad; c++) {
                        int d[4];
                        if (read_block(&r, t, -1, 4, d) < 0) { bad = 1; break; }
                        for (int b = 0; b < 4; b++) Cc[c * 64 + b * 16] = (int16_t)d[b];
                    }
                for (int c = 0; c < 2 && !bad; c++)
                    for (int b = 0; b < 4; b++) {
                        int bx = 2 * mbx + (b & 1), by = 2 * mby + (b >> 1);
                        int tcn = 0;
                        if ((cbp >> 4) == 2) {
                            int sc[15];
                            tcn = read_block(&r, t, nc_of(tcc + (size_t)c * 4 * nmb, W2, bx, by), 15, sc);
                            if (tcn < 0) { bad = 1; break; }
                            for (int q = 1; q < 16; q++) Cc[c * 64 + b * 16 + ZZ[q]] = (int16_t)sc[q - 1];
                        }
                        tcc[(size_t)c * 4 * nmb + (size_t)by * W2 + bx] = (uint8_t)tcn;
                    }
                if (bad) break;
                uint8_t py[256], pu[64], pv[64];
                mb_pred(ry, ru, rv, cw, ch, mbx, mby, pk, py, pu, pv);
                or_mb_luma_rec(y + (size_t)mby * 16 * cw + mbx * 16, cw, py, L, qp);
                chroma_rec(u + (size_t)mby * 8 * (cw / 2) + mbx * 8, cw / 2, pu, Cc, qp);
                chroma_rec(v + (size_t)mby * 8 * (cw / 2) + mbx * 8, cw / 2, pv, Cc + 64, qp);
                store_mb_mvs(mv, mb_w, mbx, mby, pk);
                done[m] = 1;
                m++;
                if (m < nmb && !br_more(&r)) { bad = 1; break; }
            }
            if (bad || r.err || m != nmb) { ret = -1; break; }
            if (st == 0 && dbf) or_deblock_frame_plain(y, u, v, cw, ch, fpk, fco, qp, offa, offb, 0);
            if (picks) memcpy(picks + (size_t)6 * nmb * nframes, fpk, sizeof(int32_t) * 6 * nmb);
            if (coeffs) memcpy(coeffs + (size_t)256 * nmb * nframes, fco, sizeof(int16_t) * 256 * nmb);
            if (ccoeffs) memcpy(ccoeffs + (size_t)128 * nmb * nframes, fcc, sizeof(int16_t) * 128 * nmb);
            nframes++;
        }
    }
    free(rbsp); free(mv); free(done); free(tcy); free(tcc); free(fpk); free(fco); free(fcc);
    return ret < 0 ? ret : nframes;
}
