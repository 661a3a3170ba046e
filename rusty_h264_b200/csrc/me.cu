// me.cu -- a10/a11/a12: motion_search (crates/rusty_h264-encoder/src/mb16.rs:
// 2433-3302), best_part (:4921) and the plain-ME frame pass.
//
// One warp runs one search.  Each lane owns one 4x4 sub-block of the
// partition (its source rows stay in registers for the whole search), so a
// pass over 32 lanes prices 32/nb candidates at once (nb = sub-blocks per
// partition); a candidate's distortion is the sum of its lanes' blocks, added
// with shared-memory atomics.  Control flow is warp-uniform and replays the
// reference exactly:
//  * fixed-centre diamond passes and batched rings price their 4/8 candidates
//    together, then take the first strict-minimum like the reference's argmin;
//  * cascading rings (the centre moves mid-ring) are priced speculatively
//    against the current centre; the first improving point is taken and the
//    remaining points are re-priced around the new centre, which is exactly
//    the order in which the reference evaluates them.
// λ·rate is computed as an IEEE double product truncated toward zero, the
// same arithmetic as `(λ·rate as f64) as i64`.
#include <algorithm>
#include <climits>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "deblock_device.cuh"
#include "hpel_device.cuh"
#include "tq_device.cuh"

namespace h264a {

constexpr int MET_SATD = 0;
constexpr int MET_SAD = 1;
// Warps per CTA of the narrow frame kernel (one MB per warp) and of the wide
// one (one MB per CTA: the 16x16 search by all its warps, each partition by
// one warp).  Four: one warp per SM sub-partition, since the warps of a team
// repeat the same control code and two of them on one sub-partition would
// share its issue slots.
constexpr int ME_WARPS = 4;
constexpr int ME_WIDE_WARPS = 4;
constexpr int ME_PART_TEAM = ME_WIDE_WARPS / 4;  // warps per partition search

// The reference picture's readiness in the pipelined closed loop: its planes
// are built segment by segment (16 picture rows by segw picture columns;
// segment (b, s)'s flag == epoch means every segment up and left of it is
// complete), and a search waits (bounded) for the segment of every pixel it
// reads.
struct BandWait {
    const int* flags;  // nbands x nseg readiness flags, band-major
    int nbands, nseg, segw, epoch, limit;
    int* status;
};

// Waits until the reference's planes (and reconstruction) are final at
// picture pixel (row, col), clamped into the picture: the flag of the band
// (16 rows) and column segment (segw columns) holding it.  Segment (b, s) is
// published after (b-1, s) and (b, s-1), so it stands for every segment up
// and left of it.  `ready` caches a segment seen ready, packed b << 12 | s
// (-1: none); any value stored there was seen ready, so a torn update between
// lanes only loses a shortcut.  Nothing when the search has no BandWait.
__device__ __forceinline__ void band_wait_px(const BandWait* bw, int* ready, int row, int col) {
    if (bw == nullptr) return;
    const int b = min(max(row, 0) >> 4, bw->nbands - 1);
    const int sg = min(max(col, 0) / bw->segw, bw->nseg - 1);
    const int c = *reinterpret_cast<volatile int*>(ready);
    if (c >= 0 && b <= (c >> 12) && sg <= (c & 4095)) return;
    wait_flag(bw->flags + b * bw->nseg + sg, bw->epoch, bw->status, 1, bw->limit);
    if (c < 0 || (b >= (c >> 12) && sg >= (c & 4095))) *reinterpret_cast<volatile int*>(ready) = (b << 12) | sg;
}

// Per-warp shared state: the round's candidates and distortions, and the
// search's cold parameters (read a few times per round, so they live here
// rather than in registers).
struct WarpScratch {
    int2 cand[32];
    int dist[32];
    const uint8_t* base;  // F|H|V|C planes
    int pw, ph, pad, cw, ch, rw, rh;
    int cx, cy;           // mvd centre, predictors[0]
    double lam_r;         // cost's λ (λ/4 for the table kinds)
    double lam_fp;        // cost_fp's λ (λ·RFF_ME_SADL under B2, else λ)
    double lam_me;        // λ itself (the batched sub-pel arms)
    int win_ok;           // the MB's reference window is staged in shared memory
    int wx0, wy0;         // its origin in padded-plane coordinates
    const BandWait* bw;   // the reference's band readiness, or nullptr (complete)
    int bready;           // a reference segment seen complete (band_wait_px)
};

// ---------------------------------------------------------------------------
// Per-MB reference window in shared memory
// ---------------------------------------------------------------------------
// The F|H|V|C planes around the MB's predicted position, copied once per MB by
// the bulk-copy (TMA) engine: WIN_H rows of WIN_W bytes per plane, every
// search of the MB (16x16 and its partitions) then reads its candidates from
// shared memory.  Candidates whose reads leave the window take the plane path
// (pred_rows), which gives the same bytes.  Rows are WIN_STRIDE = 80 bytes
// apart: a block's four rows are then load-immediate offsets of its first, and
// the rows one candidate's 16 lanes read together (four apart) fall in at most
// two lanes per bank.
constexpr int WIN_W = 64, WIN_H = 42, WIN_STRIDE = 80;
constexpr int WIN_PLANE = WIN_H * WIN_STRIDE;  // bytes per plane (a multiple of 16)
constexpr int WIN_BYTES = 4 * WIN_PLANE;
constexpr int WIN_R = 12;  // the window starts this far up/left of the predicted position
constexpr int WIN_OFF = -(1 << 30);  // window offset of a search without one: below -2^29 for any MV, so every read misses

// Rows of the 4x4 block at window position (wx, wy) (full-pel part of the MV
// applied) at phase (fx, fy): the same operand table and averaging as
// pred_rows, read from the staged window at shared address `win`.
__device__ __forceinline__ void win_rows(uint32_t win, int wx, int wy, int fx, int fy, uint32_t out[4]) {
    const uint32_t pb = phase_bits(fx, fy);
    const int pa = int(pb & 3), pbb = int((pb >> 2) & 3);
    const int xa = wx + int((pb >> 4) & 1), ya = wy + int((pb >> 5) & 1);
    const uint32_t a = win + uint32_t(pa * WIN_PLANE + ya * WIN_STRIDE + (xa & ~3));
    const uint32_t sha = uint32_t(xa & 3) * 8u;
#pragma unroll
    for (int r = 0; r < 4; r++) out[r] = __funnelshift_r(lds_u32(a + r * WIN_STRIDE), lds_u32(a + r * WIN_STRIDE + 4), sha);
    if (pbb != 0) {
        const int xb = wx + int((pb >> 6) & 1), yb = wy + int((pb >> 7) & 1);
        const uint32_t b = win + uint32_t(pbb * WIN_PLANE + yb * WIN_STRIDE + (xb & ~3));
        const uint32_t shb = uint32_t(xb & 3) * 8u;
#pragma unroll
        for (int r = 0; r < 4; r++)
            out[r] = avg_up4(out[r], __funnelshift_r(lds_u32(b + r * WIN_STRIDE), lds_u32(b + r * WIN_STRIDE + 4), shb));
    }
}

// Both operands of a block at window position (wx, wy) lie inside the window:
// x reads cover the aligned words from (wx + dx) & ~3 to +8, rows wy + dy ..
// wy + dy + 3, with dx, dy <= 1.
__device__ __forceinline__ bool win_covers(int wx, int wy) {
    return wx >= 0 && ((wx + 1) & ~3) <= WIN_W - 8 && wy >= 0 && wy + 5 <= WIN_H;
}

// Passes whose plane loads are issued together before their SATD: one, since
// the window reads are shared-memory loads and batching passes only costs
// registers.
constexpr int ME_MAX_PASS = 1;

// Register-resident part of one search (every function below is inlined, so
// nothing of it is ever addressed in local memory); the rest is in the
// warp's WarpScratch.
struct SearchGeom {
    int lx, ly, lg_nb, lane, bxo, byo;
    int wox, woy;             // this lane's block at MV (0,0) in window coordinates (WIN_OFF: no window)
    uint32_t win;             // shared address of the warp's window
    uint32_t spa[4], spb[4];  // this lane's source 4x4 rows, split into column pairs
};

__device__ __forceinline__ void geom_init(SearchGeom& g, WarpScratch& ws, const h264a_picture& pc, int x, int y, int w,
                                          int h, uint32_t win) {
    g.lx = x; g.ly = y;
    g.win = win;
    g.lane = threadIdx.x & 31;
    if (g.lane == 0) {
        ws.base = pc.d_planes;
        ws.pad = pc.pad;
        ws.pw = pc.cw + 2 * pc.pad;
        ws.ph = pc.ch + 2 * pc.pad;
        ws.cw = pc.cw;
        ws.ch = pc.ch;
        ws.rw = w;
        ws.rh = h;
    }
    g.lg_nb = (w == 16 ? 2 : (w == 8 ? 1 : 0)) + (h == 16 ? 2 : (h == 8 ? 1 : 0));
    const int nbx = w >> 2;
    const int blk = g.lane & ((1 << g.lg_nb) - 1);
    g.bxo = (blk % nbx) * 4;
    g.byo = (blk / nbx) * 4;
    if (ws.win_ok) {
        g.wox = x + g.bxo + pc.pad - ws.wx0;
        g.woy = y + g.byo + pc.pad - ws.wy0;
    } else {
        g.wox = WIN_OFF;
        g.woy = WIN_OFF;
    }
    uint32_t srow[4];
    // x + bxo is a multiple of 4 and the row lies inside the picture: aligned loads
#pragma unroll
    for (int r = 0; r < 4; r++)
        srow[r] = __ldg(reinterpret_cast<const uint32_t*>(pc.d_src + (long long)(y + g.byo + r) * pc.cw + x + g.bxo));
    split_pairs(srow, g.spa, g.spb);
    __syncwarp();
}

// Distortions of ws.cand[0..n) under `metric` into ws.dist.  All the round's
// plane loads are issued before any is consumed, so a round pays one memory
// latency however many passes it takes.
// Distortions of ws.cand[0..n) added into ws.dist (zeroed by the caller) by
// shared-memory atomics of the lanes' 4x4 blocks.
__device__ __forceinline__ void eval_round(const SearchGeom& g, WarpScratch& ws, int n, int metric) {
    const int npass = ((n << g.lg_nb) + 31) >> 5;
    for (int k0 = 0; k0 < npass; k0 += ME_MAX_PASS) {
    uint32_t pr4[ME_MAX_PASS][4];
#pragma unroll
    for (int kk = 0; kk < ME_MAX_PASS; kk++) {
        const int k = k0 + kk;
        const int c = (32 * k + g.lane) >> g.lg_nb;
        if (k < npass && c < n) {
            const int2 mv = ws.cand[c];
            const int dx = mv.x >> 2, dy = mv.y >> 2;
            const int wx = g.wox + dx, wy = g.woy + dy;
            if (win_covers(wx, wy)) {
                win_rows(g.win, wx, wy, mv.x & 3, mv.y & 3, pr4[kk]);
            } else {
                Planes P;
                P.base = ws.base; P.pw = ws.pw; P.ph = ws.ph; P.pad = ws.pad; P.ps = (long long)ws.pw * ws.ph;
                pred_rows(P, g.lx + g.bxo + dx, g.ly + g.byo + dy, mv.x & 3, mv.y & 3, pr4[kk]);
            }
        }
    }
#pragma unroll
    for (int kk = 0; kk < ME_MAX_PASS; kk++) {
        const int k = k0 + kk;
        if (k < npass) {
            const int c = (32 * k + g.lane) >> g.lg_nb;
            int d = 0;
            if (c < n) {
                if (metric == MET_SAD) {
                    uint32_t srow[4];
#pragma unroll
                    for (int r = 0; r < 4; r++) srow[r] = g.spa[r] | (g.spb[r] << 8);
                    d = sad4x4_rows(srow, pr4[kk]);
                } else {
                    d = satd4x4_packed(g.spa, g.spb, pr4[kk]);
                }
            }
            if (c < n) atomicAdd(&ws.dist[c], d);  // the candidate's blocks, summed in shared memory
        }
    }
    }
    __syncwarp();
}

// Rate of an MV against the search's mvd centre (mb16.rs:2454-2482).
__device__ __forceinline__ uint32_t rate_of(const MeParamsDev& pr, const WarpScratch& ws, int mvx, int mvy) {
    return mvbits(pr.kind, pr.tab, mvx - ws.cx) + mvbits(pr.kind, pr.tab, mvy - ws.cy);
}

// dist + (lam·rate) as i64 for candidate `lane` (< n), held in 32 bits: the
// distortions are below 2^21 and λ·rate below 2^28 for every λ the encoder
// forms (sqrt of 0.85·2^13 times a scale <= 4, rates < 2^17), so the sum
// never saturates and comparisons match the reference's i64.
__device__ __forceinline__ int lane_cost(const MeParamsDev& pr, const WarpScratch& ws, int lane, int n, double lam) {
    if (lane >= n) return INT_MAX;
    const int2 mv = ws.cand[lane];
    const long long c = (long long)ws.dist[lane] + lam_cost(lam, rate_of(pr, ws, mv.x, mv.y));
    return c > INT_MAX - 1 ? INT_MAX - 1 : int(c);
}

// The eight ring points (dx, dy) in the reference's order: (1,0) (-1,0) (0,1)
// (0,-1) (1,1) (-1,-1) (1,-1) (-1,1); the four-point diamond is the first four.
// Packed two bits per point as d+1, so a lane computes its point without a
// memory lookup.
constexpr uint32_t kRingXP = 0x2252u, kRingYP = 0x8225u;
__device__ __forceinline__ int ring_dx(int i) { return int((kRingXP >> (2 * i)) & 3u) - 1; }
__device__ __forceinline__ int ring_dy(int i) { return int((kRingYP >> (2 * i)) & 3u) - 1; }

__device__ __forceinline__ bool in_plane_window(const SearchGeom& g, const WarpScratch& ws, int mvx, int mvy) {
    const int px = g.lx + (mvx >> 2) + ws.pad, py = g.ly + (mvy >> 2) + ws.pad;
    return px >= 0 && py >= 0 && px + ws.rw + 1 <= ws.pw && py + ws.rh + 1 <= ws.ph;
}

// dist + λ·rate of candidate i as the reference's i64 (every lane the same value).
__device__ __forceinline__ long long cand_cost64(const MeParamsDev& pr, const WarpScratch& ws, int i, double lam) {
    const int2 mv = ws.cand[i];
    return (long long)ws.dist[i] + lam_cost(lam, rate_of(pr, ws, mv.x, mv.y));
}

// Search phases and what an evaluation round's results are for.
constexpr int PH_SEEDS = 0, PH_PROP = 1, PH_DIA = 2, PH_REPRICE = 3, PH_SUB = 4, PH_DONE = 5, PH_START = 6;
constexpr int EV_START = 0, EV_SEEDS = 1, EV_PROP = 2, EV_FIXED = 3, EV_RING = 4, EV_REPRICE = 5;
// Candidates of the learned search's proposal round: the median predictor
// and the network's 8 proposals.
constexpr int N_PROP = 8;
constexpr int LOOP_GUARD = 1 << 20;  // iterations of one rung / sub-pel step

// Points of a cascading ring priced per round: the first round prices
// RING_FIRST of them, later rounds (after the centre moved, or none improved)
// up to RING_REST.  A ring of eight sub-pel points usually improves once or
// twice, mostly early, so pricing a few points at a time wastes fewer
// evaluations on points the walk reaches from a different centre; the order
// of the walk and its result do not depend on these sizes.
#ifndef RING_FIRST
#define RING_FIRST 2
#endif
#ifndef RING_REST
#define RING_REST 4
#endif

// motion_search (mb16.rs:2433-3302) of the partition in `g` (warp-cooperative,
// uniform control flow).  preds: npred (x,y) pairs, preds[0] the mvd centre;
// start: refine-only start MV or nullptr.  Returns the reference's evaluation
// count in `evals`.
//
// The search is written as one loop around a single evaluation round, so the
// round's code exists once per kernel: each iteration plans the next batch of
// candidates from the phase state (seeds together with the snaps of sub-pel
// predictors, diamond ladder, B2 reprice, sub-pel rings), prices it, and folds
// the result back into the state.
//  * fixed-centre batches (the FC diamond, sp_fc rings) price all points and
//    take the first strict minimum, like the reference's argmin loops;
//  * cascading rings (the centre moves mid-ring) price the remaining points
//    against the current centre; at the first improvement the centre moves and
//    the points after it are priced again around the new centre, which is the
//    order in which the reference evaluates them.
__device__ __forceinline__ void motion_search_warp(const SearchGeom& g, const MeParamsDev& pr, WarpScratch& ws,
                                                   const int* preds, int npred, const int* start, double lambda_me,
                                                   int& out_x, int& out_y, long long& out_c, int& evals) {
    const bool refine_only = start != nullptr;
    const bool sadfp = !pr.fast && !refine_only && pr.sadfp;
    const int m_main = pr.use_sad ? MET_SAD : MET_SATD;
    if (g.lane == 0) {
        ws.cx = preds[0];
        ws.cy = preds[1];
        ws.lam_me = lambda_me;
        ws.lam_r = pr.kind != 0 ? lambda_me * 0.25 : lambda_me;
        ws.lam_fp = lambda_me * (sadfp ? pr.sadfp_lambda : 1.0);
    }
    // Seeds in ws.cand[0..npred]; with the integer snap on, the snapped
    // position of every sub-pel predictor follows them, so the snap
    // (mb16.rs:2597-2607) is priced in the seed round: slot npred+1+k holds the
    // snap of the k-th sub-pel predictor (bit i of `snaps` set for predictor i).
    unsigned snaps = 0u;
    if (!refine_only) {
        int qx = 0, qy = 0;
        const bool mine = g.lane >= 1 && g.lane <= npred;
        if (mine) {
            qx = preds[2 * (g.lane - 1)];
            qy = preds[2 * (g.lane - 1) + 1];
            ws.cand[g.lane] = make_int2(qx, qy);
        }
        snaps = __ballot_sync(0xffffffffu, pr.me_snap && mine && ((qx & 3) != 0 || (qy & 3) != 0));
        if ((snaps >> g.lane) & 1u)
            ws.cand[npred + 1 + __popc(snaps & ((1u << g.lane) - 1u))] = make_int2(((qx + 2) >> 2) * 4, ((qy + 2) >> 2) * 4);
    }
    __syncwarp();
    const int m_fp = sadfp ? MET_SAD : m_main;
    const double l_fp = sadfp ? ws.lam_fp : ws.lam_r;  // cost_fp's λ (cost's λ when B2 is off)
    const int rw = ws.rw, rh = ws.rh;
    const bool x4shape = (rw == 16 || rw == 8) && (rh == 16 || rh == 8);
    const bool fc = !pr.fast && pr.fc && x4shape;
    const uint32_t dmask = pr.fast ? 0u : ((rw < 8 || rh < 8) ? pr.dia_sub_mask : pr.dia_mask);
    const int spat = pr.subpel_pat >= 0 ? pr.subpel_pat : ((rw < 8 || rh < 8) ? pr.sub_pat : (pr.sp_single_pass ? 2 : 0));
    const bool sp_fc = pr.sp_fc && !pr.fast && x4shape;
    const int sp_nring = (spat & 1) ? 4 : 8;

    evals = 0;
    int bx = 0, by = 0, seed_x = 0, seed_y = 0;
    long long best_c = 0, seed_c = 0;
    int phase = PH_SEEDS;
    int si = -1;        // diamond rung, -1 before the first
    int sk = -1;        // sub-pel step index (0: step 2, 1: step 1), -1 before the first
    int loops = 0;      // iterations of the current rung / sub-pel step
    int iter = 0;       // sub-pel iterations of the current step
    int step = 0;
    bool ring_open = false, ring_improved = false;  // a cascading ring in progress
    int ring_i = 0, ring_n = 0;
    for (;;) {
        // ---------- plan the next round ----------
        int kind = -1, n = 0, metric = m_main;
        double lam = ws.lam_r;
        while (kind < 0 && phase != PH_DONE) {
            if (phase == PH_SEEDS) {
                // seeds (mb16.rs:2580-2596): the start MV, or (0,0) then the predictors
                if (refine_only) {
                    bx = start[0]; by = start[1];
                    if (g.lane == 0) ws.cand[0] = make_int2(bx, by);
                    kind = EV_START; n = 1; metric = m_main; lam = ws.lam_r;
                } else {
                    if (g.lane == 0) ws.cand[0] = make_int2(0, 0);
                    kind = EV_SEEDS; n = npred + 1 + __popc(snaps); metric = m_fp; lam = l_fp;
                }
            } else if (phase == PH_DIA) {
                // diamond ladder (mb16.rs:2616-2727)
                if (ring_open) {
                    kind = EV_RING; n = min(ring_n - ring_i, RING_REST); metric = m_fp; lam = l_fp;
                    if (g.lane < n)
                        ws.cand[g.lane] = make_int2(bx + ring_dx(ring_i + g.lane) * step, by + ring_dy(ring_i + g.lane) * step);
                    break;
                }
                if (si < 0 || loops >= LOOP_GUARD) {
                    // next enabled rung
                    int nsi = si + 1;
                    if (pr.fast) nsi = nsi >= 2 ? 5 : nsi;
                    else
                        while (nsi < 5 && !(dmask & (1u << nsi))) nsi++;
                    if (nsi >= 5) {
                        phase = PH_REPRICE;
                        continue;
                    }
                    si = nsi;
                    step = pr.fast ? (si == 0 ? 16 : 4) : (64 >> si);  // rungs [64,32,16,8,4] quarter-pel
                    loops = 0;
                }
                loops++;
                bool fixed = false;
                if (fc && (bx & 3) == 0 && (by & 3) == 0) {
                    const int st = step >> 2;
                    const int px = g.lx + (bx >> 2), py = g.ly + (by >> 2);
                    fixed = px - st >= 0 && py - st >= 0 && px + st + rw <= ws.cw && py + st + rh <= ws.ch;
                }
                if (g.lane < 4) ws.cand[g.lane] = make_int2(bx + ring_dx(g.lane) * step, by + ring_dy(g.lane) * step);
                if (fixed) {
                    // 16-wide: sad_x4 / satd_x4 batch priced with lam_fp (mb16.rs:2676-2690);
                    // 8-wide shapes price each point with cost_fp (mb16.rs:2691)
                    kind = EV_FIXED; n = 4;
                    metric = rw == 16 ? (sadfp ? MET_SAD : MET_SATD) : m_fp;
                    lam = rw == 16 ? ws.lam_fp : l_fp;
                } else {
                    ring_open = true; ring_improved = false; ring_i = 0; ring_n = 4;
                    kind = EV_RING; n = 4; metric = m_fp; lam = l_fp;
                }
            } else if (phase == PH_REPRICE) {
                // B2 reprice into the SATD domain (mb16.rs:2744-2747)
                if (sadfp) {
                    if (g.lane == 0) {
                        ws.cand[0] = make_int2(bx, by);
                        ws.cand[1] = make_int2(seed_x, seed_y);
                    }
                    kind = EV_REPRICE; n = 2; metric = m_main; lam = ws.lam_r;
                } else {
                    phase = PH_SUB;
                }
            } else {  // PH_SUB: sub-pel rings (mb16.rs:2956-3283)
                if (ring_open) {
                    kind = EV_RING; n = min(ring_n - ring_i, RING_REST); metric = m_main; lam = ws.lam_r;
                    if (g.lane < n)
                        ws.cand[g.lane] = make_int2(bx + ring_dx(ring_i + g.lane) * step, by + ring_dy(ring_i + g.lane) * step);
                    break;
                }
                if (!pr.subpel) {
                    phase = PH_DONE;
                    continue;
                }
                if (sk < 0 || loops >= LOOP_GUARD) {
                    if (++sk >= 2) {
                        phase = PH_DONE;
                        continue;
                    }
                    step = sk == 0 ? 2 : 1;
                    loops = 0;
                    iter = 0;
                }
                loops++;
                if (sp_fc && (spat & 1) == 0 && (step == 1 || ((bx & 3) == 0 && (by & 3) == 0))) {
                    // hpel_qpel_refs / hpel_ref resolve every ring point (inter.rs:1015, 1060):
                    // inside the +1-slack window, and at step 1 a quarter phase
                    bool all = true;
                    for (int i = 0; i < 8; i++) {
                        const int qx = bx + ring_dx(i) * step, qy = by + ring_dy(i) * step;
                        all = all && in_plane_window(g, ws, qx, qy) && (step == 2 || ((qx | qy) & 1));
                    }
                    if (all) {
                        iter++;
                        if (g.lane < 8)
                            ws.cand[g.lane] = make_int2(bx + ring_dx(g.lane) * step, by + ring_dy(g.lane) * step);
                        // 16-wide: satd_avg_x4 / satd_x4p priced with lambda_me; 8-wide: cost()
                        kind = EV_FIXED; n = 8;
                        metric = rw == 16 ? MET_SATD : m_main;
                        lam = rw == 16 ? ws.lam_me : ws.lam_r;
                        break;
                    }
                }
                iter++;
                n = min(sp_nring, RING_FIRST);
                if (g.lane < n)
                    ws.cand[g.lane] = make_int2(bx + ring_dx(g.lane) * step, by + ring_dy(g.lane) * step);
                ring_open = true; ring_improved = false; ring_i = 0; ring_n = sp_nring;
                kind = EV_RING; metric = m_main; lam = ws.lam_r;
            }
        }
        if (kind < 0) break;
        if (g.lane < n) ws.dist[g.lane] = 0;  // eval_round adds each lane's block into its candidate's slot
        __syncwarp();

        // ---------- price the round ----------
        eval_round(g, ws, n, metric);
        const int cc = lane_cost(pr, ws, g.lane, n, lam);

        // ---------- fold the result into the state ----------
        if (kind == EV_START) {
            best_c = cand_cost64(pr, ws, 0, lam);
            evals += 1;
            seed_x = bx; seed_y = by; seed_c = best_c;
            phase = PH_REPRICE;  // refine-only: no snap, no ladder, no B2 reprice; on to the sub-pel rings
        } else if (kind == EV_SEEDS) {
            // sequential strict-< scan: (0,0) first, then the predictors in order
            best_c = __shfl_sync(0xffffffffu, cc, 0);
            bx = 0; by = 0;
            int wi = 0;
            for (int i = 1; i <= npred; i++) {
                const long long ci = __shfl_sync(0xffffffffu, cc, i);
                if (ci < best_c) {
                    best_c = ci;
                    bx = ws.cand[i].x;
                    by = ws.cand[i].y;
                    wi = i;
                }
            }
            evals += npred + 1;
            seed_x = bx; seed_y = by; seed_c = best_c;
            if ((snaps >> wi) & 1u) {
                // the winner is a sub-pel predictor: take its snap, priced in this round
                const int si_ = npred + 1 + __popc(snaps & ((1u << wi) - 1u));
                bx = ws.cand[si_].x; by = ws.cand[si_].y;
                best_c = cand_cost64(pr, ws, si_, lam);
                evals += 1;
            }
            phase = PH_DIA;
        } else if (kind == EV_REPRICE) {
            best_c = cand_cost64(pr, ws, 0, lam);
            seed_c = cand_cost64(pr, ws, 1, lam);
            evals += 2;
            phase = PH_SUB;
        } else if (kind == EV_FIXED) {
            const int m = __reduce_min_sync(0xffffffffu, cc);
            const unsigned at = __ballot_sync(0xffffffffu, cc == m);
            evals += n;
            const int bi = (long long)m < best_c ? __ffs(at) - 1 : -1;
            if (bi >= 0) {
                best_c = m;
                bx += ring_dx(bi) * step;
                by += ring_dy(bi) * step;
            }
            if (phase == PH_DIA) {
                if (bi < 0) loops = LOOP_GUARD;  // rung done
            } else {
                const bool stop = bi < 0 || !pr.me_subpel_iter || (spat & 2) || (pr.sp_maxit != 0 && iter >= pr.sp_maxit);
                if (stop) loops = LOOP_GUARD;  // step done
            }
        } else {  // EV_RING
            const unsigned hit = __ballot_sync(0xffffffffu, g.lane < n && (long long)cc < best_c);
            if (hit == 0) {
                evals += n;
                ring_i += n;
                ring_open = ring_i < ring_n;  // the rest of the ring, around the same centre
            } else {
                const int j = __ffs(hit) - 1;
                best_c = __shfl_sync(0xffffffffu, cc, j);
                const int2 mv = ws.cand[j];
                evals += j + 1;
                bx = mv.x;
                by = mv.y;
                ring_improved = true;
                ring_i += j + 1;
                ring_open = ring_i < ring_n;
            }
            if (!ring_open) {
                if (phase == PH_DIA) {
                    if (!ring_improved) loops = LOOP_GUARD;  // rung done
                } else if (!ring_improved || !pr.me_subpel_iter || (spat & 2) ||
                           (pr.sp_maxit != 0 && iter >= pr.sp_maxit)) {
                    loops = LOOP_GUARD;  // step done
                }
            }
        }
        __syncwarp();
    }
    // ---- seed restore (mb16.rs:3297-3300) ----
    if (pr.me_snap && seed_c < best_c) {
        bx = seed_x; by = seed_y; best_c = seed_c;
    }
    out_x = bx; out_y = by; out_c = best_c;
}

// ---------------------------------------------------------------------------
// Searches of one MB in lane groups
// ---------------------------------------------------------------------------
// The plain-ME frame pass runs best_part's searches of an MB with this one
// search body: first the 16x16 search with the whole warp as one group (one
// lane per 4x4 block, two candidates per pass); then, when the 16x16 J
// exceeds the gate, the four partition searches (16x8 top, 16x8 bottom,
// 8x16 left, 8x16 right) side by side, lane group g = lane / 8 searching
// partition g with one candidate per pass.  The partitions share their seeds
// [pmv, mv16], mvd centre and λ (mb16.rs:8869-8913), so the four searches are
// independent; each group carries its own copy of the search state (the
// state machine of motion_search_warp, every decision taken per group) and
// the warp loops until every group is done.  Candidates and distortions of a
// group live in its slots ws.cand / ws.dist [gb, gb + group size).

struct GroupGeom {
    SearchGeom s;     // the lane's partition origin, its 4x4 block, window offsets, source rows
    int rw, rh;       // partition size
    int gb;           // first slot of the lane's group
    int gl;           // lane within the group
    int lg;           // log2 lanes per group (5: one group, 3: four groups)
    unsigned gmask;   // the group's bits in a ballot, shifted down to bit 0
};

// mode 0: the MB's 16x16 search (one group); mode 1: its four partitions,
// one lane group of 8 each; mode 2: partition `part` (0 16x8 top, 1 16x8
// bottom, 2 8x16 left, 3 8x16 right) with the whole warp as one group, four
// candidates per pass.
// pre: for mode 0, the lane's source rows already loaded (block lane & 15).
__device__ __forceinline__ void group_geom_init(GroupGeom& q, WarpScratch& ws, const h264a_picture& pc, int mx, int my,
                                                int mode, uint32_t win, const uint32_t* pre, int part = 0,
                                                const BandWait* bw = nullptr, int bready = 0) {
    const int lane = threadIdx.x & 31;
    SearchGeom& g = q.s;
    int x = mx, y = my;
    if (mode == 2) {
        q.gb = 0;
        q.gl = lane;
        q.lg = 5;
        q.gmask = 0xffffffffu;
        q.rw = part < 2 ? 16 : 8;
        q.rh = part < 2 ? 8 : 16;
        g.lg_nb = 3;
        x += part == 3 ? 8 : 0;
        y += part == 1 ? 8 : 0;
    } else if (mode == 0) {
        q.gb = 0;
        q.gl = lane;
        q.lg = 5;
        q.gmask = 0xffffffffu;
        q.rw = 16;
        q.rh = 16;
        g.lg_nb = 4;
    } else {
        const int grp = lane >> 3;
        q.gb = grp * 8;
        q.gl = lane & 7;
        q.lg = 3;
        q.gmask = 0xffu;
        q.rw = grp < 2 ? 16 : 8;
        q.rh = grp < 2 ? 8 : 16;
        g.lg_nb = 3;
        x += grp == 3 ? 8 : 0;
        y += grp == 1 ? 8 : 0;
    }
    if (lane == 0) {
        ws.bw = bw;
        ws.bready = bready;
        ws.base = pc.d_planes;
        ws.pad = pc.pad;
        ws.pw = pc.cw + 2 * pc.pad;
        ws.ph = pc.ch + 2 * pc.pad;
        ws.cw = pc.cw;
        ws.ch = pc.ch;
    }
    g.lx = x; g.ly = y;
    g.win = win;
    g.lane = lane;
    const int blk = q.gl & ((1 << g.lg_nb) - 1);
    const int nbx = q.rw >> 2;
    g.bxo = (blk % nbx) * 4;
    g.byo = (blk / nbx) * 4;
    if (ws.win_ok) {
        g.wox = x + g.bxo + pc.pad - ws.wx0;
        g.woy = y + g.byo + pc.pad - ws.wy0;
    } else {
        g.wox = WIN_OFF;
        g.woy = WIN_OFF;
    }
    uint32_t srow[4];
#pragma unroll
    for (int r = 0; r < 4; r++) srow[r] = pre ? pre[r] : ld4u(pc.d_src + (long long)(y + g.byo + r) * pc.cw + x + g.bxo);
    split_pairs(srow, g.spa, g.spb);
    __syncwarp();
}

// Distortions of each group's candidates ws.cand[gb..gb+n) (n and metric per
// group) added into ws.dist, which the caller has zeroed: each lane adds its
// 4x4 block's distortion to its candidate's slot with a shared-memory atomic
// (exact, so the order does not matter), which has a shorter dependency chain
// than a shuffle tree over the candidate's lanes.  A group prices
// 2^(lg - lg_nb) candidates per pass; passes run to the largest need over the
// groups.  SATD_ONLY: the caller's preset never prices with SAD (Balanced).
// TW > 1 (a search run by a team of TW warps with the same state, the wide
// kernel's): warp tw of the team prices, in each pass, the candidates
// [tw * cpw, (tw + 1) * cpw) of that pass's TW * cpw (cpw = the warp's
// candidates per pass), into the team's shared slots `dist` (its own slots
// only).
template <int TW>
__device__ __forceinline__ int team_cand(int k, int cpw, int sub) {
    return (k * TW + int(threadIdx.x >> 5) % TW) * cpw + sub;
}

template <bool SATD_ONLY, int TW = 1>
__device__ __forceinline__ void eval_round_group(const GroupGeom& q, WarpScratch& ws, int n, int metric,
                                                 int* dist = nullptr) {
    constexpr bool COOP = TW > 1;
    const SearchGeom& g = q.s;
    const int cps = q.lg - g.lg_nb;  // log2 candidates per pass of a group
    const int npass = COOP ? (n + (TW << cps) - 1) / (TW << cps)
                           : __reduce_max_sync(0xffffffffu, (n + (1 << cps) - 1) >> cps);
    const int sub = q.gl >> g.lg_nb;  // which of the pass's candidates the lane serves
    for (int k0 = 0; k0 < npass; k0 += ME_MAX_PASS) {
        uint32_t pr4[ME_MAX_PASS][4];
#pragma unroll
        for (int kk = 0; kk < ME_MAX_PASS; kk++) {
            const int c = COOP ? team_cand<TW>(k0 + kk, 1 << cps, sub) : ((k0 + kk) << cps) + sub;
            if (k0 + kk < npass && c < n) {
                const int2 mv = ws.cand[q.gb + c];
                const int dx = mv.x >> 2, dy = mv.y >> 2;
                const int wx = g.wox + dx, wy = g.woy + dy;
                if (win_covers(wx, wy)) {
                    win_rows(g.win, wx, wy, mv.x & 3, mv.y & 3, pr4[kk]);
                } else {
                    band_wait_px(ws.bw, &ws.bready, g.ly + g.byo + dy + 5, g.lx + g.bxo + dx + 5);
                    Planes P;
                    P.base = ws.base; P.pw = ws.pw; P.ph = ws.ph; P.pad = ws.pad; P.ps = (long long)ws.pw * ws.ph;
                    P.cg = ws.bw != nullptr;
                    pred_rows(P, g.lx + g.bxo + dx, g.ly + g.byo + dy, mv.x & 3, mv.y & 3, pr4[kk]);
                }
            }
        }
#pragma unroll
        for (int kk = 0; kk < ME_MAX_PASS; kk++) {
            const int k = k0 + kk;
            if (k < npass) {
                const int c = COOP ? team_cand<TW>(k, 1 << cps, sub) : (k << cps) + sub;
                int d = 0;
                if (c < n) {
                    if (!SATD_ONLY && metric == MET_SAD) {
                        uint32_t srow[4];
#pragma unroll
                        for (int r = 0; r < 4; r++) srow[r] = g.spa[r] | (g.spb[r] << 8);
                        d = sad4x4_rows(srow, pr4[kk]);
                    } else {
                        d = satd4x4_packed(g.spa, g.spb, pr4[kk]);
                    }
                }
                if (c < n) atomicAdd(COOP ? &dist[c] : &ws.dist[q.gb + c], d);  // the candidate's blocks, summed in shared memory
            }
        }
    }
    __syncwarp();
}

__device__ __forceinline__ bool group_in_plane_window(const GroupGeom& q, const WarpScratch& ws, int mvx, int mvy) {
    const int px = q.s.lx + (mvx >> 2) + ws.pad, py = q.s.ly + (mvy >> 2) + ws.pad;
    return px >= 0 && py >= 0 && px + q.rw + 1 <= ws.pw && py + q.rh + 1 <= ws.ph;
}

// motion_search (mb16.rs:2433-3302) of the lane's partition, every group at
// once; same phases, order and pricing as motion_search_warp.
// The search's knobs: read from the parameters, or, for the Balanced preset
// (BAL, h264a_me_params_default), compile-time constants, so that the control
// logic of every round folds to the preset's path.
template <bool BAL>
struct Knobs {
    const MeParamsDev& p;
    __device__ __forceinline__ bool fast() const { return BAL ? false : p.fast != 0; }
    __device__ __forceinline__ bool use_sad() const { return BAL ? false : p.use_sad != 0; }
    __device__ __forceinline__ bool sadfp() const { return BAL ? false : p.sadfp != 0; }
    __device__ __forceinline__ int kind() const { return BAL ? 0 : p.kind; }
    __device__ __forceinline__ bool me_snap() const { return BAL ? true : p.me_snap != 0; }
    __device__ __forceinline__ bool fc() const { return BAL ? true : p.fc != 0; }
    __device__ __forceinline__ uint32_t dia_mask() const { return BAL ? 0x1cu : p.dia_mask; }
    __device__ __forceinline__ bool subpel() const { return BAL ? true : p.subpel != 0; }
    __device__ __forceinline__ int subpel_pat() const { return BAL ? -1 : p.subpel_pat; }
    __device__ __forceinline__ bool sp_single_pass() const { return BAL ? true : p.sp_single_pass != 0; }
    __device__ __forceinline__ bool me_subpel_iter() const { return BAL ? true : p.me_subpel_iter != 0; }
    __device__ __forceinline__ int sp_maxit() const { return BAL ? 0 : p.sp_maxit; }
    __device__ __forceinline__ bool sp_fc() const { return BAL ? false : p.sp_fc != 0; }
    __device__ __forceinline__ double sadfp_lambda() const { return p.sadfp_lambda; }
    // rate of an MV against the search's mvd centre (mb16.rs:2454-2482)
    __device__ __forceinline__ uint32_t rate(const WarpScratch& ws, int mvx, int mvy) const {
        return mvbits(kind(), p.tab, mvx - ws.cx) + mvbits(kind(), p.tab, mvy - ws.cy);
    }
};

// LEARN (the learned-proposal kernels) with use_prop (their 16x16 search): the
// search first prices the median predictor preds[0..1] and the 8 proposals
// (lane gl of the group holds proposal gl - 1 in `prop`) with the search's
// own cost; when the best proposal's distortion exceeds the predictor's by
// more than prop_t it falls back to the plain search (fell = 1), otherwise it
// continues as motion_search with the cheapest of the nine as its start
// vector (mb16.rs:2445, 2579-2596: refine-only, no full-pel phase).
//
// RF / RR: the ring batches (RING_FIRST / RING_REST) of this search; wider
// batches where a pass prices more candidates at once.  TW > 1: the search is
// run by a team of TW consecutive warps with identical state (each warp its
// own `ws`, the same plan and fold), the pricing split between them
// (eval_round_group) into the team's shared distortions cdist[2][32], one
// named barrier (1 + the team's index) per round, the two halves alternating
// by round.
// Named barrier `id` (1..4) over a team of TW warps.  The barrier index is
// an immediate in each branch, so the compiler reserves barriers 1..4 only
// (an index in a register reserves all 16, and the barrier count then caps
// the CTAs per SM).
template <int TW>
__device__ __forceinline__ void team_sync(int id) {
    switch (id) {
        case 1: asm volatile("bar.sync 1, %0;" ::"n"(32 * TW) : "memory"); break;
        case 2: asm volatile("bar.sync 2, %0;" ::"n"(32 * TW) : "memory"); break;
        case 3: asm volatile("bar.sync 3, %0;" ::"n"(32 * TW) : "memory"); break;
        default: asm volatile("bar.sync 4, %0;" ::"n"(32 * TW) : "memory"); break;
    }
}

template <bool BAL, bool LEARN = false, int RF = RING_FIRST, int RR = RING_REST, int TW = 1>
__device__ __forceinline__ void motion_search_group(const GroupGeom& q, const MeParamsDev& prm, WarpScratch& ws,
                                                    const int* preds, int npred, double lambda_me, int& out_x,
                                                    int& out_y, long long& out_c, int& evals, bool use_prop = false,
                                                    int2 prop = make_int2(0, 0), int prop_t = 0, int* fell = nullptr,
                                                    int* cdist = nullptr, bool use_start = false,
                                                    int2 start = make_int2(0, 0)) {
    const Knobs<BAL> pr{prm};
    const int gl = q.gl, gb = q.gb;
    const bool sadfp = !pr.fast() && pr.sadfp();
    const int m_main = pr.use_sad() ? MET_SAD : MET_SATD;
    if (q.s.lane == 0) {
        ws.cx = preds[0];
        ws.cy = preds[1];
        ws.lam_me = lambda_me;
        ws.lam_r = pr.kind() != 0 ? lambda_me * 0.25 : lambda_me;
        ws.lam_fp = lambda_me * (sadfp ? pr.sadfp_lambda() : 1.0);
    }
    // seeds and the snaps of sub-pel predictors (as motion_search_warp), per group
    int qx = 0, qy = 0;
    const bool mine = gl >= 1 && gl <= npred;
    if (mine) {  // npred <= 2: lane 1 the first predictor, lane 2 the second
        qx = gl == 1 ? preds[0] : preds[2];
        qy = gl == 1 ? preds[1] : preds[3];
        ws.cand[gb + gl] = make_int2(qx, qy);
    }
    const unsigned snaps =
        (__ballot_sync(0xffffffffu, pr.me_snap() && mine && ((qx & 3) != 0 || (qy & 3) != 0)) >> gb) & q.gmask;
    if ((snaps >> gl) & 1u)
        ws.cand[gb + npred + 1 + __popc(snaps & ((1u << gl) - 1u))] = make_int2(((qx + 2) >> 2) * 4, ((qy + 2) >> 2) * 4);
    __syncwarp();
    const int m_fp = sadfp ? MET_SAD : m_main;
    const double l_fp = sadfp ? ws.lam_fp : ws.lam_r;
    const int rw = q.rw, rh = q.rh;
    const bool fc = !pr.fast() && pr.fc();  // 16x16, 16x8 and 8x16 are x4 shapes
    const uint32_t dmask = pr.fast() ? 0u : pr.dia_mask();
    const int spat = pr.subpel_pat() >= 0 ? pr.subpel_pat() : (pr.sp_single_pass() ? 2 : 0);
    const bool sp_fc = pr.sp_fc() && !pr.fast();
    const int sp_nring = (spat & 1) ? 4 : 8;

    evals = 0;
    int bx = 0, by = 0, seed_x = 0, seed_y = 0;
    int best_c = 0, seed_c = 0;  // costs below 2^30 (lane_cost), compared as i32
    int phase = (LEARN && use_prop) ? PH_PROP : (use_start ? PH_START : PH_SEEDS);
    int si = -1, sk = -1, loops = 0, iter = 0, step = 0;
    bool ring_open = false, ring_improved = false;
    int ring_i = 0, ring_n = 0;
    constexpr bool COOP = TW > 1;
    const int team_bar = 1 + int(threadIdx.x >> 5) / TW;
    int round = 0;
    for (;;) {
        // the round's distortion slots: the warp's own, or the team's half
        // for this round
        int* const dist = COOP ? cdist + 32 * (round & 1) : ws.dist + gb;
        round++;
        // ---------- plan (per group) ----------
        int kind = -1, n = 0, metric = m_main;
        double lam = ws.lam_r;
        while (kind < 0 && phase != PH_DONE) {
            if (phase == PH_SEEDS) {
                if (gl == 0) ws.cand[gb] = make_int2(0, 0);
                kind = EV_SEEDS; n = npred + 1 + __popc(snaps); metric = m_fp; lam = l_fp;
            } else if (LEARN && phase == PH_PROP) {
                if (gl <= N_PROP) ws.cand[gb + gl] = gl == 0 ? make_int2(preds[0], preds[1]) : prop;
                kind = EV_PROP; n = N_PROP + 1; metric = m_main; lam = ws.lam_r;
            } else if (phase == PH_START) {
                if (gl == 0) ws.cand[gb] = start;
                kind = EV_START; n = 1; metric = m_main; lam = ws.lam_r;
            } else if (phase == PH_DIA) {
                if (ring_open) {
                    kind = EV_RING; n = min(ring_n - ring_i, RR); metric = m_fp; lam = l_fp;
                    if (gl < n)
                        ws.cand[gb + gl] = make_int2(bx + ring_dx(ring_i + gl) * step, by + ring_dy(ring_i + gl) * step);
                    break;
                }
                if (si < 0 || loops >= LOOP_GUARD) {
                    int nsi = si + 1;
                    if (pr.fast()) nsi = nsi >= 2 ? 5 : nsi;
                    else
                        while (nsi < 5 && !(dmask & (1u << nsi))) nsi++;
                    if (nsi >= 5) {
                        phase = PH_REPRICE;
                        continue;
                    }
                    si = nsi;
                    step = pr.fast() ? (si == 0 ? 16 : 4) : (64 >> si);
                    loops = 0;
                }
                loops++;
                bool fixed = false;
                if (fc && (bx & 3) == 0 && (by & 3) == 0) {
                    const int st = step >> 2;
                    const int px = q.s.lx + (bx >> 2), py = q.s.ly + (by >> 2);
                    fixed = px - st >= 0 && py - st >= 0 && px + st + rw <= ws.cw && py + st + rh <= ws.ch;
                }
                if (gl < 4) ws.cand[gb + gl] = make_int2(bx + ring_dx(gl) * step, by + ring_dy(gl) * step);
                if (fixed) {
                    kind = EV_FIXED; n = 4;
                    metric = rw == 16 ? (sadfp ? MET_SAD : MET_SATD) : m_fp;
                    lam = rw == 16 ? ws.lam_fp : l_fp;
                } else {
                    ring_open = true; ring_improved = false; ring_i = 0; ring_n = 4;
                    kind = EV_RING; n = 4; metric = m_fp; lam = l_fp;
                }
            } else if (phase == PH_REPRICE) {
                if (sadfp) {
                    if (gl == 0) {
                        ws.cand[gb] = make_int2(bx, by);
                        ws.cand[gb + 1] = make_int2(seed_x, seed_y);
                    }
                    kind = EV_REPRICE; n = 2; metric = m_main; lam = ws.lam_r;
                } else {
                    phase = PH_SUB;
                }
            } else {  // PH_SUB
                if (ring_open) {
                    kind = EV_RING; n = min(ring_n - ring_i, RR); metric = m_main; lam = ws.lam_r;
                    if (gl < n)
                        ws.cand[gb + gl] = make_int2(bx + ring_dx(ring_i + gl) * step, by + ring_dy(ring_i + gl) * step);
                    break;
                }
                if (!pr.subpel()) {
                    phase = PH_DONE;
                    continue;
                }
                if (sk < 0 || loops >= LOOP_GUARD) {
                    if (++sk >= 2) {
                        phase = PH_DONE;
                        continue;
                    }
                    step = sk == 0 ? 2 : 1;
                    loops = 0;
                    iter = 0;
                }
                loops++;
                if (sp_fc && (spat & 1) == 0 && (step == 1 || ((bx & 3) == 0 && (by & 3) == 0))) {
                    bool all = true;
                    for (int i = 0; i < 8; i++) {
                        const int qx2 = bx + ring_dx(i) * step, qy2 = by + ring_dy(i) * step;
                        all = all && group_in_plane_window(q, ws, qx2, qy2) && (step == 2 || ((qx2 | qy2) & 1));
                    }
                    if (all) {
                        iter++;
                        if (gl < 8) ws.cand[gb + gl] = make_int2(bx + ring_dx(gl) * step, by + ring_dy(gl) * step);
                        kind = EV_FIXED; n = 8;
                        metric = rw == 16 ? MET_SATD : m_main;
                        lam = rw == 16 ? ws.lam_me : ws.lam_r;
                        break;
                    }
                }
                iter++;
                n = min(sp_nring, RF);
                if (gl < n) ws.cand[gb + gl] = make_int2(bx + ring_dx(gl) * step, by + ring_dy(gl) * step);
                ring_open = true; ring_improved = false; ring_i = 0; ring_n = sp_nring;
                kind = EV_RING; metric = m_main; lam = ws.lam_r;
            }
        }
        if (kind < 0) n = 0;
        if (__all_sync(0xffffffffu, kind < 0)) break;
        // which collectives this round's folds need, decided before the pricing
        // (votes off the critical path): the group minimum for fixed-centre
        // rings, the first improvement for cascading rings, the seed costs for
        // the seed and reprice rounds
        const bool need_min = __any_sync(0xffffffffu, kind == EV_FIXED);
        const bool need_hit = __any_sync(0xffffffffu, kind == EV_RING);
        const bool need_seed = __any_sync(0xffffffffu, kind == EV_SEEDS || kind == EV_REPRICE || kind == EV_START);
        if (COOP) {
            // the warp zeroes the slots of the candidates it prices (lane gl
            // < 8: pass gl / cpw, candidate gl % cpw of the warp's share)
            const int cpw = 1 << (q.lg - q.s.lg_nb);
            const int zc = team_cand<TW>(gl / cpw, cpw, gl % cpw);
            if (gl < 8 && zc < n) dist[zc] = 0;
        } else if (gl < n) {
            dist[gl] = 0;  // the pricing adds each lane's block into its candidate's slot
        }
        __syncwarp();
        __syncwarp();

        // ---------- price ----------
        eval_round_group<BAL, TW>(q, ws, n, metric, dist);
        if (COOP) team_sync<TW>(team_bar);
        int cc = INT_MAX;  // dist + λ·rate of slot gb + gl, as lane_cost prices it
        if (gl < n) {
            const int2 mv = ws.cand[gb + gl];
            const long long c = (long long)dist[gl] + lam_cost(lam, pr.rate(ws, mv.x, mv.y));
            cc = c > INT_MAX - 1 ? INT_MAX - 1 : int(c);
        }
        // group-wide collectives, taken by every lane (each only in rounds
        // where some group's fold reads it; the conditions are warp-uniform)
        int gmin = cc;
        unsigned at = 0;
        if (need_min) {
            for (int o = 1; o < (1 << q.lg); o <<= 1) gmin = min(gmin, __shfl_xor_sync(0xffffffffu, gmin, o));
            at = (__ballot_sync(0xffffffffu, cc == gmin) >> gb) & q.gmask;
        }
        unsigned hit = 0;
        int jhit = 0, cj = 0;
        if (need_hit) {
            hit = (__ballot_sync(0xffffffffu, gl < n && cc < best_c) >> gb) & q.gmask;
            jhit = hit ? __ffs(hit) - 1 : 0;
            cj = __shfl_sync(0xffffffffu, cc, gb + jhit);
        }
        int c_seed[3] = {0, 0, 0};
        if (need_seed) {
#pragma unroll
            for (int i = 0; i < 3; i++) c_seed[i] = __shfl_sync(0xffffffffu, cc, gb + i);
        }

        // ---------- fold (per group) ----------
        if (kind == EV_SEEDS) {
            best_c = c_seed[0];
            bx = 0; by = 0;
            int wi = 0;
#pragma unroll
            for (int i = 1; i < 3; i++) {
                const int ci = c_seed[i];
                if (i <= npred && ci < best_c) {
                    best_c = ci;
                    bx = ws.cand[gb + i].x;
                    by = ws.cand[gb + i].y;
                    wi = i;
                }
            }
            evals += npred + 1;
            seed_x = bx; seed_y = by; seed_c = best_c;
            if ((snaps >> wi) & 1u) {
                const int sl = gb + npred + 1 + __popc(snaps & ((1u << wi) - 1u));
                bx = ws.cand[sl].x; by = ws.cand[sl].y;
                best_c = int(((long long)dist[sl - gb] + lam_cost(lam, pr.rate(ws, ws.cand[sl].x, ws.cand[sl].y))));
                evals += 1;
            }
            phase = PH_DIA;
        } else if (kind == EV_START) {
            // a refine-only search (mb16.rs:2580-2582): the start vector
            // priced with `cost`, no full-pel phase, the sub-pel steps from it
            best_c = c_seed[0];
            bx = start.x;
            by = start.y;
            seed_x = bx; seed_y = by; seed_c = best_c;
            evals += 1;
            phase = PH_SUB;
        } else if (LEARN && kind == EV_PROP) {
            // the cheapest of the nine (first wins, the predictor first), and
            // the cheapest proposal's distortion against the predictor's
            int bi = 0, bp = 1;
            long long cbest = 0, cprop = 0;
            for (int i = 0; i <= N_PROP; i++) {
                const int2 mv = ws.cand[gb + i];
                const long long c = (long long)dist[i] + lam_cost(lam, pr.rate(ws, mv.x, mv.y));
                if (i == 0 || c < cbest) { cbest = c; bi = i; }
                if (i == 1 || (i > 1 && c < cprop)) { cprop = c; bp = i; }
            }
            evals += N_PROP + 1;
            const bool fb = (long long)dist[bp] > (long long)dist[0] + prop_t;
            if (fell) *fell = fb ? 1 : 0;
            if (fb) {
                // the plain search's seed slots again (the round above used
                // them; fb is the same in every lane of the 16x16 group)
                __syncwarp();
                if (mine) ws.cand[gb + gl] = make_int2(qx, qy);
                if ((snaps >> gl) & 1u)
                    ws.cand[gb + npred + 1 + __popc(snaps & ((1u << gl) - 1u))] =
                        make_int2(((qx + 2) >> 2) * 4, ((qy + 2) >> 2) * 4);
                phase = PH_SEEDS;
            } else {
                bx = ws.cand[gb + bi].x;
                by = ws.cand[gb + bi].y;
                best_c = cbest > INT_MAX - 1 ? INT_MAX - 1 : int(cbest);
                seed_x = bx; seed_y = by; seed_c = best_c;
                phase = PH_SUB;  // a start vector: no full-pel phase, no B2 reprice
            }
        } else if (kind == EV_REPRICE) {
            best_c = int(((long long)dist[0] + lam_cost(lam, pr.rate(ws, ws.cand[gb].x, ws.cand[gb].y))));
            seed_c = int(((long long)dist[1] + lam_cost(lam, pr.rate(ws, ws.cand[gb + 1].x, ws.cand[gb + 1].y))));
            evals += 2;
            phase = PH_SUB;
        } else if (kind == EV_FIXED) {
            evals += n;
            const int bi = gmin < best_c ? __ffs(at) - 1 : -1;
            if (bi >= 0) {
                best_c = gmin;
                bx += ring_dx(bi) * step;
                by += ring_dy(bi) * step;
            }
            if (phase == PH_DIA) {
                if (bi < 0) loops = LOOP_GUARD;
            } else {
                const bool stop = bi < 0 || !pr.me_subpel_iter() || (spat & 2) || (pr.sp_maxit() != 0 && iter >= pr.sp_maxit());
                if (stop) loops = LOOP_GUARD;
            }
        } else if (kind == EV_RING) {
            if (hit == 0) {
                evals += n;
                ring_i += n;
                ring_open = ring_i < ring_n;
            } else {
                best_c = cj;
                const int2 mv = ws.cand[gb + jhit];
                evals += jhit + 1;
                bx = mv.x;
                by = mv.y;
                ring_improved = true;
                ring_i += jhit + 1;
                ring_open = ring_i < ring_n;
            }
            if (!ring_open) {
                if (phase == PH_DIA) {
                    if (!ring_improved) loops = LOOP_GUARD;
                } else if (!ring_improved || !pr.me_subpel_iter() || (spat & 2) ||
                           (pr.sp_maxit() != 0 && iter >= pr.sp_maxit())) {
                    loops = LOOP_GUARD;
                }
            }
        }
        __syncwarp();
    }
    if (pr.me_snap() && seed_c < best_c) {
        bx = seed_x; by = seed_y; best_c = seed_c;
    }
    out_x = bx; out_y = by; out_c = best_c;
}

__device__ __forceinline__ bool job_shape_ok(int w, int h) {
    return (w == 16 && (h == 16 || h == 8)) || (w == 8 && (h == 16 || h == 8 || h == 4)) ||
           (w == 4 && (h == 8 || h == 4));
}

#ifndef ME_MIN_BLOCKS
#define ME_MIN_BLOCKS 4
#endif

__global__ void __launch_bounds__(32 * ME_WARPS) me_search_kernel(const h264a_picture* __restrict__ pics, int npics,
                                                                 const __grid_constant__ MeParamsDev prm,
                                                                 const h264a_me_job* __restrict__ jobs, int n,
                                                                 h264a_me_result* __restrict__ out) {
    __shared__ WarpScratch scratch[ME_WARPS];
    const int w = threadIdx.x >> 5;
    const long long j = (long long)blockIdx.x * ME_WARPS + w;
    if (j >= n) return;
    const h264a_me_job job = jobs[j];
    h264a_me_result res{};
    const bool ok = job.pic >= 0 && job.pic < npics && job_shape_ok(job.w, job.h) && job.npred >= 1 && job.npred <= 4;
    h264a_picture pc{};
    bool inside = false;
    if (ok) {
        pc = pics[job.pic];
        inside = job.x >= 0 && job.y >= 0 && job.x + job.w <= pc.cw && job.y + job.h <= pc.ch;
    }
    if (!ok || !inside) {
        res.status = -1;
        if ((threadIdx.x & 31) == 0) out[j] = res;
        return;
    }
    if ((threadIdx.x & 31) == 0) scratch[w].win_ok = 0;
    __syncwarp();
    SearchGeom g;
    geom_init(g, scratch[w], pc, job.x, job.y, job.w, job.h, 0u);
    int mx, my, evals;
    long long c;
    motion_search_warp(g, prm, scratch[w], job.preds, job.npred, job.has_start ? job.start : nullptr, job.lambda_me, mx,
                       my, c, evals);
    if ((threadIdx.x & 31) == 0) {
        res.mvx = mx; res.mvy = my; res.cost = c; res.evals = evals; res.status = 0;
        out[j] = res;
    }
}

// ---------------------------------------------------------------------------
// Plain-ME frames: persistent work-queue kernel
// ---------------------------------------------------------------------------

struct FrameDesc {
    // the reference picture's F|H|V|C planes as a 3D tensor (x, y, plane)
    // with an 80 x 42 x 4 box, the shape of an MB's window; tmap_ok 0 means
    // the window is staged row by row instead
    CUtensorMap tmap;
    h264a_picture pic;
    double lambda_me;
    long long split_gate;
    int32_t* picks;
    int64_t* costs;
    int flag_base;
    int mb_w, mb_h;
    // the fused MC + luma T/Q (h264a_me_tq_frames): coefficients out, or
    // nullptr for none, and the frame QP's quant row
    int16_t* coeffs;
    int16_t qff[8], qmf[8];
    // optional row completion (h264a_pixel_path_host): one counter per MB row
    // (zeroed), and a host-visible word per row set to row_token once every
    // MB of the row has its pick and coefficients stored
    int32_t* row_count;
    int32_t* row_done;
    int32_t row_token;
    int32_t tmap_ok;
    // the learned-proposal kernels (h264a_me_frames_learned): 16 i32 per MB
    // of proposals, the fallback threshold, and an optional fallback flag per MB
    const int32_t* props;
    int32_t* fallback;
    int32_t prop_t;
};

// One launch's frames, passed by value.  Frames are sorted by MB count
// (descending) and the work queue deals the k-th MB of every frame that has
// one before the (k+1)-th of any frame: segment j covers positions
// [nmb[j+1], nmb[j]) of frames 0..j, so its tickets are (nmb[j]-nmb[j+1])*(j+1),
// and segments are dealt from j = n-1 (every frame) down to j = 0 (the
// largest frame's tail).  Only the non-empty segments are stored (one per
// distinct frame size): seg_start[s] is the first ticket of segment seg_j[s],
// seg_start[nseg] the ticket count.
// Within a frame the k-th MB is taken in wavefront order (anti-diagonals
// t = x + 2y, then y): every MB's neighbours (left, top, top-left, top-right)
// lie on earlier diagonals, so a window of resident warps always holds MBs
// that are ready, and no MB ever waits on a ticket dealt after its own.
constexpr int ME_MAXF = 96;
// Launches of at most this many frames run the wide kernel (a CTA per MB):
// one frame's wavefront has at most a few dozen ready MBs, far fewer than the
// resident warps, so each MB's own latency is what counts.
constexpr int ME_WIDE_MAXF = 2;
// The pipelined closed loop: the width of a band's column segments in MBs,
// and the number of CTA pools (frames dealt round-robin to them).
#ifndef PIPE_SEGW_MBS
#define PIPE_SEGW_MBS 16
#endif
#ifndef PIPE_POOL_COUNT
#define PIPE_POOL_COUNT 8
#endif
constexpr int PIPE_SEGW = PIPE_SEGW_MBS, PIPE_POOLS = PIPE_POOL_COUNT;
struct FrameBatch {
    FrameDesc f[ME_MAXF];
    long long seg_start[ME_MAXF + 1];
    int seg_j[ME_MAXF];
    int n, nseg;
};
// The frame table as the kernel body reads it: the launch's parameters
// (FrameBatch, up to ME_MAXF frames) or arrays in device memory (any count).
struct ParamTable {
    static constexpr bool kGlobal = false;  // tensor maps in the kernel's parameters
    const FrameBatch& b;
    __device__ __forceinline__ int n() const { return b.n; }
    __device__ __forceinline__ int nseg() const { return b.nseg; }
    __device__ __forceinline__ long long seg(int s) const { return b.seg_start[s]; }
    __device__ __forceinline__ int segj(int s) const { return b.seg_j[s]; }
    __device__ __forceinline__ const FrameDesc& fr(int i) const { return b.f[i]; }
};
struct DeviceTable {
    static constexpr bool kGlobal = true;  // tensor maps in device memory
    const FrameDesc* f;
    const long long* seg_start;
    const int* seg_j;
    int nf, ns;
    __device__ __forceinline__ int n() const { return nf; }
    __device__ __forceinline__ int nseg() const { return ns; }
    __device__ __forceinline__ long long seg(int s) const { return __ldg(seg_start + s); }
    __device__ __forceinline__ int segj(int s) const { return __ldg(seg_j + s); }
    __device__ __forceinline__ const FrameDesc& fr(int i) const { return f[i]; }
};
static_assert(sizeof(FrameBatch) + 512 <= 32764, "me_frames_kernel's parameters must fit the 32 KB parameter space");

// The MV of neighbour MB `m`'s 4x4 block at (bx4, by4) under its pick.
__device__ __forceinline__ int2 pick_mv_at(const int32_t* picks, int m, int bx4, int by4) {
    const int32_t* p = picks + 6 * m;
    const int shape = __ldcg(p);
    const int part = shape == 1 ? (by4 >= 2) : (shape == 2 ? (bx4 >= 2) : 0);
    return make_int2(__ldcg(p + 1 + 2 * part), __ldcg(p + 2 + 2 * part));
}

// predict_mv (inter.rs:36-69) with every available neighbour inter, ref 0.
__device__ __forceinline__ int2 predict_mv_ref0(bool aa, int2 a, bool ba, int2 b, bool ca, int2 c) {
    int2 mva = aa ? a : make_int2(0, 0);
    int2 mvb = ba ? b : make_int2(0, 0);
    int2 mvc = ca ? c : make_int2(0, 0);
    int ra = aa ? 0 : -1, rb = ba ? 0 : -1, rc = ca ? 0 : -1;
    if (!ba && !ca && aa) { mvb = mva; rb = ra; mvc = mva; rc = ra; }
    const int matches = (ra == 0) + (rb == 0) + (rc == 0);
    if (matches == 1) return ra == 0 ? mva : (rb == 0 ? mvb : mvc);
    auto med = [](int x, int y, int z) { return x + y + z - min(min(x, y), z) - max(max(x, y), z); };
    return make_int2(med(mva.x, mvb.x, mvc.x), med(mva.y, mvb.y, mvc.y));
}

// The persistent plain-ME kernel.  Each warp takes MB tickets dealt in
// wavefront order (frames interleaved), waits (bounded, status 1) until the
// MB's left and top-right neighbours are published, derives the median
// predictor from their picks, stages the reference window around it in
// shared memory (one TMA tensor copy, or bulk copies row by row when the
// planes have no tensor map; status 3 if they do not land), runs best_part
// for 16x16 and, when its J exceeds the gate, for the four 16x8/8x16
// partitions (mb16.rs:8869-8913), and publishes the pick (then, for
// h264a_me_tq_frames, the MB's MC + T/Q).  BAL: the Balanced preset's knobs
// as constants.  Dynamic shared memory: ME_WARPS windows of WIN_BYTES.
template <bool BAL, bool LEARN, class TAB>
__device__ __forceinline__ void me_frames_body(const TAB& tab, long long total, const MeParamsDev& prm,
                                               int* __restrict__ counter, int* __restrict__ flags, int epoch,
                                               int* __restrict__ status, int spin_limit) {
    __shared__ WarpScratch scratch[ME_WARPS];
    __shared__ __align__(8) unsigned long long win_bar[ME_WARPS];
    extern __shared__ __align__(128) uint8_t me_win[];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t win = uint32_t(__cvta_generic_to_shared(me_win)) + uint32_t(w * WIN_BYTES);
    const uint32_t bar = uint32_t(__cvta_generic_to_shared(&win_bar[w]));
    if (lane == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    uint32_t parity = 0;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(counter, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) return;
        // the ticket's segment (dealt in order), frame and wavefront position
        int s = 0;
        while (s + 1 < tab.nseg() && tab.seg(s + 1) <= t) s++;
        const int j = tab.segj(s);
        const long long u = t - tab.seg(s);
        const int nxt = j + 1 < tab.n() ? tab.fr(j + 1).mb_w * tab.fr(j + 1).mb_h : 0;
        const FrameDesc& fd = tab.fr(int(u % (j + 1)));
        const int k = nxt + int(u / (j + 1));  // position in the frame's wavefront order
        int mbx, mby;
        wave_mb(fd.mb_w, fd.mb_h, k, mbx, mby);
        const int m = mby * fd.mb_w + mbx;
        int* fl = flags + fd.flag_base;
        const int lx = mbx * 16, ly = mby * 16;
        // the source rows of the lane's 4x4 block in the 16x16 search (block
        // lane & 15), loaded before the neighbour wait: the source is an input
        uint32_t src4[4];
#pragma unroll
        for (int r = 0; r < 4; r++)
            src4[r] = ld4u(fd.pic.d_src + (long long)(ly + ((lane >> 2) & 3) * 4 + r) * fd.pic.cw + lx + (lane & 3) * 4);
        // the learned search's proposal (lanes 1..8), also an input
        int2 prop = make_int2(0, 0);
        if (LEARN && lane >= 1 && lane <= N_PROP) {
            const int32_t* pp = fd.props + 16LL * m + 2 * (lane - 1);
            prop = make_int2(__ldg(pp), __ldg(pp + 1));
        }
        // dependencies: left, and top-right (or top at the right edge)
        if (lane == 0) {
            if (mbx > 0) wait_flag(fl + m - 1, epoch, status, 1, spin_limit);
            if (mby > 0) wait_flag(fl + m - fd.mb_w + (mbx < fd.mb_w - 1 ? 1 : 0), epoch, status, 1, spin_limit);
        }
        __syncwarp();
        // neighbours of the MB's top-left 4x4 block (mv_neighbors_block, mb16.rs:1871)
        const bool aa = mbx > 0, ba = mby > 0, ca = mby > 0 && mbx < fd.mb_w - 1, da = mbx > 0 && mby > 0;
        const int2 a = aa ? pick_mv_at(fd.picks, m - 1, 3, 0) : make_int2(0, 0);
        const int2 bb = ba ? pick_mv_at(fd.picks, m - fd.mb_w, 0, 3) : make_int2(0, 0);
        int2 c = ca ? pick_mv_at(fd.picks, m - fd.mb_w + 1, 0, 3) : make_int2(0, 0);
        bool cav = ca;
        if (!ca) {
            cav = da;
            c = da ? pick_mv_at(fd.picks, m - fd.mb_w - 1, 3, 3) : make_int2(0, 0);
        }
        const int2 pmv = predict_mv_ref0(aa, a, ba, bb, cav, c);
        // stage the window: WIN_R rows/columns up-left of the predicted
        // position, the x origin on a 16-byte boundary (bulk-copy alignment)
        const h264a_picture& pc = fd.pic;
        const int pw = pc.cw + 2 * pc.pad, ph = pc.ch + 2 * pc.pad;
        const bool win_ok = ((reinterpret_cast<uintptr_t>(pc.d_planes) | uintptr_t(pw)) & 15) == 0 && pw >= WIN_W &&
                            ph >= WIN_H;
        if (win_ok) {
            const int wx0 = min(max((lx + pc.pad + (pmv.x >> 2) - WIN_R) & ~15, 0), pw - WIN_W);
            const int wy0 = min(max(ly + pc.pad + (pmv.y >> 2) - WIN_R, 0), ph - WIN_H);
            if (lane == 0) {
                scratch[w].wx0 = wx0;
                scratch[w].wy0 = wy0;
                // the previous MB's window reads are complete (the warp is converged here)
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (fd.tmap_ok) {  // the whole window in one tensor copy
                    mbar_expect_tx(bar, uint32_t(WIN_BYTES));
                    // a tensor map written to device memory by the host since an
                    // earlier launch read that address: acquire it for the copy
                    if (TAB::kGlobal)
                        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&fd.tmap)
                                     : "memory");
                    tma_load_3d(win, &fd.tmap, wx0, wy0, 0, bar);
                } else {
                    mbar_expect_tx(bar, uint32_t(4 * WIN_H * WIN_W));
                }
            }
            __syncwarp();
            if (!fd.tmap_ok) {  // a bulk copy per plane row
                const long long ps = (long long)pw * ph;
                for (int i = lane; i < 4 * WIN_H; i += 32) {
                    const int pl = i / WIN_H, r = i - pl * WIN_H;
                    bulk_g2s(win + uint32_t(pl * WIN_PLANE + r * WIN_STRIDE),
                             pc.d_planes + ps * pl + (long long)(wy0 + r) * pw + wx0, WIN_W, bar);
                }
            }
        }
        if (lane == 0) scratch[w].win_ok = win_ok;
        __syncwarp();
        int preds[4] = {pmv.x, pmv.y, 0, 0};
        // best_part for 16x16 (the warp as one group), then, J above the gate,
        // the four partitions seeded with [pmv, mv16] side by side; one call
        // site, so the search body exists once in the kernel.
        int evals = 0, shape = 0, mv0x = 0, mv0y = 0, mv1x = 0, mv1y = 0, fell = 0;
        long long c16 = 0, best = 0;
        for (int mode = 0; mode < 2; mode++) {
            if (mode == 1 && !(fd.split_gate >= 0 && c16 > fd.split_gate)) break;
            GroupGeom qg;
            group_geom_init(qg, scratch[w], pc, lx, ly, mode, win, mode == 0 ? src4 : nullptr);
            if (mode == 0 && win_ok) {
                wait_window(bar, parity, status, 3, spin_limit);
                parity ^= 1u;
            }
            int rx, ry, ev;
            long long rc;
            // the learned search's partitions, when its 16x16 search took a
            // proposal: refine-only from the 16x16 MV
            const bool lstart = LEARN && mode == 1 && !fell;
            motion_search_group<BAL, LEARN>(qg, prm, scratch[w], preds, mode == 0 ? 1 : 2, fd.lambda_me, rx, ry, rc, ev,
                                            LEARN && mode == 0, prop, fd.prop_t, mode == 0 ? &fell : nullptr, nullptr,
                                            lstart, make_int2(preds[2], preds[3]));
            if (mode == 0) {
                evals = ev << 4;  // 4x4-block evaluations
                c16 = rc; best = rc;
                mv0x = mv1x = rx; mv0y = mv1y = ry;
                preds[2] = rx; preds[3] = ry;
            } else {
                int px[4], py[4];
                long long pcost[4];
#pragma unroll
                for (int gi = 0; gi < 4; gi++) {
                    px[gi] = __shfl_sync(0xffffffffu, rx, 8 * gi);
                    py[gi] = __shfl_sync(0xffffffffu, ry, 8 * gi);
                    pcost[gi] = __shfl_sync(0xffffffffu, rc, 8 * gi);
                    evals += __shfl_sync(0xffffffffu, ev, 8 * gi) << 3;
                }
                if (pcost[0] + pcost[1] < best) {  // 16x8 top + bottom
                    best = pcost[0] + pcost[1]; shape = 1;
                    mv0x = px[0]; mv0y = py[0]; mv1x = px[1]; mv1y = py[1];
                }
                if (pcost[2] + pcost[3] < best) {  // 8x16 left + right
                    best = pcost[2] + pcost[3]; shape = 2;
                    mv0x = px[2]; mv0y = py[2]; mv1x = px[3]; mv1y = py[3];
                }
            }
        }
        if (lane == 0) {
            int32_t* p = fd.picks + 6 * m;
            p[0] = shape; p[1] = mv0x; p[2] = mv0y; p[3] = mv1x; p[4] = mv1y; p[5] = evals;
            fd.costs[2 * m] = best;
            fd.costs[2 * m + 1] = c16;
            if (LEARN && fd.fallback) fd.fallback[m] = fell;
            st_release(fl + m, epoch);  // orders the pick's stores before the flag
        }
        // MC + luma T/Q of the MB under its pick (mb16.rs:3436-3450, as
        // mc_tq_frames_kernel): after the publish, so off the wavefront's
        // path; lane = 4x4 block, the prediction from the staged window
        // when it covers the block's MV.
        if (fd.coeffs != nullptr && lane < 16) {
            const int bx = (lane & 3) * 4, by = (lane >> 2) * 4;
            const int part = shape == 1 ? (by >= 8) : (shape == 2 ? (bx >= 8) : 0);
            const int mvx = part ? mv1x : mv0x, mvy = part ? mv1y : mv0y;
            const int x = lx + bx, y = ly + by;
            uint32_t pr[4];
            const uint32_t* sr = src4;  // lane < 16: the same block as the 16x16 search
            const int wx = x + pc.pad - scratch[w].wx0 + (mvx >> 2), wy = y + pc.pad - scratch[w].wy0 + (mvy >> 2);
            if (win_ok && win_covers(wx, wy)) {
                win_rows(win, wx, wy, mvx & 3, mvy & 3, pr);
            } else {
                Planes P;
                P.base = pc.d_planes; P.pw = pw; P.ph = ph; P.pad = pc.pad; P.ps = (long long)pw * ph;
                pred_rows(P, x + (mvx >> 2), y + (mvy >> 2), mvx & 3, mvy & 3, pr);
            }
            const int qi = (by >= 8 ? 2 : 0) + (bx >= 8 ? 1 : 0), k = ((by & 4) ? 2 : 0) + ((bx & 4) ? 1 : 0);
            tq4x4_store(sr, pr, fd.qff, fd.qmf, fd.coeffs + (long long)m * 256 + qi * 64 + k * 16);
        }
        __syncwarp();  // the lanes' stores ordered before lane 0's count
        if (fd.row_count != nullptr && lane == 0 && atom_add_acq_rel(fd.row_count + mby, 1) == fd.mb_w - 1)
            st_release_sys(fd.row_done + mby, fd.row_token);  // the row's last MB: tell the host
        __syncwarp();
    }
}

// The wide variant for launches of few frames (the closed loop's one frame
// at a time), where the wavefront has far fewer ready MBs than resident warps
// and an MB's own latency is the whole cost: a CTA of ME_WARPS (4) warps takes
// one MB.  Warp 0 waits for the neighbours, stages the window and runs the
// 16x16 search exactly as the narrow kernel does; when the gate opens, warp w
// searches partition w with all 32 lanes (four candidates per pass instead of
// one per 8-lane group), each warp with its own copy of the search state and
// the same seeds, centre and lambda, so every partition's result equals the
// narrow kernel's.  Warp 0 then picks the shape and publishes, as before.
// Dynamic shared memory: one window of WIN_BYTES.
// The closed loop's reconstruction of a frame, fused into the wide kernel:
// after an MB's pick is published, its luma MC + T/Q + reconstruction (warp
// 0), chroma MC + T/Q + reconstruction (warp 1), then the in-loop deblocking
// of the MB (warp 2) in shared tiles, once the deblocking of its left and
// top-right neighbours is done (bounded waits on a second run of flags, the
// same wavefront order as the search).
struct RecDesc {
    const uint8_t* src_c[2];  // the frame's chroma source (U, V)
    const uint8_t* ref_c[2];  // the chroma reconstruction of the previous frame
    uint8_t* rec_y;           // the frame's reconstruction
    uint8_t* rec_c[2];
    int16_t* ccoeffs;         // chroma levels, 128 per MB
    int qp, qpc;              // luma and chroma QP
    int16_t cff[8], cmf[8];   // the chroma QP's quant row (inter dead-zone)
    int dflag_base;           // the deblocking flags' offset in the flag array
    DbThresh th;
};

// The wide kernel's frame table (at most ME_WIDE_MAXF frames), passed by value.
struct WideBatch {
    FrameDesc f[ME_WIDE_MAXF];
    RecDesc rec[ME_WIDE_MAXF];
    long long seg_start[ME_WIDE_MAXF + 1];
    int seg_j[ME_WIDE_MAXF];
    int n, nseg;
};
struct WideTable {
    const WideBatch& b;
    __device__ __forceinline__ int n() const { return b.n; }
    __device__ __forceinline__ int nseg() const { return b.nseg; }
    __device__ __forceinline__ long long seg(int s) const { return b.seg_start[s]; }
    __device__ __forceinline__ int segj(int s) const { return b.seg_j[s]; }
    __device__ __forceinline__ const FrameDesc& fr(int i) const { return b.f[i]; }
    __device__ __forceinline__ const RecDesc& rd(int i) const { return b.rec[i]; }
};

// The wide kernel publishes each MB's pick to the wavefront as three 64-bit
// words, each the launch's epoch (high half) and one MV (x, y as i16, low
// half): the MVs of its blocks (3,0), (0,3) and (3,3), which are what its
// right, lower (and lower-left) and lower-right neighbours' median predictors
// read (mv_neighbors_block, mb16.rs:1871).  A waiting MB polls the words it
// needs until their epoch is the launch's, so the flag and the data arrive in
// one load and no release fence orders anything else.  MVs fit i16 because
// the search keeps every block inside the padded picture (at most 8191
// samples wide or high here).
constexpr int EW_PER_MB = 3;
__device__ __forceinline__ unsigned long long mv_word(int epoch, int x, int y) {
    return ((unsigned long long)(unsigned)epoch << 32) | (uint32_t(uint16_t(x)) | (uint32_t(uint16_t(y)) << 16));
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Waits (bounded; status 1 on timeout) for the word to carry `epoch`; returns its MV.
__device__ __forceinline__ int2 wait_mv_word(const unsigned long long* p, int epoch, int* status, int limit) {
    unsigned long long v = 0;
    for (int it = 0;; it++) {
        asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
        if (int(v >> 32) == epoch) break;
        if (it >= limit || ((it & 255) == 255 && *reinterpret_cast<volatile int*>(status) != 0)) {
            atomicCAS(status, 0, 1);
            break;
        }
        if (it >= 32) __nanosleep(64);
    }
    return make_int2(int(int16_t(v & 0xffffu)), int(int16_t((v >> 16) & 0xffffu)));
}

struct WideMb {
    int pmvx, pmvy;         // the median predictor
    int bready;             // a reference segment seen complete (pipelined loop, band_wait_px)
    long long c16;          // 16x16 J
    int mv16x, mv16y, ev16;
    int px[4], py[4], pev[4];
    long long pc[4];
};

// One MB of the wide kernels (a CTA per MB): the search (16x16 by all warps,
// the partitions one warp each), the pick published to the wavefront as MV
// words, and for h264a_me_tq_frames-style launches the MB's MC + T/Q; REC:
// its reconstruction and deblocking (RecDesc).  ew_frame: the frame's MV
// words; dfl: its deblocking flags; bw: the reference's band readiness
// (pipelined closed loop) or nullptr.  The caller's CTA barrier after the
// call frees the window and the shared state for the next MB.
template <bool BAL, bool LEARN, bool REC>
__device__ __forceinline__ void wide_mb(const FrameDesc& fd, const RecDesc& rd, int mbx, int mby,
                                        const MeParamsDev& prm, unsigned long long* __restrict__ ew_frame,
                                        int* __restrict__ dfl, const BandWait* bw, int epoch, int* __restrict__ status,
                                        int spin_limit, uint32_t win, uint32_t bar, uint32_t& parity,
                                        bool tmap_global = false) {
    __shared__ WarpScratch scratch[ME_WIDE_WARPS];
    __shared__ WideMb mb;
    __shared__ int coop_dist[2][32];     // the team-wide 16x16 search's distortions
    __shared__ int part_dist[4][2][32];  // each partition team's
    // REC: the MB's reconstruction tiles (deblock_device.cuh's layout), its
    // luma blocks' coefficient flags (raster order) and the edges' bS
    __shared__ __align__(16) uint8_t rec_lt[REC ? LT * LT : 4];
    __shared__ __align__(16) uint8_t rec_ct[2][REC ? CR * CT : 4];
    __shared__ int rec_nz[16];
    __shared__ int rec_bs[32];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int m = mby * fd.mb_w + mbx;
    unsigned long long* const ew = ew_frame + EW_PER_MB * m;
    const int lx = mbx * 16, ly = mby * 16;
    const h264a_picture& pc = fd.pic;
    const int pw = pc.cw + 2 * pc.pad, ph = pc.ch + 2 * pc.pad;
    const bool win_ok = ((reinterpret_cast<uintptr_t>(pc.d_planes) | uintptr_t(pw)) & 15) == 0 && pw >= WIN_W &&
                        ph >= WIN_H;
    int preds[4] = {0, 0, 0, 0};
    int fell = 0;
    // every warp's source rows of its lane's 4x4 block in the 16x16 search
    // (block lane & 15) and, for the learned search, its proposal (lane
    // gl holds proposal gl - 1), loaded before the neighbour wait
    uint32_t src4[4];
#pragma unroll
    for (int r = 0; r < 4; r++)
        src4[r] = ld4u(pc.d_src + (long long)(ly + ((lane >> 2) & 3) * 4 + r) * pc.cw + lx + (lane & 3) * 4);
    int2 prop = make_int2(0, 0);
    if (LEARN && lane >= 1 && lane <= N_PROP) {
        const int32_t* pp = fd.props + 16LL * m + 2 * (lane - 1);
        prop = make_int2(__ldg(pp), __ldg(pp + 1));
    }
    if (w == 0) {
        // the neighbours' published MVs: lane 0 the left MB's (3,0), lane
        // 1 the top MB's (0,3), lane 2 the top-right MB's (0,3), lane 3
        // the top-left MB's (3,3) when there is no top-right
        const bool aa = mbx > 0, ba = mby > 0, ca = mby > 0 && mbx < fd.mb_w - 1, da = mbx > 0 && mby > 0;
        const bool need = lane < 4 && (lane == 0 ? aa : (lane == 1 ? ba : (lane == 2 ? ca : (!ca && da))));
        const int dm = lane == 0 ? -EW_PER_MB
                                 : EW_PER_MB * (lane == 1 ? -fd.mb_w : (lane == 2 ? 1 - fd.mb_w : -1 - fd.mb_w));
        const unsigned long long* word = ew + dm + (lane == 0 ? 0 : (lane == 3 ? 2 : 1));
        // The neighbours above were published a row earlier, so the window's
        // origin is guessed from the top MB's MV and its copy overlaps the
        // wait for the left MB (on the wavefront's path).  Any origin gives
        // the same results: candidates the window misses read the planes.
        int2 nv = make_int2(0, 0);
        if (need && (lane > 0 || !ba)) nv = wait_mv_word(word, epoch, status, spin_limit);
        __syncwarp();
        const int2 bb = make_int2(__shfl_sync(0xffffffffu, nv.x, 1), __shfl_sync(0xffffffffu, nv.y, 1));
        const int2 c = make_int2(__shfl_sync(0xffffffffu, nv.x, ca ? 2 : 3), __shfl_sync(0xffffffffu, nv.y, ca ? 2 : 3));
        const int2 guess = ba ? bb : predict_mv_ref0(aa, make_int2(__shfl_sync(0xffffffffu, nv.x, 0),
                                                                   __shfl_sync(0xffffffffu, nv.y, 0)),
                                                     false, bb, false, c);
        if (lane == 0) {
            mb.bready = -1;
            scratch[0].win_ok = win_ok;
        }
        if (win_ok) {
            const int wx0 = min(max((lx + pc.pad + (guess.x >> 2) - WIN_R) & ~15, 0), pw - WIN_W);
            const int wy0 = min(max(ly + pc.pad + (guess.y >> 2) - WIN_R, 0), ph - WIN_H);
            if (lane == 0) {
                scratch[0].wx0 = wx0;
                scratch[0].wy0 = wy0;
                // the window's reference rows are built (pipelined loop), and
                // the generic-proxy writes of them are visible to the copy
                band_wait_px(bw, &mb.bready, wy0 - pc.pad + WIN_H - 1, wx0 - pc.pad + WIN_W - 1);
                if (bw != nullptr) asm volatile("fence.proxy.async.global;" ::: "memory");
                // every warp's reads of the previous MB's window are
                // complete (the CTA barrier at the end of the last MB)
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                if (fd.tmap_ok) {
                    mbar_expect_tx(bar, uint32_t(WIN_BYTES));
                    if (tmap_global)  // a tensor map in device memory, as above (once per frame and CTA)
                        asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&fd.tmap)
                                     : "memory");
                    tma_load_3d(win, &fd.tmap, wx0, wy0, 0, bar);
                } else {
                    mbar_expect_tx(bar, uint32_t(4 * WIN_H * WIN_W));
                }
            }
            __syncwarp();
            if (!fd.tmap_ok) {
                const long long ps = (long long)pw * ph;
                for (int i = lane; i < 4 * WIN_H; i += 32) {
                    const int pl = i / WIN_H, r = i - pl * WIN_H;
                    bulk_g2s(win + uint32_t(pl * WIN_PLANE + r * WIN_STRIDE),
                             pc.d_planes + ps * pl + (long long)(wy0 + r) * pw + wx0, WIN_W, bar);
                }
            }
        }
        if (need && lane == 0 && ba) nv = wait_mv_word(word, epoch, status, spin_limit);
        __syncwarp();
        const int2 a = make_int2(__shfl_sync(0xffffffffu, nv.x, 0), __shfl_sync(0xffffffffu, nv.y, 0));
        const int2 pmv = predict_mv_ref0(aa, a, ba, bb, ca || da, c);
        if (lane == 0) {
            mb.pmvx = pmv.x;
            mb.pmvy = pmv.y;
        }
    }
    __syncthreads();  // the predictor and the window's origin are in shared memory
    if (lane == 0 && w > 0) {
        scratch[w].win_ok = scratch[0].win_ok;
        scratch[w].wx0 = scratch[0].wx0;
        scratch[w].wy0 = scratch[0].wy0;
    }
    __syncwarp();
    preds[0] = mb.pmvx;
    preds[1] = mb.pmvy;
    // the 16x16 search by all warps together (2 * ME_WIDE_WARPS candidates
    // per pass)
    int rx16, ry16, ev16;
    long long c16;
    {
        GroupGeom qg;
        group_geom_init(qg, scratch[w], pc, lx, ly, 0, win, src4, 0, bw, mb.bready);
        if (win_ok) wait_window(bar, parity, status, 3, spin_limit);
        if (win_ok) parity ^= 1u;
        motion_search_group<BAL, LEARN, 2 * ME_WIDE_WARPS, 2 * ME_WIDE_WARPS, ME_WIDE_WARPS>(
            qg, prm, scratch[w], preds, 1, fd.lambda_me, rx16, ry16, c16, ev16, LEARN, prop, fd.prop_t, &fell,
            &coop_dist[0][0]);
    }
    if (w == 0 && lane == 0) {
        mb.c16 = c16;
        mb.mv16x = rx16;
        mb.mv16y = ry16;
        mb.ev16 = ev16 << 4;
    }
    // every warp holds the same 16x16 result: the gate and the partition
    // searches' seeds need no barrier
    const bool gated = fd.split_gate >= 0 && c16 > fd.split_gate;
    if (gated) {
        // partition w / ME_PART_TEAM by its team of warps
        const int part = w / ME_PART_TEAM;
        preds[2] = rx16;
        preds[3] = ry16;
        GroupGeom qg;
        group_geom_init(qg, scratch[w], pc, lx, ly, 2, win, nullptr, part, bw, mb.bready);
        int rx, ry, ev;
        long long rc;
        // the learned search's partitions, when its 16x16 search took a
        // proposal: refine-only from the 16x16 MV
        motion_search_group<BAL, false, 4 * ME_PART_TEAM, 4 * ME_PART_TEAM, ME_PART_TEAM>(
            qg, prm, scratch[w], preds, 2, fd.lambda_me, rx, ry, rc, ev, false, make_int2(0, 0), 0, nullptr,
            &part_dist[part][0][0], LEARN && !fell, make_int2(rx16, ry16));
        if (lane == 0 && w % ME_PART_TEAM == 0) {
            mb.px[part] = rx;
            mb.py[part] = ry;
            mb.pc[part] = rc;
            mb.pev[part] = ev << 3;
        }
    }
    __syncthreads();
    // the shape decision (mb16.rs:8869-8913), taken by every warp from
    // the shared results
    int evals = ev16 << 4, shape = 0;
    int mv0x = rx16, mv0y = ry16, mv1x = rx16, mv1y = ry16;
    long long best = c16;
    if (gated) {
        evals += mb.pev[0] + mb.pev[1] + mb.pev[2] + mb.pev[3];
        if (mb.pc[0] + mb.pc[1] < best) {  // 16x8 top + bottom
            best = mb.pc[0] + mb.pc[1]; shape = 1;
            mv0x = mb.px[0]; mv0y = mb.py[0]; mv1x = mb.px[1]; mv1y = mb.py[1];
        }
        if (mb.pc[2] + mb.pc[3] < best) {  // 8x16 left + right
            best = mb.pc[2] + mb.pc[3]; shape = 2;
            mv0x = mb.px[2]; mv0y = mb.py[2]; mv1x = mb.px[3]; mv1y = mb.py[3];
        }
    }
    if (w == 0) {
        if (lane == 0) {
            int32_t* p = fd.picks + 6 * m;
            p[0] = shape; p[1] = mv0x; p[2] = mv0y; p[3] = mv1x; p[4] = mv1y; p[5] = evals;
            fd.costs[2 * m] = best;
            fd.costs[2 * m + 1] = c16;
            if (LEARN && fd.fallback) fd.fallback[m] = fell;
        }
        // the pick to the wavefront: blocks (3,0), (0,3), (3,3)
        if (lane < EW_PER_MB) {
            const bool second = lane == 0 ? shape == 2 : (lane == 1 ? shape == 1 : shape != 0);
            st_relaxed_u64(ew + lane, mv_word(epoch, second ? mv1x : mv0x, second ? mv1y : mv0y));
        }
        if (fd.coeffs != nullptr && lane < 16) {
            const int bx = (lane & 3) * 4, by = (lane >> 2) * 4;
            const int part = shape == 1 ? (by >= 8) : (shape == 2 ? (bx >= 8) : 0);
            const int mvx = part ? mv1x : mv0x, mvy = part ? mv1y : mv0y;
            const int x = lx + bx, y = ly + by;
            uint32_t sr[4], pr[4];
#pragma unroll
            for (int r = 0; r < 4; r++) sr[r] = ld4u(pc.d_src + (long long)(y + r) * pc.cw + x);
            const int wx = x + pc.pad - scratch[0].wx0 + (mvx >> 2), wy = y + pc.pad - scratch[0].wy0 + (mvy >> 2);
            if (win_ok && win_covers(wx, wy)) {
                win_rows(win, wx, wy, mvx & 3, mvy & 3, pr);
            } else {
                band_wait_px(bw, &scratch[0].bready, y + (mvy >> 2) + 5, x + (mvx >> 2) + 5);
                Planes P;
                P.base = pc.d_planes; P.pw = pw; P.ph = ph; P.pad = pc.pad; P.ps = (long long)pw * ph;
                P.cg = bw != nullptr;
                pred_rows(P, x + (mvx >> 2), y + (mvy >> 2), mvx & 3, mvy & 3, pr);
            }
            const int qi = (by >= 8 ? 2 : 0) + (bx >= 8 ? 1 : 0), kk = ((by & 4) ? 2 : 0) + ((bx & 4) ? 1 : 0);
            int16_t* co = fd.coeffs + (long long)m * 256 + qi * 64 + kk * 16;
            if (REC) {
                // mb16.rs:3575-3605: the luma reconstruction into the tile
                int lv[16];
                tq4x4_store(sr, pr, fd.qff, fd.qmf, co, lv);
                int any = 0;
#pragma unroll
                for (int i = 0; i < 16; i++) any |= lv[i];
                rec_nz[lane] = any != 0;
                uint32_t r4[4];
                rec4x4(lv, pr, rd.qp, r4);
#pragma unroll
                for (int r = 0; r < 4; r++)
                    *reinterpret_cast<uint32_t*>(rec_lt + (4 + by + r) * LT + 4 + bx) = r4[r];
            } else {
                tq4x4_store(sr, pr, fd.qff, fd.qmf, co);
            }
        }
        __syncwarp();
        if (fd.row_count != nullptr && lane == 0 && atom_add_acq_rel(fd.row_count + mby, 1) == fd.mb_w - 1)
            st_release_sys(fd.row_done + mby, fd.row_token);
    }
    if (REC) {
        const int cx0 = mbx * 8, cy0 = mby * 8;
        if (w == 1) {
            // chroma: lanes 0..7 are (plane, block k); lanes 8..31 shadow
            // them so that the quads' shuffles run over the full warp
            const int c = (lane >> 2) & 1, kb = lane & 3;
            const int bx = (kb & 1) * 4, by = (kb >> 1) * 4;
            const int part = shape == 1 ? (by >= 4) : (shape == 2 ? (bx >= 4) : 0);
            const int mvx = part ? mv1x : mv0x, mvy = part ? mv1y : mv0y;
            // the previous reconstruction's chroma rows it reads are final
            // (pipelined loop: band b complete means MB rows 0..b+1 deblocked)
            band_wait_px(bw, &scratch[1].bready, 2 * min(cy0 + by + 4 + (mvy >> 3), pc.ch / 2 - 1) + 1,
                         2 * min(cx0 + bx + 4 + (mvx >> 3), pc.cw / 2 - 1) + 1);
            uint32_t r4[4];
            chroma_tq_rec(rd.src_c[c], rd.ref_c[c], pc.cw / 2, pc.ch / 2, cx0 + bx, cy0 + by, mvx, mvy, kb, rd.qpc,
                          rd.cff, rd.cmf, lane < 8 ? rd.ccoeffs + (long long)m * 128 + c * 64 + kb * 16 : nullptr,
                          r4, bw != nullptr);
            if (lane < 8) {
#pragma unroll
                for (int r = 0; r < 4; r++)
                    *reinterpret_cast<uint32_t*>(&rec_ct[c][(2 + by + r) * CT + 4 + bx]) = r4[r];
            }
        }
        const bool left = mbx > 0, top = mby > 0;
        const DbStrips strips(lane, rd.rec_y, pc.cw, lx, ly, rd.rec_c, cx0, cy0, rec_lt, rec_ct[0], rec_ct[1], left,
                              top, true);
        int nmx = 0, nmy = 0;
        bool nnz = false;
        if (w == 2) {
            // the left and top-right neighbours' deblocking (so the top
            // neighbour's too), then the strips their edges reach and the
            // neighbours' blocks on this MB's edges
            if (lane == 0 && left) wait_flag(dfl + m - 1, epoch, status, 1, spin_limit);
            if (lane == 1 && top)
                wait_flag(dfl + m - fd.mb_w + (mbx < fd.mb_w - 1 ? 1 : 0), epoch, status, 1, spin_limit);
            __syncwarp();
            strips.load();
            if (lane < 4 && left) block_state_at(fd.picks, fd.coeffs, m - 1, 3, lane, nmx, nmy, nnz);
            if (lane >= 16 && lane < 20 && top)
                block_state_at(fd.picks, fd.coeffs, m - fd.mb_w, lane - 16, 3, nmx, nmy, nnz);
        }
        __syncthreads();  // the MB's tiles and coefficient flags are complete
        if (w == 2) {
            // bS: lanes 0..15 the vertical edges (edge e, block row sg),
            // lanes 16..31 the horizontal ones (edge e, block column sg)
            const int hor = lane >> 4, e = (lane >> 2) & 3, sg = lane & 3;
            const int qbx = hor ? sg : e, qby = hor ? e : sg;
            auto own = [&](int bx4, int by4, int& mx, int& my) {
                const int part = shape == 1 ? (by4 >= 2) : (shape == 2 ? (bx4 >= 2) : 0);
                mx = part ? mv1x : mv0x;
                my = part ? mv1y : mv0y;
            };
            int bs = 0;
            if (e > 0 || (hor ? top : left)) {
                int pmx = nmx, pmy = nmy, qmx, qmy;
                bool pnz = nnz;
                if (e > 0) {
                    const int pbx = hor ? sg : e - 1, pby = hor ? e - 1 : sg;
                    own(pbx, pby, pmx, pmy);
                    pnz = rec_nz[pby * 4 + pbx] != 0;
                }
                own(qbx, qby, qmx, qmy);
                bs = bs_of(pnz, rec_nz[qby * 4 + qbx] != 0, pmx, pmy, qmx, qmy);
            }
            rec_bs[lane] = bs;
            __syncwarp();
            deblock_mb_tiles(lane, rec_lt, rec_ct[0], rec_ct[1], rec_bs, left, top, true, rd.th);
            db_store_mb(lane, rec_lt, rec_ct[0], rec_ct[1], rd.rec_y, pc.cw, lx, ly, rd.rec_c, cx0, cy0, true);
            strips.store();
            __syncwarp();  // every lane's stores ordered before lane 0's release
            if (lane == 0) st_release(dfl + m, epoch);
        }
    }
}

template <bool BAL, bool LEARN, bool REC>
__device__ __forceinline__ void me_frames_body_wide(const WideTable& tab, long long total, const MeParamsDev& prm,
                                                    int* __restrict__ counter, int* __restrict__ flags, int epoch,
                                                    int* __restrict__ status, int spin_limit) {
    __shared__ __align__(8) unsigned long long win_bar;
    __shared__ int ticket;
    extern __shared__ __align__(128) uint8_t me_win[];
    const uint32_t win = uint32_t(__cvta_generic_to_shared(me_win));
    const uint32_t bar = uint32_t(__cvta_generic_to_shared(&win_bar));
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t parity = 0;
    for (;;) {
        if (threadIdx.x == 0) ticket = atomicAdd(counter, 1);
        __syncthreads();
        const int t = ticket;
        if (t >= total) return;
        int s = 0;
        while (s + 1 < tab.nseg() && tab.seg(s + 1) <= t) s++;
        const int j = tab.segj(s);
        const long long u = t - tab.seg(s);
        const int nxt = j + 1 < tab.n() ? tab.fr(j + 1).mb_w * tab.fr(j + 1).mb_h : 0;
        const int fi = int(u % (j + 1));
        const FrameDesc& fd = tab.fr(fi);
        const int k = nxt + int(u / (j + 1));
        int mbx, mby;
        wave_mb(fd.mb_w, fd.mb_h, k, mbx, mby);
        const RecDesc& rd = tab.rd(fi);
        wide_mb<BAL, LEARN, REC>(fd, rd, mbx, mby, prm,
                                 reinterpret_cast<unsigned long long*>(flags) + EW_PER_MB * fd.flag_base,
                                 flags + rd.dflag_base, nullptr, epoch, status, spin_limit, win, bar, parity);
        __syncthreads();  // the MB's window and shared state are free for the next ticket
    }
}

template <bool BAL, bool LEARN, bool REC>
__global__ void __launch_bounds__(32 * ME_WIDE_WARPS, ME_MIN_BLOCKS)
    me_frames_wide_kernel(const __grid_constant__ WideBatch batch, long long total,
                          const __grid_constant__ MeParamsDev prm, int* __restrict__ counter, int* __restrict__ flags,
                          int epoch, int* __restrict__ status, int spin_limit) {
    me_frames_body_wide<BAL, LEARN, REC>(WideTable{batch}, total, prm, counter, flags, epoch, status, spin_limit);
}

template <bool BAL, bool LEARN = false>
__global__ void __launch_bounds__(32 * ME_WARPS, ME_MIN_BLOCKS)
    me_frames_kernel(const __grid_constant__ FrameBatch batch, long long total, const __grid_constant__ MeParamsDev prm,
                     int* __restrict__ counter, int* __restrict__ flags, int epoch, int* __restrict__ status,
                     int spin_limit) {
    me_frames_body<BAL, LEARN>(ParamTable{batch}, total, prm, counter, flags, epoch, status, spin_limit);
}

// The same kernel over a frame table in device memory (more than ME_MAXF
// frames in one wavefront launch); the frames' tensor maps are read there.
template <bool BAL, bool LEARN = false>
__global__ void __launch_bounds__(32 * ME_WARPS, ME_MIN_BLOCKS)
    me_frames_dkernel(const FrameDesc* __restrict__ frames, const long long* __restrict__ seg_start,
                      const int* __restrict__ seg_j, int nframes, int nseg, long long total,
                      const __grid_constant__ MeParamsDev prm, int* __restrict__ counter, int* __restrict__ flags,
                      int epoch, int* __restrict__ status, int spin_limit) {
    me_frames_body<BAL, LEARN>(DeviceTable{frames, seg_start, seg_j, nframes, nseg}, total, prm, counter, flags, epoch,
                               status, spin_limit);
}

// One warp waits on a flag that nothing sets; the bounded wait must give up
// after `limit` polls and record status code 2.
// ---------------------------------------------------------------------------
// The pipelined closed loop: every P frame of a clip in one launch
// ---------------------------------------------------------------------------
// Frame h searches the planes of the deblocked reconstruction of frame h-1,
// but an MB only reads the reference pixels its window (and any candidate
// off the window) reaches.  So the launch runs the frames' wavefronts
// overlapped: each frame's tickets are its MBs in wavefront order with
// segment tickets among them.  Segment (b, s) covers picture rows
// 16b .. 16b+15 (band b) and columns 16*segw*s .. (segment s, the first and
// last segments reaching into the padding); its ticket comes after the MB
// whose deblocking makes those reconstruction pixels final, MB
// (min(segw*(s+1), mb_w-1), min(b+1, mb_h-1)) (deblocking runs as a
// wavefront too, so that MB done means every MB up and left of it is), and
// builds the planes of the segment (hpel_strip_rows, its own columns only).
// An MB of frame h waits (bounded) for the segments of frame h-1 its reads
// need (band_wait_px); a segment's flag is published after the flags of the
// segments above and left of it, so one flag stands for all of those.  The
// next frame can therefore start a few MB columns and rows behind the
// previous one instead of a whole frame width behind.  The planes of nbuf
// consecutive frames live in nbuf buffers (frame h's in buffer h % nbuf),
// and a segment ticket of frame h first waits until frame h-nbuf+1, the last
// reader of the buffer's previous picture, has finished every MB.
//
// Deadlock freedom: the CTAs form `pools` pools, block i taking frames
// 1 + i % pools, 1 + i % pools + pools, ..., each pool its frames in order, a
// CTA moving to the pool's next frame only once the current frame's tickets
// are all dealt.  A ticket waits only on earlier tickets of its own frame, on
// frame h-1 and on frame h-nbuf+1's completion; the oldest unfinished frame
// therefore depends on nothing unfinished, its tickets are all dealt or held
// by CTAs of its own pool that are not blocked by a later frame, and it
// always progresses.  Every wait is still bounded, and after the first
// timeout the others give up (status 1).
struct PipeParams {
    const FrameDesc* fds;  // per frame 0..n-1 (entry 0 unused), in device memory
    const RecDesc* rds;
    const int* items;      // a frame's tickets: MB index, or -(1 + b * nseg + s)
    int nitems, n, mb_w, mb_h, nbands, nseg, segw, nbuf, pools;
    int* flags;            // per frame fstride ints: MV words, deblocking flags, segment flags
    long long fstride;
    int ew_off, dfl_off, band_off;
    int* ctr;              // n ticket counters and n completed-MB counters, zeroed
    int* done;
    const uint8_t* rec_y;  // frame h's luma reconstruction at h * fs
    long long fs;
    uint8_t* planes;       // nbuf plane buffers, pbytes apart
    long long pbytes;
    int cw, ch, pad, word_in, word_out;
    int32_t* frame_words;  // mapped host words: frame h's set to ftoken when it is final (or null)
    int32_t ftoken;
    const int32_t* arrive;  // frame h's sources uploaded once arrive[h] == atoken (or null: all resident)
    int32_t atoken;
};

// Segment (b, s) of frame h: the planes of its reconstruction for padded rows
// [pad + 16b, pad + 16b + 16) (band 0 from row 0, the last band to the end)
// and padded columns [pad + 16*segw*s, pad + 16*segw*(s+1)) (segment 0 from
// column 0, the last segment to the end), into buffer h % nbuf.
__device__ __forceinline__ void pipe_band(const PipeParams& pp, int h, int b, int sg, int epoch, int* status,
                                          int limit) {
    int* const ff = pp.flags + pp.fstride * h;
    if (threadIdx.x == 0) {
        const int r = min(b + 1, pp.mb_h - 1), x = min(pp.segw * (sg + 1), pp.mb_w - 1);
        wait_flag(ff + pp.dfl_off + r * pp.mb_w + x, epoch, status, 1, limit);
        if (h - pp.nbuf + 1 >= 1) {
            const int nmb = pp.mb_w * pp.mb_h;
            for (int it = 0; ld_acquire(pp.done + h - pp.nbuf + 1) < nmb; it++) {
                if (it >= limit || ((it & 255) == 255 && *reinterpret_cast<volatile int*>(status) != 0)) {
                    atomicCAS(status, 0, 1);
                    break;
                }
                __nanosleep(200);
            }
        }
    }
    __syncthreads();
    const int pw = pp.cw + 2 * pp.pad, ph = pp.ch + 2 * pp.pad;
    const int y0 = b == 0 ? 0 : pp.pad + 16 * b;
    const int y1 = b == pp.nbands - 1 ? ph : pp.pad + 16 * b + 16;
    const int x0 = sg == 0 ? 0 : pp.pad + 16 * pp.segw * sg;
    const int x1 = sg == pp.nseg - 1 ? pw : pp.pad + 16 * pp.segw * (sg + 1);
    for (int st = x0 / HP_STRIP + int(threadIdx.x >> 5); st * HP_STRIP < x1; st += ME_WIDE_WARPS)
        hpel_strip_rows<true>(pp.rec_y + pp.fs * h, pp.cw, pp.ch, pp.pad, pp.planes + pp.pbytes * (h % pp.nbuf), pw,
                              ph, st, y0, y1, pp.word_in, pp.word_out, x0, x1);
    // the planes' generic-proxy writes, visible to the readers' bulk copies
    asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
        int* const sf = ff + pp.band_off + b * pp.nseg + sg;
        if (b > 0) wait_flag(sf - pp.nseg, epoch, status, 1, limit);
        if (sg > 0) wait_flag(sf - 1, epoch, status, 1, limit);
        st_release(sf, epoch);
    }
}

#ifndef PIPE_MIN_BLOCKS
#define PIPE_MIN_BLOCKS ME_MIN_BLOCKS
#endif
template <bool BAL, bool LEARN>
__global__ void __launch_bounds__(32 * ME_WIDE_WARPS, PIPE_MIN_BLOCKS)
    closed_pipe_kernel(const __grid_constant__ PipeParams pp, const __grid_constant__ MeParamsDev prm, int epoch,
                       int* __restrict__ status, int spin_limit) {
    __shared__ __align__(8) unsigned long long win_bar;
    __shared__ int ticket;
    __shared__ BandWait bwait;
    extern __shared__ __align__(128) uint8_t me_win[];
    const uint32_t win = uint32_t(__cvta_generic_to_shared(me_win));
    const uint32_t bar = uint32_t(__cvta_generic_to_shared(&win_bar));
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t parity = 0;
    int fenced = -1;   // the frame whose tensor maps this CTA has acquired
    int arrived = -1;  // the frame whose sources this CTA has seen uploaded
    int h = 1 + int(blockIdx.x % unsigned(pp.pools));  // this CTA's pool: frames h, h + pools, ...
    while (h < pp.n) {
        if (threadIdx.x == 0) ticket = atomicAdd(pp.ctr + h, 1);
        __syncthreads();
        const int t = ticket;
        if (t >= pp.nitems) {
            h += pp.pools;  // every ticket of frame h is dealt: the pool's next frame
            __syncthreads();
            continue;
        }
        const int item = __ldg(pp.items + t);
        int* const ff = pp.flags + pp.fstride * h;
        if (item >= 0) {
            if (threadIdx.x == 0) {
                if (pp.arrive != nullptr && arrived != h) {
                    // the frame's sources are still being uploaded beside the launch
                    for (int it = 0; ld_acquire(pp.arrive + h) != pp.atoken; it++) {
                        if (it >= spin_limit ||
                            ((it & 255) == 255 && *reinterpret_cast<volatile int*>(status) != 0)) {
                            atomicCAS(status, 0, 1);
                            break;
                        }
                        __nanosleep(200);
                    }
                }
                bwait.flags = pp.flags + pp.fstride * (h - 1) + pp.band_off;
                bwait.nbands = pp.nbands;
                bwait.nseg = pp.nseg;
                bwait.segw = 16 * pp.segw;
                bwait.epoch = epoch;
                bwait.limit = spin_limit;
                bwait.status = status;
            }
            __syncthreads();
            // frame 1's reference (frame 0) is built before the launch
            wide_mb<BAL, LEARN, true>(pp.fds[h], pp.rds[h], item % pp.mb_w, item / pp.mb_w, prm,
                                      reinterpret_cast<unsigned long long*>(ff + pp.ew_off), ff + pp.dfl_off,
                                      h > 1 ? &bwait : nullptr, epoch, status, spin_limit, win, bar, parity,
                                      fenced != h);
            fenced = h;
            arrived = h;
            __syncthreads();  // every read and write of the MB is done
            if (threadIdx.x == 0) {
                const int c = atom_add_acq_rel(pp.done + h, 1);
                if (c == pp.mb_w * pp.mb_h - 1 && pp.frame_words != nullptr) {
                    // the frame's last MB: its outputs are final, for the host
                    __threadfence_system();
                    st_release_sys(pp.frame_words + h, pp.ftoken);
                }
            }
        } else {
            pipe_band(pp, h, (-item - 1) / pp.nseg, (-item - 1) % pp.nseg, epoch, status, spin_limit);
        }
        __syncthreads();  // the window and shared state are free for the next ticket
    }
}

__global__ void bounded_wait_selftest_kernel(const int* flag, int* status, int limit) {
    if (threadIdx.x == 0) wait_flag(flag, 1, status, 2, limit);
}

}  // namespace h264a

using namespace h264a;

namespace h264a {
int encode_u8_map_3d(CUtensorMap* map, const uint8_t* base, int w, int h, int d, int bw, int bh, int bd) {
    static const PFN_cuTensorMapEncodeTiled_v12000 encode = [] {  // looked up once, thread-safely
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
        cudaGetLastError();
        return PFN_cuTensorMapEncodeTiled_v12000(nullptr);
    }();
    if (!encode || (reinterpret_cast<uintptr_t>(base) & 15) != 0 || w % 16 != 0 || bw % 16 != 0 || w < bw || h < bh ||
        d < bd || bw > 256 || bh > 256 || bd > 256 || bd < 1)
        return 0;
    const cuuint64_t dim[3] = {cuuint64_t(w), cuuint64_t(h), cuuint64_t(d)};
    const cuuint64_t stride[2] = {cuuint64_t(w), cuuint64_t(w) * cuuint64_t(h)};  // bytes, dims 1 and 2
    const cuuint32_t box[3] = {cuuint32_t(bw), cuuint32_t(bh), cuuint32_t(bd)};
    const cuuint32_t estride[3] = {1, 1, 1};
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<uint8_t*>(base), dim, stride, box, estride,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS
               ? 1
               : 0;
}
}  // namespace h264a

// The F|H|V|C planes of a reference picture as a 3D u8 tensor (pw, ph, 4)
// whose 80 x 42 x 4 box is an MB's window in the WIN_STRIDE / WIN_PLANE
// layout.  Returns 0 when the planes cannot be described (alignment, or no
// driver entry point), and the kernel then stages the window row by row.
static int encode_window_map(CUtensorMap* map, const uint8_t* planes, int pw, int ph) {
    static_assert(WIN_STRIDE % 16 == 0 && WIN_PLANE == WIN_H * WIN_STRIDE && WIN_BYTES == 4 * WIN_PLANE,
                  "the window is one dense 3D box");
    return encode_u8_map_3d(map, planes, pw, ph, 4, WIN_STRIDE, WIN_H, 4);
}

// Dynamic shared memory of me_frames_kernel, its opt-in above 48 KB, and the
// CTAs per SM it reaches.
static int me_frames_setup_once(int& per_sm, bool learn);
// Cached per device: the attributes and the occupancy of the frame kernels
// (queried once, not on every launch).
static int me_frames_setup(int& per_sm, bool learn = false) {
    constexpr int kMaxDev = 64;
    static int cached[kMaxDev][2];  // CTAs per SM + 1, 0 while unknown
    static std::mutex mu;
    int dev = 0;
    H264A_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDev) return me_frames_setup_once(per_sm, learn);
    std::lock_guard<std::mutex> lock(mu);
    int& c = cached[dev][learn ? 1 : 0];
    if (!c) {
        const int rc = me_frames_setup_once(per_sm, learn);
        if (rc) return rc;
        c = per_sm + 1;
    }
    per_sm = c - 1;
    return H264A_OK;
}

static int me_frames_setup_once(int& per_sm, bool learn) {
    const int smem = ME_WARPS * WIN_BYTES;
    H264A_CUDA(cudaFuncSetAttribute(me_frames_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(me_frames_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(me_frames_dkernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(me_frames_dkernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(me_frames_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(me_frames_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(me_frames_dkernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(me_frames_dkernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    per_sm = 0;
    if (learn)
        H264A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, me_frames_kernel<false, true>, 32 * ME_WARPS,
                                                                 smem));
    else
        H264A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, me_frames_kernel<false>, 32 * ME_WARPS, smem));
    if (per_sm < 1) per_sm = 1;
    return H264A_OK;
}

// True when the parameters are the Balanced preset's (h264a_me_params_default):
// the frame kernel then runs its instance with those knobs as constants.
static bool balanced_preset(const MeParamsDev& p) {
    return p.fast == 0 && p.use_sad == 0 && p.sadfp == 0 && p.kind == 0 && p.me_snap == 1 && p.fc == 1 &&
           p.dia_mask == 0x1cu && p.subpel == 1 && p.subpel_pat == -1 && p.sp_single_pass == 1 &&
           p.me_subpel_iter == 1 && p.sp_maxit == 0 && p.sp_fc == 0;
}

// The non-empty segments of the ticket order of nf frames sorted by MB count,
// descending: segment j (positions [nmb(j+1), nmb(j)) of frames 0..j) has
// (nmb(j) - nmb(j+1)) * (j+1) tickets, and segments are dealt from
// j = nf-1 down.  Writes their first tickets (start[nseg] = the ticket count,
// which equals the frames' MB count) and j values; returns nseg.
static int make_segments(const FrameDesc* f, int nf, long long* start, int* segj) {
    long long acc = 0;
    int ns = 0;
    for (int j = nf - 1; j >= 0; j--) {
        const long long nj = (long long)f[j].mb_w * f[j].mb_h;
        const long long nn = j + 1 < nf ? (long long)f[j + 1].mb_w * f[j + 1].mb_h : 0;
        if (nj == nn) continue;
        start[ns] = acc;
        segj[ns] = j;
        ns++;
        acc += (nj - nn) * (j + 1);
    }
    start[ns] = acc;
    return ns;
}

// fb.nseg and the segment arrays of a batch of fb.n sorted frames; returns the
// ticket count.
static long long fill_segments(FrameBatch& fb) {
    fb.nseg = make_segments(fb.f, fb.n, fb.seg_start, fb.seg_j);
    return fb.seg_start[fb.nseg];
}

static void launch_me_frames_dtab(const MeParamsDev& prm, unsigned blocks, cudaStream_t st, const FrameDesc* frames,
                                  const long long* seg_start, const int* seg_j, int nframes, int nseg, long long total,
                                  int* counter, int* flags, int epoch, int* status, bool learn = false) {
    const size_t sm = ME_WARPS * WIN_BYTES;
    const bool bal = balanced_preset(prm);
    if (learn && bal)
        me_frames_dkernel<true, true><<<blocks, 32 * ME_WARPS, sm, st>>>(frames, seg_start, seg_j, nframes, nseg, total,
                                                                        prm, counter, flags, epoch, status, SPIN_LIMIT);
    else if (learn)
        me_frames_dkernel<false, true><<<blocks, 32 * ME_WARPS, sm, st>>>(frames, seg_start, seg_j, nframes, nseg, total,
                                                                         prm, counter, flags, epoch, status, SPIN_LIMIT);
    else if (bal)
        me_frames_dkernel<true><<<blocks, 32 * ME_WARPS, sm, st>>>(frames, seg_start, seg_j, nframes, nseg, total, prm,
                                                                  counter, flags, epoch, status, SPIN_LIMIT);
    else
        me_frames_dkernel<false><<<blocks, 32 * ME_WARPS, sm, st>>>(frames, seg_start, seg_j, nframes, nseg, total, prm,
                                                                   counter, flags, epoch, status, SPIN_LIMIT);
}

// CTAs per SM of the wide kernel (one window per CTA), cached per device
static int me_wide_setup_once(int& per_sm);
static int me_wide_setup(int& per_sm) {
    constexpr int kMaxDev = 64;
    static int cached[kMaxDev];
    static std::mutex mu;
    int dev = 0;
    H264A_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDev) return me_wide_setup_once(per_sm);
    std::lock_guard<std::mutex> lock(mu);
    if (!cached[dev]) {
        const int rc = me_wide_setup_once(per_sm);
        if (rc) return rc;
        cached[dev] = per_sm + 1;
    }
    per_sm = cached[dev] - 1;
    return H264A_OK;
}

template <bool BAL, bool LEARN, bool REC>
static int wide_attr(int smem) {
    H264A_CUDA(cudaFuncSetAttribute(me_frames_wide_kernel<BAL, LEARN, REC>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return H264A_OK;
}

static int me_wide_setup_once(int& per_sm) {
    const int smem = WIN_BYTES;
    int rc = wide_attr<false, false, false>(smem) | wide_attr<true, false, false>(smem) |
             wide_attr<false, true, false>(smem) | wide_attr<true, true, false>(smem) |
             wide_attr<false, false, true>(smem) | wide_attr<true, false, true>(smem) |
             wide_attr<false, true, true>(smem) | wide_attr<true, true, true>(smem);
    if (rc) return rc;
    // the residency of the largest variant bounds the grid of every one
    per_sm = 0;
    H264A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, me_frames_wide_kernel<false, true, true>,
                                                             32 * ME_WIDE_WARPS, smem));
    int p2 = 0;
    H264A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p2, me_frames_wide_kernel<false, true, false>,
                                                             32 * ME_WIDE_WARPS, smem));
    if (p2 < per_sm) per_sm = p2;
    if (per_sm < 1) per_sm = 1;
    return H264A_OK;
}

template <bool REC>
static void launch_wide_t(const MeParamsDev& prm, unsigned blocks, cudaStream_t st, const WideBatch& wb,
                          long long total, int* counter, int* flags, int epoch, int* status, bool learn) {
    const size_t sm = WIN_BYTES;
    const bool bal = balanced_preset(prm);
    if (learn && bal)
        me_frames_wide_kernel<true, true, REC><<<blocks, 32 * ME_WIDE_WARPS, sm, st>>>(wb, total, prm, counter, flags,
                                                                                 epoch, status, SPIN_LIMIT);
    else if (learn)
        me_frames_wide_kernel<false, true, REC><<<blocks, 32 * ME_WIDE_WARPS, sm, st>>>(wb, total, prm, counter, flags,
                                                                                  epoch, status, SPIN_LIMIT);
    else if (bal)
        me_frames_wide_kernel<true, false, REC><<<blocks, 32 * ME_WIDE_WARPS, sm, st>>>(wb, total, prm, counter, flags,
                                                                                  epoch, status, SPIN_LIMIT);
    else
        me_frames_wide_kernel<false, false, REC><<<blocks, 32 * ME_WIDE_WARPS, sm, st>>>(wb, total, prm, counter, flags,
                                                                                   epoch, status, SPIN_LIMIT);
}

static void launch_me_frames_wide(const MeParamsDev& prm, unsigned blocks, cudaStream_t st, const WideBatch& wb,
                                  long long total, int* counter, int* flags, int epoch, int* status, bool learn,
                                  bool rec) {
    if (rec)
        launch_wide_t<true>(prm, blocks, st, wb, total, counter, flags, epoch, status, learn);
    else
        launch_wide_t<false>(prm, blocks, st, wb, total, counter, flags, epoch, status, learn);
}

static void launch_me_frames(const MeParamsDev& prm, unsigned blocks, cudaStream_t st, const FrameBatch& fb,
                             long long total, int* counter, int* flags, int epoch, int* status, bool learn = false) {
    const size_t sm = ME_WARPS * WIN_BYTES;
    const bool bal = balanced_preset(prm);
    if (learn && bal)
        me_frames_kernel<true, true><<<blocks, 32 * ME_WARPS, sm, st>>>(fb, total, prm, counter, flags, epoch, status,
                                                                       SPIN_LIMIT);
    else if (learn)
        me_frames_kernel<false, true><<<blocks, 32 * ME_WARPS, sm, st>>>(fb, total, prm, counter, flags, epoch, status,
                                                                        SPIN_LIMIT);
    else if (bal)
        me_frames_kernel<true><<<blocks, 32 * ME_WARPS, sm, st>>>(fb, total, prm, counter, flags, epoch, status,
                                                                 SPIN_LIMIT);
    else
        me_frames_kernel<false><<<blocks, 32 * ME_WARPS, sm, st>>>(fb, total, prm, counter, flags, epoch, status,
                                                                  SPIN_LIMIT);
}

extern "C" int h264a_selftest_bounded_wait(h264a_ctx* ctx, int spin_limit, void* stream) {
    if (!ctx || spin_limit < 0 || spin_limit > SPIN_LIMIT) return fail(H264A_E_ARG, "selftest_bounded_wait: bad limit");
    int rc = ensure_me_scratch(ctx, 1);
    if (rc) return rc;
    cudaStream_t st = pick_stream(ctx, stream);
    // the counter word is zero-initialised scratch that no kernel of this call writes
    H264A_CUDA(cudaMemsetAsync(ctx->q[Q_MAIN].d_counter, 0, sizeof(int32_t), st));
    bounded_wait_selftest_kernel<<<1, 32, 0, st>>>(ctx->q[Q_MAIN].d_counter, ctx->d_status, spin_limit);
    return check_launch("bounded_wait_selftest_kernel");
}

extern "C" int h264a_me_search(h264a_ctx* ctx, const h264a_picture* d_pics, int npics, const h264a_me_params* params,
                               const h264a_me_job* d_jobs, int n, h264a_me_result* d_out, void* stream) {
    if (!ctx || !d_pics || !params || !d_jobs || !d_out) return fail(H264A_E_ARG, "me_search: null pointer");
    if (n < 0 || npics < 1) return fail(H264A_E_ARG, "me_search: bad count");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !params->d_mv_cost_tab)
        return fail(H264A_E_ARG, "me_search: mv cost kinds 1 and 2 need d_mv_cost_tab");
    if (n == 0) return H264A_OK;
    const MeParamsDev prm = to_dev(*params);
    me_search_kernel<<<unsigned((n + ME_WARPS - 1) / ME_WARPS), 32 * ME_WARPS, 0, pick_stream(ctx, stream)>>>(
        d_pics, npics, prm, d_jobs, n, d_out);
    return check_launch("me_search_kernel");
}

// Plain-ME of a batch of frames (h264a_me_frames); with `tq`, each frame's
// MC + luma T/Q is fused in (h264a_me_tq_frames, h264a_pixel_path_host).
// A frame table's pinned staging buffer (at least `bytes`), then its upload
// into the device copy on `st`; table_done after the launch that reads it
// records the event both wait for before they are reused.
static int table_host(h264a_ctx* ctx, size_t bytes, char** host) {
    if (!ctx->me_tab_ev) H264A_CUDA(cudaEventCreateWithFlags(&ctx->me_tab_ev, cudaEventDisableTiming));
    H264A_CUDA(cudaEventSynchronize(ctx->me_tab_ev));
    if (bytes > ctx->me_tab_cap) {
        if (ctx->me_tab) cudaFree(ctx->me_tab);
        if (ctx->me_tab_host) cudaFreeHost(ctx->me_tab_host);
        ctx->me_tab = ctx->me_tab_host = nullptr;
        ctx->me_tab_cap = 0;
        if (cudaMalloc(&ctx->me_tab, bytes) != cudaSuccess || cudaMallocHost(&ctx->me_tab_host, bytes) != cudaSuccess) {
            cudaGetLastError();
            return fail(H264A_E_NOMEM, "frame table allocation failed");
        }
        ctx->me_tab_cap = bytes;
    }
    *host = static_cast<char*>(ctx->me_tab_host);
    return H264A_OK;
}
static int table_upload(h264a_ctx* ctx, size_t bytes, cudaStream_t st) {
    H264A_CUDA(cudaMemcpyAsync(ctx->me_tab, ctx->me_tab_host, bytes, cudaMemcpyHostToDevice, st));
    return H264A_OK;
}
static int table_done(h264a_ctx* ctx, cudaStream_t st) {
    H264A_CUDA(cudaEventRecord(ctx->me_tab_ev, st));
    return H264A_OK;
}

int h264a::me_frames_run(h264a_ctx* ctx, const h264a_me_frame* h_frames, int nframes,
                         const h264a_me_params* params, const MeTqOut* tq, void* stream, const MeLearnIn* learn,
                         const MeRecIn* rec) {
    if (!ctx || !h_frames || !params) return fail(H264A_E_ARG, "me_frames: null pointer");
    if (nframes < 1) return fail(H264A_E_ARG, "me_frames: need at least one frame");
    if (rec && (!tq || nframes > ME_WIDE_MAXF))
        return fail(H264A_E_ARG, "me_frames: the fused reconstruction needs T/Q outputs and at most two frames");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !params->d_mv_cost_tab)
        return fail(H264A_E_ARG, "me_frames: mv cost kinds 1 and 2 need d_mv_cost_tab");
    for (int i = 0; i < nframes; i++) {
        const h264a_me_frame& f = h_frames[i];
        if (!f.pic.d_src || !f.pic.d_planes || !f.d_picks || !f.d_costs)
            return fail(H264A_E_ARG, "me_frames: null frame pointer");
        if (f.pic.cw < 16 || f.pic.ch < 16 || f.pic.cw % 16 || f.pic.ch % 16 || f.pic.pad < 3 || f.pic.pad > 128)
            return fail(H264A_E_ARG, "me_frames: frames must be MB-aligned with 3 <= pad <= 128");
        if ((long long)(f.pic.cw / 16) * (f.pic.ch / 16) > (1 << 24))
            return fail(H264A_E_ARG, "me_frames: frame too large");
    }
    cudaStream_t st = pick_stream(ctx, stream);
    const MeParamsDev prm = to_dev(*params);
    int per_sm = 0;
    int rc0 = me_frames_setup(per_sm, learn != nullptr);
    if (rc0) return rc0;
    // One wavefront launch over all frames, largest first: the frame table in
    // the kernel's parameters up to ME_MAXF frames, in device memory beyond.
    std::vector<int> order(nframes);
    for (int i = 0; i < nframes; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (long long)h_frames[a].pic.cw * h_frames[a].pic.ch > (long long)h_frames[b].pic.cw * h_frames[b].pic.ch;
    });
    std::vector<FrameDesc> desc(nframes);
    memset(desc.data(), 0, sizeof(FrameDesc) * nframes);
    RecDesc rdesc[ME_WIDE_MAXF];
    memset(rdesc, 0, sizeof rdesc);
    long long total = 0;
    for (int k = 0; k < nframes; k++) {
        const h264a_me_frame& f = h_frames[order[k]];
        FrameDesc& d = desc[k];
        d.pic = f.pic;
        d.tmap_ok = encode_window_map(&d.tmap, f.pic.d_planes, f.pic.cw + 2 * f.pic.pad, f.pic.ch + 2 * f.pic.pad);
        d.lambda_me = f.lambda_me;
        d.split_gate = f.split_gate;
        d.picks = f.d_picks;
        d.costs = f.d_costs;
        d.mb_w = f.pic.cw / 16;
        d.mb_h = f.pic.ch / 16;
        d.flag_base = int(total);
        if (tq) {
            const MeTqOut& t = tq[order[k]];
            d.coeffs = t.coeffs;
            make_quant_row4(t.qp, t.dz_div, d.qff, d.qmf);
            d.row_count = t.row_count;
            d.row_done = t.row_done;
            d.row_token = t.row_token;
        }
        if (learn) {
            const MeLearnIn& l = learn[order[k]];
            d.props = l.props;
            d.fallback = l.fallback;
            d.prop_t = l.prop_t;
        }
        if (rec) {
            const MeRecIn& r = rec[order[k]];
            if (!r.src_u || !r.src_v || !r.ref_u || !r.ref_v || !r.rec_y || !r.rec_u || !r.rec_v || !r.ccoeffs)
                return fail(H264A_E_ARG, "me_frames: null reconstruction pointer");
            if (((reinterpret_cast<uintptr_t>(r.src_u) | reinterpret_cast<uintptr_t>(r.src_v) |
                  reinterpret_cast<uintptr_t>(r.ref_u) | reinterpret_cast<uintptr_t>(r.ref_v) |
                  reinterpret_cast<uintptr_t>(r.rec_y) | reinterpret_cast<uintptr_t>(r.rec_u) |
                  reinterpret_cast<uintptr_t>(r.rec_v)) & 3) ||
                ((reinterpret_cast<uintptr_t>(r.ccoeffs) | reinterpret_cast<uintptr_t>(tq[order[k]].coeffs)) & 15))
                return fail(H264A_E_ARG, "me_frames: planes must be 4-byte and levels 16-byte aligned");
            const int qp = tq[order[k]].qp;
            if (qp < 0 || qp > 51) return fail(H264A_E_ARG, "me_frames: qp out of 0..51");
            RecDesc& rd = rdesc[k];
            rd.src_c[0] = r.src_u; rd.src_c[1] = r.src_v;
            rd.ref_c[0] = r.ref_u; rd.ref_c[1] = r.ref_v;
            rd.rec_y = r.rec_y;
            rd.rec_c[0] = r.rec_u; rd.rec_c[1] = r.rec_v;
            rd.ccoeffs = r.ccoeffs;
            rd.qp = qp;
            rd.qpc = chroma_qp_of(qp);
            make_quant_row4(rd.qpc, 6, rd.cff, rd.cmf);  // chroma: the inter dead-zone
            rd.th = db_thresholds(qp, 0, 0, 0);
        }
        total += (long long)d.mb_w * d.mb_h;
        if (total >= (1LL << 31)) return fail(H264A_E_ARG, "me_frames: too many macroblocks in one call");
    }
    std::vector<long long> seg(nframes + 1);
    std::vector<int> segj(nframes);
    const int nseg = make_segments(desc.data(), nframes, seg.data(), segj.data());
    if (seg[nseg] != total) return fail(H264A_E_ARG, "me_frames: internal queue layout error");
    // The wide kernel (launches of at most ME_WIDE_MAXF frames) publishes MV
    // words (2 * EW_PER_MB ints per MB), then the fused reconstruction's
    // deblocking flags, in its own queue's flag space (cleared per launch);
    // its MVs are packed as i16, so the padded pictures must be at most 8191
    // samples wide and high.
    bool wide = nframes <= ME_WIDE_MAXF;
    for (int k = 0; k < nframes; k++)
        if (desc[k].pic.cw + 2 * desc[k].pic.pad > 8191 || desc[k].pic.ch + 2 * desc[k].pic.pad > 8191) wide = false;
    if (rec && !wide) return fail(H264A_E_ARG, "me_frames: the fused reconstruction needs pictures of at most 8191 - 2 pad samples");
    if (wide) {
        // few frames: a CTA per MB, the partitions one warp each
        const size_t nflags = size_t(2 * EW_PER_MB + (rec ? 1 : 0)) * size_t(total);
        int rc = ensure_me_scratch(ctx, nflags, Q_WIDE);
        if (rc) return rc;
        WorkQueue& qw = ctx->q[Q_WIDE];
        H264A_CUDA(cudaMemsetAsync(qw.d_counter, 0, sizeof(int32_t), st));
        H264A_CUDA(cudaMemsetAsync(qw.d_flags, 0, sizeof(int32_t) * nflags, st));
        const int epoch = next_epoch(ctx, st, Q_WIDE);
        if (epoch < 0) return H264A_E_CUDA;
        int wide_sm = 0;
        rc0 = me_wide_setup(wide_sm);
        if (rc0) return rc0;
        long long wblocks = (long long)ctx->num_sms * wide_sm;
        if (wblocks > total) wblocks = total;
        WideBatch wb;
        memset(&wb, 0, sizeof wb);
        wb.n = nframes;
        memcpy(wb.f, desc.data(), sizeof(FrameDesc) * nframes);
        for (int k = 0; k < nframes; k++) {
            wb.rec[k] = rdesc[k];
            wb.rec[k].dflag_base = int(2 * EW_PER_MB * total) + desc[k].flag_base;
        }
        wb.nseg = make_segments(wb.f, wb.n, wb.seg_start, wb.seg_j);
        if (wb.seg_start[wb.nseg] != total) return fail(H264A_E_ARG, "me_frames: internal queue layout error");
        launch_me_frames_wide(prm, unsigned(wblocks), st, wb, total, qw.d_counter, qw.d_flags, epoch, ctx->d_status,
                              learn != nullptr, rec != nullptr);
        return check_launch("me_frames_wide_kernel");
    }
    int rc = ensure_me_scratch(ctx, size_t(total));
    if (rc) return rc;
    H264A_CUDA(cudaMemsetAsync(ctx->q[Q_MAIN].d_counter, 0, sizeof(int32_t), st));
    const int epoch = next_epoch(ctx, st);
    if (epoch < 0) return H264A_E_CUDA;
    long long blocks = (long long)ctx->num_sms * per_sm;
    const long long need = (total + ME_WARPS - 1) / ME_WARPS;
    if (blocks > need) blocks = need;
    if (nframes <= ME_MAXF) {
        FrameBatch fb;
        memset(&fb, 0, sizeof fb);
        fb.n = nframes;
        memcpy(fb.f, desc.data(), sizeof(FrameDesc) * nframes);
        if (fill_segments(fb) != total) return fail(H264A_E_ARG, "me_frames: internal queue layout error");
        launch_me_frames(prm, unsigned(blocks), st, fb, total, ctx->q[Q_MAIN].d_counter, ctx->q[Q_MAIN].d_flags, epoch,
                         ctx->d_status, learn != nullptr);
        return check_launch("me_frames_kernel");
    }
    // the table, its segment starts and j values in one device buffer
    const size_t b_desc = sizeof(FrameDesc) * nframes, b_seg = sizeof(long long) * (nseg + 1),
                 b_j = sizeof(int) * nseg, bytes = b_desc + b_seg + b_j;
    char* hst = nullptr;
    rc = table_host(ctx, bytes, &hst);
    if (rc) return rc;
    memcpy(hst, desc.data(), b_desc);
    memcpy(hst + b_desc, seg.data(), b_seg);
    memcpy(hst + b_desc + b_seg, segj.data(), b_j);
    rc = table_upload(ctx, bytes, st);
    if (rc) return rc;
    char* dv = static_cast<char*>(ctx->me_tab);
    launch_me_frames_dtab(prm, unsigned(blocks), st, reinterpret_cast<const FrameDesc*>(dv),
                          reinterpret_cast<const long long*>(dv + b_desc), reinterpret_cast<const int*>(dv + b_desc + b_seg),
                          nframes, nseg, total, ctx->q[Q_MAIN].d_counter, ctx->q[Q_MAIN].d_flags, epoch, ctx->d_status,
                          learn != nullptr);
    rc = check_launch("me_frames_dkernel");
    if (rc) return rc;
    return table_done(ctx, st);
}

extern "C" int h264a_me_frames(h264a_ctx* ctx, const h264a_me_frame* h_frames, int nframes,
                               const h264a_me_params* params, void* stream) {
    return me_frames_run(ctx, h_frames, nframes, params, nullptr, stream);
}

extern "C" int h264a_me_frames_learned(h264a_ctx* ctx, const h264a_me_learned_frame* h_frames, int nframes,
                                       const h264a_me_params* params, void* stream) {
    if (!ctx || !h_frames || !params) return fail(H264A_E_ARG, "me_frames_learned: null pointer");
    if (nframes < 1) return fail(H264A_E_ARG, "me_frames_learned: need at least one frame");
    std::vector<h264a_me_frame> me(nframes);
    std::vector<MeLearnIn> ln(nframes);
    for (int i = 0; i < nframes; i++) {
        const h264a_me_learned_frame& f = h_frames[i];
        if (!f.d_props) return fail(H264A_E_ARG, "me_frames_learned: null proposals");
        if (f.fallback_t < 0) return fail(H264A_E_ARG, "me_frames_learned: negative fallback threshold");
        me[i] = f.me;
        ln[i] = MeLearnIn{f.d_props, f.d_fallback, f.fallback_t};
    }
    return me_frames_run(ctx, me.data(), nframes, params, nullptr, stream, ln.data());
}

extern "C" int h264a_me_tq_frames(h264a_ctx* ctx, const h264a_me_tq_frame* h_frames, int nframes,
                                  const h264a_me_params* params, void* stream) {
    if (!ctx || !h_frames || !params) return fail(H264A_E_ARG, "me_tq_frames: null pointer");
    if (nframes < 1) return fail(H264A_E_ARG, "me_tq_frames: need at least one frame");
    std::vector<h264a_me_frame> me(nframes);
    std::vector<MeTqOut> tq(nframes);
    for (int i = 0; i < nframes; i++) {
        const h264a_me_tq_frame& f = h_frames[i];
        if (!f.d_coeffs || (reinterpret_cast<uintptr_t>(f.d_coeffs) & 15) != 0)
            return fail(H264A_E_ARG, "me_tq_frames: coefficients must be non-null and 16-byte aligned");
        if (f.qp < 0 || f.qp > 51 || f.dz_div < 1) return fail(H264A_E_ARG, "me_tq_frames: qp out of 0..51 or dz_div < 1");
        me[i] = f.me;
        tq[i] = MeTqOut{f.d_coeffs, f.qp, f.dz_div, nullptr, nullptr, 0};
    }
    return me_frames_run(ctx, me.data(), nframes, params, tq.data(), stream);
}

// ---------------------------------------------------------------------------
// Plain-ME frames without any allocation
// ---------------------------------------------------------------------------
//
// Some callers cannot allocate device memory at the moment they run motion
// estimation: a real-time encoder thread that must not block on the CUDA
// allocator (cudaMalloc can synchronise the device and take a global lock),
// or a host application that hands this library a fixed memory budget and
// owns every buffer itself.  h264a_me_frames needs a context, and the
// context allocates the persistent kernel's scratch (the work-queue counter
// and one done flag per macroblock).  The entry below runs the same kernel
// with that scratch taken from this fixed array instead: one counter word
// plus one flag word per macroblock, for at most H264A_NOALLOC_MAX_MBS
// macroblocks per call (256 KiB per device, held by every device that loads
// the library until the process exits).

namespace h264a {

// [0] work-queue counter, [1..] per-MB done flags.
static __device__ __align__(256) int g_noalloc_scratch[1 + H264A_NOALLOC_MAX_MBS];

// The device address of g_noalloc_scratch on each device (nullptr: not yet
// looked up).  It is looked up once per device and kept; a caller that resets
// a device's primary context (cudaDeviceReset) must not call this entry point
// on that device again in the same process.
struct NoallocDevice {
    int* scratch;
};
constexpr int kNoallocMaxDevices = 64;
constexpr int kNoallocFlag = 1;  // the value a published MB's flag takes
static NoallocDevice g_noalloc_dev[kNoallocMaxDevices];
static std::mutex g_noalloc_mu;

}  // namespace h264a

extern "C" int h264a_me_frames_noalloc(const h264a_me_frame* h_frames, int nframes, const h264a_me_params* params,
                                       int32_t* d_status, void* stream) {
    if (!h_frames || !params || !d_status) return fail(H264A_E_ARG, "me_frames_noalloc: null pointer");
    if (nframes < 1 || nframes > ME_MAXF)
        return fail(H264A_E_ARG, "me_frames_noalloc: 1 to " + std::to_string(ME_MAXF) + " frames per call");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !params->d_mv_cost_tab)
        return fail(H264A_E_ARG, "me_frames_noalloc: mv cost kinds 1 and 2 need d_mv_cost_tab");
    long long total = 0;
    for (int i = 0; i < nframes; i++) {
        const h264a_me_frame& f = h_frames[i];
        if (!f.pic.d_src || !f.pic.d_planes || !f.d_picks || !f.d_costs)
            return fail(H264A_E_ARG, "me_frames_noalloc: null frame pointer");
        if (f.pic.cw < 16 || f.pic.ch < 16 || f.pic.cw % 16 || f.pic.ch % 16 || f.pic.pad < 3 || f.pic.pad > 128)
            return fail(H264A_E_ARG, "me_frames_noalloc: frames must be MB-aligned with 3 <= pad <= 128");
        total += (long long)(f.pic.cw / 16) * (f.pic.ch / 16);
    }
    if (total > H264A_NOALLOC_MAX_MBS)
        return fail(H264A_E_ARG, "me_frames_noalloc: " + std::to_string(total) + " macroblocks exceed the " +
                                     std::to_string(H264A_NOALLOC_MAX_MBS) + "-macroblock scratch of this entry point");
    int dev = 0;
    H264A_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoallocMaxDevices) return fail(H264A_E_ARG, "me_frames_noalloc: device index too large");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int* scratch;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        NoallocDevice& nd = g_noalloc_dev[dev];
        if (!nd.scratch) {
            // first call on this device: the array's device address (the
            // symbol itself is only a host-side stand-in)
            void* p = nullptr;
            H264A_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            nd.scratch = static_cast<int*>(p);
        }
        scratch = nd.scratch;
    }
    // frames largest first, dealt round-robin in wavefront order (as h264a_me_frames)
    int order[ME_MAXF];
    for (int i = 0; i < nframes; i++) order[i] = i;
    for (int i = 1; i < nframes; i++) {  // stable insertion sort by size, descending
        const int v = order[i];
        const long long sv = (long long)h_frames[v].pic.cw * h_frames[v].pic.ch;
        int k = i;
        while (k > 0 && (long long)h_frames[order[k - 1]].pic.cw * h_frames[order[k - 1]].pic.ch < sv) {
            order[k] = order[k - 1];
            k--;
        }
        order[k] = v;
    }
    FrameBatch fb;
    memset(&fb, 0, sizeof fb);
    fb.n = nframes;
    total = 0;
    for (int k = 0; k < nframes; k++) {
        const h264a_me_frame& f = h_frames[order[k]];
        FrameDesc& d = fb.f[k];
        d.pic = f.pic;
        d.tmap_ok = encode_window_map(&d.tmap, f.pic.d_planes, f.pic.cw + 2 * f.pic.pad, f.pic.ch + 2 * f.pic.pad);
        d.lambda_me = f.lambda_me;
        d.split_gate = f.split_gate;
        d.picks = f.d_picks;
        d.costs = f.d_costs;
        d.mb_w = f.pic.cw / 16;
        d.mb_h = f.pic.ch / 16;
        d.flag_base = int(total);
        total += (long long)d.mb_w * d.mb_h;
    }
    fill_segments(fb);
    // The counter, this call's flags and the caller's status word start at
    // zero: they are cleared on the stream ahead of the launch (at most
    // 256 KiB), and each MB's flag is set to 1 when its pick is published.
    // Nothing of an earlier call's array contents is read.
    H264A_CUDA(cudaMemsetAsync(scratch, 0, sizeof(int) * size_t(1 + total), st));
    H264A_CUDA(cudaMemsetAsync(d_status, 0, sizeof(int32_t), st));
    int per_sm = 0, sms = 0;
    const int rc0 = me_frames_setup(per_sm);
    if (rc0) return rc0;
    H264A_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    long long blocks = (long long)sms * per_sm;
    const long long need = (total + ME_WARPS - 1) / ME_WARPS;
    if (blocks > need) blocks = need;
    const MeParamsDev prm = to_dev(*params);
    launch_me_frames(prm, unsigned(blocks), st, fb, total, scratch, scratch + 1, kNoallocFlag, d_status);
    return check_launch("me_frames_kernel (no-alloc)");
}

// ---------------------------------------------------------------------------
// The pipelined closed loop's launch
// ---------------------------------------------------------------------------

static int closed_pipe_setup_once() {
    const int smem = WIN_BYTES;
    H264A_CUDA(cudaFuncSetAttribute(closed_pipe_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(closed_pipe_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(closed_pipe_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    H264A_CUDA(cudaFuncSetAttribute(closed_pipe_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    return H264A_OK;
}

// The per-device kernel attributes and the CTAs per SM of the pipelined loop.
static int closed_pipe_setup(int& per_sm) {
    constexpr int kMaxDev = 64;
    static int cached[kMaxDev];
    static std::mutex mu;
    int dev = 0;
    H264A_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 0 || dev >= kMaxDev || !cached[dev]) {
        int rc = closed_pipe_setup_once();
        if (rc) return rc;
        int p = 0;
        H264A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, closed_pipe_kernel<false, true>,
                                                                 32 * ME_WIDE_WARPS, WIN_BYTES));
        if (p < 1) p = 1;
        if (dev < 0 || dev >= kMaxDev) {
            per_sm = p;
            return H264A_OK;
        }
        cached[dev] = p;
    }
    per_sm = cached[dev];
    return H264A_OK;
}

int h264a::closed_pipe_run(h264a_ctx* ctx, const ClosedPipeIn& in, const h264a_me_params* params, cudaStream_t st,
                           int32_t* frame_words, int32_t token) {
    const int n = in.n, cw = in.cw, ch = in.ch, pad = in.pad;
    const int pw = cw + 2 * pad, ph = ch + 2 * pad;
    if (n < 2) return H264A_OK;
    if (pw > 8191 || ph > 8191) return fail(H264A_E_ARG, "closed loop: pictures too large for the pipelined loop");
    const int mb_w = cw / 16, mb_h = ch / 16, nmb = mb_w * mb_h, nbands = mb_h;
    const long long fs = (long long)cw * ch, cs = fs / 4, pbytes = 4LL * pw * ph;
    const MeParamsDev prm = to_dev(*params);
    int per_sm = 0;
    int rc = closed_pipe_setup(per_sm);
    if (rc) return rc;
    // the frame and reconstruction descriptors (entry 0 unused)
    std::vector<FrameDesc> fds(n);
    std::vector<RecDesc> rds(n);
    memset(fds.data(), 0, sizeof(FrameDesc) * n);
    memset(rds.data(), 0, sizeof(RecDesc) * n);
    // the plane buffers (frame h's planes in buffer h % nbuf), the column
    // segments of the bands, the CTA pools
    const int nbuf = std::min(n, H264A_CLOSED_PLANE_PICTURES);
    const int segw = PIPE_SEGW, nseg = (mb_w + segw - 1) / segw;
    const int pools = std::min(PIPE_POOLS, n - 1);
    if (pad % 4) return fail(H264A_E_ARG, "closed loop: the plane padding must be a multiple of 4");
    std::vector<CUtensorMap> maps(nbuf);
    std::vector<int> maps_ok(nbuf);
    for (int k = 0; k < nbuf; k++) maps_ok[k] = encode_window_map(&maps[k], in.planes + pbytes * k, pw, ph);
    for (int h = 1; h < n; h++) {
        FrameDesc& d = fds[h];
        const int buf = (h - 1) % nbuf;
        d.tmap = maps[buf];
        d.tmap_ok = maps_ok[buf];
        d.pic = h264a_picture{in.y + fs * h, in.planes + pbytes * buf, cw, ch, pad};
        d.lambda_me = in.lambda_me;
        d.split_gate = in.split_gate;
        d.picks = in.picks + 6LL * nmb * h;
        d.costs = in.costs + 2LL * nmb * h;
        d.mb_w = mb_w;
        d.mb_h = mb_h;
        d.coeffs = in.coeffs + 256LL * nmb * h;
        make_quant_row4(in.qp, in.dz_div, d.qff, d.qmf);
        if (in.props) {
            d.props = in.props + 16LL * nmb * h;
            d.fallback = in.fallback ? in.fallback + (long long)nmb * h : nullptr;
            d.prop_t = in.prop_t;
        }
        RecDesc& r = rds[h];
        r.src_c[0] = in.u + cs * h;
        r.src_c[1] = in.v + cs * h;
        r.ref_c[0] = in.rec_u + cs * (h - 1);
        r.ref_c[1] = in.rec_v + cs * (h - 1);
        r.rec_y = in.rec_y + fs * h;
        r.rec_c[0] = in.rec_u + cs * h;
        r.rec_c[1] = in.rec_v + cs * h;
        r.ccoeffs = in.ccoeffs + 128LL * nmb * h;
        r.qp = in.qp;
        r.qpc = chroma_qp_of(in.qp);
        make_quant_row4(r.qpc, 6, r.cff, r.cmf);
        r.th = db_thresholds(in.qp, 0, 0, 0);
    }
    // a frame's tickets: its MBs in wavefront order (anti-diagonals t = x + 2y,
    // then y), and segment (b, s) right after MB (min(segw*(s+1), mb_w-1),
    // min(b+1, mb_h-1)), segments of one MB in (b, s) order
    std::vector<std::vector<int>> trig(nmb);
    for (int b = 0; b < nbands; b++)
        for (int sg = 0; sg < nseg; sg++)
            trig[std::min(b + 1, mb_h - 1) * mb_w + std::min(segw * (sg + 1), mb_w - 1)].push_back(-(1 + b * nseg + sg));
    std::vector<int> items;
    items.reserve(nmb + nbands * nseg);
    for (int t = 0; t <= (mb_w - 1) + 2 * (mb_h - 1); t++) {
        for (int y = 0; y < mb_h; y++) {
            const int x = t - 2 * y;
            if (x < 0 || x >= mb_w) continue;
            items.push_back(y * mb_w + x);
            for (int it : trig[y * mb_w + x]) items.push_back(it);
        }
    }
    if ((int)items.size() != nmb + nbands * nseg) return fail(H264A_E_ARG, "closed loop: internal ticket layout error");
    const size_t b_fd = sizeof(FrameDesc) * n, b_rd = (sizeof(RecDesc) * n + 63) & ~size_t(63),
                 b_it = sizeof(int) * items.size();
    char* hst = nullptr;
    rc = table_host(ctx, b_fd + b_rd + b_it, &hst);
    if (rc) return rc;
    memcpy(hst, fds.data(), b_fd);
    memcpy(hst + b_fd, rds.data(), sizeof(RecDesc) * n);
    memcpy(hst + b_fd + b_rd, items.data(), b_it);
    rc = table_upload(ctx, b_fd + b_rd + b_it, st);
    if (rc) return rc;
    char* dv = static_cast<char*>(ctx->me_tab);
    // flags: n ticket counters, n completed-MB counters, then per frame its
    // MV words, deblocking flags and band flags (an even count per frame)
    PipeParams pp;
    memset(&pp, 0, sizeof pp);
    pp.fds = reinterpret_cast<const FrameDesc*>(dv);
    pp.rds = reinterpret_cast<const RecDesc*>(dv + b_fd);
    pp.items = reinterpret_cast<const int*>(dv + b_fd + b_rd);
    pp.nitems = int(items.size());
    pp.n = n;
    pp.mb_w = mb_w;
    pp.mb_h = mb_h;
    pp.nbands = nbands;
    pp.nseg = nseg;
    pp.segw = segw;
    pp.nbuf = nbuf;
    pp.pools = pools;
    pp.ew_off = 0;
    pp.dfl_off = 2 * EW_PER_MB * nmb;
    pp.band_off = pp.dfl_off + nmb;
    pp.fstride = (pp.band_off + (long long)nbands * nseg + 1) & ~1LL;
    const long long head = (2LL * n + 1) & ~1LL;
    const long long need = head + pp.fstride * n;
    if (need >= (1LL << 31)) return fail(H264A_E_ARG, "closed loop: too many macroblocks for one launch");
    rc = ensure_me_scratch(ctx, size_t(need), Q_WIDE);
    if (rc) return rc;
    int* fl = ctx->q[Q_WIDE].d_flags;
    pp.ctr = fl;
    pp.done = fl + n;
    pp.flags = fl + head;
    pp.rec_y = in.rec_y;
    pp.fs = fs;
    pp.planes = in.planes;
    pp.pbytes = pbytes;
    pp.cw = cw;
    pp.ch = ch;
    pp.pad = pad;
    pp.word_in = (cw % 4 == 0) && (pad % 4 == 0) && ((reinterpret_cast<uintptr_t>(in.rec_y) & 3) == 0);
    pp.word_out = (pw % 4 == 0) && ((reinterpret_cast<uintptr_t>(in.planes) & 3) == 0) && (pbytes % 4 == 0);
    pp.frame_words = frame_words;
    pp.ftoken = token;
    pp.arrive = in.arrive;
    pp.atoken = in.atoken;
    // counters zero, and no word of an earlier launch's layout left to be
    // mistaken for a flag of this one
    H264A_CUDA(cudaMemsetAsync(fl, 0, sizeof(int) * size_t(need), st));
    const int epoch = next_epoch(ctx, st, Q_WIDE);
    if (epoch < 0) return H264A_E_CUDA;
    long long blocks = (long long)ctx->num_sms * per_sm;
    blocks -= blocks % pools;  // an equal share of CTAs per pool
    if (blocks < pools) blocks = pools;
    const bool bal = balanced_preset(prm), learn = in.props != nullptr;
    const size_t sm = WIN_BYTES;
    if (learn && bal)
        closed_pipe_kernel<true, true><<<unsigned(blocks), 32 * ME_WIDE_WARPS, sm, st>>>(pp, prm, epoch, ctx->d_status,
                                                                                        SPIN_LIMIT);
    else if (learn)
        closed_pipe_kernel<false, true><<<unsigned(blocks), 32 * ME_WIDE_WARPS, sm, st>>>(pp, prm, epoch, ctx->d_status,
                                                                                         SPIN_LIMIT);
    else if (bal)
        closed_pipe_kernel<true, false><<<unsigned(blocks), 32 * ME_WIDE_WARPS, sm, st>>>(pp, prm, epoch, ctx->d_status,
                                                                                         SPIN_LIMIT);
    else
        closed_pipe_kernel<false, false><<<unsigned(blocks), 32 * ME_WIDE_WARPS, sm, st>>>(pp, prm, epoch,
                                                                                          ctx->d_status, SPIN_LIMIT);
    rc = check_launch("closed_pipe_kernel");
    if (rc) return rc;
    return table_done(ctx, st);
}

// ---------------------------------------------------------------------------
// Plain-ME frames over several reference pictures
// ---------------------------------------------------------------------------
// best_part's loop over references (mb16.rs:4921-4960) in the frame model:
// every search (the 16x16, and the four partitions when its J exceeds the
// gate) runs on each reference r with seeds [predict_mv(a, b, c, r), extra],
// costs plus (lambda * ref_bits(r, nref)) truncated to i64, the strictly
// cheapest kept (references in order).  An MV predicts only from neighbours
// of the same reference (inter.rs:36-69), so a pick carries each half's
// reference index: 8 i32 per MB (shape, ref0, mv0x, mv0y, ref1, mv1x, mv1y,
// 4x4-block evaluations).  One warp per MB, the narrow kernel's queue and
// wavefront; the window is staged again for each reference.
constexpr int ME_MAXREF = 4;
struct FrameDescMR {
    CUtensorMap tmap[ME_MAXREF];  // each reference's planes as the window's 3D tensor
    const uint8_t* planes[ME_MAXREF];
    const uint8_t* src;
    double lambda_me;
    long long split_gate;
    int32_t* picks;
    int64_t* costs;
    int nref, cw, ch, pad, mb_w, mb_h, flag_base, tmap_ok;
};

// ref_bits (mb16.rs:5967-5981).
__device__ __forceinline__ uint32_t ref_bits_of(int r, int nref) {
    if (nref <= 1) return 0;
    if (nref == 2) return 1;
    return 1u + 2u * (31u - uint32_t(__clz(r + 1)));
}

// predict_mv (inter.rs:36-69) against reference cur: neighbours with their
// reference indices (available ones are inter, index >= 0).
__device__ __forceinline__ int2 predict_mv_ref(bool aa, int2 a, int ra, bool ba, int2 b, int rb, bool ca, int2 c, int rc,
                                               int cur) {
    int2 mva = aa ? a : make_int2(0, 0), mvb = ba ? b : make_int2(0, 0), mvc = ca ? c : make_int2(0, 0);
    int qa = aa ? ra : -1, qb = ba ? rb : -1, qc = ca ? rc : -1;
    if (!ba && !ca && aa) { mvb = mva; qb = qa; mvc = mva; qc = qa; }
    const int matches = (qa == cur) + (qb == cur) + (qc == cur);
    if (matches == 1) return qa == cur ? mva : (qb == cur ? mvb : mvc);
    auto med = [](int x, int y, int z) { return x + y + z - min(min(x, y), z) - max(max(x, y), z); };
    return make_int2(med(mva.x, mvb.x, mvc.x), med(mva.y, mvb.y, mvc.y));
}

// The MV and reference of neighbour MB `m`'s 4x4 block (bx4, by4).
__device__ __forceinline__ int2 pick_mr_at(const int32_t* picks, int m, int bx4, int by4, int& ref) {
    const int32_t* p = picks + 8 * m;
    const int shape = __ldcg(p);
    const int part = shape == 1 ? (by4 >= 2) : (shape == 2 ? (bx4 >= 2) : 0);
    ref = __ldcg(p + 1 + 3 * part);
    return make_int2(__ldcg(p + 2 + 3 * part), __ldcg(p + 3 + 3 * part));
}

// Launch shapes (the batch runtime's autotuner picks one): NW warps per CTA,
// one MB each (the MBs a CTA holds at once), and STAGE: each search's window
// staged in shared memory by TMA, or every candidate read from L2 through the
// search's global path (no window, no shared memory, the same results).
template <bool BAL, int NW, bool STAGE>
__global__ void __launch_bounds__(32 * NW, 16 / NW)
    me_frames_mr_kernel(const FrameDescMR* __restrict__ fds, const long long* __restrict__ seg_start,
                        const int* __restrict__ seg_j, int nf, int ns, long long total,
                        const __grid_constant__ MeParamsDev prm, int* __restrict__ counter, int* __restrict__ flags,
                        int epoch, int* __restrict__ status, int spin_limit) {
    __shared__ WarpScratch scratch[NW];
    __shared__ __align__(8) unsigned long long win_bar[NW];
    extern __shared__ __align__(128) uint8_t me_win[];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t win = uint32_t(__cvta_generic_to_shared(me_win)) + uint32_t(w * WIN_BYTES);
    const uint32_t bar = uint32_t(__cvta_generic_to_shared(&win_bar[w]));
    if (lane == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    uint32_t parity = 0;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(counter, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) return;
        int s = 0;
        while (s + 1 < ns && __ldg(seg_start + s + 1) <= t) s++;
        const int j = __ldg(seg_j + s);
        const long long u = t - __ldg(seg_start + s);
        const int nxt = j + 1 < nf ? fds[j + 1].mb_w * fds[j + 1].mb_h : 0;
        const FrameDescMR& fd = fds[int(u % (j + 1))];
        const int k = nxt + int(u / (j + 1));
        int mbx, mby;
        wave_mb(fd.mb_w, fd.mb_h, k, mbx, mby);
        const int m = mby * fd.mb_w + mbx;
        int* fl = flags + fd.flag_base;
        const int lx = mbx * 16, ly = mby * 16;
        uint32_t src4[4];
#pragma unroll
        for (int r = 0; r < 4; r++)
            src4[r] = ld4u(fd.src + (long long)(ly + ((lane >> 2) & 3) * 4 + r) * fd.cw + lx + (lane & 3) * 4);
        if (lane == 0) {
            if (mbx > 0) wait_flag(fl + m - 1, epoch, status, 1, spin_limit);
            if (mby > 0) wait_flag(fl + m - fd.mb_w + (mbx < fd.mb_w - 1 ? 1 : 0), epoch, status, 1, spin_limit);
        }
        __syncwarp();
        const bool aa = mbx > 0, ba = mby > 0, ca = mby > 0 && mbx < fd.mb_w - 1, da = mbx > 0 && mby > 0;
        int ra = -1, rb = -1, rc = -1;
        const int2 a = aa ? pick_mr_at(fd.picks, m - 1, 3, 0, ra) : make_int2(0, 0);
        const int2 bb = ba ? pick_mr_at(fd.picks, m - fd.mb_w, 0, 3, rb) : make_int2(0, 0);
        int2 c = make_int2(0, 0);
        if (ca) c = pick_mr_at(fd.picks, m - fd.mb_w + 1, 0, 3, rc);
        else if (da) c = pick_mr_at(fd.picks, m - fd.mb_w - 1, 3, 3, rc);
        const bool cav = ca || da;
        const int pw = fd.cw + 2 * fd.pad, ph = fd.ch + 2 * fd.pad;
        // best_part of the 16x16 over the references, then, J above the gate,
        // of each partition (lane group g = partition g) over the references
        int evals = 0, shape = 0;
        int ref16 = 0, mv16x = 0, mv16y = 0;
        long long c16 = LLONG_MAX;
        int pref = 0, pmx = 0, pmy = 0;  // the lane's partition's best (mode 1)
        long long pcost = LLONG_MAX;
        for (int mode = 0; mode < 2; mode++) {
            if (mode == 1 && !(fd.split_gate >= 0 && c16 > fd.split_gate)) break;
            for (int r = 0; r < fd.nref; r++) {
                const int2 pmv = predict_mv_ref(aa, a, ra, ba, bb, rb, cav, c, rc, r);
                h264a_picture pc{fd.src, fd.planes[r], fd.cw, fd.ch, fd.pad};
                const bool win_ok = STAGE && ((reinterpret_cast<uintptr_t>(pc.d_planes) | uintptr_t(pw)) & 15) == 0 &&
                                    pw >= WIN_W && ph >= WIN_H;
                if (win_ok) {
                    const int wx0 = min(max((lx + pc.pad + (pmv.x >> 2) - WIN_R) & ~15, 0), pw - WIN_W);
                    const int wy0 = min(max(ly + pc.pad + (pmv.y >> 2) - WIN_R, 0), ph - WIN_H);
                    if (lane == 0) {
                        scratch[w].wx0 = wx0;
                        scratch[w].wy0 = wy0;
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        if (fd.tmap_ok) {
                            mbar_expect_tx(bar, uint32_t(WIN_BYTES));
                            // a tensor map written to device memory by the host since an
                            // earlier launch read that address: acquire it for the copy
                            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(&fd.tmap[r])
                                         : "memory");
                            tma_load_3d(win, &fd.tmap[r], wx0, wy0, 0, bar);
                        } else {
                            mbar_expect_tx(bar, uint32_t(4 * WIN_H * WIN_W));
                        }
                    }
                    __syncwarp();
                    if (!fd.tmap_ok) {
                        const long long ps = (long long)pw * ph;
                        for (int i = lane; i < 4 * WIN_H; i += 32) {
                            const int pl = i / WIN_H, rr = i - pl * WIN_H;
                            bulk_g2s(win + uint32_t(pl * WIN_PLANE + rr * WIN_STRIDE),
                                     pc.d_planes + ps * pl + (long long)(wy0 + rr) * pw + wx0, WIN_W, bar);
                        }
                    }
                }
                if (lane == 0) scratch[w].win_ok = win_ok;
                __syncwarp();
                GroupGeom qg;
                group_geom_init(qg, scratch[w], pc, lx, ly, mode, win, mode == 0 ? src4 : nullptr);
                if (win_ok) {
                    wait_window(bar, parity, status, 3, spin_limit);
                    parity ^= 1u;
                }
                int preds[4] = {pmv.x, pmv.y, mv16x, mv16y};
                int rx, ry, ev;
                long long cst;
                motion_search_group<BAL>(qg, prm, scratch[w], preds, mode == 0 ? 1 : 2, fd.lambda_me, rx, ry, cst, ev);
                cst += __double2ll_rz(__dmul_rn(fd.lambda_me, double(ref_bits_of(r, fd.nref))));
                if (mode == 0) {
                    evals += ev << 4;
                    if (cst < c16) { c16 = cst; ref16 = r; mv16x = rx; mv16y = ry; }
                } else {
                    // every lane of group g holds partition g's result
                    evals += (__shfl_sync(0xffffffffu, ev, 0) + __shfl_sync(0xffffffffu, ev, 8) +
                              __shfl_sync(0xffffffffu, ev, 16) + __shfl_sync(0xffffffffu, ev, 24)) << 3;
                    if (cst < pcost) { pcost = cst; pref = r; pmx = rx; pmy = ry; }
                }
                __syncwarp();  // the window's reads are done before the next copy
            }
        }
        // the shape decision (mb16.rs:8869-8913)
        int s0r = ref16, s0x = mv16x, s0y = mv16y, s1r = ref16, s1x = mv16x, s1y = mv16y;
        long long best = c16;
        if (fd.split_gate >= 0 && c16 > fd.split_gate) {
            long long pc4[4];
            int pr4[4], px4[4], py4[4];
#pragma unroll
            for (int gi = 0; gi < 4; gi++) {
                pc4[gi] = __shfl_sync(0xffffffffu, pcost, 8 * gi);
                pr4[gi] = __shfl_sync(0xffffffffu, pref, 8 * gi);
                px4[gi] = __shfl_sync(0xffffffffu, pmx, 8 * gi);
                py4[gi] = __shfl_sync(0xffffffffu, pmy, 8 * gi);
            }
            if (pc4[0] + pc4[1] < best) {
                best = pc4[0] + pc4[1]; shape = 1;
                s0r = pr4[0]; s0x = px4[0]; s0y = py4[0]; s1r = pr4[1]; s1x = px4[1]; s1y = py4[1];
            }
            if (pc4[2] + pc4[3] < best) {
                best = pc4[2] + pc4[3]; shape = 2;
                s0r = pr4[2]; s0x = px4[2]; s0y = py4[2]; s1r = pr4[3]; s1x = px4[3]; s1y = py4[3];
            }
        }
        if (lane == 0) {
            int32_t* p = fd.picks + 8 * m;
            p[0] = shape; p[1] = s0r; p[2] = s0x; p[3] = s0y; p[4] = s1r; p[5] = s1x; p[6] = s1y; p[7] = evals;
            fd.costs[2 * m] = best;
            fd.costs[2 * m + 1] = c16;
            st_release(fl + m, epoch);  // orders the pick's stores before the flag
        }
        __syncwarp();
    }
}

// The launch shapes, variant 0 the default of h264a_me_frames_multiref.
struct MrShape {
    int nw;
    bool stage;
};
constexpr MrShape kMrShapes[H264A_BATCH_VARIANTS] = {{4, true}, {2, true}, {8, true}, {4, false}, {2, false}, {8, false}};

template <bool BAL, int NW, bool STAGE>
static int mr_attr() {
    if (STAGE)
        H264A_CUDA(cudaFuncSetAttribute(me_frames_mr_kernel<BAL, NW, STAGE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        NW * WIN_BYTES));
    return H264A_OK;
}

static int me_mr_setup_once() {
    int rc = mr_attr<false, 4, true>();
    if (!rc) rc = mr_attr<true, 4, true>();
    if (!rc) rc = mr_attr<true, 2, true>();
    if (!rc) rc = mr_attr<true, 8, true>();
    return rc;
}

template <bool BAL, int NW, bool STAGE>
static int mr_launch_t(h264a_ctx* ctx, const MeParamsDev& prm, const char* dv, const MrTable& t, int32_t* counter,
                       int32_t* flags, int epoch, cudaStream_t st) {
    const size_t sm = STAGE ? size_t(NW) * WIN_BYTES : 0;
    int per_sm = 0;
    H264A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, me_frames_mr_kernel<BAL, NW, STAGE>, 32 * NW, sm));
    if (per_sm < 1) per_sm = 1;
    long long blocks = (long long)ctx->num_sms * per_sm;
    const long long need = (t.total + NW - 1) / NW;
    if (blocks > need) blocks = need;
    me_frames_mr_kernel<BAL, NW, STAGE><<<unsigned(blocks), 32 * NW, sm, st>>>(
        reinterpret_cast<const FrameDescMR*>(dv), reinterpret_cast<const long long*>(dv + t.b_desc),
        reinterpret_cast<const int*>(dv + t.b_desc + t.b_seg), t.nframes, t.nseg, t.total, prm, counter, flags, epoch,
        ctx->d_status, SPIN_LIMIT);
    return check_launch("me_frames_mr_kernel");
}

int h264a::mr_table_build(const h264a_me_mr_frame* h_frames, int nframes, MrTable& t) {
    if (!h_frames) return fail(H264A_E_ARG, "me_frames_multiref: null pointer");
    if (nframes < 1) return fail(H264A_E_ARG, "me_frames_multiref: need at least one frame");
    for (int i = 0; i < nframes; i++) {
        const h264a_me_mr_frame& f = h_frames[i];
        if (f.nref < 1 || f.nref > ME_MAXREF) return fail(H264A_E_ARG, "me_frames_multiref: 1 to 4 references per frame");
        if (!f.d_src || !f.d_picks || !f.d_costs) return fail(H264A_E_ARG, "me_frames_multiref: null frame pointer");
        if (reinterpret_cast<uintptr_t>(f.d_src) & 3) return fail(H264A_E_ARG, "me_frames_multiref: sources must be 4-byte aligned");
        for (int r = 0; r < f.nref; r++)
            if (!f.d_planes[r]) return fail(H264A_E_ARG, "me_frames_multiref: null reference planes");
        if (f.cw < 16 || f.ch < 16 || f.cw % 16 || f.ch % 16 || f.pad < 3 || f.pad > 128)
            return fail(H264A_E_ARG, "me_frames_multiref: frames must be MB-aligned with 3 <= pad <= 128");
        if ((long long)(f.cw / 16) * (f.ch / 16) > (1 << 24)) return fail(H264A_E_ARG, "me_frames_multiref: frame too large");
    }
    std::vector<int> order(nframes);
    for (int i = 0; i < nframes; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (long long)h_frames[a].cw * h_frames[a].ch > (long long)h_frames[b].cw * h_frames[b].ch;
    });
    std::vector<FrameDescMR> desc(nframes);
    memset(desc.data(), 0, sizeof(FrameDescMR) * nframes);
    std::vector<FrameDesc> segd(nframes);  // the sizes, for the queue's segments
    memset(segd.data(), 0, sizeof(FrameDesc) * nframes);
    long long total = 0;
    for (int k = 0; k < nframes; k++) {
        const h264a_me_mr_frame& f = h_frames[order[k]];
        FrameDescMR& d = desc[k];
        const int pw = f.cw + 2 * f.pad, ph = f.ch + 2 * f.pad;
        d.tmap_ok = 1;
        for (int r = 0; r < f.nref; r++) {
            d.planes[r] = f.d_planes[r];
            d.tmap_ok &= encode_window_map(&d.tmap[r], f.d_planes[r], pw, ph);
        }
        d.src = f.d_src;
        d.lambda_me = f.lambda_me;
        d.split_gate = f.split_gate;
        d.picks = f.d_picks;
        d.costs = f.d_costs;
        d.nref = f.nref;
        d.cw = f.cw; d.ch = f.ch; d.pad = f.pad;
        d.mb_w = f.cw / 16;
        d.mb_h = f.ch / 16;
        d.flag_base = int(total);
        segd[k].mb_w = d.mb_w;
        segd[k].mb_h = d.mb_h;
        total += (long long)d.mb_w * d.mb_h;
        if (total >= (1LL << 31)) return fail(H264A_E_ARG, "me_frames_multiref: too many macroblocks in one call");
    }
    std::vector<long long> seg(nframes + 1);
    std::vector<int> segj(nframes);
    const int nseg = make_segments(segd.data(), nframes, seg.data(), segj.data());
    if (seg[nseg] != total) return fail(H264A_E_ARG, "me_frames_multiref: internal queue layout error");
    t.nframes = nframes;
    t.nseg = nseg;
    t.total = total;
    t.b_desc = sizeof(FrameDescMR) * nframes;
    t.b_seg = sizeof(long long) * (nseg + 1);
    const size_t b_j = sizeof(int) * nseg;
    t.bytes.assign(t.b_desc + t.b_seg + b_j, 0);
    memcpy(t.bytes.data(), desc.data(), t.b_desc);
    memcpy(t.bytes.data() + t.b_desc, seg.data(), t.b_seg);
    memcpy(t.bytes.data() + t.b_desc + t.b_seg, segj.data(), b_j);
    return H264A_OK;
}

int h264a::mr_launch(h264a_ctx* ctx, int variant, const MeParamsDev& prm, const void* d_table, const MrTable& t,
                     int32_t* counter, int32_t* flags, int epoch, cudaStream_t st) {
    if (variant < 0 || variant >= H264A_BATCH_VARIANTS) return fail(H264A_E_ARG, "me_frames_multiref: no such launch shape");
    static std::once_flag once;
    static int setup_rc = 0;
    std::call_once(once, [] { setup_rc = me_mr_setup_once(); });
    if (setup_rc) return setup_rc;
    const char* dv = static_cast<const char*>(d_table);
    if (!balanced_preset(prm)) return mr_launch_t<false, 4, true>(ctx, prm, dv, t, counter, flags, epoch, st);
    switch (variant) {
        case 1: return mr_launch_t<true, 2, true>(ctx, prm, dv, t, counter, flags, epoch, st);
        case 2: return mr_launch_t<true, 8, true>(ctx, prm, dv, t, counter, flags, epoch, st);
        case 3: return mr_launch_t<true, 4, false>(ctx, prm, dv, t, counter, flags, epoch, st);
        case 4: return mr_launch_t<true, 2, false>(ctx, prm, dv, t, counter, flags, epoch, st);
        case 5: return mr_launch_t<true, 8, false>(ctx, prm, dv, t, counter, flags, epoch, st);
        default: return mr_launch_t<true, 4, true>(ctx, prm, dv, t, counter, flags, epoch, st);
    }
}

extern "C" int h264a_batch_variant_shape(int variant, int* mbs_per_cta, int* staged) {
    if (variant < 0 || variant >= H264A_BATCH_VARIANTS) return fail(H264A_E_ARG, "batch_variant_shape: no such variant");
    if (mbs_per_cta) *mbs_per_cta = kMrShapes[variant].nw;
    if (staged) *staged = kMrShapes[variant].stage ? 1 : 0;
    return H264A_OK;
}

extern "C" int h264a_me_frames_multiref(h264a_ctx* ctx, const h264a_me_mr_frame* h_frames, int nframes,
                                        const h264a_me_params* params, void* stream) {
    if (!ctx || !h_frames || !params) return fail(H264A_E_ARG, "me_frames_multiref: null pointer");
    if ((params->mv_cost_kind == 1 || params->mv_cost_kind == 2) && !params->d_mv_cost_tab)
        return fail(H264A_E_ARG, "me_frames_multiref: mv cost kinds 1 and 2 need d_mv_cost_tab");
    MrTable t;
    int rc = mr_table_build(h_frames, nframes, t);
    if (rc) return rc;
    cudaStream_t st = pick_stream(ctx, stream);
    const MeParamsDev prm = to_dev(*params);
    char* hst = nullptr;
    rc = table_host(ctx, t.bytes.size(), &hst);
    if (rc) return rc;
    memcpy(hst, t.bytes.data(), t.bytes.size());
    rc = table_upload(ctx, t.bytes.size(), st);
    if (rc) return rc;
    rc = ensure_me_scratch(ctx, size_t(t.total));
    if (rc) return rc;
    H264A_CUDA(cudaMemsetAsync(ctx->q[Q_MAIN].d_counter, 0, sizeof(int32_t), st));
    const int epoch = next_epoch(ctx, st);
    if (epoch < 0) return H264A_E_CUDA;
    rc = mr_launch(ctx, 0, prm, ctx->me_tab, t, ctx->q[Q_MAIN].d_counter, ctx->q[Q_MAIN].d_flags, epoch, st);
    if (rc) return rc;
    return table_done(ctx, st);
}
