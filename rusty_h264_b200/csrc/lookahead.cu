// lookahead.cu -- a16-a19: the mb-tree lookahead's per-frame costs
// (crates/rusty_h264-encoder/src/mbtree.rs:61-263).
//
//  * downsample2x: one thread per four output pixels, 8-byte loads.
//  * intra_cost: one lane per 4x4 sub-block, Σ|Hadamard AC| reduced per MB.
//  * inter_cost + frame_costs: the seeded full-pel diamond.  The seed chain
//    (left MV, else top MV; mbtree.rs:225-231) makes every row a sequential
//    chain that starts from column 0, and column 0 a chain down the frame.
//    Frames are independent (source domain, f against f-1).  One persistent
//    kernel deals the column-0 chains first (one warp per frame, publishing
//    each MB's flag as it finishes), then the rows in row order across frames:
//    a row's warp waits (bounded) only for its own column-0 MB, so rows start
//    while column 0 is still walking down the frame.  Inside a search the warp prices the four ring
//    points of the cascading diamond together and takes the first improvement,
//    re-pricing the rest of the ring around the moved centre (the reference's
//    evaluation order).
//    In HalfRes mode (the default) each chain reads its block's candidates
//    from a shared-memory window (the block +-16 rows, 48 columns), copied by
//    TMA one block ahead; candidates outside it, or outside the picture, read
//    the clamped picture.  The kernel is instantiated per mode.
#include <cstring>
#include <vector>

#include "h264a_device.cuh"

namespace h264a {

__global__ void downsample2x_kernel(const uint8_t* __restrict__ in, int cw, int ch, size_t fstride,
                                    uint8_t* __restrict__ out) {
    const int hw = cw / 2, hh = ch / 2;
    const int f = blockIdx.z;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;  // group of 4 outputs
    const int groups_per_row = hw / 4;
    if (t >= (long long)groups_per_row * hh) return;
    const int j = int(t / groups_per_row), i4 = int(t % groups_per_row) * 4;
    const uint8_t* a = in + fstride * f + (long long)(2 * j) * cw + 2 * i4;
    const uint2 r0 = *reinterpret_cast<const uint2*>(a);
    const uint2 r1 = *reinterpret_cast<const uint2*>(a + cw);
    uint32_t o = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t w0 = k < 2 ? r0.x : r0.y, w1 = k < 2 ? r1.x : r1.y;
        const int sh = (k & 1) * 16;
        const uint32_t s = ((w0 >> sh) & 255) + ((w0 >> (sh + 8)) & 255) + ((w1 >> sh) & 255) + ((w1 >> (sh + 8)) & 255);
        o |= ((s + 2) / 4) << (8 * k);
    }
    *reinterpret_cast<uint32_t*>(out + (size_t)hw * hh * f + (long long)j * hw + i4) = o;
}

// Scoring-resolution geometry of one lookahead mode.
struct LaGeom {
    int bs;        // block size at the scoring resolution (8 HalfRes, 16 otherwise)
    int sw, sh;    // scoring picture size
};

// intra_cost (mbtree.rs:78-93) of every MB of every frame; frame 0 (IDR) also
// gets inter = intra, mv = 0 (mbtree.rs:257).
__global__ void la_intra_kernel(const uint8_t* __restrict__ pics, size_t fstride, LaGeom g, int mb_w, int mb_h, int n,
                                int32_t* __restrict__ intra, int32_t* __restrict__ inter, int32_t* __restrict__ mvs) {
    const int lg = g.bs == 16 ? 4 : 2;  // sub-blocks per MB: 16 or 4
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long gm = t >> lg;  // global MB index
    const long long nmb = (long long)mb_w * mb_h;
    const int sb = int(t & ((1 << lg) - 1));
    int v = 0;
    const bool live = gm < nmb * n;
    if (live) {
        const int f = int(gm / nmb), m = int(gm % nmb);
        const int mbx = m % mb_w, mby = m / mb_w;
        const int nbx = g.bs / 4;
        const int x = mbx * g.bs + (sb % nbx) * 4, y = mby * g.bs + (sb / nbx) * 4;
        const uint8_t* p = pics + fstride * f + (long long)y * g.sw + x;
        uint32_t s[4];
        const uint32_t z[4] = {0, 0, 0, 0};
#pragma unroll
        for (int r = 0; r < 4; r++) s[r] = ld4u(p + (long long)r * g.sw);
        const int dc = int(__vsadu4(s[0], 0) + __vsadu4(s[1], 0) + __vsadu4(s[2], 0) + __vsadu4(s[3], 0));
        v = satd4x4_rows(s, z) - dc;  // Σ|AC|: the DC coefficient is the (non-negative) block sum
    }
    v = warp_seg_sum(v, 1 << lg);
    if (live && sb == 0) {
        const int c = v < 1 ? 1 : v;
        intra[gm] = c;
        if (gm < nmb) {  // frame 0: the IDR, no reference
            inter[gm] = c;
            mvs[2 * gm] = 0;
            mvs[2 * gm + 1] = 0;
        }
    }
}

// One lane's view of the SATD search of a bs x bs block.  The warp holds two
// searches, lane group g = lane / 16 (slots 16g.. of the candidate and
// distortion arrays), each walking its own row chain; a group prices
// 16 / (bs/4)^2 candidates per pass (four 8x8 or one 16x16).
// HalfRes reference windows: per chain two buffers of LA_WIN_H rows of
// LA_WIN_W bytes (the block +-16 rows, and 48 columns from the 16-byte boundary
// at or left of the block's x - 16), filled by a TMA copy one block ahead.
constexpr int LA_WIN_W = 48, LA_WIN_H = 40, LA_WIN_BYTES = LA_WIN_W * LA_WIN_H;
constexpr int LA_WIN_BUF = 2048;  // buffer stride: 128-byte aligned, with room for a row read's second word
extern __shared__ __align__(128) uint8_t la_win[];

// The four rows of a 4x4 block at window column cx, row cy of the buffer at
// byte offset `off` of la_win (two aligned words and a funnel shift per row).
__device__ __forceinline__ void la_win_rows(int off, int cx, int cy, uint32_t p[4]) {
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int a = off + (cy + r) * LA_WIN_W + cx;
        const uint32_t* wp = reinterpret_cast<const uint32_t*>(la_win + (a & ~3));
        p[r] = __funnelshift_r(wp[0], wp[1], uint32_t(a & 3) * 8u);
    }
}

struct LaSearch {
    const uint8_t* cur;
    const uint8_t* ref;
    int w, h, bs, lg_nb, gl, gb, bxo, byo, x0, y0;
    uint32_t spa[4], spb[4];  // the source rows split into column pairs (split_pairs)
    int2* cand;
    int* dist;
    // the block's window (wbuf < 0: none): buffer offset, the lane's 4x4 block
    // at MV (0,0) in window coordinates, and the window columns/rows a 4x4
    // read may start at (inside the window and the picture) as bytes
    // xlo | xhi << 8 | ylo << 16 | yhi << 24
    int wbuf, wox, woy;
    uint32_t wlim;

    __device__ void set_window(int buf, int wx0, int wy0) {
        wbuf = buf;
        wox = x0 + bxo - wx0;
        woy = y0 + byo - wy0;
        const int xlo = max(0, -wx0), xhi = min(LA_WIN_W, w - wx0) - 4;
        const int ylo = max(0, -wy0), yhi = min(LA_WIN_H, h - wy0) - 4;
        wlim = uint32_t(xlo) | uint32_t(xhi) << 8 | uint32_t(ylo) << 16 | uint32_t(yhi) << 24;
    }

    __device__ void init(const uint8_t* c, const uint8_t* r, int pw, int ph, int b, int bx0, int by0, int2* cs,
                         int* ds) {
        cur = c; ref = r; w = pw; h = ph; bs = b; x0 = bx0; y0 = by0; cand = cs; dist = ds;
        wbuf = -1;
        const int lane = threadIdx.x & 31;
        gl = lane & 15;
        gb = lane & 16;
        lg_nb = b == 16 ? 4 : 2;
        const int nbx = b / 4;
        const int sb = gl & ((1 << lg_nb) - 1);
        bxo = (sb % nbx) * 4;
        byo = (sb / nbx) * 4;
        {
            uint32_t srow[4];
#pragma unroll
            for (int r = 0; r < 4; r++) srow[r] = ld4u(cur + (long long)(y0 + byo + r) * w + x0 + bxo);
            split_pairs(srow, spa, spb);
        }
    }

    // SATD of each group's cand[gb..gb+n) (full-pel MVs, quarter-pel units)
    // added into dist (zeroed by the caller) by shared-memory atomics of the
    // lanes' 4x4 blocks; passes run to the larger group's need.
    template <bool FULLPEL>  // FULLPEL: every candidate is a full-pel MV (HalfRes, FullRes)
    __device__ void eval(int n) {
        const int cps = 4 - lg_nb;  // log2 candidates per pass of a group
        const int npass = __reduce_max_sync(0xffffffffu, (n + (1 << cps) - 1) >> cps);
        for (int k = 0; k < npass; k++) {
            const int c = (k << cps) + (gl >> lg_nb);
            int d = 0;
            if (c < n) {
                const int2 mv = cand[gb + c];
                uint32_t p[4];
                if (FULLPEL || ((mv.x | mv.y) & 3) == 0) {
                    const int cx = wox + (mv.x >> 2), cy = woy + (mv.y >> 2);
                    if (wbuf >= 0 && cx >= int(wlim & 255u) && cx <= int((wlim >> 8) & 255u) &&
                        cy >= int((wlim >> 16) & 255u) && cy <= int(wlim >> 24))
                        la_win_rows(wbuf, cx, cy, p);
                    else
                        fullpel_rows_clamped(ref, w, h, x0 + bxo + (mv.x >> 2), y0 + byo + (mv.y >> 2), p);
                } else  // a sub-pel seed (Hybrid mode halves a full-res MV): mc_luma on the plain picture
                    subpel_rows_clamped(ref, w, h, x0 + bxo + (mv.x >> 2), y0 + byo + (mv.y >> 2), mv.x & 3, mv.y & 3, p);
                d = satd4x4_packed(spa, spb, p);
            }
            if (c < n) atomicAdd(&dist[gb + c], d);  // the candidate's blocks, summed in shared memory
        }
        __syncwarp();
    }
};

// The four-point diamond in the order mbtree.rs:181 walks it:
// right, left, down, up.
__device__ __forceinline__ int la_ring_dx(int k) { return k == 0 ? 1 : (k == 1 ? -1 : 0); }
__device__ __forceinline__ int la_ring_dy(int k) { return k == 2 ? 1 : (k == 3 ? -1 : 0); }

// inter_cost (mbtree.rs:154-197) of each group's block: (0,0) and the seed,
// then the cascading four-point diamond at steps max_step .. 1 full pixels
// (first improvement moves the centre, the rest of the ring is priced around
// it; a ring that moved is walked again at the same step), stopping at once
// when (0,0) costs nothing.  `active` false: the group takes no part.
template <bool FULLPEL>
__device__ void la_inter_cost(LaSearch& s, bool active, int seedx, int seedy, int max_step, int& cost, int& mvx,
                              int& mvy) {
    const int gl = s.gl, gb = s.gb;
    int phase = active ? 0 : 2;  // 0 seeds, 1 rings, 2 done
    int step = max_step, ri = 0, guard = 0;
    bool moved = false;
    long long best = 0;
    int bx = 0, by = 0;
    for (;;) {
        int n = 0;
        if (phase == 0) {
            if (gl == 0) {
                s.cand[gb] = make_int2(0, 0);
                s.cand[gb + 1] = make_int2(seedx, seedy);
            }
            n = 2;
        } else if (phase == 1) {
            n = 4 - ri;
            if (gl < n)
                s.cand[gb + gl] = make_int2(bx + la_ring_dx(ri + gl) * step * 4, by + la_ring_dy(ri + gl) * step * 4);
        }
        if (__all_sync(0xffffffffu, phase == 2)) break;
        if (gl < n) s.dist[gb + gl] = 0;  // eval adds each lane's block into its candidate's slot
        __syncwarp();
        s.eval<FULLPEL>(n);
        const int d = gl < n ? s.dist[gb + gl] : 0;
        const unsigned hit = (__ballot_sync(0xffffffffu, gl < n && (long long)d < best) >> gb) & 0xffffu;
        const int j = hit ? __ffs(hit) - 1 : 0;
        const int dj = __shfl_sync(0xffffffffu, d, gb + j);
        const int d0 = __shfl_sync(0xffffffffu, d, gb), d1 = __shfl_sync(0xffffffffu, d, gb + 1);
        if (phase == 0) {
            best = d0;
            if (best == 0) {
                phase = 2;
            } else {
                if ((seedx != 0 || seedy != 0) && (long long)d1 < best) {
                    best = d1;
                    bx = seedx;
                    by = seedy;
                }
                phase = 1;
            }
        } else if (phase == 1) {
            bool ring_end;
            if (hit) {
                best = dj;
                bx = s.cand[gb + j].x;
                by = s.cand[gb + j].y;
                moved = true;
                ri += j + 1;
                ring_end = ri >= 4;
            } else {
                ring_end = true;
            }
            if (ring_end) {
                if (moved && ++guard < (1 << 20)) {
                    ri = 0;  // walk the ring again at this step
                } else {
                    step >>= 1;
                    ri = 0;
                    guard = 0;
                    if (step == 0) phase = 2;
                }
                moved = false;
            }
        }
        __syncwarp();
    }
    cost = best > 0x7fffffffLL ? 0x7fffffff : int(best);
    mvx = bx;
    mvy = by;
}

struct LaBufs {
    CUtensorMap hmap;     // the half-res frames as (cw/2, ch/2, n), box LA_WIN_W x LA_WIN_H x 1
    int hmap_ok;          // HalfRes mode with a valid map: searches read windows
    const uint8_t* full;  // n frames cw x ch
    const uint8_t* half;  // n frames cw/2 x ch/2 (modes 1, 2)
    int cw, ch, mb_w, mb_h, n, mode;
    int32_t* intra;
    int32_t* inter;
    int32_t* mvs;
};

// Window origin of half-res block column mbx: 16 columns left of the block,
// rounded down to a 16-byte boundary (the TMA x alignment).
__device__ __forceinline__ int la_win_x0(int mbx) { return (mbx * 8 - 16) & ~15; }

// frame_costs for MB (mbx, mby) of frame f >= 1 given the full-res seed.
template <int MODE>
__device__ void la_mb(const LaBufs& b, bool active, int f, int mbx, int mby, int sfx, int sfy, int2* cs, int* ds,
                      int wbuf, int& outx, int& outy) {
    const long long nmb = (long long)b.mb_w * b.mb_h;
    const long long gm = nmb * f + (long long)mby * b.mb_w + mbx;
    const int cwh = b.cw / 2, chh = b.ch / 2;
    const size_t fs = (size_t)b.cw * b.ch, hs = (size_t)cwh * chh;
    LaSearch s;
    int cost, mx, my;
    // an input (la_intra_kernel's output): read before the search, used after it
    const int ic = active && (threadIdx.x & 15) == 0 ? __ldg(b.intra + gm) : 0;
    if (MODE == 0) {  // FullRes
        s.init(b.full + fs * f, b.full + fs * (f - 1), b.cw, b.ch, 16, mbx * 16, mby * 16, cs, ds);
        la_inter_cost<true>(s, active, sfx, sfy, 8, cost, mx, my);
    } else {
        s.init(b.half + hs * f, b.half + hs * (f - 1), cwh, chh, 8, mbx * 8, mby * 8, cs, ds);
        if (wbuf >= 0) s.set_window(wbuf, la_win_x0(mbx), mby * 8 - 16);
        int hx, hy;
        la_inter_cost<MODE == 2>(s, active, sfx / 2, sfy / 2, 8, cost, hx, hy);
        if (MODE == 2) {  // HalfRes
            mx = hx * 2;
            my = hy * 2;
        } else {  // Hybrid: refine at full-res from the coarse MV
            s.init(b.full + fs * f, b.full + fs * (f - 1), b.cw, b.ch, 16, mbx * 16, mby * 16, cs, ds);
            la_inter_cost<true>(s, active, hx * 2, hy * 2, 2, cost, mx, my);
        }
    }
    if (active && s.gl == 0) {
        b.inter[gm] = cost < ic ? cost : ic;
        b.mvs[2 * gm] = mx;
        b.mvs[2 * gm + 1] = my;
    }
    outx = mx;
    outy = my;
}

constexpr int LA_WARPS = 4;

// Column-0 chains and row chains in one persistent launch, two chains per
// warp (lane group g = lane / 16 walks the second).  Tickets 0 .. ceil(nf/2)-1
// walk column 0 of frames 1+2t+g and publish flag (f-1)*mb_h + y after MB
// (0, y); later tickets take rows 2p and 2p+1 of the row order (rows in
// order, frames interleaved), each group waiting for its own column-0 flag
// and walking columns 1.. seeded by the left neighbour.  In HalfRes mode each
// chain's next block window is copied (TMA, lane 0 of the group) while the
// current block is searched; every copy issued is waited for (bounded,
// status 3) before the block that reads it.
// Several streams' lookaheads in one launch: stream s's column tickets are
// col0[s] .. col0[s+1]-1, all of them before any stream's row tickets
// (rowt0[s] .. rowt0[s+1]-1 after col0[ns]), so a row ticket's column chain
// was taken earlier, by a warp that waits for nothing; stream s's flags start
// at flag0[s].
constexpr int LA_MAXS = 24;
struct LaMulti {
    LaBufs b[LA_MAXS];
    int col0[LA_MAXS + 1];
    long long rowt0[LA_MAXS + 1];
    long long flag0[LA_MAXS];
    int ns;
};

template <int MODE>  // b.mode, as a constant
__global__ void __launch_bounds__(32 * LA_WARPS, 4) la_chains_kernel(const __grid_constant__ LaMulti lm,
                                                                 int* __restrict__ counter, int* __restrict__ flags0,
                                                                 int epoch, int* __restrict__ status, int spin_limit) {
    __shared__ int2 cs[LA_WARPS][32];
    __shared__ int ds[LA_WARPS][32];
    __shared__ __align__(8) unsigned long long la_bar[LA_WARPS][2][2];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int grp = lane >> 4, gl = lane & 15;
    const int buf0 = ((w * 2 + grp) * 2) * LA_WIN_BUF;  // this chain's two buffers in la_win
    const uint32_t win0 = uint32_t(__cvta_generic_to_shared(la_win)) + uint32_t(buf0);
    const uint32_t bar0 = uint32_t(__cvta_generic_to_shared(&la_bar[w][grp][0]));
    if (gl == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    uint32_t parity = 0;  // bit k: the phase buffer k completes next
    // window of block (mbx, mby) of frame f into buffer k (lane 0 of the group);
    // the group's earlier reads of the buffer are complete (converged warp)
    auto issue = [&](const LaBufs& b, int k, int f, int mbx, int mby) {
        if (gl == 0) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar0 + 8 * k, uint32_t(LA_WIN_BYTES));
            tma_load_3d(win0 + uint32_t(k * LA_WIN_BUF), &b.hmap, la_win_x0(mbx), mby * 8 - 16, f - 1, bar0 + 8 * k);
        }
    };
    auto wait = [&](int k) {
        wait_window(bar0 + 8 * k, (parity >> k) & 1u, status, 3, spin_limit);
        parity ^= 1u << k;
    };
    const int ns = lm.ns;
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(counter, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t < lm.col0[ns]) {
            int sidx = 0;
            while (sidx + 1 < ns && lm.col0[sidx + 1] <= t) sidx++;
            const LaBufs& b = lm.b[sidx];
            int* flags = flags0 + lm.flag0[sidx];
            const int nf = b.n - 1;
            const int f = 1 + 2 * (t - lm.col0[sidx]) + grp;
            const bool active = f <= nf;
            const bool uw = active && b.hmap_ok;
            if (uw) issue(b, 0, f, 0, 0);
            int sx = 0, sy = 0;
            for (int mby = 0; mby < b.mb_h; mby++) {
                const int k = mby & 1;
                if (uw && mby + 1 < b.mb_h) issue(b, k ^ 1, f, 0, mby + 1);
                if (uw) wait(k);
                int mx, my;
                la_mb<MODE>(b, active, active ? f : 1, 0, mby, sx, sy, cs[w], ds[w], uw ? buf0 + k * LA_WIN_BUF : -1, mx, my);
                sx = mx;
                sy = my;
                if (active && gl == 0) st_release(flags + (f - 1) * b.mb_h + mby, epoch);  // after the lane's MV store
                __syncwarp();
            }
            continue;
        }
        const long long tr = (long long)t - lm.col0[ns];
        if (tr >= lm.rowt0[ns]) return;
        int sidx = 0;
        while (sidx + 1 < ns && lm.rowt0[sidx + 1] <= tr) sidx++;
        const LaBufs& b = lm.b[sidx];
        int* flags = flags0 + lm.flag0[sidx];
        const int nf = b.n - 1;
        const long long nrows = (long long)nf * b.mb_h;
        const long long r = 2 * (tr - lm.rowt0[sidx]) + grp;
        const bool active = r < nrows;
        const bool uw = active && b.hmap_ok && b.mb_w > 1;
        const int mby = active ? int(r / nf) : 0, f = active ? 1 + int(r % nf) : 1;
        if (uw) issue(b, 0, f, 1, mby);  // the window is an input: no need to wait for column 0
        if (active && gl == 0) wait_flag(flags + (f - 1) * b.mb_h + mby, epoch, status, 1, spin_limit);
        __syncwarp();
        const long long gm0 = (long long)b.mb_w * b.mb_h * f + (long long)mby * b.mb_w;
        int sx = active ? __ldcg(b.mvs + 2 * gm0) : 0, sy = active ? __ldcg(b.mvs + 2 * gm0 + 1) : 0;
        for (int mbx = 1; mbx < b.mb_w; mbx++) {
            const int k = (mbx - 1) & 1;
            if (uw && mbx + 1 < b.mb_w) issue(b, k ^ 1, f, mbx + 1, mby);
            if (uw) wait(k);
            int mx, my;
            la_mb<MODE>(b, active, f, mbx, mby, sx, sy, cs[w], ds[w], uw ? buf0 + k * LA_WIN_BUF : -1, mx, my);
            sx = mx;
            sy = my;
            __syncwarp();
        }
    }
}

}  // namespace h264a

using namespace h264a;

extern "C" int h264a_downsample2x(h264a_ctx* ctx, const uint8_t* d_frames, int cw, int ch, int n, size_t frame_stride,
                                  uint8_t* d_half, void* stream) {
    if (!ctx || !d_frames || !d_half) return fail(H264A_E_ARG, "downsample2x: null pointer");
    if (cw < 16 || ch < 16 || cw % 16 || ch % 16 || n < 1 || n > 65535)
        return fail(H264A_E_ARG, "downsample2x: frames must be MB-aligned, 1 <= n <= 65535");
    if (frame_stride % 8 || (n > 1 && frame_stride < (size_t)cw * ch) ||
        (reinterpret_cast<uintptr_t>(d_frames) & 7) || (reinterpret_cast<uintptr_t>(d_half) & 3))
        return fail(H264A_E_ARG, "downsample2x: misaligned frames");
    const long long groups = (long long)(cw / 8) * (ch / 2);
    dim3 grid(unsigned((groups + 255) / 256), 1, n);
    downsample2x_kernel<<<grid, 256, 0, pick_stream(ctx, stream)>>>(d_frames, cw, ch, frame_stride, d_half);
    return check_launch("downsample2x_kernel");
}

namespace {

// Validates one stream's lookahead and fills its LaBufs (no launch).
int la_prepare(const h264a_la_stream& q, int mode, LaBufs& b) {
    if (!q.d_full || !q.d_intra || !q.d_inter || !q.d_mvs) return fail(H264A_E_ARG, "lookahead_costs: null pointer");
    if (mode != 0 && !q.d_half) return fail(H264A_E_ARG, "lookahead_costs: modes 1 and 2 need the half-res frames");
    if (q.cw < 16 || q.ch < 16 || q.cw % 16 || q.ch % 16 || q.n < 1)
        return fail(H264A_E_ARG, "lookahead_costs: bad geometry");
    if ((long long)(q.n - 1) * (q.ch / 16) > (1 << 24)) return fail(H264A_E_ARG, "lookahead_costs: too many rows");
    memset(&b, 0, sizeof b);
    b.full = q.d_full; b.half = q.d_half; b.cw = q.cw; b.ch = q.ch; b.mb_w = q.cw / 16; b.mb_h = q.ch / 16; b.n = q.n;
    b.mode = mode;
    b.intra = q.d_intra; b.inter = q.d_inter; b.mvs = q.d_mvs;
    b.hmap_ok = mode == 2 ? encode_u8_map_3d(&b.hmap, q.d_half, q.cw / 2, q.ch / 2, q.n, LA_WIN_W, LA_WIN_H, 1) : 0;
    return H264A_OK;
}

// intra costs of every stream, then their chains in persistent launches of
// up to LA_MAXS streams each (the queue is the context's lookahead queue).
int la_run(h264a_ctx* ctx, const h264a_la_stream* qs, int nq, int mode, cudaStream_t st) {
    if (mode < 0 || mode > 2) return fail(H264A_E_ARG, "lookahead_costs: mode must be 0 (full), 1 (hybrid) or 2 (half)");
    std::vector<LaBufs> bufs(nq);
    for (int i = 0; i < nq; i++) {
        const int rc = la_prepare(qs[i], mode, bufs[i]);
        if (rc) return rc;
    }
    for (int i = 0; i < nq; i++) {
        const h264a_la_stream& q = qs[i];
        const int cw = q.cw, ch = q.ch, n = q.n;
        const LaGeom g = mode == 2 ? LaGeom{8, cw / 2, ch / 2} : LaGeom{16, cw, ch};
        const size_t fstride = mode == 2 ? (size_t)(cw / 2) * (ch / 2) : (size_t)cw * ch;
        const long long nmb = (long long)(cw / 16) * (ch / 16);
        const long long threads = nmb * n * (g.bs == 16 ? 16 : 4);
        la_intra_kernel<<<unsigned((threads + 255) / 256), 256, 0, st>>>(mode == 2 ? q.d_half : q.d_full, fstride, g,
                                                                        cw / 16, ch / 16, n, q.d_intra, q.d_inter,
                                                                        q.d_mvs);
        const int rc = check_launch("la_intra_kernel");
        if (rc) return rc;
    }
    const int smem = LA_WARPS * 2 * 2 * LA_WIN_BUF;  // two window buffers per chain
    auto kern = mode == 0 ? la_chains_kernel<0> : (mode == 1 ? la_chains_kernel<1> : la_chains_kernel<2>);
    for (int s0 = 0; s0 < nq; s0 += LA_MAXS) {
        LaMulti* lm = new LaMulti;
        memset(lm, 0, sizeof *lm);
        long long flags = 0;
        for (int i = s0; i < nq && lm->ns < LA_MAXS; i++) {
            if (qs[i].n < 2) continue;  // intra only
            const int k = lm->ns++;
            const int nf = qs[i].n - 1;
            const long long nrows = (long long)nf * (qs[i].ch / 16);
            lm->b[k] = bufs[i];
            lm->col0[k + 1] = lm->col0[k] + (nf + 1) / 2;
            lm->rowt0[k + 1] = lm->rowt0[k] + (nrows + 1) / 2;
            lm->flag0[k] = flags;
            flags += nrows;
        }
        if (lm->ns == 0) {
            delete lm;
            continue;
        }
        const long long chains = lm->col0[lm->ns] + lm->rowt0[lm->ns];  // two chains per warp
        int rc = flags > (1LL << 30) ? fail(H264A_E_ARG, "lookahead_costs: too many rows") : H264A_OK;
        if (!rc) rc = ensure_me_scratch(ctx, size_t(flags), Q_LOOKAHEAD);
        if (!rc && cudaMemsetAsync(ctx->q[Q_LOOKAHEAD].d_counter, 0, sizeof(int32_t), st) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "lookahead_costs: counter reset");
        const int epoch = rc ? -1 : next_epoch(ctx, st, Q_LOOKAHEAD);
        if (!rc && epoch < 0) rc = H264A_E_CUDA;
        int per_sm = 0;
        if (!rc && cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * LA_WARPS, smem) != cudaSuccess)
            rc = cuda_fail(cudaGetLastError(), "lookahead_costs: occupancy");
        if (!rc) {
            long long blocks = (long long)ctx->num_sms * (per_sm > 0 ? per_sm : 1);
            const long long need = (chains + LA_WARPS - 1) / LA_WARPS;
            if (blocks > need) blocks = need;
            kern<<<unsigned(blocks), 32 * LA_WARPS, smem, st>>>(*lm, ctx->q[Q_LOOKAHEAD].d_counter,
                                                                ctx->q[Q_LOOKAHEAD].d_flags, epoch, ctx->d_status,
                                                                SPIN_LIMIT);
            rc = check_launch("la_chains_kernel");
        }
        delete lm;
        if (rc) return rc;
    }
    return H264A_OK;
}

}  // namespace

extern "C" int h264a_lookahead_costs(h264a_ctx* ctx, const uint8_t* d_full, const uint8_t* d_half, int cw, int ch, int n,
                                     int mode, int32_t* d_intra, int32_t* d_inter, int32_t* d_mvs, void* stream) {
    if (!ctx) return fail(H264A_E_ARG, "lookahead_costs: null pointer");
    const h264a_la_stream q{d_full, d_half, cw, ch, n, d_intra, d_inter, d_mvs};
    return la_run(ctx, &q, 1, mode, pick_stream(ctx, stream));
}

extern "C" int h264a_lookahead_streams(h264a_ctx* ctx, const h264a_la_stream* streams, int nstreams, int mode,
                                       void* stream) {
    if (!ctx || !streams) return fail(H264A_E_ARG, "lookahead_streams: null pointer");
    if (nstreams < 1) return fail(H264A_E_ARG, "lookahead_streams: need at least one stream");
    return la_run(ctx, streams, nstreams, mode, pick_stream(ctx, stream));
}
