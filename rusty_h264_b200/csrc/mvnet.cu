// mvnet.cu -- the learned motion-vector proposal network: training and
// inference kernels (bf16 tensor-core products, fp32 accumulation) and the
// C ABI around them.
//
// The network has no counterpart in the reference encoder: rusty_h264 runs
// motion_search (crates/rusty_h264-encoder/src/mb16.rs:2433) on every MB.
// Here a small conv net looks at an MB's co-located 48x48 regions of the
// current and reference frames plus three neighbour MVs and proposes the 8
// most likely full-pel MVs; h264a_me_frames_learned prices them with the
// search's exact integer cost and refines the best one with the reference's
// own sub-pel refinement (motion_search with a start vector).
//
// Network (per MB):  X0 48x48x2 -> conv1 3x3/2 -> 24x24x16 -> conv2 3x3/2 ->
// 12x12x32 -> conv3 3x3/2 -> 6x6x32 -> [1152 features | 6 MV features | 10
// zeros] = 1168 -> FC1 -> 256 -> head -> 296 logits (289 classes: full-pel
// offsets dx, dy in -8..8, class (dy+8)*17 + dx+8).  ReLU after every layer
// but the head.  Activations are stored as bf16 (NHWC), every product runs on
// the tensor cores (tcgen05.mma, bf16 operands, fp32 accumulators in tensor
// memory).
//
// Every layer is one implicit GEMM: C[M][N] = sum_k A[m][k] B[k][n], with A
// and B gathered on the fly by a functor (im2col of a stride-2 3x3 window, a
// transposed view of a weight or activation tensor, ...) and an epilogue
// functor (bias + ReLU + bf16 store, ReLU-mask + bf16 store, or an fp32
// atomic add for weight gradients, whose K dimension -- the batch times the
// output positions -- is split over CTAs).  Weight gradients get their bias
// gradient from an extra K column of ones.
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "h264a_device.cuh"
#include "h264accel_internal.h"

namespace h264a {
namespace mvnet {

// ---- shapes and the flat parameter vector --------------------------------
constexpr int NCLS = 289, HEAD_N = 296, FEAT = 1168, HID = 256, CONVF = 1152;
constexpr int O_W1 = 0, N_W1 = 16 * 9 * 2;
constexpr int O_B1 = O_W1 + N_W1;
constexpr int O_W2 = O_B1 + 16, N_W2 = 32 * 9 * 16;
constexpr int O_B2 = O_W2 + N_W2;
constexpr int O_W3 = O_B2 + 32, N_W3 = 32 * 9 * 32;
constexpr int O_B3 = O_W3 + N_W3;
constexpr int O_W4 = O_B3 + 32, N_W4 = HID * FEAT;
constexpr int O_B4 = O_W4 + N_W4;
constexpr int O_W5 = O_B4 + HID, N_W5 = HEAD_N * HID;
constexpr int O_B5 = O_W5 + N_W5;
constexpr int NPARAMS = O_B5 + HEAD_N;
static_assert(NPARAMS == H264A_MVNET_NPARAMS, "parameter count");
static_assert((O_W1 | O_W2 | O_W3 | O_W4 | O_W5) % 2 == 0, "weights start on bf16 pairs");


typedef uint16_t bf16_t;  // raw bf16 bits

__device__ __forceinline__ bf16_t f2bf(float f) {  // round to nearest even
    uint32_t u = __float_as_uint(f);
    u += 0x7fffu + ((u >> 16) & 1u);
    return bf16_t(u >> 16);
}
__device__ __forceinline__ float bf2f(bf16_t b) { return __uint_as_float(uint32_t(b) << 16); }
__device__ __forceinline__ uint32_t pack2(bf16_t lo, bf16_t hi) { return uint32_t(lo) | (uint32_t(hi) << 16); }
__device__ __forceinline__ uint32_t ld_pair(const bf16_t* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ uint4 ld8(const bf16_t* p) { return *reinterpret_cast<const uint4*>(p); }
// 8 values (bias added, ReLU) rounded to bf16 and stored as one 16-byte word
__device__ __forceinline__ void st8_relu(bf16_t* dst, const float* v, const bf16_t* bias) {
    uint32_t w[4];
#pragma unroll
    for (int i = 0; i < 4; i++)
        w[i] = pack2(f2bf(fmaxf(v[2 * i] + bf2f(bias[2 * i]), 0.f)), f2bf(fmaxf(v[2 * i + 1] + bf2f(bias[2 * i + 1]), 0.f)));
    *reinterpret_cast<uint4*>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
}

// ---- a batch: frame pairs of one geometry, every MB a sample ---------------
// Trunk maps (NHWC bf16): A1 (ch/2)x(cw/2)x16, A2 (ch/4)x(cw/4)x32, A3
// (ch/8)x(cw/8)x32 per pair; samples are the pairs' MBs, pair-major, raster
// order within a pair.
struct Geo {
    const h264a_mvnet_pair* pairs;
    int P, cw, ch;
    int H1, W1, H2, W2, H3, W3;
    int mb_w, mb_h, nmb;
    const int16_t* nmv;     // 6 per sample
    const int16_t* labels;  // 1 per sample (training)
};

// X0 pair (reference, current) at pixel (iy, ix) of pair b; zero outside the
// frame (the conv's padding).
__device__ __forceinline__ uint32_t x0_pair(const Geo& g, int b, int iy, int ix) {
    if (iy < 0 || iy >= g.ch || ix < 0 || ix >= g.cw) return 0u;
    const h264a_mvnet_pair p = g.pairs[b];
    const long long o = (long long)iy * g.cw + ix;
    const float r = (float(p.d_ref[o]) - 128.f) * (1.f / 64.f), c = (float(p.d_cur[o]) - 128.f) * (1.f / 64.f);
    return pack2(f2bf(r), f2bf(c));  // exact: k/64 with |k| <= 128
}
__device__ __forceinline__ bf16_t x0_one(const Geo& g, int b, int iy, int ix, int ci) {
    const uint32_t v = x0_pair(g, b, iy, ix);
    return bf16_t(ci ? (v >> 16) : (v & 0xffffu));
}
__device__ __forceinline__ bf16_t mv_feat(const Geo& g, int m, int i) {
    const int v = min(max(int(g.nmv[6LL * m + i]), -128), 128);
    return f2bf(float(v) * (1.f / 64.f));  // exact
}

// ---- the tcgen05 GEMM: 128 x BN tiles, accumulators in tensor memory --------
// The GEMM of every layer, C[M][N] = sum_k A[m][k] B[k][n] (op.a(m, k) /
// op.b(k, n) gather the bf16 pair (k, k+1), zero past their tensor; op.store
// takes each fp32 result; CTA z covers k in [z*kchunk, ...)), on the sm_100
// tensor cores: per 64-wide K step all 256 threads gather the A (128 x 64)
// and B (BN x 64) tiles into one of two shared-memory stages, one thread
// issues four tcgen05.mma (M 128, N BN, K 16, bf16 in, fp32 accumulated in
// tensor memory) and commits them to the stage's mbarrier, and the gathers of
// the next step overlap them.  The epilogue reads the accumulator rows with
// tcgen05.ld: warp w may read tensor-memory lanes 32(w % 4) .. +31 (its tile
// rows), warps w and w + 4 taking half of the columns each.
constexpr int TC_BM = 128, TC_BK = 64, TC_THREADS = 256;

template <int BN>
constexpr int tc_cols() {
    return BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
}

// A K-major operand tile of R rows x 64 k (bf16) in the canonical
// no-swizzle UMMA layout: 8x8 core matrices of 128 contiguous bytes (8 rows
// of 16 bytes), the eight k-chunks of an 8-row group 128 bytes apart (the
// leading byte offset) and the groups 1024 bytes apart (the stride byte
// offset).  Byte offset of (row, k-chunk):
__device__ __forceinline__ uint32_t tc_off(int row, int chunk) {
    return uint32_t(((row >> 3) * 8 + chunk) * 128 + (row & 7) * 16);
}
// The shared-memory matrix descriptor of such a tile from shared address a:
// start >> 4 (bits 0-13), leading byte offset 128 >> 4 (16-29), stride byte
// offset 1024 >> 4 (32-45), descriptor version 1 (46-47), base offset 0,
// layout SWIZZLE_NONE (61-63).
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t a) {
    return uint64_t((a >> 4) & 0x3fffu) | (uint64_t(128 >> 4) << 16) | (uint64_t(1024 >> 4) << 32) | (1ull << 46);
}
// The instruction descriptor of kind::f16: fp32 accumulator (bits 4-5 = 1),
// A and B bf16 (7-9 = 1, 10-12 = 1), both K-major (15, 16 = 0), N >> 3
// (17-22), M >> 4 (24-28).
template <int BN>
constexpr uint32_t tc_idesc() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(BN >> 3) << 17) | (uint32_t(TC_BM >> 4) << 24);
}

__device__ __forceinline__ uint32_t tc_smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// Waits (bounded) for phase `parity` of an mbarrier; on timeout records 4 in
// status and keeps waiting up to twice as long, so that no tensor-core work
// is left reading a stage or writing tensor memory.
__device__ __forceinline__ void tc_wait(uint32_t bar, uint32_t parity, int* status) {
    constexpr int kLimit = 1 << 22;
    for (int it = 0; !mbar_try_wait(bar, parity); it++) {
        if (it == kLimit && status != nullptr) atomicCAS(status, 0, 4);
        if (it >= 2 * kLimit) break;
    }
}

// An Op with `static constexpr bool kVec = true` also gathers 8 consecutive
// k at once (op.a8(m, k), op.b8(k, n): 16 bytes, k a multiple of 8, zero past
// its tensor) and stores 8 consecutive n (op.store8(m, n, v)); the GEMM then
// moves each 16-byte chunk of a stage with one load (K and N multiples of 8).
// Such an Op also names a `Row` (what its gathers need of output row m:
// sample, position, base offset) made once per CTA row by op.row(m), so the
// per-chunk gather op.a8(row, k) does no division by a runtime size.
template <class Op, class = void>
struct VecOp : std::false_type {
    using Row = int;
};
template <class Op>
struct VecOp<Op, std::void_t<decltype(Op::kVec)>> : std::bool_constant<Op::kVec> {
    using Row = typename Op::Row;
};

template <int BN, class Op>
__global__ void __launch_bounds__(TC_THREADS) gemm_tc_kernel(const Op op, int M, int N, int K, int kchunk, int* status) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "tcgen05 N for M = 128");
    constexpr int A_BYTES = TC_BM * TC_BK * 2, B_BYTES = BN * TC_BK * 2, STAGE = A_BYTES + B_BYTES;
    constexpr int NCOL = tc_cols<BN>();
    constexpr uint32_t IDESC = tc_idesc<BN>();
    extern __shared__ __align__(128) uint8_t tc_smem[];
    __shared__ __align__(8) unsigned long long tc_bar[2];
    __shared__ uint32_t tc_tmem;
    __shared__ typename VecOp<Op>::Row tc_rows[VecOp<Op>::value ? TC_BM : 1];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * TC_BM, n0 = blockIdx.y * BN;
    if constexpr (VecOp<Op>::value) {
        for (int i = tid; i < TC_BM; i += TC_THREADS) tc_rows[i] = op.row(min(m0 + i, M - 1));
    }  // read after the __syncthreads below
    const int kb = blockIdx.z * kchunk, ke = min(K, kb + kchunk);
    const uint32_t sbase = tc_smem_u32(tc_smem), bar0 = tc_smem_u32(&tc_bar[0]);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(&tc_tmem)),
                     "r"(NCOL));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tc_tmem;
    const int nk = ke > kb ? (ke - kb + TC_BK - 1) / TC_BK : 0;
    for (int it = 0; it < nk; it++) {
        const int st = it & 1;
        const int k0 = kb + it * TC_BK;
        const uint32_t sa = sbase + uint32_t(st * STAGE), sb = sa + A_BYTES;
        // consecutive threads fill consecutive 16-byte rows of a core
        // matrix, so a warp's stores meet no bank twice
        if constexpr (VecOp<Op>::value) {
            // the step's gathers are issued before waiting for the stage, so
            // they overlap the MMAs still reading it
            constexpr int AQ = TC_BM * 8 / TC_THREADS, BQ = (BN * 8 + TC_THREADS - 1) / TC_THREADS;
            uint4 va[AQ], vb[BQ];
#pragma unroll
            for (int j = 0; j < AQ; j++) {
                const int q = tid + j * TC_THREADS;
                const int row = ((q >> 6) << 3) | (q & 7), c = (q >> 3) & 7, m = m0 + row, k = k0 + 8 * c;
                va[j] = (m < M && k < ke) ? op.a8(tc_rows[row], k) : make_uint4(0u, 0u, 0u, 0u);
            }
#pragma unroll
            for (int j = 0; j < BQ; j++) {
                const int q = tid + j * TC_THREADS;
                const int row = ((q >> 6) << 3) | (q & 7), c = (q >> 3) & 7, n = n0 + row, k = k0 + 8 * c;
                vb[j] = (q < BN * 8 && n < N && k < ke) ? op.b8(k, n) : make_uint4(0u, 0u, 0u, 0u);
            }
            // the stage's previous MMAs (step it - 2) have read it
            if (it >= 2) tc_wait(bar0 + 8 * st, uint32_t((it - 2) >> 1) & 1u, status);
#pragma unroll
            for (int j = 0; j < AQ; j++) {
                const int q = tid + j * TC_THREADS, row = ((q >> 6) << 3) | (q & 7), c = (q >> 3) & 7;
                asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sa + tc_off(row, c)), "r"(va[j].x),
                             "r"(va[j].y), "r"(va[j].z), "r"(va[j].w)
                             : "memory");
            }
#pragma unroll
            for (int j = 0; j < BQ; j++) {
                const int q = tid + j * TC_THREADS, row = ((q >> 6) << 3) | (q & 7), c = (q >> 3) & 7;
                if (q < BN * 8)
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sb + tc_off(row, c)), "r"(vb[j].x),
                                 "r"(vb[j].y), "r"(vb[j].z), "r"(vb[j].w)
                                 : "memory");
            }
        } else {
            // the stage's previous MMAs (step it - 2) have read it
            if (it >= 2) tc_wait(bar0 + 8 * st, uint32_t((it - 2) >> 1) & 1u, status);
            for (int q = tid; q < TC_BM * 8; q += TC_THREADS) {
                const int row = ((q >> 6) << 3) | (q & 7), c = (q >> 3) & 7, m = m0 + row, k = k0 + 8 * c;
                uint32_t v[4];
#pragma unroll
                for (int i = 0; i < 4; i++) v[i] = (m < M && k + 2 * i < ke) ? op.a(m, k + 2 * i) : 0u;
                asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sa + tc_off(row, c)), "r"(v[0]),
                             "r"(v[1]), "r"(v[2]), "r"(v[3])
                             : "memory");
            }
            for (int q = tid; q < BN * 8; q += TC_THREADS) {
                const int row = ((q >> 6) << 3) | (q & 7), c = (q >> 3) & 7, n = n0 + row, k = k0 + 8 * c;
                uint32_t v[4];
#pragma unroll
                for (int i = 0; i < 4; i++) v[i] = (n < N && k + 2 * i < ke) ? op.b(k + 2 * i, n) : 0u;
                asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sb + tc_off(row, c)), "r"(v[0]),
                             "r"(v[1]), "r"(v[2]), "r"(v[3])
                             : "memory");
            }
        }
        // the tiles' generic-proxy writes, visible to the tensor cores
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int j = 0; j < TC_BK / 16; j++) {
                const uint64_t da = tc_sdesc(sa + 256u * j), db = tc_sdesc(sb + 256u * j);
                const uint32_t acc = (it > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(IDESC), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar0 +
                                                                                                          8 * st)
                         : "memory");
        }
    }
    if (nk > 0) {
        // the last step's commit completes after every earlier MMA
        tc_wait(bar0 + 8 * ((nk - 1) & 1), uint32_t((nk - 1) >> 1) & 1u, status);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const int row = m0 + (warp & 3) * 32 + lane;
        const uint32_t taddr = tmem + (uint32_t((warp & 3) * 32) << 16);
        const int cb = (warp >> 2) * (BN / 2);
#pragma unroll 1
        for (int c0 = cb; c0 < cb + BN / 2; c0 += 8) {
            uint32_t r[8];
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                         : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                           "=r"(r[7])
                         : "r"(taddr + uint32_t(c0)));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if constexpr (VecOp<Op>::value) {
                if (row < M && n0 + c0 < N) {
                    float f[8];
#pragma unroll
                    for (int i = 0; i < 8; i++) f[i] = __uint_as_float(r[i]);
                    op.store8(row, n0 + c0, f);
                }
            } else if (row < M) {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const int n = n0 + c0 + i;
                    if (n < N) op.store(row, n, __uint_as_float(r[i]));
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL));
}

// ---- the layers as GEMM operands --------------------------------------------
struct Bufs {
    const bf16_t* w;  // bf16 parameters
    float* grad;      // fp32 parameter gradients (accumulated)
    bf16_t *a1, *a2, *a3, *h, *dl, *dh, *df, *da3, *da2, *da1;
    float* logits;
};

// im2col gather of a stride-2 3x3 conv over NHWC bf16 maps of H x W x C:
// row m = (pair, oy, ox) of the output, column k = tap*C + ci.
template <int C>
__device__ __forceinline__ long long im2col_off(int H, int W, int m, int k) {
    const int OW = W >> 1, OHW = (H >> 1) * OW;
    const int b = m / OHW, r = m - b * OHW, oy = r / OW, ox = r - oy * OW;
    const int tap = k / C, ci = k - tap * C, ky = tap / 3, kx = tap - ky * 3;
    const int iy = 2 * oy + ky - 1, ix = 2 * ox + kx - 1;
    if (iy < 0 || iy >= H || ix < 0 || ix >= W) return -1;
    return ((long long)(b * H + iy) * W + ix) * C + ci;
}

// conv1 forward: M = P*H1*W1, N = 16, K = 18 (padded to 32)
struct Conv1Fwd {
    Geo g; Bufs z;
    __device__ uint32_t a(int m, int k) const {
        if (k >= 18) return 0u;
        const int OHW = g.H1 * g.W1;
        const int b = m / OHW, r = m - b * OHW, oy = r / g.W1, ox = r - oy * g.W1;
        const int tap = k >> 1, ky = tap / 3, kx = tap - ky * 3;
        return x0_pair(g, b, 2 * oy + ky - 1, 2 * ox + kx - 1);
    }
    __device__ uint32_t b(int k, int n) const { return k < 18 ? ld_pair(z.w + O_W1 + n * 18 + k) : 0u; }
    __device__ void store(int m, int n, float v) const {
        z.a1[(long long)m * 16 + n] = f2bf(fmaxf(v + bf2f(z.w[O_B1 + n]), 0.f));
    }
    static constexpr bool kVec = true;
    struct Row {
        int b, y0, x0;  // pair, top-left input pixel of the 3x3 window
    };
    __device__ Row row(int m) const {
        const int OHW = g.H1 * g.W1;
        const int b = m / OHW, r = m - b * OHW, oy = r / g.W1, ox = r - oy * g.W1;
        return Row{b, 2 * oy - 1, 2 * ox - 1};
    }
    __device__ uint4 a8(const Row& w, int k) const {
        uint32_t v[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int tap = (k >> 1) + i, ky = (tap * 11) >> 5, kx = tap - ky * 3;  // ky = tap / 3 for tap < 9
            v[i] = tap < 9 ? x0_pair(g, w.b, w.y0 + ky, w.x0 + kx) : 0u;
        }
        return make_uint4(v[0], v[1], v[2], v[3]);
    }
    __device__ uint4 b8(int k, int n) const {
        uint32_t v[4];
#pragma unroll
        for (int i = 0; i < 4; i++) v[i] = b(k + 2 * i, n);
        return make_uint4(v[0], v[1], v[2], v[3]);
    }
    __device__ void store8(int m, int n, const float* v) const { st8_relu(z.a1 + (long long)m * 16 + n, v, z.w + O_B1 + n); }
};
// conv2 / conv3 forward: im2col of the previous map
template <int C, int OW, int OB, int WHICH>
struct ConvFwd {
    Geo g; Bufs z;
    __device__ uint32_t a(int m, int k) const {
        const long long o = WHICH == 2 ? im2col_off<C>(g.H1, g.W1, m, k) : im2col_off<C>(g.H2, g.W2, m, k);
        return o < 0 ? 0u : ld_pair((WHICH == 2 ? z.a1 : z.a2) + o);
    }
    __device__ uint32_t b(int k, int n) const { return ld_pair(z.w + OW + n * 9 * C + k); }
    __device__ void store(int m, int n, float v) const {
        (WHICH == 2 ? z.a2 : z.a3)[(long long)m * 32 + n] = f2bf(fmaxf(v + bf2f(z.w[OB + n]), 0.f));
    }
    // k a multiple of 8 (C = 16 or 32): the chunk is 8 channels of one tap,
    // 16 contiguous bytes of the NHWC map
    static constexpr bool kVec = true;
    struct Row {
        long long base;  // element offset of input pixel (y0, x0), channel 0 (may lie outside the map)
        int y0, x0;
    };
    __device__ Row row(int m) const {
        const int H = WHICH == 2 ? g.H1 : g.H2, W = WHICH == 2 ? g.W1 : g.W2;
        const int ow = W >> 1, ohw = (H >> 1) * ow;
        const int b = m / ohw, r = m - b * ohw, oy = r / ow, ox = r - oy * ow;
        return Row{((long long)(b * H + 2 * oy - 1) * W + 2 * ox - 1) * C, 2 * oy - 1, 2 * ox - 1};
    }
    __device__ uint4 a8(const Row& w, int k) const {
        const int H = WHICH == 2 ? g.H1 : g.H2, W = WHICH == 2 ? g.W1 : g.W2;
        const int tap = k / C, ci = k - tap * C, ky = (tap * 11) >> 5, kx = tap - ky * 3;
        const int iy = w.y0 + ky, ix = w.x0 + kx;
        if (iy < 0 || iy >= H || ix < 0 || ix >= W) return make_uint4(0u, 0u, 0u, 0u);
        return ld8((WHICH == 2 ? z.a1 : z.a2) + w.base + (long long)(ky * W + kx) * C + ci);
    }
    __device__ uint4 b8(int k, int n) const { return ld8(z.w + OW + n * 9 * C + k); }
    __device__ void store8(int m, int n, const float* v) const {
        st8_relu((WHICH == 2 ? z.a2 : z.a3) + (long long)m * 32 + n, v, z.w + OB + n);
    }
};
using Conv2Fwd = ConvFwd<16, O_W2, O_B2, 2>;
using Conv3Fwd = ConvFwd<32, O_W3, O_B3, 3>;

// offset in A3 of feature k < 1152 of sample m (its MB's 6x6-cell crop), or
// -1 outside the map
__device__ __forceinline__ long long crop_off(const Geo& g, int m, int k) {
    const int b = m / g.nmb, r = m - b * g.nmb, mby = r / g.mb_w, mbx = r - mby * g.mb_w;
    const int cy = k / 192, rem = k - cy * 192, cx = rem >> 5, c = rem & 31;
    const int y = 2 * mby - 2 + cy, x = 2 * mbx - 2 + cx;
    if (y < 0 || y >= g.H3 || x < 0 || x >= g.W3) return -1;
    return ((long long)(b * g.H3 + y) * g.W3 + x) * 32 + c;
}
// the FC1 input row of sample m, pair (k, k+1)
__device__ __forceinline__ uint32_t feat_pair(const Geo& g, const Bufs& z, int m, int k) {
    if (k < CONVF) {
        const long long o = crop_off(g, m, k);
        return o < 0 ? 0u : ld_pair(z.a3 + o);
    }
    if (k < CONVF + 6) return pack2(mv_feat(g, m, k - CONVF), mv_feat(g, m, k - CONVF + 1));
    return 0u;
}
__device__ __forceinline__ bf16_t feat_one(const Geo& g, const Bufs& z, int m, int k) {
    if (k < CONVF) {
        const long long o = crop_off(g, m, k);
        return o < 0 ? bf16_t(0) : z.a3[o];
    }
    if (k < CONVF + 6) return mv_feat(g, m, k - CONVF);
    return 0;
}
struct Fc1Fwd {
    Geo g; Bufs z;
    __device__ uint32_t a(int m, int k) const { return feat_pair(g, z, m, k); }
    __device__ uint32_t b(int k, int n) const { return ld_pair(z.w + O_W4 + (long long)n * FEAT + k); }
    __device__ void store(int m, int n, float v) const {
        z.h[(long long)m * HID + n] = f2bf(fmaxf(v + bf2f(z.w[O_B4 + n]), 0.f));
    }
    // k < 1152, a multiple of 8: 8 channels of one crop cell, 16 contiguous
    // bytes of A3; then the 6 neighbour-MV features and zeros
    static constexpr bool kVec = true;
    struct Row {
        long long base;  // element offset of the crop's top-left cell (y0, x0), channel 0
        int m, y0, x0;
    };
    __device__ Row row(int m) const {
        const int b = m / g.nmb, r = m - b * g.nmb, mby = r / g.mb_w, mbx = r - mby * g.mb_w;
        const int y0 = 2 * mby - 2, x0 = 2 * mbx - 2;
        return Row{((long long)(b * g.H3 + y0) * g.W3 + x0) * 32, m, y0, x0};
    }
    __device__ uint4 a8(const Row& w, int k) const {
        if (k < CONVF) {
            const int cy = k / 192, rem = k - cy * 192, cx = rem >> 5, c = rem & 31;
            const int y = w.y0 + cy, x = w.x0 + cx;
            if (y < 0 || y >= g.H3 || x < 0 || x >= g.W3) return make_uint4(0u, 0u, 0u, 0u);
            return ld8(z.a3 + w.base + (long long)(cy * g.W3 + cx) * 32 + c);
        }
        if (k == CONVF)
            return make_uint4(pack2(mv_feat(g, w.m, 0), mv_feat(g, w.m, 1)), pack2(mv_feat(g, w.m, 2), mv_feat(g, w.m, 3)),
                              pack2(mv_feat(g, w.m, 4), mv_feat(g, w.m, 5)), 0u);
        return make_uint4(0u, 0u, 0u, 0u);
    }
    __device__ uint4 b8(int k, int n) const { return ld8(z.w + O_W4 + (long long)n * FEAT + k); }
    __device__ void store8(int m, int n, const float* v) const { st8_relu(z.h + (long long)m * HID + n, v, z.w + O_B4 + n); }
};
struct HeadFwd {
    Bufs z;
    __device__ uint32_t a(int m, int k) const { return ld_pair(z.h + (long long)m * HID + k); }
    __device__ uint32_t b(int k, int n) const { return ld_pair(z.w + O_W5 + n * HID + k); }
    __device__ void store(int m, int n, float v) const { z.logits[(long long)m * HEAD_N + n] = v + bf2f(z.w[O_B5 + n]); }
    static constexpr bool kVec = true;
    using Row = int;
    __device__ Row row(int m) const { return m; }
    __device__ uint4 a8(Row m, int k) const { return ld8(z.h + (long long)m * HID + k); }
    __device__ uint4 b8(int k, int n) const { return ld8(z.w + O_W5 + n * HID + k); }
    __device__ void store8(int m, int n, const float* v) const {
        float4* d = reinterpret_cast<float4*>(z.logits + (long long)m * HEAD_N + n);
        const bf16_t* bias = z.w + O_B5 + n;
        d[0] = make_float4(v[0] + bf2f(bias[0]), v[1] + bf2f(bias[1]), v[2] + bf2f(bias[2]), v[3] + bf2f(bias[3]));
        d[1] = make_float4(v[4] + bf2f(bias[4]), v[5] + bf2f(bias[5]), v[6] + bf2f(bias[6]), v[7] + bf2f(bias[7]));
    }
};

// ---- backward -----------------------------------------------------------------
// Weight gradient of a layer y = W x: dW[i][j] = sum_m dy[m][i] * x[m][j], the
// GEMM's M = output channels, N = input columns (+1 for the bias, a column of
// ones), K = rows m (the samples, or the pairs times the map positions).
// a(i, m) / b(m, j) pair two consecutive rows m, m+1 (zero past K).
__device__ __forceinline__ uint32_t col_pair(const bf16_t* y, int ld, int i, int m, int K) {
    const bf16_t lo = y[(long long)m * ld + i];
    const bf16_t hi = m + 1 < K ? y[(long long)(m + 1) * ld + i] : bf16_t(0);
    return pack2(lo, hi);
}
constexpr bf16_t BF_ONE = 0x3f80;

struct HeadBwdW {  // M = 296, N = 258 (256 + bias + pad), K = B
    Bufs z; int B;
    __device__ uint32_t a(int i, int m) const { return col_pair(z.dl, HEAD_N, i, m, B); }
    __device__ uint32_t b(int m, int j) const {
        if (j < HID) return col_pair(z.h, HID, j, m, B);
        if (j == HID) return pack2(BF_ONE, m + 1 < B ? BF_ONE : bf16_t(0));
        return 0u;
    }
    __device__ void store(int i, int j, float v) const {
        if (j < HID) atomicAdd(z.grad + O_W5 + i * HID + j, v);
        else if (j == HID) atomicAdd(z.grad + O_B5 + i, v);
    }
};
struct HeadBwdData {  // dh = relu'(h) * (dl W5): M = B, N = 256, K = 296
    Bufs z;
    __device__ uint32_t a(int m, int k) const { return ld_pair(z.dl + (long long)m * HEAD_N + k); }
    __device__ uint32_t b(int k, int n) const { return pack2(z.w[O_W5 + k * HID + n], z.w[O_W5 + (k + 1) * HID + n]); }
    __device__ void store(int m, int n, float v) const {
        const long long o = (long long)m * HID + n;
        z.dh[o] = z.h[o] != 0 ? f2bf(v) : bf16_t(0);
    }
};
struct Fc1BwdW {  // M = 256, N = 1170, K = B
    Geo g; Bufs z; int B;
    __device__ uint32_t a(int i, int m) const { return col_pair(z.dh, HID, i, m, B); }
    __device__ uint32_t b(int m, int j) const {
        if (j < FEAT) return pack2(feat_one(g, z, m, j), m + 1 < B ? feat_one(g, z, m + 1, j) : bf16_t(0));
        if (j == FEAT) return pack2(BF_ONE, m + 1 < B ? BF_ONE : bf16_t(0));
        return 0u;
    }
    __device__ void store(int i, int j, float v) const {
        if (j < FEAT) atomicAdd(z.grad + O_W4 + (long long)i * FEAT + j, v);
        else if (j == FEAT) atomicAdd(z.grad + O_B4 + i, v);
    }
};
struct Fc1BwdData {  // df = (dh W4)[:, :1152]: M = B, N = 1152, K = 256
    Bufs z;
    __device__ uint32_t a(int m, int k) const { return ld_pair(z.dh + (long long)m * HID + k); }
    __device__ uint32_t b(int k, int n) const {
        return pack2(z.w[O_W4 + (long long)k * FEAT + n], z.w[O_W4 + (long long)(k + 1) * FEAT + n]);
    }
    __device__ void store(int m, int n, float v) const { z.df[(long long)m * CONVF + n] = f2bf(v); }
};
// conv weight gradient: M = CO, N = 9*C + 2 (bias column at 9*C), K = P*OH*OW
template <int C, int CO, int OW, int OB, int WHICH>
struct ConvBwdW {
    Geo g; Bufs z; int K;
    __device__ const bf16_t* dy() const { return WHICH == 1 ? z.da1 : (WHICH == 2 ? z.da2 : z.da3); }
    __device__ bf16_t xin(int m, int j) const {
        if (WHICH == 1) {  // the network input, read from the frames
            const int OHW = g.H1 * g.W1;
            const int b = m / OHW, r = m - b * OHW, oy = r / g.W1, ox = r - oy * g.W1;
            const int tap = j >> 1, ky = tap / 3, kx = tap - ky * 3;
            return x0_one(g, b, 2 * oy + ky - 1, 2 * ox + kx - 1, j & 1);
        }
        const long long o = WHICH == 2 ? im2col_off<C>(g.H1, g.W1, m, j) : im2col_off<C>(g.H2, g.W2, m, j);
        return o < 0 ? bf16_t(0) : (WHICH == 2 ? z.a1 : z.a2)[o];
    }
    __device__ uint32_t a(int i, int m) const { return col_pair(dy(), CO, i, m, K); }
    __device__ uint32_t b(int m, int j) const {
        if (j < 9 * C) return pack2(xin(m, j), m + 1 < K ? xin(m + 1, j) : bf16_t(0));
        if (j == 9 * C) return pack2(BF_ONE, m + 1 < K ? BF_ONE : bf16_t(0));
        return 0u;
    }
    __device__ void store(int i, int j, float v) const {
        if (j < 9 * C) atomicAdd(z.grad + OW + i * 9 * C + j, v);
        else if (j == 9 * C) atomicAdd(z.grad + OB + i, v);
    }
};
using Conv1BwdW = ConvBwdW<2, 16, O_W1, O_B1, 1>;
using Conv2BwdW = ConvBwdW<16, 32, O_W2, O_B2, 2>;
using Conv3BwdW = ConvBwdW<32, 32, O_W3, O_B3, 3>;
// conv input gradient (stride-2 transposed conv): rows m = (pair, iy, ix) of
// the H x W input, N = C input channels, K = 9 taps x CO output channels: tap
// (ky, kx) of input (iy, ix) feeds output ((iy + 1 - ky) / 2, (ix + 1 - kx) / 2)
// when both are even and inside the output map.
template <int C, int CO, int OW, int WHICH>
struct ConvBwdData {
    Geo g; Bufs z;
    __device__ uint32_t a(int m, int k) const {
        const int H = WHICH == 3 ? g.H2 : g.H1, W = WHICH == 3 ? g.W2 : g.W1;
        const int OH = H >> 1, OWd = W >> 1;
        const int HW = H * W, b = m / HW, r = m - b * HW, iy = r / W, ix = r - iy * W;
        const int tap = k / CO, co = k - tap * CO, ky = tap / 3, kx = tap - ky * 3;
        const int ty = iy + 1 - ky, tx = ix + 1 - kx;
        if ((ty | tx) < 0 || (ty & 1) || (tx & 1) || ty >= 2 * OH || tx >= 2 * OWd) return 0u;
        return ld_pair((WHICH == 3 ? z.da3 : z.da2) + ((long long)(b * OH + (ty >> 1)) * OWd + (tx >> 1)) * CO + co);
    }
    __device__ uint32_t b(int k, int n) const {
        const int tap = k / CO, co = k - tap * CO;
        return pack2(z.w[OW + co * 9 * C + tap * C + n], z.w[OW + (co + 1) * 9 * C + tap * C + n]);
    }
    __device__ void store(int m, int n, float v) const {
        const long long o = (long long)m * C + n;
        const bf16_t* xa = WHICH == 3 ? z.a2 : z.a1;
        (WHICH == 3 ? z.da2 : z.da1)[o] = xa[o] != 0 ? f2bf(v) : bf16_t(0);
    }
};
using Conv3BwdData = ConvBwdData<32, 32, O_W3, 3>;
using Conv2BwdData = ConvBwdData<16, 32, O_W2, 2>;

// da3 = relu'(a3) * (sum of the crop gradients of the up to 9 MBs whose 6x6
// crop holds the cell): one thread per (pair, cell, channel pair).
__global__ void uncrop_kernel(const Geo g, const bf16_t* __restrict__ df, const bf16_t* __restrict__ a3,
                              bf16_t* __restrict__ da3) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = (long long)g.P * g.H3 * g.W3 * 16;
    if (i >= total) return;
    const int c = int(i & 15) * 2;
    const long long cell = i >> 4;
    const int x = int(cell % g.W3), y = int((cell / g.W3) % g.H3), b = int(cell / ((long long)g.W3 * g.H3));
    float s0 = 0.f, s1 = 0.f;
    const int ylo = max(0, (y - 2) >> 1), yhi = min(g.mb_h - 1, (y + 2) >> 1);
    const int xlo = max(0, (x - 2) >> 1), xhi = min(g.mb_w - 1, (x + 2) >> 1);
    for (int mby = ylo; mby <= yhi; mby++) {
        const int cy = y - 2 * mby + 2;
        if (cy < 0 || cy >= 6) continue;
        for (int mbx = xlo; mbx <= xhi; mbx++) {
            const int cx = x - 2 * mbx + 2;
            if (cx < 0 || cx >= 6) continue;
            const long long m = (long long)b * g.nmb + mby * g.mb_w + mbx;
            const uint32_t v = ld_pair(df + m * CONVF + cy * 192 + cx * 32 + c);
            s0 += bf2f(bf16_t(v & 0xffffu));
            s1 += bf2f(bf16_t(v >> 16));
        }
    }
    const long long o = cell * 32 + c;
    da3[o] = a3[o] != 0 ? f2bf(s0) : bf16_t(0);
    da3[o + 1] = a3[o + 1] != 0 ? f2bf(s1) : bf16_t(0);
}

// ---- loss, proposals, optimiser -------------------------------------------------
// One warp per sample: softmax over the 289 classes, the sample's share of the
// mean cross-entropy (atomically summed into *loss) and dl = (p - onehot) / B
// in bf16 (zero for the 7 padding logits).
__global__ void loss_kernel(const float* __restrict__ logits, const int16_t* __restrict__ labels, int B,
                            bf16_t* __restrict__ dl, float* __restrict__ loss) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= B) return;
    const float* z = logits + (long long)w * HEAD_N;
    float mx = -INFINITY;
    for (int c = lane; c < NCLS; c += 32) mx = fmaxf(mx, z[c]);
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    float s = 0.f;
    for (int c = lane; c < NCLS; c += 32) s += expf(z[c] - mx);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const int label = min(max(int(labels[w]), 0), NCLS - 1);
    const float inv = 1.f / s, scale = 1.f / float(B);
    for (int c = lane; c < HEAD_N; c += 32) {
        float d = 0.f;
        if (c < NCLS) d = (expf(z[c] - mx) * inv - (c == label ? 1.f : 0.f)) * scale;
        dl[(long long)w * HEAD_N + c] = f2bf(d);
    }
    if (lane == 0) atomicAdd(loss, (logf(s) + mx - z[label]) * scale);
}

// One warp per sample: the 8 largest logits (ties to the lower class) as
// quarter-pel MVs, 16 i32 per sample; sample i of a batch is MB mb0 + i of
// the frame whose proposals out points to.
// A frame of a propose batch: its guide MVs (may be null) and its proposals.
struct PropFrame {
    const int32_t* guide;
    int32_t* props;
};

__device__ __forceinline__ void top8_one(const float* __restrict__ z, int32_t* __restrict__ o);

// top8 of every MB of P frames of nmb MBs each, into each frame's proposals
__global__ void top8_frames_kernel(const float* __restrict__ logits, int P, int nmb, const PropFrame* __restrict__ fr) {
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (w >= (long long)P * nmb) return;
    const int k = int(w / nmb), m = int(w - (long long)k * nmb);
    top8_one(logits + w * HEAD_N, fr[k].props + 16LL * m);
}

__device__ __forceinline__ void top8_one(const float* __restrict__ z, int32_t* __restrict__ o) {
    const int lane = threadIdx.x & 31;
    float v[10];
#pragma unroll
    for (int i = 0; i < 10; i++) {
        const int c = lane + 32 * i;
        v[i] = c < NCLS ? z[c] : -INFINITY;
    }
    for (int r = 0; r < 8; r++) {
        float bv = -INFINITY;
        int bc = 1 << 30;
#pragma unroll
        for (int i = 0; i < 10; i++)
            if (v[i] > bv) { bv = v[i]; bc = lane + 32 * i; }
        for (int s = 16; s; s >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, s);
            const int oc = __shfl_xor_sync(0xffffffffu, bc, s);
            if (ov > bv || (ov == bv && oc < bc)) { bv = ov; bc = oc; }
        }
        if ((bc & 31) == lane) {
#pragma unroll
            for (int i = 0; i < 10; i++)
                if (lane + 32 * i == bc) v[i] = -INFINITY;
        }
        if (lane == 0) {
            o[2 * r] = 4 * (bc % 17 - 8);
            o[2 * r + 1] = 4 * (bc / 17 - 8);
        }
    }
}

__global__ void adam_kernel(float* __restrict__ master, bf16_t* __restrict__ w, const float* __restrict__ grad,
                            float* __restrict__ m1, float* __restrict__ m2, int n, float lr, float b1, float b2,
                            float c1, float c2, float eps) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grad[i];
    const float a = b1 * m1[i] + (1.f - b1) * g, b = b2 * m2[i] + (1.f - b2) * g * g;
    m1[i] = a;
    m2[i] = b;
    const float nw = master[i] - lr * (a * c1) / (sqrtf(b * c2) + eps);
    master[i] = nw;
    w[i] = f2bf(nw);
}

__global__ void to_bf16_kernel(const float* __restrict__ src, bf16_t* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = f2bf(src[i]);
}

// The neighbour MV features of every MB of the P frames of a propose batch
// (frame k's MBs at samples k * nmb ..) from their guide MVs (2 i32 per MB):
// left, top, top-right MB, zero outside the frame or when the frame has no
// guide MVs.
__global__ void guide_frames_kernel(const PropFrame* __restrict__ fr, int P, int mb_w, int mb_h,
                                    int16_t* __restrict__ nmv) {
    const int nmb = mb_w * mb_h;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)P * nmb) return;
    const int k = int(t / nmb), m = int(t - (long long)k * nmb);
    const int32_t* guide = fr[k].guide;
    const int mbx = m % mb_w, mby = m / mb_w;
    const int nb[3] = {mbx > 0 ? m - 1 : -1, mby > 0 ? m - mb_w : -1, (mby > 0 && mbx + 1 < mb_w) ? m - mb_w + 1 : -1};
    int16_t* o = nmv + 6 * t;
    for (int j = 0; j < 3; j++) {
        int vx = 0, vy = 0;
        if (guide && nb[j] >= 0) {
            vx = guide[2 * nb[j]];
            vy = guide[2 * nb[j] + 1];
        }
        o[2 * j] = int16_t(min(max(vx, -32768), 32767));
        o[2 * j + 1] = int16_t(min(max(vy, -32768), 32767));
    }
}

template <int BN, class Op>
static void gemm(const Op& op, int M, int N, int K, cudaStream_t st, int splits = 1) {
    constexpr int smem = 2 * (TC_BM * TC_BK * 2 + BN * TC_BK * 2);
    static const bool attr_ok = [] {  // once per instantiation (the dynamic shared memory above 48 KB)
        return cudaFuncSetAttribute(gemm_tc_kernel<BN, Op>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) ==
               cudaSuccess;
    }();
    (void)attr_ok;
    int kchunk = K;
    if (splits > 1) {
        kchunk = (K + splits - 1) / splits;
        kchunk = (kchunk + TC_BK - 1) / TC_BK * TC_BK;
        splits = (K + kchunk - 1) / kchunk;
    }
    dim3 grid((M + TC_BM - 1) / TC_BM, (N + BN - 1) / BN, splits);
    gemm_tc_kernel<BN, Op><<<grid, TC_THREADS, smem, st>>>(op, M, N, K, kchunk, nullptr);
}

// split count of a weight-gradient GEMM: about 4 waves of CTAs
static int wsplits(int M, int N, int BN, long long K, int sms) {
    const long long tiles = (long long)((M + TC_BM - 1) / TC_BM) * ((N + BN - 1) / BN);
    long long s = (4LL * sms + tiles - 1) / tiles;
    const long long maxs = (K + 1023) / 1024;  // at least 1024 rows per CTA
    if (s > maxs) s = maxs;
    return int(s < 1 ? 1 : s);
}

}  // namespace mvnet
}  // namespace h264a

using namespace h264a;
using namespace h264a::mvnet;

constexpr long long MAXPIX = H264A_MVNET_MAX_PIXELS;
constexpr long long MAXS = MAXPIX / 256;  // samples (MBs) per batch

struct h264a_mvnet {
    int device = 0, sms = 0;
    float* master = nullptr;  // fp32 parameters
    bf16_t* w = nullptr;      // their bf16 copy (what the kernels read)
    float *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
    long long step = 0;
    // maps, activations and gradients of one batch
    bf16_t *a1 = nullptr, *a2 = nullptr, *a3 = nullptr, *h = nullptr, *dl = nullptr, *dh = nullptr, *df = nullptr;
    bf16_t *da3 = nullptr, *da2 = nullptr, *da1 = nullptr;
    float* logits = nullptr;
    float* loss = nullptr;
    // inference: the batch's pair table and neighbour features
    h264a_mvnet_pair* ipairs = nullptr;
    PropFrame* iprop = nullptr;  // a propose batch's frames: guide MVs and proposals
    int16_t* inmv = nullptr;
};

namespace {

template <class T>
int dmalloc(T** p, size_t n) {
    if (cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        return fail(H264A_E_NOMEM, "mvnet: cudaMalloc failed");
    }
    return H264A_OK;
}

void free_net(h264a_mvnet* n) {
    void* ps[] = {n->master, n->w, n->grad, n->m1, n->m2, n->a1, n->a2, n->a3, n->h, n->dl, n->dh, n->df,
                  n->da3, n->da2, n->da1, n->logits, n->loss, n->ipairs, n->inmv, n->iprop};
    for (void* p : ps)
        if (p) cudaFree(p);
    delete n;
}

uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// He-normal weights (Box-Muller over splitmix64), zero biases, and zero rows /
// columns that only pad (FC1 inputs 1158..1167, head rows 289..295).
void init_params(std::vector<float>& p, uint64_t seed) {
    uint64_t s = seed;
    auto normal = [&]() {
        const double u1 = (double(splitmix(s) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
        const double u2 = double(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    p.assign(NPARAMS, 0.f);
    auto fill = [&](int off, int n, int fan_in) {
        const double sd = std::sqrt(2.0 / fan_in);
        for (int i = 0; i < n; i++) p[off + i] = float(normal() * sd);
    };
    fill(O_W1, N_W1, 18);
    fill(O_W2, N_W2, 144);
    fill(O_W3, N_W3, 288);
    fill(O_W4, N_W4, CONVF + 6);
    fill(O_W5, N_W5, HID);
    for (int o = 0; o < HID; o++)
        for (int k = CONVF + 6; k < FEAT; k++) p[O_W4 + o * FEAT + k] = 0.f;
    for (int r = NCLS; r < HEAD_N; r++)
        for (int k = 0; k < HID; k++) p[O_W5 + r * HID + k] = 0.f;
}

int upload_params(h264a_mvnet* n, const float* h) {
    H264A_CUDA(cudaMemcpy(n->master, h, sizeof(float) * NPARAMS, cudaMemcpyHostToDevice));
    to_bf16_kernel<<<(NPARAMS + 255) / 256, 256>>>(n->master, n->w, NPARAMS);
    H264A_CUDA(cudaGetLastError());
    H264A_CUDA(cudaDeviceSynchronize());
    return H264A_OK;
}

Bufs bufs(h264a_mvnet* n) {
    Bufs z;
    z.w = n->w; z.grad = n->grad;
    z.a1 = n->a1; z.a2 = n->a2; z.a3 = n->a3; z.h = n->h; z.dl = n->dl; z.dh = n->dh; z.df = n->df;
    z.da3 = n->da3; z.da2 = n->da2; z.da1 = n->da1;
    z.logits = n->logits;
    return z;
}

Geo make_geo(const h264a_mvnet_pair* pairs, int P, int cw, int ch, const int16_t* nmv, const int16_t* labels) {
    Geo g;
    g.pairs = pairs; g.P = P; g.cw = cw; g.ch = ch;
    g.H1 = ch / 2; g.W1 = cw / 2; g.H2 = ch / 4; g.W2 = cw / 4; g.H3 = ch / 8; g.W3 = cw / 8;
    g.mb_w = cw / 16; g.mb_h = ch / 16; g.nmb = g.mb_w * g.mb_h;
    g.nmv = nmv; g.labels = labels;
    return g;
}

int check_geo(const h264a_mvnet* n, const h264a_mvnet_pair* d_pairs, int P, int cw, int ch, const void* nmv) {
    if (!n || !d_pairs || !nmv) return fail(H264A_E_ARG, "mvnet: null pointer");
    if (P < 1 || cw < 16 || ch < 16 || cw % 16 || ch % 16 || cw > 8192 || ch > 8192)
        return fail(H264A_E_ARG, "mvnet: frames must be MB-aligned, 16 to 8192 pixels a side, at least one pair");
    if ((long long)P * cw * ch > MAXPIX)
        return fail(H264A_E_ARG, "mvnet: a batch holds at most " + std::to_string(MAXPIX) + " luma pixels");
    return H264A_OK;
}

void trunk_forward(h264a_mvnet* n, const Geo& g, cudaStream_t st) {
    const Bufs z = bufs(n);
    gemm<16>(Conv1Fwd{g, z}, g.P * g.H1 * g.W1, 16, 32, st);
    gemm<32>(Conv2Fwd{g, z}, g.P * g.H2 * g.W2, 32, 144, st);
    gemm<32>(Conv3Fwd{g, z}, g.P * g.H3 * g.W3, 32, 288, st);
}

void head_forward(h264a_mvnet* n, const Geo& g, cudaStream_t st) {
    const Bufs z = bufs(n);
    const int B = g.P * g.nmb;
    gemm<256>(Fc1Fwd{g, z}, B, HID, FEAT, st);
    gemm<160>(HeadFwd{z}, B, HEAD_N, HID, st);
}

void backward(h264a_mvnet* n, const Geo& g, cudaStream_t st) {
    const Bufs z = bufs(n);
    const int B = g.P * g.nmb, S = n->sms;
    const int K3 = g.P * g.H3 * g.W3, K2 = g.P * g.H2 * g.W2, K1 = g.P * g.H1 * g.W1;
    gemm<160>(HeadBwdW{z, B}, HEAD_N, HID + 2, B, st, wsplits(HEAD_N, HID + 2, 160, B, S));
    gemm<256>(HeadBwdData{z}, B, HID, HEAD_N, st);
    gemm<256>(Fc1BwdW{g, z, B}, HID, FEAT + 2, B, st, wsplits(HID, FEAT + 2, 256, B, S));
    gemm<256>(Fc1BwdData{z}, B, CONVF, HID, st);
    const long long cells = (long long)K3 * 16;
    uncrop_kernel<<<unsigned((cells + 255) / 256), 256, 0, st>>>(g, n->df, n->a3, n->da3);
    gemm<160>(Conv3BwdW{g, z, K3}, 32, 9 * 32 + 2, K3, st, wsplits(32, 290, 160, K3, S));
    gemm<32>(Conv3BwdData{g, z}, K2, 32, 288, st);
    gemm<160>(Conv2BwdW{g, z, K2}, 32, 9 * 16 + 2, K2, st, wsplits(32, 146, 160, K2, S));
    gemm<16>(Conv2BwdData{g, z}, K1, 16, 288, st);
    gemm<32>(Conv1BwdW{g, z, K1}, 16, 9 * 2 + 2, K1, st, wsplits(16, 20, 32, K1, S));
}

}  // namespace

extern "C" int h264a_mvnet_create(int device, uint64_t seed, h264a_mvnet** out) {
    if (!out) return fail(H264A_E_ARG, "mvnet_create: null out");
    *out = nullptr;
    H264A_CUDA(cudaSetDevice(device));
    h264a_mvnet* n = new h264a_mvnet();
    n->device = device;
    cudaDeviceGetAttribute(&n->sms, cudaDevAttrMultiProcessorCount, device);
    int rc = H264A_OK;
    if (!rc) rc = dmalloc(&n->master, NPARAMS);
    if (!rc) rc = dmalloc(&n->w, NPARAMS);
    if (!rc) rc = dmalloc(&n->grad, NPARAMS);
    if (!rc) rc = dmalloc(&n->m1, NPARAMS);
    if (!rc) rc = dmalloc(&n->m2, NPARAMS);
    if (!rc) rc = dmalloc(&n->a1, size_t(MAXPIX / 4 * 16));
    if (!rc) rc = dmalloc(&n->da1, size_t(MAXPIX / 4 * 16));
    if (!rc) rc = dmalloc(&n->a2, size_t(MAXPIX / 16 * 32));
    if (!rc) rc = dmalloc(&n->da2, size_t(MAXPIX / 16 * 32));
    if (!rc) rc = dmalloc(&n->a3, size_t(MAXPIX / 64 * 32));
    if (!rc) rc = dmalloc(&n->da3, size_t(MAXPIX / 64 * 32));
    if (!rc) rc = dmalloc(&n->h, size_t(MAXS * HID));
    if (!rc) rc = dmalloc(&n->dh, size_t(MAXS * HID));
    if (!rc) rc = dmalloc(&n->dl, size_t(MAXS * HEAD_N));
    if (!rc) rc = dmalloc(&n->df, size_t(MAXS * CONVF));
    if (!rc) rc = dmalloc(&n->logits, size_t(MAXS * HEAD_N));
    if (!rc) rc = dmalloc(&n->loss, 1);
    if (!rc) rc = dmalloc(&n->inmv, size_t(MAXS * 6));
    if (!rc) rc = dmalloc(&n->ipairs, size_t(MAXPIX / 256));
    if (!rc) rc = dmalloc(&n->iprop, size_t(MAXPIX / 256));
    if (rc) {
        free_net(n);
        return rc;
    }
    std::vector<float> p;
    init_params(p, seed);
    rc = upload_params(n, p.data());
    if (!rc && cudaMemset(n->m1, 0, sizeof(float) * NPARAMS) != cudaSuccess) rc = fail(H264A_E_CUDA, "mvnet: memset");
    if (!rc && cudaMemset(n->m2, 0, sizeof(float) * NPARAMS) != cudaSuccess) rc = fail(H264A_E_CUDA, "mvnet: memset");
    if (rc) {
        free_net(n);
        return rc;
    }
    *out = n;
    return H264A_OK;
}

extern "C" int h264a_mvnet_destroy(h264a_mvnet* n) {
    if (!n) return H264A_OK;
    cudaSetDevice(n->device);
    cudaDeviceSynchronize();
    free_net(n);
    return H264A_OK;
}

extern "C" int h264a_mvnet_set_params(h264a_mvnet* n, const float* h_params) {
    if (!n || !h_params) return fail(H264A_E_ARG, "mvnet_set_params: null pointer");
    H264A_CUDA(cudaSetDevice(n->device));
    const int rc = upload_params(n, h_params);
    if (rc) return rc;
    H264A_CUDA(cudaMemset(n->m1, 0, sizeof(float) * NPARAMS));
    H264A_CUDA(cudaMemset(n->m2, 0, sizeof(float) * NPARAMS));
    n->step = 0;
    return H264A_OK;
}

extern "C" int h264a_mvnet_get_params(h264a_mvnet* n, float* h_params) {
    if (!n || !h_params) return fail(H264A_E_ARG, "mvnet_get_params: null pointer");
    H264A_CUDA(cudaSetDevice(n->device));
    H264A_CUDA(cudaDeviceSynchronize());
    H264A_CUDA(cudaMemcpy(h_params, n->master, sizeof(float) * NPARAMS, cudaMemcpyDeviceToHost));
    return H264A_OK;
}

extern "C" int h264a_mvnet_forward(h264a_mvnet* n, const h264a_mvnet_pair* d_pairs, int npairs, int cw, int ch,
                                   const int16_t* d_nmv, float* d_logits, void* stream) {
    int rc = check_geo(n, d_pairs, npairs, cw, ch, d_nmv);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const Geo g = make_geo(d_pairs, npairs, cw, ch, d_nmv, nullptr);
    trunk_forward(n, g, st);
    head_forward(n, g, st);
    if (d_logits)
        H264A_CUDA(cudaMemcpyAsync(d_logits, n->logits, sizeof(float) * HEAD_N * npairs * g.nmb,
                                   cudaMemcpyDeviceToDevice, st));
    return check_launch("mvnet forward");
}

extern "C" int h264a_mvnet_grads(h264a_mvnet* n, const h264a_mvnet_pair* d_pairs, int npairs, int cw, int ch,
                                 const int16_t* d_nmv, const int16_t* d_labels, float* d_grads, float* d_loss,
                                 void* stream) {
    int rc = check_geo(n, d_pairs, npairs, cw, ch, d_nmv);
    if (rc) return rc;
    if (!d_labels) return fail(H264A_E_ARG, "mvnet_grads: null labels");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const Geo g = make_geo(d_pairs, npairs, cw, ch, d_nmv, d_labels);
    const int B = npairs * g.nmb;
    H264A_CUDA(cudaMemsetAsync(n->grad, 0, sizeof(float) * NPARAMS, st));
    H264A_CUDA(cudaMemsetAsync(n->loss, 0, sizeof(float), st));
    trunk_forward(n, g, st);
    head_forward(n, g, st);
    loss_kernel<<<(B * 32 + 255) / 256, 256, 0, st>>>(n->logits, d_labels, B, n->dl, n->loss);
    backward(n, g, st);
    if (d_grads) H264A_CUDA(cudaMemcpyAsync(d_grads, n->grad, sizeof(float) * NPARAMS, cudaMemcpyDeviceToDevice, st));
    if (d_loss) H264A_CUDA(cudaMemcpyAsync(d_loss, n->loss, sizeof(float), cudaMemcpyDeviceToDevice, st));
    return check_launch("mvnet grads");
}

extern "C" int h264a_mvnet_train_step(h264a_mvnet* n, const h264a_mvnet_pair* d_pairs, int npairs, int cw, int ch,
                                      const int16_t* d_nmv, const int16_t* d_labels, float lr, float* d_loss,
                                      void* stream) {
    if (!(lr > 0.f)) return fail(H264A_E_ARG, "mvnet_train_step: lr must be positive");
    int rc = h264a_mvnet_grads(n, d_pairs, npairs, cw, ch, d_nmv, d_labels, nullptr, d_loss, stream);
    if (rc) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    n->step++;
    const double b1 = 0.9, b2 = 0.999;
    const float c1 = float(1.0 / (1.0 - std::pow(b1, double(n->step))));
    const float c2 = float(1.0 / (1.0 - std::pow(b2, double(n->step))));
    adam_kernel<<<(NPARAMS + 255) / 256, 256, 0, st>>>(n->master, n->w, n->grad, n->m1, n->m2, NPARAMS, lr, float(b1),
                                                       float(b2), c1, c2, 1e-8f);
    return check_launch("mvnet adam");
}

extern "C" int h264a_mvnet_propose(h264a_mvnet* n, const h264a_mvnet_frame* h_frames, int nframes, void* stream) {
    if (!n || !h_frames) return fail(H264A_E_ARG, "mvnet_propose: null pointer");
    if (nframes < 1) return fail(H264A_E_ARG, "mvnet_propose: need at least one frame");
    for (int i = 0; i < nframes; i++) {
        const h264a_mvnet_frame& f = h_frames[i];
        if (!f.d_cur || !f.d_ref || !f.d_props) return fail(H264A_E_ARG, "mvnet_propose: null frame pointer");
        if (f.cw < 16 || f.ch < 16 || f.cw % 16 || f.ch % 16 || f.cw > 8192 || f.ch > 8192 ||
            (long long)f.cw * f.ch > MAXPIX)
            return fail(H264A_E_ARG, "mvnet_propose: frames must be MB-aligned, at most 8192 pixels a side");
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    // consecutive frames of one geometry, up to MAXPIX pixels, form a batch:
    // their trunk maps in one pass, then FC1 + head over their MBs, then each
    // frame's top-8 into its own d_props
    std::vector<h264a_mvnet_pair> pr;
    std::vector<PropFrame> pf;
    int i = 0;
    while (i < nframes) {
        const int cw = h_frames[i].cw, ch = h_frames[i].ch;
        int j = i;
        pr.clear();
        pf.clear();
        while (j < nframes && h_frames[j].cw == cw && h_frames[j].ch == ch && (long long)(j - i + 1) * cw * ch <= MAXPIX) {
            pr.push_back(h264a_mvnet_pair{h_frames[j].d_cur, h_frames[j].d_ref});
            pf.push_back(PropFrame{h_frames[j].d_guide_mvs, h_frames[j].d_props});
            j++;
        }
        const int P = j - i;
        // the previous batch's kernels read the tables on this stream, so the
        // uploads are stream-ordered after them (pageable sources: the copies
        // are staged before the call returns)
        H264A_CUDA(cudaMemcpyAsync(n->ipairs, pr.data(), sizeof(h264a_mvnet_pair) * P, cudaMemcpyHostToDevice, st));
        H264A_CUDA(cudaMemcpyAsync(n->iprop, pf.data(), sizeof(PropFrame) * P, cudaMemcpyHostToDevice, st));
        const Geo g = make_geo(n->ipairs, P, cw, ch, n->inmv, nullptr);
        const long long samples = (long long)P * g.nmb;
        guide_frames_kernel<<<unsigned((samples + 255) / 256), 256, 0, st>>>(n->iprop, P, g.mb_w, g.mb_h, n->inmv);
        trunk_forward(n, g, st);
        head_forward(n, g, st);
        top8_frames_kernel<<<unsigned((samples * 32 + 255) / 256), 256, 0, st>>>(n->logits, P, g.nmb, n->iprop);
        i = j;
    }
    return check_launch("mvnet propose");
}
