// h264a_device.cuh -- device building blocks shared by the sm_100a kernels.
//
// All codec arithmetic is integer and bit-exact with the reference
// (Remade-With-Rust/rusty_h264); each helper names the reference function
// whose value it reproduces.
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "h264accel_internal.h"

namespace h264a {

// ---------------------------------------------------------------------------
// Byte access
// ---------------------------------------------------------------------------

// Four consecutive bytes at any alignment, little-endian, from read-only global
// memory: two aligned 32-bit loads and a funnel shift.  Reads stay inside the
// 4-byte words that hold p[0..3].
__device__ __forceinline__ uint32_t ld4u(const uint8_t* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    const uint32_t sh = uint32_t(a & 3) * 8u;
    const uint32_t lo = __ldg(w);
    if (sh == 0) return lo;
    const uint32_t hi = __ldg(w + 1);
    return __funnelshift_r(lo, hi, sh);
}

// ld4u through L2 (buffers written during the launch).
__device__ __forceinline__ uint32_t ld4u_cg(const uint8_t* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    const uint32_t sh = uint32_t(a & 3) * 8u;
    const uint32_t lo = __ldcg(w);
    if (sh == 0) return lo;
    const uint32_t hi = __ldcg(w + 1);
    return __funnelshift_r(lo, hi, sh);
}

// Branch-free form of ld4u for reads whose following aligned word is known to
// lie inside the buffer (plane reads inside the padded window).
__device__ __forceinline__ uint32_t ld4u_nb(const uint8_t* p) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
    return __funnelshift_r(__ldg(w), __ldg(w + 1), uint32_t(a & 3) * 8u);
}

__device__ __forceinline__ int byte_of(uint32_t w, int k) { return int((w >> (8 * k)) & 0xffu); }

// 32-bit load from a shared-memory address (the 32-bit shared window).
__device__ __forceinline__ uint32_t lds_u32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr));
    return v;
}


__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---------------------------------------------------------------------------
// 4x4 Hadamard SATD
// ---------------------------------------------------------------------------

// Σ|H·(s−p)·Hᵀ| of one 4x4 block given as four packed rows: the unrounded
// value of satd_4x4_sum (transform.rs:701); the openh264 per-block SATD
// (satd_sad.rs:39) is (this + 1) >> 1.  Butterfly order as satd4x4_scalar.
__device__ __forceinline__ int satd4x4_rows(const uint32_t s[4], const uint32_t p[4]) {
    int m[4][4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int d0 = byte_of(s[r], 0) - byte_of(p[r], 0);
        const int d1 = byte_of(s[r], 1) - byte_of(p[r], 1);
        const int d2 = byte_of(s[r], 2) - byte_of(p[r], 2);
        const int d3 = byte_of(s[r], 3) - byte_of(p[r], 3);
        const int s0 = d0 + d2, s1 = d1 + d3, s2 = d0 - d2, s3 = d1 - d3;
        m[r][0] = s0 + s1; m[r][1] = s2 + s3; m[r][2] = s2 - s3; m[r][3] = s0 - s1;
    }
    int sum = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int s0 = m[0][j] + m[2][j], s1 = m[1][j] + m[3][j];
        const int s2 = m[0][j] - m[2][j], s3 = m[1][j] - m[3][j];
        sum += abs(s0 + s1) + abs(s2 + s3) + abs(s2 - s3) + abs(s0 - s1);
    }
    return sum;
}

// Per-byte (a+b+1)>>1 (what pavgb and the reference's avg_rows compute):
// (a|b) − ((a^b)>>1) per byte, which never borrows across bytes.
__device__ __forceinline__ uint32_t avg_up4(uint32_t a, uint32_t b) {
    return (a | b) - (((a ^ b) >> 1) & 0x7f7f7f7fu);
}

// Source rows of a 4x4 block split into column pairs (c0|c2) and (c1|c3) in
// 16-bit halves, the operand form of satd4x4_packed.
__device__ __forceinline__ void split_pairs(const uint32_t s[4], uint32_t a[4], uint32_t b[4]) {
#pragma unroll
    for (int r = 0; r < 4; r++) {
        a[r] = __byte_perm(s[r], 0u, 0x4240);
        b[r] = __byte_perm(s[r], 0u, 0x4341);
    }
}

// Low 16 bits, sign-extended (the low half of a packed pair).
__device__ __forceinline__ int sext16(int v) { return int(int16_t(uint16_t(uint32_t(v) & 0xffffu))); }

// Σ|H·(s−p)·Hᵀ| of a 4x4 block with the source pre-split (split_pairs): the
// same value as satd4x4_rows.  Each 32-bit register carries two columns as
// hi·2^16 + lo; the butterflies are linear, so plain 32-bit adds keep both
// halves exact (|half| <= 2040 here).  The last butterfly of every row is
// folded into |x+y| + |x−y| = 2·max(|x|,|y|).
__device__ __forceinline__ int satd4x4_packed(const uint32_t sa[4], const uint32_t sb[4], const uint32_t p[4]) {
    int A[4], B[4];
#pragma unroll
    for (int r = 0; r < 4; r++) {
        A[r] = int(sa[r]) - int(__byte_perm(p[r], 0u, 0x4240));
        B[r] = int(sb[r]) - int(__byte_perm(p[r], 0u, 0x4341));
    }
    {
        const int t0 = A[0] + A[1], t1 = A[0] - A[1], t2 = A[2] + A[3], t3 = A[2] - A[3];
        A[0] = t0 + t2; A[1] = t1 + t3; A[2] = t0 - t2; A[3] = t1 - t3;
        const int u0 = B[0] + B[1], u1 = B[0] - B[1], u2 = B[2] + B[3], u3 = B[2] - B[3];
        B[0] = u0 + u2; B[1] = u1 + u3; B[2] = u0 - u2; B[3] = u1 - u3;
    }
    int sum = 0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int pp = A[r] + B[r], qq = A[r] - B[r];
        const int pl = sext16(pp), ph = (pp - pl) >> 16;
        const int ql = sext16(qq), qh = (qq - ql) >> 16;
        sum += max(abs(pl), abs(ph)) + max(abs(ql), abs(qh));
    }
    return 2 * sum;
}

// Σ|s−p| of one 4x4 block (sad_scalar, satd_sad.rs:74).
__device__ __forceinline__ int sad4x4_rows(const uint32_t s[4], const uint32_t p[4]) {
    return int(__vsadu4(s[0], p[0]) + __vsadu4(s[1], p[1]) + __vsadu4(s[2], p[2]) + __vsadu4(s[3], p[3]));
}

// ---------------------------------------------------------------------------
// Quarter-pel prediction from the cached planes
// ---------------------------------------------------------------------------

// Plane set of one reference picture: F|H|V|C, each pw×ph, stride pw, the
// layout HpelPlanes holds (inter.rs:707).
struct Planes {
    const uint8_t* base;  // F at base, H at +ps, V at +2ps, C at +3ps
    int pw, ph, pad;
    long long ps;
    // read through L2 rather than the read-only path: the planes are written
    // during the launch that reads them (the pipelined closed loop)
    bool cg = false;
    __device__ __forceinline__ const uint8_t* plane(int i) const { return base + ps * i; }
};

// A word or byte of a buffer through the read-only path, or through L2 for
// buffers written during the launch.
__device__ __forceinline__ uint32_t ldw(const uint32_t* p, bool cg) { return cg ? __ldcg(p) : __ldg(p); }
__device__ __forceinline__ int ldb(const uint8_t* p, bool cg) { return cg ? __ldcg(p) : __ldg(p); }

// Operand table of the quarter phases (inter.rs:1086-1099, mectx.rs:143-156):
// plane a at (+dxa,+dya), plane b at (+dxb,+dyb); planes 0=F 1=H 2=V 3=C.
// Half/full phases use one plane (inter.rs:1024-1035).
struct PhaseOps { int8_t pa, dxa, dya, pb, dxb, dyb; };

__device__ __forceinline__ PhaseOps phase_ops(int fx, int fy) {
    switch (fx * 4 + fy) {
        case 0 * 4 + 0: return {0, 0, 0, -1, 0, 0};
        case 2 * 4 + 0: return {1, 0, 0, -1, 0, 0};
        case 0 * 4 + 2: return {2, 0, 0, -1, 0, 0};
        case 2 * 4 + 2: return {3, 0, 0, -1, 0, 0};
        case 1 * 4 + 0: return {0, 0, 0, 1, 0, 0};
        case 3 * 4 + 0: return {0, 1, 0, 1, 0, 0};
        case 0 * 4 + 1: return {0, 0, 0, 2, 0, 0};
        case 0 * 4 + 3: return {0, 0, 1, 2, 0, 0};
        case 1 * 4 + 1: return {1, 0, 0, 2, 0, 0};
        case 3 * 4 + 1: return {1, 0, 0, 2, 1, 0};
        case 1 * 4 + 3: return {1, 0, 1, 2, 0, 0};
        case 3 * 4 + 3: return {1, 0, 1, 2, 1, 0};
        case 2 * 4 + 1: return {1, 0, 0, 3, 0, 0};
        case 2 * 4 + 3: return {1, 0, 1, 3, 0, 0};
        case 1 * 4 + 2: return {2, 0, 0, 3, 0, 0};
        default:        return {2, 1, 0, 3, 0, 0};  // (3,2)
    }
}

// The same table packed into two 64-bit words, one byte per phase fx*4+fy:
// bits 0-1 plane a, bits 2-3 plane b (0 = single plane; b is never F),
// bit 4 dx_a, bit 5 dy_a, bit 6 dx_b, bit 7 dy_b.  A byte extract replaces the
// divergent switch when the lanes of a warp hold different phases.
__host__ __device__ constexpr uint32_t phase_byte(int pa, int pb, int dxa, int dya, int dxb, int dyb) {
    return uint32_t(pa | (pb << 2) | (dxa << 4) | (dya << 5) | (dxb << 6) | (dyb << 7));
}
constexpr unsigned long long kPhaseLo =
    (unsigned long long)phase_byte(0, 0, 0, 0, 0, 0) | ((unsigned long long)phase_byte(0, 2, 0, 0, 0, 0) << 8) |
    ((unsigned long long)phase_byte(2, 0, 0, 0, 0, 0) << 16) | ((unsigned long long)phase_byte(0, 2, 0, 1, 0, 0) << 24) |
    ((unsigned long long)phase_byte(0, 1, 0, 0, 0, 0) << 32) | ((unsigned long long)phase_byte(1, 2, 0, 0, 0, 0) << 40) |
    ((unsigned long long)phase_byte(2, 3, 0, 0, 0, 0) << 48) | ((unsigned long long)phase_byte(1, 2, 0, 1, 0, 0) << 56);
constexpr unsigned long long kPhaseHi =
    (unsigned long long)phase_byte(1, 0, 0, 0, 0, 0) | ((unsigned long long)phase_byte(1, 3, 0, 0, 0, 0) << 8) |
    ((unsigned long long)phase_byte(3, 0, 0, 0, 0, 0) << 16) | ((unsigned long long)phase_byte(1, 3, 0, 1, 0, 0) << 24) |
    ((unsigned long long)phase_byte(0, 1, 1, 0, 0, 0) << 32) | ((unsigned long long)phase_byte(1, 2, 0, 0, 1, 0) << 40) |
    ((unsigned long long)phase_byte(2, 3, 1, 0, 0, 0) << 48) | ((unsigned long long)phase_byte(1, 2, 0, 1, 1, 0) << 56);

__device__ __forceinline__ uint32_t phase_bits(int fx, int fy) {
    const int idx = fx * 4 + fy;
    const unsigned long long w = idx < 8 ? kPhaseLo : kPhaseHi;
    return uint32_t(w >> ((idx & 7) * 8)) & 0xffu;
}

// The four packed prediction rows of the 4x4 block whose top-left full-pel
// sample is (ix, iy) in picture coordinates, at phase (fx, fy).  Equal to
// mc_luma (inter.rs:1193) for every position: inside the padded planes the rows
// are plane reads (and the (a+b+1)>>1 average, computed per byte by
// avg_up4); outside, every operand coordinate is clamped to the plane, which
// reproduces mc_luma's per-tap clamping because the planes are built from the
// edge-replicated picture with a pad of at least 3.
__device__ __forceinline__ void pred_rows(const Planes& P, int ix, int iy, int fx, int fy, uint32_t out[4]) {
    const int px = ix + P.pad, py = iy + P.pad;
    // inside: both aligned words ld4u_nb touches for an operand starting at
    // px+dx (dx <= 1) end by px+8, so they stay in the operand's row
    const bool inside = px >= 0 && py >= 0 && px + 9 <= P.pw && py + 5 <= P.ph;
    if (inside) {
        const uint32_t pb = phase_bits(fx, fy);
        const int pa = int(pb & 3), pbb = int((pb >> 2) & 3);
        const uint8_t* a = P.base + P.ps * pa + (long long)(py + int((pb >> 5) & 1)) * P.pw + px + int((pb >> 4) & 1);
        auto rd4 = [&](const uint8_t* q) {
            const uintptr_t ad = reinterpret_cast<uintptr_t>(q);
            const uint32_t* w = reinterpret_cast<const uint32_t*>(ad & ~uintptr_t(3));
            return __funnelshift_r(ldw(w, P.cg), ldw(w + 1, P.cg), uint32_t(ad & 3) * 8u);
        };
        if (pbb == 0) {
#pragma unroll
            for (int r = 0; r < 4; r++) out[r] = rd4(a + (long long)r * P.pw);
        } else {
            const uint8_t* b =
                P.base + P.ps * pbb + (long long)(py + int((pb >> 7) & 1)) * P.pw + px + int((pb >> 6) & 1);
#pragma unroll
            for (int r = 0; r < 4; r++) out[r] = avg_up4(rd4(a + (long long)r * P.pw), rd4(b + (long long)r * P.pw));
        }
        return;
    }
    const PhaseOps op = phase_ops(fx, fy);
    const uint8_t* A = P.plane(op.pa);
    const uint8_t* B = P.plane(op.pb < 0 ? op.pa : op.pb);
#pragma unroll
    for (int r = 0; r < 4; r++) {
        uint32_t w = 0;
        const int ya = clampi(py + r + op.dya, 0, P.ph - 1);
        const int yb = clampi(py + r + op.dyb, 0, P.ph - 1);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            int v = ldb(A + (long long)ya * P.pw + clampi(px + c + op.dxa, 0, P.pw - 1), P.cg);
            if (op.pb >= 0) {
                const int u = ldb(B + (long long)yb * P.pw + clampi(px + c + op.dxb, 0, P.pw - 1), P.cg);
                v = (v + u + 1) >> 1;
            }
            w |= uint32_t(v) << (8 * c);
        }
        out[r] = w;
    }
}

// Packed rows of a full-pel 4x4 block read from a plain picture with clamped
// coordinates (mc_luma's full-pel arm, inter.rs:1213-1243).
__device__ __forceinline__ void fullpel_rows_clamped(const uint8_t* pic, int w, int h, int x, int y, uint32_t out[4]) {
    if (x >= 0 && y >= 0 && x + 4 <= w && y + 4 <= h) {
#pragma unroll
        for (int r = 0; r < 4; r++) out[r] = ld4u(pic + (long long)(y + r) * w + x);
        return;
    }
#pragma unroll
    for (int r = 0; r < 4; r++) {
        const int yy = clampi(y + r, 0, h - 1);
        uint32_t v = 0;
#pragma unroll
        for (int c = 0; c < 4; c++) v |= uint32_t(__ldg(pic + (long long)yy * w + clampi(x + c, 0, w - 1))) << (8 * c);
        out[r] = v;
    }
}

// Quarter-pel prediction rows of a 4x4 block straight from a plain picture
// (no cached planes), every tap clamped: luma_sample (inter.rs:134-176), the
// value mc_luma returns.  Used where the reference interpolates a picture it
// keeps no planes for (the lookahead's sub-pel seed probes).
__device__ __forceinline__ int pic_at(const uint8_t* pic, int w, int h, int x, int y) {
    return __ldg(pic + (long long)clampi(y, 0, h - 1) * w + clampi(x, 0, w - 1));
}
__device__ __forceinline__ int clip255d(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }
// value of plane `pl` (0 full-pel, 1 horizontal half, 2 vertical half, 3 centre) at (x, y)
__device__ __forceinline__ int half_sample(const uint8_t* pic, int w, int h, int pl, int x, int y) {
    if (pl == 0) return pic_at(pic, w, h, x, y);
    if (pl == 1) {
        const int s = pic_at(pic, w, h, x - 2, y) - 5 * pic_at(pic, w, h, x - 1, y) + 20 * pic_at(pic, w, h, x, y) +
                      20 * pic_at(pic, w, h, x + 1, y) - 5 * pic_at(pic, w, h, x + 2, y) + pic_at(pic, w, h, x + 3, y);
        return clip255d((s + 16) >> 5);
    }
    if (pl == 2) {
        const int s = pic_at(pic, w, h, x, y - 2) - 5 * pic_at(pic, w, h, x, y - 1) + 20 * pic_at(pic, w, h, x, y) +
                      20 * pic_at(pic, w, h, x, y + 1) - 5 * pic_at(pic, w, h, x, y + 2) + pic_at(pic, w, h, x, y + 3);
        return clip255d((s + 16) >> 5);
    }
    const int tap[6] = {1, -5, 20, 20, -5, 1};
    int acc = 0;
#pragma unroll
    for (int k = 0; k < 6; k++) {
        int v = 0;
#pragma unroll
        for (int j = 0; j < 6; j++) v += tap[j] * pic_at(pic, w, h, x - 2 + k, y - 2 + j);
        acc += tap[k] * v;
    }
    return clip255d((acc + 512) >> 10);
}
__device__ __noinline__ static void subpel_rows_clamped(const uint8_t* pic, int w, int h, int x, int y, int fx, int fy, uint32_t out[4]) {
    const PhaseOps op = phase_ops(fx, fy);
    for (int r = 0; r < 4; r++) {
        uint32_t wd = 0;
        for (int c = 0; c < 4; c++) {
            int v = half_sample(pic, w, h, op.pa, x + c + op.dxa, y + r + op.dya);
            if (op.pb >= 0) v = (v + half_sample(pic, w, h, op.pb, x + c + op.dxb, y + r + op.dyb) + 1) >> 1;
            wd |= uint32_t(v) << (8 * c);
        }
        out[r] = wd;
    }
}

// ---------------------------------------------------------------------------
// Rate model and λ pricing (mb16.rs:2454-2482, 2540-2578)
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t mvbits(int kind, const uint16_t* tab, int d) {
    if (kind == 1 || kind == 2) {
        unsigned a = unsigned(d < 0 ? -d : d);
        if (a > 4095u) a = 4095u;
        return __ldg(tab + a);
    }
    const uint32_t codenum = d > 0 ? uint32_t(2 * d - 1) : uint32_t(-2 * d);
    return 1u + 2u * (31u - uint32_t(__clz(int(codenum + 1u))));
}

// (λ·rate as f64) as i64: one IEEE double multiply rounded to nearest, then
// truncation toward zero, the same two steps the reference performs.
__device__ __forceinline__ long long lam_cost(double lam, uint32_t rate) {
    return __double2ll_rz(__dmul_rn(lam, double(rate)));
}

// ---------------------------------------------------------------------------
// Wavefront queues of the persistent kernels
// ---------------------------------------------------------------------------
// An MB that depends on its left and top-right neighbours (motion-vector
// prediction, in-loop deblocking) is dealt in anti-diagonal order t = x + 2y:
// both neighbours lie on earlier diagonals.  Readiness is a per-MB flag set to
// the launch's epoch with release semantics and polled with acquire loads.

constexpr int SPIN_LIMIT = 1000 * 1000;  // ~0.5 s of polling (a 200 ns sleep per poll)

// Number of MBs (x, y) of a W x H frame with x + 2y < t: rows y < a are
// full (t - 2y >= W), rows a <= y < b hold t - 2y MBs.
__device__ __forceinline__ int wave_prefix(int W, int H, int t) {
    const int a = t >= W ? min((t - W) / 2 + 1, H) : 0;
    const int b = t >= 1 ? min((t - 1) / 2 + 1, H) : 0;
    return a * W + (b - a) * t - (b - a) * (a + b - 1);
}

// The k-th MB of a W x H frame in wavefront order.
__device__ __forceinline__ void wave_mb(int W, int H, int k, int& x, int& y) {
    int lo = 0, hi = (W - 1) + 2 * (H - 1);  // find the diagonal t with prefix(t) <= k < prefix(t+1)
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (wave_prefix(W, H, mid) <= k) lo = mid; else hi = mid - 1;
    }
    const int t = lo;
    const int ylo = t - (W - 1) > 0 ? (t - (W - 1) + 1) >> 1 : 0;
    y = ylo + (k - wave_prefix(W, H, t));
    x = t - 2 * y;
}

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// Fetch-and-add at GPU scope with acquire and release semantics.
__device__ __forceinline__ int atom_add_acq_rel(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
// Release store at system scope (a word the host polls in mapped memory).
__device__ __forceinline__ void st_release_sys(int* p, int v) {
    asm volatile("st.release.sys.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// Release store at GPU scope: the thread's earlier stores, and those of the
// lanes that a __syncwarp ordered before it, are visible to any thread whose
// ld_acquire reads the value (a release fence and a store in one; no separate
// __threadfence is needed).
__device__ __forceinline__ void st_release(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits (bounded) until flag == epoch; on timeout records `code` in status.
// Once any wait of the launch has timed out (status non-zero, checked every
// 256 polls) the others give up too, so a failed launch ends promptly.
static __device__ void wait_flag(const int* flag, int epoch, int* status, int code, int limit) {
    for (int it = 0;; it++) {
        if (ld_acquire(flag) == epoch) return;
        if (it >= limit || ((it & 255) == 255 && *reinterpret_cast<volatile int*>(status) != 0)) {
            atomicCAS(status, 0, code);
            return;
        }
        __nanosleep(200);
    }
}

// ---------------------------------------------------------------------------
// Warp helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ int warp_seg_sum(int v, int seg) {
    // sum over aligned groups of `seg` lanes (seg a power of two <= 32)
    for (int o = seg >> 1; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// Bulk copies into shared memory (ME reference windows, lookahead windows)
// ---------------------------------------------------------------------------

// mbarrier and bulk-copy primitives (shared addresses are 32-bit).
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// One tiled TMA copy of the box at (x, y, z) of `map` into shared memory,
// completing on `bar` (no multicast).  x * 1 byte must be a multiple of 16.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int x, int y, int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
            dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

// Waits (bounded) for the phase `parity` of the warp's window barrier; on
// timeout records `code` in status and keeps waiting (again bounded) so that
// no copy is left in flight into the window.
__device__ __forceinline__ void wait_window(uint32_t bar, uint32_t parity, int* status, int code, int limit) {
    for (int it = 0; !mbar_try_wait(bar, parity); it++) {
        if (it == limit) atomicCAS(status, 0, code);
        if (it >= 2 * limit) break;
    }
}

}  // namespace h264a
