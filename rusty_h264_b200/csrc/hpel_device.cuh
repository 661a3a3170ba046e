// hpel_device.cuh -- the warp body that writes a strip of the edge-padded
// full-pel plane F and the half-pel planes H, V, C (pad_plane_into +
// build_hpel_fused, crates/rusty_h264-common/src/inter.rs:798-991), shared by
// hpel_build_kernel and the closed loop's pipelined kernel, which builds the
// planes of each reconstructed picture band by band.
#pragma once

#include "h264a_device.cuh"

namespace h264a {

constexpr int HP_STRIP = 120;  // output columns per warp (30 lanes x 4)
constexpr int HP_BAND = 48;    // output rows per warp, a multiple of 6
constexpr int HP_WARPS = 4;
constexpr uint32_t HP_BIAS = 0x20102010u;  // 8208 = 256 * 32 + 16 in each half

__device__ __forceinline__ uint32_t max_u16x2(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("max.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t min_u16x2(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// Both halves of a 6-tap sum t biased by 8208: clipped to [8192, 16383] and
// shifted right by 5, the low byte of each half (bits 0-7 and 16-23) is
// clip((t + 16) >> 5); bits above it are discarded by the caller's byte_perm.
__device__ __forceinline__ uint32_t clip5_16x2(uint32_t sb) {
    return min_u16x2(max_u16x2(sb, 0x20002000u), 0x3fff3fffu) >> 5;
}

// biased 6-tap [1,-5,20,20,-5,1] over six 16x2 words
__device__ __forceinline__ uint32_t tap6_16x2(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t e,
                                              uint32_t f) {
    return (a + f + HP_BIAS) + 20u * (c + d) - 5u * (b + e);
}

// (biased C sum) >> 10 of one column from six vt values biased by 8208: the
// result plus 256 (8208 * 32 = 256 * 1024 + 512, the rounding term)
__device__ __forceinline__ uint32_t centre_q(int a, int b, int c, int d, int e, int f) {
    return uint32_t((a + f + 20 * (c + d) - 5 * (b + e)) >> 10);
}

struct HpelRow {
    uint32_t raw, ev, od;  // the source word, its even and odd bytes as 16x2
};

// Rows [y0, y1) of strip `strip` (plane columns strip * HP_STRIP ..) of the
// four planes F of picture Y, one warp: see the file comment of hpel.cu.
// Only the 4-byte words whose plane column lies in [xlo, xhi) are written
// (xlo, xhi multiples of 4): a strip shared by two column segments is
// written by each for its own columns.
// CG: read the picture through L2 rather than the read-only path (a picture
// written during the launch, whose rows below the strip's may still change:
// the look-ahead loads past y1 must not leave stale lines in L1).
template <bool CG = false>
__device__ __forceinline__ void hpel_strip_rows(const uint8_t* __restrict__ Y, int cw, int ch, int pad,
                                                uint8_t* __restrict__ F, int pw, int ph, int strip, int y0, int y1,
                                                int word_in, int word_out, int xlo = 0, int xhi = 1 << 30) {
    const int lane = threadIdx.x & 31;
    const long long ps = (long long)pw * ph;
    const int X = strip * HP_STRIP + 4 * (lane - 1);  // plane column of the lane's word
    const int sx = X - pad;                           // its first picture column
    const bool inner = word_in && sx >= 0 && sx + 3 <= cw - 1;
    const int c0 = clampi(sx, 0, cw - 1), c1 = clampi(sx + 1, 0, cw - 1), c2 = clampi(sx + 2, 0, cw - 1),
              c3 = clampi(sx + 3, 0, cw - 1);
    auto ldraw = [&](int yp) {
        const uint8_t* row = Y + (long long)clampi(yp - pad, 0, ch - 1) * cw;
        return inner ? ldw(reinterpret_cast<const uint32_t*>(row + sx), CG)
                     : uint32_t(ldb(row + c0, CG)) | uint32_t(ldb(row + c1, CG)) << 8 |
                           uint32_t(ldb(row + c2, CG)) << 16 | uint32_t(ldb(row + c3, CG)) << 24;
    };
    auto mk = [](uint32_t raw) {
        HpelRow r;
        r.raw = raw;
        r.ev = __byte_perm(raw, 0u, 0x4240);
        r.od = __byte_perm(raw, 0u, 0x4341);
        return r;
    };
    auto load = [&](int yp) { return mk(ldraw(yp)); };
    const bool owner = lane >= 1 && lane <= 30 && X < pw && X >= xlo && X < xhi;
    // the four planes' words of row y from the rows y-2 .. y+3
    auto emit = [&](int y, const HpelRow& a, const HpelRow& b, const HpelRow& c, const HpelRow& d, const HpelRow& e,
                    const HpelRow& f) {
        const uint32_t vte = tap6_16x2(a.ev, b.ev, c.ev, d.ev, e.ev, f.ev);
        const uint32_t vto = tap6_16x2(a.od, b.od, c.od, d.od, e.od, f.od);
        const uint32_t vw = __byte_perm(clip5_16x2(vte), clip5_16x2(vto), 0x6240);
        // H: the centre row's bytes x-2 .. x+6 as pairs of columns two apart
        const uint32_t wl = __shfl_up_sync(0xffffffffu, c.raw, 1), wr = __shfl_down_sync(0xffffffffu, c.raw, 1);
        const uint32_t el = __byte_perm(wl, 0u, 0x4240), ol = __byte_perm(wl, 0u, 0x4341);
        const uint32_t er = __byte_perm(wr, 0u, 0x4240), orr = __byte_perm(wr, 0u, 0x4341);
        const uint32_t q0 = __funnelshift_r(el, c.ev, 16), q1 = __funnelshift_r(ol, c.od, 16);
        const uint32_t q4 = __funnelshift_r(c.ev, er, 16), q5 = __funnelshift_r(c.od, orr, 16);
        const uint32_t he = tap6_16x2(q0, q1, c.ev, c.od, q4, q5);
        const uint32_t ho = tap6_16x2(q1, c.ev, c.od, q4, q5, er);
        const uint32_t hw = __byte_perm(clip5_16x2(he), clip5_16x2(ho), 0x6240);
        // C: vt of columns x-2, x-1 (left lane) and x+4 .. x+6 (right lane)
        const uint32_t lw = __shfl_up_sync(0xffffffffu, __byte_perm(vte, vto, 0x7632), 1);
        const uint32_t rw = __shfl_down_sync(0xffffffffu, __byte_perm(vte, vto, 0x5410), 1);
        const uint32_t re = __shfl_down_sync(0xffffffffu, vte, 1);
        const int v_2 = int(lw & 0xffffu), v_1 = int(lw >> 16);
        const int v0 = int(vte & 0xffffu), v1 = int(vto & 0xffffu), v2 = int(vte >> 16), v3 = int(vto >> 16);
        const int v4 = int(rw & 0xffffu), v5 = int(rw >> 16), v6 = int(re >> 16);
        // columns x, x+2 and x+1, x+3 as 16x2 pairs (each below 800), clipped
        // to [256, 511]: the low bytes are the four C samples
        const uint32_t ce = __byte_perm(centre_q(v_2, v_1, v0, v1, v2, v3), centre_q(v0, v1, v2, v3, v4, v5), 0x5410);
        const uint32_t co = __byte_perm(centre_q(v_1, v0, v1, v2, v3, v4), centre_q(v1, v2, v3, v4, v5, v6), 0x5410);
        const uint32_t cwd = __byte_perm(min_u16x2(max_u16x2(ce, 0x01000100u), 0x01ff01ffu),
                                         min_u16x2(max_u16x2(co, 0x01000100u), 0x01ff01ffu), 0x6240);
        if (!owner) return;
        const long long off = (long long)y * pw + X;
        if (word_out) {
            *reinterpret_cast<uint32_t*>(F + off) = c.raw;
            *reinterpret_cast<uint32_t*>(F + ps + off) = hw;
            *reinterpret_cast<uint32_t*>(F + 2 * ps + off) = vw;
            *reinterpret_cast<uint32_t*>(F + 3 * ps + off) = cwd;
        } else {
            const int nb = pw - X < 4 ? pw - X : 4;
            for (int i = 0; i < nb; i++) {
                F[off + i] = uint8_t(c.raw >> (8 * i));
                F[ps + off + i] = uint8_t(hw >> (8 * i));
                F[2 * ps + off + i] = uint8_t(vw >> (8 * i));
                F[3 * ps + off + i] = uint8_t(cwd >> (8 * i));
            }
        }
    };
    HpelRow r0 = load(y0 - 2), r1 = load(y0 - 1), r2 = load(y0), r3 = load(y0 + 1), r4 = load(y0 + 2), r5;
    // six rows per iteration, the window rotating through r0..r5 by name
    for (int y = y0; y < y1; y += 6) {
        // the iteration's six rows in flight at once (rows past the band are
        // clamped reads, discarded)
        const uint32_t n0 = ldraw(y + 3), n1 = ldraw(y + 4), n2 = ldraw(y + 5), n3 = ldraw(y + 6), n4 = ldraw(y + 7),
                       n5 = ldraw(y + 8);
        r5 = mk(n0);
        emit(y, r0, r1, r2, r3, r4, r5);
        if (y + 1 >= y1) break;
        r0 = mk(n1);
        emit(y + 1, r1, r2, r3, r4, r5, r0);
        if (y + 2 >= y1) break;
        r1 = mk(n2);
        emit(y + 2, r2, r3, r4, r5, r0, r1);
        if (y + 3 >= y1) break;
        r2 = mk(n3);
        emit(y + 3, r3, r4, r5, r0, r1, r2);
        if (y + 4 >= y1) break;
        r3 = mk(n4);
        emit(y + 4, r4, r5, r0, r1, r2, r3);
        if (y + 5 >= y1) break;
        r4 = mk(n5);
        emit(y + 5, r5, r0, r1, r2, r3, r4);
    }
}

}  // namespace h264a
