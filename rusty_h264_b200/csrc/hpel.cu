// hpel.cu -- a1/a2: edge-padded full-pel plane F and the half-pel planes
// H, V, C of reference pictures (pad_plane_into + build_hpel_fused,
// crates/rusty_h264-common/src/inter.rs:798-991; AVX2 twin
// crates/rusty_h264-accel/src/hpel.rs:34-203).
//
// One warp writes a strip of HP_STRIP columns and HP_BAND rows of all four
// planes.  Lanes 1..30 own one 4-byte word of a row each; lanes 0 and 31 hold
// the words either side of the strip, so that the 6-tap filters read their
// neighbours' samples with shuffles.  Each lane keeps the six source rows its
// filters span in registers and slides them down the strip: one 4-byte load
// per row, no shared memory.  Sample columns and rows are clamped to the
// picture, which is exactly the replication pad_plane performs.
//
// Arithmetic on pairs of 16-bit columns (even bytes 0/2, odd bytes 1/3 of a
// word): the vertical intermediate vt and the horizontal sum of H, biased by
// 2560 = 80 * 32 so that no half goes negative (|taps| <= 2550 <= 2560), stay
// below 13,270 per half; (s + 16) >> 5 of the biased sum is the result plus
// 80 and is clipped with 16x2 min/max.  C sums six biased vt values per
// column in 32 bits (the bias adds 2560 * 32 = 80 * 1024).
// HBM traffic is one read of the picture (the band halo mostly from L2) and
// one write of the four planes.
#include "h264a_device.cuh"

namespace h264a {

constexpr int HP_STRIP = 120;  // output columns per warp (30 lanes x 4)
constexpr int HP_BAND = 48;    // output rows per warp, a multiple of 6
constexpr int HP_WARPS = 4;
constexpr uint32_t HP_BIAS = 0x0A000A00u;  // 2560 in each half

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

// clip((s + 16) >> 5) of both halves of a biased 6-tap sum (halves < 13,271)
__device__ __forceinline__ uint32_t round5_clip(uint32_t sb) {
    const uint32_t q = ((sb + 0x00100010u) >> 5) & 0x07ff07ffu;  // per half: result + 80
    return min_u16x2(max_u16x2(q, 0x00500050u), 0x014f014fu) - 0x00500050u;
}

// biased 6-tap [1,-5,20,20,-5,1] over six 16x2 words
__device__ __forceinline__ uint32_t tap6_16x2(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t e,
                                              uint32_t f) {
    return (a + f + HP_BIAS) + 20u * (c + d) - 5u * (b + e);
}

// C of one column from six biased vt values
__device__ __forceinline__ uint32_t centre_px(int a, int b, int c, int d, int e, int f) {
    const int s = a + f - 81408 + 20 * (c + d) - 5 * (b + e);  // 81408 = 80 * 1024 - 512
    return uint32_t(clampi(s >> 10, 0, 255));
}

struct HpelRow {
    uint32_t raw, ev, od;  // the source word, its even and odd bytes as 16x2
};

__global__ void __launch_bounds__(32 * HP_WARPS) hpel_build_kernel(const uint8_t* __restrict__ ref, int cw, int ch,
                                                                   int pad, size_t ref_fstride,
                                                                   uint8_t* __restrict__ planes, int pw, int ph,
                                                                   int strips, int bands, long long nwarps,
                                                                   int word_in, int word_out) {
    const long long wid = (long long)blockIdx.x * HP_WARPS + (threadIdx.x >> 5);
    if (wid >= nwarps) return;  // warp-uniform
    const int lane = threadIdx.x & 31;
    const long long per_pic = (long long)strips * bands;
    const int pic = int(wid / per_pic);
    const int rem = int(wid - per_pic * pic);
    const int band = rem / strips, strip = rem - band * strips;
    const uint8_t* Y = ref + ref_fstride * pic;
    const long long ps = (long long)pw * ph;
    uint8_t* F = planes + 4 * ps * pic;
    const int X = strip * HP_STRIP + 4 * (lane - 1);  // plane column of the lane's word
    const int sx = X - pad;                           // its first picture column
    const bool inner = word_in && sx >= 0 && sx + 3 <= cw - 1;
    const int c0 = clampi(sx, 0, cw - 1), c1 = clampi(sx + 1, 0, cw - 1), c2 = clampi(sx + 2, 0, cw - 1),
              c3 = clampi(sx + 3, 0, cw - 1);
    auto load = [&](int yp) {
        const uint8_t* row = Y + (long long)clampi(yp - pad, 0, ch - 1) * cw;
        HpelRow r;
        r.raw = inner ? __ldg(reinterpret_cast<const uint32_t*>(row + sx))
                      : uint32_t(__ldg(row + c0)) | uint32_t(__ldg(row + c1)) << 8 | uint32_t(__ldg(row + c2)) << 16 |
                            uint32_t(__ldg(row + c3)) << 24;
        r.ev = __byte_perm(r.raw, 0u, 0x4240);
        r.od = __byte_perm(r.raw, 0u, 0x4341);
        return r;
    };
    const bool owner = lane >= 1 && lane <= 30 && X < pw;
    // the four planes' words of row y from the rows y-2 .. y+3
    auto emit = [&](int y, const HpelRow& a, const HpelRow& b, const HpelRow& c, const HpelRow& d, const HpelRow& e,
                    const HpelRow& f) {
        const uint32_t vte = tap6_16x2(a.ev, b.ev, c.ev, d.ev, e.ev, f.ev);
        const uint32_t vto = tap6_16x2(a.od, b.od, c.od, d.od, e.od, f.od);
        const uint32_t vw = round5_clip(vte) | (round5_clip(vto) << 8);
        // H: the centre row's bytes x-2 .. x+6 as pairs of columns two apart
        const uint32_t wl = __shfl_up_sync(0xffffffffu, c.raw, 1), wr = __shfl_down_sync(0xffffffffu, c.raw, 1);
        const uint32_t el = __byte_perm(wl, 0u, 0x4240), ol = __byte_perm(wl, 0u, 0x4341);
        const uint32_t er = __byte_perm(wr, 0u, 0x4240), orr = __byte_perm(wr, 0u, 0x4341);
        const uint32_t q0 = __funnelshift_r(el, c.ev, 16), q1 = __funnelshift_r(ol, c.od, 16);
        const uint32_t q4 = __funnelshift_r(c.ev, er, 16), q5 = __funnelshift_r(c.od, orr, 16);
        const uint32_t he = tap6_16x2(q0, q1, c.ev, c.od, q4, q5);
        const uint32_t ho = tap6_16x2(q1, c.ev, c.od, q4, q5, er);
        const uint32_t hw = round5_clip(he) | (round5_clip(ho) << 8);
        // C: vt of columns x-2, x-1 (left lane) and x+4 .. x+6 (right lane)
        const uint32_t lw = __shfl_up_sync(0xffffffffu, __byte_perm(vte, vto, 0x7632), 1);
        const uint32_t rw = __shfl_down_sync(0xffffffffu, __byte_perm(vte, vto, 0x5410), 1);
        const uint32_t re = __shfl_down_sync(0xffffffffu, vte, 1);
        const int v_2 = int(lw & 0xffffu), v_1 = int(lw >> 16);
        const int v0 = int(vte & 0xffffu), v1 = int(vto & 0xffffu), v2 = int(vte >> 16), v3 = int(vto >> 16);
        const int v4 = int(rw & 0xffffu), v5 = int(rw >> 16), v6 = int(re >> 16);
        const uint32_t cwd = centre_px(v_2, v_1, v0, v1, v2, v3) | centre_px(v_1, v0, v1, v2, v3, v4) << 8 |
                             centre_px(v0, v1, v2, v3, v4, v5) << 16 | centre_px(v1, v2, v3, v4, v5, v6) << 24;
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
    const int y0 = band * HP_BAND;
    const int y1 = y0 + HP_BAND < ph ? y0 + HP_BAND : ph;
    HpelRow r0 = load(y0 - 2), r1 = load(y0 - 1), r2 = load(y0), r3 = load(y0 + 1), r4 = load(y0 + 2), r5;
    // six rows per iteration, the window rotating through r0..r5 by name
    for (int y = y0; y < y1; y += 6) {
        r5 = load(y + 3);
        emit(y, r0, r1, r2, r3, r4, r5);
        if (y + 1 >= y1) break;
        r0 = load(y + 4);
        emit(y + 1, r1, r2, r3, r4, r5, r0);
        if (y + 2 >= y1) break;
        r1 = load(y + 5);
        emit(y + 2, r2, r3, r4, r5, r0, r1);
        if (y + 3 >= y1) break;
        r2 = load(y + 6);
        emit(y + 3, r3, r4, r5, r0, r1, r2);
        if (y + 4 >= y1) break;
        r3 = load(y + 7);
        emit(y + 4, r4, r5, r0, r1, r2, r3);
        if (y + 5 >= y1) break;
        r4 = load(y + 8);
        emit(y + 5, r5, r0, r1, r2, r3, r4);
    }
}

}  // namespace h264a

using namespace h264a;

extern "C" int h264a_hpel_build(h264a_ctx* ctx, const uint8_t* d_ref, int cw, int ch, int pad, int n,
                                size_t ref_frame_stride, uint8_t* d_planes, void* stream) {
    if (!ctx || !d_ref || !d_planes) return fail(H264A_E_ARG, "hpel_build: null pointer");
    if (cw < 1 || ch < 1 || n < 1 || pad < 3 || pad > 128)
        return fail(H264A_E_ARG, "hpel_build: need cw, ch, n >= 1 and 3 <= pad <= 128");
    if (n > 65535) return fail(H264A_E_ARG, "hpel_build: at most 65535 pictures per call");
    if (n > 1 && ref_frame_stride < (size_t)cw * ch) return fail(H264A_E_ARG, "hpel_build: frame stride < cw*ch");
    const int pw = cw + 2 * pad, ph = ch + 2 * pad;
    const int word_in = (cw % 4 == 0) && (pad % 4 == 0) && (ref_frame_stride % 4 == 0) &&
                        ((reinterpret_cast<uintptr_t>(d_ref) & 3) == 0);
    const int word_out = (pw % 4 == 0) && ((reinterpret_cast<uintptr_t>(d_planes) & 3) == 0);
    const int strips = (pw + HP_STRIP - 1) / HP_STRIP, bands = (ph + HP_BAND - 1) / HP_BAND;
    const long long nwarps = (long long)strips * bands * n;
    const long long blocks = (nwarps + HP_WARPS - 1) / HP_WARPS;
    hpel_build_kernel<<<unsigned(blocks), 32 * HP_WARPS, 0, pick_stream(ctx, stream)>>>(
        d_ref, cw, ch, pad, ref_frame_stride, d_planes, pw, ph, strips, bands, nwarps, word_in, word_out);
    return check_launch("hpel_build_kernel");
}
