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
// per row, the six loads of an unrolled step issued together, no shared
// memory.  Sample columns and rows are clamped to the picture, which is
// exactly the replication pad_plane performs.
//
// Arithmetic on pairs of 16-bit columns (even bytes 0/2, odd bytes 1/3 of a
// word): the vertical intermediate vt and the horizontal sum of H are biased
// by 8208 = 256 * 32 + 16, so that no half goes negative (|taps| <= 2550) and
// every half stays below 18,920.  Clipped to [8192, 16383] and shifted right
// by 5, a half's low byte is clip((t + 16) >> 5), and one byte_perm gathers
// the four bytes of a word.  C sums six biased vt values per column in 32
// bits: the bias adds 8208 * 32 = 256 * 1024 + 512, the rounding term, so
// the sum >> 10, clipped to [256, 511], again has the sample in its low byte.
// HBM traffic is one read of the picture (the band halo mostly from L2) and
// one write of the four planes.
#include "hpel_device.cuh"

namespace h264a {

__global__ void __launch_bounds__(32 * HP_WARPS) hpel_build_kernel(const uint8_t* __restrict__ ref, int cw, int ch,
                                                                   int pad, size_t ref_fstride,
                                                                   uint8_t* __restrict__ planes, int pw, int ph,
                                                                   int strips, int bands, long long nwarps,
                                                                   int word_in, int word_out) {
    const long long wid = (long long)blockIdx.x * HP_WARPS + (threadIdx.x >> 5);
    if (wid >= nwarps) return;  // warp-uniform
    const long long per_pic = (long long)strips * bands;
    const int pic = int(wid / per_pic);
    const int rem = int(wid - per_pic * pic);
    const int band = rem / strips, strip = rem - band * strips;
    const int y0 = band * HP_BAND;
    hpel_strip_rows(ref + ref_fstride * pic, cw, ch, pad, planes + 4LL * pw * ph * pic, pw, ph, strip, y0,
                    y0 + HP_BAND < ph ? y0 + HP_BAND : ph, word_in, word_out);
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
