// hpel.cu -- a1/a2: edge-padded full-pel plane F and the half-pel planes
// H, V, C of reference pictures (pad_plane_into + build_hpel_fused,
// crates/rusty_h264-common/src/inter.rs:798-991; AVX2 twin
// crates/rusty_h264-accel/src/hpel.rs:34-203).
//
// One CTA writes a TILE_W x TILE_H tile of all four planes.  The source halo
// ((TILE_H+5) x (TILE_W+5) bytes, edge-clamped, which is exactly the
// replication pad_plane performs) is staged once in shared memory; every
// thread then produces 16 consecutive bytes of one row of F, H, V and C and
// writes each with one 16-byte store.  HBM traffic is one read of the picture
// (plus the halo) and one write of the four planes.
#include "h264a_device.cuh"

namespace h264a {

constexpr int HP_TILE_W = 64;
constexpr int HP_TILE_H = 32;
constexpr int HP_PITCH = 72;  // >= TILE_W + 5, multiple of 4
constexpr int HP_ROWS = HP_TILE_H + 5;

__device__ __forceinline__ int clip255(int v) { return v < 0 ? 0 : (v > 255 ? 255 : v); }

__global__ void __launch_bounds__(128) hpel_build_kernel(const uint8_t* __restrict__ ref, int cw, int ch, int pad,
                                                        size_t ref_fstride, uint8_t* __restrict__ planes,
                                                        int pw, int ph, int vec_ok) {
    __shared__ __align__(16) uint8_t S[HP_ROWS * HP_PITCH];
    const int pic = blockIdx.z;
    const uint8_t* Y = ref + ref_fstride * pic;
    const long long ps = (long long)pw * ph;
    uint8_t* F = planes + 4 * ps * pic;
    uint8_t* H = F + ps;
    uint8_t* V = F + 2 * ps;
    uint8_t* C = F + 3 * ps;
    const int x0 = blockIdx.x * HP_TILE_W, y0 = blockIdx.y * HP_TILE_H;

    // Stage the clamped halo: S[ty][tx] = Y[clamp(y0+ty-2-pad)][clamp(x0+tx-2-pad)].
    for (int i = threadIdx.x; i < HP_ROWS * (HP_TILE_W + 5); i += blockDim.x) {
        const int ty = i / (HP_TILE_W + 5), tx = i - ty * (HP_TILE_W + 5);
        const int sy = clampi(y0 + ty - 2 - pad, 0, ch - 1);
        const int sx = clampi(x0 + tx - 2 - pad, 0, cw - 1);
        S[ty * HP_PITCH + tx] = __ldg(Y + (long long)sy * cw + sx);
    }
    __syncthreads();

    const int ty = threadIdx.x >> 2;          // output row within the tile
    const int cx = (threadIdx.x & 3) * 16;    // first output column within the tile
    const int y = y0 + ty, x = x0 + cx;
    if (y >= ph || x >= pw) return;

    // Vertical 6-tap intermediates (exact, unrounded) for tile columns cx..cx+20
    // (plane columns x-2..x+18): vt[j] = Σ tap·S[ty+k][cx+j].
    int vt[21];
#pragma unroll
    for (int j = 0; j < 21; j++) {
        const uint8_t* s = S + ty * HP_PITCH + cx + j;
        vt[j] = s[0] - 5 * s[HP_PITCH] + 20 * s[2 * HP_PITCH] + 20 * s[3 * HP_PITCH] - 5 * s[4 * HP_PITCH] +
                s[5 * HP_PITCH];
    }
    const uint8_t* mid = S + (ty + 2) * HP_PITCH + cx;
    uint32_t fw[4], hw[4], vw[4], cwd[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        uint32_t f = 0, h = 0, v = 0, c = 0;
#pragma unroll
        for (int b = 0; b < 4; b++) {
            const int i = q * 4 + b;
            const uint8_t* m = mid + i;  // m[2] is the sample at plane column x+i
            const int hs = m[0] - 5 * m[1] + 20 * m[2] + 20 * m[3] - 5 * m[4] + m[5];
            const int cs = vt[i] - 5 * vt[i + 1] + 20 * vt[i + 2] + 20 * vt[i + 3] - 5 * vt[i + 4] + vt[i + 5];
            f |= uint32_t(m[2]) << (8 * b);
            h |= uint32_t(clip255((hs + 16) >> 5)) << (8 * b);
            v |= uint32_t(clip255((vt[i + 2] + 16) >> 5)) << (8 * b);
            c |= uint32_t(clip255((cs + 512) >> 10)) << (8 * b);
        }
        fw[q] = f; hw[q] = h; vw[q] = v; cwd[q] = c;
    }
    const long long off = (long long)y * pw + x;
    if (vec_ok) {
        *reinterpret_cast<uint4*>(F + off) = make_uint4(fw[0], fw[1], fw[2], fw[3]);
        *reinterpret_cast<uint4*>(H + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
        *reinterpret_cast<uint4*>(V + off) = make_uint4(vw[0], vw[1], vw[2], vw[3]);
        *reinterpret_cast<uint4*>(C + off) = make_uint4(cwd[0], cwd[1], cwd[2], cwd[3]);
    } else {
        const int n = pw - x < 16 ? pw - x : 16;
        for (int i = 0; i < n; i++) {
            F[off + i] = uint8_t(fw[i >> 2] >> (8 * (i & 3)));
            H[off + i] = uint8_t(hw[i >> 2] >> (8 * (i & 3)));
            V[off + i] = uint8_t(vw[i >> 2] >> (8 * (i & 3)));
            C[off + i] = uint8_t(cwd[i >> 2] >> (8 * (i & 3)));
        }
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
    const int vec_ok = (pw % 16 == 0) && ((reinterpret_cast<uintptr_t>(d_planes) & 15) == 0);
    dim3 grid((pw + HP_TILE_W - 1) / HP_TILE_W, (ph + HP_TILE_H - 1) / HP_TILE_H, n);
    hpel_build_kernel<<<grid, 128, 0, pick_stream(ctx, stream)>>>(d_ref, cw, ch, pad, ref_frame_stride, d_planes, pw,
                                                                  ph, vec_ok);
    return check_launch("hpel_build_kernel");
}
