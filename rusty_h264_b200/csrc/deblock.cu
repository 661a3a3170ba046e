// deblock.cu -- §8f row 3: in-loop deblocking of the plain-ME P pictures
// (crates/rusty_h264-common/src/deblock.rs).
//
// The reference filters MBs in raster order, in place: per MB the luma
// vertical edges, the luma horizontal edges, then per chroma plane its
// vertical and horizontal edges.  An MB's filtering reads and writes three
// samples into its left and top neighbours, and the top edge reads samples
// that the top-right MB's left edge wrote, so an MB is ready once its left
// and top-right neighbours are done: the same wavefront as motion-vector
// prediction.  One persistent kernel deals MB tickets in that order (frames
// interleaved, bounded waits on the neighbours' flags); a warp filters its MB
// on shared-memory tiles (20x20 luma and 10x12 per chroma plane, the MB plus
// the samples its edges reach) and writes them back through L2.  No MB
// earlier in the order writes an MB's own samples, so they and bS are loaded
// before the wait; after it only the neighbours' strips are fetched, and luma
// (lanes 0..15) and chroma (lanes 16..31) are filtered side by side, one line
// per lane through all edges of a direction.
#include <algorithm>
#include <cstring>
#include <vector>

#include "deblock_device.cuh"

namespace h264a {

struct DbFrameDesc {
    uint8_t* y;
    uint8_t* uv[2];
    const int32_t* picks;
    const int16_t* coeffs;
    int cw, ch, mb_w, mb_h, flag_base;
    DbThresh th;
};
constexpr int DB_MAXF = 64;
struct DbBatch {
    DbFrameDesc f[DB_MAXF];
    long long seg_start[DB_MAXF + 1];
    int n;
};

constexpr int DB_WARPS = 4;
// Resident CTAs per SM: 8 x 4 warps hold about two and a half wavefront steps
// of a 59-picture 1080p batch; more only adds warps polling flags.
constexpr int DB_BLOCKS_PER_SM = 8;

__device__ __forceinline__ void block_state(const DbFrameDesc& fd, int m, int bx, int by, int& mvx, int& mvy,
                                            bool& nz) {
    block_state_at(fd.picks, fd.coeffs, m, bx, by, mvx, mvy, nz);
}

__global__ void __launch_bounds__(32 * DB_WARPS) deblock_frames_kernel(const __grid_constant__ DbBatch batch,
                                                                       long long total, int* __restrict__ counter,
                                                                       int* __restrict__ flags, int epoch,
                                                                       int* __restrict__ status, int spin_limit) {
    __shared__ __align__(16) uint8_t ltile[DB_WARPS][LT * LT];
    __shared__ __align__(16) uint8_t ctile[DB_WARPS][2][CR * CT];
    __shared__ int bsw[DB_WARPS][32];
    const int w = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    uint8_t* lt = ltile[w];
    for (;;) {
        int t = 0;
        if (lane == 0) t = atomicAdd(counter, 1);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) return;
        // segments are dealt from s = 0 (every frame, j = n - 1) on
        int s = 0;
        while (s + 1 < batch.n && batch.seg_start[s + 1] <= t) s++;
        const int j = batch.n - 1 - s;
        const long long u = t - batch.seg_start[s];
        const int nxt = j + 1 < batch.n ? batch.f[j + 1].mb_w * batch.f[j + 1].mb_h : 0;
        const DbFrameDesc& fd = batch.f[int(u % (j + 1))];
        const int k = nxt + int(u / (j + 1));
        int mbx, mby;
        wave_mb(fd.mb_w, fd.mb_h, k, mbx, mby);
        const int m = mby * fd.mb_w + mbx;
        int* fl = flags + fd.flag_base;
        const int y0 = mby * 16, x0 = mbx * 16;
        const int cy0 = mby * 8, cx0 = mbx * 8, ccw = fd.cw / 2;
        const bool has_c = fd.uv[0] != nullptr;
        // ---- before the wait: the MB's own samples (no MB earlier in the
        // order writes them) and bS: lanes 0..15 the vertical edges (edge
        // e = lane / 4, block row lane % 4), lanes 16..31 the horizontal ones ----
        for (int i = lane; i < 64; i += 32) {
            const int r = i >> 2, c4 = (i & 3) * 4;
            *reinterpret_cast<uint32_t*>(lt + (4 + r) * LT + 4 + c4) =
                __ldcg(reinterpret_cast<const unsigned int*>(fd.y + (long long)(y0 + r) * fd.cw + x0 + c4));
        }
        if (has_c) {
            const int pl = lane >> 4, r = (lane >> 1) & 7, c4 = (lane & 1) * 4;
            *reinterpret_cast<uint32_t*>(&ctile[w][pl][(2 + r) * CT + 4 + c4]) =
                __ldcg(reinterpret_cast<const unsigned int*>(fd.uv[pl] + (long long)(cy0 + r) * ccw + cx0 + c4));
        }
        {
            const int hor = lane >> 4, e = (lane >> 2) & 3, sg = lane & 3;
            int bs = 0;
            if (e > 0 || (hor ? mby > 0 : mbx > 0)) {
                int pmx, pmy, qmx, qmy;
                bool pnz, qnz;
                if (hor) {
                    block_state(fd, e > 0 ? m : m - fd.mb_w, sg, e > 0 ? e - 1 : 3, pmx, pmy, pnz);
                    block_state(fd, m, sg, e, qmx, qmy, qnz);
                } else {
                    block_state(fd, e > 0 ? m : m - 1, e > 0 ? e - 1 : 3, sg, pmx, pmy, pnz);
                    block_state(fd, m, e, sg, qmx, qmy, qnz);
                }
                bs = bs_of(pnz, qnz, pmx, pmy, qmx, qmy);
            }
            bsw[w][lane] = bs;
        }
        // ---- wait for the left (lane 0) and top-right (lane 1) neighbours ----
        if (lane == 0 && mbx > 0) wait_flag(fl + m - 1, epoch, status, 1, spin_limit);
        if (lane == 1 && mby > 0)
            wait_flag(fl + m - fd.mb_w + (mbx < fd.mb_w - 1 ? 1 : 0), epoch, status, 1, spin_limit);
        __syncwarp();
        // ---- the neighbours' samples the edges reach, through L2 ----
        const DbStrips strips(lane, fd.y, fd.cw, x0, y0, fd.uv, cx0, cy0, lt, ctile[w][0], ctile[w][1], mbx > 0,
                              mby > 0, has_c);
        strips.load();
        __syncwarp();
        deblock_mb_tiles(lane, lt, ctile[w][0], ctile[w][1], bsw[w], mbx > 0, mby > 0, has_c, fd.th);
        // ---- write back: the MB and the strips ----
        db_store_mb(lane, lt, ctile[w][0], ctile[w][1], fd.y, fd.cw, x0, y0, fd.uv, cx0, cy0, has_c);
        strips.store();
        __syncwarp();  // every lane's stores ordered before lane 0's release
        if (lane == 0) st_release(fl + m, epoch);
        __syncwarp();
    }
}

}  // namespace h264a

using namespace h264a;

extern "C" int h264a_deblock_frames(h264a_ctx* ctx, const h264a_deblock_frame* h_frames, int nframes, void* stream) {
    if (!ctx || !h_frames || nframes < 1) return fail(H264A_E_ARG, "deblock_frames: bad arguments");
    for (int i = 0; i < nframes; i++) {
        const h264a_deblock_frame& f = h_frames[i];
        if (!f.d_y || !f.d_picks || !f.d_coeffs) return fail(H264A_E_ARG, "deblock_frames: null frame pointer");
        if ((f.d_u == nullptr) != (f.d_v == nullptr))
            return fail(H264A_E_ARG, "deblock_frames: give both chroma planes or neither");
        if (f.cw < 16 || f.ch < 16 || f.cw % 16 || f.ch % 16 || (long long)(f.cw / 16) * (f.ch / 16) > (1 << 24))
            return fail(H264A_E_ARG, "deblock_frames: frames must be MB-aligned");
        const uintptr_t a = reinterpret_cast<uintptr_t>(f.d_y) | reinterpret_cast<uintptr_t>(f.d_u) |
                            reinterpret_cast<uintptr_t>(f.d_v);
        if ((a & 3) != 0 || (reinterpret_cast<uintptr_t>(f.d_coeffs) & 15) != 0)
            return fail(H264A_E_ARG, "deblock_frames: planes must be 4-byte and coefficients 16-byte aligned");
        if (f.qp < 0 || f.qp > 51) return fail(H264A_E_ARG, "deblock_frames: qp out of 0..51");
    }
    cudaStream_t st = pick_stream(ctx, stream);
    std::vector<int> order(nframes);
    for (int i = 0; i < nframes; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return (long long)h_frames[a].cw * h_frames[a].ch > (long long)h_frames[b].cw * h_frames[b].ch;
    });
    for (int g0 = 0; g0 < nframes; g0 += DB_MAXF) {
        const int gn = nframes - g0 < DB_MAXF ? nframes - g0 : DB_MAXF;
        DbBatch b;
        memset(&b, 0, sizeof b);
        b.n = gn;
        long long total = 0;
        for (int k = 0; k < gn; k++) {
            const h264a_deblock_frame& f = h_frames[order[g0 + k]];
            DbFrameDesc& d = b.f[k];
            d.y = f.d_y;
            d.uv[0] = f.d_u;
            d.uv[1] = f.d_v;
            d.picks = f.d_picks;
            d.coeffs = f.d_coeffs;
            d.cw = f.cw;
            d.ch = f.ch;
            d.mb_w = f.cw / 16;
            d.mb_h = f.ch / 16;
            d.flag_base = int(total);
            d.th = db_thresholds(f.qp, f.offset_a, f.offset_b, f.chroma_qp_offset);
            total += (long long)d.mb_w * d.mb_h;
        }
        long long acc = 0;
        for (int s = 0; s < gn; s++) {
            const int jj = gn - 1 - s;
            b.seg_start[s] = acc;
            const long long nj = (long long)b.f[jj].mb_w * b.f[jj].mb_h;
            const long long nn = jj + 1 < gn ? (long long)b.f[jj + 1].mb_w * b.f[jj + 1].mb_h : 0;
            acc += (nj - nn) * (jj + 1);
        }
        b.seg_start[gn] = acc;
        if (acc != total) return fail(H264A_E_ARG, "deblock_frames: internal queue layout error");
        int rc = ensure_me_scratch(ctx, size_t(total));
        if (rc) return rc;
        H264A_CUDA(cudaMemsetAsync(ctx->q[Q_MAIN].d_counter, 0, sizeof(int32_t), st));
        const int epoch = next_epoch(ctx, st);
        if (epoch < 0) return H264A_E_CUDA;
        int per_sm = 0;
        H264A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, deblock_frames_kernel, 32 * DB_WARPS, 0));
        if (per_sm > DB_BLOCKS_PER_SM) per_sm = DB_BLOCKS_PER_SM;
        long long blocks = (long long)ctx->num_sms * (per_sm > 0 ? per_sm : 1);
        const long long need = (total + DB_WARPS - 1) / DB_WARPS;
        if (blocks > need) blocks = need;
        deblock_frames_kernel<<<unsigned(blocks), 32 * DB_WARPS, 0, st>>>(b, total, ctx->q[Q_MAIN].d_counter, ctx->q[Q_MAIN].d_flags,
                                                                          epoch, ctx->d_status, SPIN_LIMIT);
        rc = check_launch("deblock_frames_kernel");
        if (rc) return rc;
    }
    return H264A_OK;
}
