// superres.cu — §7.16 horizontal super-resolution upscaling.
//
// Replaces upscale_frame / upscale_plane / upscale_sample
// (src/superres.rs:282-445) as called at frame_driver.rs:906-966: both the
// CDEF output and (when loop restoration is on) the deblocked frame are
// upscaled from the padded FrameWidth-wide planes to exact UpscaledWidth x
// FrameHeight planes.  A tile is 256, 512 or 1024 output samples (the launch
// shape's tile width) of one row of one plane of one source set: the CTA
// stages the source window those outputs read (clamped to the mi-padded
// width exactly as the reference clamps every tap) and the 64-phase filter
// table in shared memory, then each thread produces groups of four adjacent
// outputs with the 8-tap polyphase kernel at the 14-bit fixed-point step and
// stores each group as one vector.
#include "common.cuh"
#include "av1_spec_tables.h"

namespace av1g {

__constant__ AV1T_UPSCALE_FILTER_TYPE c_upscale AV1T_UPSCALE_FILTER_DIMS = AV1T_UPSCALE_FILTER_INIT;

namespace {

__device__ __forceinline__ int r2u(int x, int n) { return n ? (x + (1 << (n - 1))) >> n : x; }

constexpr int kSrMaxOut = 1024;          // output samples of a row per tile: 256, 512 or 1024 (launch shape)
constexpr int kSrThreads = 128;          // groups of 4 outputs per thread
constexpr int kSrWin = kSrMaxOut + 16;   // source window: the step is below 1, plus 8 taps, rounded up

// Output segments of a plane row.
__device__ __host__ __forceinline__ int sr_segs(int uw, int tile) { return (uw + tile - 1) / tile; }

// A plane of one source set, as a run of tiles: its step, start phase and
// the clamp bound shared by all its rows.
struct SrPlane {
    int first, rows, segs;  // tiles [first, first + rows * segs) of the frame
    int set, plane, step_x, init, lim, uw, maxv;
};

__device__ SrPlane sr_plane(const av1g_frame_header& h, int local, int cap_w, int tile) {
    SrPlane P{};
    int first = 0;
    const int nsets = h.uses_lr ? 2 : 1;
    for (int s = 0; s < nsets; s++)
        for (int p = 0; p < h.num_planes; p++) {
            const int ssx = p ? h.subsampling_x : 0;
            const int rows = r2u(h.frame_height, p ? h.subsampling_y : 0);
            const int uw = r2u(h.upscaled_width, ssx), segs = sr_segs(uw, tile);
            if (local < first + rows * segs || (s == nsets - 1 && p == h.num_planes - 1)) {
                // upscale_plane's step and start (superres.rs:363-377)
                const int dw = r2u(h.frame_width, ssx);
                const long long stepx_num = ((long long)dw << 14) + uw / 2;
                const int step_x = (int)(stepx_num / uw);
                const int err = (int)((long long)uw * step_x - ((long long)dw << 14));
                const long long num = -(((long long)uw - dw) << 13) + uw / 2;
                int init = (int)(num / uw) + (1 << 7) - err / 2;
                init &= (1 << 14) - 1;
                const int max_x = (h.mi_cols >> ssx) * 4 - 1;
                return SrPlane{first, rows, segs, s, p, step_x, init, min(max_x, cap_w - 1), uw, (1 << h.bit_depth) - 1};
            }
            first += rows * segs;
        }
    return P;
}

__global__ void __launch_bounds__(kSrThreads) superres_kernel(const FrameDev* __restrict__ frames,
                                                              const int32_t* __restrict__ starts, int n, int total,
                                                              int tile) {
    __shared__ __align__(16) int16_t filt[64][8];
    __shared__ uint16_t win[kSrWin];
    for (int i = threadIdx.x; i < 64 * 8; i += kSrThreads) filt[i >> 3][i & 7] = (int16_t)c_upscale[i >> 3][i & 7];
    // each CTA walks a contiguous run of tiles: the frame, plane and its
    // parameters change rarely, the row and segment advance by one
    const int per = (total + gridDim.x - 1) / gridDim.x;
    const int t0 = blockIdx.x * per, t1 = min(total, t0 + per);
    int f = -1, fend = 0, y = 0, seg = 0;
    SrPlane P{};
    const FrameDev* F = nullptr;
    for (int t = t0; t < t1; t++) {
        if (f < 0 || t >= fend || t - starts[f] >= P.first + P.rows * P.segs) {
            if (f < 0 || t >= fend) {
                f = find_frame(starts, n, t);
                fend = starts[f + 1];
                F = &frames[f];
            }
            const int local = t - starts[f];
            P = sr_plane(F->h, local, 1 << 30, tile);
            const PlaneDev& S0 = P.set == 0 ? F->cdef[P.plane] : F->deb[P.plane];
            P.lim = min(P.lim, S0.w - 1);
            y = (local - P.first) / P.segs;
            seg = (local - P.first) % P.segs;
        }
        const PlaneDev& S = P.set == 0 ? F->cdef[P.plane] : F->deb[P.plane];
        const PlaneDev& D = P.set == 0 ? F->upcdef[P.plane] : F->updeb[P.plane];
        const int hbd = F->hbd;
        const int x0 = seg * tile, x1 = min(P.uw, x0 + tile);
        const int lo = ((-(1 << 14) + P.init + x0 * P.step_x) >> 14) - 3;
        const int hi = ((-(1 << 14) + P.init + (x1 - 1) * P.step_x) >> 14) + 4;
        __syncthreads();  // the previous tile's window is no longer read
        const uint8_t* srow = S.p + (size_t)y * S.stride;
        for (int i = threadIdx.x; i <= hi - lo && i < kSrWin; i += kSrThreads) {
            const int sx = clip3(0, P.lim, lo + i);
            win[i] = hbd ? reinterpret_cast<const uint16_t*>(srow)[sx] : srow[sx];
        }
        __syncthreads();
        for (int xb = x0 + 4 * threadIdx.x; xb < x1; xb += 4 * kSrThreads) {
            int v[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int src_x = -(1 << 14) + P.init + (xb + j) * P.step_x;
                const int base = (src_x >> 14) - 3 - lo;
                const int sub = ((src_x & ((1 << 14) - 1)) >> 8) & 63;
                const int4 fr = *reinterpret_cast<const int4*>(filt[sub]);
                const int c[4] = {fr.x, fr.y, fr.z, fr.w};
                int sum = 0;
#pragma unroll
                for (int k = 0; k < 8; k++) sum += (int)win[base + k] * (int)(int16_t)(c[k >> 1] >> (16 * (k & 1)));
                v[j] = clip3(0, P.maxv, round2(sum, 7));
            }
            uint8_t* drow = D.p + (size_t)y * D.stride;
            const bool vec = xb + 4 <= x1 && !(((uintptr_t)drow | (unsigned)D.stride) & 7);
            if (vec) {
                if (hbd)
                    *reinterpret_cast<uint2*>(reinterpret_cast<uint16_t*>(drow) + xb) =
                        make_uint2((uint32_t)v[0] | ((uint32_t)v[1] << 16), (uint32_t)v[2] | ((uint32_t)v[3] << 16));
                else
                    *reinterpret_cast<uint32_t*>(drow + xb) =
                        (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
            } else {
                for (int j = 0; j < 4 && xb + j < x1; j++) st_px(D, hbd, y, xb + j, v[j]);
            }
        }
        if (++seg == P.segs) {
            seg = 0;
            y++;
        }
    }
}

}  // namespace

int tiles_superres(const FrameDev& f, int tile) {
    int tiles = 0;
    for (int p = 0; p < f.h.num_planes; p++) {
        const int ssy = p ? f.h.subsampling_y : 0, ssx = p ? f.h.subsampling_x : 0;
        const int rows = ssy ? (f.h.frame_height + 1) >> 1 : f.h.frame_height;
        const int uw = ssx ? (f.h.upscaled_width + 1) >> 1 : f.h.upscaled_width;
        tiles += rows * sr_segs(uw, tile);
    }
    return tiles * (f.h.uses_lr ? 2 : 1);
}

void launch_superres(const FrameDev* frames, const int32_t* starts, int n, int total, const StageShape& sh,
                     cudaStream_t s) {
    if (total <= 0) return;
    superres_kernel<<<shape_grid(sh, total), kSrThreads, 0, s>>>(frames, starts, n, total, sh.tile);
}

}  // namespace av1g
