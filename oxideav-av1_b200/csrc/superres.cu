// superres.cu — §7.16 horizontal super-resolution upscaling.
//
// Replaces upscale_frame / upscale_plane / upscale_sample
// (src/superres.rs:282-445) as called at frame_driver.rs:906-966: both the
// CDEF output and (when loop restoration is on) the deblocked frame are
// upscaled from the padded FrameWidth-wide planes to exact UpscaledWidth x
// FrameHeight planes.  One CTA row-tile per (source set, plane, row); each
// thread produces output samples of the row with the 8-tap polyphase kernel
// at the 14-bit fixed-point step, clamping source positions to the mi-padded
// width exactly as the reference does.
#include "common.cuh"
#include "av1_spec_tables.h"

namespace av1g {

__constant__ AV1T_UPSCALE_FILTER_TYPE c_upscale AV1T_UPSCALE_FILTER_DIMS = AV1T_UPSCALE_FILTER_INIT;

namespace {

__device__ __forceinline__ int r2u(int x, int n) { return n ? (x + (1 << (n - 1))) >> n : x; }

__global__ void __launch_bounds__(256) superres_kernel(const FrameDev* __restrict__ frames,
                                                       const int32_t* __restrict__ starts, int n, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        int f = find_frame(starts, n, t);
        const FrameDev& F = frames[f];
        const av1g_frame_header& h = F.h;
        int local = t - starts[f];
        int nsets = h.uses_lr ? 2 : 1;
        // tile -> (set, plane, row)
        int set = 0, plane = 0, y = 0;
        {
            int rem = local;
            bool found = false;
            for (int s = 0; s < nsets && !found; s++)
                for (int p = 0; p < h.num_planes && !found; p++) {
                    int ph = r2u(h.frame_height, p ? h.subsampling_y : 0);
                    if (rem < ph) { set = s; plane = p; y = rem; found = true; }
                    else rem -= ph;
                }
        }
        int ssx = plane ? h.subsampling_x : 0;
        int dw = r2u(h.frame_width, ssx), uw = r2u(h.upscaled_width, ssx);
        long long stepx_num = ((long long)dw << 14) + uw / 2;
        int step_x = (int)(stepx_num / uw);
        int err = (int)((long long)uw * step_x - ((long long)dw << 14));
        long long num = -(((long long)uw - dw) << 13) + uw / 2;
        int init = (int)(num / uw) + (1 << 7) - err / 2;
        init &= (1 << 14) - 1;
        int max_x = (h.mi_cols >> ssx) * 4 - 1;
        int maxv = (1 << h.bit_depth) - 1;
        const PlaneDev& S = set == 0 ? F.cdef[plane] : F.deb[plane];
        const PlaneDev& D = set == 0 ? F.upcdef[plane] : F.updeb[plane];
        const int hbd = F.hbd;
        for (int x = threadIdx.x; x < uw; x += blockDim.x) {
            int src_x = -(1 << 14) + init + x * step_x;
            int px = src_x >> 14;
            int sub = ((src_x & ((1 << 14) - 1)) >> 8) & 63;
            int sum = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                int sx = clip3(0, max_x, px + k - 3);
                sx = clip3(0, S.w - 1, sx);
                sum += ld_px(S, hbd, y, sx) * c_upscale[sub][k];
            }
            st_px(D, hbd, y, x, clip3(0, maxv, round2(sum, 7)));
        }
    }
}

}  // namespace

int tiles_superres(const FrameDev& f) {
    int rows = 0;
    for (int p = 0; p < f.h.num_planes; p++) {
        int ssy = p ? f.h.subsampling_y : 0;
        rows += ssy ? (f.h.frame_height + 1) >> 1 : f.h.frame_height;
    }
    return rows * (f.h.uses_lr ? 2 : 1);
}

void launch_superres(const FrameDev* frames, const int32_t* starts, int n, int total, cudaStream_t s) {
    if (total <= 0) return;
    int grid = total < kSMs * 8 ? total : kSMs * 8;
    superres_kernel<<<grid, 256, 0, s>>>(frames, starts, n, total);
}

}  // namespace av1g
