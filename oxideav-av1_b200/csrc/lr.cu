// lr.cu — §7.17 loop restoration (Wiener and self-guided filters).
//
// Replaces loop_restoration_frame / loop_restore_block / wiener_filter /
// self_guided_filter / box_filter / get_source_sample
// (src/loop_restoration.rs:268-883) as driven by loop_restore_frame_from_grid
// (src/cdf.rs:20624).
//
// The reference filters 4x4 blocks (MI_SIZE walk), each recomputing its
// 7-tap Wiener rows and its box sums over a halo.  Every quantity it computes
// is a function of the sample position, the restoration unit and the 64-row
// stripe only (stripe boundaries fall on 4x4 block boundaries and unit
// boundaries on stripe boundaries), so the B200 kernel computes each quantity
// once per position: one CTA owns (plane, stripe, column tile) where the tile
// width min(unit size, 64) lies inside a single restoration unit.  The CTA
// stages the stripe's source window with a 3-sample halo in shared memory —
// rows inside the stripe from the CDEF frame, up to 2 rows beyond it from the
// deblocked frame, clamped to the plane, exactly get_source_sample — and then
// runs the separable Wiener filter or the two box-filter passes and the
// projection.  Units of type RESTORE_NONE copy the CDEF samples through.
#include "common.cuh"

namespace av1g {

namespace {

constexpr int TW = 64, TH = 64, H3 = 3;
constexpr int SW = TW + 2 * H3, SH = TH + 2 * H3, SP = SW + 1;  // source window
constexpr int AW = TW + 2, AH = TH + 2, AP = AW + 1;             // A/B grid

__constant__ int8_t c_sgr_params[16][4] = {
    {2, 12, 1, 4}, {2, 15, 1, 6}, {2, 18, 1, 8}, {2, 21, 1, 9}, {2, 24, 1, 10}, {2, 29, 1, 11},
    {2, 36, 1, 12}, {2, 45, 1, 13}, {2, 56, 1, 14}, {2, 68, 1, 15}, {0, 0, 1, 5}, {0, 0, 1, 8},
    {0, 0, 1, 11}, {0, 0, 1, 14}, {2, 30, 0, 0}, {2, 75, 0, 0}};

// source window + A + B + the two filtered outputs
constexpr size_t kSmemBytes = sizeof(int) * (SH * SP + 2 * AH * AP + 2 * TH * TW);

struct LrTile {
    int plane, stripe, ct;
};

__device__ __forceinline__ int r2u(int x, int n) { return n ? (x + (1 << (n - 1))) >> n : x; }

__device__ __forceinline__ int tile_w(const av1g_frame_header& h, int p) {
    int us = h.lr_unit_size[p] > 0 ? h.lr_unit_size[p] : 1;
    return us < TW ? us : TW;
}

__device__ __forceinline__ int n_stripes(const av1g_frame_header& h, int p) {
    int ssy = p ? h.subsampling_y : 0;
    int ph = r2u(h.frame_height, ssy);
    return ((((ph - 1) << ssy) + 8) >> 6) + 1;
}

__device__ __forceinline__ int count_units(int us, int sz) {
    int n = (sz + (us >> 1)) / us;
    return n > 1 ? n : 1;
}

// box_filter A/B + weighting (loop_restoration.rs:594-736) for one radius over
// the tile, leaving F[i][j] (the filtered value before projection) in `out`.
__device__ void box_pass(const int* src, int* A, int* B, int* out, int th, int tw, int bd, int r,
                         int eps, int pass, int y0) {
    int n = (2 * r + 1) * (2 * r + 1);
    long long n2e = (long long)n * n * eps;
    unsigned s = (unsigned)(((1LL << 20) + n2e / 2) / n2e);
    int one_over_n = ((1 << 12) + n / 2) / n;
    int sa = 2 * (bd - 8), sb = bd - 8;
    for (int k = threadIdx.x; k < (th + 2) * (tw + 2); k += blockDim.x) {
        int i = k / (tw + 2), j = k % (tw + 2);  // position (i-1, j-1) in tile coords
        const int* w = src + (i - 1 + H3) * SP + (j - 1 + H3);
        int a = 0, b = 0;
        for (int dy = -r; dy <= r; dy++)
            for (int dx = -r; dx <= r; dx++) {
                int c = w[dy * SP + dx];
                a += c * c;
                b += c;
            }
        int ar = sa ? (a + (1 << (sa - 1))) >> sa : a;
        int dr = sb ? (b + (1 << (sb - 1))) >> sb : b;
        long long p = (long long)ar * n - (long long)dr * dr;
        if (p < 0) p = 0;
        int z = (int)(((unsigned long long)p * s + (1ULL << 19)) >> 20);
        int a2 = z >= 255 ? 256 : (z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1));
        long long b2 = (long long)(256 - a2) * b * one_over_n;
        A[i * AP + j] = a2;
        B[i * AP + j] = (int)((b2 + (1 << 11)) >> 12);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < th * tw; k += blockDim.x) {
        int i = k / tw, j = k % tw;
        int odd = (y0 + i) & 1;
        int as = 0, bs = 0;
        if (pass == 0) {
            if (odd) {
                const int* a = A + (i + 1) * AP + j;
                const int* bb = B + (i + 1) * AP + j;
                as = 5 * a[0] + 6 * a[1] + 5 * a[2];
                bs = 5 * bb[0] + 6 * bb[1] + 5 * bb[2];
            } else {
                const int* a0 = A + i * AP + j;
                const int* a2 = A + (i + 2) * AP + j;
                const int* b0 = B + i * AP + j;
                const int* b2 = B + (i + 2) * AP + j;
                as = 5 * (a0[0] + a0[2] + a2[0] + a2[2]) + 6 * (a0[1] + a2[1]);
                bs = 5 * (b0[0] + b0[2] + b2[0] + b2[2]) + 6 * (b0[1] + b2[1]);
            }
        } else {
            const int* a = A + i * AP + j;
            const int* bb = B + i * AP + j;
            as = 3 * (a[0] + a[2] + a[2 * AP] + a[2 * AP + 2]) + 4 * (a[1] + a[AP] + a[AP + 1] + a[AP + 2] + a[2 * AP + 1]);
            bs = 3 * (bb[0] + bb[2] + bb[2 * AP] + bb[2 * AP + 2]) + 4 * (bb[1] + bb[AP] + bb[AP + 1] + bb[AP + 2] + bb[2 * AP + 1]);
        }
        int shift = (pass == 0 && odd) ? 4 : 5;
        int u = src[(i + H3) * SP + j + H3];
        int v = as * u + bs;
        int sh = 8 + shift - 4;
        out[k] = (v + (1 << (sh - 1))) >> sh;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(256) lr_kernel(const FrameDev* __restrict__ frames,
                                                 const int32_t* __restrict__ starts, int n, int total) {
    extern __shared__ int smem[];
    int* src = smem;
    int* A = src + SH * SP;
    int* B = A + AH * AP;
    int* F0 = B + AH * AP;
    int* inter = A;  // Wiener reuses the A/B space
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        int f = find_frame(starts, n, t);
        const FrameDev& F = frames[f];
        const av1g_frame_header& h = F.h;
        int local = t - starts[f];
        int plane = 0, stripe = 0, ct = 0;
        for (int p = 0; p < h.num_planes; p++) {
            if (h.lr_type[p] == 0) continue;
            int pw = r2u(h.upscaled_width, p ? h.subsampling_x : 0);
            int nct = (pw + tile_w(h, p) - 1) / tile_w(h, p);
            int cnt = nct * n_stripes(h, p);
            if (local < cnt) { plane = p; stripe = local / nct; ct = local % nct; break; }
            local -= cnt;
        }
        const int ssx = plane ? h.subsampling_x : 0, ssy = plane ? h.subsampling_y : 0;
        const int pw = r2u(h.upscaled_width, ssx), ph = r2u(h.frame_height, ssy);
        const int tw_ = tile_w(h, plane);
        const int x0 = ct * tw_, x1 = min(x0 + tw_, pw);
        const int sstart = (-8 + stripe * 64) >> ssy, send = sstart + (64 >> ssy) - 1;
        const int y0 = max(0, sstart), y1 = min(ph, send + 1);
        const int tw = x1 - x0, th = y1 - y0;
        const int hbd = F.hbd, bd = h.bit_depth;
        const PlaneDev& C = F.upcdef[plane];
        const PlaneDev& Dq = F.updeb[plane];
        const PlaneDev& O = F.lr[plane];
        // restoration unit of this tile (derive_block_geometry, loop_restoration.rs:370-428)
        int us = h.lr_unit_size[plane] > 0 ? h.lr_unit_size[plane] : 1;
        int urows = count_units(us, ph), ucols = count_units(us, pw);
        int ur = min(urows - 1, ((((y0 << ssy) + 8) >> ssy) / us));
        int uc = min(ucols - 1, x0 / us);
        av1g_lr_unit u{};
        if (F.lr_units[plane] && ur < F.lr_unit_rows[plane] && uc < F.lr_unit_cols[plane])
            u = F.lr_units[plane][ur * F.lr_unit_cols[plane] + uc];
        __syncthreads();
        if (u.type != 1 && u.type != 2) {
            for (int k = threadIdx.x; k < th * tw; k += blockDim.x) {
                int i = k / tw, j = k % tw;
                st_px(O, hbd, y0 + i, x0 + j, ld_px(C, hbd, y0 + i, x0 + j));
            }
            continue;
        }
        // source window: get_source_sample (loop_restoration.rs:862-883)
        for (int k = threadIdx.x; k < (th + 2 * H3) * (tw + 2 * H3); k += blockDim.x) {
            int i = k / (tw + 2 * H3), j = k % (tw + 2 * H3);
            int x = clip3(0, pw - 1, x0 - H3 + j), y = clip3(0, ph - 1, y0 - H3 + i);
            int v;
            if (y < sstart) v = ld_px(Dq, hbd, clip3(0, Dq.h - 1, max(y, sstart - 2)), min(x, Dq.w - 1));
            else if (y > send) v = ld_px(Dq, hbd, clip3(0, Dq.h - 1, min(y, send + 2)), min(x, Dq.w - 1));
            else v = ld_px(C, hbd, min(y, C.h - 1), min(x, C.w - 1));
            src[i * SP + j] = v;
        }
        __syncthreads();
        const int maxv = (1 << bd) - 1;
        if (u.type == 1) {
            int hf[7], vf[7];
            hf[3] = vf[3] = 128;
#pragma unroll
            for (int i = 0; i < 3; i++) {
                vf[i] = vf[6 - i] = u.wiener[0][i];
                vf[3] -= 2 * u.wiener[0][i];
                hf[i] = hf[6 - i] = u.wiener[1][i];
                hf[3] -= 2 * u.wiener[1][i];
            }
            int rr0 = bd == 12 ? 5 : 3, rr1 = bd == 12 ? 9 : 11;
            int off = 1 << (bd + 7 - rr0 - 1);
            int lim = (1 << (bd + 1 + 7 - rr0)) - 1;
            for (int k = threadIdx.x; k < (th + 6) * tw; k += blockDim.x) {
                int i = k / tw, j = k % tw;
                const int* w = src + i * SP + j;
                int s = 0;
#pragma unroll
                for (int q = 0; q < 7; q++) s += hf[q] * w[q];
                inter[i * TW + j] = clip3(-off, lim - off, (s + (1 << (rr0 - 1))) >> rr0);
            }
            __syncthreads();
            for (int k = threadIdx.x; k < th * tw; k += blockDim.x) {
                int i = k / tw, j = k % tw;
                int s = 0;
#pragma unroll
                for (int q = 0; q < 7; q++) s += vf[q] * inter[(i + q) * TW + j];
                st_px(O, hbd, y0 + i, x0 + j, clip3(0, maxv, (s + (1 << (rr1 - 1))) >> rr1));
            }
            continue;
        }
        // self-guided (loop_restoration.rs:485-588)
        int set = u.sgr_set < 16 ? u.sgr_set : 15;
        int r0 = c_sgr_params[set][0], e0 = c_sgr_params[set][1];
        int r1 = c_sgr_params[set][2], e1 = c_sgr_params[set][3];
        int w0 = u.sgr_xqd[0], w1 = u.sgr_xqd[1], w2 = 128 - w0 - w1;
        int* F1 = F0 + TH * TW;
        if (r0) box_pass(src, A, B, F0, th, tw, bd, r0, e0, 0, y0);
        if (r1) box_pass(src, A, B, F1, th, tw, bd, r1, e1, 1, y0);
        for (int k = threadIdx.x; k < th * tw; k += blockDim.x) {
            int i = k / tw, j = k % tw;
            int uu = src[(i + H3) * SP + j + H3] << 4;
            int v = w1 * uu + w0 * (r0 ? F0[k] : uu) + w2 * (r1 ? F1[k] : uu);
            st_px(O, hbd, y0 + i, x0 + j, clip3(0, maxv, (v + (1 << 10)) >> 11));
        }
    }
}

}  // namespace

size_t lr_smem_bytes() { return kSmemBytes; }

int tiles_lr(const FrameDev& f) {
    const av1g_frame_header& h = f.h;
    int n = 0;
    for (int p = 0; p < h.num_planes; p++) {
        if (h.lr_type[p] == 0) continue;
        int ssx = p ? h.subsampling_x : 0, ssy = p ? h.subsampling_y : 0;
        int pw = ssx ? (h.upscaled_width + 1) >> 1 : h.upscaled_width;
        int ph = ssy ? (h.frame_height + 1) >> 1 : h.frame_height;
        int us = h.lr_unit_size[p] > 0 ? h.lr_unit_size[p] : 1;
        int tw = us < TW ? us : TW;
        int ns = ((((ph - 1) << ssy) + 8) >> 6) + 1;
        n += ((pw + tw - 1) / tw) * ns;
    }
    return n;
}

void launch_lr(const FrameDev* frames, const int32_t* starts, int n, int total, cudaStream_t s) {
    if (total <= 0) return;
    size_t bytes = lr_smem_bytes();
    cudaFuncSetAttribute(lr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    int grid = total < kSMs * 2 ? total : kSMs * 2;
    lr_kernel<<<grid, 256, bytes, s>>>(frames, starts, n, total);
}

}  // namespace av1g
