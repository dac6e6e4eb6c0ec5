// intra.cu — §7.11.2 intra prediction, §7.11.5 chroma from luma and intra
// reconstruction as a superblock-diagonal wavefront.
//
// Replaces predict_intra_into_curr_frame (src/cdf.rs:16789),
// intra_predict_block_samples (cdf.rs:16990-17250), the mode kernels
// (cdf.rs:1348-3120) and predict_chroma_from_luma_into_curr_frame
// (cdf.rs:17256) in the order transform_block_emit runs them per TU
// (cdf.rs:32540-32910): predict, CfL, dequant + inverse transform + merge.
//
// An intra TU reads the final samples of the row above and the column to its
// left, up to twice its size (above-right / below-left when already decoded).
// Within a superblock that forces decode order; across superblocks every
// reference points at the same or an earlier superblock row and at most one
// superblock to the right in the row above, so superblock (c, r) only depends
// on superblocks of level c + 2r - 1 or lower.  The host groups each frame's
// TUs by superblock and launches one kernel per level over all frames of the
// batch (no inter-CTA waiting); one 64-thread CTA runs its superblock's TUs in
// decode order, parallel within each TU.
#include <algorithm>
#include <cstring>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "common.cuh"
#include "itx.cuh"
#include "wedge.cuh"

namespace av1g {

namespace {

using namespace itx;

constexpr int kT = 64;
constexpr int kEdge = 272;  // 2 * (64 + 64) + 2 rounded up; index 0 == position -2

__constant__ AV1T_MODE_TO_ANGLE_TYPE c_mode_angle AV1T_MODE_TO_ANGLE_DIMS = AV1T_MODE_TO_ANGLE_INIT;
__constant__ AV1T_DR_INTRA_DERIVATIVE_TYPE c_dr AV1T_DR_INTRA_DERIVATIVE_DIMS = AV1T_DR_INTRA_DERIVATIVE_INIT;
__constant__ AV1T_INTRA_EDGE_KERNEL_TYPE c_edge_k AV1T_INTRA_EDGE_KERNEL_DIMS = AV1T_INTRA_EDGE_KERNEL_INIT;
__constant__ AV1T_INTRA_FILTER_TAPS_TYPE c_fi_taps AV1T_INTRA_FILTER_TAPS_DIMS = AV1T_INTRA_FILTER_TAPS_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_4X4_TYPE c_sm4 AV1T_SM_WEIGHTS_TX_4X4_DIMS = AV1T_SM_WEIGHTS_TX_4X4_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_8X8_TYPE c_sm8 AV1T_SM_WEIGHTS_TX_8X8_DIMS = AV1T_SM_WEIGHTS_TX_8X8_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_16X16_TYPE c_sm16 AV1T_SM_WEIGHTS_TX_16X16_DIMS = AV1T_SM_WEIGHTS_TX_16X16_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_32X32_TYPE c_sm32 AV1T_SM_WEIGHTS_TX_32X32_DIMS = AV1T_SM_WEIGHTS_TX_32X32_INIT;
__constant__ AV1T_SM_WEIGHTS_TX_64X64_TYPE c_sm64 AV1T_SM_WEIGHTS_TX_64X64_DIMS = AV1T_SM_WEIGHTS_TX_64X64_INIT;
__constant__ AV1T_SUBPEL_FILTERS_TYPE c_subpel AV1T_SUBPEL_FILTERS_DIMS = AV1T_SUBPEL_FILTERS_INIT;

struct IntraFrame {
    ReconFrame rf;
    int32_t ssx, ssy;
    const uint8_t* maps;  // palette colour-index pool
    PlaneDev side[3];     // inter halves of inter-intra blocks
};

__device__ const AV1T_II_WEIGHTS_1D_TYPE g_ii_w AV1T_II_WEIGHTS_1D_DIMS = AV1T_II_WEIGHTS_1D_INIT;
__device__ const wedge::Master g_wmaster = wedge::kMaster;

// The intra half of an inter-intra block: blend of the intra prediction
// with the inter half (mask_blend_interintra, src/inter_pred.rs:3272).  The
// mask is the §7.11.3.13 smooth mask on the plane block (read at [i][j]
// directly) or the §7.11.3.11 wedge mask on the luma grid (orientation
// resolved by the host into palette_map).
template <int W, int H>
__device__ __forceinline__ int interintra_px(const IntraFrame& F, const av1g_intra_tu& t, int i, int j, int intra,
                                             int inter, int maxv) {
    int m;
    if (t.interintra == 2) {
        const uint32_t o = t.palette_map;
        const wedge::Orient w{(uint8_t)(o & 0xff), (uint8_t)((o >> 8) & 0xff), (uint8_t)((o >> 16) & 0xff),
                              (uint8_t)(o >> 24)};
        m = wedge::mask_px(g_wmaster, w, t.plane ? F.ssx : 0, t.plane ? F.ssy : 0, i, j);
    } else {
        constexpr int scale = 128 / (W > H ? W : H);
        const int mode = t.interintra_mode;
        m = mode == 1 ? __ldg(&g_ii_w[i * scale]) : mode == 2 ? __ldg(&g_ii_w[j * scale])
          : mode == 3 ? __ldg(&g_ii_w[min(i, j) * scale]) : 32;
    }
    return min(max((m * intra + (64 - m) * inter + 32) >> 6, 0), maxv);
}

struct IntraItem {
    int32_t frame, first, count, level;
};

struct Smem {
    uint16_t above[kEdge], left[kEdge], dup[kEdge];
    uint16_t pred[64 * 64];
    int buf[64 * 64];
    long long red[kT / 32];
    av1g_intra_tu tu;
};

__device__ __forceinline__ const uint8_t* sm_weights(int log2n) {
    return log2n == 2 ? c_sm4 : log2n == 3 ? c_sm8 : log2n == 4 ? c_sm16 : log2n == 5 ? c_sm32 : c_sm64;
}

// CTA-wide sum (all threads call)
__device__ long long block_sum(Smem& s, long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffff, v, o);
    if ((threadIdx.x & 31) == 0) s.red[threadIdx.x >> 5] = v;
    __syncthreads();
    long long t = 0;
#pragma unroll
    for (int k = 0; k < kT / 32; k++) t += s.red[k];
    __syncthreads();
    return t;
}

// intra_edge_filter_strength_selection (cdf.rs:2610)
__device__ int strength_sel(int w, int h, int ft, int delta) {
    int d = abs(delta), wh = w + h, st = 0;
    if (ft == 0) {
        if (wh <= 8) { if (d >= 56) st = 1; }
        else if (wh <= 16) { if (d >= 40) st = 1; }
        else if (wh <= 24) { if (d >= 8) st = 1; if (d >= 16) st = 2; if (d >= 32) st = 3; }
        else if (wh <= 32) { st = 1; if (d >= 4) st = 2; if (d >= 32) st = 3; }
        else st = 3;
    } else {
        if (wh <= 8) { if (d >= 40) st = 1; if (d >= 64) st = 2; }
        else if (wh <= 16) { if (d >= 20) st = 1; if (d >= 48) st = 2; }
        else if (wh <= 24) { if (d >= 4) st = 3; }
        else st = 3;
    }
    return st;
}
// intra_edge_upsample_selection (cdf.rs:2588)
__device__ int upsample_sel(int w, int h, int ft, int delta) {
    int d = abs(delta);
    if (d == 0 || d >= 40) return 0;
    return ft == 0 ? (w + h <= 16) : (w + h <= 8);
}

// intra_edge_filter (cdf.rs:2760) on an edge array (index 0 == position -2), in parallel
__device__ void edge_filter(Smem& s, uint16_t* e, int sz, int strength) {
    if (strength == 0 || sz == 0) return;  // uniform
    for (int i = threadIdx.x; i < sz; i += kT) s.dup[i] = e[i + 1];
    __syncthreads();
    for (int i = 1 + threadIdx.x; i < sz; i += kT) {
        int acc = 0;
#pragma unroll
        for (int j = 0; j < 5; j++) acc += c_edge_k[strength - 1][j] * s.dup[clip3(0, sz - 1, i - 2 + j)];
        e[i + 1] = (uint16_t)max((acc + 8) >> 4, 0);
    }
    __syncthreads();
}

// intra_edge_upsample (cdf.rs:2700), in parallel
__device__ void edge_upsample(Smem& s, uint16_t* e, int n, int bd) {
    if (threadIdx.x == 0) {
        s.dup[0] = e[1];
        s.dup[1] = e[1];
        s.dup[n + 2] = e[n + 1];
    }
    for (int i = threadIdx.x; i < n; i += kT) s.dup[i + 2] = e[i + 2];
    __syncthreads();
    const int maxv = (1 << bd) - 1;
    if (threadIdx.x == 0) e[0] = s.dup[0];
    for (int i = threadIdx.x; i < n; i += kT) {
        int sum = -s.dup[i] + 9 * s.dup[i + 1] + 9 * s.dup[i + 2] - s.dup[i + 3];
        int r = sum >= 0 ? (sum + 8) >> 4 : -(((-sum) + 8) >> 4);
        e[2 * i + 1] = (uint16_t)clip3(0, maxv, r);
        e[2 * i + 2] = (uint16_t)min((int)s.dup[i + 2], maxv);
    }
    __syncthreads();
}

// One TU: prediction (+ CfL) into the plane, then the residual.
template <int TX>
__device__ void intra_tu(Smem& s, const IntraFrame& F, const av1g_intra_tu& t) {
    constexpr int W = kTxW[TX], H = kTxH[TX], L = W > H ? W : H;
    constexpr int LW = ilog2<W>(), LH = ilog2<H>();
    const int tid = threadIdx.x;
    const PlaneDev& P = F.rf.planes[t.plane];
    const int hbd = F.rf.hbd, bd = F.rf.bd;
    const int sx = t.x, sy = t.y;
    if (t.mode < 13) {
        const int max_x = P.w - 1, max_y = P.h - 1;
        auto rd = [&](int yy, int xx) { return ld_px(P, hbd, min(yy, max_y), min(xx, max_x)); };
        const bool ha = (t.flags & AV1G_INTRA_HAVE_ABOVE) && sy > 0;
        const bool hl = (t.flags & AV1G_INTRA_HAVE_LEFT) && sx > 0;
        const bool har = t.flags & AV1G_INTRA_HAVE_ABOVE_RIGHT, hbl = t.flags & AV1G_INTRA_HAVE_BELOW_LEFT;
        const bool eief = t.flags & AV1G_INTRA_EDGE_FILTER;
        const int ft = (t.flags & AV1G_INTRA_FILTER_TYPE) ? 1 : 0;
        const int corner = ha && hl ? rd(sy - 1, sx - 1) : ha ? rd(sy - 1, sx) : hl ? rd(sy, sx - 1) : 1 << (bd - 1);
        constexpr int span = W + H;
        // edge arrays (intra_predict_block_samples, cdf.rs:17030-17075)
        for (int i = tid; i < span; i += kT) {
            int a, l;
            if (!ha && hl) a = rd(sy, sx - 1);
            else if (!ha && !hl) a = (1 << (bd - 1)) - 1;
            else a = rd(sy - 1, min(min(max_x, sx + (har ? 2 * W : W) - 1), sx + i));
            if (!hl && ha) l = rd(sy - 1, sx);
            else if (!hl && !ha) l = (1 << (bd - 1)) + 1;
            else l = rd(min(min(max_y, sy + (hbl ? 2 * H : H) - 1), sy + i), sx - 1);
            s.above[2 + i] = (uint16_t)a;
            s.left[2 + i] = (uint16_t)l;
        }
        if (tid < 2) s.above[tid] = s.left[tid] = (uint16_t)corner;
        __syncthreads();
        const bool dir = t.mode >= 1 && t.mode <= 8;
        const int pa = c_mode_angle[t.mode] + t.angle_delta * 3;
        int ua = 0, ul = 0;
        if (dir && eief && pa != 90 && pa != 180) {
            if (pa > 90 && pa < 180 && span >= 24) {
                if (tid == 0) {
                    uint16_t fc = (uint16_t)((s.left[2] * 5 + s.above[1] * 6 + s.above[2] * 5 + 8) >> 4);
                    s.above[1] = fc;
                    s.left[1] = fc;
                }
                __syncthreads();
            }
            if (ha) edge_filter(s, s.above, min(W, max_x - sx + 1) + (pa < 90 ? H : 0) + 1, strength_sel(W, H, ft, pa - 90));
            if (hl) edge_filter(s, s.left, min(H, max_y - sy + 1) + (pa > 180 ? W : 0) + 1, strength_sel(W, H, ft, pa - 180));
            ua = upsample_sel(W, H, ft, pa - 90);
            if (ua) edge_upsample(s, s.above, W + (pa < 90 ? H : 0), bd);
            ul = upsample_sel(W, H, ft, pa - 180);
            if (ul) edge_upsample(s, s.left, H + (pa > 180 ? W : 0), bd);
        }
        const uint16_t* A = s.above + 2;  // A[k] == AboveRow[k]
        const uint16_t* Lc = s.left + 2;
        const int fim = (t.plane == 0 && t.filter_intra_mode < 5) ? t.filter_intra_mode : -1;
        if (fim >= 0) {
            // predict_intra_recursive (cdf.rs:2145): 4x2 cells, wavefront over i2 + j4
            constexpr int W4 = W >> 2, H2 = H >> 1;
            const int maxv = (1 << bd) - 1;
            for (int d = 0; d < W4 + H2 - 1; d++) {
                int b = tid >> 3, o = tid & 7;
                int i2 = max(0, d - (W4 - 1)) + b, j4 = d - i2;
                if (i2 < H2 && j4 >= 0) {
                    int p[7];
#pragma unroll
                    for (int i = 0; i < 7; i++) {
                        if (i < 5) {
                            if (i2 == 0) p[i] = A[(j4 << 2) + i - 1];
                            else if (j4 == 0 && i == 0) p[i] = Lc[(i2 << 1) - 1];
                            else p[i] = s.pred[((i2 << 1) - 1) * W + (j4 << 2) + i - 1];
                        } else if (j4 == 0) {
                            p[i] = Lc[(i2 << 1) + i - 5];
                        } else {
                            p[i] = s.pred[((i2 << 1) + i - 5) * W + (j4 << 2) - 1];
                        }
                    }
                    int i1 = o >> 2, j1 = o & 3;
                    int acc = 0;
#pragma unroll
                    for (int i = 0; i < 7; i++) acc += c_fi_taps[fim][(i1 << 2) + j1][i] * p[i];
                    int v = acc >= 0 ? (acc + 8) >> 4 : -(((-acc) + 8) >> 4);
                    s.pred[((i2 << 1) + i1) * W + (j4 << 2) + j1] = (uint16_t)clip3(0, maxv, v);
                }
                __syncthreads();
            }
        } else if (t.mode == 0) {
            // predict_intra_dc_pred (cdf.rs:1348)
            long long part = 0;
            for (int i = tid; i < span; i += kT) {
                if (hl && i < H) part += Lc[i];
                if (ha && i < W) part += A[i];
            }
            long long sum = block_sum(s, part);
            unsigned avg;
            if (hl && ha) avg = (unsigned)((sum + (span >> 1)) / span);
            else if (hl) avg = min((unsigned)((sum + (H >> 1)) >> LH), (1u << bd) - 1);
            else if (ha) avg = min((unsigned)((sum + (W >> 1)) >> LW), (1u << bd) - 1);
            else avg = 1u << (bd - 1);
            for (int k = tid; k < W * H; k += kT) s.pred[k] = (uint16_t)avg;
        } else {
            const int dx = pa < 90 ? c_dr[pa] : (pa < 180 ? c_dr[180 - pa] : 0);
            const int dy = (pa >= 90 && pa < 180) ? c_dr[pa - 90] : (pa > 180 ? c_dr[270 - pa] : 0);
            const uint8_t* swx = sm_weights(LW);
            const uint8_t* swy = sm_weights(LH);
            for (int k = tid; k < W * H; k += kT) {
                int i = k >> LW, j = k & (W - 1);
                int v;
                if (t.mode == 1 && t.angle_delta == 0) {
                    v = A[j];
                } else if (t.mode == 2 && t.angle_delta == 0) {
                    v = Lc[i];
                } else if (dir) {
                    // predict_intra_directional (cdf.rs:2879-3010)
                    if (pa < 90) {
                        int maxb = (W + H - 1) << ua;
                        int idx = (i + 1) * dx;
                        int base = (idx >> (6 - ua)) + j * (1 << ua);
                        int sh = ((idx * (1 << ua)) >> 1) & 0x1F;
                        v = base < maxb ? (A[base] * (32 - sh) + A[base + 1] * sh + 16) >> 5 : A[maxb];
                    } else if (pa < 180) {
                        int ix = (j << 6) - (i + 1) * dx;
                        int bx = ix >> (6 - ua);
                        if (bx >= -(1 << ua)) {
                            int sh = ((ix * (1 << ua)) >> 1) & 0x1F;
                            v = (A[bx] * (32 - sh) + A[bx + 1] * sh + 16) >> 5;
                        } else {
                            int iy = (i << 6) - (j + 1) * dy;
                            int by = iy >> (6 - ul);
                            int sh = ((iy * (1 << ul)) >> 1) & 0x1F;
                            v = (Lc[by] * (32 - sh) + Lc[by + 1] * sh + 16) >> 5;
                        }
                    } else {
                        int maxb = (W + H - 1) << ul;
                        int idx = (j + 1) * dy;
                        int base = (idx >> (6 - ul)) + i * (1 << ul);
                        int sh = ((idx * (1 << ul)) >> 1) & 0x1F;
                        v = base < maxb ? (Lc[base] * (32 - sh) + Lc[base + 1] * sh + 16) >> 5 : Lc[maxb];
                    }
                } else if (t.mode == 9) {  // SMOOTH (cdf.rs:2267)
                    unsigned sp = swy[i] * A[j] + (256 - swy[i]) * Lc[H - 1] + swx[j] * Lc[i] + (256 - swx[j]) * A[W - 1];
                    v = (int)((sp + 256) >> 9);
                } else if (t.mode == 10) {  // SMOOTH_V
                    v = (int)((swy[i] * A[j] + (256 - swy[i]) * Lc[H - 1] + 128) >> 8);
                } else if (t.mode == 11) {  // SMOOTH_H
                    v = (int)((swx[j] * Lc[i] + (256 - swx[j]) * A[W - 1] + 128) >> 8);
                } else {  // PAETH (cdf.rs:2077)
                    int base = A[j] + Lc[i] - corner;
                    int pl = abs(base - Lc[i]), pt = abs(base - A[j]), ptl = abs(base - corner);
                    v = (pl <= pt && pl <= ptl) ? Lc[i] : (pt <= ptl ? A[j] : corner);
                }
                s.pred[k] = (uint16_t)v;
            }
        }
        __syncthreads();
        if (t.interintra) {
            const PlaneDev& SD = F.side[t.plane];
            const int maxv = (1 << bd) - 1;
            for (int k = tid; k < W * H; k += kT) {
                int i = k >> LW, j = k & (W - 1);
                if (sy + i < P.h && sx + j < P.w)
                    st_px(P, hbd, sy + i, sx + j,
                          interintra_px<W, H>(F, t, i, j, s.pred[k], ld_px(SD, hbd, sy + i, sx + j), maxv));
            }
        } else {
            for (int k = tid; k < W * H; k += kT) {
                int i = k >> LW, j = k & (W - 1);
                if (sy + i < P.h && sx + j < P.w) st_px(P, hbd, sy + i, sx + j, s.pred[k]);
            }
        }
        __syncthreads();
    }
    if (t.mode == AV1G_INTRA_MODE_PALETTE || t.mode == AV1G_INTRA_MODE_INTRABC) {
        const int maxv = (1 << bd) - 1;
        if (t.mode == AV1G_INTRA_MODE_PALETTE) {
            // predict_palette (cdf.rs:11907); indices checked on the host
            const uint8_t* m = F.maps + t.palette_map;
            for (int k = tid; k < W * H; k += kT) {
                int i = k >> LW, j = k & (W - 1);
                s.pred[k] = s.tu.palette_colors[m[i * t.palette_stride + j]];
            }
        } else {
            // predict_intrabc_leaf_into_curr_frame (cdf.rs:19235): BILINEAR
            // block_inter_prediction from the pre-filter plane at unit scale,
            // start = (x << 10) + (((2 * mv) >> ss) << 6) + 32, clamped to the
            // mi-padded plane (the reference's window clamp is the same set).
            const int pss_x = t.plane ? F.ssx : 0, pss_y = t.plane ? F.ssy : 0;
            const int stx = (sx << 10) + ((2 * t.mv[1]) >> pss_x) * 64 + 32;
            const int sty = (sy << 10) + ((2 * t.mv[0]) >> pss_y) * 64 + 32;
            const int r0 = bd == 12 ? 5 : 3, r1 = bd == 12 ? 9 : 11;
            const int hph = (stx >> 6) & 15, vph = (sty >> 6) & 15;
            for (int k = tid; k < W * H; k += kT) {
                int i = k >> LW, j = k & (W - 1);
                int xi = ((stx >> 10) + j) - 3, yi = ((sty >> 10) + i) - 3;
                int acc = 0;
                for (int tt = 0; tt < 8; tt++) {
                    int vc = c_subpel[3][vph][tt];
                    if (!vc) continue;
                    int yy = min(max(yi + tt, 0), P.h - 1);
                    int hsum = 0;
                    for (int u = 0; u < 8; u++) {
                        int hc = c_subpel[3][hph][u];
                        if (hc) hsum += hc * ld_px(P, hbd, yy, min(max(xi + u, 0), P.w - 1));
                    }
                    acc += vc * ((hsum + ((1 << r0) >> 1)) >> r0);
                }
                s.pred[k] = (uint16_t)min(max((acc + (1 << (r1 - 1))) >> r1, 0), maxv);
            }
        }
        __syncthreads();
        for (int k = tid; k < W * H; k += kT) {
            int i = k >> LW, j = k & (W - 1);
            if (sy + i < P.h && sx + j < P.w) st_px(P, hbd, sy + i, sx + j, s.pred[k]);
        }
        __syncthreads();
    }
    if ((t.flags & AV1G_INTRA_CFL) && t.plane > 0) {
        // predict_chroma_from_luma_into_curr_frame (cdf.rs:17256-17340); luma
        // outside the luma plane reads as 0
        const PlaneDev& Y = F.rf.planes[0];
        const int ssx = F.ssx, ssy = F.ssy;
        const int cx = max((int)t.max_luma_w - (1 << ssx), 0), cy = max((int)t.max_luma_h - (1 << ssy), 0);
        long long part = 0;
        for (int k = tid; k < W * H; k += kT) {
            int i = k >> LW, j = k & (W - 1);
            int ly = min((sy + i) << ssy, cy), lx = min((sx + j) << ssx, cx);
            int acc = 0;
            for (int ddy = 0; ddy <= ssy; ddy++)
                for (int ddx = 0; ddx <= ssx; ddx++) {
                    int yy = ly + ddy, xx = lx + ddx;
                    acc += (yy < Y.h && xx < Y.w) ? ld_px(Y, hbd, yy, xx) : 0;
                }
            int v = acc << (3 - ssx - ssy);
            s.buf[k] = v;
            part += v;
        }
        long long sum = block_sum(s, part);
        long long half = 1LL << (LW + LH - 1);
        long long avg = sum >= 0 ? (sum + half) >> (LW + LH) : -(((-sum) + half) >> (LW + LH));
        const int maxv = (1 << bd) - 1;
        for (int k = tid; k < W * H; k += kT) {
            int i = k >> LW, j = k & (W - 1);
            if (sy + i >= P.h || sx + j >= P.w) continue;
            long long d = (long long)t.cfl_alpha * (s.buf[k] - avg);
            long long sc = d >= 0 ? (d + 32) >> 6 : -(((-d) + 32) >> 6);
            long long v = ld_px(P, hbd, sy + i, sx + j) + sc;
            st_px(P, hbd, sy + i, sx + j, (int)min(max(v, 0LL), (long long)maxv));
        }
        __syncthreads();
    }
    if (t.flags & AV1G_INTRA_RESIDUAL) {
        const int slot = tid / L, lane = tid % L;
        recon_core<TX>(F.rf, t.res, slot == 0, lane, s.buf + slot * W * H);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kT) intra_kernel(const IntraFrame* __restrict__ frames,
                                                   const av1g_intra_tu* __restrict__ tus,
                                                   const IntraItem* __restrict__ items, int nitems) {
    __shared__ Smem s;
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const IntraItem item = items[it];
        const IntraFrame& F = frames[item.frame];
        for (int k = item.first; k < item.first + item.count; k++) {
            __syncthreads();
            if (threadIdx.x == 0) s.tu = tus[k];
            __syncthreads();
            const av1g_intra_tu t = s.tu;
            switch (t.tx_size) {
                case 0: intra_tu<0>(s, F, t); break;
                case 1: intra_tu<1>(s, F, t); break;
                case 2: intra_tu<2>(s, F, t); break;
                case 3: intra_tu<3>(s, F, t); break;
                case 4: intra_tu<4>(s, F, t); break;
                case 5: intra_tu<5>(s, F, t); break;
                case 6: intra_tu<6>(s, F, t); break;
                case 7: intra_tu<7>(s, F, t); break;
                case 8: intra_tu<8>(s, F, t); break;
                case 9: intra_tu<9>(s, F, t); break;
                case 10: intra_tu<10>(s, F, t); break;
                case 11: intra_tu<11>(s, F, t); break;
                case 12: intra_tu<12>(s, F, t); break;
                case 13: intra_tu<13>(s, F, t); break;
                case 14: intra_tu<14>(s, F, t); break;
                case 15: intra_tu<15>(s, F, t); break;
                case 16: intra_tu<16>(s, F, t); break;
                case 17: intra_tu<17>(s, F, t); break;
                default: intra_tu<18>(s, F, t); break;
            }
        }
    }
}

}  // namespace

// Host side of av1g_run_intra: validation, superblock grouping, level order, launches.
av1g_status intra_run(const av1g_intra_job* jobs, int n, cudaStream_t st, std::string& err) {
    std::vector<IntraFrame> frames(n);
    std::vector<av1g_intra_tu> all;
    std::vector<IntraItem> items;
    std::vector<std::pair<size_t, uint32_t>> wedge_pack;  // (TU index, packed wedge window)
    std::vector<uint8_t> maps;            // palette colour indices of all jobs
    std::vector<size_t> map_base(n, 0);
    for (int i = 0; i < n; i++) {
        const av1g_intra_job& j = jobs[i];
        if (!j.hdr || !j.quant || j.num_tus < 0 || (j.num_tus > 0 && !j.tus) || (j.sb_size != 64 && j.sb_size != 128) ||
            j.palette_map_bytes < 0 || (j.palette_map_bytes > 0 && !j.palette_maps)) {
            err = "intra job " + std::to_string(i) + ": missing header/quantizer/TUs/maps or superblock size not 64/128";
            return AV1G_EINVAL;
        }
        const av1g_frame_header& h = *j.hdr;
        if (h.bit_depth != 8 && h.bit_depth != 10 && h.bit_depth != 12) {
            err = "intra job " + std::to_string(i) + ": bit depth";
            return AV1G_EINVAL;
        }
        IntraFrame& F = frames[i];
        memset(&F, 0, sizeof F);
        F.rf.bd = h.bit_depth;
        F.rf.hbd = h.bit_depth > 8;
        F.rf.q = *j.quant;
        F.rf.coeffs = j.coeffs;
        F.ssx = h.subsampling_x;
        F.ssy = h.subsampling_y;
        for (int p = 0; p < h.num_planes; p++) {
            int sx = p ? h.subsampling_x : 0, sy = p ? h.subsampling_y : 0;
            int pw = (h.mi_cols * 4) >> sx, ph = (h.mi_rows * 4) >> sy;
            const av1g_plane& pl = j.planes[p];
            if (!pl.data || pl.width < pw || pl.height < ph || pl.stride < pw * (F.rf.hbd ? 2 : 1) || (pl.stride & 15)) {
                err = "intra job " + std::to_string(i) + ": plane " + std::to_string(p);
                return AV1G_EINVAL;
            }
            F.rf.planes[p] = PlaneDev{(uint8_t*)pl.data, pl.stride, pw, ph};
        }
        map_base[i] = maps.size();
        if (j.palette_map_bytes > 0) maps.insert(maps.end(), j.palette_maps, j.palette_maps + j.palette_map_bytes);
        // superblocks in decode order, and the intra block copy windows
        struct Sb {
            int sbx, sby, seq;
        };
        std::vector<Sb> sbs;
        std::unordered_map<long long, int> sb_index;
        struct Bc {
            int sb, x0, y0, x1, y1;  // luma-sample window, inclusive
        };
        std::vector<Bc> bcs;
        int base = (int)all.size();
        int first_item = (int)items.size();
        long long prev = -1;
        for (int k = 0; k < j.num_tus; k++) {
            const av1g_intra_tu& t = j.tus[k];
            bool res = t.flags & AV1G_INTRA_RESIDUAL;
            bool fi_ok = !(t.plane == 0 && t.filter_intra_mode < 5) || (t.tx_size != 4 && t.tx_size != 11 &&
                                                                        t.tx_size != 12 && t.tx_size != 17 &&
                                                                        t.tx_size != 18);
            if (t.tx_size >= 19 || t.plane >= h.num_planes || !fi_ok ||
                (res && (t.res.tx_size != t.tx_size || t.res.plane != t.plane || t.res.x != t.x || t.res.y != t.y ||
                         t.res.tx_type >= 16 || !j.coeffs))) {
                err = "intra job " + std::to_string(i) + ": TU " + std::to_string(k) + " is malformed";
                return AV1G_EINVAL;
            }
            const int tw = kTxW[t.tx_size], th = kTxH[t.tx_size];
            const int pss_x = t.plane ? h.subsampling_x : 0, pss_y = t.plane ? h.subsampling_y : 0;
            if (t.interintra) {
                // the intra half of an inter-intra block: an II mode's intra
                // mode (DC, V, H, SMOOTH) over the whole block, then the blend
                static const uint8_t ii_to_intra[4] = {0, 1, 2, 9};
                const av1g_plane& sp = j.interintra_in[t.plane];
                wedge::Orient o{};
                bool ok = t.interintra <= 2 && t.interintra_mode <= 3 && t.mode == ii_to_intra[t.interintra_mode] &&
                          t.filter_intra_mode >= 5 && !(t.flags & AV1G_INTRA_CFL) && sp.data &&
                          sp.width >= F.rf.planes[t.plane].w && sp.height >= F.rf.planes[t.plane].h &&
                          sp.stride >= F.rf.planes[t.plane].w * (F.rf.hbd ? 2 : 1) && !(sp.stride & 15);
                if (ok && t.interintra == 2)
                    ok = wedge::orient(t.mi_size, t.wedge_index, 0, tw, th, pss_x, pss_y, o);
                if (!ok) {
                    err = "intra job " + std::to_string(i) + ": inter-intra TU " + std::to_string(k) + " is malformed";
                    return AV1G_EINVAL;
                }
                F.side[t.plane] = PlaneDev{(uint8_t*)sp.data, sp.stride, F.rf.planes[t.plane].w, F.rf.planes[t.plane].h};
                // the device copy of the TU carries the wedge window in
                // palette_map (an inter-intra TU has no palette)
                wedge_pack.emplace_back((size_t)(base + k), (uint32_t)o.dir | ((uint32_t)o.xoff << 8) |
                                                                ((uint32_t)o.yoff << 16) | ((uint32_t)o.invert << 24));
            }
            if (t.mode == AV1G_INTRA_MODE_PALETTE) {
                // predict_palette's checks (cdf.rs:11907-11960)
                long long last = (long long)t.palette_map + (long long)(th - 1) * t.palette_stride + (tw - 1);
                bool ok = t.palette_size >= 1 && t.palette_size <= 8 && t.palette_stride >= tw &&
                          last < j.palette_map_bytes;
                for (int r = 0; ok && r < th; r++)
                    for (int c = 0; ok && c < tw; c++)
                        ok = j.palette_maps[t.palette_map + (long long)r * t.palette_stride + c] < t.palette_size;
                if (!ok) {
                    err = "intra job " + std::to_string(i) + ": palette TU " + std::to_string(k) + " is malformed";
                    return AV1G_EINVAL;
                }
            }
            int lx = t.x << pss_x, ly = t.y << pss_y;
            long long sb = ((long long)(ly / j.sb_size) << 32) | (unsigned)(lx / j.sb_size);
            if (sb != prev) {
                if (sb_index.count(sb)) {
                    err = "intra job " + std::to_string(i) + ": TUs of a superblock are not contiguous in decode order";
                    return AV1G_EINVAL;
                }
                int sbx = lx / j.sb_size, sby = ly / j.sb_size;
                sb_index[sb] = (int)sbs.size();
                sbs.push_back(Sb{sbx, sby, (int)sbs.size()});
                items.push_back(IntraItem{i, base + k, 0, 0});
                prev = sb;
            }
            if (t.mode == AV1G_INTRA_MODE_INTRABC) {
                if (std::abs((int)t.mv[0]) >= (1 << 14) || std::abs((int)t.mv[1]) >= (1 << 14)) {
                    err = "intra job " + std::to_string(i) + ": intra block copy TU " + std::to_string(k) +
                          " has a motion vector out of range";
                    return AV1G_EINVAL;
                }
                // the window the BILINEAR filter reads, in luma samples
                int pw = (h.mi_cols * 4) >> pss_x, ph = (h.mi_rows * 4) >> pss_y;
                int stx = (t.x << 10) + ((2 * t.mv[1]) >> pss_x) * 64 + 32;
                int sty = (t.y << 10) + ((2 * t.mv[0]) >> pss_y) * 64 + 32;
                int x0 = std::min(std::max((stx >> 10) - 3, 0), pw - 1);
                int x1 = std::min(std::max((stx >> 10) + tw - 1 + 4, 0), pw - 1);
                int y0 = std::min(std::max((sty >> 10) - 3, 0), ph - 1);
                int y1 = std::min(std::max((sty >> 10) + th - 1 + 4, 0), ph - 1);
                bcs.push_back(Bc{sb_index[sb], x0 << pss_x, y0 << pss_y, ((x1 + 1) << pss_x) - 1,
                                 ((y1 + 1) << pss_y) - 1});
            }
            items.back().count++;
            all.push_back(t);
        }
        // Superblock (c, r) gets level c + k r.  k = 2 covers the intra edge
        // reads (above-right is one superblock up and right).  An intra block
        // copy may read any earlier superblock, so every superblock its window
        // touches must sit on the same side of it in level order as in decode
        // order; steeper slopes follow the spec's intra-block-copy wavefront
        // delay, and decode order itself (one superblock per level) always
        // reproduces sequential decoding.
        auto level_ok = [&](auto level) {
            for (const Bc& b : bcs) {
                const Sb& cur = sbs[b.sb];
                for (int by = b.y0 / j.sb_size; by <= b.y1 / j.sb_size; by++)
                    for (int bx = b.x0 / j.sb_size; bx <= b.x1 / j.sb_size; bx++) {
                        auto it = sb_index.find(((long long)by << 32) | (unsigned)bx);
                        if (it == sb_index.end() || it->second == b.sb) continue;
                        const Sb& o = sbs[it->second];
                        int lo = level(o), lc = level(cur);
                        if (lo == lc || (o.seq < cur.seq) != (lo < lc)) return false;
                    }
            }
            return true;
        };
        int slope = 0;
        for (int k : {2, 3, 4, 5, 6, 8})
            if (level_ok([k](const Sb& b) { return b.sbx + k * b.sby; })) {
                slope = k;
                break;
            }
        for (int q = first_item; q < (int)items.size(); q++) {
            const Sb& b = sbs[q - first_item];
            items[q].level = slope ? b.sbx + slope * b.sby : b.seq;
        }
    }
    if (items.empty()) return AV1G_OK;
    for (const auto& wp : wedge_pack) all[wp.first].palette_map = wp.second;
    std::stable_sort(items.begin(), items.end(), [](const IntraItem& a, const IntraItem& b) { return a.level < b.level; });
    size_t off_tus = (sizeof(IntraFrame) * n + 255) & ~(size_t)255;
    size_t off_items = (off_tus + sizeof(av1g_intra_tu) * all.size() + 255) & ~(size_t)255;
    size_t off_maps = (off_items + sizeof(IntraItem) * items.size() + 255) & ~(size_t)255;
    size_t bytes = off_maps + maps.size();
    uint8_t* dev = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dev, bytes, st);
    if (e != cudaSuccess) {
        err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    for (int i = 0; i < n; i++) frames[i].maps = dev + off_maps + map_base[i];
    std::vector<uint8_t> host(bytes);
    memcpy(host.data(), frames.data(), sizeof(IntraFrame) * n);
    memcpy(host.data() + off_tus, all.data(), sizeof(av1g_intra_tu) * all.size());
    memcpy(host.data() + off_items, items.data(), sizeof(IntraItem) * items.size());
    if (!maps.empty()) memcpy(host.data() + off_maps, maps.data(), maps.size());
    e = upload(dev, host.data(), bytes, st);
    const IntraFrame* df = (const IntraFrame*)dev;
    const av1g_intra_tu* dt = (const av1g_intra_tu*)(dev + off_tus);
    const IntraItem* di = (const IntraItem*)(dev + off_items);
    for (size_t lo = 0; e == cudaSuccess && lo < items.size();) {
        size_t hi = lo;
        while (hi < items.size() && items[hi].level == items[lo].level) hi++;
        int cnt = (int)(hi - lo);
        intra_kernel<<<cnt, kT, 0, st>>>(df, dt, di + lo, cnt);
        e = cudaGetLastError();
        lo = hi;
    }
    cudaFreeAsync(dev, st);
    if (e != cudaSuccess) {
        err = std::string("intra launch: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    return AV1G_OK;
}

}  // namespace av1g
