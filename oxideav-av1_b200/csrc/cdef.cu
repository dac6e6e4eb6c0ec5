// cdef.cu — §7.15 constrained directional enhancement filter.
//
// Replaces cdef_frame / cdef_block / cdef_direction / cdef_filter_block
// (src/cdef.rs:180-606) as driven by cdef_frame_from_idx (src/cdf.rs:20300).
// One CTA owns one 64x64 filter block (the cdef_idx granularity) across all
// planes: it stages the deblocked samples of the block plus a 2-sample halo
// (the furthest tap of Cdef_Directions) for every plane in shared memory,
// marking samples outside the plane as unavailable (the reference's
// CdefAvailable == 0 arm, cdef.rs:564-590), runs the direction search of the
// 64 luma 8x8 blocks, then filters every sample of every plane and writes the
// CDEF frame.  Samples of skipped blocks (cdef_idx == -1, or all four 4x4
// cells skipped) are copied through, as cdef_block does (cdef.rs:229-262).
#include "common.cuh"

namespace av1g {

namespace {

constexpr int FB = 64, H2 = 2, WMAX = FB + 2 * H2, WP = WMAX + 2;
constexpr int16_t NA = -32768;

__constant__ int8_t c_cdef_dirs[8][2][2] = {
    {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
    {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}}};
__constant__ int16_t c_div_table[9] = {0, 840, 420, 280, 210, 168, 140, 120, 105};
__constant__ int8_t c_uv_dir[2][2][8] = {{{0, 1, 2, 3, 4, 5, 6, 7}, {1, 2, 2, 2, 3, 4, 6, 0}},
                                         {{7, 0, 2, 4, 5, 6, 6, 6}, {0, 1, 2, 3, 4, 5, 6, 7}}};

struct BlockParams {
    int8_t active;  // 0: copy through
    int8_t ydir;
    int16_t pad;
    int32_t var;
};

__device__ __forceinline__ int constrain_adj(int diff, int threshold, int adj) {
    // constrain (cdef.rs:592-606) with dampingAdj precomputed
    int ad = abs(diff);
    int inner = max(threshold - (ad >> adj), 0);
    int v = min(ad, inner);
    return diff < 0 ? -v : v;
}

// cdef_direction (cdef.rs:366-456) on an 8x8 luma block in shared memory.
__device__ void direction(const int16_t* w, int shift, int* ydir, int* var) {
    int partial[8][15];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int b = 0; b < 15; b++) partial[a][b] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
            int x = (w[i * WP + j] >> shift) - 128;
            partial[0][i + j] += x;
            partial[1][i + j / 2] += x;
            partial[2][i] += x;
            partial[3][3 + i - j / 2] += x;
            partial[4][7 + i - j] += x;
            partial[5][3 - i / 2 + j] += x;
            partial[6][j] += x;
            partial[7][i / 2 + j] += x;
        }
    int cost[8];
#pragma unroll
    for (int k = 0; k < 8; k++) cost[k] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        cost[2] += partial[2][i] * partial[2][i];
        cost[6] += partial[6][i] * partial[6][i];
    }
    cost[2] *= 105;
    cost[6] *= 105;
#pragma unroll
    for (int i = 0; i < 7; i++) {
        cost[0] += (partial[0][i] * partial[0][i] + partial[0][14 - i] * partial[0][14 - i]) * c_div_table[i + 1];
        cost[4] += (partial[4][i] * partial[4][i] + partial[4][14 - i] * partial[4][14 - i]) * c_div_table[i + 1];
    }
    cost[0] += partial[0][7] * partial[0][7] * 105;
    cost[4] += partial[4][7] * partial[4][7] * 105;
#pragma unroll
    for (int i = 1; i < 8; i += 2) {
#pragma unroll
        for (int j = 0; j < 5; j++) cost[i] += partial[i][3 + j] * partial[i][3 + j];
        cost[i] *= 105;
#pragma unroll
        for (int j = 0; j < 3; j++)
            cost[i] += (partial[i][j] * partial[i][j] + partial[i][10 - j] * partial[i][10 - j]) * c_div_table[2 * j + 2];
    }
    int best = 0, d = 0;
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (cost[k] > best) { best = cost[k]; d = k; }
    *ydir = d;
    *var = (best - cost[(d + 4) & 7]) >> 10;
}

__global__ void __launch_bounds__(256) cdef_kernel(const FrameDev* __restrict__ frames,
                                                   const int32_t* __restrict__ starts, int n, int total) {
    __shared__ int16_t win[3][WMAX * WP];
    __shared__ BlockParams bp[64];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        int f = find_frame(starts, n, t);
        const FrameDev& F = frames[f];
        const av1g_frame_header& h = F.h;
        int local = t - starts[f];
        int fcols = (h.mi_cols + 15) >> 4;
        int fbr = local / fcols, fbc = local % fcols;
        int idx = F.cdef_idx[fbr * fcols + fbc];
        if (idx > 7) idx = -1;  // not a strength-set index: malformed, copied through
        const int hbd = F.hbd, np = h.num_planes;
        const int ssx = h.subsampling_x, ssy = h.subsampling_y;
        const int cs = h.bit_depth - 8;
        __syncthreads();
        for (int p = 0; p < np; p++) {
            int px = p ? ssx : 0, py = p ? ssy : 0;
            int bw = FB >> px, bh = FB >> py;
            int x0 = (fbc * FB) >> px, y0 = (fbr * FB) >> py;
            const PlaneDev& S = F.deb[p];
            int ww = bw + 2 * H2, wh = bh + 2 * H2;
            for (int i = threadIdx.x; i < ww * wh; i += blockDim.x) {
                int r = i / ww, c = i % ww;
                int gy = y0 - H2 + r, gx = x0 - H2 + c;
                win[p][r * WP + c] = (gy >= 0 && gy < S.h && gx >= 0 && gx < S.w) ? (int16_t)ld_px(S, hbd, gy, gx) : NA;
            }
        }
        __syncthreads();
        if (threadIdx.x < 64) {
            int bi = threadIdx.x >> 3, bj = threadIdx.x & 7;
            int r = fbr * 16 + bi * 2, c = fbc * 16 + bj * 2;
            BlockParams b{0, 0, 0, 0};
            if (idx >= 0 && r < h.mi_rows && c < h.mi_cols) {
                const uint8_t* sk = F.g.skip;
                int mc = h.mi_cols;
                bool skip = sk[r * mc + c] && (r + 1 >= h.mi_rows || sk[(r + 1) * mc + c]) &&
                            (c + 1 >= mc || sk[r * mc + c + 1]) &&
                            (r + 1 >= h.mi_rows || c + 1 >= mc || sk[(r + 1) * mc + c + 1]);
                if (!skip) {
                    int yd, var;
                    direction(&win[0][(H2 + bi * 8) * WP + H2 + bj * 8], cs, &yd, &var);
                    b.active = 1;
                    b.ydir = (int8_t)yd;
                    b.var = var;
                }
            }
            bp[threadIdx.x] = b;
        }
        __syncthreads();
        int pri_y = 0, sec_y = 0, pri_uv = 0, sec_uv = 0;
        if (idx >= 0) {
            pri_y = h.cdef_y_pri[idx] << cs;
            sec_y = h.cdef_y_sec[idx] << cs;
            pri_uv = h.cdef_uv_pri[idx] << cs;
            sec_uv = h.cdef_uv_sec[idx] << cs;
        }
        for (int p = 0; p < np; p++) {
            int px = p ? ssx : 0, py = p ? ssy : 0;
            int bw = FB >> px, bh = FB >> py;
            int x0 = (fbc * FB) >> px, y0 = (fbr * FB) >> py;
            const PlaneDev& D = F.cdef[p];
            const int dh = min(D.h, F.deb[p].h), dw = min(D.w, F.deb[p].w);
            const int16_t* W = win[p];
            int damping = h.cdef_damping + cs - (p ? 1 : 0);
            for (int i = threadIdx.x; i < bw * bh; i += blockDim.x) {
                int r = i / bw, c = i % bw;
                int gy = y0 + r, gx = x0 + c;
                if (gy >= dh || gx >= dw) continue;
                int xv = W[(r + H2) * WP + c + H2];
                const BlockParams b = bp[(r >> (3 - py)) * 8 + (c >> (3 - px))];
                int out = xv;
                if (b.active) {
                    int pri, sec, dir;
                    if (p == 0) {
                        int vs = (b.var >> 6) > 0 ? min(floor_log2u((unsigned)(b.var >> 6)), 12) : 0;
                        pri = b.var != 0 ? (pri_y * (4 + vs) + 8) >> 4 : 0;
                        sec = sec_y;
                        dir = pri_y == 0 ? 0 : b.ydir;
                    } else {
                        pri = pri_uv;
                        sec = sec_uv;
                        dir = pri_uv == 0 ? 0 : c_uv_dir[ssx][ssy][b.ydir];
                    }
                    int prow = (pri >> cs) & 1;
                    int pt0 = prow ? 3 : 4, pt1 = prow ? 3 : 2;
                    int padj = pri ? max(damping - floor_log2u((unsigned)pri), 0) : 0;
                    int sadj = sec ? max(damping - floor_log2u((unsigned)sec), 0) : 0;
                    int sum = 0, mx = xv, mn = xv;
#pragma unroll
                    for (int k = 0; k < 2; k++) {
#pragma unroll
                        for (int sg = -1; sg <= 1; sg += 2) {
#pragma unroll
                            for (int tt = 0; tt < 3; tt++) {
                                int d = tt == 0 ? dir : ((dir + (tt == 1 ? -2 : 2)) & 7);
                                int yy = r + H2 + sg * c_cdef_dirs[d][k][0];
                                int xx = c + H2 + sg * c_cdef_dirs[d][k][1];
                                int v = W[yy * WP + xx];
                                if (v == NA) continue;
                                if (tt == 0) {
                                    if (pri) sum += (k ? pt1 : pt0) * constrain_adj(v - xv, pri, padj);
                                } else {
                                    if (sec) sum += (k ? 1 : 2) * constrain_adj(v - xv, sec, sadj);
                                }
                                mx = max(mx, v);
                                mn = min(mn, v);
                            }
                        }
                    }
                    out = clip3(mn, mx, xv + ((8 + sum - (sum < 0)) >> 4));
                }
                st_px(D, hbd, gy, gx, out);
            }
        }
    }
}

}  // namespace

int tiles_cdef(const FrameDev& f) { return ((f.h.mi_rows + 15) >> 4) * ((f.h.mi_cols + 15) >> 4); }

void launch_cdef(const FrameDev* frames, const int32_t* starts, int n, int total, cudaStream_t s) {
    if (total <= 0) return;
    int grid = total < kSMs * 4 ? total : kSMs * 4;
    cdef_kernel<<<grid, 256, 0, s>>>(frames, starts, n, total);
}

}  // namespace av1g
