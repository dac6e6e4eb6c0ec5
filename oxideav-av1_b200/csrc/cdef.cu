// cdef.cu — §7.15 constrained directional enhancement filter.
//
// Replaces cdef_frame / cdef_block / cdef_direction / cdef_filter_block
// (src/cdef.rs:180-606) as driven by cdef_frame_from_idx (src/cdf.rs:20300).
// One CTA owns one 64x64 filter block (the cdef_idx granularity) across all
// planes.  It stages the deblocked samples of the block plus a 2-sample halo
// (the furthest tap of Cdef_Directions) for every plane in shared memory,
// marking samples outside the plane as unavailable (the reference's
// CdefAvailable == 0 arm, cdef.rs:564-590).
//
// Direction search (cdef.rs:366-456): eight threads per 8x8 luma block, one
// per direction, each accumulating its own partial-sum line set and cost;
// the block's direction is the arg-max over the eight lanes with the lowest
// index winning ties, exactly the reference's first-strictly-greater scan.
// Filtering (cdef.rs:465-590): one thread per sample with the block's
// primary / secondary tap offsets read from a per-direction table; tiles
// whose halo lies inside the plane take a path without availability tests.
// Samples of skipped blocks (cdef_idx == -1, or all four 4x4 cells skipped)
// are copied through, as cdef_block does (cdef.rs:229-262).
#include "common.cuh"

namespace av1g {

namespace {

constexpr int FB = 64, H2 = 2, WMAX = FB + 2 * H2, WP = WMAX + 4;
constexpr int16_t NA = -32768;

__constant__ int8_t c_cdef_dirs[8][2][2] = {
    {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
    {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}}};
__constant__ int8_t c_uv_dir[2][2][8] = {{{0, 1, 2, 3, 4, 5, 6, 7}, {1, 2, 2, 2, 3, 4, 6, 0}},
                                         {{7, 0, 2, 4, 5, 6, 6, 6}, {0, 1, 2, 3, 4, 5, 6, 7}}};

struct BlockParams {
    int8_t active;  // 0: copy through
    int8_t ydir;
    int8_t uvdir;
    int8_t pad;
    int32_t pri_y;  // variance-scaled luma primary strength
};

// Cost of direction D over an 8x8 block (cdef.rs:366-440), bins fixed at compile time.
template <int D>
__device__ __forceinline__ int dir_cost(const int16_t* w, int shift) {
    constexpr int NB = (D == 2 || D == 6) ? 8 : ((D & 1) ? 11 : 15);
    int p[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) p[k] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) {
            int x = (w[i * WP + j] >> shift) - 128;
            int b = D == 0 ? i + j : D == 1 ? i + j / 2 : D == 2 ? i : D == 3 ? 3 + i - j / 2
                  : D == 4 ? 7 + i - j : D == 5 ? 3 - i / 2 + j : D == 6 ? j : i / 2 + j;
            p[b] += x;
        }
    int cost = 0;
    if (D == 2 || D == 6) {
#pragma unroll
        for (int k = 0; k < 8; k++) cost += p[k] * p[k];
        cost *= 105;
    } else if (D == 0 || D == 4) {
        constexpr int div[8] = {840, 420, 280, 210, 168, 140, 120, 105};
#pragma unroll
        for (int k = 0; k < 7; k++) cost += (p[k] * p[k] + p[14 - k] * p[14 - k]) * div[k];
        cost += p[7] * p[7] * 105;
    } else {
        constexpr int div2[3] = {420, 210, 140};
#pragma unroll
        for (int k = 0; k < 5; k++) cost += p[3 + k] * p[3 + k];
        cost *= 105;
#pragma unroll
        for (int k = 0; k < 3; k++) cost += (p[k] * p[k] + p[10 - k] * p[10 - k]) * div2[k];
    }
    return cost;
}

__device__ __forceinline__ int constrain_adj(int diff, int threshold, int adj) {
    // constrain (cdef.rs:592-606) with dampingAdj precomputed
    int ad = abs(diff);
    int v = min(ad, max(threshold - (ad >> adj), 0));
    return diff < 0 ? -v : v;
}

template <bool BORDER>
__device__ __forceinline__ int filter_px(const int16_t* c, int xv, const int16_t* toff, int dir, int pri, int sec,
                                         int padj, int sadj, int pt0, int pt1) {
    int sum = 0, mx = xv, mn = xv;
    const int d2a = (dir + 2) & 7, d2b = (dir + 6) & 7;
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const int op = toff[dir * 2 + k], oa = toff[d2a * 2 + k], ob = toff[d2b * 2 + k];
        const int v[6] = {c[op], c[-op], c[oa], c[-oa], c[ob], c[-ob]};
#pragma unroll
        for (int t = 0; t < 6; t++) {
            int x = v[t];
            if (BORDER && x == NA) continue;
            if (t < 2) sum += (k ? pt1 : pt0) * constrain_adj(x - xv, pri, padj);
            else sum += (k ? 1 : 2) * constrain_adj(x - xv, sec, sadj);
            mx = max(mx, x);
            mn = min(mn, x);
        }
    }
    return clip3(mn, mx, xv + ((8 + sum - (sum < 0)) >> 4));
}

__global__ void __launch_bounds__(256, 3) cdef_kernel(const FrameDev* __restrict__ frames,
                                                      const int32_t* __restrict__ starts, int n, int total) {
    __shared__ int16_t win[3][WMAX * WP];
    __shared__ BlockParams bp[64];
    __shared__ int16_t toff[16];
    if (threadIdx.x < 16) toff[threadIdx.x] = c_cdef_dirs[threadIdx.x >> 1][threadIdx.x & 1][0] * WP +
                                              c_cdef_dirs[threadIdx.x >> 1][threadIdx.x & 1][1];
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
        const int lx0 = fbc * FB, ly0 = fbr * FB;
        const bool border = lx0 < H2 || ly0 < H2 || lx0 + FB + H2 > F.deb[0].w || ly0 + FB + H2 > F.deb[0].h;
        __syncthreads();
        for (int p = 0; p < np; p++) {
            int px = p ? ssx : 0, py = p ? ssy : 0;
            int bw = FB >> px, bh = FB >> py;
            int x0 = lx0 >> px, y0 = ly0 >> py;
            const PlaneDev& S = F.deb[p];
            int ww = bw + 2 * H2, wh = bh + 2 * H2;
            for (int i = threadIdx.x; i < WMAX * wh; i += blockDim.x) {
                int r = i / WMAX, c = i - r * WMAX;
                if (c >= ww) continue;
                int gy = y0 - H2 + r, gx = x0 - H2 + c;
                win[p][r * WP + c] = (gy >= 0 && gy < S.h && gx >= 0 && gx < S.w) ? (int16_t)ld_px(S, hbd, gy, gx) : NA;
            }
        }
        __syncthreads();
        // direction search: 8 lanes per block, 32 blocks per pass
        for (int b0 = 0; b0 < 64; b0 += 32) {
            int blk = b0 + (threadIdx.x >> 3), d = threadIdx.x & 7;
            int bi = blk >> 3, bj = blk & 7;
            int r = fbr * 16 + bi * 2, c = fbc * 16 + bj * 2;
            bool live = idx >= 0 && r < h.mi_rows && c < h.mi_cols;
            bool skip = true;
            if (live) {
                const uint8_t* sk = F.g.skip;
                int mc = h.mi_cols;
                skip = sk[r * mc + c] && (r + 1 >= h.mi_rows || sk[(r + 1) * mc + c]) &&
                       (c + 1 >= mc || sk[r * mc + c + 1]) &&
                       (r + 1 >= h.mi_rows || c + 1 >= mc || sk[(r + 1) * mc + c + 1]);
            }
            int cost = 0;
            if (live && !skip) {
                const int16_t* w = &win[0][(H2 + bi * 8) * WP + H2 + bj * 8];
                switch (d) {
                    case 0: cost = dir_cost<0>(w, cs); break;
                    case 1: cost = dir_cost<1>(w, cs); break;
                    case 2: cost = dir_cost<2>(w, cs); break;
                    case 3: cost = dir_cost<3>(w, cs); break;
                    case 4: cost = dir_cost<4>(w, cs); break;
                    case 5: cost = dir_cost<5>(w, cs); break;
                    case 6: cost = dir_cost<6>(w, cs); break;
                    default: cost = dir_cost<7>(w, cs); break;
                }
            }
            int best = cost, bd = d;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                int oc = __shfl_xor_sync(0xffffffff, best, o, 8);
                int od = __shfl_xor_sync(0xffffffff, bd, o, 8);
                if (oc > best || (oc == best && od < bd)) { best = oc; bd = od; }
            }
            int opp = __shfl_sync(0xffffffff, cost, (threadIdx.x & ~7) | ((bd + 4) & 7), 32);
            if (d == 0) {
                BlockParams b{0, 0, 0, 0, 0};
                if (live && !skip) {
                    int var = (best - opp) >> 10;
                    int pri_y = h.cdef_y_pri[idx] << cs;
                    int vs = (var >> 6) > 0 ? min(floor_log2u((unsigned)(var >> 6)), 12) : 0;
                    b.active = 1;
                    b.pri_y = var != 0 ? (pri_y * (4 + vs) + 8) >> 4 : 0;
                    b.ydir = (int8_t)(pri_y == 0 ? 0 : bd);
                    int pri_uv = h.cdef_uv_pri[idx] << cs;
                    b.uvdir = (int8_t)(pri_uv == 0 ? 0 : c_uv_dir[ssx][ssy][bd]);
                }
                bp[blk] = b;
            }
        }
        __syncthreads();
        const int sec_y = idx >= 0 ? h.cdef_y_sec[idx] << cs : 0;
        const int pri_uv = idx >= 0 ? h.cdef_uv_pri[idx] << cs : 0;
        const int sec_uv = idx >= 0 ? h.cdef_uv_sec[idx] << cs : 0;
        for (int p = 0; p < np; p++) {
            int px = p ? ssx : 0, py = p ? ssy : 0;
            int bw = FB >> px, bh = FB >> py;
            int x0 = lx0 >> px, y0 = ly0 >> py;
            const PlaneDev& D = F.cdef[p];
            const int dh = min(D.h, F.deb[p].h), dw = min(D.w, F.deb[p].w);
            const int16_t* W = win[p];
            const int damping = h.cdef_damping + cs - (p ? 1 : 0);
            const int sadj = (p ? sec_uv : sec_y) ? max(damping - floor_log2u((unsigned)(p ? sec_uv : sec_y)), 0) : 0;
            const int sec = p ? sec_uv : sec_y;
            const int lbw = 6 - px;  // log2 of the block width in this plane
            for (int i = threadIdx.x; i < bw * bh; i += blockDim.x) {
                int r = i >> lbw, c = i & (bw - 1);
                int gy = y0 + r, gx = x0 + c;
                if (gy >= dh || gx >= dw) continue;
                const int16_t* cp = W + (r + H2) * WP + c + H2;
                int xv = *cp;
                const BlockParams b = bp[(r >> (3 - py)) * 8 + (c >> (3 - px))];
                int out = xv;
                if (b.active) {
                    int pri = p ? pri_uv : b.pri_y;
                    int dir = p ? b.uvdir : b.ydir;
                    int prow = (pri >> cs) & 1;
                    int padj = pri ? max(damping - floor_log2u((unsigned)pri), 0) : 0;
                    out = border ? filter_px<true>(cp, xv, toff, dir, pri, sec, padj, sadj, prow ? 3 : 4, prow ? 3 : 2)
                                 : filter_px<false>(cp, xv, toff, dir, pri, sec, padj, sadj, prow ? 3 : 4, prow ? 3 : 2);
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
    int grid = total < kSMs * 6 ? total : kSMs * 6;
    cdef_kernel<<<grid, 256, 0, s>>>(frames, starts, n, total);
}

}  // namespace av1g
