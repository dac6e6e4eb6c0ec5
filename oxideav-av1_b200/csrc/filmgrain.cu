// filmgrain.cu — §7.18.3 film grain synthesis.
//
// Replaces film_grain_synthesis / generate_grain / scaling_lookup_init /
// add_noise_synthesis (src/film_grain.rs:100-873) as called at
// frame_driver.rs:1060-1096.
//
// Two kernels:
//  * grain_template_kernel — one CTA per frame builds the 82x73 luma and the
//    chroma grain templates, the three scaling LUTs and the per-stripe random
//    block offsets into a per-frame scratch area.  The reference draws the
//    white noise from one 16-bit LFSR in raster order; the LFSR is linear over
//    GF(2), so the state at the start of row y is M^(W*y) applied to the seed
//    and every row is generated by its own thread after a jump of at most
//    seven precomputed matrix-vector products.  The auto-regressive filter
//    (lag <= 3) reads only earlier rows and earlier samples of the same row,
//    so samples with equal x + 4y are independent and one warp sweeps the
//    template in ~350 wavefront steps.
//  * grain_blend_kernel — every thread owns one chroma-resolution position
//    and the (1 << ssx) x (1 << ssy) luma samples it covers.  The noise value
//    of a sample is evaluated in closed form from the template, the random
//    offsets of the (at most two) 32-sample blocks that wrote it in each
//    direction and the 27/17, 17/27 and 23/22 overlap blends, which is exactly
//    what the reference's materialised noise stripes and noise image hold
//    (film_grain.rs:599-760).  Chroma is blended first from the un-noised
//    luma, then luma, as the reference orders it (film_grain.rs:758-828).
#include "common.cuh"
#include "av1_spec_tables.h"

namespace av1g {

__constant__ AV1T_GAUSSIAN_SEQUENCE_TYPE c_gauss AV1T_GAUSSIAN_SEQUENCE_DIMS = AV1T_GAUSSIAN_SEQUENCE_INIT;

namespace {

constexpr int LW = 82, LH = 73;

// ---- LFSR jump tables: M^(w * 2^b) for row widths 82 and 44 ---------------
struct Jumps {
    uint16_t m[2][7][16];  // [width 82 / 44][bit][column]
};

constexpr uint16_t mat_apply(const uint16_t* cols, uint16_t v) {
    uint16_t r = 0;
    for (int k = 0; k < 16; k++)
        if ((v >> k) & 1) r ^= cols[k];
    return r;
}

constexpr uint16_t lfsr_step(uint16_t r) {
    unsigned bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1;
    return (uint16_t)((r >> 1) | (bit << 15));
}

constexpr Jumps make_jumps() {
    Jumps j{};
    const int widths[2] = {LW, 44};
    for (int wi = 0; wi < 2; wi++) {
        // M^w by stepping each basis vector w times
        for (int k = 0; k < 16; k++) {
            uint16_t v = (uint16_t)(1u << k);
            for (int s = 0; s < widths[wi]; s++) v = lfsr_step(v);
            j.m[wi][0][k] = v;
        }
        for (int b = 1; b < 7; b++)
            for (int k = 0; k < 16; k++)
                j.m[wi][b][k] = mat_apply(j.m[wi][b - 1], j.m[wi][b - 1][k]);
    }
    return j;
}

__constant__ Jumps c_jumps = make_jumps();

__device__ __forceinline__ uint16_t row_state(uint16_t seed, int row, int wi) {
    uint16_t s = seed;
    for (int b = 0; b < 7; b++)
        if ((row >> b) & 1) s = mat_apply(c_jumps.m[wi][b], s);
    return s;
}

__device__ __forceinline__ int r2(int x, int n) { return n ? (x + (1 << (n - 1))) >> n : x; }

// scaling_lookup_fill (film_grain.rs:490-540)
__device__ void scaling_fill(uint8_t* t, int np, const uint8_t* xv, const uint8_t* yv) {
    if (np == 0) {
        for (int v = 0; v < 256; v++) t[v] = 0;
        return;
    }
    for (int v = 0; v < xv[0]; v++) t[v] = yv[0];
    for (int i = 0; i + 1 < np; i++) {
        int dx = xv[i + 1] - xv[i], dy = yv[i + 1] - yv[i];
        if (dx <= 0) continue;
        int delta = dy * ((65536 + (dx >> 1)) / dx);
        for (int x = 0; x < dx; x++) {
            int idx = xv[i] + x;
            if (idx < 256) t[idx] = (uint8_t)clip3(0, 255, yv[i] + ((x * delta + 32768) >> 16));
        }
    }
    for (int v = xv[np - 1]; v < 256; v++) t[v] = yv[np - 1];
}

// AR filter of one template by one warp: wavefront over t = x + 4y, the
// coefficients (minus 128) held in registers.
template <int LAG>
__device__ void ar_luma(int16_t* L, const av1g_film_grain& fg, int gmin, int gmax) {
    constexpr int NC = 2 * LAG * (LAG + 1);
    int c[NC > 0 ? NC : 1];
#pragma unroll
    for (int i = 0; i < NC; i++) c[i] = fg.ar_coeffs_y_plus_128[i] - 128;
    const int shift = fg.ar_coeff_shift, lane = threadIdx.x & 31;
    for (int T = 3 + 4 * 3; T <= (LW - 4) + 4 * (LH - 1); T++) {
        const int ylo = max(3, (T - (LW - 4) + 3) >> 2), yhi = min(LH - 1, (T - 3) >> 2);
        const int y = ylo + lane;
        if (y <= yhi) {
            const int x = T - 4 * y;
            int s = 0;
#pragma unroll
            for (int dr = -LAG; dr <= 0; dr++)
#pragma unroll
                for (int dc = -LAG; dc <= LAG; dc++) {
                    const int pos = (dr + LAG) * (2 * LAG + 1) + dc + LAG;
                    if (pos < NC) s += L[(y + dr) * LW + x + dc] * c[pos];
                }
            L[y * LW + x] = (int16_t)clip3(gmin, gmax, L[y * LW + x] + r2(s, shift));
        }
        __syncwarp();
    }
}

template <int LAG>
__device__ void ar_chroma(int16_t* C, const int16_t* L, const uint8_t* coef, const av1g_film_grain& fg, int cw,
                          int ch, int ssx, int ssy, int gmin, int gmax) {
    constexpr int NC = 2 * LAG * (LAG + 1);  // the last coefficient weighs the co-located luma
    int c[NC + 1];
#pragma unroll
    for (int i = 0; i <= NC; i++) c[i] = coef[i] - 128;
    const bool luma = fg.num_y_points > 0;
    const int shift = fg.ar_coeff_shift, lane = threadIdx.x & 31;
    for (int T = 3 + 4 * 3; T <= (cw - 4) + 4 * (ch - 1); T++) {
        const int ylo = max(3, (T - (cw - 4) + 3) >> 2), yhi = min(ch - 1, (T - 3) >> 2);
        for (int y = ylo + lane; y <= yhi; y += 32) {
            const int x = T - 4 * y;
            int s = 0;
#pragma unroll
            for (int dr = -LAG; dr <= 0; dr++)
#pragma unroll
                for (int dc = -LAG; dc <= LAG; dc++) {
                    const int pos = (dr + LAG) * (2 * LAG + 1) + dc + LAG;
                    if (pos < NC) s += C[(y + dr) * cw + x + dc] * c[pos];
                }
            if (luma) {
                const int lx = ((x - 3) << ssx) + 3, ly = ((y - 3) << ssy) + 3;
                int l = 0;
                for (int i = 0; i <= ssy; i++)
                    for (int j = 0; j <= ssx; j++) l += L[(ly + i) * LW + lx + j];
                s += r2(l, ssx + ssy) * c[NC];
            }
            C[y * cw + x] = (int16_t)clip3(gmin, gmax, C[y * cw + x] + r2(s, shift));
        }
        __syncwarp();
    }
}

__global__ void __launch_bounds__(128) grain_template_kernel(const FrameDev* __restrict__ frames,
                                                             const int32_t* __restrict__ starts, int n, int total) {
    __shared__ int16_t T[3][LH * LW];
    __shared__ int16_t gauss[2048];  // the lanes draw different entries: shared, not constant, memory
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) gauss[i] = (int16_t)c_gauss[i];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        int f = find_frame(starts, n, t);
        const FrameDev& F = frames[f];
        const av1g_film_grain& fg = F.h.film_grain;
        const int bd = F.h.bit_depth, ssx = F.h.subsampling_x, ssy = F.h.subsampling_y;
        const int center = 128 << (bd - 8), gmin = -center, gmax = (256 << (bd - 8)) - 1 - center;
        const int shift = 12 - bd + fg.grain_scale_shift;
        const int cw = ssx ? 44 : 82, ch = ssy ? 38 : 73;
        __syncthreads();
        if (threadIdx.x < 3) {
            int p = threadIdx.x;
            uint8_t* lut = F.grain_lut + p * 256;
            if (p < F.h.num_planes) {
                if (p == 0 || fg.chroma_scaling_from_luma) scaling_fill(lut, fg.num_y_points, fg.point_y_value, fg.point_y_scaling);
                else if (p == 1) scaling_fill(lut, fg.num_cb_points, fg.point_cb_value, fg.point_cb_scaling);
                else scaling_fill(lut, fg.num_cr_points, fg.point_cr_value, fg.point_cr_scaling);
            } else {
                for (int v = 0; v < 256; v++) lut[v] = 0;
            }
        }
        // white noise (generate_grain, film_grain.rs:245-300)
        for (int job = threadIdx.x; job < LH + 2 * ch; job += blockDim.x) {
            int p = job < LH ? 0 : (job < LH + ch ? 1 : 2);
            int y = p == 0 ? job : (p == 1 ? job - LH : job - LH - ch);
            int w = p == 0 ? LW : cw;
            bool on = p == 0 ? fg.num_y_points > 0
                             : (p == 1 ? (fg.num_cb_points > 0 || fg.chroma_scaling_from_luma)
                                       : (fg.num_cr_points > 0 || fg.chroma_scaling_from_luma));
            uint16_t seed = p == 0 ? fg.grain_seed : (uint16_t)(fg.grain_seed ^ (p == 1 ? 0xb524 : 0x49d8));
            uint16_t s = on ? row_state(seed, y, (p == 0 || cw == LW) ? 0 : 1) : 0;
            int16_t* row = &T[p][y * w];
            for (int x = 0; x < w; x++) {
                int g = 0;
                if (on) {
                    s = lfsr_step(s);
                    g = gauss[(s >> 5) & 2047];
                }
                row[x] = (int16_t)r2(g, shift);
            }
        }
        __syncthreads();
        if (fg.num_y_points > 0 && threadIdx.x < 32) {
            switch (fg.ar_coeff_lag) {
                case 0: ar_luma<0>(T[0], fg, gmin, gmax); break;
                case 1: ar_luma<1>(T[0], fg, gmin, gmax); break;
                case 2: ar_luma<2>(T[0], fg, gmin, gmax); break;
                default: ar_luma<3>(T[0], fg, gmin, gmax); break;
            }
        }
        __syncthreads();
        if (fg.chroma_scaling_from_luma || fg.num_cb_points > 0 || fg.num_cr_points > 0) {
            int warp = threadIdx.x >> 5;
            if (warp < 2) {
                int16_t* C = T[1 + warp];
                const uint8_t* cf = warp == 0 ? fg.ar_coeffs_cb_plus_128 : fg.ar_coeffs_cr_plus_128;
                switch (fg.ar_coeff_lag) {
                    case 0: ar_chroma<0>(C, T[0], cf, fg, cw, ch, ssx, ssy, gmin, gmax); break;
                    case 1: ar_chroma<1>(C, T[0], cf, fg, cw, ch, ssx, ssy, gmin, gmax); break;
                    case 2: ar_chroma<2>(C, T[0], cf, fg, cw, ch, ssx, ssy, gmin, gmax); break;
                    default: ar_chroma<3>(C, T[0], cf, fg, cw, ch, ssx, ssy, gmin, gmax); break;
                }
            }
        }
        __syncthreads();
        int16_t* out = F.grain_tmpl;
        for (int i = threadIdx.x; i < LH * LW; i += blockDim.x) out[i] = T[0][i];
        for (int i = threadIdx.x; i < ch * cw; i += blockDim.x) {
            out[LH * LW + i] = T[1][i];
            out[2 * LH * LW + i] = T[2][i];
        }
        // per-stripe block offsets (add_noise_synthesis, film_grain.rs:604-615)
        const int w = F.out[0].w, h = F.out[0].h;
        const int nstripes = ((h + 1) / 2 + 15) / 16, nblocks = F.grain_nblocks;
        for (int s = threadIdx.x; s < nstripes; s += blockDim.x) {
            uint16_t st = fg.grain_seed;
            st ^= (uint16_t)((((unsigned)s * 37 + 178) & 255) << 8);
            st ^= (uint16_t)(((unsigned)s * 173 + 105) & 255);
            for (int k = 0; k < nblocks; k++) {
                st = lfsr_step(st);
                F.grain_offs[s * nblocks + k] = (uint8_t)(st >> 8);
            }
        }
        (void)w;
    }
}

// Noise of N adjacent samples of one plane, (y, x0 .. x0 + N - 1): the
// materialised noiseImage of the reference (film_grain.rs:599-760) in closed
// form.  x0 is a multiple of N and N divides the 16- or 32-sample noise block,
// so the group lies in one block: one offset lookup serves all N samples.
template <int N>
struct Noise {
    const int16_t* tmpl;
    const uint8_t* offs;
    int nblocks, tw;  // blocks per stripe, template row width
    int psx, psy, overlap, gmin, gmax;

    __device__ __forceinline__ const int16_t* block_row(int s, int k, int i) const {
        const int o = offs[s * nblocks + k];
        const int ox = o >> 4, oy = o & 15;
        const int pox = psx ? 6 + ox : 9 + ox * 2, poy = psy ? 6 + oy : 9 + oy * 2;
        return tmpl + (poy + i) * tw + pox;
    }
    // noise stripe s, row i, after the horizontal overlap blend
    __device__ __forceinline__ void stripe(int s, int i, int x0, int (&v)[N]) const {
        const int bs = psx ? 4 : 5;
        const int k = x0 >> bs, j0 = x0 & ((1 << bs) - 1);
        const int16_t* row = block_row(s, k, i) + j0;
#pragma unroll
        for (int e = 0; e < N; e++) v[e] = __ldg(row + e);
        if (overlap && k > 0 && j0 == 0) {
            const int16_t* old = block_row(s, k - 1, i);
            if (psx == 0) {  // columns 0 and 1 blend with columns 32 and 33 of the left block
                v[0] = clip3(gmin, gmax, r2(__ldg(old + 32) * 27 + v[0] * 17, 5));
                if (N > 1) v[1] = clip3(gmin, gmax, r2(__ldg(old + 33) * 17 + v[1] * 27, 5));
            } else {  // column 0 blends with column 16 of the left block
                v[0] = clip3(gmin, gmax, r2(__ldg(old + 16) * 23 + v[0] * 22, 5));
            }
        }
    }
    __device__ __forceinline__ void noise(int y, int x0, int (&v)[N]) const {
        const int bs = psy ? 4 : 5;
        const int s = y >> bs, i = y & ((1 << bs) - 1);
        stripe(s, i, x0, v);
        if (overlap && s > 0 && (psy ? i == 0 : i < 2)) {
            int old[N];
            stripe(s - 1, psy ? 16 : i + 32, x0, old);
#pragma unroll
            for (int e = 0; e < N; e++) {
                const int m = psy ? old[e] * 23 + v[e] * 22 : (i == 0 ? old[e] * 27 + v[e] * 17 : old[e] * 17 + v[e] * 27);
                v[e] = clip3(gmin, gmax, r2(m, 5));
            }
        }
    }
};

__device__ __forceinline__ int scale_lut(const uint8_t* lut, int index, int bd) {
    int shift = bd - 8, x = index >> shift;
    if (bd == 8 || x >= 255) return lut[x < 255 ? x : 255];
    int rem = index - (x << shift);
    int a = lut[x], b = lut[x + 1];
    return a + r2((b - a) * rem, shift);
}

// N samples of a row at x0: one vector access when the group is whole and the
// row keeps it aligned, else sample by sample (x < w only).
template <int N>
__device__ __forceinline__ void ld_n(const PlaneDev& P, int hbd, int y, int x0, int w, int (&v)[N]) {
    const uint8_t* row = P.p + (size_t)y * P.stride;
    if (x0 + N <= w) {
        if (hbd) {
            if constexpr (N == 4) {
                const uint2 u = *reinterpret_cast<const uint2*>(reinterpret_cast<const uint16_t*>(row) + x0);
                v[0] = u.x & 0xffff; v[1] = u.x >> 16; v[2] = u.y & 0xffff; v[3] = u.y >> 16;
                return;
            } else if constexpr (N == 2) {
                const uint32_t u = *reinterpret_cast<const uint32_t*>(reinterpret_cast<const uint16_t*>(row) + x0);
                v[0] = u & 0xffff; v[1] = u >> 16;
                return;
            }
        } else {
            if constexpr (N == 4) {
                const uint32_t u = *reinterpret_cast<const uint32_t*>(row + x0);
                v[0] = u & 0xff; v[1] = (u >> 8) & 0xff; v[2] = (u >> 16) & 0xff; v[3] = u >> 24;
                return;
            } else if constexpr (N == 2) {
                const uint16_t u = *reinterpret_cast<const uint16_t*>(row + x0);
                v[0] = u & 0xff; v[1] = u >> 8;
                return;
            }
        }
    }
#pragma unroll
    for (int e = 0; e < N; e++) v[e] = x0 + e < w ? ld_px(P, hbd, y, x0 + e) : 0;
}
template <int N>
__device__ __forceinline__ void st_n(const PlaneDev& P, int hbd, int y, int x0, int w, const int (&v)[N]) {
    uint8_t* row = P.p + (size_t)y * P.stride;
    if (x0 + N <= w) {
        if (hbd) {
            if constexpr (N == 4) {
                *reinterpret_cast<uint2*>(reinterpret_cast<uint16_t*>(row) + x0) =
                    make_uint2((uint32_t)v[0] | ((uint32_t)v[1] << 16), (uint32_t)v[2] | ((uint32_t)v[3] << 16));
                return;
            } else if constexpr (N == 2) {
                *reinterpret_cast<uint32_t*>(reinterpret_cast<uint16_t*>(row) + x0) =
                    (uint32_t)v[0] | ((uint32_t)v[1] << 16);
                return;
            }
        } else {
            if constexpr (N == 4) {
                *reinterpret_cast<uint32_t*>(row + x0) =
                    (uint32_t)v[0] | ((uint32_t)v[1] << 8) | ((uint32_t)v[2] << 16) | ((uint32_t)v[3] << 24);
                return;
            } else if constexpr (N == 2) {
                *reinterpret_cast<uint16_t*>(row + x0) = (uint16_t)(v[0] | (v[1] << 8));
                return;
            }
        }
    }
#pragma unroll
    for (int e = 0; e < N; e++)
        if (x0 + e < w) st_px(P, hbd, y, x0 + e, v[e]);
}

constexpr int BR = 8;      // chroma-resolution rows per tile
constexpr int QPT = 256;   // groups of 4 luma columns per tile (one per thread)

// One chroma-resolution row yc of a group: CQ = 4 >> ssx chroma samples of
// each chroma plane (blended from the un-noised luma first), then the
// 4 x (1 << ssy) luma samples they cover, as the reference orders it
// (film_grain.rs:758-828).
template <int CQ>
__device__ __forceinline__ void blend_group(const FrameDev& F, const av1g_film_grain& fg, const uint8_t (*lut)[256],
                                            int q, int yc, int gmin, int gmax, int minv, int maxl, int maxc) {
    const int bd = F.h.bit_depth, hbd = F.hbd;
    const int np = F.h.num_planes;
    const int ssx = np > 1 ? F.h.subsampling_x : 0, ssy = np > 1 ? F.h.subsampling_y : 0;
    const int w = F.out[0].w, h = F.out[0].h;
    const int gw = (w + ssx) >> ssx;
    const int x0 = q * 4, xc0 = q * CQ, ly = yc << ssy;
    if (np >= 3 && xc0 < gw) {
        const bool chroma = fg.num_cb_points > 0 || fg.num_cr_points > 0 || fg.chroma_scaling_from_luma;
        int avg[CQ];
        if (chroma) {
            int l[4];
            ld_n<4>(F.lr[0], hbd, ly, x0, w, l);
            if (ssx) {
                // average of the two luma columns, the right one clamped to the plane
#pragma unroll
                for (int c = 0; c < CQ; c++) {
                    const int bx = 2 * c + 1;
                    avg[c] = r2(l[2 * c] + (x0 + bx < w ? l[bx] : l[min(w - 1 - x0, 3)]), 1);
                }
            } else {
#pragma unroll
                for (int c = 0; c < CQ; c++) avg[c] = l[c];
            }
        }
        for (int p = 1; p <= 2; p++) {
            int orig[CQ];
            ld_n<CQ>(F.lr[p], hbd, yc, xc0, gw, orig);
            const int npts = p == 1 ? fg.num_cb_points : fg.num_cr_points;
            if (!(npts > 0 || fg.chroma_scaling_from_luma)) {
                st_n<CQ>(F.out[p], hbd, yc, xc0, gw, orig);
                continue;
            }
            const Noise<CQ> nc{F.grain_tmpl + p * LH * LW, F.grain_offs, F.grain_nblocks, F.h.subsampling_x ? 44 : 82,
                               F.h.subsampling_x, F.h.subsampling_y, fg.overlap_flag, gmin, gmax};
            int nz[CQ];
            nc.noise(yc, xc0, nz);
            const int lm = p == 1 ? fg.cb_luma_mult : fg.cr_luma_mult;
            const int m = p == 1 ? fg.cb_mult : fg.cr_mult;
            const int off = p == 1 ? fg.cb_offset : fg.cr_offset;
            int o[CQ];
#pragma unroll
            for (int c = 0; c < CQ; c++) {
                int merged;
                if (fg.chroma_scaling_from_luma) {
                    merged = avg[c];
                } else {
                    const int comb = avg[c] * (lm - 128) + orig[c] * (m - 128);
                    merged = clip3(0, (1 << bd) - 1, (comb >> 6) + (off - 256) * (1 << (bd - 8)));
                }
                o[c] = clip3(minv, maxc, orig[c] + r2(scale_lut(lut[p], merged, bd) * nz[c], fg.grain_scaling));
            }
            st_n<CQ>(F.out[p], hbd, yc, xc0, gw, o);
        }
    }
    if (x0 >= w) return;
    const Noise<4> nl{F.grain_tmpl, F.grain_offs, F.grain_nblocks, LW, 0, 0, fg.overlap_flag, gmin, gmax};
    for (int dy = 0; dy <= ssy; dy++) {
        const int y = ly + dy;
        if (y >= h) break;
        int orig[4];
        ld_n<4>(F.lr[0], hbd, y, x0, w, orig);
        if (fg.num_y_points > 0) {
            int nz[4];
            nl.noise(y, x0, nz);
#pragma unroll
            for (int e = 0; e < 4; e++)
                orig[e] = clip3(minv, maxl, orig[e] + r2(scale_lut(lut[0], orig[e], bd) * nz[e], fg.grain_scaling));
        }
        st_n<4>(F.out[0], hbd, y, x0, w, orig);
    }
}

__global__ void __launch_bounds__(256) grain_blend_kernel(const FrameDev* __restrict__ frames,
                                                          const int32_t* __restrict__ starts, int n, int total) {
    __shared__ uint8_t lut[3][256];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int f = find_frame(starts, n, t);
        const FrameDev& F = frames[f];
        const av1g_film_grain& fg = F.h.film_grain;
        const int bd = F.h.bit_depth;
        const int np = F.h.num_planes;
        const int ssx = np > 1 ? F.h.subsampling_x : 0, ssy = np > 1 ? F.h.subsampling_y : 0;
        const int w = F.out[0].w, h = F.out[0].h;
        const int gh = (h + ssy) >> ssy, nq = (w + 3) >> 2;
        const int ntc = (nq + QPT - 1) / QPT;
        const int local = t - starts[f];
        const int tr = local / ntc, tc = local % ntc;
        __syncthreads();  // the previous tile's LUTs are no longer read
        for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) lut[i >> 8][i & 255] = F.grain_lut[i];
        __syncthreads();
        const int q = tc * QPT + threadIdx.x;
        if (q >= nq) continue;
        const int center = 128 << (bd - 8), gmin = -center, gmax = (256 << (bd - 8)) - 1 - center;
        int minv, maxl, maxc;
        if (fg.clip_to_restricted_range) {
            minv = 16 << (bd - 8);
            maxl = 235 << (bd - 8);
            maxc = F.h.matrix_coefficients == 0 ? maxl : 240 << (bd - 8);
        } else {
            minv = 0;
            maxl = maxc = (256 << (bd - 8)) - 1;
        }
        for (int yc = tr * BR; yc < min(gh, tr * BR + BR); yc++) {
            if (ssx) blend_group<2>(F, fg, lut, q, yc, gmin, gmax, minv, maxl, maxc);
            else blend_group<4>(F, fg, lut, q, yc, gmin, gmax, minv, maxl, maxc);
        }
    }
}

}  // namespace

int tiles_grain_blend(const FrameDev& f) {
    int ssy = f.h.num_planes > 1 ? f.h.subsampling_y : 0;
    int gh = (f.out[0].h + ssy) >> ssy, nq = (f.out[0].w + 3) >> 2;
    return ((gh + BR - 1) / BR) * ((nq + QPT - 1) / QPT);
}

void launch_grain(const FrameDev* frames, const int32_t* starts_tmpl, const int32_t* starts_blend, int n,
                  int total_tmpl, int total_blend, const StageShape& sh, cudaStream_t s) {
    if (total_tmpl > 0) grain_template_kernel<<<total_tmpl, 128, 0, s>>>(frames, starts_tmpl, n, total_tmpl);
    if (total_blend > 0) grain_blend_kernel<<<shape_grid(sh, total_blend), 256, 0, s>>>(frames, starts_blend, n, total_blend);
}

}  // namespace av1g
