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
// Direction search (cdef.rs:366-456): one thread per (8x8 luma block,
// direction), laid out so that every warp evaluates a single direction for
// 32 blocks (the cost's bin pattern is fixed at compile time per direction,
// so a warp never diverges); the block's direction is then the arg-max over
// the eight costs with the lowest index winning ties, exactly the reference's
// first-strictly-greater scan.
// Filtering (cdef.rs:465-590): one thread per sample with the block's
// primary / secondary tap offsets read from a per-direction table; tiles
// whose halo lies inside the plane take a path without availability tests.
// Samples of skipped blocks (cdef_idx == -1, or all four 4x4 cells skipped)
// are copied through, as cdef_block does (cdef.rs:229-262).
//
// 8- and 10-bit frames filter two horizontally adjacent samples per thread in
// packed half-precision registers, so each add / fma / min / max serves both
// samples.  The window holds 1024 + v as half-precision bits (0x6400 | v;
// unavailable samples are NaN), every difference, threshold, weighted sum
// and clip bound is an integer below 2048 (exact in half precision), and the
// two roundings the reference asks for — floor(|d| >> damping) inside
// constrain and the (8 + sum - (sum < 0)) >> 4 of the tap sum — are each one
// round-to-nearest addition of 1536 to an exactly computed value whose
// fraction cannot be a tie.  The maximum with zero that ends constrain turns
// a NaN (unavailable) tap into a zero contribution and the clip range's min
// / max skip NaNs, which is the reference's CdefAvailable == 0 arm.  A warp
// filters 64 consecutive samples of a row (8 luma blocks, each with its own
// direction); in interior tiles a luma tap is one aligned 32-bit load from
// the window or from a copy of it shifted by one sample (per-block byte
// offsets), elsewhere two aligned words and a byte permute.  12-bit frames
// keep the 32-bit integer path (their sums pass 2048).
#include <cuda_fp16.h>

#include "common.cuh"

namespace av1g {

namespace {

constexpr int FB = 64, H2 = 2, WMAX = FB + 2 * H2, WP = WMAX + 4;
constexpr int kCdefThreads = 256;  // cdef_kernel's CTA size
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
    int8_t padj_y;  // primary damping shift of pri_y
    int32_t pri_y;  // variance-scaled luma primary strength
    uint16_t htb, hk, hc;  // half-precision constants of pri_y (HalfStrength, one lane)
    uint16_t pad;
};

// Cost of direction D over an 8x8 block (cdef.rs:366-440), bins fixed at
// compile time.  blk: the block's 64 samples, row-major, already shifted to
// 8 bits and centred ((v >> (bitDepth - 8)) - 128), 8-byte aligned.
template <int D>
__device__ __forceinline__ int dir_cost(const int16_t* blk) {
    constexpr int NB = (D == 2 || D == 6) ? 8 : ((D & 1) ? 11 : 15);
    int p[NB];
#pragma unroll
    for (int k = 0; k < NB; k++) p[k] = 0;
    const uint2* q = reinterpret_cast<const uint2*>(blk);
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int hh = 0; hh < 2; hh++) {
            const uint2 w = q[i * 2 + hh];
            const int xs[4] = {(int)(int16_t)(w.x & 0xffffu), (int)w.x >> 16, (int)(int16_t)(w.y & 0xffffu),
                               (int)w.y >> 16};
#pragma unroll
            for (int e = 0; e < 4; e++) {
                const int j = hh * 4 + e;
                const int b = D == 0 ? i + j : D == 1 ? i + j / 2 : D == 2 ? i : D == 3 ? 3 + i - j / 2
                            : D == 4 ? 7 + i - j : D == 5 ? 3 - i / 2 + j : D == 6 ? j : i / 2 + j;
                p[b] += xs[e];
            }
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
    // constrain (cdef.rs:592-606) with dampingAdj precomputed:
    // min(|d|, max(t - (|d| >> adj), 0)) == max(min(|d|, t - (|d| >> adj)), 0) as |d| >= 0
    int ad = abs(diff);
    int v = __vimin_s32_relu(ad, threshold - (ad >> adj));
    return diff < 0 ? -v : v;
}

// Tap offsets of one direction: primary (k = 0, 1), then the two secondary
// directions (dir + 2, dir - 2) for k = 0, 1.
struct Taps {
    int p0, p1, a0, a1, b0, b1;
};

__device__ __forceinline__ Taps taps_of(const int16_t* toff, int dir) {
    const int da = (dir + 2) & 7, db = (dir + 6) & 7;
    return Taps{toff[dir * 2], toff[dir * 2 + 1], toff[da * 2], toff[da * 2 + 1], toff[db * 2], toff[db * 2 + 1]};
}

// One tap pair (+o and -o) of weight w: constrain (cdef.rs:592-606) with the
// damping shift precomputed, accumulated into sum; with MINMAX, min / max of
// the samples taken (the reference's clip range, cdef.rs:540-560).
template <bool BORDER, bool MINMAX>
__device__ __forceinline__ void tap2(const int16_t* c, int o, int xv, int w, int thr, int adj, int& sum, int& mn,
                                     int& mx) {
    if (!BORDER) {  // both taps available: one weight product, three-input min / max
        const int x0 = c[o], x1 = c[-o];
        sum += w * (constrain_adj(x0 - xv, thr, adj) + constrain_adj(x1 - xv, thr, adj));
        if (MINMAX) {
            mx = __vimax3_s32(mx, x0, x1);
            mn = __vimin3_s32(mn, x0, x1);
        }
        return;
    }
#pragma unroll
    for (int s = 0; s < 2; s++) {
        const int x = s ? c[-o] : c[o];
        if (x == NA) continue;
        sum += w * constrain_adj(x - xv, thr, adj);
        if (MINMAX) {
            mx = max(mx, x);
            mn = min(mn, x);
        }
    }
}

// One sample of cdef_filter (cdef.rs:465-590).  MODE 3: primary and
// secondary taps, clipped to the taps' range as the reference always does.
// MODE 1 / 2: only the primary / only the secondary strength is non-zero;
// the taps of a zero strength add nothing (constrain with threshold 0 is 0)
// and the clip is the identity, so both are left out: the remaining taps'
// weights sum to 12 (2 x (4 + 2), 2 x (3 + 3), or 2 x 2 x (2 + 1)), each
// constrained difference has its tap's sign and at most its magnitude, so
// with D the largest positive difference sum <= 12 D and
// (8 + sum) >> 4 <= D (and symmetrically below): x + offset stays inside
// [min, max] of the taps, and the unclipped value is the clipped one.
template <bool BORDER, int MODE>
__device__ __forceinline__ int filter_px(const int16_t* c, int xv, const Taps& T, int pri, int sec, int padj,
                                         int sadj, int pt0, int pt1) {
    constexpr bool MM = MODE == 3;
    int sum = 0, mx = xv, mn = xv;
    if (MODE & 1) {
        tap2<BORDER, MM>(c, T.p0, xv, pt0, pri, padj, sum, mn, mx);
        tap2<BORDER, MM>(c, T.p1, xv, pt1, pri, padj, sum, mn, mx);
    }
    if (MODE & 2) {
        tap2<BORDER, MM>(c, T.a0, xv, 2, sec, sadj, sum, mn, mx);
        tap2<BORDER, MM>(c, T.b0, xv, 2, sec, sadj, sum, mn, mx);
        tap2<BORDER, MM>(c, T.a1, xv, 1, sec, sadj, sum, mn, mx);
        tap2<BORDER, MM>(c, T.b1, xv, 1, sec, sadj, sum, mn, mx);
    }
    const int y = xv + ((8 + sum - (sum < 0)) >> 4);
    return MM ? clip3(mn, mx, y) : y;
}

// ---- half-precision path (8- and 10-bit) ---------------------------------

constexpr uint16_t kHalfNA = 0x7E00;        // NaN: a tap outside the plane
constexpr uint32_t kH1536 = 0x66006600u;    // 1536, 1536
constexpr uint32_t kHNeg1 = 0xBC00BC00u;    // -1, -1
constexpr uint32_t kH1_16 = 0x2C002C00u;    // 1/16, 1/16
constexpr uint32_t kH1_32 = 0x28002800u;    // 1/32, 1/32
constexpr uint32_t kSign2 = 0x80008000u;

__device__ __forceinline__ __half2 u2h(uint32_t u) {
    __half2 h;
    memcpy(&h, &u, 4);
    return h;
}
__device__ __forceinline__ uint32_t h2u(__half2 h) {
    uint32_t u;
    memcpy(&u, &h, 4);
    return u;
}

// Half-precision constants of one strength: 1536 + t, 2^-adj and
// -(2^adj - 1) / 2^(adj + 1), each in both lanes.
struct HalfStrength {
    uint32_t tb, k, c;
};

__device__ __forceinline__ HalfStrength half_strength(int t, int adj) {
    const uint32_t tb = __half_as_ushort(__int2half_rn(1536 + t));
    const uint32_t k = (uint32_t)(15 - adj) << 10;  // 2^-adj (adj <= 9)
    const uint32_t c = __half_as_ushort(__float2half_rn(-(float)((1 << adj) - 1) / (float)(2 << adj)));
    return HalfStrength{tb * 0x10001u, k * 0x10001u, c * 0x10001u};
}

// constrain (cdef.rs:592-606) of two taps against two centres, both
// biased by 1024: |d| * 2^-adj - (2^adj - 1) / 2^(adj+1) is exact, adding
// 1536 rounds it to 1536 + (|d| >> adj), the threshold minus that is exact,
// and the result takes d's sign bit.  BORDER: NaN taps (outside the plane)
// give 0 through the NaN-skipping maximum with zero.
template <bool BORDER>
__device__ __forceinline__ __half2 constrain_h(__half2 x, __half2 xv, const HalfStrength& S) {
    const __half2 d = __hsub2(x, xv);
    const __half2 ad = __habs2(d);
    const __half2 v2 = __hadd2(__hfma2(ad, u2h(S.k), u2h(S.c)), u2h(kH1536));
    const __half2 m = BORDER ? __hmax2(__hsub2(u2h(S.tb), v2), u2h(0u)) : __hfma2_relu(v2, u2h(kHNeg1), u2h(S.tb));
    return u2h(h2u(__hmin2(ad, m)) | (h2u(d) & kSign2));
}

// The two samples at base + o, base + o + 1 (base even): two aligned words
// and a byte permute (o's parity differs between lanes).
__device__ __forceinline__ __half2 ld_pair(const uint16_t* base, int o) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(base + (o & ~1));
    return u2h(__byte_perm(w[0], w[1], (o & 1) ? 0x5432 : 0x3210));
}

// One tap pair (+o and -o) of weight w for two samples, with the clip range.
template <bool BORDER, bool MINMAX>
__device__ __forceinline__ void tap2_h(const uint16_t* cp, int o, __half2 xv, uint32_t w, const HalfStrength& S,
                                       __half2& sum, __half2& mn, __half2& mx) {
    const __half2 x0 = ld_pair(cp, o), x1 = ld_pair(cp, -o);
    sum = __hfma2(u2h(w), __hadd2(constrain_h<BORDER>(x0, xv, S), constrain_h<BORDER>(x1, xv, S)), sum);
    if (MINMAX) {
        mx = __hmax2(mx, __hmax2(x0, x1));
        mn = __hmin2(mn, __hmin2(x0, x1));
    }
}

// cdef_filter (cdef.rs:465-590) of two adjacent samples; MODE as filter_px.
// Returns the two filtered samples as half-precision bits 0x6400 | value.
template <bool BORDER, int MODE>
__device__ __forceinline__ uint32_t filter_pair_h(const uint16_t* cp, __half2 xv, const Taps& T, const HalfStrength& P,
                                                  uint32_t pw0, uint32_t pw1, const HalfStrength& Sc) {
    constexpr bool MM = MODE == 3;
    __half2 sum = u2h(0u), mn = xv, mx = xv;
    if (MODE & 1) {
        tap2_h<BORDER, MM>(cp, T.p0, xv, pw0, P, sum, mn, mx);
        tap2_h<BORDER, MM>(cp, T.p1, xv, pw1, P, sum, mn, mx);
    }
    if (MODE & 2) {
        tap2_h<BORDER, MM>(cp, T.a0, xv, 0x40004000u, Sc, sum, mn, mx);  // weight 2
        tap2_h<BORDER, MM>(cp, T.b0, xv, 0x40004000u, Sc, sum, mn, mx);
        tap2_h<BORDER, MM>(cp, T.a1, xv, 0x3C003C00u, Sc, sum, mn, mx);  // weight 1
        tap2_h<BORDER, MM>(cp, T.b1, xv, 0x3C003C00u, Sc, sum, mn, mx);
    }
    // (8 + sum - (sum < 0)) >> 4: sum / 16 + copysign(1/32, sum) is exact and
    // never a half-integer; adding 1536 rounds it to the reference's offset
    const __half2 g = __hfma2(sum, u2h(kH1_16), u2h((h2u(sum) & kSign2) | kH1_32));
    __half2 y = __hadd2(__hadd2(g, u2h(kH1536)), __hsub2(xv, u2h(kH1536)));
    if (MM) y = __hmin2(__hmax2(y, mn), mx);
    return h2u(y);
}

template <bool BORDER>
__device__ __forceinline__ uint32_t filter_pair_modes(const uint16_t* cp, __half2 xv, const Taps& T, int mode,
                                                      const HalfStrength& P, uint32_t pw0, uint32_t pw1,
                                                      const HalfStrength& Sc) {
    switch (mode) {
        case 3: return filter_pair_h<BORDER, 3>(cp, xv, T, P, pw0, pw1, Sc);
        case 1: return filter_pair_h<BORDER, 1>(cp, xv, T, P, pw0, pw1, Sc);
        case 2: return filter_pair_h<BORDER, 2>(cp, xv, T, P, pw0, pw1, Sc);
        default: return h2u(xv);
    }
}

// ---- luma, interior: per-lane tap offsets into the window and its shifted copy
// eo (per 8x8 block, bytes from the centre pair): for each tap of the
// block's direction, +offset then -offset, primary k = 0, 1, secondary
// (dir + 2) k = 0, 1, secondary (dir - 2) k = 0, 1; an odd column offset
// points into the shifted copy, so every tap is one aligned 32-bit load.

__device__ __forceinline__ __half2 ld_at(const uint16_t* cp, int byteoff) {
    return u2h(*reinterpret_cast<const uint32_t*>(reinterpret_cast<const char*>(cp) + byteoff));
}

template <bool MINMAX>
__device__ __forceinline__ void tap2_eo(const uint16_t* cp, int e0, int e1, __half2 xv, uint32_t w,
                                        const HalfStrength& S, __half2& sum, __half2& mn, __half2& mx) {
    const __half2 x0 = ld_at(cp, e0), x1 = ld_at(cp, e1);
    sum = __hfma2(u2h(w), __hadd2(constrain_h<false>(x0, xv, S), constrain_h<false>(x1, xv, S)), sum);
    if (MINMAX) {
        mx = __hmax2(mx, __hmax2(x0, x1));
        mn = __hmin2(mn, __hmin2(x0, x1));
    }
}

template <int MODE>
__device__ __forceinline__ uint32_t filter_pair_eo(const uint16_t* cp, __half2 xv, const int* eo,
                                                   const HalfStrength& P, uint32_t pw0, uint32_t pw1,
                                                   const HalfStrength& Sc) {
    constexpr bool MM = MODE == 3;
    __half2 sum = u2h(0u), mn = xv, mx = xv;
    if (MODE & 1) {
        tap2_eo<MM>(cp, eo[0], eo[1], xv, pw0, P, sum, mn, mx);
        tap2_eo<MM>(cp, eo[2], eo[3], xv, pw1, P, sum, mn, mx);
    }
    if (MODE & 2) {
        tap2_eo<MM>(cp, eo[4], eo[5], xv, 0x40004000u, Sc, sum, mn, mx);   // weight 2
        tap2_eo<MM>(cp, eo[8], eo[9], xv, 0x40004000u, Sc, sum, mn, mx);
        tap2_eo<MM>(cp, eo[6], eo[7], xv, 0x3C003C00u, Sc, sum, mn, mx);   // weight 1
        tap2_eo<MM>(cp, eo[10], eo[11], xv, 0x3C003C00u, Sc, sum, mn, mx);
    }
    const __half2 g = __hfma2(sum, u2h(kH1_16), u2h((h2u(sum) & kSign2) | kH1_32));
    __half2 y = __hadd2(__hadd2(g, u2h(kH1536)), __hsub2(xv, u2h(kH1536)));
    if (MM) y = __hmin2(__hmax2(y, mn), mx);
    return h2u(y);
}

__device__ __forceinline__ uint32_t filter_pair_eo_modes(const uint16_t* cp, __half2 xv, const int* eo, int mode,
                                                         const HalfStrength& P, uint32_t pw0, uint32_t pw1,
                                                         const HalfStrength& Sc) {
    switch (mode) {
        case 3: return filter_pair_eo<3>(cp, xv, eo, P, pw0, pw1, Sc);
        case 1: return filter_pair_eo<1>(cp, xv, eo, P, pw0, pw1, Sc);
        case 2: return filter_pair_eo<2>(cp, xv, eo, P, pw0, pw1, Sc);
        default: return h2u(xv);
    }
}

template <bool BORDER>
__device__ __forceinline__ void filter_two(const int16_t* cp, int xv0, int xv1, const Taps& T, int pri, int sec,
                                           int padj, int sadj, int pt0, int pt1, int& out0, int& out1) {
    if (pri && sec) {
        out0 = filter_px<BORDER, 3>(cp, xv0, T, pri, sec, padj, sadj, pt0, pt1);
        out1 = filter_px<BORDER, 3>(cp + 1, xv1, T, pri, sec, padj, sadj, pt0, pt1);
    } else if (pri) {
        out0 = filter_px<BORDER, 1>(cp, xv0, T, pri, sec, padj, sadj, pt0, pt1);
        out1 = filter_px<BORDER, 1>(cp + 1, xv1, T, pri, sec, padj, sadj, pt0, pt1);
    } else if (sec) {
        out0 = filter_px<BORDER, 2>(cp, xv0, T, pri, sec, padj, sadj, pt0, pt1);
        out1 = filter_px<BORDER, 2>(cp + 1, xv1, T, pri, sec, padj, sadj, pt0, pt1);
    }
}

__global__ void __launch_bounds__(kCdefThreads, 4) cdef_kernel(const FrameDev* __restrict__ frames,
                                                      const int32_t* __restrict__ starts, int n, int total) {
    // the three planes' windows, then the luma window shifted by one sample
    // (win[3][i] = win[0][i + 1], so a pair of samples starting at an odd
    // column is one aligned word); win[3] holds the direction search's
    // block-major luma until the search ends
    __shared__ __align__(16) int16_t win[4][WMAX * WP];
    __shared__ BlockParams bp[64];
    __shared__ __align__(16) int beo[64][12];  // luma tap byte offsets (interior, half path)
    __shared__ int costs[64][8];
    // luma of the 64 8x8 blocks, block-major with a 136-byte block stride so
    // that 32 lanes reading 8 bytes each from 32 blocks hit distinct banks
    static_assert(64 * 68 <= WMAX * WP, "blkx does not fit");
    int16_t (*blkx)[68] = reinterpret_cast<int16_t (*)[68]>(win[3]);
    __shared__ int16_t toff[16];
    __shared__ int8_t blive[64];  // 8x8 luma block filtered (inside the mi grid, not all skip)
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
        const bool half = h.bit_depth <= 10;  // the half-precision filter path
        const int lx0 = fbc * FB, ly0 = fbr * FB;
        const bool border = lx0 < H2 || ly0 < H2 || lx0 + FB + H2 > F.deb[0].w || ly0 + FB + H2 > F.deb[0].h;
        __syncthreads();
        for (int p = 0; p < np; p++) {
            int px = p ? ssx : 0, py = p ? ssy : 0;
            int bw = FB >> px, bh = FB >> py;
            int x0 = lx0 >> px, y0 = ly0 >> py;
            const PlaneDev& S = F.deb[p];
            int ww = bw + 2 * H2, wh = bh + 2 * H2;
            if (x0 >= 4 && y0 >= H2 && x0 + bw + 4 <= S.w && y0 + bh + H2 <= S.h) {
                // interior: aligned 4-sample loads over [x0 - 4, x0 + bw + 4),
                // every one inside the plane
                // every thread issues its (at most 5) loads before it unpacks
                // any, so their latencies overlap
                const int ng = (bw + 8) >> 2, items = wh * ng;
                const unsigned mag = (1u << 16) / ng + 1;  // i / ng for i < 4096
                constexpr int PER = (WMAX * ((FB + 8) >> 2) + kCdefThreads - 1) / kCdefThreads;
                int16_t* wrow = win[p];
                uint2 q[PER];
#pragma unroll
                for (int k = 0; k < PER; k++) {
                    const int i = threadIdx.x + k * kCdefThreads;
                    if (i >= items) break;
                    const int r = (int)(((unsigned)i * mag) >> 16), g = i - r * ng;
                    const uint8_t* row = S.p + (size_t)(y0 - H2 + r) * S.stride;
                    if (hbd) q[k] = *reinterpret_cast<const uint2*>(row + 2 * (x0 - 4 + 4 * g));
                    else q[k].x = *reinterpret_cast<const uint32_t*>(row + x0 - 4 + 4 * g);
                }
#pragma unroll
                for (int k = 0; k < PER; k++) {
                    const int i = threadIdx.x + k * kCdefThreads;
                    if (i >= items) break;
                    const int r = (int)(((unsigned)i * mag) >> 16), g = i - r * ng;
                    if (p == 0 && r >= H2 && r < H2 + FB && g >= 1 && g <= FB / 4) {
                        // the four luma samples also go to the direction
                        // search's block-major array, centred: (v >> cs) - 128
                        int t[4];
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const int v = hbd ? (int)(((e < 2 ? q[k].x : q[k].y) >> (16 * (e & 1))) & 0xffff)
                                              : (int)((q[k].x >> (8 * e)) & 0xff);
                            t[e] = (v >> cs) - 128;
                        }
                        const int sr = r - H2, sc = 4 * g - 4;
                        *reinterpret_cast<uint2*>(&blkx[((sr >> 3) << 3) + (sc >> 3)][((sr & 7) << 3) + (sc & 7)]) =
                            make_uint2(((uint32_t)t[0] & 0xffffu) | ((uint32_t)t[1] << 16),
                                       ((uint32_t)t[2] & 0xffffu) | ((uint32_t)t[3] << 16));
                    }
                    if (half) {
                        // samples 4g - 2 .. 4g + 1 of the window row as two
                        // words of biased half-precision pairs (0x6400 | v);
                        // a pair lies wholly inside or outside [0, ww)
                        uint32_t lo, hi;
                        if (hbd) {
                            lo = q[k].x | 0x64006400u;
                            hi = q[k].y | 0x64006400u;
                        } else {
                            lo = __byte_perm(q[k].x, 0x64u, 0x4140);
                            hi = __byte_perm(q[k].x, 0x64u, 0x4342);
                        }
                        uint32_t* wr = reinterpret_cast<uint32_t*>(wrow + r * WP);
                        const int c0 = 4 * g - 2;
                        if (c0 >= 0) wr[c0 >> 1] = lo;
                        if (c0 + 2 < ww) wr[(c0 + 2) >> 1] = hi;
                        continue;
                    }
                    int v[4];
                    if (hbd) {
                        v[0] = q[k].x & 0xffff;
                        v[1] = q[k].x >> 16;
                        v[2] = q[k].y & 0xffff;
                        v[3] = q[k].y >> 16;
                    } else {
                        v[0] = q[k].x & 0xff;
                        v[1] = (q[k].x >> 8) & 0xff;
                        v[2] = (q[k].x >> 16) & 0xff;
                        v[3] = q[k].x >> 24;
                    }
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        int c = 4 * g + e - 2;
                        if (c >= 0 && c < ww) wrow[r * WP + c] = (int16_t)v[e];
                    }
                }
            } else {
                for (int i = threadIdx.x; i < WMAX * wh; i += blockDim.x) {
                    int r = i / WMAX, c = i - r * WMAX;
                    if (c >= ww) continue;
                    int gy = y0 - H2 + r, gx = x0 - H2 + c;
                    const bool in = gy >= 0 && gy < S.h && gx >= 0 && gx < S.w;
                    const int v = in ? ld_px(S, hbd, gy, gx) : 0;
                    win[p][r * WP + c] = half ? (int16_t)(in ? 0x6400 | v : kHalfNA) : (in ? (int16_t)v : NA);
                }
            }
        }
        __syncthreads();
        // which 8x8 blocks are filtered (cdef_block's skip test, cdef.rs:229-262):
        // the four mi skip flags loaded together, out-of-grid ones read as skip
        if (threadIdx.x < 64) {
            const int blk = threadIdx.x, r = fbr * 16 + (blk >> 3) * 2, c = fbc * 16 + (blk & 7) * 2;
            bool live = idx >= 0 && r < h.mi_rows && c < h.mi_cols;
            if (live) {
                const uint8_t* sk = F.g.skip;
                const int mc = h.mi_cols;
                const bool rn = r + 1 < h.mi_rows, cn = c + 1 < mc;
                const int s00 = sk[r * mc + c];
                const int s10 = rn ? sk[(r + 1) * mc + c] : 1;
                const int s01 = cn ? sk[r * mc + c + 1] : 1;
                const int s11 = rn && cn ? sk[(r + 1) * mc + c + 1] : 1;
                live = !(s00 && s10 && s01 && s11);
            }
            blive[blk] = live;
        }
        // block-major centred luma for the direction search (only blocks
        // inside the mi grid are searched, and those lie inside the plane);
        // an interior luma window wrote it while staging
        const bool luma_staged = lx0 >= 4 && ly0 >= H2 && lx0 + FB + 4 <= F.deb[0].w && ly0 + FB + H2 <= F.deb[0].h;
        if (!luma_staged)
            for (int k = threadIdx.x; k < 64 * 64; k += blockDim.x) {
                int b = k >> 6, e = k & 63;
                int r = ((b >> 3) << 3) + (e >> 3), c = ((b & 7) << 3) + (e & 7);
                const int w = win[0][(r + H2) * WP + c + H2];
                blkx[b][e] = (int16_t)(((half ? w & 0x3FF : w) >> cs) - 128);
            }
        __syncthreads();
        // direction search: each warp computes one direction for 32 blocks
        // (warp-uniform direction, no divergence); costs go to shared memory
        // and one thread per block takes the arg-max
        for (int q = threadIdx.x; q < 64 * 8; q += blockDim.x) {
            const int d = (q >> 5) & 7, blk = (q >> 8) * 32 + (q & 31);
            int cost = -1;  // marks a block that is not filtered
            if (blive[blk]) {
                const int16_t* w = blkx[blk];
                switch (d) {
                    case 0: cost = dir_cost<0>(w); break;
                    case 1: cost = dir_cost<1>(w); break;
                    case 2: cost = dir_cost<2>(w); break;
                    case 3: cost = dir_cost<3>(w); break;
                    case 4: cost = dir_cost<4>(w); break;
                    case 5: cost = dir_cost<5>(w); break;
                    case 6: cost = dir_cost<6>(w); break;
                    default: cost = dir_cost<7>(w); break;
                }
            }
            costs[blk][d] = cost;
        }
        __syncthreads();
        if (threadIdx.x < 64) {
            const int blk = threadIdx.x;
            BlockParams b{0, 0, 0, 0, 0};
            if (costs[blk][0] >= 0) {
                // first strictly greater wins (cdef.rs:440-456)
                int best = costs[blk][0], bd = 0;
#pragma unroll
                for (int d = 1; d < 8; d++)
                    if (costs[blk][d] > best) {
                        best = costs[blk][d];
                        bd = d;
                    }
                int opp = costs[blk][(bd + 4) & 7];
                int var = (best - opp) >> 10;
                int pri_y = h.cdef_y_pri[idx] << cs;
                int vs = (var >> 6) > 0 ? min(floor_log2u((unsigned)(var >> 6)), 12) : 0;
                b.active = 1;
                b.pri_y = var != 0 ? (pri_y * (4 + vs) + 8) >> 4 : 0;
                b.padj_y = (int8_t)(b.pri_y ? max(h.cdef_damping + cs - floor_log2u((unsigned)b.pri_y), 0) : 0);
                b.ydir = (int8_t)(pri_y == 0 ? 0 : bd);
                int pri_uv = h.cdef_uv_pri[idx] << cs;
                b.uvdir = (int8_t)(pri_uv == 0 ? 0 : c_uv_dir[ssx][ssy][bd]);
                if (half && b.pri_y) {
                    const HalfStrength hs = half_strength(b.pri_y, b.padj_y);
                    b.htb = (uint16_t)hs.tb;
                    b.hk = (uint16_t)hs.k;
                    b.hc = (uint16_t)hs.c;
                }
                if (half && !border) {
                    const Taps T = taps_of(toff, b.ydir);
                    const int o[6] = {T.p0, T.p1, T.a0, T.a1, T.b0, T.b1};
#pragma unroll
                    for (int t = 0; t < 6; t++)
#pragma unroll
                        for (int sgn = 0; sgn < 2; sgn++) {
                            const int v = sgn ? -o[t] : o[t];
                            beo[blk][2 * t + sgn] = 2 * ((v & 1) ? v - 1 + 3 * WMAX * WP : v);
                        }
                }
            }
            bp[blk] = b;
        } else if (half && !border) {
            // the shifted luma window for the direction-specialised filter
            const uint32_t* we = reinterpret_cast<const uint32_t*>(win[0]);
            uint32_t* wo = reinterpret_cast<uint32_t*>(win[3]);
            for (int i = threadIdx.x - 64; i < WMAX * WP / 2 - 1; i += blockDim.x - 64)
                wo[i] = __byte_perm(we[i], we[i + 1], 0x5432);
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
            const int padj_uv = pri_uv ? max(damping - floor_log2u((unsigned)pri_uv), 0) : 0;
            if (half) {
                // pairs of horizontally adjacent samples, a warp on 64
                // consecutive samples of a row (8 blocks of luma)
                const HalfStrength Sc = half_strength(sec, sadj);
                const HalfStrength Puv = half_strength(pri_uv, padj_uv);
                const uint16_t* Wh = reinterpret_cast<const uint16_t*>(W);
                const int lbw = 6 - px;
                const bool shifted = p == 0 && !border;  // luma taps through beo
                for (int i = threadIdx.x; i < (bw * bh) >> 1; i += blockDim.x) {
                    const int r = (2 * i) >> lbw, c = (2 * i) & (bw - 1);
                    const int gy = y0 + r, gx = x0 + c;
                    if (gy >= dh || gx >= dw) continue;
                    const uint16_t* cp = Wh + (r + H2) * WP + c + H2;
                    const __half2 xv = u2h(*reinterpret_cast<const uint32_t*>(cp));
                    const int blk = (r >> (3 - py)) * 8 + (c >> (3 - px));
                    const BlockParams b = bp[blk];
                    uint32_t out = h2u(xv);
                    if (b.active) {
                        const int pri = p ? pri_uv : b.pri_y;
                        const HalfStrength P = p ? Puv : HalfStrength{b.htb * 0x10001u, b.hk * 0x10001u,
                                                                       b.hc * 0x10001u};
                        const bool prow = (pri >> cs) & 1;
                        const uint32_t pw0 = prow ? 0x42004200u : 0x44004400u;  // 3 : 4
                        const uint32_t pw1 = prow ? 0x42004200u : 0x40004000u;  // 3 : 2
                        const int mode = (pri ? 1 : 0) | (sec ? 2 : 0);
                        if (shifted) {
                            int eo[12];
                            const int4* e4 = reinterpret_cast<const int4*>(beo[blk]);
#pragma unroll
                            for (int t = 0; t < 3; t++) {
                                const int4 v = e4[t];
                                eo[4 * t] = v.x;
                                eo[4 * t + 1] = v.y;
                                eo[4 * t + 2] = v.z;
                                eo[4 * t + 3] = v.w;
                            }
                            out = filter_pair_eo_modes(cp, xv, eo, mode, P, pw0, pw1, Sc);
                        } else {
                            const Taps T = taps_of(toff, p ? b.uvdir : b.ydir);
                            out = border ? filter_pair_modes<true>(cp, xv, T, mode, P, pw0, pw1, Sc)
                                         : filter_pair_modes<false>(cp, xv, T, mode, P, pw0, pw1, Sc);
                        }
                    }
                    // out holds 0x6400 | value per lane
                    uint8_t* row = D.p + (size_t)gy * D.stride;
                    if (gx + 1 < dw) {  // gx is even: one aligned 2- or 4-byte store
                        if (hbd) *reinterpret_cast<uint32_t*>(row + 2 * gx) = out & 0x03FF03FFu;
                        else *reinterpret_cast<uint16_t*>(row + gx) = (uint16_t)__byte_perm(out, 0u, 0x0020);
                    } else {
                        st_px(D, hbd, gy, gx, (int)(out & 0x3FFu));
                    }
                }
                continue;
            }
            const int lbw = 6 - px;  // log2 of the block width in this plane
            // two horizontally adjacent samples per thread: same 8x8 block,
            // so one parameter and tap-offset fetch serves both
            for (int i = threadIdx.x; i < (bw * bh) >> 1; i += blockDim.x) {
                int r = (2 * i) >> lbw, c = (2 * i) & (bw - 1);
                int gy = y0 + r, gx = x0 + c;
                if (gy >= dh || gx >= dw) continue;
                const int16_t* cp = W + (r + H2) * WP + c + H2;
                int xv0 = cp[0], xv1 = cp[1];
                const BlockParams b = bp[(r >> (3 - py)) * 8 + (c >> (3 - px))];
                int out0 = xv0, out1 = xv1;
                if (b.active) {
                    const int pri = p ? pri_uv : b.pri_y;
                    const int padj = p ? padj_uv : b.padj_y;
                    const Taps T = taps_of(toff, p ? b.uvdir : b.ydir);
                    const int prow = (pri >> cs) & 1, pt0 = prow ? 3 : 4, pt1 = prow ? 3 : 2;
                    if (border) filter_two<true>(cp, xv0, xv1, T, pri, sec, padj, sadj, pt0, pt1, out0, out1);
                    else filter_two<false>(cp, xv0, xv1, T, pri, sec, padj, sadj, pt0, pt1, out0, out1);
                }
                if (gx + 1 < dw) {  // gx is even: one aligned 2- or 4-byte store
                    uint8_t* row = D.p + (size_t)gy * D.stride;
                    if (hbd) *reinterpret_cast<uint32_t*>(row + 2 * gx) = (uint32_t)out0 | (uint32_t)out1 << 16;
                    else *reinterpret_cast<uint16_t*>(row + gx) = (uint16_t)(out0 | out1 << 8);
                } else {
                    st_px(D, hbd, gy, gx, out0);
                }
            }
        }
    }
}

}  // namespace

int tiles_cdef(const FrameDev& f) { return ((f.h.mi_rows + 15) >> 4) * ((f.h.mi_cols + 15) >> 4); }

void launch_cdef(const FrameDev* frames, const int32_t* starts, int n, int total, const StageShape& sh,
                 cudaStream_t s) {
    if (total <= 0) return;
    cdef_kernel<<<shape_grid(sh, total), kCdefThreads, 0, s>>>(frames, starts, n, total);
}

}  // namespace av1g
