// inter.cu — §7.11.3 inter prediction for lists of predict_inter calls.
//
// The reference predicts one block at a time (predict_inter,
// src/inter_pred.rs:2100): per reference list a w x h int32 prediction
// (block_inter_prediction, inter_pred.rs:654, or block_warp per 8x8,
// inter_pred.rs:4276), a blend (average / distance / wedge / difference
// weight / inter-intra, inter_pred.rs:1289-1419 and 2844-3553), then OBMC
// (obmc_walk_axis, inter_pred.rs:1911, and overlap_blending,
// inter_pred.rs:4613).
//
// Every one of those outputs is a per-sample function of the call's scalar
// parameters: the sub-sample position of output column c is
// startX + stepX * c whatever block it sits in, and the vertical filter of
// output row r reads reference rows ((startY + stepY * r) >> 10) - 3 + t.  So
// the GPU cuts each call into 8x8 tiles (the block_warp grid) and gives each
// tile to one warp: the warp filters the reference rows its 8 rows need into
// shared memory, filters them vertically, blends both lists and any OBMC
// neighbour overlapping the tile in registers, and writes the tile.  Tiles
// of all calls of all frames run in one launch; the scalar per-call work
// (motion-vector scaling, useWarp, setupShear, wedge orientation, OBMC
// geometry) runs once per call on the host while the list is validated.
// A DIFFWTD block's chroma calls read the mask its luma call wrote into a
// luma-grid mask plane, so they run in a second launch.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "av1_spec_tables.h"
#include "common.cuh"
#include "wedge.cuh"

namespace av1g {
namespace {

constexpr int kWarps = 4;          // tiles per CTA
constexpr int kRows = 24;          // intermediate rows held per chunk
constexpr int kMaskMargin = 256;   // DIFFWTD mask plane margin past the luma plane

// ---- tables ---------------------------------------------------------------

__device__ const AV1T_SUBPEL_FILTERS_TYPE g_subpel AV1T_SUBPEL_FILTERS_DIMS = AV1T_SUBPEL_FILTERS_INIT;
__device__ const AV1T_WARPED_FILTERS_TYPE g_warped AV1T_WARPED_FILTERS_DIMS = AV1T_WARPED_FILTERS_INIT;
__device__ const AV1T_II_WEIGHTS_1D_TYPE g_ii AV1T_II_WEIGHTS_1D_DIMS = AV1T_II_WEIGHTS_1D_INIT;

const AV1T_DIV_LUT_TYPE h_div_lut AV1T_DIV_LUT_DIMS = AV1T_DIV_LUT_INIT;
const AV1T_WEDGE_CODEBOOK_TYPE h_codebook AV1T_WEDGE_CODEBOOK_DIMS = AV1T_WEDGE_CODEBOOK_INIT;
const AV1T_WEDGE_BITS_TYPE h_wedge_bits AV1T_WEDGE_BITS_DIMS = AV1T_WEDGE_BITS_INIT;
const AV1T_NUM_4X4_BLOCKS_WIDE_TYPE h_n4w AV1T_NUM_4X4_BLOCKS_WIDE_DIMS = AV1T_NUM_4X4_BLOCKS_WIDE_INIT;
const AV1T_NUM_4X4_BLOCKS_HIGH_TYPE h_n4h AV1T_NUM_4X4_BLOCKS_HIGH_DIMS = AV1T_NUM_4X4_BLOCKS_HIGH_INIT;

// OBMC masks of lengths 2, 4, 8, 16, 32 back to back (get_obmc_mask,
// inter_pred.rs:4532); offset of length L is L - 2.
struct ObmcMasks {
    uint8_t m[62];
};
constexpr ObmcMasks make_obmc_masks() {
    ObmcMasks o{};
    const uint8_t a2[] = AV1T_OBMC_MASK_2_INIT;
    const uint8_t a4[] = AV1T_OBMC_MASK_4_INIT;
    const uint8_t a8[] = AV1T_OBMC_MASK_8_INIT;
    const uint8_t a16[] = AV1T_OBMC_MASK_16_INIT;
    const uint8_t a32[] = AV1T_OBMC_MASK_32_INIT;
    for (int i = 0; i < 2; i++) o.m[i] = a2[i];
    for (int i = 0; i < 4; i++) o.m[2 + i] = a4[i];
    for (int i = 0; i < 8; i++) o.m[6 + i] = a8[i];
    for (int i = 0; i < 16; i++) o.m[14 + i] = a16[i];
    for (int i = 0; i < 32; i++) o.m[30 + i] = a32[i];
    return o;
}
__device__ const ObmcMasks g_obmc = make_obmc_masks();

// The wedge master masks (wedge.cuh), one device copy for this kernel.
using wedge::Master;
using wedge::kMaster;
__device__ const Master g_master = kMaster;

// ---- device records -------------------------------------------------------

struct RefPlane {
    const uint8_t* p;
    int32_t stride;  // bytes
    int32_t last_x, last_y;
};

struct InterFrame {
    PlaneDev planes[3];
    PlaneDev side[3];    // inter halves of inter-intra calls (when requested)
    RefPlane refs[7][3];
    uint8_t* mask;       // luma-grid DIFFWTD mask plane
    int32_t mask_stride;
    int32_t hbd, maxv;
};

// One reference list of one call: translational (start/step from
// motion_vector_scaling) or warp (w = index of its WarpRec).
struct RefCall {
    int32_t sx, sy, stx, sty;
    uint8_t ref, hf, vf, warp;
};

struct WarpRec {
    int32_t p[6];
    int32_t alpha, beta, gamma, delta;
};

// One OBMC neighbour prediction: region (ox, oy, fw, fh) of its block.
struct Seg {
    int32_t sx, sy, stx, sty;
    uint16_t ox, oy, fw, fh;
    uint8_t ref, hf, vf, left, mlen, pad[3];
};

enum Blend : uint8_t { B_SINGLE, B_AVG, B_DIST, B_WEDGE, B_DIFF_LUMA, B_DIFF_CHROMA, B_II, B_II_WEDGE };

struct Call {
    int32_t frame;
    uint16_t x, y, w, h;
    uint8_t plane, nref, blend, r0, r1, post, ssx, ssy;
    uint8_t fwd, bck, mask_type, ii_mode, ii_scale, wdir, wxoff, wyoff;
    uint8_t winv, nseg, side, pad;  // side: store the inter half of an inter-intra call
    uint32_t seg_first;
    RefCall ref[2];
};

__device__ __forceinline__ int ld_ref(const RefPlane& R, int hbd, int y, int x) {
    const uint8_t* row = R.p + (size_t)y * R.stride;
    return hbd ? (int)__ldg(reinterpret_cast<const uint16_t*>(row) + x) : (int)__ldg(row + x);
}

__device__ __forceinline__ int rnd(int v, int n) { return (v + ((1 << n) >> 1)) >> n; }

// Translational prediction (block_inter_prediction, inter_pred.rs:654) of
// the tile pixels (i, j), i in [i0, i1), j in [j0, j1), whose position in the
// predicted region is (roff + i, coff + j).  Lane pixel k is tile pixel
// (p >> 3, p & 7) with p = lane + 32 k.
__device__ void pred_trans(const RefPlane& R, int hbd, const RefCall& rc, int r0s, int r1s, int roff, int coff,
                           int i0, int i1, int j0, int j1, int32_t* buf, int lane, int32_t out[2]) {
    const int16_t* hfl = &g_subpel[rc.hf][0][0];
    const int16_t* vfl = &g_subpel[rc.vf][0][0];
    int rs = i0;
    while (rs < i1) {
        int base = ((rc.sy + rc.sty * (roff + rs)) >> 10) - 3;
        int re = rs + 1;
        while (re < i1 && ((rc.sy + rc.sty * (roff + re)) >> 10) + 5 - base <= kRows) re++;
        int span = ((rc.sy + rc.sty * (roff + re - 1)) >> 10) + 5 - base;
        for (int e = lane; e < span * 8; e += 32) {
            int ri = e >> 3, c = e & 7;
            if (c >= j0 && c < j1) {
                int ry = min(max(base + ri, 0), R.last_y);
                int p = rc.sx + rc.stx * (coff + c);
                const int16_t* f = hfl + ((p >> 6) & 15) * 8;
                int pint = (p >> 10) - 3;
                int s = 0;
#pragma unroll
                for (int t = 0; t < 8; t++) s += (int)__ldg(f + t) * ld_ref(R, hbd, ry, min(max(pint + t, 0), R.last_x));
                buf[ri * 8 + c] = rnd(s, r0s);
            }
        }
        __syncwarp();
#pragma unroll
        for (int k = 0; k < 2; k++) {
            int p = lane + 32 * k, i = p >> 3, j = p & 7;
            if (i >= rs && i < re && j >= j0 && j < j1) {
                int py = rc.sy + rc.sty * (roff + i);
                const int16_t* f = vfl + ((py >> 6) & 15) * 8;
                const int32_t* col = buf + (((py >> 10) - 3 - base) * 8 + j);
                int s = 0;
#pragma unroll
                for (int t = 0; t < 8; t++) s += (int)__ldg(f + t) * col[t * 8];
                out[k] = rnd(s, r1s);
            }
        }
        __syncwarp();
        rs = re;
    }
}

// block_warp (inter_pred.rs:4276) of the 8x8 block (ty, tx) of a call.
__device__ void pred_warp(const RefPlane& R, int hbd, const WarpRec& W, int ssx, int ssy, int bx, int by, int r0s,
                          int r1s, int th, int tw, int32_t* buf, int lane, int32_t out[2]) {
    int src_x = (bx + 4) << ssx, src_y = (by + 4) << ssy;
    long long dst_x = (long long)W.p[2] * src_x + (long long)W.p[3] * src_y + W.p[0];
    long long dst_y = (long long)W.p[4] * src_x + (long long)W.p[5] * src_y + W.p[1];
    long long x4 = dst_x >> ssx, y4 = dst_y >> ssy;
    int ix4 = (int)(x4 >> 16), sx4 = (int)(x4 & 0xffff);
    int iy4 = (int)(y4 >> 16), sy4 = (int)(y4 & 0xffff);
    for (int e = lane; e < 120; e += 32) {
        int i1 = (e >> 3) - 7, i2 = (e & 7) - 4;
        int sx = sx4 + W.alpha * i2 + W.beta * i1;
        int offs = min(max(((sx + 512) >> 10) + 64, 0), 192);
        const int16_t* f = &g_warped[offs][0];
        int ry = min(max(iy4 + i1, 0), R.last_y);
        int s = 0;
#pragma unroll
        for (int t = 0; t < 8; t++) s += (int)__ldg(f + t) * ld_ref(R, hbd, ry, min(max(ix4 + i2 - 3 + t, 0), R.last_x));
        buf[e] = rnd(s, r0s);
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 2; k++) {
        int p = lane + 32 * k, i = p >> 3, j = p & 7;
        if (i < th && j < tw) {
            int sy = sy4 + W.gamma * (j - 4) + W.delta * (i - 4);
            int offs = min(max(((sy + 512) >> 10) + 64, 0), 192);
            const int16_t* f = &g_warped[offs][0];
            int s = 0;
#pragma unroll
            for (int t = 0; t < 8; t++) s += (int)__ldg(f + t) * buf[(i + t) * 8 + j];
            out[k] = rnd(s, r1s);
        }
    }
    __syncwarp();
}

__device__ __forceinline__ int wedge_at(const Call& C, int yy, int xx) {
    int raw = __ldg(&g_master.m[C.wdir][C.wyoff + yy][C.wxoff + xx]);
    return C.winv ? 64 - raw : raw;
}

// The mask read of mask_blend (inter_pred.rs:3136) at plane sample (i, j)
// of a wedge mask on the luma grid.
__device__ __forceinline__ int wedge_mask_px(const Call& C, int i, int j) {
    if (!C.ssx && !C.ssy) return wedge_at(C, i, j);
    if (C.ssx && !C.ssy) return (wedge_at(C, i, 2 * j) + wedge_at(C, i, 2 * j + 1) + 1) >> 1;
    if (!C.ssx) return (wedge_at(C, 2 * i, j) + wedge_at(C, 2 * i + 1, j) + 1) >> 1;
    return (wedge_at(C, 2 * i, 2 * j) + wedge_at(C, 2 * i, 2 * j + 1) + wedge_at(C, 2 * i + 1, 2 * j) +
            wedge_at(C, 2 * i + 1, 2 * j + 1) + 2) >> 2;
}

__device__ __forceinline__ int diff_mask_px(const InterFrame& F, const Call& C, int i, int j) {
    const uint8_t* m = F.mask + (size_t)((C.y + i) << C.ssy) * F.mask_stride + ((C.x + j) << C.ssx);
    int s = F.mask_stride;
    if (!C.ssx && !C.ssy) return m[0];
    if (C.ssx && !C.ssy) return (m[0] + m[1] + 1) >> 1;
    if (!C.ssx) return (m[0] + m[s] + 1) >> 1;
    return (m[0] + m[1] + m[s] + m[s + 1] + 2) >> 2;
}

__global__ void __launch_bounds__(kWarps * 32) inter_kernel(const InterFrame* __restrict__ frames,
                                                             const Call* __restrict__ calls,
                                                             const uint32_t* __restrict__ starts, int ncalls,
                                                             uint32_t total, const WarpRec* __restrict__ warps,
                                                             const Seg* __restrict__ segs) {
    __shared__ int32_t smem[kWarps][kRows * 8];
    const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tile = blockIdx.x * kWarps + wid;
    if (tile >= total) return;
    int lo = 0, hi = ncalls - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(starts + mid) <= tile) lo = mid;
        else hi = mid - 1;
    }
    const Call C = calls[lo];
    const InterFrame& F = frames[C.frame];
    int32_t* buf = smem[wid];
    const int ntx = (C.w + 7) >> 3;
    const int li = (int)(tile - starts[lo]);
    const int ty = li / ntx, tx = li - ty * ntx;
    const int r0 = ty * 8, c0 = tx * 8;
    const int th = min(8, C.h - r0), tw = min(8, C.w - c0);
    const int hbd = F.hbd, maxv = F.maxv;

    int32_t pv[2][2] = {{0, 0}, {0, 0}};
#pragma unroll
    for (int l = 0; l < 2; l++) {
        if (l >= C.nref) break;
        const RefCall& rc = C.ref[l];
        const RefPlane& R = F.refs[rc.ref][C.plane];
        if (rc.warp) pred_warp(R, hbd, warps[rc.sx], C.ssx, C.ssy, C.x + c0, C.y + r0, C.r0, C.r1, th, tw, buf, lane,
                               pv[l]);
        else pred_trans(R, hbd, rc, C.r0, C.r1, r0, c0, 0, th, 0, tw, buf, lane, pv[l]);
    }

    const PlaneDev& P = F.planes[C.plane];
    int val[2] = {0, 0};
#pragma unroll
    for (int k = 0; k < 2; k++) {
        int p = lane + 32 * k, i = p >> 3, j = p & 7;
        if (i >= th || j >= tw) continue;
        int bi = r0 + i, bj = c0 + j;
        int a = pv[0][k], b = pv[1][k], v;
        switch (C.blend) {
        case B_AVG: v = rnd(a + b, 1 + C.post); break;
        case B_DIST: v = rnd(C.fwd * a + C.bck * b, 4 + C.post); break;
        case B_WEDGE: {
            int m = wedge_mask_px(C, bi, bj);
            v = rnd(m * a + (64 - m) * b, 6 + C.post);
            break;
        }
        case B_DIFF_LUMA: {
            // difference_weight_mask, inter_pred.rs:2958
            int d = rnd(abs(a - b), (hbd ? (maxv == 1023 ? 2 : 4) : 0) + C.post);
            int m = min(38 + d / 16, 64);
            if (C.mask_type) m = 64 - m;
            F.mask[(size_t)(C.y + bi) * F.mask_stride + C.x + bj] = (uint8_t)m;
            v = rnd(m * a + (64 - m) * b, 6 + C.post);
            break;
        }
        case B_DIFF_CHROMA: {
            int m = diff_mask_px(F, C, bi, bj);
            v = rnd(m * a + (64 - m) * b, 6 + C.post);
            break;
        }
        case B_II:
        case B_II_WEDGE: {
            // mask_blend_interintra, inter_pred.rs:3272
            if (C.side) {  // the blend happens once the intra half exists
                v = min(max(rnd(a, C.post), 0), maxv);
                break;
            }
            int m;
            if (C.blend == B_II_WEDGE) m = wedge_mask_px(C, bi, bj);
            else if (C.ii_mode == 1) m = g_ii[bi * C.ii_scale];
            else if (C.ii_mode == 2) m = g_ii[bj * C.ii_scale];
            else if (C.ii_mode == 3) m = g_ii[min(bi, bj) * C.ii_scale];
            else m = 32;
            int cl = min(max(rnd(a, C.post), 0), maxv);
            int gy = C.y + bi, gx = C.x + bj;
            int cur = (gy < P.h && gx < P.w) ? ld_px(P, hbd, gy, gx) : 0;
            v = rnd(m * cur + (64 - m) * cl, 6);
            break;
        }
        default: v = a; break;
        }
        val[k] = min(max(v, 0), maxv);
    }

    // OBMC: above neighbours then left ones (obmc_walk_axis order).
    for (int s = 0; s < C.nseg; s++) {
        const Seg S = segs[C.seg_first + s];
        int i0 = max(S.oy - r0, 0), i1 = min(S.oy + S.fh - r0, th);
        int j0 = max(S.ox - c0, 0), j1 = min(S.ox + S.fw - c0, tw);
        if (i0 >= i1 || j0 >= j1) continue;
        RefCall rc{S.sx, S.sy, S.stx, S.sty, S.ref, S.hf, S.vf, 0};
        int32_t ob[2] = {0, 0};
        pred_trans(F.refs[S.ref][C.plane], hbd, rc, C.r0, C.r1, r0 - S.oy, c0 - S.ox, i0, i1, j0, j1, buf, lane, ob);
        const uint8_t* mask = g_obmc.m + (S.mlen - 2);
#pragma unroll
        for (int k = 0; k < 2; k++) {
            int p = lane + 32 * k, i = p >> 3, j = p & 7;
            if (i < i0 || i >= i1 || j < j0 || j >= j1) continue;
            int m = S.left ? mask[c0 + j - S.ox] : mask[r0 + i - S.oy];
            int o = min(max(ob[k], 0), maxv);
            val[k] = (m * val[k] + (64 - m) * o + 32) >> 6;
        }
    }

#pragma unroll
    for (int k = 0; k < 2; k++) {
        int p = lane + 32 * k, i = p >> 3, j = p & 7;
        if (i >= th || j >= tw) continue;
        int gy = C.y + r0 + i, gx = C.x + c0 + j;
        if (gy < P.h && gx < P.w) st_px(C.side ? F.side[C.plane] : P, hbd, gy, gx, val[k]);
    }
}

// ---- host: the scalar per-call work ---------------------------------------

long long rnd2s(long long x, int n) {
    if (n == 0) return x;
    return x >= 0 ? (x + (1LL << (n - 1))) >> n : -((-x + (1LL << (n - 1))) >> n);
}
int clip3i(int lo, int hi, int v) { return v < lo ? lo : (v > hi ? hi : v); }

// setup_shear (inter_pred.rs:3982) with resolve_divisor (inter_pred.rs:3885).
bool setup_shear(const int32_t p[6], bool* valid, int32_t abcd[4]) {
    if (p[2] == 0) return false;
    uint32_t a = p[2] < 0 ? (uint32_t)(-(long long)p[2]) : (uint32_t)p[2];
    int n = 31 - __builtin_clz(a);
    long long e = (long long)a - (1LL << n);
    long long f = n > 8 ? (e + (1LL << (n - 9))) >> (n - 8) : e << (8 - n);
    if (f > 256) f = 256;
    long long fac = p[2] < 0 ? -h_div_lut[f] : h_div_lut[f];
    int sh = n + 14;
    auto sat = [](long long x, long long y) {
        __int128 q = (__int128)x * y;
        if (q > (__int128)INT64_MAX) return (long long)INT64_MAX;
        if (q < (__int128)INT64_MIN) return (long long)INT64_MIN;
        return (long long)q;
    };
    int32_t alpha0 = clip3i(-32768, 32767, p[2] - (1 << 16));
    int32_t beta0 = clip3i(-32768, 32767, p[3]);
    int32_t gamma0 = clip3i(-32768, 32767, (int32_t)rnd2s(sat((long long)p[4] * 65536, fac), sh));
    int32_t corr = (int32_t)rnd2s(sat((long long)p[3] * p[4], fac), sh);
    int32_t delta0 = clip3i(-32768, 32767, (int32_t)((uint32_t)p[5] - (uint32_t)corr - (1u << 16)));
    const int32_t v0[4] = {alpha0, beta0, gamma0, delta0};
    for (int i = 0; i < 4; i++) abcd[i] = (int32_t)rnd2s(v0[i], 6) * 64;
    *valid = 4 * std::abs(abcd[0]) + 7 * std::abs(abcd[1]) < (1 << 16) &&
             4 * std::abs(abcd[2]) + 4 * std::abs(abcd[3]) < (1 << 16);
    return true;
}

// motion_vector_scaling (inter_pred.rs:318).
// xScale / yScale of motion_vector_scaling (inter_pred.rs:318-330); false
// for a zero frame or reference extent.
bool ref_scale(long long fw, long long fh, long long ruw, long long rh, long long& xs, long long& ys) {
    if (fw <= 0 || fh <= 0 || ruw <= 0 || rh <= 0) return false;
    xs = ((ruw << 14) + fw / 2) / fw;
    ys = ((rh << 14) + fh / 2) / fh;
    return true;
}

void mv_scale(int ssx, int ssy, long long xs, long long ys, int x, int y, const int16_t mv[2], RefCall& rc) {
    long long ox = ((long long)x << 4) + ((2 * (long long)mv[1]) >> ssx) + 8;
    long long oy = ((long long)y << 4) + ((2 * (long long)mv[0]) >> ssy) + 8;
    rc.sx = (int32_t)(rnd2s(ox * xs - (8LL << 14), 8) + 32);
    rc.sy = (int32_t)(rnd2s(oy * ys - (8LL << 14), 8) + 32);
    rc.stx = (int32_t)rnd2s(xs, 4);
    rc.sty = (int32_t)rnd2s(ys, 4);
}

int small_filter(int f, int n) {
    if (n > 4) return f;
    return (f == 0 || f == 2) ? 4 : (f == 1 ? 5 : f);
}

struct Builder {
    const av1g_inter_job& job;
    int fi;
    int ssx_frame, ssy_frame;
    int hbd;
    std::vector<Call>& a;
    std::vector<Call>& b;
    std::vector<WarpRec>& warps;
    std::vector<Seg>& segs;
    std::string& err;
    bool any_diff = false;
    // per reference, computed once: its scale factors and whether each plane is usable
    long long xs[7] = {}, ys[7] = {};
    int8_t scale_ok[7] = {}, plane_ok[7][3] = {};

    void init() {
        const av1g_frame_header& hd = *job.hdr;
        for (int r = 0; r < 7; r++) {
            scale_ok[r] = ref_scale(hd.frame_width, hd.frame_height, job.refs[r].upscaled_width,
                                    job.refs[r].frame_height, xs[r], ys[r]);
            for (int p = 0; p < 3; p++) plane_ok[r][p] = p < hd.num_planes && ref_ok(r, p);
        }
    }

    bool bad(int k, const char* what) {
        err = "inter job " + std::to_string(fi) + ": call " + std::to_string(k) + ": " + what;
        return false;
    }

    // block_inter_prediction's reference-plane checks (inter_pred.rs:680-700).
    bool ref_ok(int ref, int plane) {
        const av1g_ref_frame& R = job.refs[ref];
        int g = plane ? ssx_frame : 0, gy = plane ? ssy_frame : 0;
        if (R.upscaled_width <= 0 || R.frame_height <= 0) return false;
        const av1g_plane& pl = R.planes[plane];
        int pw = (R.upscaled_width + g) >> g, ph = (R.frame_height + gy) >> gy;
        return pl.data && pl.width >= pw && pl.height >= ph && pl.stride >= pl.width * (hbd ? 2 : 1) &&
               !(pl.stride & 15);
    }

    bool trans(int k, int plane, int ref, const int16_t mv[2], int x, int y, int w, int h, int fx, int fy,
               RefCall& rc) {
        int sx = plane ? ssx_frame : 0, sy = plane ? ssy_frame : 0;
        if (!scale_ok[ref]) return bad(k, "zero frame or reference extent");
        mv_scale(sx, sy, xs[ref], ys[ref], x, y, mv, rc);
        if (!plane_ok[ref][plane]) return bad(k, "reference plane smaller than its extent");
        if (fx >= 6 || fy >= 6) return bad(k, "interpolation filter");
        // The kernel's int32 position arithmetic covers references up to 16x
        // larger than the frame; conformant streams stay within 2x.
        if (rc.stx <= 0 || rc.sty <= 0 || rc.stx > 16384 || rc.sty > 16384)
            return bad(k, "reference scale outside 1/16..16");
        rc.ref = (uint8_t)ref;
        rc.hf = (uint8_t)small_filter(fx, w);
        rc.vf = (uint8_t)small_filter(fy, h);
        rc.warp = 0;
        return true;
    }

    // predict_inter_one_ref with derive_use_warp (inter_pred.rs:1633-1910).
    bool one_ref(int k, const av1g_inter_pred& d, int list, bool local_valid, RefCall& rc) {
        int decision = 0;
        const av1g_warp_ctx* wp = d.warp >= 0 ? &job.warps[d.warp] : nullptr;
        if (wp) {
            int ym = wp->y_mode[list];
            bool yg = ym == 16 || ym == 24, gmw = wp->gm_type[list] > 1, scaled = wp->ref_is_scaled[list];
            bool gvalid = false;
            if (yg && gmw && !scaled) {
                int32_t sh[4];
                bool v;
                gvalid = setup_shear(wp->gm_params[list], &v, sh) && v;
            }
            if (d.w < 8 || d.h < 8 || wp->force_integer_mv) decision = 0;
            else if (d.motion_mode == 2 && local_valid) decision = 1;
            else if (yg && gmw && !scaled && gvalid) decision = 2;
        }
        int ref = d.ref[list];
        if (!decision) return trans(k, d.plane, ref, d.mv[list], d.x, d.y, d.w, d.h, d.filter_x, d.filter_y, rc);
        if (d.w > 128 || d.h > 128) return bad(k, "warp block larger than 128");
        const int32_t* params = decision == 1 ? wp->local_warp_params : wp->gm_params[list];
        WarpRec W{};
        bool v;
        if (!setup_shear(params, &v, &W.alpha)) return bad(k, "warp divisor");
        memcpy(W.p, params, sizeof W.p);
        const av1g_ref_frame& R = job.refs[ref];
        int sx = d.plane ? ssx_frame : 0, sy = d.plane ? ssy_frame : 0;
        if (R.upscaled_width <= 0 || R.frame_height <= 0) return bad(k, "zero reference extent");
        const av1g_plane& pl = R.planes[d.plane];
        if (!pl.data || pl.width < ((R.upscaled_width + sx) >> sx) || pl.height < ((R.frame_height + sy) >> sy) ||
            pl.stride < pl.width * (hbd ? 2 : 1) || (pl.stride & 15))
            return bad(k, "reference plane smaller than its extent");
        rc = RefCall{(int32_t)warps.size(), 0, 0, 0, (uint8_t)ref, 0, 0, 1};
        warps.push_back(W);
        return true;
    }

    // wedge_mask orientation (inter_pred.rs:2844): direction, offsets, sign.
    bool wedge(int k, int mi_size, int idx, int sign, Call& c) {
        if (mi_size >= 22 || h_wedge_bits[mi_size] == 0 || idx >= 16 || sign > 1) return bad(k, "wedge parameters");
        int n4w = h_n4w[mi_size], n4h = h_n4h[mi_size], w = n4w * 4, h = n4h * 4;
        int shape = n4h > n4w ? 0 : (n4h < n4w ? 1 : 2);
        const uint8_t* e = h_codebook[shape][idx];
        int dir = e[0], xoff = 32 - ((e[1] * w) >> 3), yoff = 32 - ((e[2] * h) >> 3);
        long long sum = 0;
        for (int i = 0; i < w; i++) sum += kMaster.m[dir][yoff][xoff + i];
        for (int i = 1; i < h; i++) sum += kMaster.m[dir][yoff + i][xoff];
        long long avg = (sum + (w + h - 1) / 2) / (w + h - 1);
        int flip = avg < 32;
        c.wdir = (uint8_t)dir;
        c.wxoff = (uint8_t)xoff;
        c.wyoff = (uint8_t)yoff;
        c.winv = (uint8_t)(sign != flip);
        // mask_blend's extent check against the luma-grid mask
        int mw = c.ssx ? 2 * c.w : c.w, mh = c.ssy ? 2 * c.h : c.h;
        if (mw > w || (long long)w * (mh - 1) + mw > (long long)w * h) return bad(k, "block larger than its wedge mask");
        return true;
    }

    // obmc_walk_axis (inter_pred.rs:1911) geometry of one pass.
    bool obmc_pass(int k, const av1g_inter_pred& d, bool left, uint32_t first, int count, Call& c) {
        const av1g_frame_header& hd = *job.hdr;
        int sx = c.ssx, sy = c.ssy, bw = d.w, bh = d.h;
        uint32_t lg = left ? d.mi_height_log2 : d.mi_width_log2;
        uint32_t start = left ? d.mi_row : d.mi_col;
        uint32_t limit = std::min<uint32_t>(left ? (uint32_t)hd.mi_rows : (uint32_t)hd.mi_cols, start + (1u << lg));
        uint32_t n_limit = std::min<uint32_t>(4, lg), n = 0;
        for (int q = 0; q < count && n < n_limit; q++) {
            const av1g_obmc_neighbour& nb = job.neighbours[first + q];
            uint32_t pos = nb.axis_pos4;
            if (pos < start || pos >= limit || nb.step4 < 2 || nb.step4 > 16 || nb.ref > 6)
                return bad(k, "OBMC neighbour outside the block's edge");
            n++;
            int px, py, pw, ph, mlen;
            if (!left) {
                px = (int)((pos * 4) >> sx);
                py = (int)((d.mi_row * 4u) >> sy);
                pw = std::min(bw, (int)((nb.step4 * 4u) >> sx));
                ph = std::min(bh >> 1, 32 >> sy);
                mlen = ph;
            } else {
                px = (int)((d.mi_col * 4u) >> sx);
                py = (int)((pos * 4) >> sy);
                pw = std::min(bw >> 1, 32 >> sx);
                ph = std::min(bh, (int)((nb.step4 * 4u) >> sy));
                mlen = pw;
            }
            if (pw == 0 || ph == 0) continue;
            int ox = px - d.x, oy = py - d.y;
            if (ox < 0 || oy < 0 || ox >= bw || oy >= bh) return bad(k, "OBMC region outside the block");
            int fw = std::min(pw, bw - ox), fh = std::min(ph, bh - oy);
            if (!fw || !fh) continue;
            RefCall rc;
            if (!trans(k, d.plane, nb.ref, nb.mv, px, py, fw, fh, nb.filter_x, nb.filter_y, rc)) return false;
            Seg s{rc.sx, rc.sy, rc.stx, rc.sty, (uint16_t)ox, (uint16_t)oy, (uint16_t)fw, (uint16_t)fh,
                  rc.ref, rc.hf, rc.vf, (uint8_t)left,
                  (uint8_t)(mlen == 2 || mlen == 4 || mlen == 8 || mlen == 16 ? mlen : 32), {0, 0, 0}};
            segs.push_back(s);
            c.nseg++;
        }
        return true;
    }

    bool add(int k) {
        const av1g_inter_pred& d = job.preds[k];
        const av1g_frame_header& hd = *job.hdr;
        if (d.plane >= hd.num_planes || d.w == 0 || d.h == 0 || d.w > 256 || d.h > 256) return bad(k, "plane or size");
        const av1g_plane& P = job.planes[d.plane];
        if (d.x >= P.width || d.y >= P.height) return bad(k, "position outside the plane");
        if (d.kind > 2) return bad(k, "kind");
        bool comp = d.kind == AV1G_INTER_COMPOUND, ii = d.kind == AV1G_INTER_INTRA;
        if (d.ref[0] > 6 || (comp && d.ref[1] > 6)) return bad(k, "reference index");
        if (comp && d.compound_type != 0 && d.compound_type != 1 && d.compound_type != 2 && d.compound_type != 4)
            return bad(k, "compound type");
        if (ii && d.interintra_mode > 3) return bad(k, "inter-intra mode");
        if (d.warp >= job.num_warps || (d.motion_mode == 2 && d.warp < 0)) return bad(k, "warp context");
        if (d.motion_mode == 1 &&
            (uint64_t)d.obmc_first + d.obmc_above + d.obmc_left > (uint64_t)std::max(job.num_neighbours, 0))
            return bad(k, "OBMC neighbour range");
        Call c{};
        c.frame = fi;
        c.x = d.x;
        c.y = d.y;
        c.w = d.w;
        c.h = d.h;
        c.plane = d.plane;
        c.ssx = (uint8_t)(d.plane ? ssx_frame : 0);
        c.ssy = (uint8_t)(d.plane ? ssy_frame : 0);
        int bd = hd.bit_depth;
        int r0 = bd == 12 ? 5 : 3, r1 = comp ? 7 : (bd == 12 ? 9 : 11);
        c.r0 = (uint8_t)r0;
        c.r1 = (uint8_t)r1;
        c.post = (uint8_t)(14 - r0 - r1);
        bool local_valid = d.warp >= 0 && job.warps[d.warp].local_valid;
        if (d.warp >= 0 && d.motion_mode == 2 && local_valid) {
            int32_t sh[4];
            bool v;
            if (!setup_shear(job.warps[d.warp].local_warp_params, &v, sh) || !v) local_valid = false;
        }
        c.nref = comp ? 2 : 1;
        for (int l = 0; l < c.nref; l++)
            if (!one_ref(k, d, l, local_valid, c.ref[l])) return false;
        bool chroma_diff = false;
        if (ii) {
            if (d.wedge_interintra) {
                c.blend = B_II_WEDGE;
                if (!wedge(k, d.mi_size, d.wedge_index, 0, c)) return false;
            } else {
                if (d.w > 128 || d.h > 128) return bad(k, "inter-intra block larger than 128");
                c.blend = B_II;
                c.ii_mode = d.interintra_mode;
                c.ii_scale = (uint8_t)(128 / std::max(d.w, d.h));
            }
            if (job.interintra_out[d.plane].data) {
                if (d.motion_mode == 1) return bad(k, "inter-intra call with OBMC cannot use the side plane");
                c.side = 1;
            }
        } else if (comp) {
            switch (d.compound_type) {
            case 2: c.blend = B_AVG; break;
            case 4:
                c.blend = B_DIST;
                c.fwd = d.fwd_weight;
                c.bck = d.bck_weight;
                break;
            case 0:
                c.blend = B_WEDGE;
                if (!wedge(k, d.mi_size, d.wedge_index, d.wedge_sign, c)) return false;
                break;
            default: {
                int lw = d.w << c.ssx, lh = d.h << c.ssy;
                if ((d.y << c.ssy) + lh > job.planes[0].height + kMaskMargin ||
                    (d.x << c.ssx) + lw > job.planes[0].width + kMaskMargin)
                    return bad(k, "difference-weight block past the mask plane");
                chroma_diff = d.plane != 0;
                c.blend = chroma_diff ? B_DIFF_CHROMA : B_DIFF_LUMA;
                c.mask_type = d.mask_type;
                any_diff = true;
            }
            }
        } else {
            c.blend = B_SINGLE;
        }
        if (d.motion_mode == 1) {
            c.seg_first = (uint32_t)segs.size();
            if (d.avail_u && d.plane_residual_ge_8x8 && !obmc_pass(k, d, false, d.obmc_first, d.obmc_above, c))
                return false;
            if (d.avail_l && !obmc_pass(k, d, true, d.obmc_first + d.obmc_above, d.obmc_left, c)) return false;
        }
        (chroma_diff ? b : a).push_back(c);
        return true;
    }
};

uint32_t tiles_of(const Call& c) { return (uint32_t)((c.w + 7) >> 3) * (uint32_t)((c.h + 7) >> 3); }

}  // namespace

av1g_status inter_run(const av1g_inter_job* jobs, int n, cudaStream_t st, std::string& err) {
    std::vector<InterFrame> frames(n);
    std::vector<Call> a, b;
    std::vector<WarpRec> warps;
    std::vector<Seg> segs;
    std::vector<int> diff_frames;
    {
        size_t np = 0;
        for (int i = 0; i < n; i++) np += jobs[i].num_preds > 0 ? (size_t)jobs[i].num_preds : 0;
        a.reserve(np);
    }
    for (int i = 0; i < n; i++) {
        const av1g_inter_job& j = jobs[i];
        if (!j.hdr || !j.refs || j.num_preds < 0 || (j.num_preds > 0 && !j.preds) || j.num_neighbours < 0 ||
            (j.num_neighbours > 0 && !j.neighbours) || j.num_warps < 0 || (j.num_warps > 0 && !j.warps)) {
            err = "inter job " + std::to_string(i) + ": missing header, references or lists";
            return AV1G_EINVAL;
        }
        const av1g_frame_header& h = *j.hdr;
        if ((h.bit_depth != 8 && h.bit_depth != 10 && h.bit_depth != 12) || h.frame_width <= 0 ||
            h.frame_height <= 0 || h.frame_width > 65535 || h.frame_height > 65535 || h.subsampling_x > 1 ||
            h.subsampling_y > 1 || h.num_planes < 1 || h.num_planes > 3) {
            err = "inter job " + std::to_string(i) + ": bit depth, subsampling or frame size";
            return AV1G_EINVAL;
        }
        InterFrame& F = frames[i];
        memset(&F, 0, sizeof F);
        F.hbd = h.bit_depth > 8;
        F.maxv = (1 << h.bit_depth) - 1;
        for (int p = 0; p < h.num_planes; p++) {
            const av1g_plane& pl = j.planes[p];
            if (!pl.data || pl.width <= 0 || pl.height <= 0 || pl.stride < pl.width * (F.hbd ? 2 : 1) ||
                (pl.stride & 15)) {
                err = "inter job " + std::to_string(i) + ": plane " + std::to_string(p);
                return AV1G_EINVAL;
            }
            F.planes[p] = PlaneDev{(uint8_t*)pl.data, pl.stride, pl.width, pl.height};
            const av1g_plane& sp = j.interintra_out[p];
            if (sp.data) {
                if (sp.width < pl.width || sp.height < pl.height || sp.stride < pl.width * (F.hbd ? 2 : 1) ||
                    (sp.stride & 15) || ((uintptr_t)sp.data & 15)) {
                    err = "inter job " + std::to_string(i) + ": inter-intra side plane " + std::to_string(p);
                    return AV1G_EINVAL;
                }
                F.side[p] = PlaneDev{(uint8_t*)sp.data, sp.stride, pl.width, pl.height};
            }
            for (int r = 0; r < 7; r++) {
                const av1g_ref_frame& R = j.refs[r];
                int sx = p ? h.subsampling_x : 0, sy = p ? h.subsampling_y : 0;
                F.refs[r][p] = RefPlane{(const uint8_t*)R.planes[p].data, R.planes[p].stride,
                                        ((R.upscaled_width + sx) >> sx) - 1, ((R.frame_height + sy) >> sy) - 1};
            }
        }
        Builder B{j, i, h.subsampling_x, h.subsampling_y, F.hbd, a, b, warps, segs, err};
        B.init();
        for (int k = 0; k < j.num_preds; k++)
            if (!B.add(k)) return AV1G_EINVAL;
        if (B.any_diff) {
            F.mask_stride = ((j.planes[0].width + kMaskMargin) + 15) & ~15;
            diff_frames.push_back(i);
        }
    }
    if (a.empty() && b.empty()) return AV1G_OK;

    std::vector<uint32_t> sa(a.size() + 1, 0), sb(b.size() + 1, 0);
    for (size_t k = 0; k < a.size(); k++) sa[k + 1] = sa[k] + tiles_of(a[k]);
    for (size_t k = 0; k < b.size(); k++) sb[k + 1] = sb[k] + tiles_of(b[k]);

    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    size_t o_frames = 0;
    size_t o_a = al(o_frames + sizeof(InterFrame) * n);
    size_t o_b = al(o_a + sizeof(Call) * a.size());
    size_t o_sa = al(o_b + sizeof(Call) * b.size());
    size_t o_sb = al(o_sa + sizeof(uint32_t) * sa.size());
    size_t o_w = al(o_sb + sizeof(uint32_t) * sb.size());
    size_t o_s = al(o_w + sizeof(WarpRec) * warps.size());
    size_t o_m = al(o_s + sizeof(Seg) * segs.size());
    size_t host_bytes = o_m;
    std::vector<size_t> mask_off(n, 0);
    size_t bytes = o_m;
    for (int i : diff_frames) {
        mask_off[i] = bytes;
        bytes = al(bytes + (size_t)frames[i].mask_stride * (jobs[i].planes[0].height + kMaskMargin));
    }
    uint8_t* dev = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&dev, bytes, st);
    if (e != cudaSuccess) {
        err = std::string("cudaMallocAsync: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    for (int i : diff_frames) frames[i].mask = dev + mask_off[i];
    e = upload_with(dev, host_bytes, st, [&](uint8_t* host) {
        memcpy(host + o_frames, frames.data(), sizeof(InterFrame) * n);
        if (!a.empty()) memcpy(host + o_a, a.data(), sizeof(Call) * a.size());
        if (!b.empty()) memcpy(host + o_b, b.data(), sizeof(Call) * b.size());
        memcpy(host + o_sa, sa.data(), sizeof(uint32_t) * sa.size());
        memcpy(host + o_sb, sb.data(), sizeof(uint32_t) * sb.size());
        if (!warps.empty()) memcpy(host + o_w, warps.data(), sizeof(WarpRec) * warps.size());
        if (!segs.empty()) memcpy(host + o_s, segs.data(), sizeof(Seg) * segs.size());
    });
    if (e == cudaSuccess && bytes > host_bytes) e = cudaMemsetAsync(dev + host_bytes, 0, bytes - host_bytes, st);
    const InterFrame* df = (const InterFrame*)(dev + o_frames);
    const WarpRec* dw = (const WarpRec*)(dev + o_w);
    const Seg* ds = (const Seg*)(dev + o_s);
    if (e == cudaSuccess && sa.back()) {
        unsigned grid = (sa.back() + kWarps - 1) / kWarps;
        inter_kernel<<<grid, kWarps * 32, 0, st>>>(df, (const Call*)(dev + o_a), (const uint32_t*)(dev + o_sa),
                                                  (int)a.size(), sa.back(), dw, ds);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && sb.back()) {
        unsigned grid = (sb.back() + kWarps - 1) / kWarps;
        inter_kernel<<<grid, kWarps * 32, 0, st>>>(df, (const Call*)(dev + o_b), (const uint32_t*)(dev + o_sb),
                                                  (int)b.size(), sb.back(), dw, ds);
        e = cudaGetLastError();
    }
    cudaFreeAsync(dev, st);
    if (e != cudaSuccess) {
        err = std::string("inter launch: ") + cudaGetErrorString(e);
        return AV1G_EDEVICE;
    }
    return AV1G_OK;
}

}  // namespace av1g

