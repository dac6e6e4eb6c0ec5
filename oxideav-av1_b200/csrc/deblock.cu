// deblock.cu — §7.14 deblocking filter, both passes fused per tile.
//
// Replaces loop_filter_frame (src/loop_filter.rs:271) as driven by
// loop_filter_frame_from_grid (src/cdf.rs:20449).  The reference walks every
// 4-sample edge segment in raster order, vertical pass then horizontal pass,
// filtering in place.  Within one pass no two edges touch the same samples:
// an edge's filter length is capped by the smaller of the two adjoining
// transform dimensions (loop_filter.rs:434-443) and its taps reach at most 7
// samples back and 6 forward (loop_filter.rs:643-671, 800-821), so every edge
// of a pass is independent and the sequential order is immaterial.
//
// B200 mapping: one CTA owns a 64x64 output tile of one plane and stages a
// 96x96 window (16-sample halo: an output sample can be moved by an edge up to
// 6 samples away whose taps reach 7 further) in shared memory.  It computes
// the per-4x4 edge parameters (filter length, limit, blimit, thresh) for the
// window from the mi grid, runs the vertical pass over all window rows, then
// the horizontal pass over the tile's columns, and writes the tile.  The
// frame is filtered out of place (recon -> deblocked) so halo reads never
// observe another tile's output.
#include "common.cuh"
#include "av1_spec_tables.h"

namespace av1g {

__constant__ AV1T_SUBSAMPLED_SIZE_TYPE c_subsampled AV1T_SUBSAMPLED_SIZE_DIMS = AV1T_SUBSAMPLED_SIZE_INIT;
__constant__ AV1T_MAX_TX_SIZE_RECT_TYPE c_max_tx_rect AV1T_MAX_TX_SIZE_RECT_DIMS = AV1T_MAX_TX_SIZE_RECT_INIT;
__constant__ AV1T_NUM_4X4_BLOCKS_WIDE_TYPE c_n4w AV1T_NUM_4X4_BLOCKS_WIDE_DIMS = AV1T_NUM_4X4_BLOCKS_WIDE_INIT;
__constant__ AV1T_NUM_4X4_BLOCKS_HIGH_TYPE c_n4h AV1T_NUM_4X4_BLOCKS_HIGH_DIMS = AV1T_NUM_4X4_BLOCKS_HIGH_INIT;
__constant__ AV1T_TX_WIDTH_TYPE c_txw AV1T_TX_WIDTH_DIMS = AV1T_TX_WIDTH_INIT;
__constant__ AV1T_TX_HEIGHT_TYPE c_txh AV1T_TX_HEIGHT_DIMS = AV1T_TX_HEIGHT_INIT;

namespace {

// window rows hold u16 samples at an odd number of 32-bit words per row
// (49), so a warp walking down a column touches 32 distinct banks; a row
// starts on a 4-byte (not always 8-byte) boundary, so the window is moved in
// 32-bit words
constexpr int TILE = 64, HALO = 16, WIN = TILE + 2 * HALO, PITCH = WIN + 2, CELLS = WIN / 4;
constexpr int kDbThreads = 256;  // deblock_kernel's CTA size
static_assert(WIN * (WIN / 4) % kDbThreads == 0, "window groups split evenly over the CTA");
constexpr int BLOCK_SIZES = 22, BLOCK_INVALID = 22;

struct Grid {
    const av1g_frame_header& h;
    const av1g_mi_grid& g;
    __device__ bool in(int r, int c) const { return r >= 0 && c >= 0 && r < h.mi_rows && c < h.mi_cols; }
    __device__ int at(int r, int c) const { return r * h.mi_cols + c; }
    __device__ int mi_size(int r, int c) const { return in(r, c) ? g.mi_size[at(r, c)] : BLOCK_INVALID; }
    __device__ int lf_tx(int plane, int sr, int sc) const {
        // loopfilter_tx_size_at (cdf.rs:20559-20594)
        int ssx = h.subsampling_x, ssy = h.subsampling_y;
        int lr = plane ? sr << ssy : sr, lc = plane ? sc << ssx : sc;
        int tx = 0;
        if (in(lr, lc)) tx = g.is_inter[at(lr, lc)] ? g.inter_tx_size[at(lr, lc)] : g.tx_size[at(lr, lc)];
        if (tx >= 19) tx = 0;  // not a TX_* ordinal: malformed grid, filtered as TX_4X4
        if (plane == 0) return tx;
        int ms = mi_size(lr, lc);
        if (ms >= BLOCK_SIZES) return 0;
        int psz = c_subsampled[ms][ssx ? 1 : 0][ssy ? 1 : 0];
        if (psz == BLOCK_INVALID) return 0;
        int uv = c_max_tx_rect[psz];
        int w = c_txw[uv], hh = c_txh[uv];
        if (w == 64 || hh == 64) return w == 16 ? 9 : (hh == 16 ? 10 : 3);
        return uv;
    }
    // adaptive_filter_strength(_selection) (loop_filter.rs:465-580): lvl only
    __device__ int level(int r, int c, int plane, int pass) const {
        int seg = in(r, c) ? g.segment_id[at(r, c)] : -1;
        int ref = in(r, c) ? g.ref_frame0[at(r, c)] : 0;
        if (ref < 0) ref = 0;
        int m = in(r, c) ? g.y_mode[at(r, c)] : 0;
        int mode_type = (m >= 14 && m != 16 && m != 24) ? 1 : 0;
        int i = plane == 0 ? pass : plane + 1;
        int dl = in(r, c) ? g.delta_lf[at(r, c) * 4 + (h.delta_lf_multi ? i : 0)] : 0;
        int lvl = clip3(0, 63, dl + h.lf_level[i]);
        if (seg >= 0 && seg < 8 && h.seg_lf_active[seg][i]) lvl = clip3(0, 63, h.seg_lf_data[seg][i] + lvl);
        if (h.lf_delta_enabled) {
            int ns = lvl >> 5;
            if (ref == 0) {
                lvl += h.lf_ref_deltas[0] * (1 << ns);
            } else {
                lvl += h.lf_ref_deltas[ref < 7 ? ref : 7] * (1 << ns);
                lvl += h.lf_mode_deltas[mode_type] * (1 << ns);
            }
            lvl = clip3(0, 63, lvl);
        }
        return lvl;
    }
};

// Packed edge parameters: filter length | limit << 8 | blimit << 16 | thresh << 24.
// Follows loop_filter_edge (loop_filter.rs:302-423) up to the sample loop.
__device__ uint32_t edge_param(const FrameDev& F, int plane, int pass, int cy, int cx) {
    const av1g_frame_header& h = F.h;
    Grid G{h, F.g};
    int ssx = plane ? h.subsampling_x : 0, ssy = plane ? h.subsampling_y : 0;
    int row = cy << ssy, col = cx << ssx;
    int x = col * 4, y = row * 4;
    row |= ssy;
    col |= ssx;
    if (cy < 0 || cx < 0 || x >= h.frame_width || y >= h.frame_height) return 0;
    if (pass == 0 && x == 0) return 0;
    if (pass == 1 && y == 0) return 0;
    int dx = pass == 0, dy = pass == 1;
    int xp = x >> ssx, yp = y >> ssy;
    int prow = row - (dy << ssy), pcol = col - (dx << ssx);
    if (prow < 0 || pcol < 0) return 0;
    if (row >= h.mi_rows || col >= h.mi_cols) return 0;
    int ms = G.mi_size(row, col);
    int tx = G.lf_tx(plane, row >> ssy, col >> ssx);
    int psz = ms < BLOCK_SIZES ? c_subsampled[ms][ssx][ssy] : BLOCK_INVALID;
    if (psz == BLOCK_INVALID) psz = ms;
    int skip = G.in(row, col) ? F.g.skip[G.at(row, col)] : 0;
    int ref0 = G.in(row, col) ? F.g.ref_frame0[G.at(row, col)] : 0;
    int ptx = G.lf_tx(plane, prow >> ssy, pcol >> ssx);
    int bw = psz >= BLOCK_SIZES ? 4 : c_n4w[psz] * 4;
    int bh = psz >= BLOCK_SIZES ? 4 : c_n4h[psz] * 4;
    bool block_edge = pass == 0 ? (xp % bw == 0) : (yp % bh == 0);
    bool tx_edge = pass == 0 ? (xp % c_txw[tx] == 0) : (yp % c_txh[tx] == 0);
    bool apply = tx_edge && (block_edge || !skip || ref0 <= 0);
    if (!apply) return 0;
    int lvl = G.level(row, col, plane, pass);
    if (lvl == 0) lvl = G.level(prow, pcol, plane, pass);
    if (lvl == 0) return 0;
    int base = pass == 0 ? min((int)c_txw[tx], (int)c_txw[ptx]) : min((int)c_txh[tx], (int)c_txh[ptx]);
    int fsize = min(base, plane == 0 ? 16 : 8);
    // one byte: filter length class (1: 4, 2: 8 or chroma 6, 3: 16) << 6 | lvl (1..63)
    return (uint32_t)((fsize == 4 ? 1 : (fsize == 8 ? 2 : 3)) << 6) | (uint32_t)lvl;
}

// Unpacks a cell code into filter length | limit << 8 | blimit << 16 |
// thresh << 24 (adaptive_filter_strength, loop_filter.rs:500-525).
__device__ __forceinline__ uint32_t decode_code(uint32_t code, int sharp) {
    if (code == 0) return 0;
    int lvl = code & 63, fsc = code >> 6;
    int fsize = fsc == 1 ? 4 : (fsc == 2 ? 8 : 16);
    int sh = sharp > 4 ? 2 : (sharp > 0 ? 1 : 0);
    int limit = sharp > 0 ? clip3(1, 9 - sharp, lvl >> sh) : max(lvl >> sh, 1);
    int blimit = (2 * (lvl + 2) + limit) & 0xff;
    return (uint32_t)fsize | ((uint32_t)limit << 8) | ((uint32_t)blimit << 16) | ((uint32_t)(lvl >> 4) << 24);
}

// Per-cell edge codes of every deblocked plane of a frame: u16 per 4x4 cell,
// vertical-edge code in the low byte, horizontal-edge code in the high byte.
// blockIdx.y is the frame; cells are numbered plane by plane.
__global__ void __launch_bounds__(256) lf_prep_kernel(const FrameDev* __restrict__ frames) {
    const FrameDev& F = frames[blockIdx.y];
    if (!F.do_stage[ST_DEBLOCK]) return;
    int cell = blockIdx.x * blockDim.x + threadIdx.x;
    for (int p = 0; p < F.h.num_planes; p++) {
        int cw = F.recon[p].w >> 2, ch = F.recon[p].h >> 2;
        if (cell < cw * ch) {
            if (p > 0 && F.h.lf_level[1 + p] == 0) return;
            int cy = cell / cw, cx = cell % cw;
            uint32_t v = edge_param(F, p, 0, cy, cx), hh = edge_param(F, p, 1, cy, cx);
            F.lf_codes[p][cell] = (uint16_t)(v | (hh << 8));
            return;
        }
        cell -= cw * ch;
    }
}

__device__ __forceinline__ int f4clamp(int v, int bd) { return clip3(-(1 << (bd - 1)), (1 << (bd - 1)) - 1, v); }

// wide_filter (loop_filter.rs:789-822) for one (n, log2Size) case: outputs
// i in [-n, n) from taps j in [-n, n] weighted 2 for |j| <= n2 else 1, source
// positions clamped to [-(n + 1), n].  All indices are compile-time.
template <int N, int LOG2, int N2>
__device__ __forceinline__ void wide(uint16_t* b, int st) {
    int v[2 * N + 2];
#pragma unroll
    for (int k = 0; k < 2 * N + 2; k++) v[k] = b[(k - N - 1) * st];
    int o[2 * N];
#pragma unroll
    for (int i = -N; i < N; i++) {
        int t = 0;
#pragma unroll
        for (int j = -N; j <= N; j++) {
            int pp = i + j < -(N + 1) ? -(N + 1) : (i + j > N ? N : i + j);
            t += v[pp + N + 1] * ((j <= N2 && j >= -N2) ? 2 : 1);
        }
        o[i + N] = (t + (1 << (LOG2 - 1))) >> LOG2;
    }
#pragma unroll
    for (int i = -N; i < N; i++) b[i * st] = (uint16_t)o[i + N];
}

// sample_filtering + filter_mask + narrow/wide filters (loop_filter.rs:582-822)
// on a line of shared-memory samples; b points at q0, st is the step.
__device__ void filter_line(uint16_t* b, int st, uint32_t prm, int plane, int bd) {
    int fs = prm & 0xff;
    int limit = (prm >> 8) & 0xff, blimit = (prm >> 16) & 0xff, thresh = prm >> 24;
    int bds = bd - 8;
    int q0 = b[0], q1 = b[st], q2 = b[2 * st], q3 = b[3 * st];
    int p0 = b[-st], p1 = b[-2 * st], p2 = b[-3 * st], p3 = b[-4 * st];
    // every test below is "some |difference| > bound": the largest
    // difference against the bound, the shared ones computed once
    const int d1 = max(abs(p1 - p0), abs(q1 - q0));
    int thr = thresh << bds;
    bool hev = d1 > thr;
    int flen = fs == 4 ? 4 : (plane ? 6 : (fs == 8 ? 8 : 16));
    int lim = limit << bds, blim = blimit << bds;
    int dl = d1;
    if (flen >= 6) dl = __vimax3_s32(dl, abs(p2 - p1), abs(q2 - q1));
    if (flen >= 8) dl = __vimax3_s32(dl, abs(p3 - p2), abs(q3 - q2));
    if (dl > lim || abs(p0 - q0) * 2 + abs(p1 - q1) / 2 > blim) return;
    int one = 1 << bds;
    bool flat = false, flat2 = false;
    if (fs >= 8) {
        int df = __vimax3_s32(d1, abs(p2 - p0), abs(q2 - q0));
        if (flen >= 8) df = __vimax3_s32(df, abs(p3 - p0), abs(q3 - q0));
        flat = df <= one;
    }
    if (fs >= 16 && flat) {
        int q4 = b[4 * st], q5 = b[5 * st], q6 = b[6 * st];
        int p4 = b[-5 * st], p5 = b[-6 * st], p6 = b[-7 * st];
        const int d2 = __vimax3_s32(__vimax3_s32(abs(p6 - p0), abs(q6 - q0), abs(p5 - p0)),
                                    __vimax3_s32(abs(q5 - q0), abs(p4 - p0), abs(q4 - q0)), 0);
        flat2 = d2 <= one;
    }
    if (fs == 4 || !flat) {
        int half = 0x80 << bds;
        int ps1 = p1 - half, ps0 = p0 - half, qs0 = q0 - half, qs1 = q1 - half;
        int f = hev ? f4clamp(ps1 - qs1, bd) : 0;
        f = f4clamp(f + 3 * (qs0 - ps0), bd);
        int f1 = f4clamp(f + 4, bd) >> 3;
        int f2 = f4clamp(f + 3, bd) >> 3;
        b[0] = (uint16_t)(f4clamp(qs0 - f1, bd) + half);
        b[-st] = (uint16_t)(f4clamp(ps0 + f2, bd) + half);
        if (!hev) {
            int ff = (f1 + 1) >> 1;
            b[st] = (uint16_t)(f4clamp(qs1 - ff, bd) + half);
            b[-2 * st] = (uint16_t)(f4clamp(ps1 + ff, bd) + half);
        }
        return;
    }
    if (fs == 8 || !flat2) {
        if (plane == 0) wide<3, 3, 0>(b, st);
        else wide<2, 3, 1>(b, st);
    } else {
        wide<6, 4, 1>(b, st);
    }
}

__global__ void __launch_bounds__(kDbThreads, 6) deblock_kernel(const FrameDev* __restrict__ frames,
                                                      const int32_t* __restrict__ starts, int n, int total) {
    __shared__ __align__(16) uint16_t win[WIN * PITCH];
    __shared__ uint32_t ev[CELLS * CELLS], eh[CELLS * CELLS];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        int f = find_frame(starts, n, t);
        const FrameDev& F = frames[f];
        int local = t - starts[f];
        // tile -> (plane, ty, tx); planes with no deblock work have no tiles
        int plane = 0, tx = 0, ty = 0;
        for (int p = 0; p < F.h.num_planes; p++) {
            if (p > 0 && F.h.lf_level[1 + p] == 0) continue;
            int ntx = (F.recon[p].w + TILE - 1) / TILE, nty = (F.recon[p].h + TILE - 1) / TILE;
            if (local < ntx * nty) { plane = p; ty = local / ntx; tx = local % ntx; break; }
            local -= ntx * nty;
        }
        const PlaneDev& S = F.recon[plane];
        const PlaneDev& D = F.deb[plane];
        const int hbd = F.hbd, bd = F.h.bit_depth;
        const int gx0 = tx * TILE - HALO, gy0 = ty * TILE - HALO;
        __syncthreads();  // previous tile done with shared memory
        // window: 4 consecutive samples per thread, one vector load when the
        // group lies inside the plane (rows are 4-sample aligned: gx0 % 4 == 0).
        // A window inside the plane horizontally (almost every tile) issues
        // all of a thread's loads before it unpacks any, so their latencies
        // overlap instead of adding up.
        if (gx0 >= 0 && gx0 + WIN <= S.w) {
            constexpr int G = WIN / 4, PER = WIN * G / kDbThreads;
            const uint8_t* base = S.p + (size_t)(hbd ? 2 : 1) * gx0;
            if (hbd) {
                uint2 v[PER];
#pragma unroll
                for (int q = 0; q < PER; q++) {
                    const int i = threadIdx.x + q * kDbThreads, r = i / G, c = (i - r * G) * 4;
                    v[q] = *reinterpret_cast<const uint2*>(base + (size_t)clip3(0, S.h - 1, gy0 + r) * S.stride + 2 * c);
                }
#pragma unroll
                for (int q = 0; q < PER; q++) {
                    const int i = threadIdx.x + q * kDbThreads, r = i / G, c = (i - r * G) * 4;
                    uint32_t* w = reinterpret_cast<uint32_t*>(&win[r * PITCH + c]);  // 4-byte aligned
                    w[0] = v[q].x;
                    w[1] = v[q].y;
                }
            } else {
                uint32_t v[PER];
#pragma unroll
                for (int q = 0; q < PER; q++) {
                    const int i = threadIdx.x + q * kDbThreads, r = i / G, c = (i - r * G) * 4;
                    v[q] = *reinterpret_cast<const uint32_t*>(base + (size_t)clip3(0, S.h - 1, gy0 + r) * S.stride + c);
                }
#pragma unroll
                for (int q = 0; q < PER; q++) {
                    const int i = threadIdx.x + q * kDbThreads, r = i / G, c = (i - r * G) * 4;
                    uint32_t* w = reinterpret_cast<uint32_t*>(&win[r * PITCH + c]);  // 4-byte aligned
                    w[0] = __byte_perm(v[q], 0u, 0x4140);
                    w[1] = __byte_perm(v[q], 0u, 0x4342);
                }
            }
        } else
        for (int i = threadIdx.x; i < WIN * (WIN / 4); i += blockDim.x) {
            int r = i / (WIN / 4), c = (i % (WIN / 4)) * 4;
            int gy = clip3(0, S.h - 1, gy0 + r), gx = gx0 + c;
            uint16_t* w = &win[r * PITCH + c];
            const uint8_t* row = S.p + (size_t)gy * S.stride;
            if (gx >= 0 && gx + 3 < S.w) {
                uint32_t* w32 = reinterpret_cast<uint32_t*>(w);  // 4-byte aligned
                if (hbd) {
                    const uint2 v = *reinterpret_cast<const uint2*>(row + 2 * gx);
                    w32[0] = v.x;
                    w32[1] = v.y;
                } else {
                    const uint32_t v = *reinterpret_cast<const uint32_t*>(row + gx);
                    w32[0] = __byte_perm(v, 0u, 0x4140);
                    w32[1] = __byte_perm(v, 0u, 0x4342);
                }
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++) w[k] = (uint16_t)ld_px(S, hbd, gy, clip3(0, S.w - 1, gx + k));
            }
        }
        const int cy0 = gy0 / 4, cx0 = gx0 / 4;  // gx0,gy0 are multiples of 4 (may be negative)
        const int cw = S.w >> 2, ch = S.h >> 2, sharp = F.h.lf_sharpness;
        const uint16_t* codes = F.lf_codes[plane];
        {
            // the edge codes: a thread's (at most 3) loads first, then the decodes
            constexpr int PER = (CELLS * CELLS + kDbThreads - 1) / kDbThreads;
            uint32_t code[PER];
#pragma unroll
            for (int q = 0; q < PER; q++) {
                const int i = threadIdx.x + q * kDbThreads, cr = i / CELLS, cc = i - cr * CELLS;
                const int cy = cy0 + cr, cx = cx0 + cc;
                code[q] = (i < CELLS * CELLS && cy >= 0 && cx >= 0 && cy < ch && cx < cw) ? codes[cy * cw + cx] : 0;
            }
#pragma unroll
            for (int q = 0; q < PER; q++) {
                const int i = threadIdx.x + q * kDbThreads;
                if (i >= CELLS * CELLS) break;
                ev[i] = decode_code(code[q] & 0xff, sharp);
                eh[i] = decode_code(code[q] >> 8, sharp);
            }
        }
        __syncthreads();
        // vertical pass: window rows x edge columns 12..84 (cells 3..21: a
        // filter moves at most 6 samples from its edge, so only those edges
        // move tile columns; all window rows keep each warp's rows aligned to
        // the 4-row cells)
        constexpr int VR = WIN, VE = CELLS - 5;
        for (int i = threadIdx.x; i < VR * VE; i += blockDim.x) {
            int r = i % VR, cc = 3 + i / VR;
            uint32_t prm = ev[(r >> 2) * CELLS + cc];
            if (prm & 0xff) filter_line(&win[r * PITCH + cc * 4], 1, prm, plane, bd);
        }
        __syncthreads();
        // horizontal pass: tile columns x edge rows 12..84
        constexpr int HE = CELLS - 5;  // cells 3..21
        for (int i = threadIdx.x; i < TILE * HE; i += blockDim.x) {
            int c = HALO + i % TILE, cr = 3 + i / TILE;
            uint32_t prm = eh[cr * CELLS + (c >> 2)];
            if (prm & 0xff) filter_line(&win[cr * 4 * PITCH + c], PITCH, prm, plane, bd);
        }
        __syncthreads();
        // write the tile, four samples per thread (one vector store inside the plane)
        const int dh = min(D.h, S.h), dw = min(D.w, S.w);
        for (int i = threadIdx.x; i < TILE * (TILE / 4); i += blockDim.x) {
            int r = i / (TILE / 4), c = (i % (TILE / 4)) * 4;
            int gy = ty * TILE + r, gx = tx * TILE + c;
            if (gy >= dh) continue;
            const uint16_t* w = &win[(r + HALO) * PITCH + c + HALO];
            uint8_t* row = D.p + (size_t)gy * D.stride;
            if (gx + 3 < dw) {
                const uint32_t* w32 = reinterpret_cast<const uint32_t*>(w);  // 4-byte aligned
                const uint2 v = make_uint2(w32[0], w32[1]);
                if (hbd) *reinterpret_cast<uint2*>(row + 2 * gx) = v;
                else *reinterpret_cast<uint32_t*>(row + gx) = __byte_perm(v.x, v.y, 0x6420);
            } else {
                for (int k = 0; k < 4 && gx + k < dw; k++) st_px(D, hbd, gy, gx + k, w[k]);
            }
        }
    }
}

}  // namespace

int tiles_deblock(const FrameDev& f) {
    int n = 0;
    for (int p = 0; p < f.h.num_planes; p++) {
        if (p > 0 && f.h.lf_level[1 + p] == 0) continue;
        n += ((f.recon[p].w + TILE - 1) / TILE) * ((f.recon[p].h + TILE - 1) / TILE);
    }
    return n;
}

int cells_deblock(const FrameDev& f) {
    int n = 0;
    for (int p = 0; p < f.h.num_planes; p++) n += (f.recon[p].w >> 2) * (f.recon[p].h >> 2);
    return n;
}

void launch_deblock(const FrameDev* frames, const int32_t* starts, int n, int total, int max_cells,
                    const StageShape& sh, cudaStream_t s) {
    if (total <= 0) return;
    lf_prep_kernel<<<dim3((max_cells + 255) / 256, n), 256, 0, s>>>(frames);
    deblock_kernel<<<shape_grid(sh, total), kDbThreads, 0, s>>>(frames, starts, n, total);
}

}  // namespace av1g
