/*
 * postfilter.c — CPU oracle for the §7.4 post-filter chain.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  A plain restatement of the
 * reference crate's sample-by-sample loops:
 *   §7.14 deblock        src/loop_filter.rs:271-822, src/cdf.rs:20449-20594
 *   §7.15 CDEF           src/cdef.rs:180-606,        src/cdf.rs:20300-20330
 *   §7.16 superres       src/superres.rs:282-445
 *   §7.17 restoration    src/loop_restoration.rs:268-883, src/cdf.rs:20624
 *   §7.18.3 film grain   src/film_grain.rs:100-873
 *   chain + crop         src/decoder/frame_driver.rs:790-1116
 * including the reference's own choices where it departs from a literal
 * reading of the spec (e.g. the raw box sum in the self-guided b2 term,
 * loop_restoration.rs:660-661; the secondary tap row keyed on priStr,
 * cdef.rs:493-498).
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "av1_spec_tables.h"

static const AV1T_UPSCALE_FILTER_TYPE UPSCALE_FILTER AV1T_UPSCALE_FILTER_DIMS = AV1T_UPSCALE_FILTER_INIT;
static const AV1T_GAUSSIAN_SEQUENCE_TYPE GAUSSIAN_SEQUENCE AV1T_GAUSSIAN_SEQUENCE_DIMS = AV1T_GAUSSIAN_SEQUENCE_INIT;
static const AV1T_SUBSAMPLED_SIZE_TYPE SUBSAMPLED_SIZE AV1T_SUBSAMPLED_SIZE_DIMS = AV1T_SUBSAMPLED_SIZE_INIT;
static const AV1T_MAX_TX_SIZE_RECT_TYPE MAX_TX_SIZE_RECT AV1T_MAX_TX_SIZE_RECT_DIMS = AV1T_MAX_TX_SIZE_RECT_INIT;
static const AV1T_NUM_4X4_BLOCKS_WIDE_TYPE NUM4W AV1T_NUM_4X4_BLOCKS_WIDE_DIMS = AV1T_NUM_4X4_BLOCKS_WIDE_INIT;
static const AV1T_NUM_4X4_BLOCKS_HIGH_TYPE NUM4H AV1T_NUM_4X4_BLOCKS_HIGH_DIMS = AV1T_NUM_4X4_BLOCKS_HIGH_INIT;
static const AV1T_TX_WIDTH_TYPE TXW AV1T_TX_WIDTH_DIMS = AV1T_TX_WIDTH_INIT;
static const AV1T_TX_HEIGHT_TYPE TXH AV1T_TX_HEIGHT_DIMS = AV1T_TX_HEIGHT_INIT;

enum { BLOCK_SIZES = 22, BLOCK_INVALID = 22, TX_4X4 = 0, TX_32X32 = 3, TX_16X32 = 9, TX_32X16 = 10 };
enum { NEARESTMV = 14, GLOBALMV = 16, GLOBAL_GLOBALMV = 24 };

static int clip3(int lo, int hi, int x) { return x < lo ? lo : (x > hi ? hi : x); }
static int round2(int x, int n) { return n == 0 ? x : (x + (1 << (n - 1))) >> n; }
static int64_t round2_64(int64_t x, int n) { return n == 0 ? x : (x + ((int64_t)1 << (n - 1))) >> n; }
static int floor_log2(uint32_t x) { int n = 0; if (!x) return 0; while (x >>= 1) n++; return n; }
static int iabs(int x) { return x < 0 ? -x : x; }

/* ===================================================================== */
/* §7.14 deblocking                                                      */
/* ===================================================================== */

/* PlaneBuffer::get / ::set (loop_filter.rs:137-160): clamped read,
 * dropped out-of-range write. */
static int pget(const ora_plane* p, int y, int x) {
    int yc = clip3(0, p->rows - 1, y), xc = clip3(0, p->cols - 1, x);
    return p->s[(size_t)yc * p->cols + xc];
}
static void pset(ora_plane* p, int y, int x, int v) {
    if (y < 0 || x < 0 || y >= p->rows || x >= p->cols) return;
    p->s[(size_t)y * p->cols + x] = v;
}

typedef struct { const av1g_frame_header* h; const av1g_mi_grid* g; } lf_ctx;

static int mi_idx(const lf_ctx* c, int r, int col) { return r * c->h->mi_cols + col; }
static int in_grid(const lf_ctx* c, int r, int col) {
    return r >= 0 && col >= 0 && r < c->h->mi_rows && col < c->h->mi_cols;
}
/* grid accessors with the walker's out-of-range defaults (cdf.rs:19404,
 * 19496, 20766, 20935, 21513, 21892, 28172, 28189) */
static int g_skip(const lf_ctx* c, int r, int col) { return in_grid(c, r, col) ? c->g->skip[mi_idx(c, r, col)] : 0; }
static int g_is_inter(const lf_ctx* c, int r, int col) { return in_grid(c, r, col) ? c->g->is_inter[mi_idx(c, r, col)] : 0; }
static int g_ref0(const lf_ctx* c, int r, int col) { return in_grid(c, r, col) ? c->g->ref_frame0[mi_idx(c, r, col)] : 0; }
static int g_mode(const lf_ctx* c, int r, int col) { return in_grid(c, r, col) ? c->g->y_mode[mi_idx(c, r, col)] : 0; }
static int g_seg(const lf_ctx* c, int r, int col) { return in_grid(c, r, col) ? c->g->segment_id[mi_idx(c, r, col)] : -1; }
static int g_dlf(const lf_ctx* c, int r, int col, int i) { return in_grid(c, r, col) ? c->g->delta_lf[mi_idx(c, r, col) * 4 + i] : 0; }
static int g_misize(const lf_ctx* c, int r, int col) { return in_grid(c, r, col) ? c->g->mi_size[mi_idx(c, r, col)] : BLOCK_INVALID; }
static int g_tx(const lf_ctx* c, int r, int col) { return in_grid(c, r, col) ? c->g->tx_size[mi_idx(c, r, col)] : TX_4X4; }
static int g_itx(const lf_ctx* c, int r, int col) { return in_grid(c, r, col) ? c->g->inter_tx_size[mi_idx(c, r, col)] : TX_4X4; }

/* get_plane_residual_size (cdf.rs:1250) — BLOCK_INVALID for None. */
static int plane_residual_size(int mi_size, int plane, int ssx, int ssy) {
    if (mi_size >= BLOCK_SIZES) return BLOCK_INVALID;
    int sx = plane > 0 ? (ssx != 0) : 0, sy = plane > 0 ? (ssy != 0) : 0;
    return SUBSAMPLED_SIZE[mi_size][sx][sy];
}

/* get_tx_size (cdf.rs:12976) with the caller's unwrap_or(TX_4X4). */
static int get_tx_size(int plane, int tx, int mi_size, int ssx, int ssy) {
    if (plane == 0) return tx;
    int psz = plane_residual_size(mi_size, plane, ssx, ssy);
    if (psz == BLOCK_INVALID) return TX_4X4;
    int uv = MAX_TX_SIZE_RECT[psz];
    int w = TXW[uv], h = TXH[uv];
    if (w == 64 || h == 64) {
        if (w == 16) return TX_16X32;
        if (h == 16) return TX_32X16;
        return TX_32X32;
    }
    return uv;
}

/* loopfilter_tx_size_at (cdf.rs:20559-20594). */
static int lf_tx_size(const lf_ctx* c, int plane, int sub_row, int sub_col) {
    int ssx = c->h->subsampling_x, ssy = c->h->subsampling_y;
    int lr = plane == 0 ? sub_row : (sub_row << ssy);
    int lc = plane == 0 ? sub_col : (sub_col << ssx);
    int luma_tx = g_is_inter(c, lr, lc) ? g_itx(c, lr, lc) : g_tx(c, lr, lc);
    if (plane == 0) return luma_tx;
    int ms = g_misize(c, lr, lc);
    if (ms >= BLOCK_SIZES) return TX_4X4;
    return get_tx_size(plane, luma_tx, ms, ssx, ssy);
}

typedef struct { int lvl, limit, blimit, thresh; } lf_strength;

/* adaptive_filter_strength_selection (loop_filter.rs:527-580). */
static int strength_selection(const lf_ctx* c, int segment, int ref, int mode_type, int delta_lf,
                              int plane, int pass) {
    const av1g_frame_header* h = c->h;
    int i = plane == 0 ? pass : plane + 1;
    int base = clip3(0, 63, delta_lf + h->lf_level[i]);
    int lvl_seg = base;
    if (segment >= 0 && segment < 8 && h->seg_lf_active[segment][i])
        lvl_seg = clip3(0, 63, h->seg_lf_data[segment][i] + lvl_seg);
    if (h->lf_delta_enabled) {
        int n_shift = lvl_seg >> 5;
        if (ref == 0) {
            lvl_seg += h->lf_ref_deltas[0] * (1 << n_shift);
        } else {
            int ri = ref < 7 ? ref : 7;
            int mi = mode_type < 1 ? mode_type : 1;
            lvl_seg += h->lf_ref_deltas[ri] * (1 << n_shift);
            lvl_seg += h->lf_mode_deltas[mi] * (1 << n_shift);
        }
        lvl_seg = clip3(0, 63, lvl_seg);
    }
    return clip3(0, 255, lvl_seg);
}

/* adaptive_filter_strength (loop_filter.rs:465-525). */
static lf_strength filter_strength(const lf_ctx* c, int row, int col, int plane, int pass) {
    const av1g_frame_header* h = c->h;
    int segment = g_seg(c, row, col); /* -1 -> u8::MAX: never an active segment */
    int ref = g_ref0(c, row, col);
    if (ref < 0) ref = 0;
    int m = g_mode(c, row, col);
    int mode_type = (m >= NEARESTMV && m != GLOBALMV && m != GLOBAL_GLOBALMV) ? 1 : 0;
    int dl_idx = h->delta_lf_multi ? (plane == 0 ? pass : plane + 1) : 0;
    int dl = g_dlf(c, row, col, dl_idx);
    lf_strength s;
    s.lvl = strength_selection(c, segment < 0 ? 255 : segment, ref, mode_type, dl, plane, pass);
    int shift = h->lf_sharpness > 4 ? 2 : (h->lf_sharpness > 0 ? 1 : 0);
    int limit = h->lf_sharpness > 0 ? clip3(1, 9 - h->lf_sharpness, s.lvl >> shift)
                                     : ((s.lvl >> shift) > 1 ? (s.lvl >> shift) : 1);
    s.limit = limit;
    s.blimit = (2 * (s.lvl + 2) + limit) & 0xff; /* stored as u8 in the reference */
    s.thresh = s.lvl >> 4;
    return s;
}

static int filter4_clamp(int v, int bd) { return clip3(-(1 << (bd - 1)), (1 << (bd - 1)) - 1, v); }

/* narrow_filter (loop_filter.rs:743-787). */
static void narrow_filter(ora_plane* p, int x, int y, int dx, int dy, int hev, int bd) {
    int half = 0x80 << (bd - 8);
    int q0 = pget(p, y, x), q1 = pget(p, y + dy, x + dx);
    int p0 = pget(p, y - dy, x - dx), p1 = pget(p, y - 2 * dy, x - 2 * dx);
    int ps1 = p1 - half, ps0 = p0 - half, qs0 = q0 - half, qs1 = q1 - half;
    int f = hev ? filter4_clamp(ps1 - qs1, bd) : 0;
    f = filter4_clamp(f + 3 * (qs0 - ps0), bd);
    int f1 = filter4_clamp(f + 4, bd) >> 3;
    int f2 = filter4_clamp(f + 3, bd) >> 3;
    pset(p, y, x, filter4_clamp(qs0 - f1, bd) + half);
    pset(p, y - dy, x - dx, filter4_clamp(ps0 + f2, bd) + half);
    if (!hev) {
        int ff = round2(f1, 1);
        pset(p, y + dy, x + dx, filter4_clamp(qs1 - ff, bd) + half);
        pset(p, y - 2 * dy, x - 2 * dx, filter4_clamp(ps1 + ff, bd) + half);
    }
}

/* wide_filter (loop_filter.rs:789-822). */
static void wide_filter(ora_plane* p, int x, int y, int plane, int dx, int dy, int log2_size) {
    int n = log2_size == 4 ? 6 : (plane == 0 ? 3 : 2);
    int n2 = (log2_size == 3 && plane == 0) ? 0 : 1;
    int f[12];
    for (int i = -n; i < n; i++) {
        int64_t t = 0;
        for (int j = -n; j <= n; j++) {
            int pp = clip3(-(n + 1), n, i + j);
            int tap = iabs(j) <= n2 ? 2 : 1;
            t += (int64_t)pget(p, y + pp * dy, x + pp * dx) * tap;
        }
        f[i + n] = (int)round2_64(t, log2_size);
    }
    for (int i = -n; i < n; i++) pset(p, y + i * dy, x + i * dx, f[i + n]);
}

/* filter_mask + sample_filtering (loop_filter.rs:582-741). */
static void sample_filtering(ora_plane* p, int x, int y, int plane, int limit, int blimit,
                             int thresh, int dx, int dy, int filter_size, int bd) {
    int q[7], pp[7];
    for (int k = 0; k < 7; k++) {
        q[k] = pget(p, y + k * dy, x + k * dx);
        pp[k] = pget(p, y - (k + 1) * dy, x - (k + 1) * dx);
    }
    int bds = bd - 8;
    int thr = thresh << bds;
    int hev = iabs(pp[1] - pp[0]) > thr || iabs(q[1] - q[0]) > thr;
    int flen = filter_size == 4 ? 4 : (plane != 0 ? 6 : (filter_size == 8 ? 8 : 16));
    int lim = limit << bds, blim = blimit << bds;
    int mask = iabs(pp[1] - pp[0]) > lim || iabs(q[1] - q[0]) > lim ||
               iabs(pp[0] - q[0]) * 2 + iabs(pp[1] - q[1]) / 2 > blim;
    if (flen >= 6) mask |= iabs(pp[2] - pp[1]) > lim || iabs(q[2] - q[1]) > lim;
    if (flen >= 8) mask |= iabs(pp[3] - pp[2]) > lim || iabs(q[3] - q[2]) > lim;
    if (mask) return;
    int one = 1 << bds;
    int flat = 0, flat2 = 0;
    if (filter_size >= 8) {
        int m = iabs(pp[1] - pp[0]) > one || iabs(q[1] - q[0]) > one ||
                iabs(pp[2] - pp[0]) > one || iabs(q[2] - q[0]) > one;
        if (flen >= 8) m |= iabs(pp[3] - pp[0]) > one || iabs(q[3] - q[0]) > one;
        flat = !m;
    }
    if (filter_size >= 16) {
        int m = iabs(pp[6] - pp[0]) > one || iabs(q[6] - q[0]) > one ||
                iabs(pp[5] - pp[0]) > one || iabs(q[5] - q[0]) > one ||
                iabs(pp[4] - pp[0]) > one || iabs(q[4] - q[0]) > one;
        flat2 = !m;
    }
    if (filter_size == 4 || !flat) narrow_filter(p, x, y, dx, dy, hev, bd);
    else if (filter_size == 8 || !flat2) wide_filter(p, x, y, plane, dx, dy, 3);
    else wide_filter(p, x, y, plane, dx, dy, 4);
}

/* loop_filter_edge (loop_filter.rs:302-423). */
static void loop_filter_edge(const lf_ctx* c, ora_plane* planes, int plane, int pass, int row,
                             int col) {
    const av1g_frame_header* h = c->h;
    int ssx = plane ? h->subsampling_x : 0, ssy = plane ? h->subsampling_y : 0;
    int dx = pass == 0 ? 1 : 0, dy = pass == 0 ? 0 : 1;
    int x = col * 4, y = row * 4;
    row |= ssy;
    col |= ssx;
    if (x >= h->frame_width || y >= h->frame_height) return;
    if (pass == 0 && x == 0) return;
    if (pass == 1 && y == 0) return;
    int xp = x >> ssx, yp = y >> ssy;
    int prev_row = row - (dy << ssy), prev_col = col - (dx << ssx);
    if (prev_row < 0 || prev_col < 0) return;
    if (row >= h->mi_rows || col >= h->mi_cols) return;
    int mi_size = g_misize(c, row, col);
    int tx = lf_tx_size(c, plane, row >> ssy, col >> ssx);
    int psz = plane_residual_size(mi_size, plane, ssx, ssy);
    if (psz == BLOCK_INVALID) psz = mi_size;
    int skip = g_skip(c, row, col);
    int is_intra = g_ref0(c, row, col) <= 0;
    int prev_tx = lf_tx_size(c, plane, prev_row >> ssy, prev_col >> ssx);
    int bw = psz >= BLOCK_SIZES ? 4 : NUM4W[psz] * 4;
    int bh = psz >= BLOCK_SIZES ? 4 : NUM4H[psz] * 4;
    int is_block_edge = pass == 0 ? (xp % bw == 0) : (yp % bh == 0);
    int is_tx_edge = pass == 0 ? (xp % TXW[tx] == 0) : (yp % TXH[tx] == 0);
    int apply = is_tx_edge && (is_block_edge || !skip || is_intra);
    /* filter_size (loop_filter.rs:434-443) */
    int base = pass == 0 ? (TXW[tx] < TXW[prev_tx] ? TXW[tx] : TXW[prev_tx])
                         : (TXH[tx] < TXH[prev_tx] ? TXH[tx] : TXH[prev_tx]);
    int cap = plane == 0 ? 16 : 8;
    int fsize = base < cap ? base : cap;
    lf_strength s = filter_strength(c, row, col, plane, pass);
    if (s.lvl == 0) s = filter_strength(c, prev_row, prev_col, plane, pass);
    if (!apply || s.lvl == 0) return;
    for (int i = 0; i < 4; i++)
        sample_filtering(&planes[plane], xp + dy * i, yp + dx * i, plane, s.limit, s.blimit,
                         s.thresh, dx, dy, fsize, h->bit_depth);
}

/* loop_filter_frame (loop_filter.rs:271-300). */
void ora_loop_filter_frame(const av1g_frame_header* hdr, const av1g_mi_grid* grid,
                           ora_plane planes[3]) {
    lf_ctx c = {hdr, grid};
    for (int plane = 0; plane < hdr->num_planes; plane++) {
        if (plane > 0 && hdr->lf_level[1 + plane] == 0) continue;
        int ssx = plane ? hdr->subsampling_x : 0, ssy = plane ? hdr->subsampling_y : 0;
        int rs = plane == 0 ? 1 : 1 << ssy, cs = plane == 0 ? 1 : 1 << ssx;
        for (int pass = 0; pass < 2; pass++)
            for (int row = 0; row < hdr->mi_rows; row += rs)
                for (int col = 0; col < hdr->mi_cols; col += cs)
                    loop_filter_edge(&c, planes, plane, pass, row, col);
    }
}

/* ===================================================================== */
/* §7.15 CDEF                                                            */
/* ===================================================================== */

static const int CDEF_PRI_TAPS[2][2] = {{4, 2}, {3, 3}};          /* cdef.rs:64 */
static const int CDEF_SEC_TAPS[2][2] = {{2, 1}, {2, 1}};          /* cdef.rs:70 */
static const int CDEF_DIRECTIONS[8][2][2] = {                     /* cdef.rs:76 */
    {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}}, {{0, 1}, {0, 2}}, {{0, 1}, {1, 2}},
    {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},  {{1, 0}, {2, 0}}, {{1, 0}, {2, -1}}};
static const int DIV_TABLE[9] = {0, 840, 420, 280, 210, 168, 140, 120, 105}; /* cdef.rs:90 */
static const int CDEF_UV_DIR[2][2][8] = {                         /* cdef.rs:99 */
    {{0, 1, 2, 3, 4, 5, 6, 7}, {1, 2, 2, 2, 3, 4, 6, 0}},
    {{7, 0, 2, 4, 5, 6, 6, 6}, {0, 1, 2, 3, 4, 5, 6, 7}}};

/* constrain (cdef.rs:592-606). */
static int constrain(int diff, int threshold, int damping) {
    if (threshold == 0) return 0;
    int adj = damping - floor_log2((uint32_t)threshold);
    if (adj < 0) adj = 0;
    int sign = diff < 0 ? -1 : 1;
    int ad = iabs(diff);
    int shifted = adj >= 31 ? 0 : ad >> adj;
    int inner = threshold - shifted;
    if (inner < 0) inner = 0;
    return sign * clip3(0, ad, inner);
}

/* cdef_direction (cdef.rs:366-456). */
static void cdef_direction(const av1g_frame_header* h, const ora_plane* p0, int r, int c,
                           int* y_dir, int* var) {
    int partial[8][15];
    int cost[8];
    memset(partial, 0, sizeof partial);
    memset(cost, 0, sizeof cost);
    int x0 = c << 2, y0 = r << 2, shift = h->bit_depth - 8;
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) {
            int sx = clip3(0, p0->cols - 1, x0 + j), sy = clip3(0, p0->rows - 1, y0 + i);
            int x = (p0->s[(size_t)sy * p0->cols + sx] >> shift) - 128;
            partial[0][i + j] += x;
            partial[1][i + j / 2] += x;
            partial[2][i] += x;
            partial[3][3 + i - j / 2] += x;
            partial[4][7 + i - j] += x;
            partial[5][3 - i / 2 + j] += x;
            partial[6][j] += x;
            partial[7][i / 2 + j] += x;
        }
    for (int i = 0; i < 8; i++) {
        cost[2] += partial[2][i] * partial[2][i];
        cost[6] += partial[6][i] * partial[6][i];
    }
    cost[2] *= DIV_TABLE[8];
    cost[6] *= DIV_TABLE[8];
    for (int i = 0; i < 7; i++) {
        cost[0] += (partial[0][i] * partial[0][i] + partial[0][14 - i] * partial[0][14 - i]) * DIV_TABLE[i + 1];
        cost[4] += (partial[4][i] * partial[4][i] + partial[4][14 - i] * partial[4][14 - i]) * DIV_TABLE[i + 1];
    }
    cost[0] += partial[0][7] * partial[0][7] * DIV_TABLE[8];
    cost[4] += partial[4][7] * partial[4][7] * DIV_TABLE[8];
    for (int i = 1; i < 8; i += 2) {
        for (int j = 0; j < 5; j++) cost[i] += partial[i][3 + j] * partial[i][3 + j];
        cost[i] *= DIV_TABLE[8];
        for (int j = 0; j < 3; j++)
            cost[i] += (partial[i][j] * partial[i][j] + partial[i][10 - j] * partial[i][10 - j]) * DIV_TABLE[2 * j + 2];
    }
    int best = 0, d = 0;
    for (int k = 0; k < 8; k++)
        if (cost[k] > best) { best = cost[k]; d = k; }
    *y_dir = d;
    *var = (best - cost[(d + 4) & 7]) >> 10;
}

/* cdef_filter_block + cdef_sample_at (cdef.rs:465-590). */
static void cdef_filter_block(const av1g_frame_header* h, const ora_plane* src, ora_plane* dst,
                              int plane, int r, int c, int pri, int sec, int damping, int dir) {
    int ssx = plane ? h->subsampling_x : 0, ssy = plane ? h->subsampling_y : 0;
    int coeff_shift = h->bit_depth - 8;
    int x0 = (c * 4) >> ssx, y0 = (r * 4) >> ssy, w = 8 >> ssx, hh = 8 >> ssy;
    int row = (pri >> coeff_shift) & 1;
    int pw = src->cols, ph = src->rows;
    for (int i = 0; i < hh; i++)
        for (int j = 0; j < w; j++) {
            int py = y0 + i, px = x0 + j;
            if (py < 0 || py >= ph || px < 0 || px >= pw) continue;
            int x = src->s[(size_t)py * pw + px];
            int sum = 0, mx = x, mn = x;
            for (int k = 0; k < 2; k++)
                for (int sgn = -1; sgn <= 1; sgn += 2) {
                    for (int t = 0; t < 3; t++) {
                        int d = t == 0 ? dir : ((dir + (t == 1 ? -2 : 2)) & 7);
                        int yy = y0 + i + sgn * CDEF_DIRECTIONS[d][k][0];
                        int xx = x0 + j + sgn * CDEF_DIRECTIONS[d][k][1];
                        if (yy < 0 || yy >= ph || xx < 0 || xx >= pw) continue;
                        int v = src->s[(size_t)yy * pw + xx];
                        if (t == 0) sum += CDEF_PRI_TAPS[row][k] * constrain(v - x, pri, damping);
                        else sum += CDEF_SEC_TAPS[row][k] * constrain(v - x, sec, damping);
                        if (v > mx) mx = v;
                        if (v < mn) mn = v;
                    }
                }
            int delta = (8 + sum - (sum < 0)) >> 4;
            dst->s[(size_t)py * dst->cols + px] = clip3(mn, mx, x + delta);
        }
}

static void cdef_copy(const ora_plane* src, ora_plane* dst, int r, int c, int ssx, int ssy) {
    int sy = (r * 4) >> ssy, ey = ((r + 2) * 4) >> ssy, sx = (c * 4) >> ssx, ex = ((c + 2) * 4) >> ssx;
    int cols = src->cols < dst->cols ? src->cols : dst->cols;
    int rows = src->rows < dst->rows ? src->rows : dst->rows;
    for (int y = sy; y < ey; y++) {
        if (y < 0 || y >= rows) continue;
        for (int x = sx; x < ex; x++) {
            if (x < 0 || x >= cols) continue;
            dst->s[(size_t)y * dst->cols + x] = src->s[(size_t)y * src->cols + x];
        }
    }
}

/* cdef_frame + cdef_block (cdef.rs:180-330). */
void ora_cdef_frame(const av1g_frame_header* h, const av1g_mi_grid* grid, const int8_t* cdef_idx,
                    const ora_plane src[3], ora_plane dst[3]) {
    int cdef_cols = (h->mi_cols + 15) >> 4;
    lf_ctx lc = {h, grid};
    for (int r = 0; r < h->mi_rows; r += 2)
        for (int c = 0; c < h->mi_cols; c += 2) {
            int br = r & ~15, bc = c & ~15;
            int idx = cdef_idx[(br >> 4) * cdef_cols + (bc >> 4)];
            cdef_copy(&src[0], &dst[0], r, c, 0, 0);
            if (h->num_planes > 1) {
                cdef_copy(&src[1], &dst[1], r, c, h->subsampling_x, h->subsampling_y);
                cdef_copy(&src[2], &dst[2], r, c, h->subsampling_x, h->subsampling_y);
            }
            if (idx < 0) continue;
            int cs = h->bit_depth - 8;
            int skip = g_skip(&lc, r, c) && (r + 1 >= h->mi_rows || g_skip(&lc, r + 1, c)) &&
                       (c + 1 >= h->mi_cols || g_skip(&lc, r, c + 1)) &&
                       (r + 1 >= h->mi_rows || c + 1 >= h->mi_cols || g_skip(&lc, r + 1, c + 1));
            if (skip) continue;
            int y_dir, var;
            cdef_direction(h, &src[0], r, c, &y_dir, &var);
            int pri_y = h->cdef_y_pri[idx] << cs, sec_y = h->cdef_y_sec[idx] << cs;
            int dir_y = pri_y == 0 ? 0 : y_dir;
            int var_str = (var >> 6) > 0 ? floor_log2((uint32_t)(var >> 6)) : 0;
            if (var_str > 12) var_str = 12;
            int pri_y_s = var != 0 ? (pri_y * (4 + var_str) + 8) >> 4 : 0;
            int damp_y = h->cdef_damping + cs;
            cdef_filter_block(h, &src[0], &dst[0], 0, r, c, pri_y_s, sec_y, damp_y, dir_y);
            if (h->num_planes == 1) continue;
            int pri_uv = h->cdef_uv_pri[idx] << cs, sec_uv = h->cdef_uv_sec[idx] << cs;
            int sx = h->subsampling_x ? 1 : 0, sy = h->subsampling_y ? 1 : 0;
            int dir_uv = pri_uv == 0 ? 0 : CDEF_UV_DIR[sx][sy][y_dir];
            int damp_uv = h->cdef_damping + cs - 1;
            cdef_filter_block(h, &src[1], &dst[1], 1, r, c, pri_uv, sec_uv, damp_uv, dir_uv);
            cdef_filter_block(h, &src[2], &dst[2], 2, r, c, pri_uv, sec_uv, damp_uv, dir_uv);
        }
}

/* ===================================================================== */
/* §7.16 superres                                                        */
/* ===================================================================== */

static uint32_t round2u(uint32_t x, int n) { return n == 0 ? x : (x + (1u << (n - 1))) >> n; }

/* upscale_plane + upscale_sample (superres.rs:326-445). */
static int upscale_plane(const av1g_frame_header* h, int plane, const ora_plane* in, ora_plane* out) {
    int ssx = plane ? h->subsampling_x : 0, ssy = plane ? h->subsampling_y : 0;
    int dw = (int)round2u((uint32_t)h->frame_width, ssx);
    int uw = (int)round2u((uint32_t)h->upscaled_width, ssx);
    int ph = (int)round2u((uint32_t)h->frame_height, ssy);
    if (in->rows < ph || in->cols < dw || out->rows != ph || out->cols != uw) return 1;
    if (uw == 0 || ph == 0) return 0;
    if (uw <= dw) return 1;
    int64_t stepx_num = ((int64_t)dw << 14) + uw / 2;
    int step_x = (int)(stepx_num / uw);
    int err = (int)((int64_t)uw * step_x - ((int64_t)dw << 14));
    int64_t diff = (int64_t)uw - dw;
    int64_t num = -(diff << 13) + uw / 2;
    int division = (int)(num / uw); /* truncates toward zero like Rust */
    int init = division + (1 << (8 - 1)) - err / 2;
    init &= (1 << 14) - 1;
    int mi_w = h->mi_cols >> ssx;
    int max_x = mi_w * 4 - 1;
    int maxv = (1 << h->bit_depth) - 1;
    for (int y = 0; y < ph; y++) {
        const int32_t* row = in->s + (size_t)y * in->cols;
        for (int x = 0; x < uw; x++) {
            int src_x = -(1 << 14) + init + x * step_x;
            int px = src_x >> 14;
            int sub = (src_x & ((1 << 14) - 1)) >> 8;
            int sum = 0;
            for (int k = 0; k < 8; k++) {
                int sxx = clip3(0, max_x, px + (k - 3));
                int idx = clip3(0, in->cols - 1, sxx);
                sum += row[idx] * UPSCALE_FILTER[sub & 63][k];
            }
            out->s[(size_t)y * out->cols + x] = clip3(0, maxv, round2(sum, 7));
        }
    }
    return 0;
}

int ora_upscale_frame(const av1g_frame_header* h, const ora_plane in[3], ora_plane out[3]) {
    for (int p = 0; p < h->num_planes; p++) {
        if (!h->use_superres || h->frame_width == h->upscaled_width) {
            if (in[p].rows != out[p].rows || in[p].cols != out[p].cols) return 1;
            memcpy(out[p].s, in[p].s, sizeof(int32_t) * (size_t)in[p].rows * in[p].cols);
            continue;
        }
        if (h->upscaled_width <= h->frame_width) return 1;
        if (upscale_plane(h, p, &in[p], &out[p])) return 1;
    }
    return 0;
}

/* ===================================================================== */
/* §7.17 loop restoration                                                */
/* ===================================================================== */

static const int SGR_PARAMS[16][4] = {                       /* loop_restoration.rs:165 */
    {2, 12, 1, 4}, {2, 15, 1, 6}, {2, 18, 1, 8}, {2, 21, 1, 9}, {2, 24, 1, 10}, {2, 29, 1, 11},
    {2, 36, 1, 12}, {2, 45, 1, 13}, {2, 56, 1, 14}, {2, 68, 1, 15}, {0, 0, 1, 5}, {0, 0, 1, 8},
    {0, 0, 1, 11}, {0, 0, 1, 14}, {2, 30, 0, 0}, {2, 75, 0, 0}};

typedef struct {
    int unit_row, unit_col, x, y, w, h, stripe_start, stripe_end, plane_end_x, plane_end_y;
} lr_geom;

static int count_units(int unit_size, int frame_size) {
    if (unit_size == 0) return 1;
    int n = (frame_size + (unit_size >> 1)) / unit_size;
    return n > 1 ? n : 1;
}

/* derive_block_geometry (loop_restoration.rs:370-428). */
static lr_geom lr_geometry(const av1g_frame_header* h, int plane, int row, int col) {
    lr_geom g;
    int luma_y = row * 4;
    int stripe_num = (luma_y + 8) / 64;
    int ssx = plane ? h->subsampling_x : 0, ssy = plane ? h->subsampling_y : 0;
    g.stripe_start = (-8 + stripe_num * 64) >> ssy;
    g.stripe_end = g.stripe_start + (64 >> ssy) - 1;
    int unit_size = h->lr_unit_size[plane] > 0 ? h->lr_unit_size[plane] : 1;
    int unit_rows = count_units(unit_size, (int)round2u((uint32_t)h->frame_height, ssy));
    int unit_cols = count_units(unit_size, (int)round2u((uint32_t)h->upscaled_width, ssx));
    int ur = ((row * 4 + 8) >> ssy) / unit_size;
    g.unit_row = ur < unit_rows - 1 ? ur : unit_rows - 1;
    int uc = ((col * 4) >> ssx) / unit_size;
    g.unit_col = uc < unit_cols - 1 ? uc : unit_cols - 1;
    g.plane_end_x = (int)round2u((uint32_t)h->upscaled_width, ssx) - 1;
    g.plane_end_y = (int)round2u((uint32_t)h->frame_height, ssy) - 1;
    g.x = (col * 4) >> ssx;
    g.y = (row * 4) >> ssy;
    int wr = g.plane_end_x + 1 - g.x, hr = g.plane_end_y + 1 - g.y;
    if (wr < 0) wr = 0;
    if (hr < 0) hr = 0;
    g.w = (4 >> ssx) < wr ? (4 >> ssx) : wr;
    g.h = (4 >> ssy) < hr ? (4 >> ssy) : hr;
    return g;
}

static int sample_at(const ora_plane* p, int x, int y) {
    if (p->rows == 0 || p->cols == 0) return 0;
    int yc = clip3(0, p->rows - 1, y), xc = clip3(0, p->cols - 1, x);
    return p->s[(size_t)yc * p->cols + xc];
}

/* get_source_sample (loop_restoration.rs:862-883). */
static int source_sample(const ora_plane* curr, const ora_plane* cdef, int x, int y, const lr_geom* g) {
    x = clip3(0, g->plane_end_x > 0 ? g->plane_end_x : 0, x);
    y = clip3(0, g->plane_end_y > 0 ? g->plane_end_y : 0, y);
    if (y < g->stripe_start) {
        if (y < g->stripe_start - 2) y = g->stripe_start - 2;
        return sample_at(curr, x, y);
    } else if (y > g->stripe_end) {
        if (y > g->stripe_end + 2) y = g->stripe_end + 2;
        return sample_at(curr, x, y);
    }
    return sample_at(cdef, x, y);
}

/* box_filter (loop_restoration.rs:594-736). f: h*w outputs. */
static void box_filter(const ora_plane* curr, const ora_plane* cdef, const lr_geom* g, int bd, int r,
                       int eps, int pass, int32_t* f) {
    int h = g->h, w = g->w;
    memset(f, 0, sizeof(int32_t) * (size_t)h * w);
    if (r == 0) return;
    int n = (2 * r + 1) * (2 * r + 1);
    int64_t n2e = (int64_t)n * n * eps;
    int64_t s = (((int64_t)1 << 20) + n2e / 2) / (n2e > 1 ? n2e : 1);
    int one_over_n = ((1 << 12) + n / 2) / n;
    int aw = w + 2;
    int32_t A[6 * 6], B[6 * 6];
    int bdsa = 2 * (bd - 8 > 0 ? bd - 8 : 0), bdsb = bd - 8 > 0 ? bd - 8 : 0;
    for (int i = -1; i <= h; i++)
        for (int j = -1; j <= w; j++) {
            int64_t a = 0, b = 0;
            for (int dy = -r; dy <= r; dy++)
                for (int dx = -r; dx <= r; dx++) {
                    int64_t c = source_sample(curr, cdef, g->x + j + dx, g->y + i + dy, g);
                    a += c * c;
                    b += c;
                }
            int a_r = (int)round2_64(a, bdsa);
            int d_r = (int)round2_64(b, bdsb);
            int64_t p = (int64_t)a_r * n - (int64_t)d_r * d_r;
            if (p < 0) p = 0;
            int z = (int)round2_64(p * s, 20);
            int a2 = z >= 255 ? 256 : (z == 0 ? 1 : ((z << 8) + z / 2) / (z + 1));
            int64_t b2 = (int64_t)(256 - a2) * b * one_over_n; /* raw box sum b, as the reference */
            A[(i + 1) * aw + (j + 1)] = a2;
            B[(i + 1) * aw + (j + 1)] = (int32_t)round2_64(b2, 12);
        }
    for (int i = 0; i < h; i++) {
        int shift = (pass == 0 && (i & 1)) ? 4 : 5;
        for (int j = 0; j < w; j++) {
            int64_t as = 0, bs = 0;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    int wt;
                    if (pass == 0) wt = ((i + dy) & 1) ? (dx == 0 ? 6 : 5) : 0;
                    else wt = (dx == 0 || dy == 0) ? 4 : 3;
                    int ai = (i + dy + 1) * aw + (j + dx + 1);
                    as += (int64_t)wt * A[ai];
                    bs += (int64_t)wt * B[ai];
                }
            int py = g->y + i, px = g->x + j;
            int64_t u = (py >= 0 && py < cdef->rows && px >= 0 && px < cdef->cols)
                            ? cdef->s[(size_t)py * cdef->cols + px] : 0;
            int64_t v = as * u + bs;
            f[i * w + j] = (int32_t)round2_64(v, 8 + shift - 4);
        }
    }
}

/* self_guided_filter (loop_restoration.rs:485-588). */
static void self_guided(const av1g_frame_header* hd, const av1g_lr_unit* u, const ora_plane* curr,
                        const ora_plane* cdef, ora_plane* lr, const lr_geom* g) {
    int set = u->sgr_set < 16 ? u->sgr_set : 15;
    int r0 = SGR_PARAMS[set][0], e0 = SGR_PARAMS[set][1], r1 = SGR_PARAMS[set][2], e1 = SGR_PARAMS[set][3];
    int w0 = u->sgr_xqd[0], w1 = u->sgr_xqd[1], w2 = (1 << 7) - w0 - w1;
    int32_t f0[16], f1[16];
    box_filter(curr, cdef, g, hd->bit_depth, r0, e0, 0, f0);
    box_filter(curr, cdef, g, hd->bit_depth, r1, e1, 1, f1);
    int maxv = (1 << hd->bit_depth) - 1;
    for (int i = 0; i < g->h; i++)
        for (int j = 0; j < g->w; j++) {
            int py = g->y + i, px = g->x + j;
            int uu = (py >= 0 && py < cdef->rows && px >= 0 && px < cdef->cols)
                         ? cdef->s[(size_t)py * cdef->cols + px] << 4 : 0;
            int v = w1 * uu;
            v += r0 ? w0 * f0[i * g->w + j] : w0 * uu;
            v += r1 ? w2 * f1[i * g->w + j] : w2 * uu;
            int s = round2(v, 4 + 7);
            if (py >= 0 && py < lr->rows && px >= 0 && px < lr->cols)
                lr->s[(size_t)py * lr->cols + px] = clip3(0, maxv, s);
        }
}

/* wiener_filter + wiener_coefficients (loop_restoration.rs:742-857). */
static void wiener(const av1g_frame_header* hd, const av1g_lr_unit* u, const ora_plane* curr,
                   const ora_plane* cdef, ora_plane* lr, const lr_geom* g) {
    int vf[7], hf[7];
    vf[3] = hf[3] = 128;
    for (int i = 0; i < 3; i++) {
        vf[i] = vf[6 - i] = u->wiener[0][i];
        vf[3] -= 2 * u->wiener[0][i];
        hf[i] = hf[6 - i] = u->wiener[1][i];
        hf[3] -= 2 * u->wiener[1][i];
    }
    int bd = hd->bit_depth;
    int r0 = bd == 12 ? 5 : 3, r1 = bd == 12 ? 9 : 11;
    int offset = 1 << (bd + 7 - r0 - 1);
    int limit = (1 << (bd + 1 + 7 - r0)) - 1;
    int32_t inter[10 * 4];
    int w = g->w, h = g->h;
    for (int r = 0; r < h + 6; r++)
        for (int c = 0; c < w; c++) {
            int s = 0;
            for (int t = 0; t < 7; t++)
                s += hf[t] * source_sample(curr, cdef, g->x + c + t - 3, g->y + r - 3, g);
            inter[r * w + c] = clip3(-offset, limit - offset, round2(s, r0));
        }
    int maxv = (1 << bd) - 1;
    for (int r = 0; r < h; r++)
        for (int c = 0; c < w; c++) {
            int s = 0;
            for (int t = 0; t < 7; t++) s += vf[t] * inter[(r + t) * w + c];
            int out = clip3(0, maxv, round2(s, r1));
            int dy = g->y + r, dx = g->x + c;
            if (dy < 0 || dy >= lr->rows || dx < 0 || dx >= lr->cols) continue;
            lr->s[(size_t)dy * lr->cols + dx] = out;
        }
}

/* loop_restoration_frame + loop_restore_block (loop_restoration.rs:268-470),
 * with lr_unit lookups as cdf.rs:20273 (RESTORE_NONE outside the grid). */
void ora_lr_frame(const av1g_frame_header* h, const av1g_lr_unit* const units[3],
                  const int32_t unit_rows[3], const int32_t unit_cols[3], const ora_plane curr[3],
                  const ora_plane cdef[3], ora_plane lr[3]) {
    for (int p = 0; p < h->num_planes; p++) {
        int rows = cdef[p].rows < lr[p].rows ? cdef[p].rows : lr[p].rows;
        int cols = cdef[p].cols < lr[p].cols ? cdef[p].cols : lr[p].cols;
        for (int y = 0; y < rows; y++)
            memcpy(lr[p].s + (size_t)y * lr[p].cols, cdef[p].s + (size_t)y * cdef[p].cols, sizeof(int32_t) * cols);
    }
    if (!h->uses_lr) return;
    for (int y = 0; y < h->frame_height; y += 4)
        for (int x = 0; x < h->upscaled_width; x += 4)
            for (int p = 0; p < h->num_planes; p++) {
                if (h->lr_type[p] == 0) continue;
                lr_geom g = lr_geometry(h, p, y >> 2, x >> 2);
                if (g.w == 0 || g.h == 0) continue;
                av1g_lr_unit none = {0};
                const av1g_lr_unit* u = &none;
                if (units[p] && g.unit_row < unit_rows[p] && g.unit_col < unit_cols[p])
                    u = &units[p][g.unit_row * unit_cols[p] + g.unit_col];
                if (u->type == 1) wiener(h, u, &curr[p], &cdef[p], &lr[p], &g);
                else if (u->type == 2) self_guided(h, u, &curr[p], &cdef[p], &lr[p], &g);
            }
}

/* ===================================================================== */
/* §7.18.3 film grain                                                    */
/* ===================================================================== */

/* RandomRegister::next (film_grain.rs:119-131). */
uint32_t ora_random_next(uint16_t* state, int bits) {
    uint32_t r = *state;
    uint32_t bit = (r ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1;
    r = (r >> 1) | (bit << 15);
    *state = (uint16_t)r;
    return (r >> (16 - bits)) & ((1u << bits) - 1);
}

/* generate_grain (film_grain.rs:230-400). */
void ora_generate_grain(const av1g_film_grain* fg, int bd, int ssx, int ssy, int32_t* luma,
                        int32_t* cb, int32_t* cr) {
    const int LW = 82, LH = 73;
    int center = 128 << (bd - 8), gmin = -center, gmax = (256 << (bd - 8)) - 1 - center;
    int shift = 12 - bd + fg->grain_scale_shift;
    uint16_t st = fg->grain_seed;
    for (int y = 0; y < LH; y++)
        for (int x = 0; x < LW; x++) {
            int g = 0;
            if (fg->num_y_points > 0) g = GAUSSIAN_SEQUENCE[ora_random_next(&st, 11)];
            luma[y * LW + x] = round2(g, shift);
        }
    int lag = fg->ar_coeff_lag;
    if (fg->num_y_points > 0) {
        for (int y = 3; y < LH; y++)
            for (int x = 3; x < LW - 3; x++) {
                int s = 0, pos = 0;
                for (int dr = -lag; dr <= 0; dr++)
                    for (int dc = -lag; dc <= lag; dc++) {
                        if (dr == 0 && dc == 0) goto done_l;
                        s += luma[(y + dr) * LW + x + dc] * (fg->ar_coeffs_y_plus_128[pos] - 128);
                        pos++;
                    }
            done_l:
                luma[y * LW + x] = clip3(gmin, gmax, luma[y * LW + x] + round2(s, fg->ar_coeff_shift));
            }
    }
    int cw = ssx ? 44 : 82, ch = ssy ? 38 : 73;
    int any_c = fg->num_cb_points > 0 || fg->chroma_scaling_from_luma;
    st = fg->grain_seed ^ 0xb524;
    for (int y = 0; y < ch; y++)
        for (int x = 0; x < cw; x++) {
            int g = any_c ? GAUSSIAN_SEQUENCE[ora_random_next(&st, 11)] : 0;
            cb[y * cw + x] = round2(g, shift);
        }
    any_c = fg->num_cr_points > 0 || fg->chroma_scaling_from_luma;
    st = fg->grain_seed ^ 0x49d8;
    for (int y = 0; y < ch; y++)
        for (int x = 0; x < cw; x++) {
            int g = any_c ? GAUSSIAN_SEQUENCE[ora_random_next(&st, 11)] : 0;
            cr[y * cw + x] = round2(g, shift);
        }
    if (fg->chroma_scaling_from_luma || fg->num_cb_points > 0 || fg->num_cr_points > 0) {
        for (int y = 3; y < ch; y++)
            for (int x = 3; x < cw - 3; x++) {
                int s0 = 0, s1 = 0, pos = 0;
                for (int dr = -lag; dr <= 0; dr++)
                    for (int dc = -lag; dc <= lag; dc++) {
                        int c0 = fg->ar_coeffs_cb_plus_128[pos] - 128;
                        int c1 = fg->ar_coeffs_cr_plus_128[pos] - 128;
                        if (dr == 0 && dc == 0) {
                            if (fg->num_y_points > 0) {
                                int lx = ((x - 3) << ssx) + 3, ly = ((y - 3) << ssy) + 3, l = 0;
                                for (int i = 0; i <= ssy; i++)
                                    for (int j = 0; j <= ssx; j++) l += luma[(ly + i) * LW + lx + j];
                                l = round2(l, ssx + ssy);
                                s0 += l * c0;
                                s1 += l * c1;
                            }
                            goto done_c;
                        }
                        s0 += cb[(y + dr) * cw + x + dc] * c0;
                        s1 += cr[(y + dr) * cw + x + dc] * c1;
                        pos++;
                    }
            done_c:
                cb[y * cw + x] = clip3(gmin, gmax, cb[y * cw + x] + round2(s0, fg->ar_coeff_shift));
                cr[y * cw + x] = clip3(gmin, gmax, cr[y * cw + x] + round2(s1, fg->ar_coeff_shift));
            }
    }
}

/* scaling_lookup_fill (film_grain.rs:490-540). */
static void scaling_fill(uint8_t* t, int np, const uint8_t* xv, const uint8_t* yv) {
    if (np == 0) { memset(t, 0, 256); return; }
    for (int v = 0; v < xv[0] && v < 256; v++) t[v] = yv[0];
    for (int i = 0; i + 1 < np; i++) {
        int dx = xv[i + 1] - xv[i], dy = yv[i + 1] - yv[i];
        if (dx <= 0) continue;
        int delta = dy * ((65536 + (dx >> 1)) / dx);
        for (int x = 0; x < dx; x++) {
            int v = yv[i] + ((x * delta + 32768) >> 16);
            int idx = xv[i] + x;
            if (idx < 256) t[idx] = (uint8_t)clip3(0, 255, v);
        }
    }
    for (int v = xv[np - 1]; v < 256; v++) t[v] = yv[np - 1];
}

/* scaling_lookup_init (film_grain.rs:418-470). */
void ora_scaling_lookup_init(const av1g_film_grain* fg, int num_planes, uint8_t lut[3][256]) {
    memset(lut, 0, 3 * 256);
    for (int p = 0; p < num_planes && p < 3; p++) {
        if (p == 0 || fg->chroma_scaling_from_luma)
            scaling_fill(lut[p], fg->num_y_points, fg->point_y_value, fg->point_y_scaling);
        else if (p == 1)
            scaling_fill(lut[p], fg->num_cb_points, fg->point_cb_value, fg->point_cb_scaling);
        else
            scaling_fill(lut[p], fg->num_cr_points, fg->point_cr_value, fg->point_cr_scaling);
    }
}

/* scale_lut (film_grain.rs:543-556). */
static int scale_lut(uint8_t lut[3][256], int plane, int index, int bd) {
    int shift = bd - 8;
    int x = index >> shift;
    if (bd == 8 || x >= 255) return lut[plane][x < 255 ? x : 255];
    int rem = index - (x << shift);
    int start = lut[plane][x], end = lut[plane][x + 1];
    return start + round2((end - start) * rem, shift);
}

/* add_noise_synthesis (film_grain.rs:570-829). */
static void add_noise(const av1g_film_grain* fg, const int32_t* gl, const int32_t* gcb,
                      const int32_t* gcr, int cw, uint8_t lut[3][256], int bd, int num_planes,
                      int ssx, int ssy, int mc, ora_plane* out) {
    int w = out[0].cols, h = out[0].rows;
    if (w == 0 || h == 0) return;
    int center = 128 << (bd - 8), gmin = -center, gmax = (256 << (bd - 8)) - 1 - center;
    int np = num_planes < 3 ? num_planes : 3;
    int nstripes = ((h + 1) / 2 + 15) / 16;
    int sh[3], sw[3];
    for (int p = 0; p < np; p++) {
        int psx = p ? ssx : 0, psy = p ? ssy : 0;
        sh[p] = 34 >> psy;
        sw[p] = ((w + psx) >> psx) + 34;
    }
    int32_t* stripes[3];
    for (int p = 0; p < np; p++) stripes[p] = (int32_t*)calloc((size_t)nstripes * sh[p] * sw[p], sizeof(int32_t));
    int luma_num = 0;
    for (int ys = 0; ys < (h + 1) / 2; ys += 16, luma_num++) {
        uint16_t st = fg->grain_seed;
        st ^= (uint16_t)((((uint32_t)luma_num * 37 + 178) & 255) << 8);
        st ^= (uint16_t)(((uint32_t)luma_num * 173 + 105) & 255);
        for (int xb = 0; xb < (w + 1) / 2; xb += 16) {
            uint32_t rnd = ora_random_next(&st, 8);
            int ox = rnd >> 4, oy = rnd & 15;
            for (int p = 0; p < np; p++) {
                int psx = p ? ssx : 0, psy = p ? ssy : 0;
                int pox = psx ? 6 + ox : 9 + ox * 2, poy = psy ? 6 + oy : 9 + oy * 2;
                int32_t* ns = stripes[p] + (size_t)luma_num * sh[p] * sw[p];
                for (int i = 0; i < (34 >> psy); i++)
                    for (int j = 0; j < (34 >> psx); j++) {
                        int yi = poy + i, xi = pox + j;
                        int g = p == 0 ? gl[yi * 82 + xi] : (p == 1 ? gcb[yi * cw + xi] : gcr[yi * cw + xi]);
                        if (psx == 0) {
                            int col = xb * 2 + j;
                            if (j < 2 && fg->overlap_flag && xb > 0) {
                                int old = ns[i * sw[p] + col];
                                g = j == 0 ? old * 27 + g * 17 : old * 17 + g * 27;
                                g = clip3(gmin, gmax, round2(g, 5));
                            }
                            if (col < sw[p]) ns[i * sw[p] + col] = g;
                        } else {
                            int col = xb + j;
                            if (j == 0 && fg->overlap_flag && xb > 0) {
                                int old = ns[i * sw[p] + col];
                                g = old * 23 + g * 22;
                                g = clip3(gmin, gmax, round2(g, 5));
                            }
                            if (col < sw[p]) ns[i * sw[p] + col] = g;
                        }
                    }
            }
        }
    }
    int32_t* img[3];
    for (int p = 0; p < np; p++) {
        int psx = p ? ssx : 0, psy = p ? ssy : 0;
        int ph = (h + psy) >> psy, pw = (w + psx) >> psx;
        img[p] = (int32_t*)calloc((size_t)ph * pw, sizeof(int32_t));
        for (int yy = 0; yy < ph; yy++) {
            int si = yy >> (5 - psy);
            int i = yy - (si << (5 - psy));
            if (si >= nstripes) continue;
            const int32_t* cur = stripes[p] + (size_t)si * sh[p] * sw[p];
            for (int xx = 0; xx < pw; xx++) {
                int g = cur[i * sw[p] + xx];
                if (psy == 0) {
                    if (i < 2 && si > 0 && fg->overlap_flag) {
                        int old = stripes[p][(size_t)(si - 1) * sh[p] * sw[p] + (i + 32) * sw[p] + xx];
                        g = i == 0 ? old * 27 + g * 17 : old * 17 + g * 27;
                        g = clip3(gmin, gmax, round2(g, 5));
                    }
                } else if (i < 1 && si > 0 && fg->overlap_flag) {
                    int old = stripes[p][(size_t)(si - 1) * sh[p] * sw[p] + (i + 16) * sw[p] + xx];
                    g = old * 23 + g * 22;
                    g = clip3(gmin, gmax, round2(g, 5));
                }
                img[p][yy * pw + xx] = g;
            }
        }
    }
    int minv, maxl, maxc;
    if (fg->clip_to_restricted_range) {
        minv = 16 << (bd - 8);
        maxl = 235 << (bd - 8);
        maxc = mc == 0 ? maxl : 240 << (bd - 8);
    } else {
        minv = 0;
        maxl = maxc = (256 << (bd - 8)) - 1;
    }
    int sshift = fg->grain_scaling;
    if (np >= 3 && (fg->num_cb_points > 0 || fg->num_cr_points > 0 || fg->chroma_scaling_from_luma)) {
        int pwc = (w + ssx) >> ssx, phc = (h + ssy) >> ssy;
        for (int yy = 0; yy < phc; yy++)
            for (int xx = 0; xx < pwc; xx++) {
                int lx = xx << ssx, ly = yy << ssy;
                int lnx = lx + 1 < w - 1 ? lx + 1 : w - 1;
                const int32_t* Y = out[0].s;
                int avg = ssx ? round2(Y[(size_t)ly * out[0].cols + lx] + Y[(size_t)ly * out[0].cols + lnx], 1)
                              : Y[(size_t)ly * out[0].cols + lx];
                for (int p = 1; p <= 2; p++) {
                    int np_ = p == 1 ? fg->num_cb_points : fg->num_cr_points;
                    if (!(np_ > 0 || fg->chroma_scaling_from_luma)) continue;
                    int32_t* o = &out[p].s[(size_t)yy * out[p].cols + xx];
                    int orig = *o, merged;
                    if (fg->chroma_scaling_from_luma) merged = avg;
                    else {
                        int lm = p == 1 ? fg->cb_luma_mult : fg->cr_luma_mult;
                        int m = p == 1 ? fg->cb_mult : fg->cr_mult;
                        int off = p == 1 ? fg->cb_offset : fg->cr_offset;
                        int comb = avg * (lm - 128) + orig * (m - 128);
                        merged = clip3(0, (1 << bd) - 1, (comb >> 6) + ((off - 256) * (1 << (bd - 8))));
                    }
                    int noise = img[p][yy * pwc + xx];
                    noise = round2(scale_lut(lut, p, merged, bd) * noise, sshift);
                    *o = clip3(minv, maxc, orig + noise);
                }
            }
    }
    if (fg->num_y_points > 0)
        for (int yy = 0; yy < h; yy++)
            for (int xx = 0; xx < w; xx++) {
                int32_t* o = &out[0].s[(size_t)yy * out[0].cols + xx];
                int orig = *o;
                int noise = round2(scale_lut(lut, 0, orig, bd) * img[0][yy * w + xx], sshift);
                *o = clip3(minv, maxl, orig + noise);
            }
    for (int p = 0; p < np; p++) { free(stripes[p]); free(img[p]); }
}

void ora_film_grain(const av1g_film_grain* fg, int bd, int num_planes, int ssx, int ssy, int mc,
                    ora_plane out[3]) {
    if (!fg->apply_grain) return;
    int32_t luma[73 * 82], cb[73 * 82], cr[73 * 82];
    ora_generate_grain(fg, bd, ssx, ssy, luma, cb, cr);
    uint8_t lut[3][256];
    ora_scaling_lookup_init(fg, num_planes, lut);
    add_noise(fg, luma, cb, cr, ssx ? 44 : 82, lut, bd, num_planes, ssx, ssy, mc, out);
}

/* ===================================================================== */
/* Chain (frame_driver.rs:790-1116)                                       */
/* ===================================================================== */

int ora_postfilter_frame(const av1g_frame_header* h, const av1g_mi_grid* grid,
                         const int8_t* cdef_idx, const av1g_lr_unit* const units[3],
                         const int32_t* const recon[3], int32_t* ref_out[3], int32_t* out[3]) {
    int np = h->num_planes;
    if (np != 1 && np != 3) return 1;
    int ssx = h->subsampling_x, ssy = h->subsampling_y;
    ora_plane cur[3], deb[3];
    int pw[3], ph[3];
    for (int p = 0; p < np; p++) {
        pw[p] = (h->mi_cols * 4) >> (p ? ssx : 0);
        ph[p] = (h->mi_rows * 4) >> (p ? ssy : 0);
        size_t n = (size_t)pw[p] * ph[p];
        cur[p].s = (int32_t*)malloc(n * sizeof(int32_t));
        memcpy(cur[p].s, recon[p], n * sizeof(int32_t));
        cur[p].rows = ph[p];
        cur[p].cols = pw[p];
        deb[p].s = NULL;
    }
    /* §7.4 step 1 gate (frame_driver.rs:832-836) */
    if ((h->lf_level[0] != 0 || h->lf_level[1] != 0) && !h->coded_lossless && !h->allow_intrabc)
        ora_loop_filter_frame(h, grid, cur);
    if (h->uses_lr)
        for (int p = 0; p < np; p++) {
            size_t n = (size_t)pw[p] * ph[p];
            deb[p] = cur[p];
            deb[p].s = (int32_t*)malloc(n * sizeof(int32_t));
            memcpy(deb[p].s, cur[p].s, n * sizeof(int32_t));
        }
    /* CDEF gate (frame_driver.rs:870) */
    if (!h->coded_lossless && !h->allow_intrabc && h->enable_cdef && !h->cdef_short_circuited) {
        ora_plane src[3];
        for (int p = 0; p < np; p++) {
            size_t n = (size_t)pw[p] * ph[p];
            src[p] = cur[p];
            src[p].s = (int32_t*)malloc(n * sizeof(int32_t));
            memcpy(src[p].s, cur[p].s, n * sizeof(int32_t));
        }
        ora_cdef_frame(h, grid, cdef_idx, src, cur);
        for (int p = 0; p < np; p++) free(src[p].s);
    }
    /* superres (frame_driver.rs:906-966) */
    if (h->use_superres && h->upscaled_width > h->frame_width) {
        ora_plane up[3], upd[3];
        for (int p = 0; p < np; p++) {
            int ow = p ? (h->upscaled_width + ssx) >> ssx : h->upscaled_width;
            int oh = p ? (h->frame_height + ssy) >> ssy : h->frame_height;
            up[p].rows = upd[p].rows = oh;
            up[p].cols = upd[p].cols = ow;
            up[p].s = (int32_t*)calloc((size_t)ow * oh, sizeof(int32_t));
            upd[p].s = h->uses_lr ? (int32_t*)calloc((size_t)ow * oh, sizeof(int32_t)) : NULL;
        }
        if (ora_upscale_frame(h, cur, up)) return 2;
        if (h->uses_lr && ora_upscale_frame(h, deb, upd)) return 2;
        for (int p = 0; p < np; p++) {
            free(cur[p].s);
            cur[p] = up[p];
            if (h->uses_lr) { free(deb[p].s); deb[p] = upd[p]; }
            pw[p] = up[p].cols;
            ph[p] = up[p].rows;
        }
    }
    /* loop restoration (frame_driver.rs:971-1011) */
    if (h->uses_lr) {
        ora_plane lr[3];
        int32_t urows[3] = {0, 0, 0}, ucols[3] = {0, 0, 0};
        for (int p = 0; p < np; p++) {
            lr[p] = cur[p];
            lr[p].s = (int32_t*)malloc((size_t)pw[p] * ph[p] * sizeof(int32_t));
            int us = h->lr_unit_size[p] > 0 ? h->lr_unit_size[p] : 1;
            urows[p] = count_units(us, (int)round2u((uint32_t)h->frame_height, p ? ssy : 0));
            ucols[p] = count_units(us, (int)round2u((uint32_t)h->upscaled_width, p ? ssx : 0));
        }
        ora_lr_frame(h, units, urows, ucols, deb, cur, lr);
        for (int p = 0; p < np; p++) {
            free(cur[p].s);
            free(deb[p].s);
            cur[p] = lr[p];
        }
    }
    /* crop (frame_driver.rs:1018-1042) and the pre-grain store payload */
    ora_plane o[3];
    for (int p = 0; p < np; p++) {
        int ow = p ? (h->upscaled_width + ssx) >> ssx : h->upscaled_width;
        int oh = p ? (h->frame_height + ssy) >> ssy : h->frame_height;
        if (cur[p].cols < ow || cur[p].rows < oh) return 3;
        for (int y = 0; y < oh; y++) {
            memcpy(ref_out[p] + (size_t)y * ow, cur[p].s + (size_t)y * cur[p].cols, sizeof(int32_t) * ow);
            memcpy(out[p] + (size_t)y * ow, cur[p].s + (size_t)y * cur[p].cols, sizeof(int32_t) * ow);
        }
        for (size_t i = 0; i < (size_t)ow * oh; i++) if (ref_out[p][i] < 0) ref_out[p][i] = 0;
        o[p].s = out[p];
        o[p].rows = oh;
        o[p].cols = ow;
        free(cur[p].s);
    }
    /* film grain on the output copy (frame_driver.rs:1060-1096) */
    ora_film_grain(&h->film_grain, h->bit_depth, np, ssx, ssy, h->matrix_coefficients, o);
    /* narrow (frame_driver.rs:1101-1116) */
    int maxv = (1 << h->bit_depth) - 1;
    for (int p = 0; p < np; p++)
        for (size_t i = 0; i < (size_t)o[p].rows * o[p].cols; i++) out[p][i] = clip3(0, maxv, out[p][i]);
    return 0;
}

/* ===================================================================== */
/* Internals exposed for the known-answer tests that restate the         */
/* reference's module unit tests (loop_filter.rs, cdef.rs,               */
/* loop_restoration.rs tests).                                           */
/* ===================================================================== */

void ora_lf_strength(const av1g_frame_header* hdr, const av1g_mi_grid* grid, int row, int col, int plane,
                     int pass, int32_t out[4]) {
    lf_ctx c = {hdr, grid};
    lf_strength s = filter_strength(&c, row, col, plane, pass);
    out[0] = s.lvl;
    out[1] = s.limit;
    out[2] = s.blimit;
    out[3] = s.thresh;
}

int ora_lf_filter_size(int tx, int prev_tx, int pass, int plane) {
    int base = pass == 0 ? (TXW[tx] < TXW[prev_tx] ? TXW[tx] : TXW[prev_tx])
                         : (TXH[tx] < TXH[prev_tx] ? TXH[tx] : TXH[prev_tx]);
    int cap = plane == 0 ? 16 : 8;
    return base < cap ? base : cap;
}

void ora_lf_narrow(ora_plane* p, int x, int y, int dx, int dy, int hev, int bd) {
    narrow_filter(p, x, y, dx, dy, hev, bd);
}

void ora_lf_wide(ora_plane* p, int x, int y, int plane, int dx, int dy, int log2_size) {
    wide_filter(p, x, y, plane, dx, dy, log2_size);
}

int ora_cdef_constrain(int diff, int threshold, int damping) { return constrain(diff, threshold, damping); }

void ora_cdef_direction(const av1g_frame_header* hdr, const ora_plane* p0, int r, int c, int32_t out[2]) {
    int d, v;
    cdef_direction(hdr, p0, r, c, &d, &v);
    out[0] = d;
    out[1] = v;
}

int ora_lr_count_units(int unit_size, int frame_size) { return count_units(unit_size, frame_size); }

void ora_lr_geometry(const av1g_frame_header* hdr, int plane, int row, int col, int32_t out[10]) {
    lr_geom g = lr_geometry(hdr, plane, row, col);
    int32_t v[10] = {g.unit_row, g.unit_col, g.x, g.y, g.w, g.h, g.stripe_start, g.stripe_end, g.plane_end_x,
                     g.plane_end_y};
    memcpy(out, v, sizeof v);
}

int ora_lr_source_sample(const av1g_frame_header* hdr, int plane, int row, int col, const ora_plane* curr,
                         const ora_plane* cdef, int x, int y) {
    lr_geom g = lr_geometry(hdr, plane, row, col);
    return source_sample(curr, cdef, x, y, &g);
}
