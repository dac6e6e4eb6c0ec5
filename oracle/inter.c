/*
 * inter.c — CPU restatement of the reference's §7.11.3 inter prediction.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Every function follows the
 * reference's per-block formulation in src/inter_pred.rs, cited at each
 * definition; the driver at the bottom executes av1g_inter_pred calls in
 * list order the way the reference's reconstruct_inter_block* functions do
 * (predict into a w x h buffer, then copy the part inside the plane).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "av1_spec_tables.h"

static const AV1T_SUBPEL_FILTERS_TYPE SUBPEL AV1T_SUBPEL_FILTERS_DIMS = AV1T_SUBPEL_FILTERS_INIT;
static const AV1T_WARPED_FILTERS_TYPE WARPED AV1T_WARPED_FILTERS_DIMS = AV1T_WARPED_FILTERS_INIT;
static const AV1T_DIV_LUT_TYPE DIV_LUT AV1T_DIV_LUT_DIMS = AV1T_DIV_LUT_INIT;
static const AV1T_WEDGE_CODEBOOK_TYPE CODEBOOK AV1T_WEDGE_CODEBOOK_DIMS = AV1T_WEDGE_CODEBOOK_INIT;
static const AV1T_WEDGE_MASTER_OBLIQUE_ODD_TYPE M_ODD AV1T_WEDGE_MASTER_OBLIQUE_ODD_DIMS =
    AV1T_WEDGE_MASTER_OBLIQUE_ODD_INIT;
static const AV1T_WEDGE_MASTER_OBLIQUE_EVEN_TYPE M_EVEN AV1T_WEDGE_MASTER_OBLIQUE_EVEN_DIMS =
    AV1T_WEDGE_MASTER_OBLIQUE_EVEN_INIT;
static const AV1T_WEDGE_MASTER_VERTICAL_TYPE M_VERT AV1T_WEDGE_MASTER_VERTICAL_DIMS =
    AV1T_WEDGE_MASTER_VERTICAL_INIT;
static const AV1T_WEDGE_BITS_TYPE WEDGE_BITS AV1T_WEDGE_BITS_DIMS = AV1T_WEDGE_BITS_INIT;
static const AV1T_II_WEIGHTS_1D_TYPE II_W AV1T_II_WEIGHTS_1D_DIMS = AV1T_II_WEIGHTS_1D_INIT;
static const AV1T_OBMC_MASK_2_TYPE OM2 AV1T_OBMC_MASK_2_DIMS = AV1T_OBMC_MASK_2_INIT;
static const AV1T_OBMC_MASK_4_TYPE OM4 AV1T_OBMC_MASK_4_DIMS = AV1T_OBMC_MASK_4_INIT;
static const AV1T_OBMC_MASK_8_TYPE OM8 AV1T_OBMC_MASK_8_DIMS = AV1T_OBMC_MASK_8_INIT;
static const AV1T_OBMC_MASK_16_TYPE OM16 AV1T_OBMC_MASK_16_DIMS = AV1T_OBMC_MASK_16_INIT;
static const AV1T_OBMC_MASK_32_TYPE OM32 AV1T_OBMC_MASK_32_DIMS = AV1T_OBMC_MASK_32_INIT;
static const AV1T_NUM_4X4_BLOCKS_WIDE_TYPE N4W AV1T_NUM_4X4_BLOCKS_WIDE_DIMS = AV1T_NUM_4X4_BLOCKS_WIDE_INIT;
static const AV1T_NUM_4X4_BLOCKS_HIGH_TYPE N4H AV1T_NUM_4X4_BLOCKS_HIGH_DIMS = AV1T_NUM_4X4_BLOCKS_HIGH_INIT;

#define ERR (-1)

static int64_t rnd2(int64_t x, int n) { return n == 0 ? x : (x + ((int64_t)1 << (n - 1))) >> n; }
/* round2_signed, inter_pred.rs:256 */
static int64_t rnd2s(int64_t x, int n) {
    if (n == 0) return x;
    return x >= 0 ? (x + ((int64_t)1 << (n - 1))) >> n : -((-x + ((int64_t)1 << (n - 1))) >> n);
}
static int32_t clip3(int32_t lo, int32_t hi, int32_t v) { return v < lo ? lo : (v > hi ? hi : v); }
static int64_t clip3l(int64_t lo, int64_t hi, int64_t v) { return v < lo ? lo : (v > hi ? hi : v); }

/* rounding_variables, inter_pred.rs:205 */
static void rounding(int bd, int compound, int* r0, int* r1, int* post) {
    *r0 = 3;
    *r1 = compound ? 7 : 11;
    if (bd == 12) {
        *r0 += 2;
        if (!compound) *r1 -= 2;
    }
    *post = 14 - (*r0 + *r1);
}

/* motion_vector_scaling, inter_pred.rs:318 */
static int mv_scaling(int plane, int ssx, int ssy, int64_t fw, int64_t fh, int64_t ruw, int64_t rh, int x,
                      int y, const int16_t mv[2], int32_t out[4]) {
    if (fw <= 0 || fh <= 0 || ruw <= 0 || rh <= 0) return ERR;
    int64_t xs = ((ruw << 14) + fw / 2) / fw;
    int64_t ys = ((rh << 14) + fh / 2) / fh;
    int sx = plane ? ssx : 0, sy = plane ? ssy : 0;
    int64_t half = 8;
    int64_t ox = ((int64_t)x << 4) + ((2 * (int64_t)mv[1]) >> sx) + half;
    int64_t oy = ((int64_t)y << 4) + ((2 * (int64_t)mv[0]) >> sy) + half;
    int64_t bx = ox * xs - (half << 14);
    int64_t by = oy * ys - (half << 14);
    int64_t off = (1 << 6) / 2;
    out[0] = (int32_t)(rnd2s(bx, 8) + off);
    out[1] = (int32_t)(rnd2s(by, 8) + off);
    out[2] = (int32_t)rnd2s(xs, 4);
    out[3] = (int32_t)rnd2s(ys, 4);
    return 0;
}

/* select_interp_filter_small_block, inter_pred.rs:550 */
static int small_filter(int f) {
    if (f == 0 || f == 2) return 4;
    if (f == 1) return 5;
    return f;
}

typedef struct {
    const ora_plane* p;   /* this plane of the reference */
    int32_t uw, h;        /* luma RefUpscaledWidth / RefFrameHeight */
} ref_view;

/* block_inter_prediction, inter_pred.rs:654 */
static int block_inter(int plane, int ssx, int ssy, ref_view r, int32_t sx, int32_t sy, int32_t stx, int32_t sty,
                       int w, int h, int fx, int fy, int r0, int r1, int32_t* pred) {
    int gx = plane ? ssx : 0, gy = plane ? ssy : 0;
    int pw = (r.uw + gx) >> gx, ph = (r.h + gy) >> gy;
    if (r.uw <= 0 || r.h <= 0 || r.p->cols < pw || r.p->rows < ph) return ERR;
    if (w <= 0 || h <= 0 || w > 256 || h > 256 || stx <= 0 || sty <= 0) return ERR;
    if (fx >= 6 || fy >= 6) return ERR;
    int last_x = pw - 1, last_y = ph - 1;
    int64_t ih = ((((int64_t)h - 1) * sty + (1 << 10) - 1) >> 10) + 8;
    int hf = w <= 4 ? small_filter(fx) : fx;
    int vf = h <= 4 ? small_filter(fy) : fy;
    int32_t* im = (int32_t*)malloc(sizeof(int32_t) * (size_t)ih * (size_t)w);
    int ybase = (sy >> 10) - 3;
    for (int64_t rr = 0; rr < ih; rr++) {
        const int32_t* row = r.p->s + (size_t)clip3(0, last_y, ybase + (int32_t)rr) * r.p->cols;
        for (int c = 0; c < w; c++) {
            int32_t p = sx + stx * c;
            int phase = (p >> 6) & 15;
            int pint = p >> 10;
            int64_t s = 0;
            for (int t = 0; t < 8; t++)
                s += (int64_t)SUBPEL[hf][phase][t] * row[clip3(0, last_x, pint + t - 3)];
            im[rr * w + c] = (int32_t)rnd2(s, r0);
        }
    }
    for (int rr = 0; rr < h; rr++) {
        int32_t p = (sy & 1023) + sty * rr;
        int phase = (p >> 6) & 15;
        int pint = p >> 10;
        for (int c = 0; c < w; c++) {
            int64_t s = 0;
            for (int t = 0; t < 8; t++) s += (int64_t)SUBPEL[vf][phase][t] * im[(size_t)(pint + t) * w + c];
            pred[rr * w + c] = (int32_t)rnd2(s, r1);
        }
    }
    free(im);
    return 0;
}

/* resolve_divisor, inter_pred.rs:3885 */
static int resolve_divisor(int32_t d, int32_t* factor, int* shift) {
    if (d == 0) return ERR;
    uint32_t a = d < 0 ? (uint32_t)(-(int64_t)d) : (uint32_t)d;
    int n = 31 - __builtin_clz(a);
    int64_t e = (int64_t)a - ((int64_t)1 << n);
    int64_t f = n > 8 ? (e + ((int64_t)1 << (n - 8 - 1))) >> (n - 8) : e << (8 - n);
    if (f > 256) f = 256;
    *factor = d < 0 ? -DIV_LUT[f] : DIV_LUT[f];
    *shift = n + 14;
    return 0;
}

static int64_t sat_mul(int64_t a, int64_t b) {
    __int128 p = (__int128)a * b;
    if (p > INT64_MAX) return INT64_MAX;
    if (p < INT64_MIN) return INT64_MIN;
    return (int64_t)p;
}

/* setup_shear, inter_pred.rs:3982.  Returns 0 (Some) or ERR (None). */
static int setup_shear(const int32_t p[6], int* valid, int32_t abcd[4]) {
    int32_t alpha0 = clip3(-32768, 32767, p[2] - (1 << 16));
    int32_t beta0 = clip3(-32768, 32767, p[3]);
    int32_t fac;
    int sh;
    if (resolve_divisor(p[2], &fac, &sh)) return ERR;
    int64_t v = (int64_t)p[4] * 65536;
    int32_t gamma0 = clip3(-32768, 32767, (int32_t)rnd2s(sat_mul(v, fac), sh));
    int64_t w = (int64_t)p[3] * p[4];
    int32_t corr = (int32_t)rnd2s(sat_mul(w, fac), sh);
    int32_t draw = (int32_t)((uint32_t)p[5] - (uint32_t)corr - (uint32_t)(1 << 16));
    int32_t delta0 = clip3(-32768, 32767, draw);
#define REDUCE(x) ((int32_t)rnd2s((x), 6) * 64)
    abcd[0] = REDUCE(alpha0);
    abcd[1] = REDUCE(beta0);
    abcd[2] = REDUCE(gamma0);
    abcd[3] = REDUCE(delta0);
#undef REDUCE
    *valid = 4 * abs(abcd[0]) + 7 * abs(abcd[1]) < (1 << 16) && 4 * abs(abcd[2]) + 4 * abs(abcd[3]) < (1 << 16);
    return 0;
}

/* block_warp, inter_pred.rs:4276 */
static int block_warp(int plane, int ssx, int ssy, int x, int y, int i8b, int j8b, int w, int h, ref_view r,
                      const int32_t wp[6], int r0, int r1, int32_t* pred) {
    if (w <= 0 || h <= 0 || w > 128 || h > 128) return ERR;
    if (r.uw <= 0 || r.h <= 0) return ERR;
    int sub_x = plane ? ssx : 0, sub_y = plane ? ssy : 0;
    int last_x = ((r.uw + sub_x) >> sub_x) - 1;
    int last_y = ((r.h + sub_y) >> sub_y) - 1;
    if (last_x >= r.p->cols || last_y + 1 > r.p->rows) return ERR;
    int32_t src_x = (x + j8b * 8 + 4) << sub_x;
    int32_t src_y = (y + i8b * 8 + 4) << sub_y;
    int64_t dst_x = (int64_t)wp[2] * src_x + (int64_t)wp[3] * src_y + wp[0];
    int64_t dst_y = (int64_t)wp[4] * src_x + (int64_t)wp[5] * src_y + wp[1];
    int valid;
    int32_t sh[4];
    if (setup_shear(wp, &valid, sh)) return ERR;
    int64_t alpha = sh[0], beta = sh[1], gamma = sh[2], delta = sh[3];
    int64_t x4 = dst_x >> sub_x, y4 = dst_y >> sub_y;
    int32_t ix4 = (int32_t)(x4 >> 16);
    int64_t sx4 = x4 & 0xffff;
    int32_t iy4 = (int32_t)(y4 >> 16);
    int64_t sy4 = y4 & 0xffff;
    int32_t im[15][8];
    for (int i1 = -7; i1 < 8; i1++) {
        for (int i2 = -4; i2 < 4; i2++) {
            int64_t sx = sx4 + alpha * i2 + beta * i1;
            int64_t o = rnd2(sx, 10) + 64;
            int offs = (int)clip3l(0, 192, o);
            const int32_t* row = r.p->s + (size_t)clip3(0, last_y, iy4 + i1) * r.p->cols;
            int64_t s = 0;
            for (int t = 0; t < 8; t++) s += (int64_t)WARPED[offs][t] * row[clip3(0, last_x, ix4 + i2 - 3 + t)];
            im[i1 + 7][i2 + 4] = (int32_t)rnd2(s, r0);
        }
    }
    int il = h - i8b * 8 - 4, jl = w - j8b * 8 - 4;
    if (il > 4) il = 4;
    if (jl > 4) jl = 4;
    for (int i1 = -4; i1 < il; i1++) {
        for (int i2 = -4; i2 < jl; i2++) {
            int64_t sy = sy4 + gamma * i2 + delta * i1;
            int offs = (int)clip3l(0, 192, rnd2(sy, 10) + 64);
            int64_t s = 0;
            for (int t = 0; t < 8; t++) s += (int64_t)WARPED[offs][t] * im[i1 + t + 4][i2 + 4];
            pred[(size_t)(i8b * 8 + i1 + 4) * w + j8b * 8 + i2 + 4] = (int32_t)rnd2(s, r1);
        }
    }
    return 0;
}

/* build_master_mask, inter_pred.rs:2712 */
static uint8_t MASTER[6][64][64];
static int master_ready = 0;
static void build_master(void) {
    if (master_ready) return;
    for (int j = 0; j < 64; j++) {
        int shift = 16;
        for (int i = 0; i < 64; i += 2) {
            MASTER[3][i][j] = M_EVEN[clip3(0, 63, j - shift)];
            shift -= 1;
            MASTER[3][i + 1][j] = M_ODD[clip3(0, 63, j - shift)];
            MASTER[1][i][j] = M_VERT[j];
            MASTER[1][i + 1][j] = M_VERT[j];
        }
    }
    for (int i = 0; i < 64; i++)
        for (int j = 0; j < 64; j++) {
            uint8_t m = MASTER[3][i][j];
            MASTER[2][j][i] = m;
            MASTER[4][i][63 - j] = 64 - m;
            MASTER[5][63 - j][i] = 64 - m;
            MASTER[0][j][i] = MASTER[1][i][j];
        }
    master_ready = 1;
}

/* wedge_mask, inter_pred.rs:2844 */
static int wedge_mask(int mi_size, int idx, int sign, uint8_t* mask) {
    if (mi_size >= 22 || WEDGE_BITS[mi_size] == 0 || idx >= 16 || sign > 1) return ERR;
    int n4w = N4W[mi_size], n4h = N4H[mi_size];
    int w = n4w * 4, h = n4h * 4;
    if (w > 64 || h > 64) return ERR;
    build_master();
    int shape = n4h > n4w ? 0 : (n4h < n4w ? 1 : 2);
    const uint8_t* e = CODEBOOK[shape][idx];
    int dir = e[0];
    int xoff = 32 - ((e[1] * w) >> 3);
    int yoff = 32 - ((e[2] * h) >> 3);
    int64_t sum = 0;
    for (int i = 0; i < w; i++) sum += MASTER[dir][yoff][xoff + i];
    for (int i = 1; i < h; i++) sum += MASTER[dir][yoff + i][xoff];
    int64_t avg = (sum + (w + h - 1) / 2) / (w + h - 1);
    int flip = avg < 32;
    int invert = sign != flip;
    for (int i = 0; i < h; i++)
        for (int j = 0; j < w; j++) {
            uint8_t raw = MASTER[dir][yoff + i][xoff + j];
            mask[i * w + j] = invert ? 64 - raw : raw;
        }
    return 0;
}

/* the mask read of mask_blend / mask_blend_interintra, inter_pred.rs:3136-3356 */
static int64_t mask_at(const uint8_t* m, int stride, int sx, int sy, int y, int x) {
    if (!sx && !sy) return m[y * stride + x];
    if (sx && !sy) return rnd2((int64_t)m[y * stride + 2 * x] + m[y * stride + 2 * x + 1], 1);
    if (!sx && sy) return rnd2((int64_t)m[2 * y * stride + x] + m[(2 * y + 1) * stride + x], 1);
    return rnd2((int64_t)m[2 * y * stride + 2 * x] + m[2 * y * stride + 2 * x + 1] + m[(2 * y + 1) * stride + 2 * x] +
                    m[(2 * y + 1) * stride + 2 * x + 1],
                2);
}

static const uint8_t* obmc_mask(int len) {
    switch (len) {
    case 2: return OM2;
    case 4: return OM4;
    case 8: return OM8;
    case 16: return OM16;
    default: return OM32;
    }
}

typedef struct {
    const av1g_frame_header* hdr;
    const av1g_ref_frame* refs;
    const ora_plane* ref_planes;  /* [7][3] */
    const av1g_obmc_neighbour* nb;
    int32_t n_nb;
    const av1g_warp_ctx* warps;
    int32_t n_warps;
    uint8_t* diffwtd;             /* luma-grid mask plane */
    int32_t dw_stride, dw_rows;
} ctx_t;

static ref_view view(const ctx_t* c, int ref, int plane) {
    ref_view r = {&c->ref_planes[ref * 3 + plane], c->refs[ref].upscaled_width, c->refs[ref].frame_height};
    return r;
}

/* predict_inter_per_ref, inter_pred.rs:1221 */
static int per_ref(const ctx_t* c, int ref, const int16_t mv[2], int plane, int x, int y, int w, int h, int fx, int fy,
                   int r0, int r1, int32_t* pred) {
    int ssx = plane ? c->hdr->subsampling_x : 0, ssy = plane ? c->hdr->subsampling_y : 0;
    int32_t s[4];
    if (mv_scaling(plane, ssx, ssy, c->hdr->frame_width, c->hdr->frame_height, c->refs[ref].upscaled_width,
                   c->refs[ref].frame_height, x, y, mv, s))
        return ERR;
    return block_inter(plane, ssx, ssy, view(c, ref, plane), s[0], s[1], s[2], s[3], w, h, fx, fy, r0, r1, pred);
}

/* predict_inter_one_ref with derive_use_warp, inter_pred.rs:1633-1910 */
static int one_ref(const ctx_t* c, const av1g_inter_pred* d, int list, int local_valid, int r0, int r1, int32_t* pred) {
    int plane = d->plane;
    int ssx = plane ? c->hdr->subsampling_x : 0, ssy = plane ? c->hdr->subsampling_y : 0;
    int ref = d->ref[list];
    int decision = 0; /* 0 translational, 1 local, 2 global */
    const av1g_warp_ctx* wp = d->warp >= 0 ? &c->warps[d->warp] : NULL;
    if (wp) {
        int ymode = wp->y_mode[list];
        int y_global = ymode == 16 || ymode == 24;
        int gm_warp = wp->gm_type[list] > 1;
        int scaled = wp->ref_is_scaled[list];
        int global_valid = 0;
        if (y_global && gm_warp && !scaled) {
            int v;
            int32_t sh[4];
            global_valid = setup_shear(wp->gm_params[list], &v, sh) == 0 && v;
        }
        if (d->w < 8 || d->h < 8) decision = 0;
        else if (wp->force_integer_mv) decision = 0;
        else if (d->motion_mode == 2 && local_valid) decision = 1;
        else if (y_global && gm_warp && !scaled && global_valid) decision = 2;
    }
    if (decision == 0)
        return per_ref(c, ref, d->mv[list], plane, d->x, d->y, d->w, d->h, d->filter_x, d->filter_y, r0, r1, pred);
    const int32_t* params = decision == 1 ? wp->local_warp_params : wp->gm_params[list];
    ref_view rv = view(c, ref, plane);
    for (int i = 0; i < (d->h + 7) / 8; i++)
        for (int j = 0; j < (d->w + 7) / 8; j++)
            if (block_warp(plane, ssx, ssy, d->x, d->y, i, j, d->w, d->h, rv, params, r0, r1, pred)) return ERR;
    return 0;
}

/* obmc_walk_axis + overlap_blending, inter_pred.rs:1911-2099, 4613-4880 */
static int obmc_axis(const ctx_t* c, const av1g_inter_pred* d, int left, const av1g_obmc_neighbour* list, int count,
                     int r0, int r1, uint16_t* out) {
    int plane = d->plane;
    int sx = plane ? c->hdr->subsampling_x : 0, sy = plane ? c->hdr->subsampling_y : 0;
    int bw = d->w, bh = d->h;
    uint32_t limit_log2 = left ? d->mi_height_log2 : d->mi_width_log2;
    uint32_t start = left ? d->mi_row : d->mi_col;
    uint32_t ext = 1u << limit_log2;
    uint32_t frame_limit = left ? (uint32_t)c->hdr->mi_rows : (uint32_t)c->hdr->mi_cols;
    if (start + ext < frame_limit) frame_limit = start + ext;
    uint32_t n_limit = limit_log2 < 4 ? limit_log2 : 4;
    uint32_t n = 0;
    int maxv = (1 << c->hdr->bit_depth) - 1;
    for (int k = 0; k < count; k++) {
        if (n >= n_limit) break;
        const av1g_obmc_neighbour* nb = &list[k];
        uint32_t pos = nb->axis_pos4;
        if (pos < start || pos >= frame_limit) return ERR;
        if (nb->step4 < 2 || nb->step4 > 16) return ERR;
        if (nb->ref > 6) return ERR;
        n++;
        int px, py, pw, ph, mlen;
        if (!left) {
            px = (int)((pos * 4) >> sx);
            py = (int)((d->mi_row * 4u) >> sy);
            pw = bw < (int)((nb->step4 * 4u) >> sx) ? bw : (int)((nb->step4 * 4u) >> sx);
            ph = (bh >> 1) < (32 >> sy) ? (bh >> 1) : (32 >> sy);
            mlen = ph;
        } else {
            px = (int)((d->mi_col * 4u) >> sx);
            py = (int)((pos * 4) >> sy);
            pw = (bw >> 1) < (32 >> sx) ? (bw >> 1) : (32 >> sx);
            ph = bh < (int)((nb->step4 * 4u) >> sy) ? bh : (int)((nb->step4 * 4u) >> sy);
            mlen = pw;
        }
        if (pw == 0 || ph == 0) continue;
        int ox = px - d->x, oy = py - d->y;
        if (ox < 0 || oy < 0 || ox >= bw || oy >= bh) return ERR;
        int fw = pw < bw - ox ? pw : bw - ox;
        int fh = ph < bh - oy ? ph : bh - oy;
        if (fw == 0 || fh == 0) continue;
        int32_t* p = (int32_t*)malloc(sizeof(int32_t) * (size_t)fw * fh);
        int e = per_ref(c, nb->ref, nb->mv, plane, px, py, fw, fh, nb->filter_x, nb->filter_y, r0, r1, p);
        if (e) {
            free(p);
            return ERR;
        }
        const uint8_t* m = obmc_mask(mlen);
        for (int i = 0; i < fh; i++)
            for (int j = 0; j < fw; j++) {
                uint32_t mm = left ? m[j] : m[i];
                uint32_t ob = (uint32_t)clip3(0, maxv, p[i * fw + j]);
                uint16_t* cur = &out[(oy + i) * bw + ox + j];
                *cur = (uint16_t)((mm * *cur + (64 - mm) * ob + 32) >> 6);
            }
        free(p);
    }
    return 0;
}

/* predict_inter, inter_pred.rs:2100, for one call; out holds the CurrFrame
 * region on entry (read by the inter-intra blend) and the prediction on
 * return. */
static int predict_inter(const ctx_t* c, const av1g_inter_pred* d, uint16_t* out, uint16_t* side_out) {
    const av1g_frame_header* hdr = c->hdr;
    int plane = d->plane, w = d->w, h = d->h, bd = hdr->bit_depth;
    if (plane > 2 || (bd != 8 && bd != 10 && bd != 12)) return ERR;
    if (hdr->frame_width <= 0 || hdr->frame_height <= 0) return ERR;
    if (w == 0 || h == 0 || w > 256 || h > 256) return ERR;
    if (d->kind > 2) return ERR;
    int compound = d->kind == AV1G_INTER_COMPOUND, ii = d->kind == AV1G_INTER_INTRA;
    if (d->ref[0] > 6 || (compound && d->ref[1] > 6)) return ERR;
    if (compound && d->compound_type != 0 && d->compound_type != 1 && d->compound_type != 2 && d->compound_type != 4)
        return ERR;
    if (ii && d->interintra_mode > 3) return ERR;
    if (d->warp >= c->n_warps) return ERR;
    if (d->motion_mode == 2 && d->warp < 0) return ERR;
    if (d->motion_mode == 1 && (uint64_t)d->obmc_first + d->obmc_above + d->obmc_left > (uint64_t)c->n_nb) return ERR;
    int ssx = plane ? hdr->subsampling_x : 0, ssy = plane ? hdr->subsampling_y : 0;
    int r0, r1, post;
    rounding(bd, compound, &r0, &r1, &post);
    int local_valid = d->warp >= 0 && c->warps[d->warp].local_valid;
    if (d->warp >= 0 && d->motion_mode == 2 && local_valid) {
        int v;
        int32_t sh[4];
        if (setup_shear(c->warps[d->warp].local_warp_params, &v, sh) || !v) local_valid = 0;
    }
    int maxv = (1 << bd) - 1;
    size_t n = (size_t)w * h;
    int32_t* p0 = (int32_t*)malloc(sizeof(int32_t) * n);
    int32_t* p1 = (int32_t*)malloc(sizeof(int32_t) * n);
    uint8_t* mask = NULL;
    int rc = one_ref(c, d, 0, local_valid, r0, r1, p0);
    if (rc) goto done;
    if (ii) {
        /* mask_blend_interintra, inter_pred.rs:3272 */
        int mstride, msx = 0, msy = 0;
        if (d->wedge_interintra) {
            if (d->mi_size >= 22) { rc = ERR; goto done; }
            int lw = N4W[d->mi_size] * 4, lh = N4H[d->mi_size] * 4;
            mask = (uint8_t*)malloc((size_t)lw * lh);
            if (wedge_mask(d->mi_size, d->wedge_index, 0, mask)) { rc = ERR; goto done; }
            msx = ssx;
            msy = ssy;
            mstride = lw;
            if ((msx ? 2 * w : w) > mstride || (size_t)mstride * ((msy ? 2 * h : h) - 1) + (msx ? 2 * w : w) >
                                                   (size_t)lw * lh) {
                rc = ERR;
                goto done;
            }
        } else {
            /* intra_mode_variant_mask, inter_pred.rs:3052 */
            if (w > 128 || h > 128) { rc = ERR; goto done; }
            mask = (uint8_t*)malloc(n);
            int scale = 128 / (w > h ? w : h);
            for (int i = 0; i < h; i++)
                for (int j = 0; j < w; j++) {
                    int m = 32;
                    if (d->interintra_mode == 1) m = II_W[i * scale];
                    else if (d->interintra_mode == 2) m = II_W[j * scale];
                    else if (d->interintra_mode == 3) m = II_W[(i < j ? i : j) * scale];
                    mask[i * w + j] = (uint8_t)m;
                }
            mstride = w;
        }
        if (side_out) {
            /* the blend's inter operand, kept for the intra half (no OBMC on such calls) */
            if (d->motion_mode == 1) { rc = ERR; goto done; }
            for (size_t i = 0; i < n; i++) side_out[i] = (uint16_t)clip3(0, maxv, (int32_t)rnd2(p0[i], post));
            goto done;
        }
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                int64_t m = mask_at(mask, mstride, msx, msy, y, x);
                int64_t cl = clip3(0, maxv, (int32_t)rnd2(p0[y * w + x], post));
                int32_t b = (int32_t)rnd2(m * out[y * w + x] + (64 - m) * cl, 6);
                out[y * w + x] = (uint16_t)clip3(0, maxv, b);
            }
    } else if (compound) {
        rc = one_ref(c, d, 1, local_valid, r0, r1, p1);
        if (rc) goto done;
        int ct = d->compound_type;
        if (ct == 2) {
            for (size_t i = 0; i < n; i++)
                out[i] = (uint16_t)clip3(0, maxv, (int32_t)rnd2((int64_t)p0[i] + p1[i], 1 + post));
        } else if (ct == 4) {
            /* compound_distance_blend, inter_pred.rs:3503 */
            for (size_t i = 0; i < n; i++)
                out[i] = (uint16_t)clip3(
                    0, maxv, (int32_t)rnd2((int64_t)d->fwd_weight * p0[i] + (int64_t)d->bck_weight * p1[i], 4 + post));
        } else {
            const uint8_t* m;
            int mstride;
            if (ct == 0) {
                if (d->mi_size >= 22) { rc = ERR; goto done; }
                int lw = N4W[d->mi_size] * 4, lh = N4H[d->mi_size] * 4;
                mask = (uint8_t*)malloc((size_t)lw * lh);
                if (wedge_mask(d->mi_size, d->wedge_index, d->wedge_sign, mask)) { rc = ERR; goto done; }
                m = mask;
                mstride = lw;
                if ((ssx ? 2 * w : w) > mstride ||
                    (size_t)mstride * ((ssy ? 2 * h : h) - 1) + (ssx ? 2 * w : w) > (size_t)lw * lh) {
                    rc = ERR;
                    goto done;
                }
            } else {
                /* predict_inter_compound_blend DIFFWTD arm, inter_pred.rs:1340-1370 */
                int lw = w << ssx, lh = h << ssy;
                if (d->y * (1 << ssy) + lh > c->dw_rows || d->x * (1 << ssx) + lw > c->dw_stride) {
                    rc = ERR;
                    goto done;
                }
                uint8_t* dm = c->diffwtd + (size_t)(d->y << ssy) * c->dw_stride + (d->x << ssx);
                if (plane == 0) {
                    /* difference_weight_mask, inter_pred.rs:2958 */
                    int shift = (bd - 8) + post;
                    for (int i = 0; i < h; i++)
                        for (int j = 0; j < w; j++) {
                            int64_t diff = llabs((int64_t)p0[i * w + j] - p1[i * w + j]);
                            int mm = clip3(0, 64, 38 + (int32_t)(rnd2(diff, shift) / 16));
                            dm[i * c->dw_stride + j] = (uint8_t)(d->mask_type ? 64 - mm : mm);
                        }
                }
                m = dm;
                mstride = c->dw_stride;
            }
            /* mask_blend, inter_pred.rs:3136 */
            for (int y = 0; y < h; y++)
                for (int x = 0; x < w; x++) {
                    int64_t mm = mask_at(m, mstride, ssx, ssy, y, x);
                    int64_t acc = mm * p0[y * w + x] + (64 - mm) * p1[y * w + x];
                    out[y * w + x] = (uint16_t)clip3(0, maxv, (int32_t)rnd2(acc, 6 + post));
                }
        }
    } else {
        for (size_t i = 0; i < n; i++) out[i] = (uint16_t)clip3(0, maxv, p0[i]);
    }
    if (d->motion_mode == 1) {
        const av1g_obmc_neighbour* nb = c->nb + d->obmc_first;
        if (d->avail_u && d->plane_residual_ge_8x8) {
            rc = obmc_axis(c, d, 0, nb, d->obmc_above, r0, r1, out);
            if (rc) goto done;
        }
        if (d->avail_l) rc = obmc_axis(c, d, 1, nb + d->obmc_above, d->obmc_left, r0, r1, out);
    }
done:
    free(p0);
    free(p1);
    free(mask);
    return rc;
}

int ora_inter_frame(const av1g_frame_header* hdr, const av1g_ref_frame* refs, const ora_plane* ref_planes,
                    const av1g_inter_pred* preds, int n, const av1g_obmc_neighbour* nb, int n_nb,
                    const av1g_warp_ctx* warps, int n_warps, ora_plane planes[3], ora_plane* side) {
    ctx_t c = {hdr, refs, ref_planes, nb, n_nb, warps, n_warps, NULL, 0, 0};
    c.dw_stride = planes[0].cols + 256;
    c.dw_rows = planes[0].rows + 256;
    c.diffwtd = (uint8_t*)calloc((size_t)c.dw_stride * c.dw_rows, 1);
    int rc = 0;
    for (int k = 0; k < n && !rc; k++) {
        const av1g_inter_pred* d = &preds[k];
        if (d->plane > 2 || d->w == 0 || d->h == 0 || d->w > 256 || d->h > 256) { rc = k + 1; break; }
        ora_plane* P = &planes[d->plane];
        if (d->x >= P->cols || d->y >= P->rows) { rc = k + 1; break; }
        int w = d->w, h = d->h;
        int fw = w < P->cols - d->x ? w : P->cols - d->x;
        int fh = h < P->rows - d->y ? h : P->rows - d->y;
        uint16_t* out = (uint16_t*)calloc((size_t)w * h, sizeof(uint16_t));
        for (int i = 0; i < fh; i++)
            for (int j = 0; j < fw; j++) out[i * w + j] = (uint16_t)P->s[(size_t)(d->y + i) * P->cols + d->x + j];
        ora_plane* S = (side && d->kind == AV1G_INTER_INTRA && side[d->plane].s) ? &side[d->plane] : NULL;
        uint16_t* so = S ? (uint16_t*)calloc((size_t)w * h, sizeof(uint16_t)) : NULL;
        if (predict_inter(&c, d, out, so)) rc = k + 1;
        else
            for (int i = 0; i < fh; i++)
                for (int j = 0; j < fw; j++) {
                    if (S) S->s[(size_t)(d->y + i) * S->cols + d->x + j] = so[i * w + j];
                    else P->s[(size_t)(d->y + i) * P->cols + d->x + j] = out[i * w + j];
                }
        free(out);
        free(so);
    }
    free(c.diffwtd);
    return rc;
}

/* exposed for the known-answer pins */
int ora_mv_scaling(int plane, int ssx, int ssy, int fw, int fh, int ruw, int rh, int x, int y, int mv_row,
                   int mv_col, int32_t out[4]) {
    int16_t mv[2] = {(int16_t)mv_row, (int16_t)mv_col};
    return mv_scaling(plane, ssx, ssy, fw, fh, ruw, rh, x, y, mv, out);
}
int ora_setup_shear(const int32_t p[6], int32_t out[5]) {
    int v;
    if (setup_shear(p, &v, out)) return ERR;
    out[4] = v;
    return 0;
}
int ora_wedge_mask(int mi_size, int idx, int sign, uint8_t* mask) { return wedge_mask(mi_size, idx, sign, mask); }

/* predict_intrabc_leaf_into_curr_frame (src/cdf.rs:19235-19370) for one
 * w x h region of plane p at (x, y): BILINEAR prediction from the window of
 * the pre-filter CurrFrame the filter can reach, clamped to the mi-padded
 * plane.  Returns 0 or ERR. */
int ora_intrabc_predict(const ora_plane* p, int plane, int ssx, int ssy, int mi_cols, int mi_rows, int x, int y,
                        int w, int h, int mv_row, int mv_col, int bd, uint16_t* pred) {
    if (abs(mv_row) >= (1 << 14) || abs(mv_col) >= (1 << 14)) return ERR;
    int sub_x = plane ? ssx : 0, sub_y = plane ? ssy : 0;
    int plane_rows = (mi_rows * 4) >> sub_y, plane_cols = (mi_cols * 4) >> sub_x;
    if (plane_rows == 0 || plane_cols == 0) return ERR;
    int32_t s[4];
    int16_t mv[2] = {(int16_t)mv_row, (int16_t)mv_col};
    if (mv_scaling(plane, ssx, ssy, mi_cols * 4, mi_rows * 4, mi_cols * 4, mi_rows * 4, x, y, mv, s)) return ERR;
    int last_x = plane_cols - 1, last_y = plane_rows - 1;
    int ih = (int)((((int64_t)h - 1) * s[3] + 1023) >> 10) + 8;
    int y_raw0 = (s[1] >> 10) - 3, x_raw0 = (s[0] >> 10) - 3;
    int x_raw1 = (int)(((int64_t)s[0] + (int64_t)s[2] * (w - 1)) >> 10) + 4;
    int y0 = clip3(0, last_y, y_raw0), y1 = clip3(0, last_y, y_raw0 + ih - 1);
    int x0 = clip3(0, last_x, x_raw0), x1 = clip3(0, last_x, x_raw1);
    int ww = x1 - x0 + 1, wh = y1 - y0 + 1;
    ora_plane win = {(int32_t*)malloc(sizeof(int32_t) * (size_t)ww * wh), wh, ww};
    for (int yy = y0; yy <= y1; yy++)
        for (int xx = x0; xx <= x1; xx++) win.s[(size_t)(yy - y0) * ww + xx - x0] = p->s[(size_t)yy * p->cols + xx];
    int r0, r1, post;
    rounding(bd, 0, &r0, &r1, &post);
    int32_t* pr = (int32_t*)malloc(sizeof(int32_t) * (size_t)w * h);
    ref_view rv = {&win, ww << sub_x, wh << sub_y};
    int rc = block_inter(plane, ssx, ssy, rv, s[0] - (x0 << 10), s[1] - (y0 << 10), s[2], s[3], w, h, 3, 3, r0, r1, pr);
    int maxv = (1 << bd) - 1;
    if (!rc)
        for (int i = 0; i < w * h; i++) pred[i] = (uint16_t)clip3(0, maxv, pr[i]);
    free(pr);
    free(win.s);
    return rc;
}

/* warp_estimation, inter_pred.rs:4083-4226, with the reference's release-
 * build integer semantics (wrapping +, -, *; saturating where it says so). */
static int64_t ls_product(int32_t a, int32_t b) { return (((int64_t)a * b) >> 2) + a + b; }
static int64_t wadd64(int64_t a, int64_t b) { return (int64_t)((uint64_t)a + (uint64_t)b); }
static int64_t wsub64(int64_t a, int64_t b) { return (int64_t)((uint64_t)a - (uint64_t)b); }
static int64_t wmul64(int64_t a, int64_t b) { return (int64_t)((uint64_t)a * (uint64_t)b); }
static int32_t wsub32(int32_t a, int32_t b) { return (int32_t)((uint32_t)a - (uint32_t)b); }
static int32_t wabs32(int32_t v) { return v == INT32_MIN ? v : (v < 0 ? -v : v); }

int ora_warp_estimation(const av1g_warp_sample* cand, int n, int mi_row, int mi_col, int bw4, int bh4, int mv_row,
                        int mv_col, int32_t params[6]) {
    if (n > 8) n = 8;
    int32_t mid_y = (int32_t)((uint32_t)mi_row * 4u + (uint32_t)bh4 * 2u - 1u);
    int32_t mid_x = (int32_t)((uint32_t)mi_col * 4u + (uint32_t)bw4 * 2u - 1u);
    int32_t suy = (int32_t)((uint32_t)mid_y * 8u), sux = (int32_t)((uint32_t)mid_x * 8u);
    int32_t duy = (int32_t)((uint32_t)suy + (uint32_t)(int32_t)(int16_t)mv_row);
    int32_t dux = (int32_t)((uint32_t)sux + (uint32_t)(int32_t)(int16_t)mv_col);
    int64_t A00 = 0, A01 = 0, A11 = 0, Bx0 = 0, Bx1 = 0, By0 = 0, By1 = 0;
    for (int i = 0; i < n; i++) {
        int32_t sy = wsub32(cand[i].sy, suy), sx = wsub32(cand[i].sx, sux);
        int32_t dy = wsub32(cand[i].dy, duy), dx = wsub32(cand[i].dx, dux);
        if (wabs32(wsub32(sx, dx)) < 256 && wabs32(wsub32(sy, dy)) < 256) {
            A00 = wadd64(A00, ls_product(sx, sx) + 8);
            A01 = wadd64(A01, ls_product(sx, sy) + 4);
            A11 = wadd64(A11, ls_product(sy, sy) + 8);
            Bx0 = wadd64(Bx0, ls_product(sx, dx) + 8);
            Bx1 = wadd64(Bx1, ls_product(sy, dx) + 4);
            By0 = wadd64(By0, ls_product(sx, dy) + 4);
            By1 = wadd64(By1, ls_product(sy, dy) + 8);
        }
    }
    int64_t det = wsub64(sat_mul(A00, A11), sat_mul(A01, A01));
    memset(params, 0, 6 * sizeof(int32_t));
    if (det == 0) return 0;
    uint64_t ad = det < 0 ? 0ull - (uint64_t)det : (uint64_t)det;
    int nb = 63 - __builtin_clzll(ad);
    int64_t e = (int64_t)(ad - (1ull << nb));
    int64_t f = nb > 8 ? (e + ((int64_t)1 << (nb - 8 - 1))) >> (nb - 8) : e << (8 - nb);
    if (f > 256) f = 256;
    int64_t fac = DIV_LUT[f];
    if (det < 0) fac = -fac;
    int shift = nb + 14 - 16;
    if (shift < 0) {
        fac = wmul64(fac, (int64_t)1 << -shift);
        shift = 0;
    }
    int32_t one = 1 << 16, ndc = 1 << 13;
#define DIAG(v) clip3(one - ndc + 1, one + ndc - 1, (int32_t)rnd2s(sat_mul((v), fac), shift))
#define NONDIAG(v) clip3(-ndc + 1, ndc - 1, (int32_t)rnd2s(sat_mul((v), fac), shift))
    params[2] = DIAG(wsub64(wmul64(A11, Bx0), wmul64(A01, Bx1)));
    params[3] = NONDIAG(wadd64(wmul64(wsub64(0, A01), Bx0), wmul64(A00, Bx1)));
    params[4] = NONDIAG(wsub64(wmul64(A11, By0), wmul64(A01, By1)));
    params[5] = DIAG(wadd64(wmul64(wsub64(0, A01), By0), wmul64(A00, By1)));
#undef DIAG
#undef NONDIAG
    int64_t vx = (int64_t)(int16_t)mv_col * (1 << 13) - ((int64_t)mid_x * (params[2] - one) + (int64_t)mid_y * params[3]);
    int64_t vy = (int64_t)(int16_t)mv_row * (1 << 13) - ((int64_t)mid_x * params[4] + (int64_t)mid_y * (params[5] - one));
    int64_t tc = 1 << 23;
    params[0] = (int32_t)(vx < -tc ? -tc : (vx > tc - 1 ? tc - 1 : vx));
    params[1] = (int32_t)(vy < -tc ? -tc : (vy > tc - 1 ? tc - 1 : vy));
    return 1;
}

/* The intra half of an inter-intra block of one plane: intra (the block's
 * intra prediction, w x h) blended with the stored inter half in side,
 * written to out within the plane (mask_blend_interintra,
 * inter_pred.rs:3272, with the masks of predict_inter's inter-intra arm,
 * inter_pred.rs:2230-2290).  Returns 0 or ERR. */
int ora_interintra_blend(const av1g_frame_header* hdr, const av1g_intra_tu* t, int w, int h, const uint16_t* intra,
                         const ora_plane* side, ora_plane* out) {
    int ssx = t->plane ? hdr->subsampling_x : 0, ssy = t->plane ? hdr->subsampling_y : 0;
    int maxv = (1 << hdr->bit_depth) - 1;
    uint8_t* mask = NULL;
    int mstride, msx = 0, msy = 0;
    if (t->interintra == 2) {
        if (t->mi_size >= 22) return ERR;
        int lw = N4W[t->mi_size] * 4, lh = N4H[t->mi_size] * 4;
        mask = (uint8_t*)malloc((size_t)lw * lh);
        if (wedge_mask(t->mi_size, t->wedge_index, 0, mask) || (ssx ? 2 * w : w) > lw ||
            (size_t)lw * ((ssy ? 2 * h : h) - 1) + (ssx ? 2 * w : w) > (size_t)lw * lh) {
            free(mask);
            return ERR;
        }
        msx = ssx;
        msy = ssy;
        mstride = lw;
    } else {
        mask = (uint8_t*)malloc((size_t)w * h);
        int scale = 128 / (w > h ? w : h);
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) {
                int m = 32;
                if (t->interintra_mode == 1) m = II_W[i * scale];
                else if (t->interintra_mode == 2) m = II_W[j * scale];
                else if (t->interintra_mode == 3) m = II_W[(i < j ? i : j) * scale];
                mask[i * w + j] = (uint8_t)m;
            }
        mstride = w;
    }
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int yy = t->y + y, xx = t->x + x;
            if (yy >= out->rows || xx >= out->cols) continue;
            int64_t m = mask_at(mask, mstride, msx, msy, y, x);
            int64_t cl = side->s[(size_t)yy * side->cols + xx];
            int32_t b = (int32_t)rnd2(m * intra[y * w + x] + (64 - m) * cl, 6);
            out->s[(size_t)yy * out->cols + xx] = clip3(0, maxv, b);
        }
    free(mask);
    return 0;
}
