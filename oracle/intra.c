/*
 * intra.c — CPU oracle for intra prediction, chroma-from-luma and intra
 * reconstruction.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates:
 *   intra_predict_block_samples           src/cdf.rs:16990-17250
 *   predict_intra_dc_pred                 src/cdf.rs:1348
 *   predict_intra_v_pred / _h_pred        src/cdf.rs:1680-1730
 *   predict_intra_paeth_pred              src/cdf.rs:2077
 *   predict_intra_recursive               src/cdf.rs:2145
 *   predict_intra_smooth(_v/_h)_pred      src/cdf.rs:2267-2387
 *   intra_edge_*_selection, filter_corner, intra_edge_upsample,
 *   intra_edge_filter                     src/cdf.rs:2588-2878
 *   predict_intra_directional             src/cdf.rs:2879-3010
 *   predict_chroma_from_luma_into_curr_frame   src/cdf.rs:17256-17340
 * and the per-TU order of transform_block_emit (src/cdf.rs:32540-32910):
 * predict, CfL, then dequant + inverse transform + merge.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "av1_spec_tables.h"

static const AV1T_TX_WIDTH_TYPE TW_ AV1T_TX_WIDTH_DIMS = AV1T_TX_WIDTH_INIT;
static const AV1T_TX_HEIGHT_TYPE TH_ AV1T_TX_HEIGHT_DIMS = AV1T_TX_HEIGHT_INIT;
static const AV1T_MODE_TO_ANGLE_TYPE MODE_TO_ANGLE AV1T_MODE_TO_ANGLE_DIMS = AV1T_MODE_TO_ANGLE_INIT;
static const AV1T_DR_INTRA_DERIVATIVE_TYPE DR_DERIV AV1T_DR_INTRA_DERIVATIVE_DIMS = AV1T_DR_INTRA_DERIVATIVE_INIT;
static const AV1T_INTRA_EDGE_KERNEL_TYPE EDGE_KERNEL AV1T_INTRA_EDGE_KERNEL_DIMS = AV1T_INTRA_EDGE_KERNEL_INIT;
static const AV1T_INTRA_FILTER_TAPS_TYPE FI_TAPS AV1T_INTRA_FILTER_TAPS_DIMS = AV1T_INTRA_FILTER_TAPS_INIT;
static const AV1T_SM_WEIGHTS_TX_4X4_TYPE SM4 AV1T_SM_WEIGHTS_TX_4X4_DIMS = AV1T_SM_WEIGHTS_TX_4X4_INIT;
static const AV1T_SM_WEIGHTS_TX_8X8_TYPE SM8 AV1T_SM_WEIGHTS_TX_8X8_DIMS = AV1T_SM_WEIGHTS_TX_8X8_INIT;
static const AV1T_SM_WEIGHTS_TX_16X16_TYPE SM16 AV1T_SM_WEIGHTS_TX_16X16_DIMS = AV1T_SM_WEIGHTS_TX_16X16_INIT;
static const AV1T_SM_WEIGHTS_TX_32X32_TYPE SM32 AV1T_SM_WEIGHTS_TX_32X32_DIMS = AV1T_SM_WEIGHTS_TX_32X32_INIT;
static const AV1T_SM_WEIGHTS_TX_64X64_TYPE SM64 AV1T_SM_WEIGHTS_TX_64X64_DIMS = AV1T_SM_WEIGHTS_TX_64X64_INIT;

enum { DC_PRED = 0, V_PRED = 1, H_PRED = 2, D67_PRED = 8, SMOOTH_PRED = 9, SMOOTH_V_PRED = 10, SMOOTH_H_PRED = 11,
       PAETH_PRED = 12, INTRA_MODES = 13 };

static const uint8_t* sm_weights(int log2n) {
    switch (log2n) {
        case 2: return SM4;
        case 3: return SM8;
        case 4: return SM16;
        case 5: return SM32;
        default: return SM64;
    }
}
static int ilog2(int v) { int n = 0; while ((1 << n) < v) n++; return n; }
static int64_t r2s(int64_t x, int n) {  /* round2_signed, cdf.rs:35247 */
    if (n == 0) return x;
    int64_t half = (int64_t)1 << (n - 1);
    return x >= 0 ? (x + half) >> n : -(((-x) + half) >> n);
}

/* intra_edge_upsample_selection (cdf.rs:2588) */
static int upsample_sel(int w, int h, int ft, int delta) {
    int d = delta < 0 ? -delta : delta;
    if (d == 0 || d >= 40) return 0;
    int wh = w + h;
    return ft == 0 ? (wh <= 16) : (wh <= 8);
}
/* intra_edge_filter_strength_selection (cdf.rs:2610) */
static int strength_sel(int w, int h, int ft, int delta) {
    int d = delta < 0 ? -delta : delta, wh = w + h, s = 0;
    if (ft == 0) {
        if (wh <= 8) { if (d >= 56) s = 1; }
        else if (wh <= 16) { if (d >= 40) s = 1; }
        else if (wh <= 24) { if (d >= 8) s = 1; if (d >= 16) s = 2; if (d >= 32) s = 3; }
        else if (wh <= 32) { s = 1; if (d >= 4) s = 2; if (d >= 32) s = 3; }
        else s = 3;
    } else {
        if (wh <= 8) { if (d >= 40) s = 1; if (d >= 64) s = 2; }
        else if (wh <= 16) { if (d >= 20) s = 1; if (d >= 48) s = 2; }
        else if (wh <= 24) { if (d >= 4) s = 3; }
        else s = 3;
    }
    return s;
}
/* intra_edge_upsample (cdf.rs:2700) on buf (index 0 == position -2) */
static void edge_upsample(int num_px, int bd, uint16_t* buf) {
    int dup[132];
    dup[0] = buf[1];
    for (int i = 0; i < num_px; i++) dup[i + 2] = buf[i + 2];
    dup[1] = buf[1];
    dup[num_px + 2] = buf[num_px + 1];
    buf[0] = (uint16_t)dup[0];
    int maxv = (1 << bd) - 1;
    for (int i = 0; i < num_px; i++) {
        int s = -dup[i] + 9 * dup[i + 1] + 9 * dup[i + 2] - dup[i + 3];
        int r = s >= 0 ? (s + 8) >> 4 : -(((-s) + 8) >> 4);
        buf[2 * i + 1] = (uint16_t)(r < 0 ? 0 : (r > maxv ? maxv : r));
        int c = dup[i + 2];
        buf[2 * i + 2] = (uint16_t)(c > maxv ? maxv : c);
    }
}
/* intra_edge_filter (cdf.rs:2760) on buf (index 0 == position -2) */
static void edge_filter(int sz, int strength, uint16_t* buf) {
    if (strength == 0 || sz == 0) return;
    int edge[132];
    for (int i = 0; i < sz; i++) edge[i] = buf[i + 1];
    for (int i = 1; i < sz; i++) {
        int s = 0;
        for (int j = 0; j < 5; j++) {
            int k = i - 2 + j;
            k = k < 0 ? 0 : (k > sz - 1 ? sz - 1 : k);
            s += EDGE_KERNEL[strength - 1][j] * edge[k];
        }
        int o = (s + 8) >> 4;
        buf[i + 1] = (uint16_t)(o < 0 ? 0 : o);
    }
}

/* predict_intra_directional (cdf.rs:2879-3010); above/left are the extended
 * arrays with index 0 == position -2. */
static void directional(int w, int h, int pa, int ua, int ul, const uint16_t* above, const uint16_t* left,
                        uint16_t* pred) {
    int dx = pa < 90 ? DR_DERIV[pa] : (pa < 180 ? DR_DERIV[180 - pa] : 0);
    int dy = (pa >= 90 && pa < 180) ? DR_DERIV[pa - 90] : (pa > 180 ? DR_DERIV[270 - pa] : 0);
#define A(k) above[(k) + 2]
#define L(k) left[(k) + 2]
    if (pa < 90) {
        int maxb = (w + h - 1) << ua;
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) {
                int idx = (i + 1) * dx;
                int base = (idx >> (6 - ua)) + j * (1 << ua);
                int sh = ((idx * (1 << ua)) >> 1) & 0x1F;
                pred[i * w + j] = base < maxb ? (uint16_t)((A(base) * (32 - sh) + A(base + 1) * sh + 16) >> 5) : A(maxb);
            }
    } else if (pa < 180) {
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) {
                int ix = (j << 6) - (i + 1) * dx;
                int bx = ix >> (6 - ua);
                if (bx >= -(1 << ua)) {
                    int sh = ((ix * (1 << ua)) >> 1) & 0x1F;
                    pred[i * w + j] = (uint16_t)((A(bx) * (32 - sh) + A(bx + 1) * sh + 16) >> 5);
                } else {
                    int iy = (i << 6) - (j + 1) * dy;
                    int by = iy >> (6 - ul);
                    int sh = ((iy * (1 << ul)) >> 1) & 0x1F;
                    pred[i * w + j] = (uint16_t)((L(by) * (32 - sh) + L(by + 1) * sh + 16) >> 5);
                }
            }
    } else {
        int maxb = (w + h - 1) << ul;
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) {
                int idx = (j + 1) * dy;
                int base = (idx >> (6 - ul)) + i * (1 << ul);
                int sh = ((idx * (1 << ul)) >> 1) & 0x1F;
                pred[i * w + j] = base < maxb ? (uint16_t)((L(base) * (32 - sh) + L(base + 1) * sh + 16) >> 5) : L(maxb);
            }
    }
#undef A
#undef L
}

/* predict_intra_recursive (cdf.rs:2145-2200) */
static void recursive(int w, int h, int fim, int bd, const uint16_t* above, const uint16_t* left, uint16_t* pred) {
    int w4 = w >> 2, h2 = h >> 1, maxv = (1 << bd) - 1;
    for (int i2 = 0; i2 < h2; i2++)
        for (int j4 = 0; j4 < w4; j4++) {
            int p[7];
            for (int i = 0; i < 7; i++) {
                if (i < 5) {
                    if (i2 == 0) p[i] = above[(j4 << 2) + i - 1 + 2];
                    else if (j4 == 0 && i == 0) p[i] = left[(i2 << 1) - 1 + 2];
                    else p[i] = pred[((i2 << 1) - 1) * w + (j4 << 2) + i - 1];
                } else if (j4 == 0) {
                    p[i] = left[(i2 << 1) + i - 5 + 2];
                } else {
                    p[i] = pred[((i2 << 1) + i - 5) * w + (j4 << 2) - 1];
                }
            }
            for (int i1 = 0; i1 < 2; i1++)
                for (int j1 = 0; j1 < 4; j1++) {
                    int64_t acc = 0;
                    for (int i = 0; i < 7; i++) acc += (int64_t)FI_TAPS[fim][(i1 << 2) + j1][i] * p[i];
                    int64_t v = r2s(acc, 4);
                    pred[((i2 << 1) + i1) * w + (j4 << 2) + j1] = (uint16_t)(v < 0 ? 0 : (v > maxv ? maxv : v));
                }
        }
}

/* intra_predict_block_samples (cdf.rs:16990-17250) reading plane p (int32). */
void ora_intra_predict(const ora_plane* p, int sx, int sy, int tx, int mode, int angle_delta, int bd, int flags,
                       int filter_intra_mode, uint16_t* pred) {
    int w = TW_[tx], h = TH_[tx];
    int lw = ilog2(w), lh = ilog2(h);
    int max_x = p->cols - 1, max_y = p->rows - 1;
    int have_above = (flags & AV1G_INTRA_HAVE_ABOVE) && sy > 0;
    int have_left = (flags & AV1G_INTRA_HAVE_LEFT) && sx > 0;
    int have_ar = (flags & AV1G_INTRA_HAVE_ABOVE_RIGHT) != 0, have_bl = (flags & AV1G_INTRA_HAVE_BELOW_LEFT) != 0;
    int eief = (flags & AV1G_INTRA_EDGE_FILTER) != 0, ft = (flags & AV1G_INTRA_FILTER_TYPE) ? 1 : 0;
#define RD(yy, xx) ((uint16_t)p->s[(size_t)((yy) < max_y ? (yy) : max_y) * p->cols + ((xx) < max_x ? (xx) : max_x)])
    uint16_t half = (uint16_t)(1 << (bd - 1));
    uint16_t corner = have_above && have_left ? RD(sy - 1, sx - 1) : have_above ? RD(sy - 1, sx) : have_left ? RD(sy, sx - 1) : half;
    int span = w + h, cap = 2 * span + 2;
    uint16_t above[260], left[260];
    memset(above, 0, sizeof above);
    memset(left, 0, sizeof left);
    above[0] = above[1] = corner;
    if (!have_above && have_left) {
        uint16_t v = RD(sy, sx - 1);
        for (int i = 0; i < span; i++) above[2 + i] = v;
    } else if (!have_above && !have_left) {
        for (int i = 0; i < span; i++) above[2 + i] = (uint16_t)((1 << (bd - 1)) - 1);
    } else {
        int lim = sx + (have_ar ? 2 * w : w) - 1;
        lim = lim < max_x ? lim : max_x;
        for (int i = 0; i < span; i++) above[2 + i] = RD(sy - 1, (sx + i) < lim ? sx + i : lim);
    }
    left[0] = left[1] = corner;
    if (!have_left && have_above) {
        uint16_t v = RD(sy - 1, sx);
        for (int i = 0; i < span; i++) left[2 + i] = v;
    } else if (!have_left && !have_above) {
        for (int i = 0; i < span; i++) left[2 + i] = (uint16_t)((1 << (bd - 1)) + 1);
    } else {
        int lim = sy + (have_bl ? 2 * h : h) - 1;
        lim = lim < max_y ? lim : max_y;
        for (int i = 0; i < span; i++) left[2 + i] = RD((sy + i) < lim ? sy + i : lim, sx - 1);
    }
#undef RD
    (void)cap;
    int ua = 0, ul = 0;
    if (mode >= V_PRED && mode <= D67_PRED) {
        int pa = MODE_TO_ANGLE[mode] + angle_delta * 3;
        if (eief && pa != 90 && pa != 180) {
            if (pa > 90 && pa < 180 && (w + h) >= 24) {
                uint16_t fc = (uint16_t)((left[2] * 5 + above[1] * 6 + above[2] * 5 + 8) >> 4);
                above[1] = fc;
                left[1] = fc;
            }
            if (have_above) {
                int st = strength_sel(w, h, ft, pa - 90);
                int n = (w < max_x - sx + 1 ? w : max_x - sx + 1) + (pa < 90 ? h : 0) + 1;
                edge_filter(n, st, above);
            }
            if (have_left) {
                int st = strength_sel(w, h, ft, pa - 180);
                int n = (h < max_y - sy + 1 ? h : max_y - sy + 1) + (pa > 180 ? w : 0) + 1;
                edge_filter(n, st, left);
            }
            ua = upsample_sel(w, h, ft, pa - 90);
            if (ua) edge_upsample(w + (pa < 90 ? h : 0), bd, above);
            ul = upsample_sel(w, h, ft, pa - 180);
            if (ul) edge_upsample(h + (pa > 180 ? w : 0), bd, left);
        }
    }
    const uint16_t* ar = above + 2;
    const uint16_t* lc = left + 2;
    if (filter_intra_mode < 5) {
        recursive(w, h, filter_intra_mode, bd, above, left, pred);
        return;
    }
    if (mode == DC_PRED) {
        uint32_t avg;
        if (have_left && have_above) {
            uint32_t s = 0;
            for (int i = 0; i < h; i++) s += lc[i];
            for (int j = 0; j < w; j++) s += ar[j];
            s += (uint32_t)(w + h) >> 1;
            avg = s / (uint32_t)(w + h);
        } else if (have_left) {
            uint32_t s = 0;
            for (int i = 0; i < h; i++) s += lc[i];
            avg = (s + ((uint32_t)h >> 1)) >> lh;
            if (avg > (uint32_t)(1 << bd) - 1) avg = (1 << bd) - 1;
        } else if (have_above) {
            uint32_t s = 0;
            for (int j = 0; j < w; j++) s += ar[j];
            avg = (s + ((uint32_t)w >> 1)) >> lw;
            if (avg > (uint32_t)(1 << bd) - 1) avg = (1 << bd) - 1;
        } else {
            avg = 1u << (bd - 1);
        }
        for (int k = 0; k < w * h; k++) pred[k] = (uint16_t)avg;
    } else if (mode == V_PRED && angle_delta == 0) {
        for (int i = 0; i < h; i++) memcpy(pred + i * w, ar, sizeof(uint16_t) * w);
    } else if (mode == H_PRED && angle_delta == 0) {
        for (int i = 0; i < h; i++) for (int j = 0; j < w; j++) pred[i * w + j] = lc[i];
    } else if (mode >= V_PRED && mode <= D67_PRED) {
        directional(w, h, MODE_TO_ANGLE[mode] + angle_delta * 3, ua, ul, above, left, pred);
    } else if (mode == SMOOTH_PRED) {
        const uint8_t *swx = sm_weights(lw), *swy = sm_weights(lh);
        uint32_t bl = lc[h - 1], tr = ar[w - 1];
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) {
                uint32_t s = swy[i] * ar[j] + (256 - swy[i]) * bl + swx[j] * lc[i] + (256 - swx[j]) * tr;
                pred[i * w + j] = (uint16_t)((s + 256) >> 9);
            }
    } else if (mode == SMOOTH_V_PRED) {
        const uint8_t* sw = sm_weights(lh);
        uint32_t bl = lc[h - 1];
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) pred[i * w + j] = (uint16_t)((sw[i] * ar[j] + (256 - sw[i]) * bl + 128) >> 8);
    } else if (mode == SMOOTH_H_PRED) {
        const uint8_t* sw = sm_weights(lw);
        uint32_t tr = ar[w - 1];
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) pred[i * w + j] = (uint16_t)((sw[j] * lc[i] + (256 - sw[j]) * tr + 128) >> 8);
    } else if (mode == PAETH_PRED) {
        for (int i = 0; i < h; i++)
            for (int j = 0; j < w; j++) {
                int base = ar[j] + lc[i] - corner;
                int pl = abs(base - lc[i]), pt = abs(base - ar[j]), ptl = abs(base - corner);
                pred[i * w + j] = (pl <= pt && pl <= ptl) ? lc[i] : (pt <= ptl ? ar[j] : corner);
            }
    }
}

/* The luma a transform writes past the mi-grid plane (LumaOverhang,
 * cdf.rs:15938-15990: up to 64 samples right of and below the plane), kept
 * for chroma from luma. */
typedef struct {
    int32_t* s;
    int rows, cols; /* plane rows + 64, plane cols + 64 */
} overhang;

static int32_t luma_at(const ora_plane* luma, const overhang* oh, int yy, int xx) {
    if (yy < luma->rows && xx < luma->cols) return luma->s[(size_t)yy * luma->cols + xx];
    if (oh && yy < oh->rows && xx < oh->cols) return oh->s[(size_t)yy * oh->cols + xx];
    return 0;
}

/* predict_chroma_from_luma_into_curr_frame (cdf.rs:17256-17340): luma past
 * the plane comes from the overhang store (read at cdf.rs:17292-17305). */
static void cfl(ora_plane* luma, const overhang* oh, ora_plane* p, int sx, int sy, int tx, int ssx, int ssy,
                int alpha, int bd, int max_luma_w, int max_luma_h) {
    int w = TW_[tx], h = TH_[tx];
    int cx = max_luma_w - (1 << ssx), cy = max_luma_h - (1 << ssy);
    if (cx < 0) cx = 0;
    if (cy < 0) cy = 0;
    int64_t* l = (int64_t*)malloc(sizeof(int64_t) * w * h);
    int64_t avg = 0;
    for (int i = 0; i < h; i++) {
        int ly = (sy + i) << ssy;
        ly = ly < cy ? ly : cy;
        for (int j = 0; j < w; j++) {
            int lx = (sx + j) << ssx;
            lx = lx < cx ? lx : cx;
            int64_t t = 0;
            for (int dy = 0; dy <= ssy; dy++)
                for (int dx = 0; dx <= ssx; dx++) {
                    int yy = ly + dy, xx = lx + dx;
                    t += luma_at(luma, oh, yy, xx);
                }
            int64_t v = t << (3 - ssx - ssy);
            l[i * w + j] = v;
            avg += v;
        }
    }
    avg = r2s(avg, ilog2(w) + ilog2(h));
    int64_t maxv = (1 << bd) - 1;
    for (int i = 0; i < h; i++) {
        int dy = sy + i;
        if (dy >= p->rows) break;
        for (int j = 0; j < w; j++) {
            int dx = sx + j;
            if (dx >= p->cols) break;
            int32_t* s = &p->s[(size_t)dy * p->cols + dx];
            int64_t v = *s + r2s((int64_t)alpha * (l[i * w + j] - avg), 6);
            *s = (int32_t)(v < 0 ? 0 : (v > maxv ? maxv : v));
        }
    }
    free(l);
}

void ora_recon_frame(const av1g_frame_header* hdr, const av1g_quant_params* q, const av1g_tu* tus, int n,
                     const int32_t* coeffs, ora_plane planes[3]);

/* Every intra TU of a frame in decode order: predict (writing the TU area
 * inside the plane), CfL, residual. */
int ora_intra_frame(const av1g_frame_header* hdr, const av1g_quant_params* q, const av1g_intra_tu* tus, int n,
                    const int32_t* coeffs, ora_plane planes[3], const uint8_t* maps, int64_t map_bytes,
                    const ora_plane* side) {
    uint16_t* pred = (uint16_t*)malloc(sizeof(uint16_t) * 64 * 64);
    int32_t* full = (int32_t*)malloc(sizeof(int32_t) * 64 * 64);
    overhang oh = {NULL, planes[0].rows + 64, planes[0].cols + 64};
    oh.s = (int32_t*)calloc((size_t)oh.rows * oh.cols, sizeof(int32_t));
    int rc = 0;
    for (int k = 0; k < n; k++) {
        const av1g_intra_tu* t = &tus[k];
        ora_plane* p = &planes[t->plane];
        int w = TW_[t->tx_size], h = TH_[t->tx_size];
        int have_pred = t->mode < INTRA_MODES;
        int luma_overhang = t->plane == 0 && !t->interintra && (t->x + w > p->cols || t->y + h > p->rows);
        if (t->interintra) {
            static const int ii_to_intra[4] = {0, 1, 2, 9};
            if (t->interintra > 2 || t->interintra_mode > 3 || t->mode != ii_to_intra[t->interintra_mode] ||
                t->filter_intra_mode < 5 || (t->flags & AV1G_INTRA_CFL) || !side || !side[t->plane].s) {
                rc = k + 1;
                break;
            }
            ora_intra_predict(p, t->x, t->y, t->tx_size, t->mode, 0, hdr->bit_depth, t->flags, 255, pred);
            if (ora_interintra_blend(hdr, t, w, h, pred, &side[t->plane], p)) {
                rc = k + 1;
                break;
            }
            have_pred = 0;  /* already written */
        } else if (t->mode == AV1G_INTRA_MODE_PALETTE) {
            /* predict_palette (cdf.rs:11907) */
            int64_t last = (int64_t)t->palette_map + (int64_t)(h - 1) * t->palette_stride + (w - 1);
            if (t->palette_size == 0 || t->palette_size > 8 || t->palette_stride < w || last >= map_bytes) {
                rc = k + 1;
                break;
            }
            for (int i = 0; i < h && !rc; i++)
                for (int j = 0; j < w; j++) {
                    int idx = maps[t->palette_map + (int64_t)i * t->palette_stride + j];
                    if (idx >= t->palette_size) {
                        rc = k + 1;
                        break;
                    }
                    pred[i * w + j] = t->palette_colors[idx];
                }
            if (rc) break;
            have_pred = 1;
        } else if (t->mode == AV1G_INTRA_MODE_INTRABC) {
            if (ora_intrabc_predict(p, t->plane, hdr->subsampling_x, hdr->subsampling_y, hdr->mi_cols, hdr->mi_rows,
                                    t->x, t->y, w, h, t->mv[0], t->mv[1], hdr->bit_depth, pred)) {
                rc = k + 1;
                break;
            }
            have_pred = 1;
        } else if (t->mode < INTRA_MODES) {
            int fim = (t->plane == 0 && t->filter_intra_mode < 5) ? t->filter_intra_mode : 255;
            ora_intra_predict(p, t->x, t->y, t->tx_size, t->mode, t->angle_delta, hdr->bit_depth, t->flags, fim,
                              pred);
        }
        if (have_pred) {
            for (int i = 0; i < h; i++)
                for (int j = 0; j < w; j++) {
                    int yy = t->y + i, xx = t->x + j;
                    if (yy < p->rows && xx < p->cols) p->s[(size_t)yy * p->cols + xx] = pred[i * w + j];
                }
        }
        if ((t->flags & AV1G_INTRA_CFL) && t->plane > 0)
            cfl(&planes[0], &oh, p, t->x, t->y, t->tx_size, hdr->subsampling_x, hdr->subsampling_y, t->cfl_alpha,
                hdr->bit_depth, t->max_luma_w, t->max_luma_h);
        if (luma_overhang && have_pred) {
            /* the whole transform (prediction + residual) for the samples past
             * the plane (the merge's side-store writes, cdf.rs:17441-17477) */
            for (int i = 0; i < w * h; i++) full[i] = pred[i];
            if (t->flags & AV1G_INTRA_RESIDUAL) {
                av1g_tu r = t->res;
                r.x = 0;
                r.y = 0;
                r.plane = 0;
                ora_plane tp[3] = {{full, h, w}, {full, h, w}, {full, h, w}};
                ora_recon_frame(hdr, q, &r, 1, coeffs, tp);
            }
            for (int i = 0; i < h; i++)
                for (int j = 0; j < w; j++) {
                    int yy = t->y + i, xx = t->x + j;
                    if ((yy >= p->rows || xx >= p->cols) && yy < oh.rows && xx < oh.cols)
                        oh.s[(size_t)yy * oh.cols + xx] = full[i * w + j];
                }
        }
        if (t->flags & AV1G_INTRA_RESIDUAL) ora_recon_frame(hdr, q, &t->res, 1, coeffs, planes);
    }
    free(pred);
    free(full);
    free(oh.s);
    return rc;
}
