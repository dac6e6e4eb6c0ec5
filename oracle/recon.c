/*
 * recon.c — CPU oracle for dequantization, inverse transform and the
 * reconstruction merge.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates, in the reference's own
 * formulation and with its 64-bit intermediates:
 *   §7.12.3 step 1   dc_q / ac_q / get_qindex / get_dc_quant / get_ac_quant /
 *                    dequant_denom / dequantize_step1   src/cdf.rs:13384-13703
 *                    qmatrix_value                      src/qmatrix.rs:4888
 *   §7.13            inverse_transform_2d and the 1-D kernels
 *                                                       src/transform.rs:96-847
 *   §7.12.3 step 3   curr_frame_step3_merge             src/cdf.rs:17398-17470
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"
#include "av1_spec_tables.h"

static const AV1T_DC_QLOOKUP_TYPE DC_Q AV1T_DC_QLOOKUP_DIMS = AV1T_DC_QLOOKUP_INIT;
static const AV1T_AC_QLOOKUP_TYPE AC_Q AV1T_AC_QLOOKUP_DIMS = AV1T_AC_QLOOKUP_INIT;
static const AV1T_QM_OFFSET_TYPE QM_OFF AV1T_QM_OFFSET_DIMS = AV1T_QM_OFFSET_INIT;
static const AV1T_QUANTIZER_MATRIX_TYPE QM AV1T_QUANTIZER_MATRIX_DIMS = AV1T_QUANTIZER_MATRIX_INIT;
static const AV1T_COS128_LOOKUP_TYPE COS128 AV1T_COS128_LOOKUP_DIMS = AV1T_COS128_LOOKUP_INIT;
static const AV1T_TRANSFORM_ROW_SHIFT_TYPE ROW_SHIFT AV1T_TRANSFORM_ROW_SHIFT_DIMS = AV1T_TRANSFORM_ROW_SHIFT_INIT;
static const AV1T_TX_WIDTH_TYPE TXW_ AV1T_TX_WIDTH_DIMS = AV1T_TX_WIDTH_INIT;
static const AV1T_TX_HEIGHT_TYPE TXH_ AV1T_TX_HEIGHT_DIMS = AV1T_TX_HEIGHT_INIT;

enum { DCT_DCT, ADST_DCT, DCT_ADST, ADST_ADST, FLIPADST_DCT, DCT_FLIPADST, FLIPADST_FLIPADST, ADST_FLIPADST,
       FLIPADST_ADST, IDTX, V_DCT, H_DCT, V_ADST, H_ADST, V_FLIPADST, H_FLIPADST };

static int64_t r2(int64_t x, int n) { return n == 0 ? x : (x + ((int64_t)1 << (n - 1))) >> n; }
static int64_t clip64(int64_t lo, int64_t hi, int64_t x) { return x < lo ? lo : (x > hi ? hi : x); }
static int clampi(int lo, int hi, int x) { return x < lo ? lo : (x > hi ? hi : x); }

/* ---- §7.12.3 step 1 ------------------------------------------------------ */

/* dc_q / ac_q (cdf.rs:13384-13403) */
static int dc_q(int bd, int b) { int row = (bd < 8 ? 0 : (bd - 8) >> 1); row = row > 2 ? 2 : row; return DC_Q[row][clampi(0, 255, b)]; }
static int ac_q(int bd, int b) { int row = (bd < 8 ? 0 : (bd - 8) >> 1); row = row > 2 ? 2 : row; return AC_Q[row][clampi(0, 255, b)]; }

/* get_qindex (cdf.rs:13527-13550); ignore_delta_q = false */
static int get_qindex(const av1g_quant_params* q, int segment_id, int current_q_index) {
    int seg = segment_id < 7 ? segment_id : 7;
    if (seg < 0) seg = 0;
    if (q->segmentation_enabled && q->seg_alt_q_active[seg]) {
        int data = q->seg_alt_q_data[seg];
        int qi = q->delta_q_present ? current_q_index + data : q->base_q_idx + data;
        return clampi(0, 255, qi);
    }
    if (q->delta_q_present) return current_q_index;
    return q->base_q_idx;
}

/* dequant_denom (cdf.rs:13582) */
static int64_t dq_denom(int tx) {
    if (tx == 3 || tx == 9 || tx == 10 || tx == 17 || tx == 18) return 2;
    if (tx == 4 || tx == 11 || tx == 12) return 4;
    return 1;
}

/* dequantize_step1 (cdf.rs:13655-13703): compact tw-stride levels -> dense w*h */
void ora_dequantize(const av1g_quant_params* q, int bit_depth, const int32_t* levels, int tx, int plane,
                    int segment_id, int current_q_index, int plane_tx_type, int64_t* out) {
    int w = TXW_[tx], h = TXH_[tx];
    int tw = w < 32 ? w : 32, th = h < 32 ? h : 32;
    int64_t denom = dq_denom(tx);
    int64_t cmin = -((int64_t)1 << (7 + bit_depth)), cmax = ((int64_t)1 << (7 + bit_depth)) - 1;
    int base = get_qindex(q, segment_id, current_q_index);
    int ddc = plane == 0 ? q->delta_q_y_dc : (plane == 1 ? q->delta_q_u_dc : q->delta_q_v_dc);
    int dac = plane == 0 ? 0 : (plane == 1 ? q->delta_q_u_ac : q->delta_q_v_ac);
    int64_t dcq = dc_q(bit_depth, base + ddc), acq = ac_q(bit_depth, base + dac);
    int seg = segment_id < 0 ? 0 : (segment_id > 7 ? 7 : segment_id);
    int qm_level = q->seg_qm_level[plane][seg];
    int qm_active = q->using_qmatrix && plane_tx_type < IDTX && qm_level < 15;
    memset(out, 0, sizeof(int64_t) * (size_t)w * h);
    for (int i = 0; i < th; i++)
        for (int j = 0; j < tw; j++) {
            int64_t qq = (i == 0 && j == 0) ? dcq : acq;
            if (qm_active) {
                int64_t m = QM[qm_level][plane > 0][QM_OFF[tx] + i * tw + j];
                qq = (qq * m + 16) >> 5;
            }
            int64_t dq = (int64_t)levels[i * tw + j] * qq;
            int64_t sign = dq < 0 ? -1 : 1;
            int64_t mag = (int64_t)((uint64_t)(dq < 0 ? -dq : dq) & 0xFFFFFF);
            int64_t dq2 = (sign * mag) / denom;
            out[i * w + j] = clip64(cmin, cmax, dq2);
        }
}

/* ---- §7.13 1-D kernels (transform.rs) ------------------------------------ */

static int cos128(int angle) {                          /* transform.rs:170-185 */
    int a = angle & 255;
    if (a <= 64) return COS128[a];
    if (a <= 128) return -COS128[128 - a];
    if (a <= 192) return -COS128[a - 128];
    return COS128[256 - a];
}
static int sin128(int angle) { return cos128(angle - 64); }
static unsigned brev(int nbits, unsigned x) {
    unsigned t = 0;
    for (int i = 0; i < nbits; i++) t |= ((x >> i) & 1) << (nbits - 1 - i);
    return t;
}

static void B(int64_t* t, int a, int b, int angle, int flip) {   /* butterfly_b, transform.rs:196-209 */
    int64_t c = cos128(angle), s = sin128(angle);
    int64_t x = t[a] * c - t[b] * s, y = t[a] * s + t[b] * c;
    t[a] = r2(x, 12);
    t[b] = r2(y, 12);
    if (flip) { int64_t tmp = t[a]; t[a] = t[b]; t[b] = tmp; }
}
static void H(int64_t* t, int a, int b, int flip, int r) {       /* butterfly_h, transform.rs:211-219 */
    int ai = flip ? b : a, bi = flip ? a : b;
    int64_t x = t[ai], y = t[bi];
    int64_t lo = -((int64_t)1 << (r - 1)), hi = ((int64_t)1 << (r - 1)) - 1;
    t[ai] = clip64(lo, hi, x + y);
    t[bi] = clip64(lo, hi, x - y);
}

/* inverse_dct (transform.rs:238-460) */
static void idct(int64_t* t, int n, int r) {
    int len = 1 << n;
    int64_t cp[64];
    memcpy(cp, t, sizeof(int64_t) * len);
    for (int i = 0; i < len; i++) t[i] = cp[brev(n, i)];
    if (n == 6) for (int i = 0; i < 16; i++) B(t, 32 + i, 63 - i, 63 - 4 * (int)brev(4, i), 0);
    if (n >= 5) for (int i = 0; i < 8; i++) B(t, 16 + i, 31 - i, 6 + ((int)brev(3, 7 - i) << 3), 0);
    if (n == 6) for (int i = 0; i < 16; i++) H(t, 32 + i * 2, 33 + i * 2, i & 1, r);
    if (n >= 4) for (int i = 0; i < 4; i++) B(t, 8 + i, 15 - i, 12 + ((int)brev(2, 3 - i) << 4), 0);
    if (n >= 5) for (int i = 0; i < 8; i++) H(t, 16 + 2 * i, 17 + 2 * i, i & 1, r);
    if (n == 6) for (int i = 0; i < 4; i++) for (int j = 0; j < 2; j++)
        B(t, 62 - i * 4 - j, 33 + i * 4 + j, 60 - 16 * (int)brev(2, i) + 64 * j, 1);
    if (n >= 3) for (int i = 0; i < 2; i++) B(t, 4 + i, 7 - i, 56 - 32 * i, 0);
    if (n >= 4) for (int i = 0; i < 4; i++) H(t, 8 + 2 * i, 9 + 2 * i, i & 1, r);
    if (n >= 5) for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
        B(t, 30 - 4 * i - j, 17 + 4 * i + j, 24 + (j << 6) + ((1 - i) << 5), 1);
    if (n == 6) for (int i = 0; i < 8; i++) for (int j = 0; j < 2; j++) H(t, 32 + i * 4 + j, 35 + i * 4 - j, i & 1, r);
    for (int i = 0; i < 2; i++) B(t, 2 * i, 2 * i + 1, 32 + 16 * i, 1 - i);
    if (n >= 3) for (int i = 0; i < 2; i++) H(t, 4 + 2 * i, 5 + 2 * i, i, r);
    if (n >= 4) for (int i = 0; i < 2; i++) B(t, 14 - i, 9 + i, 48 + 64 * i, 1);
    if (n >= 5) for (int i = 0; i < 4; i++) for (int j = 0; j < 2; j++) H(t, 16 + 4 * i + j, 19 + 4 * i - j, i & 1, r);
    if (n == 6) for (int i = 0; i < 2; i++) for (int j = 0; j < 4; j++)
        B(t, 61 - i * 8 - j, 34 + i * 8 + j, 56 - i * 32 + (j >> 1) * 64, 1);
    for (int i = 0; i < 2; i++) H(t, i, 3 - i, 0, r);
    if (n >= 3) B(t, 6, 5, 32, 1);
    if (n >= 4) for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) H(t, 8 + 4 * i + j, 11 + 4 * i - j, i, r);
    if (n >= 5) for (int i = 0; i < 4; i++) B(t, 29 - i, 18 + i, 48 + (i >> 1) * 64, 1);
    if (n == 6) for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) H(t, 32 + 8 * i + j, 39 + 8 * i - j, i & 1, r);
    if (n >= 3) for (int i = 0; i < 4; i++) H(t, i, 7 - i, 0, r);
    if (n >= 4) for (int i = 0; i < 2; i++) B(t, 13 - i, 10 + i, 32, 1);
    if (n >= 5) for (int i = 0; i < 2; i++) for (int j = 0; j < 4; j++) H(t, 16 + i * 8 + j, 23 + i * 8 - j, i, r);
    if (n == 6) for (int i = 0; i < 8; i++) B(t, 59 - i, 36 + i, i < 4 ? 48 : 112, 1);
    if (n >= 4) for (int i = 0; i < 8; i++) H(t, i, 15 - i, 0, r);
    if (n >= 5) for (int i = 0; i < 4; i++) B(t, 27 - i, 20 + i, 32, 1);
    if (n == 6) for (int i = 0; i < 8; i++) { H(t, 32 + i, 47 - i, 0, r); H(t, 48 + i, 63 - i, 1, r); }
    if (n >= 5) for (int i = 0; i < 16; i++) H(t, i, 31 - i, 0, r);
    if (n == 6) for (int i = 0; i < 8; i++) B(t, 55 - i, 40 + i, 32, 1);
    if (n == 6) for (int i = 0; i < 32; i++) H(t, i, 63 - i, 0, r);
}

static void adst_in_perm(int64_t* t, int n) {            /* transform.rs:465-474 */
    int n0 = 1 << n;
    int64_t cp[16];
    memcpy(cp, t, sizeof(int64_t) * n0);
    for (int i = 0; i < n0; i++) t[i] = cp[(i & 1) ? i - 1 : n0 - i - 1];
}
static void adst_out_perm(int64_t* t, int n) {           /* transform.rs:476-492 */
    int n0 = 1 << n;
    int64_t cp[16];
    memcpy(cp, t, sizeof(int64_t) * n0);
    for (int i = 0; i < n0; i++) {
        unsigned a = (i >> 3) & 1, b = ((i >> 2) & 1) ^ ((i >> 3) & 1), c = ((i >> 1) & 1) ^ ((i >> 2) & 1),
                 d = (i & 1) ^ ((i >> 1) & 1);
        unsigned idx = ((d << 3) | (c << 2) | (b << 1) | a) >> (4 - n);
        t[i] = (i & 1) ? -cp[idx] : cp[idx];
    }
}
static void iadst4(int64_t* t) {                          /* transform.rs:494-525 */
    const int64_t S1 = 1321, S2 = 2482, S3 = 3344, S4 = 3803;
    int64_t t0 = t[0], t1 = t[1], t2 = t[2], t3 = t[3], s[7];
    s[0] = S1 * t0; s[1] = S2 * t0; s[2] = S3 * t1; s[3] = S4 * t2; s[4] = S1 * t2; s[5] = S2 * t3; s[6] = S4 * t3;
    int64_t b7 = t0 - t2 + t3;
    s[0] += s[3]; s[1] -= s[4]; s[3] = s[2]; s[2] = S3 * b7; s[0] += s[5]; s[1] -= s[6];
    t[0] = r2(s[0] + s[3], 12); t[1] = r2(s[1] + s[3], 12); t[2] = r2(s[2], 12); t[3] = r2(s[0] + s[1] - s[3], 12);
}
static void iadst8(int64_t* t, int r) {                   /* transform.rs:527-556 */
    adst_in_perm(t, 3);
    for (int i = 0; i < 4; i++) B(t, 2 * i, 2 * i + 1, 60 - 16 * i, 1);
    for (int i = 0; i < 4; i++) H(t, i, 4 + i, 0, r);
    for (int i = 0; i < 2; i++) B(t, 4 + 3 * i, 5 + i, 48 - 32 * i, 1);
    for (int j = 0; j < 2; j++) for (int i = 0; i < 2; i++) H(t, 4 * j + i, 2 + 4 * j + i, 0, r);
    for (int i = 0; i < 2; i++) B(t, 2 + 4 * i, 3 + 4 * i, 32, 1);
    adst_out_perm(t, 3);
}
static void iadst16(int64_t* t, int r) {                  /* transform.rs:558-616 */
    adst_in_perm(t, 4);
    for (int i = 0; i < 8; i++) B(t, 2 * i, 2 * i + 1, 62 - 8 * i, 1);
    for (int i = 0; i < 8; i++) H(t, i, 8 + i, 0, r);
    for (int i = 0; i < 2; i++) { B(t, 8 + 2 * i, 9 + 2 * i, 56 - 32 * i, 1); B(t, 13 + 2 * i, 12 + 2 * i, 8 + 32 * i, 1); }
    for (int j = 0; j < 2; j++) for (int i = 0; i < 4; i++) H(t, 8 * j + i, 4 + 8 * j + i, 0, r);
    for (int j = 0; j < 2; j++) for (int i = 0; i < 2; i++) B(t, 4 + 8 * j + 3 * i, 5 + 8 * j + i, 48 - 32 * i, 1);
    for (int j = 0; j < 4; j++) for (int i = 0; i < 2; i++) H(t, 4 * j + i, 2 + 4 * j + i, 0, r);
    for (int i = 0; i < 4; i++) B(t, 2 + 4 * i, 3 + 4 * i, 32, 1);
    adst_out_perm(t, 4);
}
static void iwht4(int64_t* t, int shift) {                /* transform.rs:622-643 */
    int64_t a = t[0] >> shift, c = t[1] >> shift, d = t[2] >> shift, b = t[3] >> shift;
    a += c; d -= b;
    int64_t e = (a - d) >> 1;
    b = e - b;
    int64_t c2 = e - c;
    a -= b; d += c2;
    t[0] = a; t[1] = b; t[2] = c2; t[3] = d;
}
static void iidentity(int64_t* t, int n) {                /* transform.rs:645-682 */
    int len = 1 << n;
    for (int i = 0; i < len; i++) {
        if (n == 2) t[i] = r2(t[i] * 5793, 12);
        else if (n == 3) t[i] *= 2;
        else if (n == 4) t[i] = r2(t[i] * 11586, 12);
        else t[i] *= 4;
    }
}
static int row_is_dct(int tt) { return tt == DCT_DCT || tt == ADST_DCT || tt == FLIPADST_DCT || tt == H_DCT; }
static int row_is_adst(int tt) {
    return tt == DCT_ADST || tt == ADST_ADST || tt == DCT_FLIPADST || tt == FLIPADST_FLIPADST || tt == ADST_FLIPADST ||
           tt == FLIPADST_ADST || tt == H_ADST || tt == H_FLIPADST;
}
static int col_is_dct(int tt) { return tt == DCT_DCT || tt == DCT_ADST || tt == DCT_FLIPADST || tt == V_DCT; }
static int col_is_adst(int tt) {
    return tt == ADST_DCT || tt == ADST_ADST || tt == FLIPADST_DCT || tt == FLIPADST_FLIPADST || tt == ADST_FLIPADST ||
           tt == FLIPADST_ADST || tt == V_ADST || tt == V_FLIPADST;
}
static void iadst(int64_t* t, int n, int r) { if (n == 2) iadst4(t); else if (n == 3) iadst8(t, r); else iadst16(t, r); }

/* inverse_transform_2d (transform.rs:707-789) */
void ora_inverse_transform_2d(const int64_t* dq, int tx, int tt, int bit_depth, int lossless, int64_t* res) {
    int w = TXW_[tx], h = TXH_[tx];
    int lw = 0, lh = 0;
    while ((1 << lw) < w) lw++;
    while ((1 << lh) < h) lh++;
    int row_shift = lossless ? 0 : ROW_SHIFT[tx], col_shift = lossless ? 0 : 4;
    int rr = bit_depth + 8, cr = bit_depth + 6 > 16 ? bit_depth + 6 : 16;
    int64_t tb[64];
    for (int i = 0; i < h; i++) {
        for (int j = 0; j < w; j++) tb[j] = (i < 32 && j < 32) ? dq[i * w + j] : 0;
        if (abs(lw - lh) == 1) for (int j = 0; j < w; j++) tb[j] = r2(tb[j] * 2896, 12);
        if (lossless) iwht4(tb, 2);
        else if (row_is_dct(tt)) idct(tb, lw, rr);
        else if (row_is_adst(tt)) iadst(tb, lw, rr);
        else iidentity(tb, lw);
        for (int j = 0; j < w; j++) res[i * w + j] = r2(tb[j], row_shift);
    }
    int64_t lo = -((int64_t)1 << (cr - 1)), hi = ((int64_t)1 << (cr - 1)) - 1;
    for (int k = 0; k < w * h; k++) res[k] = clip64(lo, hi, res[k]);
    for (int j = 0; j < w; j++) {
        for (int i = 0; i < h; i++) tb[i] = res[i * w + j];
        if (lossless) iwht4(tb, 0);
        else if (col_is_dct(tt)) idct(tb, lh, cr);
        else if (col_is_adst(tt)) iadst(tb, lh, cr);
        else iidentity(tb, lh);
        for (int i = 0; i < h; i++) res[i * w + j] = r2(tb[i], col_shift);
    }
}

/* curr_frame_step3_merge (cdf.rs:17398-17470) inside the plane; ora_intra_frame
 * keeps the luma past the plane (the overhang store) itself */
static void merge(ora_plane* p, int x0, int y0, int tx, int tt, const int64_t* res, int bit_depth) {
    int w = TXW_[tx], h = TXH_[tx];
    int fud = tt == FLIPADST_DCT || tt == FLIPADST_ADST || tt == V_FLIPADST || tt == FLIPADST_FLIPADST;
    int flr = tt == DCT_FLIPADST || tt == ADST_FLIPADST || tt == H_FLIPADST || tt == FLIPADST_FLIPADST;
    int64_t maxv = (1 << bit_depth) - 1;
    for (int i = 0; i < h; i++)
        for (int j = 0; j < w; j++) {
            int yy = fud ? h - i - 1 : i, xx = flr ? w - j - 1 : j;
            int dy = y0 + yy, dx = x0 + xx;
            if (dy >= p->rows || dx >= p->cols) continue;
            int32_t* s = &p->s[(size_t)dy * p->cols + dx];
            int64_t v = (int64_t)*s + res[i * w + j];
            *s = (int32_t)clip64(0, maxv, v);
        }
}

/* transform_block_emit's reconstruct tail (cdf.rs:32874-32910) for every TU of
 * a frame: dequant, inverse transform, merge into the planes (in place). */
void ora_recon_frame(const av1g_frame_header* hdr, const av1g_quant_params* q, const av1g_tu* tus, int n,
                     const int32_t* coeffs, ora_plane planes[3]) {
    int64_t* dq = (int64_t*)malloc(sizeof(int64_t) * 4096);
    int64_t* res = (int64_t*)malloc(sizeof(int64_t) * 4096);
    for (int k = 0; k < n; k++) {
        const av1g_tu* t = &tus[k];
        int seg = t->segment_id > 7 ? 7 : t->segment_id;
        ora_dequantize(q, hdr->bit_depth, coeffs + t->coeff_offset, t->tx_size, t->plane, t->segment_id,
                       t->current_q_index, t->tx_type, dq);
        ora_inverse_transform_2d(dq, t->tx_size, t->tx_type, hdr->bit_depth, q->lossless[seg], res);
        merge(&planes[t->plane], t->x, t->y, t->tx_size, t->tx_type, res, hdr->bit_depth);
    }
    free(dq);
    free(res);
}
