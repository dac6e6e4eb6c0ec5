/*
 * mfmv.c — CPU oracle for motion-field motion vectors.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Restates, sequentially and in the
 * reference's order:
 *   get_relative_dist                 src/inter_pred.rs:3383-3390
 *   §7.19 motion vector storage       src/decoder/frame_driver.rs:1119-1160
 *   §7.9  motion_field_estimation_core
 *         (project_ref, get_mv_projection, get_block_position, the source
 *          selection and ref_stamp budget)  src/inter_pred.rs:7592-7742
 *   §7.9.3 get_mv_projection          src/cdf.rs:35101-35114
 * The av1g_mf_* job structs are reused with HOST pointers.  Products are
 * formed in 64 bits like the cdf.rs version; for the stored candidates
 * (|mv| <= 4095) they equal the 32-bit products of inter_pred.rs.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

enum { LAST = 1, LAST2 = 2, GOLDEN = 4, BWDREF = 5, ALTREF2 = 6, ALTREF = 7 };
#define MAX_FRAME_DISTANCE 31
#define MAX_OFFSET_WIDTH 8
#define MAX_OFFSET_HEIGHT 0

/* §7.9.3 Div_Mult, a table of the specification. */
static const int DIV_MULT[32] = {0,    16384, 8192, 5461, 4096, 3276, 2730, 2340, 2048, 1820, 1638,
                                 1489, 1365,  1260, 1170, 1092, 1024, 963,  910,  862,  819,  780,
                                 744,  712,   682,  655,  630,  606,  585,  564,  546,  528};

int ora_relative_dist(int a, int b, int bits) {
    if (bits == 0) return 0;
    int diff = a - b, m = 1 << (bits - 1);
    return (diff & (m - 1)) - (diff & m);
}

void ora_mv_projection(const int mv[2], int numerator, int denominator, int out[2]) {
    int den = denominator < MAX_FRAME_DISTANCE ? denominator : MAX_FRAME_DISTANCE;
    int num = numerator;
    if (num < -MAX_FRAME_DISTANCE) num = -MAX_FRAME_DISTANCE;
    if (num > MAX_FRAME_DISTANCE) num = MAX_FRAME_DISTANCE;
    for (int i = 0; i < 2; i++) {
        long long v = (long long)mv[i] * num * DIV_MULT[den];
        long long scaled = v >= 0 ? (v + (1 << 13)) >> 14 : -((-v + (1 << 13)) >> 14);
        long long lim = (1 << 14) - 1;
        out[i] = (int)(scaled < -lim ? -lim : (scaled > lim ? lim : scaled));
    }
}

void ora_mf_store(const av1g_mf_store_job* j) {
    const int limit = (1 << 12) - 1; /* REFMVS_LIMIT */
    long long cells = (long long)j->mi_rows * j->mi_cols;
    for (long long c = 0; c < cells; c++) {
        j->mf_ref_frames[c] = -1;
        j->mf_mvs[2 * c] = 0;
        j->mf_mvs[2 * c + 1] = 0;
        if (!j->is_inter_frame) continue;
        for (int list = 0; list < 2; list++) {
            int r = j->ref_frames[2 * c + list];
            if (r <= 0 || r > 7) continue;
            if (ora_relative_dist(j->ref_order_hint[r - 1], j->order_hint, j->hint_bits) >= 0) continue;
            int mr = j->mvs[(2 * c + list) * 2], mc = j->mvs[(2 * c + list) * 2 + 1];
            if (abs(mr) <= limit && abs(mc) <= limit) {
                j->mf_ref_frames[c] = (int8_t)r;
                j->mf_mvs[2 * c] = (int16_t)mr;
                j->mf_mvs[2 * c + 1] = (int16_t)mc;
            }
        }
    }
}

/* §7.9.4 project() of get_block_position. */
static int block_position(int v8, int delta, int sign, int max8, int max_off8, int* out) {
    int base8 = (v8 >> 3) << 3;
    int off8 = delta >= 0 ? delta >> 6 : -((-delta) >> 6);
    v8 += sign * off8;
    *out = v8;
    return !(v8 < 0 || v8 >= max8 || v8 < base8 - max_off8 || v8 >= base8 + 8 + max_off8);
}

/* get_block_position (cdf.rs:35141): 1 and the position when it is valid. */
int ora_block_position(int x8, int y8, int sign, int pr, int pc, int mi_rows, int mi_cols, int* py, int* px) {
    int vy = block_position(y8, pr, sign, mi_rows >> 1, MAX_OFFSET_HEIGHT, py);
    int vx = block_position(x8, pc, sign, mi_cols >> 1, MAX_OFFSET_WIDTH, px);
    return vy && vx;
}

/* project_ref: returns 0 when the source slot is skipped. */
static int project_ref(const av1g_mf_project_job* j, int src, int sign) {
    const av1g_mf_slot* s = &j->slots[j->ref_frame_idx[src - LAST]];
    if (!s->mf_ref_frames || s->mi_rows != j->mi_rows || s->mi_cols != j->mi_cols || s->frame_is_intra) return 0;
    int w8 = j->mi_cols >> 1, h8 = j->mi_rows >> 1;
    for (int y8 = 0; y8 < h8; y8++)
        for (int x8 = 0; x8 < w8; x8++) {
            long long cell = (long long)(2 * y8 + 1) * j->mi_cols + (2 * x8 + 1);
            int sref = s->mf_ref_frames[cell];
            if (sref <= 0 || sref > 7) continue;
            int ref_to_cur = ora_relative_dist(j->order_hints[src], j->order_hint, j->hint_bits);
            int ref_offset = ora_relative_dist(j->order_hints[src], s->saved_order_hints[sref], j->hint_bits);
            if (!(abs(ref_to_cur) <= MAX_FRAME_DISTANCE && abs(ref_offset) <= MAX_FRAME_DISTANCE && ref_offset > 0))
                continue;
            int mv[2] = {s->mf_mvs[2 * cell], s->mf_mvs[2 * cell + 1]}, proj[2];
            ora_mv_projection(mv, ref_to_cur * sign, ref_offset, proj);
            int py, px;
            int vy = block_position(y8, proj[0], sign, h8, MAX_OFFSET_HEIGHT, &py);
            int vx = block_position(x8, proj[1], sign, w8, MAX_OFFSET_WIDTH, &px);
            if (!(vy && vx)) continue;
            for (int dst = LAST; dst <= ALTREF; dst++) {
                int ref_to_dst = ora_relative_dist(j->order_hint, j->order_hints[dst], j->hint_bits);
                int o[2];
                ora_mv_projection(mv, ref_to_dst, ref_offset, o);
                size_t at = (((size_t)(dst - 1) * h8 + py) * w8 + px) * 2;
                j->out[at] = (int16_t)o[0];
                j->out[at + 1] = (int16_t)o[1];
            }
        }
    return 1;
}

void ora_mf_project(const av1g_mf_project_job* j) {
    int w8 = j->mi_cols >> 1, h8 = j->mi_rows >> 1;
    size_t total = (size_t)7 * h8 * w8 * 2;
    for (size_t k = 0; k < total; k++) j->out[k] = AV1G_MFMV_INVALID;
    if (w8 <= 0 || h8 <= 0) return;
    const av1g_mf_slot* last = &j->slots[j->ref_frame_idx[0]];
    int last_alt = last->mf_ref_frames ? last->saved_order_hints[ALTREF] : 0;
    if (last_alt != j->order_hints[GOLDEN]) project_ref(j, LAST, -1);
    int stamp = 1; /* MFMV_STACK_SIZE - 2 */
    if (ora_relative_dist(j->order_hints[BWDREF], j->order_hint, j->hint_bits) > 0 && project_ref(j, BWDREF, 1))
        stamp--;
    if (ora_relative_dist(j->order_hints[ALTREF2], j->order_hint, j->hint_bits) > 0 && project_ref(j, ALTREF2, 1))
        stamp--;
    if (ora_relative_dist(j->order_hints[ALTREF], j->order_hint, j->hint_bits) > 0 && stamp >= 0 &&
        project_ref(j, ALTREF, 1))
        stamp--;
    if (stamp >= 0) project_ref(j, LAST2, -1);
}
