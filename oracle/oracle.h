/*
 * oracle.h — CPU restatement of the reference decoder's pixel path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity oracle for the CUDA
 * engine: tests, the smoke check and the bench's CPU-baseline arm call it to
 * produce the expected output on the same inputs.  The engine never links,
 * loads or calls it.
 *
 * Every function restates the reference crate's CPU code (Rust, not buildable
 * here: no rustc/cargo and the `oxideav-core` dependency is not vendored) in
 * the reference's own per-sample formulation, with the file:line it follows
 * cited at each definition.  Planes are int32 row-major, like the reference's
 * `PlaneBuffer` (src/loop_filter.rs:119-126).
 */
#ifndef AV1_ORACLE_H
#define AV1_ORACLE_H

#include <stdint.h>
#include "av1g.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_plane {
    int32_t* s;
    int32_t rows;
    int32_t cols;
} ora_plane;

/* §7.14 — loop_filter_frame (src/loop_filter.rs:271) driven by
 * loop_filter_frame_from_grid (src/cdf.rs:20449).  In place. */
void ora_loop_filter_frame(const av1g_frame_header* hdr, const av1g_mi_grid* grid,
                           ora_plane planes[3]);

/* §7.15 — cdef_frame (src/cdef.rs:180) driven by cdef_frame_from_idx
 * (src/cdf.rs:20300).  cdef_idx per 64x64: ceil(mi_rows/16) x ceil(mi_cols/16). */
void ora_cdef_frame(const av1g_frame_header* hdr, const av1g_mi_grid* grid,
                    const int8_t* cdef_idx, const ora_plane src[3], ora_plane dst[3]);

/* §7.16 — upscale_frame (src/superres.rs:282).  Returns 0 on success. */
int ora_upscale_frame(const av1g_frame_header* hdr, const ora_plane in[3], ora_plane out[3]);

/* §7.17 — loop_restoration_frame (src/loop_restoration.rs:268) driven by
 * loop_restore_frame_from_grid (src/cdf.rs:20624). */
void ora_lr_frame(const av1g_frame_header* hdr, const av1g_lr_unit* const units[3],
                  const int32_t unit_rows[3], const int32_t unit_cols[3],
                  const ora_plane curr[3], const ora_plane cdef[3], ora_plane lr[3]);

/* §7.18.3 — film_grain_synthesis (src/film_grain.rs:848), in place on the
 * cropped output planes. */
void ora_film_grain(const av1g_film_grain* fg, int bit_depth, int num_planes, int sub_x,
                    int sub_y, int matrix_coefficients, ora_plane out[3]);

/* §7.18.3.3 generate_grain (src/film_grain.rs:230) — exposed for the
 * template-level known-answer tests.  luma: 73x82, cb/cr: chroma_h x chroma_w. */
void ora_generate_grain(const av1g_film_grain* fg, int bit_depth, int sub_x, int sub_y,
                        int32_t* luma, int32_t* cb, int32_t* cr);

/* §7.18.3.4 scaling_lookup_init (src/film_grain.rs:418): 3 x 256 table. */
void ora_scaling_lookup_init(const av1g_film_grain* fg, int num_planes, uint8_t lut[3][256]);

/* §7.18.3.2 RandomRegister::next (src/film_grain.rs:119). */
uint32_t ora_random_next(uint16_t* state, int bits);

/* The §7.4 chain of decode_frame_spec_tiles (src/decoder/frame_driver.rs:
 * 790-1116): deblock, CDEF, superres, LR, crop, pre-grain store, grain.
 * recon: padded-extent planes (not modified).  ref_out / out: cropped
 * UpscaledWidth x FrameHeight planes (chroma subsampled), row stride = width;
 * ref_out is the §7.20 pre-grain payload, out the post-grain output.
 * Returns 0 on success, nonzero on a malformed header. */
int ora_postfilter_frame(const av1g_frame_header* hdr, const av1g_mi_grid* grid,
                         const int8_t* cdef_idx, const av1g_lr_unit* const units[3],
                         const int32_t* const recon[3], int32_t* ref_out[3],
                         int32_t* out[3]);

/* §7.12.3 step 1 — dequantize_step1 (src/cdf.rs:13655): compact levels ->
 * dense w*h int64. */
void ora_dequantize(const av1g_quant_params* q, int bit_depth, const int32_t* levels, int tx, int plane,
                    int segment_id, int current_q_index, int plane_tx_type, int64_t* out);

/* §7.13.3 — inverse_transform_2d (src/transform.rs:707): w*h int64 -> w*h int64. */
void ora_inverse_transform_2d(const int64_t* dq, int tx, int tx_type, int bit_depth, int lossless, int64_t* res);

/* dequant + inverse transform + step-3 merge of every TU (in place on planes). */
void ora_recon_frame(const av1g_frame_header* hdr, const av1g_quant_params* q, const av1g_tu* tus, int n,
                     const int32_t* coeffs, ora_plane planes[3]);

/* intra_predict_block_samples (src/cdf.rs:16990-17250) reading plane p;
 * filter_intra_mode 0..4 or 255; pred receives w*h samples. */
void ora_intra_predict(const ora_plane* p, int sx, int sy, int tx, int mode, int angle_delta, int bd, int flags,
                       int filter_intra_mode, uint16_t* pred);

/* Every intra TU of a frame in decode order: prediction (intra modes,
 * palette from `maps`, intra block copy), chroma from luma, residual
 * (transform_block_emit order, src/cdf.rs:32540-32910).  Returns 0, or
 * 1 + the index of the first TU the reference rejects. */
int ora_intra_frame(const av1g_frame_header* hdr, const av1g_quant_params* q, const av1g_intra_tu* tus, int n,
                    const int32_t* coeffs, ora_plane planes[3], const uint8_t* maps, int64_t map_bytes,
                    const ora_plane* side);

/* The intra half of an inter-intra block: intra blended with the inter half
 * in side (mask_blend_interintra, inter_pred.rs:3272), written to out. */
int ora_interintra_blend(const av1g_frame_header* hdr, const av1g_intra_tu* t, int w, int h, const uint16_t* intra,
                         const ora_plane* side, ora_plane* out);

/* predict_intrabc_leaf_into_curr_frame (cdf.rs:19235) for one w x h region. */
int ora_intrabc_predict(const ora_plane* p, int plane, int ssx, int ssy, int mi_cols, int mi_rows, int x, int y,
                        int w, int h, int mv_row, int mv_col, int bd, uint16_t* pred);

/* Every inter prediction call of a frame in list order (predict_inter,
 * src/inter_pred.rs:2100, with the CurrFrame copy of its
 * reconstruct_inter_block* caller).  refs: dims of the 7 references;
 * ref_planes: their int32 planes, [ref * 3 + plane].  side: NULL, or 3
 * planes; an inter-intra call whose plane has one stores its clipped inter
 * prediction there instead of blending.  Returns 0, or 1 + the index of the
 * first call the reference rejects. */
int ora_inter_frame(const av1g_frame_header* hdr, const av1g_ref_frame* refs, const ora_plane* ref_planes,
                    const av1g_inter_pred* preds, int n, const av1g_obmc_neighbour* nb, int n_nb,
                    const av1g_warp_ctx* warps, int n_warps, ora_plane planes[3], ora_plane* side);

/* motion_vector_scaling (inter_pred.rs:318): out = startX, startY, stepX, stepY. */
int ora_mv_scaling(int plane, int ssx, int ssy, int fw, int fh, int ruw, int rh, int x, int y, int mv_row,
                   int mv_col, int32_t out[4]);
/* setup_shear (inter_pred.rs:3982): out = alpha, beta, gamma, delta, warpValid; -1 for None. */
int ora_setup_shear(const int32_t p[6], int32_t out[5]);
/* warp_estimation (inter_pred.rs:4083): returns LocalValid, fills params. */
int ora_warp_estimation(const av1g_warp_sample* cand, int n, int mi_row, int mi_col, int bw4, int bh4, int mv_row,
                        int mv_col, int32_t params[6]);
/* wedge_mask (inter_pred.rs:2844) into a block_width x block_height mask. */
int ora_wedge_mask(int mi_size, int idx, int sign, uint8_t* mask);

/* get_relative_dist (inter_pred.rs:3383). */
int ora_relative_dist(int a, int b, int bits);
/* §7.9.3 get_mv_projection (cdf.rs:35101). */
void ora_mv_projection(const int mv[2], int numerator, int denominator, int out[2]);
/* get_block_position (cdf.rs:35141): 1 and (*py, *px) when valid, else 0. */
int ora_block_position(int x8, int y8, int sign, int pr, int pc, int mi_rows, int mi_cols, int* py, int* px);
/* §7.19 storage (frame_driver.rs:1119-1160) for one job, host pointers. */
void ora_mf_store(const av1g_mf_store_job* job);
/* §7.9 motion_field_estimation_core (inter_pred.rs:7592) for one job, host
 * pointers; fills all of job->out. */
void ora_mf_project(const av1g_mf_project_job* job);

#ifdef __cplusplus
}
#endif

#endif
