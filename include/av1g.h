/*
 * av1g.h — C ABI of the B200 AV1 reconstruction + post-filter engine.
 *
 * The engine replaces the pixel stages of the reference decoder's frame
 * driver: everything in `decode_frame_spec_tiles` after the tile walk has
 * parsed the symbols (src/decoder/frame_driver.rs:790-1116 — deblock, CDEF,
 * superres, loop restoration, crop, pre-grain reference store, film grain,
 * narrow) plus the per-TU dequant / inverse transform / reconstruction merge
 * that the walker interleaves with parsing (src/cdf.rs:32482-32973).
 *
 * Conventions
 *  - Plain C types only; no CUDA or torch types appear in signatures.  Where a
 *    CUDA stream is accepted it is passed as `void*` (a cudaStream_t, NULL =
 *    legacy default stream).
 *  - Every entry point returns an av1g_status; nothing aborts the process.  A
 *    malformed descriptor yields AV1G_EINVAL, mirroring the reference's
 *    "typed error, never panic" contract (src/lib.rs:1937).
 *  - Sample planes hold 8-bit content as uint8_t and 10/12-bit content as
 *    uint16_t (little-endian), the same layout the reference surfaces
 *    (frame_driver.rs:1101-1116).  Strides are in bytes.
 *  - Per-mi grids are row-major MiRows x MiCols with stride MiCols, one entry
 *    per 4x4 luma cell, as the tile walker stores them (cdf.rs:15391-15940).
 */
#ifndef AV1G_H
#define AV1G_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AV1G_ABI_VERSION 1

typedef enum av1g_status {
    AV1G_OK = 0,
    AV1G_EINVAL = 1,         /* malformed descriptor or argument            */
    AV1G_ENOMEM_BUDGET = 2,  /* admission would exceed the engine HBM budget */
    AV1G_EBUSY = 3,          /* no free slot; retry after a poll/fetch       */
    AV1G_TIMEOUT = 4,        /* bounded wait expired                         */
    AV1G_EDEVICE = 5,        /* CUDA error (launch, copy, allocation)        */
    AV1G_EPARITY = 6,        /* debug self-check mismatch                    */
    AV1G_ENOTSUP = 7,        /* feature not handled by this build            */
    AV1G_ENOTREADY = 8,      /* ticket not finished yet (non-blocking poll);
                                av1g_decoder_receive_frame: no frame queued
                                (the reference's NeedMore)                    */
    AV1G_EOF = 9             /* av1g_decoder_receive_frame after flush with
                                nothing left (the reference's Eof)            */
} av1g_status;

/* ---------------------------------------------------------------------
 * Frame-level parameters (resolved header state)
 * ------------------------------------------------------------------- */

/* Film grain parameters after §5.9.30 resolution (the `update_grain == 0`
 * predicted path already applied by the caller, frame_driver.rs:1060-1075).
 * Field meaning follows FilmGrainParams (src/uncompressed_header_tail.rs:1763):
 * grain_scaling is GrainScaling (8..11), ar_coeff_shift is ArCoeffShift
 * (6..9). */
typedef struct av1g_film_grain {
    uint8_t apply_grain;
    uint8_t chroma_scaling_from_luma;
    uint16_t grain_seed;
    uint8_t num_y_points;
    uint8_t point_y_value[14];
    uint8_t point_y_scaling[14];
    uint8_t num_cb_points;
    uint8_t point_cb_value[10];
    uint8_t point_cb_scaling[10];
    uint8_t num_cr_points;
    uint8_t point_cr_value[10];
    uint8_t point_cr_scaling[10];
    uint8_t grain_scaling;
    uint8_t ar_coeff_lag;
    uint8_t ar_coeffs_y_plus_128[24];
    uint8_t ar_coeffs_cb_plus_128[25];
    uint8_t ar_coeffs_cr_plus_128[25];
    uint8_t ar_coeff_shift;
    uint8_t grain_scale_shift;
    uint8_t cb_mult;
    uint8_t cb_luma_mult;
    uint8_t cr_mult;
    uint8_t cr_luma_mult;
    uint8_t overlap_flag;
    uint8_t clip_to_restricted_range;
    uint16_t cb_offset;
    uint16_t cr_offset;
} av1g_film_grain;

/* Everything the post-filter chain reads from the sequence and frame
 * headers.  Names follow the spec / reference structs:
 *   sizes            — FrameSize (frame_header.rs), MiRows/MiCols
 *   loop filter      — LoopFilterParams (uncompressed_header_tail.rs:261)
 *   segmentation     — the SEG_LVL_ALT_LF_* features (1..4) of
 *                      SegmentationParams (uncompressed_header_tail.rs:554)
 *   cdef             — CdefParams (uncompressed_header_tail.rs:876); the
 *                      secondary strengths are the adjusted {0,1,2,4} values
 *   restoration      — LrParams (uncompressed_header_tail.rs:1079)
 *   film grain       — av1g_film_grain above. */
typedef struct av1g_frame_header {
    int32_t frame_width;      /* FrameWidth (post superres downscale)      */
    int32_t frame_height;     /* FrameHeight                               */
    int32_t upscaled_width;   /* UpscaledWidth (== frame_width w/o superres) */
    int32_t mi_rows;          /* MiRows                                    */
    int32_t mi_cols;          /* MiCols                                    */
    uint8_t bit_depth;        /* 8, 10 or 12                               */
    uint8_t subsampling_x;
    uint8_t subsampling_y;
    uint8_t num_planes;       /* 1 (monochrome) or 3                       */
    uint8_t matrix_coefficients;
    uint8_t use_superres;
    uint8_t coded_lossless;
    uint8_t allow_intrabc;
    uint8_t enable_cdef;      /* sequence header enable_cdef               */
    /* §5.9.11 loop filter */
    uint8_t lf_level[4];
    uint8_t lf_sharpness;
    uint8_t lf_delta_enabled;
    uint8_t delta_lf_multi;
    int8_t lf_ref_deltas[8];
    int8_t lf_mode_deltas[2];
    /* §5.9.14 segmentation, loop-filter features only: [segment][i] for
     * feature SEG_LVL_ALT_LF_Y_V + i, i = 0..3 */
    uint8_t seg_lf_active[8][4];
    int16_t seg_lf_data[8][4];
    /* §5.9.19 cdef */
    uint8_t cdef_short_circuited;
    uint8_t cdef_damping;
    uint8_t cdef_bits;
    uint8_t cdef_y_pri[8];
    uint8_t cdef_y_sec[8];
    uint8_t cdef_uv_pri[8];
    uint8_t cdef_uv_sec[8];
    /* §5.9.20 loop restoration: FrameRestorationType (0 none, 1 wiener,
     * 2 sgrproj, 3 switchable) and LoopRestorationSize per plane */
    uint8_t uses_lr;
    uint8_t lr_type[3];
    int32_t lr_unit_size[3];
    av1g_film_grain film_grain;
} av1g_frame_header;

/* Per-unit loop-restoration parameters (LrUnit, src/cdf.rs:15225).
 * type: 0 RESTORE_NONE, 1 RESTORE_WIENER, 2 RESTORE_SGRPROJ.
 * wiener[pass][i]: pass 0 vertical, pass 1 horizontal coefficients. */
typedef struct av1g_lr_unit {
    uint8_t type;
    uint8_t sgr_set;
    int8_t wiener[2][3];
    int16_t sgr_xqd[2];
} av1g_lr_unit;

/* Per-mi decode grids the post filters read (cdf.rs:15391-15940).  Each
 * pointer addresses mi_rows * mi_cols entries (delta_lf: 4 per cell). */
typedef struct av1g_mi_grid {
    const uint8_t* mi_size;       /* MiSizes, BLOCK_* ordinal               */
    const uint8_t* skip;          /* Skips                                  */
    const uint8_t* is_inter;      /* IsInters                               */
    const int8_t* ref_frame0;     /* RefFrames[.][.][0] (0 = INTRA_FRAME)   */
    const uint8_t* y_mode;        /* YModes                                 */
    const int8_t* segment_id;     /* SegmentIds (-1 = none)                 */
    const int8_t* delta_lf;       /* DeltaLFs[.][.][0..3]                   */
    const uint8_t* tx_size;       /* TxSizes (intra cells)                  */
    const uint8_t* inter_tx_size; /* InterTxSizes (inter cells)             */
} av1g_mi_grid;

/* One sample plane.  data is a device pointer for the av1g_run_* entry
 * points and a host pointer for av1g_submit_frame / av1g_fetch_output. */
typedef struct av1g_plane {
    void* data;
    int32_t stride;   /* bytes between rows                               */
    int32_t width;    /* samples                                          */
    int32_t height;   /* rows                                             */
} av1g_plane;

/* A frame's post-filter work in device memory.  The chain reads `recon`
 * (CurrFrame at the padded mi extent, (MiCols*4 >> ssx) x (MiRows*4 >> ssy))
 * and writes the intermediate planes named below.  Stages that the header
 * gates off (frame_driver.rs:832-836, 870, 906, 971, 1060) are skipped and the
 * next stage reads the previous stage's buffer instead.
 *   deblocked    — §7.14 output (padded extent)
 *   cdef         — §7.15 output (padded extent)
 *   up_deblocked — §7.16 upscale of `deblocked` (UpscaledWidth x FrameHeight)
 *   up_cdef      — §7.16 upscale of `cdef`      (UpscaledWidth x FrameHeight)
 *   lr           — §7.17 output; its crop to UpscaledWidth x FrameHeight is
 *                  the §7.20 reference payload (pre grain)
 *   out          — §7.18.3 film grain applied to the cropped frame
 * Buffers a frame does not need may be left NULL. */
typedef struct av1g_frame_job {
    const av1g_frame_header* hdr;   /* host pointer                        */
    av1g_mi_grid grid;              /* device pointers                     */
    const int8_t* cdef_idx;         /* device; cdef_idx per 64x64 luma
                                       block, ceil(MiRows/16) rows x
                                       ceil(MiCols/16) cols, -1 = off      */
    const av1g_lr_unit* lr_units[3]; /* device; unit_rows x unit_cols each  */
    av1g_plane recon[3];
    av1g_plane deblocked[3];
    av1g_plane cdef[3];
    av1g_plane up_deblocked[3];
    av1g_plane up_cdef[3];
    av1g_plane lr[3];
    av1g_plane out[3];
} av1g_frame_job;

/* ---------------------------------------------------------------------
 * Reconstruction (dequant, inverse transform, merge)
 * ------------------------------------------------------------------- */

/* Frame-level quantizer state (QuantizerParams, src/cdf.rs:13405) plus the
 * per-segment LosslessArray.  seg_qm_level[plane][segment]; a level of 15
 * means no quantizer matrix. */
typedef struct av1g_quant_params {
    uint8_t base_q_idx;
    int8_t delta_q_y_dc;
    int8_t delta_q_u_dc;
    int8_t delta_q_u_ac;
    int8_t delta_q_v_dc;
    int8_t delta_q_v_ac;
    uint8_t using_qmatrix;
    uint8_t delta_q_present;
    uint8_t segmentation_enabled;
    uint8_t seg_alt_q_active[8];
    uint8_t pad;
    int16_t seg_alt_q_data[8];
    uint8_t seg_qm_level[3][8];
    uint8_t lossless[8];
} av1g_quant_params;

/* One transform unit with coefficients (the reference reconstructs a TU only
 * when eob > 0, cdf.rs:32874; TUs without coefficients are not listed).
 * x, y: plane sample position of the TU; tx_type is PlaneTxType;
 * current_q_index is CurrentQIndex where the TU's block was decoded.
 * Its quantized levels are min(32,w) x min(32,h) int32 at coeff_offset in the
 * job's coefficient pool (row stride min(32,w), dequantize_step1's layout). */
typedef struct av1g_tu {
    uint16_t x;
    uint16_t y;
    uint8_t plane;
    uint8_t tx_size;
    uint8_t tx_type;
    uint8_t segment_id;
    uint8_t current_q_index;
    uint8_t pad[3];
    uint32_t coeff_offset;
} av1g_tu;

/* A frame's residual work: tus is a host array (the library buckets the TUs
 * by size and type and uploads them), coeffs a device array; planes hold the
 * prediction on entry (CurrFrame at the padded mi extent) and the
 * reconstruction on return. */
typedef struct av1g_recon_job {
    const av1g_frame_header* hdr;    /* host: bit depth, subsampling, mi dims */
    const av1g_quant_params* quant;  /* host */
    const av1g_tu* tus;              /* host */
    int32_t num_tus;
    const int32_t* coeffs;           /* device */
    av1g_plane planes[3];            /* device, updated in place */
} av1g_recon_job;

/* §7.12.3 dequantization + §7.13.3 inverse transform + §7.12.3 step-3 merge
 * for every listed TU of `n` frames.  Replaces the reconstruct tail of
 * transform_block_emit (src/cdf.rs:32874-32910): dequantize_step1
 * (cdf.rs:13655), inverse_transform_2d (src/transform.rs:707),
 * curr_frame_step3_merge (cdf.rs:17398). */
av1g_status av1g_run_recon(const av1g_recon_job* jobs, int32_t n, void* stream);

/* ---------------------------------------------------------------------
 * Intra prediction + reconstruction
 * ------------------------------------------------------------------- */

/* flags of av1g_intra_tu */
#define AV1G_INTRA_HAVE_ABOVE        0x01
#define AV1G_INTRA_HAVE_LEFT         0x02
#define AV1G_INTRA_HAVE_ABOVE_RIGHT  0x04
#define AV1G_INTRA_HAVE_BELOW_LEFT   0x08
#define AV1G_INTRA_EDGE_FILTER       0x10  /* enable_intra_edge_filter        */
#define AV1G_INTRA_FILTER_TYPE       0x20  /* get_filter_type() == 1 (smooth)  */
#define AV1G_INTRA_RESIDUAL          0x40  /* the TU has coefficients (eob>0)  */
#define AV1G_INTRA_CFL               0x80  /* chroma-from-luma on top of DC    */

/* mode values of av1g_intra_tu beyond the intra modes 0..12 */
#define AV1G_INTRA_MODE_PALETTE  64   /* §7.11.4 palette prediction              */
#define AV1G_INTRA_MODE_INTRABC  65   /* intra block copy from CurrFrame          */
#define AV1G_INTRA_MODE_NONE     255  /* no prediction (residual / CfL only)     */

/* One intra transform unit, in decode order, with the prediction inputs the
 * tile walker derives at transform_block_emit (src/cdf.rs:32540-32700):
 * mode is YMode for luma and UVMode for chroma with UV_CFL_PRED mapped to
 * DC_PRED; haveAbove / haveLeft are `avail || x/y > 0`; filter_intra_mode is
 * 0..4 or 255 for none (luma only).  For CfL TUs, cfl_alpha is CflAlphaU/V and
 * max_luma_w/h are MaxLumaW/H (luma samples) of the block.  `res` is the
 * residual (used when AV1G_INTRA_RESIDUAL is set); res.x/y/plane/tx_size must
 * equal the TU's.
 * AV1G_INTRA_MODE_PALETTE (predict_palette_tu_into_curr_frame,
 * cdf.rs:18603): the TU's colour indices start at palette_map in the job's
 * map pool with row stride palette_stride; palette_colors[0..palette_size).
 * AV1G_INTRA_MODE_INTRABC (predict_intrabc_leaf_into_curr_frame,
 * cdf.rs:19235): the TU-sized piece at (x, y) of a block predicted from the
 * pre-filter CurrFrame with the block's mv = {row, col} (1/8 luma samples);
 * list one piece per transform-sized part of the block, before its residual
 * TUs.
 * interintra != 0: the TU is a whole inter-intra block of one plane (tx_size
 * = the block size, mode = the intra mode of interintra_mode: DC, V, H or
 * SMOOTH): its intra prediction is blended with the inter prediction the
 * inter pass left in the job's interintra_in plane (mask_blend_interintra,
 * inter_pred.rs:3272), which is what predict_inter does with the intra
 * prediction in CurrFrame; list the block's residual TUs after it (mode
 * AV1G_INTRA_MODE_NONE). */
typedef struct av1g_intra_tu {
    uint16_t x;
    uint16_t y;
    uint8_t plane;
    uint8_t tx_size;
    uint8_t mode;
    uint8_t flags;
    int8_t angle_delta;
    int8_t cfl_alpha;
    uint8_t filter_intra_mode;
    uint8_t pad;
    uint16_t max_luma_w;
    uint16_t max_luma_h;
    av1g_tu res;
    int16_t mv[2];
    uint32_t palette_map;
    uint16_t palette_stride;
    uint8_t palette_size;
    uint8_t pad2;
    uint16_t palette_colors[8];
    uint8_t interintra;          /* 0, or the intra half of an inter-intra block:
                                    1 smooth mask, 2 wedge mask */
    uint8_t interintra_mode;     /* II_DC_PRED..II_SMOOTH_PRED (mask of kind 1) */
    uint8_t wedge_index;         /* kind 2 (wedge_sign 0) */
    uint8_t mi_size;             /* kind 2: the luma block size */
} av1g_intra_tu;

/* A frame's intra work, reconstructed in place on top of whatever the
 * planes already hold (inter predictions + residuals of inter blocks).
 * tus: host array in decode order; coeffs: device pool; planes: device. */
typedef struct av1g_intra_job {
    const av1g_frame_header* hdr;    /* host */
    const av1g_quant_params* quant;  /* host */
    const av1g_intra_tu* tus;        /* host, decode order */
    int32_t num_tus;
    int32_t sb_size;                 /* 64 or 128 (luma samples) */
    const int32_t* coeffs;           /* device */
    av1g_plane planes[3];            /* device, updated in place */
    const uint8_t* palette_maps;     /* host: colour-index pool of palette TUs */
    int64_t palette_map_bytes;
    av1g_plane interintra_in[3];     /* device: inter halves of inter-intra blocks */
} av1g_intra_job;

/* §7.11.2 intra prediction (DC, V, H, directional with edge filter and
 * upsampling, SMOOTH*, PAETH, recursive filter intra), §7.11.5 chroma from
 * luma, then dequant + inverse transform + merge, for every intra TU of `n`
 * frames.  Returns once the launch has finished: AV1G_EDEVICE names the job
 * one of whose superblock dependency waits ran out of time (a bounded wait,
 * 2 s; only that job's samples are incomplete, and later calls are not
 * affected).  Replaces predict_intra_into_curr_frame (src/cdf.rs:16789),
 * intra_predict_block_samples (cdf.rs:16990-17250), the kernels at
 * cdf.rs:1348-3120 and predict_chroma_from_luma_into_curr_frame
 * (cdf.rs:17256) as called from transform_block_emit (cdf.rs:32482).
 * One persistent launch for all frames: the host plan records, per
 * superblock, which levels of which earlier superblocks its TUs read (the
 * edges and copies the TUs' availability flags and vectors name), and a
 * superblock waits only for those, so superblocks of different tiles (whose
 * TUs read nothing across the tile edge) run side by side. */
av1g_status av1g_run_intra(const av1g_intra_job* jobs, int32_t n, void* stream);

/* The plan av1g_run_intra would build for these jobs, without running it
 * (host only; the jobs' device pointers are not read).  depth: superblocks
 * on the longest chain of waits; width: most superblocks at one depth. */
typedef struct av1g_intra_plan_stats {
    int32_t superblocks;
    int32_t tus;
    int32_t waits;
    int32_t depth;
    int32_t width;
    int32_t pad;
} av1g_intra_plan_stats;
av1g_status av1g_intra_plan_stats_get(const av1g_intra_job* jobs, int32_t n, av1g_intra_plan_stats* out);

/* Test hook for the wait bound above, on the current device: wait_ns sets
 * the bound (<= 0 restores 2 s) and, while frame_width > 0, every intra job
 * whose frame is that wide gets a superblock wait that nothing satisfies, so
 * its wait runs out after wait_ns.  No counterpart in the reference (its
 * decode is single-threaded and never waits). */
av1g_status av1g_test_intra_wait_fault(int64_t wait_ns, int32_t frame_width);

/* ---------------------------------------------------------------------
 * Inter prediction
 * ------------------------------------------------------------------- */

/* One reference-store entry as the inter predictor reads it: the stored
 * (cropped, upscaled, pre-grain) planes and the stored frame's LUMA extents,
 * which serve both as RefUpscaledWidth / RefFrameHeight of the §7.11.3.3
 * scale and as the clamp extents of §7.11.3.4 / §7.11.3.5
 * (RefFrameStoreEntry as built at src/decoder/frame_driver.rs:566-583).
 * Each plane must hold at least ((upscaled_width + ss) >> ss) x
 * ((frame_height + ss) >> ss) samples.  planes: device. */
typedef struct av1g_ref_frame {
    av1g_plane planes[3];
    int32_t upscaled_width;
    int32_t frame_height;
} av1g_ref_frame;

/* WarpDriverParams (src/inter_pred.rs:1420-1429): the useWarp inputs of one
 * prediction, per reference list. */
typedef struct av1g_warp_ctx {
    int32_t gm_params[2][6];
    int32_t local_warp_params[6];
    uint8_t y_mode[2];
    uint8_t gm_type[2];
    uint8_t local_valid;
    uint8_t ref_is_scaled[2];
    uint8_t force_integer_mv;
} av1g_warp_ctx;

/* ObmcNeighbour (src/inter_pred.rs:1430-1437): one above or left neighbour
 * of an OBMC block.  ref: 0..6 = LAST_FRAME..ALTREF_FRAME; axis_pos4: the
 * neighbour's mi column (above pass) or mi row (left pass). */
typedef struct av1g_obmc_neighbour {
    int16_t mv[2];
    uint16_t axis_pos4;
    uint8_t ref;
    uint8_t step4;
    uint8_t filter_x;
    uint8_t filter_y;
    uint8_t pad[2];
} av1g_obmc_neighbour;

/* kind of av1g_inter_pred */
#define AV1G_INTER_SINGLE     0
#define AV1G_INTER_COMPOUND   1
#define AV1G_INTER_INTRA      2   /* IsInterIntra: blends with CurrFrame */

/* One predict_inter call (src/inter_pred.rs:2100-2510) together with the
 * CurrFrame write of its caller (reconstruct_inter_block*,
 * inter_pred.rs:4881-6010: the w x h prediction clipped to the plane).
 * x, y, w, h are in the plane's samples; the subsampling of plane > 0 is the
 * header's.  filter_x = InterpFilter[1], filter_y = InterpFilter[0], 0..5.
 * mv[list] = {row, col} in 1/8 luma samples.  compound_type: 0 WEDGE,
 * 1 DIFFWTD, 2 AVERAGE, 4 DISTANCE (with fwd/bck_weight).  Wedge masks use
 * mi_size (the luma block size), wedge_index and wedge_sign; an inter-intra
 * wedge uses wedge_sign 0.  A DIFFWTD chroma call reads the mask its block's
 * plane-0 call computed (the mask of the luma samples at (x << ss, y << ss)),
 * so list the plane-0 call of each DIFFWTD block too.  AV1G_INTER_INTRA
 * blends with the intra prediction the CurrFrame region holds on entry — or,
 * when the job's interintra_out plane of that plane is given, stores its
 * clipped inter prediction Clip1(Round2(preds[0], InterPostRound)) there
 * instead (CurrFrame untouched) for av1g_run_intra to blend once the intra
 * half exists (no OBMC on such calls).
 * warp: index into the job's warps (-1: no warp context).  motion_mode 1
 * (OBMC) uses obmc_above + obmc_left neighbours from obmc_first (above ones
 * first) with the ObmcParams fields below (inter_pred.rs:1438-1450).
 * Calls of one job must cover disjoint CurrFrame regions. */
typedef struct av1g_inter_pred {
    uint16_t x;
    uint16_t y;
    uint16_t w;
    uint16_t h;
    uint8_t plane;
    uint8_t kind;
    uint8_t motion_mode;        /* 0 SIMPLE, 1 OBMC, 2 WARPED_CAUSAL */
    uint8_t filter_x;
    uint8_t filter_y;
    uint8_t ref[2];
    uint8_t compound_type;
    int16_t mv[2][2];
    uint8_t mi_size;
    uint8_t wedge_index;
    uint8_t wedge_sign;
    uint8_t mask_type;
    uint8_t interintra_mode;    /* II_DC_PRED..II_SMOOTH_PRED */
    uint8_t wedge_interintra;
    uint8_t fwd_weight;
    uint8_t bck_weight;
    int32_t warp;
    uint32_t obmc_first;
    uint8_t obmc_above;
    uint8_t obmc_left;
    uint8_t avail_u;
    uint8_t avail_l;
    uint8_t plane_residual_ge_8x8;
    uint8_t mi_width_log2;
    uint8_t mi_height_log2;
    uint8_t pad;
    uint16_t mi_row;
    uint16_t mi_col;
} av1g_inter_pred;

/* A frame's inter predictions.  hdr gives bit depth, subsampling, FrameWidth
 * / FrameHeight (frame_width, frame_height: the §7.11.3.3 scale divisors)
 * and mi dims; refs: 7 entries, LAST_FRAME..ALTREF_FRAME. */
typedef struct av1g_inter_job {
    const av1g_frame_header* hdr;           /* host */
    const av1g_ref_frame* refs;             /* host array of 7 */
    const av1g_inter_pred* preds;           /* host */
    int32_t num_preds;
    const av1g_obmc_neighbour* neighbours;  /* host */
    int32_t num_neighbours;
    const av1g_warp_ctx* warps;             /* host */
    int32_t num_warps;
    av1g_plane planes[3];                   /* CurrFrame, device, written */
    av1g_plane interintra_out[3];           /* device or NULL, see below */
} av1g_inter_job;

/* WarpSampleCand (src/inter_pred.rs:4030): one §7.10.4 warp sample. */
typedef struct av1g_warp_sample {
    int32_t sy, sx, dy, dx;
} av1g_warp_sample;

/* The §7.11.3.8 least-squares local warp fit of a WARPED_CAUSAL block
 * (warp_estimation, src/inter_pred.rs:4083, called by the tile walker at
 * cdf.rs:30929): at most 8 samples are used.  Writes LocalWarpParams and
 * LocalValid.  A host function (eight samples per block); its output feeds
 * av1g_warp_ctx.local_warp_params / local_valid. */
av1g_status av1g_warp_estimation(const av1g_warp_sample* cands, int32_t n, int32_t mi_row, int32_t mi_col,
                                 int32_t block_w4, int32_t block_h4, int16_t mv_row, int16_t mv_col,
                                 int32_t params[6], uint8_t* valid);

/* §7.11.3 inter prediction for every listed call of `n` frames: motion
 * vector scaling (§7.11.3.3), 8-tap sub-sample interpolation with scaled
 * references (§7.11.3.4), local / global warp (§7.11.3.5-6), OBMC
 * (§7.11.3.9-10), wedge / difference-weight / inter-intra masks and blends
 * (§7.11.3.11-14), distance weights (§7.11.3.15).  Replaces predict_inter
 * (src/inter_pred.rs:2100) as called by reconstruct_inter_block,
 * _warp, _obmc, _compound and _interintra (inter_pred.rs:4881-6010).
 * One launch for all frames, plus one for DIFFWTD chroma calls. */
av1g_status av1g_run_inter(const av1g_inter_job* jobs, int32_t n, void* stream);

/* ---------------------------------------------------------------------
 * Motion-field motion vectors: §7.19 storage and §7.9 projection
 * ------------------------------------------------------------------- */

/* MotionFieldMvs entry of a position no projection reached (MFMV_INVALID,
 * src/cdf.rs:515). */
#define AV1G_MFMV_INVALID (-32768)

/* One decoded frame's §7.19 motion field motion vector storage: filters the
 * block walker's per-4x4-cell RefFrames[2] / Mvs[2][2] down to the one
 * candidate per cell that a later frame's §7.9 projection reads.  Per cell,
 * the last list whose reference (1..7) lies in the past
 * (get_relative_dist(ref_order_hint[r - 1], order_hint) < 0) and whose MV
 * components are within +-(1 << 12) - 1; -1 / {0, 0} otherwise, and for every
 * cell of a frame that is not an inter frame.  Cell values outside 1..7 are no
 * reference.  Arrays are device memory, row-major over mi_rows x mi_cols
 * cells; ref_frames 2-byte, mvs 8-byte and mf_mvs 4-byte aligned. */
typedef struct av1g_mf_store_job {
    int32_t mi_rows, mi_cols;
    int32_t is_inter_frame;
    int32_t order_hint;          /* OrderHint of the frame */
    int32_t hint_bits;           /* OrderHintBits, 0 when enable_order_hint is 0 */
    int32_t ref_order_hint[7];   /* RefOrderHint[ref_frame_idx[i]], LAST..ALTREF */
    const int8_t* ref_frames;    /* device: [cell][list] */
    const int16_t* mvs;          /* device: [cell][list][row, col] */
    int8_t* mf_ref_frames;       /* device out: [cell] */
    int16_t* mf_mvs;             /* device out: [cell][row, col] */
} av1g_mf_store_job;

/* Replaces the §7.19 loop of decode_frame_spec_tiles
 * (src/decoder/frame_driver.rs:1119-1160) for `n` frames in one launch. */
av1g_status av1g_run_mf_store(const av1g_mf_store_job* jobs, int32_t n, void* stream);

/* One §7.20 reference slot as the projection reads it (MotionFieldSlot,
 * src/inter_pred.rs:7567-7586): the stored frame's av1g_mf_store_job outputs
 * (device, 4-byte aligned mf_mvs), SavedOrderHints[0..8], mi extent and
 * FrameIsIntra.  mf_ref_frames == NULL marks an empty slot; stored
 * reference values outside 1..7 are no candidate. */
typedef struct av1g_mf_slot {
    const int16_t* mf_mvs;
    const int8_t* mf_ref_frames;
    int32_t saved_order_hints[8];
    int32_t mi_rows, mi_cols;
    int32_t frame_is_intra;
    int32_t pad;
} av1g_mf_slot;

/* The current frame's §7.9 motion_field_estimation inputs
 * (motion_field_estimation_core, src/inter_pred.rs:7592): the eight slots,
 * ref_frame_idx[0..7], OrderHints[0..8] (index LAST_FRAME + i holds the
 * order hint of reference i), OrderHint, OrderHintBits (0 when order hints
 * are off) and the frame's mi extent.  out is a device array of
 * 7 x (mi_rows >> 1) x (mi_cols >> 1) x 2 int16, MotionFieldMvs layout
 * [ref - LAST_FRAME][y8][x8][row, col] (src/cdf.rs:34989), 4-byte aligned;
 * every entry is written (AV1G_MFMV_INVALID where no projection lands). */
typedef struct av1g_mf_project_job {
    av1g_mf_slot slots[8];
    int32_t ref_frame_idx[7];
    int32_t pad;
    int32_t order_hints[8];
    int32_t order_hint;
    int32_t hint_bits;
    int32_t mi_rows, mi_cols;
    int16_t* out;
} av1g_mf_project_job;

/* §7.9.1-§7.9.4 for `n` frames: the projection passes (LAST, BWDREF,
 * ALTREF2, ALTREF, LAST2 with the reference's selection and stamp rules,
 * src/inter_pred.rs:7716-7741) over every stored cell at once.  Where several
 * cells land on one position the reference's sequential order decides — the
 * last pass, then the last cell in raster order, wins — so the result equals
 * the reference's grid entry for entry. */
av1g_status av1g_run_mf_project(const av1g_mf_project_job* jobs, int32_t n, void* stream);

/* ---------------------------------------------------------------------
 * Large-scale tile (§7.3): output assembly of decoded camera tiles
 * ------------------------------------------------------------------- */

/* Where one decoded camera tile lies: the CurrFrame planes its §7.3.2
 * decode wrote (device, the camera frame's extent) and the tile's luma
 * origin in them (MiColStart * 4, MiRowStart * 4). */
typedef struct av1g_tile_list_entry {
    av1g_plane src[3];
    int32_t x0, y0;
} av1g_tile_list_entry;

/* One tile list's output frame (decode_tile_list, src/tile_list.rs:651-740):
 * tile_width x tile_height luma samples per tile (TileWidth, TileHeight),
 * an output of width_in_tiles x height_in_tiles tiles
 * (output_frame_*_in_tiles_minus_1 + 1), num_entries decoded tiles (host
 * array) placed in raster order; output tile positions no entry covers are
 * zero, as the reference's output buffer starts.  out: device planes of
 * width_in_tiles * tile_width x height_in_tiles * tile_height luma samples
 * (chroma >> subsampling), u8 for 8-bit content, u16 otherwise. */
typedef struct av1g_tile_list_job {
    int32_t tile_width, tile_height;
    int32_t width_in_tiles, height_in_tiles;
    int32_t num_planes, subsampling_x, subsampling_y, bit_depth;
    int32_t num_entries;
    int32_t pad;
    const av1g_tile_list_entry* entries;
    av1g_plane out[3];
} av1g_tile_list_job;

/* The §7.3.1 output placement for `n` tile lists in one launch; the camera
 * tiles themselves are decoded by the batched reconstruction entry points
 * (each tile an independent job with its anchor frame as reference), not one
 * after the other as the reference does. */
av1g_status av1g_run_tile_list_output(const av1g_tile_list_job* jobs, int32_t n, void* stream);

/* ---------------------------------------------------------------------
 * Serving engine: streams, device-resident reference slots, tickets
 * ------------------------------------------------------------------- */

typedef struct av1g_engine av1g_engine;
typedef struct av1g_stream av1g_stream;

typedef struct av1g_config {
    int32_t device;              /* CUDA device ordinal                           */
    int32_t max_batch;           /* frames (one per stream) per step; 0 = 64      */
    int64_t hbm_budget_bytes;    /* admission budget; 0 = 80% of free memory      */
    int32_t max_inflight_steps;  /* steps enqueued ahead of completion, per lane;
                                    0 = 3                                         */
    int32_t lanes;               /* worker threads, each with a CUDA stream; a
                                    stream of frames stays on one lane; 0 = 4     */
    const char* autotune_cache;  /* NULL, or a file av1g_autotune_postfilter
                                    wrote: loaded at create                       */
    int64_t max_step_samples;    /* a step takes frames until their luma samples
                                    would pass this (at least one frame):
                                    small frames batch, large ones pipeline;
                                    0 = 4,194,304 (two 1080p frames), < 0 =
                                    no limit                                      */
} av1g_config;

/* What a stream's sequence header fixes: the largest upscaled frame and the
 * sample format.  When the stream opens, the engine reserves in its budget
 * nine slot payloads of that size (the eight reference slots and the one a
 * refresh writes before it replaces an older one). */
typedef struct av1g_seq_info {
    int32_t max_width;
    int32_t max_height;
    uint8_t bit_depth;
    uint8_t subsampling_x;
    uint8_t subsampling_y;
    uint8_t num_planes;
    int32_t sb_size;             /* 64 or 128 */
} av1g_seq_info;

/* One frame as the tile walker hands it over (all pointers HOST memory; the
 * engine copies what it needs before av1g_submit_frame returns).  Decoding
 * runs: inter predictions (references: the stream's slots named by
 * ref_frame_idx), inter residuals, the intra wavefront, then the §7.4
 * post-filter chain (decode_frame_spec_tiles, frame_driver.rs:790-1116),
 * the §7.20 slot refresh with the pre-grain frame (reference_frame_update,
 * frame_driver.rs:1409) and, if shown, the output.  show_existing_frame
 * outputs slot frame_to_show_map_idx with its stored grain parameters
 * (output_existing_frame, frame_driver.rs:1495) and refreshes the slots in
 * refresh_frame_flags with it. */
typedef struct av1g_frame_desc {
    const av1g_frame_header* hdr;
    const av1g_quant_params* quant;
    av1g_mi_grid grid;
    const int8_t* cdef_idx;
    const av1g_lr_unit* lr_units[3];
    const av1g_inter_pred* inter_preds;
    int32_t num_inter_preds;
    const av1g_obmc_neighbour* neighbours;
    int32_t num_neighbours;
    const av1g_warp_ctx* warps;
    int32_t num_warps;
    const av1g_tu* inter_tus;           /* residuals of inter blocks            */
    int32_t num_inter_tus;
    const av1g_intra_tu* intra_tus;     /* decode order                          */
    int32_t num_intra_tus;
    const uint8_t* palette_maps;
    int64_t palette_map_bytes;
    const int32_t* coeffs;              /* pool indexed by coeff_offset          */
    int64_t num_coeffs;
    uint8_t ref_frame_idx[7];           /* slot of LAST_FRAME..ALTREF_FRAME      */
    uint8_t refresh_frame_flags;
    uint8_t show_frame;
    uint8_t show_existing_frame;
    uint8_t frame_to_show_map_idx;
    uint8_t pad;
} av1g_frame_desc;

/* A finished frame: cropped planes with tight strides (width x 1 or 2 bytes,
 * SpecFrame layout, frame_driver.rs:64-77) in engine-owned pinned host memory,
 * valid until av1g_release_output.  latency_ms: submit to completion. */
typedef struct av1g_frame_out {
    av1g_plane planes[3];
    int32_t num_planes;
    int32_t bit_depth;
    int32_t shown;
    int32_t pad;
    double latency_ms;
} av1g_frame_out;

typedef struct av1g_engine_stats {
    int64_t frames_done;
    int64_t steps_done;
    int64_t bytes_reserved;     /* reference slots of open streams             */
    int64_t bytes_in_flight;    /* work buffers of enqueued steps              */
    int64_t budget;
    int32_t streams_open;
    int32_t pad;
    double host_ms;             /* worker time spent preparing and enqueuing steps */
    double device_ms;           /* device time of the finished steps (events)      */
    double host_stage_ms[6];    /* host_ms by part: uploads, inter, residual, intra,
                                   post-filter, slots + outputs                    */
} av1g_engine_stats;

av1g_status av1g_engine_create(const av1g_config* cfg, av1g_engine** out);
/* Waits (bounded) for enqueued work, then frees everything. */
void av1g_engine_destroy(av1g_engine* e);
av1g_status av1g_engine_get_stats(av1g_engine* e, av1g_engine_stats* out);

/* AV1G_ENOMEM_BUDGET when the stream's reference slots do not fit the
 * remaining budget (retry after another stream closes). */
av1g_status av1g_stream_open(av1g_engine* e, const av1g_seq_info* seq, av1g_stream** out);
/* Waits for the stream's frames, then releases its slots and outputs. */
av1g_status av1g_stream_close(av1g_stream* s);
/* reset_references (frame_driver.rs:1401), ordered after frames already
 * submitted on the stream. */
av1g_status av1g_stream_reset_refs(av1g_stream* s);

/* Queues a frame; *ticket identifies it.  Frames of one stream run in
 * submission order; frames of different streams are batched into shared
 * launches (one per stage per step). */
av1g_status av1g_submit_frame(av1g_stream* s, const av1g_frame_desc* d, uint64_t* ticket);
/* Waits up to timeout_ns (0: no wait) for the ticket.  Returns AV1G_OK with
 * *result = the frame's status once finished, AV1G_TIMEOUT (timeout > 0) or
 * AV1G_ENOTREADY (timeout 0) otherwise. */
av1g_status av1g_poll(av1g_engine* e, uint64_t ticket, int64_t timeout_ns, av1g_status* result);
/* The finished frame of a ticket (its status is returned).  When a frame
 * failed, av1g_poll and av1g_fetch_output leave the reason in the calling
 * thread's av1g_last_error(). */
av1g_status av1g_fetch_output(av1g_stream* s, uint64_t ticket, av1g_frame_out* out);
/* Frees a finished ticket and its output buffer. */
av1g_status av1g_release_output(av1g_stream* s, uint64_t ticket);

/* Launch modes for av1g_run_postfilter. */
#define AV1G_MODE_BATCHED 0     /* one launch per stage across all jobs    */
#define AV1G_MODE_PER_FRAME 1   /* one launch per stage per frame          */

/* ---------------------------------------------------------------------
 * Framing (host functions, no device work): IVF files, §5.3 OBUs,
 * Annex B length-delimited streams, §5.5 sequence headers, the §7.5
 * temporal-unit OBU walk and the leading fields of §5.9.2 frame headers.
 * A malformed input returns AV1G_EINVAL; av1g_framing_error() then names
 * the reference's error variant and av1g_last_error() gives the text.
 * ------------------------------------------------------------------- */

#define AV1G_FE_NONE 0
#define AV1G_FE_UNEXPECTED_END 1          /* Error::UnexpectedEnd, IvfReadError::UnexpectedEnd */
#define AV1G_FE_FORBIDDEN_BIT_SET 2       /* Error::ForbiddenBitSet                            */
#define AV1G_FE_MISSING_SIZE_FIELD 3      /* Error::MissingSizeField                           */
#define AV1G_FE_LEB128_OVERFLOW 4         /* Error::Leb128Overflow (value > 2^32 - 1)          */
#define AV1G_FE_LEB128_TOO_LONG 5         /* Error::Leb128TooLong (8 continuation bytes)       */
#define AV1G_FE_SIZE_OVERFLOW 6           /* Error::SizeOverflow                               */
#define AV1G_FE_ANNEXB_INVALID 7          /* Error::AnnexBInvalid                              */
#define AV1G_FE_IVF_BAD_MAGIC 8           /* IvfReadError::BadMagic                            */
#define AV1G_FE_IVF_UNSUPPORTED_VERSION 9 /* IvfReadError::UnsupportedVersion                  */
#define AV1G_FE_IVF_UNSUPPORTED_HEADER_LENGTH 10 /* IvfReadError::UnsupportedHeaderLength      */
#define AV1G_FE_RESERVED_PROFILE 11       /* Error::ReservedProfile (seq_profile > 2)          */
#define AV1G_FE_REDUCED_STILL_REQUIRES_STILL 12 /* Error::ReducedStillRequiresStill            */
#define AV1G_FE_OPERATING_POINT_OUT_OF_RANGE 13 /* Error::OperatingPointOutOfRange             */
#define AV1G_FE_OUTPUT_TOO_SMALL 14       /* the caller's output buffer (no reference variant) */
#define AV1G_FE_UNSUPPORTED_OBU 15        /* a reserved OBU type in a temporal unit (the
                                             reference's walk rejects it as well)             */
#define AV1G_FE_TEMPORAL_POINT_INFO_UNSUPPORTED 16 /* Error::TemporalPointInfoUnsupported      */
int32_t av1g_framing_error(void);

/* OBU type values (§6.2.2, ObuType, src/obu.rs). */
#define AV1G_OBU_SEQUENCE_HEADER 1
#define AV1G_OBU_TEMPORAL_DELIMITER 2
#define AV1G_OBU_FRAME_HEADER 3
#define AV1G_OBU_TILE_GROUP 4
#define AV1G_OBU_METADATA 5
#define AV1G_OBU_FRAME 6
#define AV1G_OBU_REDUNDANT_FRAME_HEADER 7
#define AV1G_OBU_TILE_LIST 8
#define AV1G_OBU_PADDING 15

/* One OBU (ObuDescriptor, src/obu.rs): the raw 4-bit type, the header
 * flags, temporal / spatial id (0 without an extension), header_len (header +
 * extension + obu_size bytes), and where its payload lies: payload_offset
 * bytes from the start of the buffer the call parsed. */
typedef struct av1g_obu {
    int32_t obu_type;
    int32_t extension_flag;
    int32_t has_size_field;
    int32_t temporal_id;
    int32_t spatial_id;
    int32_t header_len;
    uint64_t payload_offset;
    uint64_t payload_len;
} av1g_obu;

/* §4.10.5 leb128 (parse_leb128, src/obu.rs): value and bytes used. */
av1g_status av1g_leb128(const uint8_t* p, size_t n, uint64_t* value, int32_t* len);
/* §5.3.1-§5.3.3 one OBU at p (parse_obu, src/obu.rs): the low-overhead
 * format, so obu_has_size_field must be 1.  *consumed = header + payload. */
av1g_status av1g_parse_obu(const uint8_t* p, size_t n, av1g_obu* out, uint64_t* consumed);

/* IVF file header (IvfFileHeader, src/encoder/ivf.rs:205). */
typedef struct av1g_ivf_header {
    uint16_t version;
    uint16_t header_length;
    uint8_t fourcc[4];
    uint16_t width;
    uint16_t height;
    uint32_t fps_num;
    uint32_t fps_den;
    uint32_t frame_count;
} av1g_ivf_header;
/* One IVF frame record: its timestamp and the payload's place in the file. */
typedef struct av1g_ivf_frame {
    uint64_t pts;
    uint64_t offset;
    uint64_t size;
} av1g_ivf_frame;
/* parse_file_header (ivf.rs:242): DKIF magic, version 0, 32-byte header. */
av1g_status av1g_ivf_parse_header(const uint8_t* p, size_t n, av1g_ivf_header* out);
/* IvfReader::read_next_frame (ivf.rs:309): *cursor starts at 32; on return
 * *got = 1 with the frame and *cursor past it, or *got = 0 at the end. */
av1g_status av1g_ivf_next_frame(const uint8_t* p, size_t n, uint64_t* cursor, av1g_ivf_frame* out, int32_t* got);

/* Annex B -> §7.5 low-overhead temporal units (split_temporal_units,
 * src/annexb.rs:66): every OBU gains an obu_size field where it had none, a
 * temporal unit must open with its temporal delimiter and sizes must nest
 * exactly.  The units are written back to back into out (never longer than
 * the input, so cap >= n always suffices); tu_end[i] is the end offset of
 * unit i in out; at most tu_cap units. */
av1g_status av1g_annexb_split(const uint8_t* p, size_t n, uint8_t* out, size_t cap, uint64_t* tu_end,
                              int32_t tu_cap, int32_t* n_tu, uint64_t* out_len);
/* Low-overhead temporal units -> Annex B (build_from_temporal_units,
 * annexb.rs:185): unit i is tus[tu_end[i-1] .. tu_end[i]).  out == NULL
 * only measures: *out_len receives the size the stream needs. */
av1g_status av1g_annexb_build(const uint8_t* tus, const uint64_t* tu_end, int32_t n_tu, uint8_t* out, size_t cap,
                              uint64_t* out_len);

/* §5.5 sequence header (SequenceHeader, src/sequence_header.rs), flattened:
 * one entry per operating point (at most 32). */
typedef struct av1g_operating_point {
    uint16_t idc;                  /* operating_point_idc                     */
    uint8_t seq_level_idx;
    uint8_t seq_tier;
    uint8_t decoder_model_present;
    uint8_t initial_display_delay_present;
    uint8_t initial_display_delay_minus_1;
    uint8_t low_delay_mode_flag;
    uint64_t decoder_buffer_delay;
    uint64_t encoder_buffer_delay;
} av1g_operating_point;

typedef struct av1g_sequence_header {
    uint8_t seq_profile, still_picture, reduced_still_picture_header;
    uint8_t timing_info_present_flag, equal_picture_interval;
    uint8_t decoder_model_info_present_flag, initial_display_delay_present_flag;
    uint8_t operating_points_cnt_minus_1;
    uint32_t num_units_in_display_tick, time_scale, num_ticks_per_picture_minus_1;
    uint8_t buffer_delay_length_minus_1, buffer_removal_time_length_minus_1;
    uint8_t frame_presentation_time_length_minus_1, pad0;
    uint32_t num_units_in_decoding_tick;
    av1g_operating_point operating_points[32];
    uint8_t frame_width_bits_minus_1, frame_height_bits_minus_1;
    uint8_t frame_id_numbers_present_flag, delta_frame_id_length_minus_2, additional_frame_id_length_minus_1;
    uint8_t use_128x128_superblock, enable_filter_intra, enable_intra_edge_filter;
    uint32_t max_frame_width_minus_1, max_frame_height_minus_1;
    uint8_t enable_interintra_compound, enable_masked_compound, enable_warped_motion, enable_dual_filter;
    uint8_t enable_order_hint, enable_jnt_comp, enable_ref_frame_mvs;
    uint8_t seq_force_screen_content_tools, seq_force_integer_mv, order_hint_bits;
    uint8_t enable_superres, enable_cdef, enable_restoration;
    /* §5.5.2 color config */
    uint8_t high_bitdepth, twelve_bit, bit_depth, mono_chrome, num_planes;
    uint8_t color_description_present_flag, color_primaries, transfer_characteristics, matrix_coefficients;
    uint8_t color_range, subsampling_x, subsampling_y, chroma_sample_position, separate_uv_delta_q;
    uint8_t film_grain_params_present;
    uint8_t pad1[3];
    uint32_t bits_consumed;
} av1g_sequence_header;

/* parse_sequence_header (src/sequence_header.rs) of an OBU payload. */
av1g_status av1g_parse_sequence_header(const uint8_t* payload, size_t n, av1g_sequence_header* out);
/* The engine's stream parameters from a sequence header: the largest frame,
 * sample format and superblock size (what av1g_stream_open needs). */
av1g_status av1g_seq_info_from_header(const av1g_sequence_header* sh, av1g_seq_info* out);

/* The OBU walk of one temporal unit (decode_temporal_unit_spec,
 * src/decoder/frame_driver.rs:1590-1650): OBUs outside the chosen operating
 * point are dropped (an extension header whose temporal / spatial id is not
 * in *op_idc), a sequence header is parsed into *seq (*have_seq = 1) and
 * selects *op_idc = operating_points[chosen_op].idc, and the OBUs the frame
 * decode acts on — sequence header, frame header, redundant frame header,
 * tile group, frame — are listed in order (temporal delimiters, padding,
 * metadata and tile lists are passed over).  *op_idc, *seq and *have_seq
 * carry from one unit of a stream to the next. */
av1g_status av1g_temporal_unit_obus(const uint8_t* tu, size_t n, int32_t chosen_op, uint16_t* op_idc,
                                    av1g_sequence_header* seq, int32_t* have_seq, av1g_obu* obus, int32_t cap,
                                    int32_t* count);

/* The leading fields of a §5.9.2 uncompressed header (frame header OBU or
 * frame OBU payload) under sequence header sh: show_existing_frame and
 * frame_to_show_map_idx, or frame_type, show_frame, showable_frame and
 * error_resilient_mode.  Enough to know which frames a stream shows. */
typedef struct av1g_frame_prefix {
    int32_t show_existing_frame;
    int32_t frame_to_show_map_idx;
    int32_t frame_type;            /* 0 KEY, 1 INTER, 2 INTRA_ONLY, 3 SWITCH */
    int32_t show_frame;
    int32_t showable_frame;
    int32_t error_resilient_mode;
} av1g_frame_prefix;
av1g_status av1g_frame_header_prefix(const uint8_t* payload, size_t n, const av1g_sequence_header* sh,
                                     av1g_frame_prefix* out);

/* §5.9 uncompressed header (parse_frame_header_with_refs,
 * src/frame_header.rs:726; the parameter blocks of
 * src/uncompressed_header_tail.rs and src/tile_info.rs).  The §7.20
 * reference state the header reads (RefInfo) is caller-owned: initialise it
 * with av1g_ref_state_init, parse each frame header against it and apply
 * av1g_ref_state_update once the frame is decoded (or at once for a shown
 * existing frame). */
typedef struct av1g_ref_state {
    int32_t valid[8];
    int32_t frame_id[8];
    int32_t frame_type[8];
    int32_t order_hint[8];
    int32_t saved_order_hints[8][8];
    int32_t upscaled_width[8], frame_width[8], frame_height[8], render_width[8], render_height[8];
    int32_t mi_cols[8], mi_rows[8];
    int32_t gm_params[8][8][6];       /* [slot][ref LAST..ALTREF at 1..7][i] */
    int8_t lf_ref_deltas[8][8];
    int8_t lf_mode_deltas[8][2];
    uint8_t seg_feature_enabled[8][8][8];
    int16_t seg_feature_data[8][8][8];
    av1g_film_grain film_grain[8];
} av1g_ref_state;

/* Everything a frame header fixes, flattened.  pf is the post-filter header
 * the chain kernels take (sizes, format, loop filter, segmentation loop-filter
 * features, CDEF, loop restoration, resolved film grain), filled from the
 * bitstream; the rest are the §5.9 syntax elements and derived values the
 * reconstruction needs. */
typedef struct av1g_parsed_frame_header {
    av1g_frame_header pf;
    int32_t show_existing_frame, frame_to_show_map_idx, frame_type, show_frame, showable_frame;
    int32_t error_resilient_mode, disable_cdf_update, allow_screen_content_tools, force_integer_mv;
    int32_t current_frame_id, frame_size_override_flag, order_hint, primary_ref_frame, refresh_frame_flags;
    int32_t frame_refs_short_signaling, ref_frame_idx[7];
    int32_t allow_high_precision_mv, interpolation_filter, is_motion_mode_switchable, use_ref_frame_mvs;
    int32_t order_hints[8];                   /* OrderHints[LAST_FRAME + i] at [1 + i] */
    int32_t render_width, render_height, superres_denom, disable_frame_end_update_cdf;
    int32_t tile_cols, tile_rows, tile_cols_log2, tile_rows_log2, context_update_tile_id, tile_size_bytes;
    int32_t mi_col_starts[65], mi_row_starts[65];
    int32_t base_q_idx, delta_q_y_dc, delta_q_u_dc, delta_q_u_ac, delta_q_v_dc, delta_q_v_ac;
    int32_t using_qmatrix, qm_y, qm_u, qm_v;
    int32_t segmentation_enabled, segmentation_update_map, segmentation_temporal_update;
    int32_t segmentation_update_data;
    uint8_t seg_feature_enabled[8][8];
    int16_t seg_feature_data[8][8];
    int32_t delta_q_present, delta_q_res, delta_lf_present, delta_lf_res;
    int32_t lossless[8], all_lossless;
    int32_t lr_unit_shift, lr_uv_shift;
    int32_t tx_mode, reference_select, skip_mode_present, skip_mode_frame[2];
    int32_t allow_warped_motion, reduced_tx_set;
    int32_t gm_type[8];
    int32_t gm_params[8][6];
    int32_t update_grain, film_grain_params_ref_idx;
    int32_t temporal_id, spatial_id;          /* of the OBU that carried it (input) */
    uint32_t header_bits;                     /* bits the uncompressed header took */
} av1g_parsed_frame_header;

#define AV1G_FE_FRAME_HEADER_INVALID 20   /* a header the reference rejects (invalid syntax or
                                             state it does not handle)                        */
void av1g_ref_state_init(av1g_ref_state* st);
/* temporal_id / spatial_id: the carrying OBU's extension ids (0 without). */
av1g_status av1g_parse_frame_header(const uint8_t* payload, size_t n, const av1g_sequence_header* sh,
                                    const av1g_ref_state* st, int32_t temporal_id, int32_t spatial_id,
                                    av1g_parsed_frame_header* out);
/* §7.20 reference_frame_update of the header state (and §7.21 for a shown
 * existing key frame). */
av1g_status av1g_ref_state_update(av1g_ref_state* st, const av1g_parsed_frame_header* fh);

/* §5.11.1 tile group: the tile range and each tile's bytes in the payload
 * (a tile group OBU, or the rest of a frame OBU after its byte-aligned
 * header). */
typedef struct av1g_tile_span {
    int32_t tile_num;
    int32_t pad;
    uint64_t offset, size;
} av1g_tile_span;
av1g_status av1g_parse_tile_group(const uint8_t* payload, size_t n, const av1g_parsed_frame_header* fh,
                                  int32_t* tg_start, int32_t* tg_end, av1g_tile_span* tiles, int32_t cap);

/* §8.2 symbol decoder (SymbolDecoder, src/symbol_decoder.rs), the first
 * piece of the host parse layer: the arithmetic decoder the tile walker reads
 * every symbol with.  The state is caller-owned and plain; `data` must stay
 * valid while it is in use.  A CDF of an n-symbol alphabet is n + 1 uint16
 * values: the n cumulative values (the last 32768) and the adaptation
 * counter. */
typedef struct av1g_symbol_decoder {
    const uint8_t* data;
    uint64_t size;               /* sz: the tile's byte count                 */
    uint64_t pos;                /* bits consumed from data                   */
    int64_t max_bits;            /* SymbolMaxBits                             */
    uint32_t value;              /* SymbolValue                               */
    uint32_t range;              /* SymbolRange                               */
    int32_t disable_cdf_update;
    int32_t pad;
} av1g_symbol_decoder;
#define AV1G_FE_SYMBOL_STATE_INVARIANT 18 /* Error::SymbolStateInvariantBroken                */
#define AV1G_FE_SYMBOL_EXIT_UNDERFLOW 19  /* Error::SymbolExitUnderflow                       */
/* init_symbol(sz) (§8.2.2, symbol_decoder.rs init_symbol). */
av1g_status av1g_symbol_init(av1g_symbol_decoder* d, const uint8_t* data, size_t sz, int32_t disable_cdf_update);
/* read_symbol (§8.2.6) with the §8.3 CDF update unless disabled. */
av1g_status av1g_symbol_read(av1g_symbol_decoder* d, uint16_t* cdf, int32_t n, uint32_t* symbol);
av1g_status av1g_symbol_read_bool(av1g_symbol_decoder* d, uint32_t* bit);
av1g_status av1g_symbol_read_literal(av1g_symbol_decoder* d, int32_t n, uint32_t* value);
av1g_status av1g_symbol_read_ns(av1g_symbol_decoder* d, uint32_t n, uint32_t* value);
/* decode_signed_subexp_with_ref_bool (low, high, k, r) (§5.9.26-§5.9.28 with
 * bools from the symbol decoder). */
av1g_status av1g_symbol_read_signed_subexp(av1g_symbol_decoder* d, int64_t low, int64_t high, uint32_t k, int64_t r,
                                           int64_t* value);
/* exit_symbol (§8.2.4): the trailing-bit position and the padding end. */
av1g_status av1g_symbol_exit(av1g_symbol_decoder* d, uint64_t* trailing_bit_position, uint64_t* padding_end);
/* The §8.3 CDF adaptation after decoding `symbol` of an n-symbol CDF. */
void av1g_update_cdf(uint16_t* cdf, uint32_t symbol, int32_t n);

/* §5.12 tile list OBU (TileListObu / TileListEntry, src/tile_list.rs): the
 * output size in tiles and, per entry, the anchor and tile it names and
 * where its coded tile data lies in the payload. */
typedef struct av1g_tile_list_header {
    int32_t output_frame_width_in_tiles_minus_1;
    int32_t output_frame_height_in_tiles_minus_1;
    int32_t tile_count_minus_1;
    int32_t pad;
} av1g_tile_list_header;
typedef struct av1g_tile_list_obu_entry {
    int32_t anchor_frame_idx;
    int32_t anchor_tile_row;
    int32_t anchor_tile_col;
    int32_t pad;
    uint64_t data_offset;
    uint64_t data_size;
} av1g_tile_list_obu_entry;
#define AV1G_FE_TILE_LIST_INVALID 17      /* Error::TileListInvalid                            */
/* parse_tile_list_obu (tile_list.rs:102): at most cap entries are written;
 * the conformance bounds tile_count_minus_1 <= 511 and anchor_frame_idx <=
 * 127 are enforced and the payload must end with the last entry. */
av1g_status av1g_parse_tile_list(const uint8_t* payload, size_t n, av1g_tile_list_header* hdr,
                                 av1g_tile_list_obu_entry* entries, int32_t cap);
/* write_tile_list_obu (tile_list.rs:156): 1..512 entries, anchor_frame_idx <=
 * 127, 1..65536 bytes of tile data each (entries[i].data_offset indexes
 * `data`).  out == NULL only measures. */
av1g_status av1g_write_tile_list(const av1g_tile_list_header* hdr, const av1g_tile_list_obu_entry* entries,
                                 int32_t count, const uint8_t* data, uint8_t* out, size_t cap, uint64_t* out_len);

/* ---------------------------------------------------------------------
 * Stream decoder: the registry Decoder API over the whole path
 * ------------------------------------------------------------------- */

/* The reference's oxideav_core::Decoder implementation (Av1Decoder,
 * src/registry.rs:103-195) over its decode session (SpecDecodeSession,
 * src/decoder/frame_driver.rs:1295-1400): packets in, shown frames out.
 * Host side per frame: the §7.5 OBU walk, the §5.9 header, the §5.11 tile
 * walk (symbols, CDF contexts, motion vector prediction) producing the
 * av1g_frame_desc of the frame; the GPU engine then reconstructs, filters and
 * stores it.  engine == NULL gives a parse-only decoder that records every
 * frame's descriptor (av1g_decoder_parsed_frame) and produces no pixels.
 * operating_point: the §6.7.5 choice (0 = the preferred point). */
typedef struct av1g_decoder av1g_decoder;
av1g_status av1g_decoder_create(av1g_engine* engine, int32_t operating_point, av1g_decoder** out);
/* Waits (bounded) for the frames in flight and frees the decoder. */
void av1g_decoder_destroy(av1g_decoder* d);
/* send_packet (registry.rs:132-166): a whole IVF file (DKIF magic) is split
 * into its frame records, anything else is one §7.5 temporal unit; pts is
 * carried to the frame (IVF records carry their own).  A malformed packet
 * returns AV1G_EINVAL (av1g_last_error names the cause); the reference maps
 * its typed errors to CoreError::invalid the same way. */
av1g_status av1g_decoder_send_packet(av1g_decoder* d, const uint8_t* data, size_t n, int64_t pts);
/* receive_frame (registry.rs:168-179): AV1G_OK with the next shown frame in
 * output order (cropped planes, tight strides, u8 or little-endian u16 —
 * the SpecFrame layout), valid until the next call; AV1G_ENOTREADY when no
 * frame is queued (NeedMore); AV1G_EOF after av1g_decoder_flush once the
 * queue is empty.  Waits (bounded) for the frame's GPU work. */
av1g_status av1g_decoder_receive_frame(av1g_decoder* d, av1g_frame_out* out, int64_t* pts);
/* flush (registry.rs:181-184): no more packets; receive drains, then EOF. */
av1g_status av1g_decoder_flush(av1g_decoder* d);
/* reset (registry.rs:186-195): drops queued frames and the reference state
 * (reset_references, frame_driver.rs:1401), keeps the sequence header. */
av1g_status av1g_decoder_reset(av1g_decoder* d);
/* Parse-only decoders: the number of frames parsed so far and frame i's
 * descriptor (pointers valid while the decoder lives) with its header. */
int32_t av1g_decoder_parsed_count(const av1g_decoder* d);
av1g_status av1g_decoder_parsed_frame(const av1g_decoder* d, int32_t i, av1g_frame_desc* out,
                                      av1g_parsed_frame_header* fh);
/* The current sequence header. */
av1g_status av1g_decoder_sequence(const av1g_decoder* d, av1g_sequence_header* out);
/* Host milliseconds spent in send_packet (framing, headers, tile walk). */
double av1g_decoder_host_ms(const av1g_decoder* d);
/* Frames so far whose tile data did not end at its §8.2.4 trailing bit
 * after the walk (a stream the walk read differently from its encoder). */
int32_t av1g_decoder_frames_out_of_sync(const av1g_decoder* d);

/* ---------------------------------------------------------------------
 * Library
 * ------------------------------------------------------------------- */

/* ABI version of the loaded library (AV1G_ABI_VERSION at build time). */
int32_t av1g_abi_version(void);

/* sizeof() of a public struct by name ("av1g_frame_header", ...), or -1.
 * Lets bindings in other languages verify their struct mirrors. */
int32_t av1g_struct_size(const char* name);

/* Human-readable text of the last error on this thread. */
const char* av1g_last_error(void);

/* Number of units an LR plane of `plane_size` samples holds at
 * `unit_size` (§5.9.20 count_units_in_frame, loop_restoration.rs:888). */
int32_t av1g_lr_units_in_frame(int32_t unit_size, int32_t plane_size);

/* ---------------------------------------------------------------------
 * Stage entry points on device-resident frames.  Each runs one stage for
 * `n` jobs as one launch (or one launch per plane group) on `stream`.
 * ------------------------------------------------------------------- */

/* §7.14 deblock: recon -> deblocked.  Replaces loop_filter_frame
 * (src/loop_filter.rs:271) as driven by loop_filter_frame_from_grid
 * (src/cdf.rs:20449). */
av1g_status av1g_run_deblock(const av1g_frame_job* jobs, int32_t n, void* stream);

/* §7.15 CDEF: deblocked -> cdef.  Replaces cdef_frame (src/cdef.rs:180) as
 * driven by cdef_frame_from_idx (src/cdf.rs:20300). */
av1g_status av1g_run_cdef(const av1g_frame_job* jobs, int32_t n, void* stream);

/* §7.16 superres: deblocked -> up_deblocked and cdef -> up_cdef.
 * Replaces upscale_frame (src/superres.rs:282) as called at
 * frame_driver.rs:906-966. */
av1g_status av1g_run_superres(const av1g_frame_job* jobs, int32_t n, void* stream);

/* §7.17 loop restoration: (up_)cdef + (up_)deblocked -> lr.  Replaces
 * loop_restoration_frame (src/loop_restoration.rs:268) as driven by
 * loop_restore_frame_from_grid (src/cdf.rs:20624). */
av1g_status av1g_run_lr(const av1g_frame_job* jobs, int32_t n, void* stream);

/* §7.18.3 film grain: lr (cropped) -> out.  Replaces film_grain_synthesis
 * (src/film_grain.rs:848) as called at frame_driver.rs:1060-1096. */
av1g_status av1g_run_film_grain(const av1g_frame_job* jobs, int32_t n, void* stream);

/* The whole §7.4 chain of frame_driver.rs:830-1096 for `n` jobs:
 * deblock, CDEF, superres, loop restoration, film grain, with the
 * reference's gating.  mode = AV1G_MODE_BATCHED or AV1G_MODE_PER_FRAME.
 * *launches (optional) receives the number of stage kernels launched; the
 * frame records of a batch up to 32 KB (about 28 frames) travel as the
 * parameters of one small store kernel per 16 KB (no copy engine), larger
 * ones by a copy. */
av1g_status av1g_run_postfilter(const av1g_frame_job* jobs, int32_t n, int32_t mode,
                                void* stream, int32_t* launches);

/* Launch-shape autotuner for the post-filter stages.  Each stage is a
 * grid-stride launch over a flattened tile list: its grid size (resident CTAs
 * per SM) is a free parameter, and so is superres's tile width (256, 512 or
 * 1024 output samples of a row).  av1g_autotune_postfilter runs the whole
 * chain on the jobs once per candidate shape of each stage, in chain order
 * (the stages are idempotent on their inputs), times three launches per
 * candidate with CUDA events, and keeps the fastest for that stage and the
 * batch's sample width (8-bit or high bit depth) for every later call in
 * this process; it synchronizes `stream`.  cache_path (optional) receives
 * the table as text ("stage hbd ctas_per_sm tile" per line);
 * av1g_autotune_load reads such a file (av1g_engine_create does when
 * av1g_config.autotune_cache names one); av1g_autotune_get reads one entry
 * (stage 0 deblock, 1 CDEF, 2 superres, 3 LR, 4 film grain). */
av1g_status av1g_autotune_postfilter(const av1g_frame_job* jobs, int32_t n, void* stream, const char* cache_path);
av1g_status av1g_autotune_load(const char* cache_path);
av1g_status av1g_autotune_get(int32_t stage, int32_t hbd, int32_t* ctas_per_sm, int32_t* tile);

/* The §7.4 chain for a fixed set of jobs, captured once as a CUDA graph.
 * The frame records, tile prefixes and stage scratch live in one device
 * allocation the graph owns, so each av1g_chain_graph_launch is a single
 * graph launch on `stream` that replays every stage launch — no record upload
 * and no allocation per call (frame_driver.rs:830-1096 for the same frames
 * step after step, e.g. a serving slot set or a benchmark batch).  The jobs'
 * plane pointers, sizes and headers are baked in; the caller may rewrite the
 * planes' samples between launches.  stage_mask: bit s runs stage s
 * (0 deblock, 1 CDEF, 2 superres, 3 loop restoration, 4 film grain) with the
 * reference's gating; mode: AV1G_MODE_BATCHED (one launch per stage) or
 * AV1G_MODE_PER_FRAME (a launch per stage per frame, all in the graph).
 * create runs the chain once, uncaptured, before capturing it. */
typedef struct av1g_chain_graph av1g_chain_graph;
av1g_status av1g_chain_graph_create(const av1g_frame_job* jobs, int32_t n, int32_t stage_mask, int32_t mode,
                                    void* stream, av1g_chain_graph** out);
av1g_status av1g_chain_graph_launch(av1g_chain_graph* g, void* stream);
/* Kernel launches one replay performs. */
int32_t av1g_chain_graph_launches(const av1g_chain_graph* g);
/* Frees the graph; its device memory is released once the device is idle
 * (cudaFree synchronizes), so launches still in flight complete first. */
av1g_status av1g_chain_graph_destroy(av1g_chain_graph* g);

/* Film grain (as av1g_run_film_grain) without any device allocation.  No
 * counterpart in the reference: it exists for callers that may not allocate
 * device memory on the per-frame path, such as a host application that
 * reserves the whole device-memory budget at start-up and forbids its
 * plug-ins to allocate while frames flow (an allocation there can stall on
 * the allocator or fail once the pool is full).
 * The frame records and grain scratch live in one static device array of
 * AV1G_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit.  The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture.  The address is kept per device ordinal for the
 * life of the process, so calls must run in the device's primary context
 * (the CUDA runtime's default) and not after cudaDeviceReset.  At most
 * AV1G_NOALLOC_MAX_FRAMES jobs per call,
 * and the batch's scratch must fit the array; larger requests return
 * AV1G_EINVAL with a message naming the limit.  All calls on a device share
 * the array: calls that overlap on the GPU race on it. */
#define AV1G_NOALLOC_MAX_FRAMES 16
#define AV1G_NOALLOC_SCRATCH_BYTES (2 * 1024 * 1024)
av1g_status av1g_run_film_grain_noalloc(const av1g_frame_job* jobs, int32_t n, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* AV1G_H */
