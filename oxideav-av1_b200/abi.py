"""ctypes mirror of ``include/av1g.h`` and the loader of the CUDA library.

The structures below are field-for-field copies of the C structs; the loader
checks their sizes against ``av1g_struct_size`` exported by the library so a
drift between the header and this file fails at load time rather than
corrupting a launch.  There is no CPU fallback: if the library is missing or
fails to load, ``load()`` raises.
"""
import ctypes as C
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "liboxav1_b200.so"

AV1G_OK = 0
AV1G_EINVAL = 1
AV1G_ENOMEM_BUDGET = 2
AV1G_EBUSY = 3
AV1G_TIMEOUT = 4
AV1G_EDEVICE = 5
AV1G_EPARITY = 6
AV1G_ENOTSUP = 7
AV1G_ENOTREADY = 8
AV1G_EOF = 9
STATUS_NAMES = {0: "OK", 1: "EINVAL", 2: "ENOMEM_BUDGET", 3: "EBUSY", 4: "TIMEOUT", 5: "EDEVICE", 9: "EOF",
                6: "EPARITY", 7: "ENOTSUP", 8: "ENOTREADY"}

MODE_BATCHED = 0
MODE_PER_FRAME = 1


class FilmGrain(C.Structure):
    _fields_ = [
        ("apply_grain", C.c_uint8), ("chroma_scaling_from_luma", C.c_uint8), ("grain_seed", C.c_uint16),
        ("num_y_points", C.c_uint8), ("point_y_value", C.c_uint8 * 14), ("point_y_scaling", C.c_uint8 * 14),
        ("num_cb_points", C.c_uint8), ("point_cb_value", C.c_uint8 * 10), ("point_cb_scaling", C.c_uint8 * 10),
        ("num_cr_points", C.c_uint8), ("point_cr_value", C.c_uint8 * 10), ("point_cr_scaling", C.c_uint8 * 10),
        ("grain_scaling", C.c_uint8), ("ar_coeff_lag", C.c_uint8),
        ("ar_coeffs_y_plus_128", C.c_uint8 * 24), ("ar_coeffs_cb_plus_128", C.c_uint8 * 25),
        ("ar_coeffs_cr_plus_128", C.c_uint8 * 25), ("ar_coeff_shift", C.c_uint8), ("grain_scale_shift", C.c_uint8),
        ("cb_mult", C.c_uint8), ("cb_luma_mult", C.c_uint8), ("cr_mult", C.c_uint8), ("cr_luma_mult", C.c_uint8),
        ("overlap_flag", C.c_uint8), ("clip_to_restricted_range", C.c_uint8),
        ("cb_offset", C.c_uint16), ("cr_offset", C.c_uint16),
    ]


class FrameHeader(C.Structure):
    _fields_ = [
        ("frame_width", C.c_int32), ("frame_height", C.c_int32), ("upscaled_width", C.c_int32),
        ("mi_rows", C.c_int32), ("mi_cols", C.c_int32),
        ("bit_depth", C.c_uint8), ("subsampling_x", C.c_uint8), ("subsampling_y", C.c_uint8),
        ("num_planes", C.c_uint8), ("matrix_coefficients", C.c_uint8), ("use_superres", C.c_uint8),
        ("coded_lossless", C.c_uint8), ("allow_intrabc", C.c_uint8), ("enable_cdef", C.c_uint8),
        ("lf_level", C.c_uint8 * 4), ("lf_sharpness", C.c_uint8), ("lf_delta_enabled", C.c_uint8),
        ("delta_lf_multi", C.c_uint8), ("lf_ref_deltas", C.c_int8 * 8), ("lf_mode_deltas", C.c_int8 * 2),
        ("seg_lf_active", (C.c_uint8 * 4) * 8), ("seg_lf_data", (C.c_int16 * 4) * 8),
        ("cdef_short_circuited", C.c_uint8), ("cdef_damping", C.c_uint8), ("cdef_bits", C.c_uint8),
        ("cdef_y_pri", C.c_uint8 * 8), ("cdef_y_sec", C.c_uint8 * 8),
        ("cdef_uv_pri", C.c_uint8 * 8), ("cdef_uv_sec", C.c_uint8 * 8),
        ("uses_lr", C.c_uint8), ("lr_type", C.c_uint8 * 3), ("lr_unit_size", C.c_int32 * 3),
        ("film_grain", FilmGrain),
    ]


class LrUnit(C.Structure):
    _fields_ = [("type", C.c_uint8), ("sgr_set", C.c_uint8), ("wiener", (C.c_int8 * 3) * 2),
                ("sgr_xqd", C.c_int16 * 2)]


class MiGrid(C.Structure):
    _fields_ = [
        ("mi_size", C.c_void_p), ("skip", C.c_void_p), ("is_inter", C.c_void_p), ("ref_frame0", C.c_void_p),
        ("y_mode", C.c_void_p), ("segment_id", C.c_void_p), ("delta_lf", C.c_void_p), ("tx_size", C.c_void_p),
        ("inter_tx_size", C.c_void_p),
    ]


class Plane(C.Structure):
    _fields_ = [("data", C.c_void_p), ("stride", C.c_int32), ("width", C.c_int32), ("height", C.c_int32)]


class FrameJob(C.Structure):
    _fields_ = [
        ("hdr", C.POINTER(FrameHeader)), ("grid", MiGrid), ("cdef_idx", C.c_void_p),
        ("lr_units", C.c_void_p * 3),
        ("recon", Plane * 3), ("deblocked", Plane * 3), ("cdef", Plane * 3), ("up_deblocked", Plane * 3),
        ("up_cdef", Plane * 3), ("lr", Plane * 3), ("out", Plane * 3),
    ]


class QuantParams(C.Structure):
    _fields_ = [
        ("base_q_idx", C.c_uint8), ("delta_q_y_dc", C.c_int8), ("delta_q_u_dc", C.c_int8),
        ("delta_q_u_ac", C.c_int8), ("delta_q_v_dc", C.c_int8), ("delta_q_v_ac", C.c_int8),
        ("using_qmatrix", C.c_uint8), ("delta_q_present", C.c_uint8), ("segmentation_enabled", C.c_uint8),
        ("seg_alt_q_active", C.c_uint8 * 8), ("pad", C.c_uint8), ("seg_alt_q_data", C.c_int16 * 8),
        ("seg_qm_level", (C.c_uint8 * 8) * 3), ("lossless", C.c_uint8 * 8),
    ]


class Tu(C.Structure):
    _fields_ = [("x", C.c_uint16), ("y", C.c_uint16), ("plane", C.c_uint8), ("tx_size", C.c_uint8),
                ("tx_type", C.c_uint8), ("segment_id", C.c_uint8), ("current_q_index", C.c_uint8),
                ("pad", C.c_uint8 * 3), ("coeff_offset", C.c_uint32)]


class ReconJob(C.Structure):
    _fields_ = [("hdr", C.POINTER(FrameHeader)), ("quant", C.POINTER(QuantParams)), ("tus", C.c_void_p),
                ("num_tus", C.c_int32), ("coeffs", C.c_void_p), ("planes", Plane * 3)]


class IntraTu(C.Structure):
    _fields_ = [("x", C.c_uint16), ("y", C.c_uint16), ("plane", C.c_uint8), ("tx_size", C.c_uint8),
                ("mode", C.c_uint8), ("flags", C.c_uint8), ("angle_delta", C.c_int8), ("cfl_alpha", C.c_int8),
                ("filter_intra_mode", C.c_uint8), ("pad", C.c_uint8), ("max_luma_w", C.c_uint16),
                ("max_luma_h", C.c_uint16), ("res", Tu), ("mv", C.c_int16 * 2), ("palette_map", C.c_uint32),
                ("palette_stride", C.c_uint16), ("palette_size", C.c_uint8), ("pad2", C.c_uint8),
                ("palette_colors", C.c_uint16 * 8), ("interintra", C.c_uint8), ("interintra_mode", C.c_uint8),
                ("wedge_index", C.c_uint8), ("mi_size", C.c_uint8)]


class IntraJob(C.Structure):
    _fields_ = [("hdr", C.POINTER(FrameHeader)), ("quant", C.POINTER(QuantParams)), ("tus", C.c_void_p),
                ("num_tus", C.c_int32), ("sb_size", C.c_int32), ("coeffs", C.c_void_p), ("planes", Plane * 3),
                ("palette_maps", C.c_void_p), ("palette_map_bytes", C.c_int64), ("interintra_in", Plane * 3)]


class IntraPlanStats(C.Structure):
    _fields_ = [("superblocks", C.c_int32), ("tus", C.c_int32), ("waits", C.c_int32), ("depth", C.c_int32),
                ("width", C.c_int32), ("pad", C.c_int32)]


class RefFrame(C.Structure):
    _fields_ = [("planes", Plane * 3), ("upscaled_width", C.c_int32), ("frame_height", C.c_int32)]


class WarpCtx(C.Structure):
    _fields_ = [("gm_params", (C.c_int32 * 6) * 2), ("local_warp_params", C.c_int32 * 6),
                ("y_mode", C.c_uint8 * 2), ("gm_type", C.c_uint8 * 2), ("local_valid", C.c_uint8),
                ("ref_is_scaled", C.c_uint8 * 2), ("force_integer_mv", C.c_uint8)]


class ObmcNeighbour(C.Structure):
    _fields_ = [("mv", C.c_int16 * 2), ("axis_pos4", C.c_uint16), ("ref", C.c_uint8), ("step4", C.c_uint8),
                ("filter_x", C.c_uint8), ("filter_y", C.c_uint8), ("pad", C.c_uint8 * 2)]


class InterPred(C.Structure):
    _fields_ = [("x", C.c_uint16), ("y", C.c_uint16), ("w", C.c_uint16), ("h", C.c_uint16),
                ("plane", C.c_uint8), ("kind", C.c_uint8), ("motion_mode", C.c_uint8), ("filter_x", C.c_uint8),
                ("filter_y", C.c_uint8), ("ref", C.c_uint8 * 2), ("compound_type", C.c_uint8),
                ("mv", (C.c_int16 * 2) * 2), ("mi_size", C.c_uint8), ("wedge_index", C.c_uint8),
                ("wedge_sign", C.c_uint8), ("mask_type", C.c_uint8), ("interintra_mode", C.c_uint8),
                ("wedge_interintra", C.c_uint8), ("fwd_weight", C.c_uint8), ("bck_weight", C.c_uint8),
                ("warp", C.c_int32), ("obmc_first", C.c_uint32), ("obmc_above", C.c_uint8),
                ("obmc_left", C.c_uint8), ("avail_u", C.c_uint8), ("avail_l", C.c_uint8),
                ("plane_residual_ge_8x8", C.c_uint8), ("mi_width_log2", C.c_uint8),
                ("mi_height_log2", C.c_uint8), ("pad", C.c_uint8), ("mi_row", C.c_uint16), ("mi_col", C.c_uint16)]


class WarpSample(C.Structure):
    _fields_ = [("sy", C.c_int32), ("sx", C.c_int32), ("dy", C.c_int32), ("dx", C.c_int32)]


class InterJob(C.Structure):
    _fields_ = [("hdr", C.POINTER(FrameHeader)), ("refs", C.POINTER(RefFrame)), ("preds", C.c_void_p),
                ("num_preds", C.c_int32), ("neighbours", C.c_void_p), ("num_neighbours", C.c_int32),
                ("warps", C.c_void_p), ("num_warps", C.c_int32), ("planes", Plane * 3),
                ("interintra_out", Plane * 3)]


INTER_SINGLE, INTER_COMPOUND, INTER_INTRA = 0, 1, 2


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("max_batch", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("max_inflight_steps", C.c_int32), ("lanes", C.c_int32), ("autotune_cache", C.c_char_p),
                ("max_step_samples", C.c_int64)]


class SeqInfo(C.Structure):
    _fields_ = [("max_width", C.c_int32), ("max_height", C.c_int32), ("bit_depth", C.c_uint8),
                ("subsampling_x", C.c_uint8), ("subsampling_y", C.c_uint8), ("num_planes", C.c_uint8),
                ("sb_size", C.c_int32)]


class FrameDesc(C.Structure):
    _fields_ = [("hdr", C.POINTER(FrameHeader)), ("quant", C.POINTER(QuantParams)), ("grid", MiGrid),
                ("cdef_idx", C.c_void_p), ("lr_units", C.c_void_p * 3), ("inter_preds", C.c_void_p),
                ("num_inter_preds", C.c_int32), ("neighbours", C.c_void_p), ("num_neighbours", C.c_int32),
                ("warps", C.c_void_p), ("num_warps", C.c_int32), ("inter_tus", C.c_void_p),
                ("num_inter_tus", C.c_int32), ("intra_tus", C.c_void_p), ("num_intra_tus", C.c_int32),
                ("palette_maps", C.c_void_p), ("palette_map_bytes", C.c_int64), ("coeffs", C.c_void_p),
                ("num_coeffs", C.c_int64), ("ref_frame_idx", C.c_uint8 * 7), ("refresh_frame_flags", C.c_uint8),
                ("show_frame", C.c_uint8), ("show_existing_frame", C.c_uint8), ("frame_to_show_map_idx", C.c_uint8),
                ("pad", C.c_uint8)]


class FrameOut(C.Structure):
    _fields_ = [("planes", Plane * 3), ("num_planes", C.c_int32), ("bit_depth", C.c_int32), ("shown", C.c_int32),
                ("pad", C.c_int32), ("latency_ms", C.c_double)]


class EngineStats(C.Structure):
    _fields_ = [("frames_done", C.c_int64), ("steps_done", C.c_int64), ("bytes_reserved", C.c_int64),
                ("bytes_in_flight", C.c_int64), ("budget", C.c_int64), ("streams_open", C.c_int32),
                ("pad", C.c_int32), ("host_ms", C.c_double), ("device_ms", C.c_double),
                ("host_stage_ms", C.c_double * 6)]

class MfStoreJob(C.Structure):
    _fields_ = [("mi_rows", C.c_int32), ("mi_cols", C.c_int32), ("is_inter_frame", C.c_int32),
                ("order_hint", C.c_int32), ("hint_bits", C.c_int32), ("ref_order_hint", C.c_int32 * 7),
                ("ref_frames", C.c_void_p), ("mvs", C.c_void_p), ("mf_ref_frames", C.c_void_p),
                ("mf_mvs", C.c_void_p)]


class MfSlot(C.Structure):
    _fields_ = [("mf_mvs", C.c_void_p), ("mf_ref_frames", C.c_void_p), ("saved_order_hints", C.c_int32 * 8),
                ("mi_rows", C.c_int32), ("mi_cols", C.c_int32), ("frame_is_intra", C.c_int32), ("pad", C.c_int32)]


class MfProjectJob(C.Structure):
    _fields_ = [("slots", MfSlot * 8), ("ref_frame_idx", C.c_int32 * 7), ("pad", C.c_int32),
                ("order_hints", C.c_int32 * 8), ("order_hint", C.c_int32), ("hint_bits", C.c_int32),
                ("mi_rows", C.c_int32), ("mi_cols", C.c_int32), ("out", C.c_void_p)]


MFMV_INVALID = -32768


class Obu(C.Structure):
    _fields_ = [("obu_type", C.c_int32), ("extension_flag", C.c_int32), ("has_size_field", C.c_int32),
                ("temporal_id", C.c_int32), ("spatial_id", C.c_int32), ("header_len", C.c_int32),
                ("payload_offset", C.c_uint64), ("payload_len", C.c_uint64)]


class IvfHeader(C.Structure):
    _fields_ = [("version", C.c_uint16), ("header_length", C.c_uint16), ("fourcc", C.c_uint8 * 4),
                ("width", C.c_uint16), ("height", C.c_uint16), ("fps_num", C.c_uint32), ("fps_den", C.c_uint32),
                ("frame_count", C.c_uint32)]


class IvfFrame(C.Structure):
    _fields_ = [("pts", C.c_uint64), ("offset", C.c_uint64), ("size", C.c_uint64)]


class OperatingPoint(C.Structure):
    _fields_ = [("idc", C.c_uint16), ("seq_level_idx", C.c_uint8), ("seq_tier", C.c_uint8),
                ("decoder_model_present", C.c_uint8), ("initial_display_delay_present", C.c_uint8),
                ("initial_display_delay_minus_1", C.c_uint8), ("low_delay_mode_flag", C.c_uint8),
                ("decoder_buffer_delay", C.c_uint64), ("encoder_buffer_delay", C.c_uint64)]


_U8 = C.c_uint8


class SequenceHeader(C.Structure):
    _fields_ = [(n, _U8) for n in ("seq_profile", "still_picture", "reduced_still_picture_header",
                                   "timing_info_present_flag", "equal_picture_interval",
                                   "decoder_model_info_present_flag", "initial_display_delay_present_flag",
                                   "operating_points_cnt_minus_1")] + \
              [(n, C.c_uint32) for n in ("num_units_in_display_tick", "time_scale",
                                         "num_ticks_per_picture_minus_1")] + \
              [(n, _U8) for n in ("buffer_delay_length_minus_1", "buffer_removal_time_length_minus_1",
                                  "frame_presentation_time_length_minus_1", "pad0")] + \
              [("num_units_in_decoding_tick", C.c_uint32), ("operating_points", OperatingPoint * 32)] + \
              [(n, _U8) for n in ("frame_width_bits_minus_1", "frame_height_bits_minus_1",
                                  "frame_id_numbers_present_flag", "delta_frame_id_length_minus_2",
                                  "additional_frame_id_length_minus_1", "use_128x128_superblock",
                                  "enable_filter_intra", "enable_intra_edge_filter")] + \
              [("max_frame_width_minus_1", C.c_uint32), ("max_frame_height_minus_1", C.c_uint32)] + \
              [(n, _U8) for n in ("enable_interintra_compound", "enable_masked_compound", "enable_warped_motion",
                                  "enable_dual_filter", "enable_order_hint", "enable_jnt_comp",
                                  "enable_ref_frame_mvs", "seq_force_screen_content_tools",
                                  "seq_force_integer_mv", "order_hint_bits", "enable_superres", "enable_cdef",
                                  "enable_restoration", "high_bitdepth", "twelve_bit", "bit_depth", "mono_chrome",
                                  "num_planes", "color_description_present_flag", "color_primaries",
                                  "transfer_characteristics", "matrix_coefficients", "color_range",
                                  "subsampling_x", "subsampling_y", "chroma_sample_position",
                                  "separate_uv_delta_q", "film_grain_params_present")] + \
              [("pad1", _U8 * 3), ("bits_consumed", C.c_uint32)]


class FramePrefix(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("show_existing_frame", "frame_to_show_map_idx", "frame_type", "show_frame",
                                         "showable_frame", "error_resilient_mode")]


class TileListEntry(C.Structure):
    _fields_ = [("src", Plane * 3), ("x0", C.c_int32), ("y0", C.c_int32)]


class TileListJob(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("tile_width", "tile_height", "width_in_tiles", "height_in_tiles",
                                         "num_planes", "subsampling_x", "subsampling_y", "bit_depth", "num_entries",
                                         "pad")] + [("entries", C.POINTER(TileListEntry)), ("out", Plane * 3)]


class TileListHeader(C.Structure):
    _fields_ = [(n, C.c_int32) for n in ("output_frame_width_in_tiles_minus_1",
                                         "output_frame_height_in_tiles_minus_1", "tile_count_minus_1", "pad")]


class TileListObuEntry(C.Structure):
    _fields_ = [("anchor_frame_idx", C.c_int32), ("anchor_tile_row", C.c_int32), ("anchor_tile_col", C.c_int32),
                ("pad", C.c_int32), ("data_offset", C.c_uint64), ("data_size", C.c_uint64)]


FE_TILE_LIST_INVALID = 17
FE_SYMBOL_STATE_INVARIANT, FE_SYMBOL_EXIT_UNDERFLOW = 18, 19


_I32 = C.c_int32


class RefState(C.Structure):
    _fields_ = [(n, _I32 * 8) for n in ("valid", "frame_id", "frame_type", "order_hint")] + \
              [("saved_order_hints", (_I32 * 8) * 8)] + \
              [(n, _I32 * 8) for n in ("upscaled_width", "frame_width", "frame_height", "render_width",
                                       "render_height", "mi_cols", "mi_rows")] + \
              [("gm_params", ((_I32 * 6) * 8) * 8), ("lf_ref_deltas", (C.c_int8 * 8) * 8),
               ("lf_mode_deltas", (C.c_int8 * 2) * 8), ("seg_feature_enabled", ((C.c_uint8 * 8) * 8) * 8),
               ("seg_feature_data", ((C.c_int16 * 8) * 8) * 8), ("film_grain", FilmGrain * 8)]


class ParsedFrameHeader(C.Structure):
    _fields_ = [("pf", FrameHeader)] + \
              [(n, _I32) for n in ("show_existing_frame", "frame_to_show_map_idx", "frame_type", "show_frame",
                                   "showable_frame", "error_resilient_mode", "disable_cdf_update",
                                   "allow_screen_content_tools", "force_integer_mv", "current_frame_id",
                                   "frame_size_override_flag", "order_hint", "primary_ref_frame",
                                   "refresh_frame_flags", "frame_refs_short_signaling")] + \
              [("ref_frame_idx", _I32 * 7)] + \
              [(n, _I32) for n in ("allow_high_precision_mv", "interpolation_filter", "is_motion_mode_switchable",
                                   "use_ref_frame_mvs")] + \
              [("order_hints", _I32 * 8)] + \
              [(n, _I32) for n in ("render_width", "render_height", "superres_denom",
                                   "disable_frame_end_update_cdf", "tile_cols", "tile_rows", "tile_cols_log2",
                                   "tile_rows_log2", "context_update_tile_id", "tile_size_bytes")] + \
              [("mi_col_starts", _I32 * 65), ("mi_row_starts", _I32 * 65)] + \
              [(n, _I32) for n in ("base_q_idx", "delta_q_y_dc", "delta_q_u_dc", "delta_q_u_ac", "delta_q_v_dc",
                                   "delta_q_v_ac", "using_qmatrix", "qm_y", "qm_u", "qm_v", "segmentation_enabled",
                                   "segmentation_update_map", "segmentation_temporal_update",
                                   "segmentation_update_data")] + \
              [("seg_feature_enabled", (C.c_uint8 * 8) * 8), ("seg_feature_data", (C.c_int16 * 8) * 8)] + \
              [(n, _I32) for n in ("delta_q_present", "delta_q_res", "delta_lf_present", "delta_lf_res")] + \
              [("lossless", _I32 * 8)] + \
              [(n, _I32) for n in ("all_lossless", "lr_unit_shift", "lr_uv_shift", "tx_mode", "reference_select",
                                   "skip_mode_present")] + \
              [("skip_mode_frame", _I32 * 2), ("allow_warped_motion", _I32), ("reduced_tx_set", _I32),
               ("gm_type", _I32 * 8), ("gm_params", (_I32 * 6) * 8)] + \
              [(n, _I32) for n in ("update_grain", "film_grain_params_ref_idx", "temporal_id", "spatial_id")] + \
              [("header_bits", C.c_uint32)]


class TileSpan(C.Structure):
    _fields_ = [("tile_num", _I32), ("pad", _I32), ("offset", C.c_uint64), ("size", C.c_uint64)]


FE_FRAME_HEADER_INVALID = 20


class SymbolDecoder(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size", C.c_uint64), ("pos", C.c_uint64), ("max_bits", C.c_int64),
                ("value", C.c_uint32), ("range", C.c_uint32), ("disable_cdf_update", C.c_int32),
                ("pad", C.c_int32)]
FE_NONE, FE_UNEXPECTED_END, FE_FORBIDDEN_BIT_SET, FE_MISSING_SIZE_FIELD = 0, 1, 2, 3
FE_LEB128_OVERFLOW, FE_LEB128_TOO_LONG, FE_SIZE_OVERFLOW, FE_ANNEXB_INVALID = 4, 5, 6, 7
FE_IVF_BAD_MAGIC, FE_IVF_UNSUPPORTED_VERSION, FE_IVF_UNSUPPORTED_HEADER_LENGTH = 8, 9, 10
FE_RESERVED_PROFILE, FE_REDUCED_STILL_REQUIRES_STILL, FE_OPERATING_POINT_OUT_OF_RANGE = 11, 12, 13
FE_OUTPUT_TOO_SMALL, FE_UNSUPPORTED_OBU, FE_TEMPORAL_POINT_INFO_UNSUPPORTED = 14, 15, 16

INTRA_HAVE_ABOVE, INTRA_HAVE_LEFT, INTRA_HAVE_ABOVE_RIGHT, INTRA_HAVE_BELOW_LEFT = 1, 2, 4, 8
INTRA_EDGE_FILTER, INTRA_FILTER_TYPE, INTRA_RESIDUAL, INTRA_CFL = 16, 32, 64, 128
INTRA_MODE_PALETTE, INTRA_MODE_INTRABC, INTRA_MODE_NONE = 64, 65, 255

_STRUCTS = {"av1g_film_grain": FilmGrain, "av1g_frame_header": FrameHeader, "av1g_lr_unit": LrUnit,
            "av1g_mi_grid": MiGrid, "av1g_plane": Plane, "av1g_frame_job": FrameJob,
            "av1g_quant_params": QuantParams, "av1g_tu": Tu, "av1g_recon_job": ReconJob,
            "av1g_intra_tu": IntraTu, "av1g_intra_job": IntraJob, "av1g_ref_frame": RefFrame,
            "av1g_intra_plan_stats": IntraPlanStats,
            "av1g_warp_ctx": WarpCtx, "av1g_obmc_neighbour": ObmcNeighbour, "av1g_inter_pred": InterPred,
            "av1g_inter_job": InterJob, "av1g_warp_sample": WarpSample, "av1g_config": Config,
            "av1g_seq_info": SeqInfo, "av1g_frame_desc": FrameDesc, "av1g_frame_out": FrameOut,
            "av1g_engine_stats": EngineStats, "av1g_mf_store_job": MfStoreJob, "av1g_mf_slot": MfSlot,
            "av1g_mf_project_job": MfProjectJob, "av1g_obu": Obu, "av1g_ivf_header": IvfHeader,
            "av1g_ivf_frame": IvfFrame, "av1g_operating_point": OperatingPoint,
            "av1g_sequence_header": SequenceHeader, "av1g_frame_prefix": FramePrefix,
            "av1g_tile_list_entry": TileListEntry, "av1g_tile_list_job": TileListJob,
            "av1g_tile_list_header": TileListHeader, "av1g_tile_list_obu_entry": TileListObuEntry,
            "av1g_symbol_decoder": SymbolDecoder, "av1g_ref_state": RefState,
            "av1g_parsed_frame_header": ParsedFrameHeader, "av1g_tile_span": TileSpan}

# exported entry points and their ctypes signatures
_SIGS = {
    "av1g_abi_version": (C.c_int32, []),
    "av1g_struct_size": (C.c_int32, [C.c_char_p]),
    "av1g_last_error": (C.c_char_p, []),
    "av1g_lr_units_in_frame": (C.c_int32, [C.c_int32, C.c_int32]),
    "av1g_run_deblock": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_void_p]),
    "av1g_run_cdef": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_void_p]),
    "av1g_run_superres": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_void_p]),
    "av1g_run_lr": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_void_p]),
    "av1g_run_film_grain": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_void_p]),
    "av1g_run_postfilter": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_int32, C.c_void_p,
                                      C.POINTER(C.c_int32)]),
    "av1g_run_film_grain_noalloc": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_void_p]),
    "av1g_autotune_postfilter": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_void_p, C.c_char_p]),
    "av1g_autotune_load": (C.c_int, [C.c_char_p]),
    "av1g_autotune_get": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "av1g_chain_graph_create": (C.c_int, [C.POINTER(FrameJob), C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                                          C.POINTER(C.c_void_p)]),
    "av1g_chain_graph_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "av1g_chain_graph_launches": (C.c_int32, [C.c_void_p]),
    "av1g_chain_graph_destroy": (C.c_int, [C.c_void_p]),
    "av1g_run_recon": (C.c_int, [C.POINTER(ReconJob), C.c_int32, C.c_void_p]),
    "av1g_run_intra": (C.c_int, [C.POINTER(IntraJob), C.c_int32, C.c_void_p]),
    "av1g_run_inter": (C.c_int, [C.POINTER(InterJob), C.c_int32, C.c_void_p]),
    "av1g_run_mf_store": (C.c_int, [C.POINTER(MfStoreJob), C.c_int32, C.c_void_p]),
    "av1g_run_mf_project": (C.c_int, [C.POINTER(MfProjectJob), C.c_int32, C.c_void_p]),
    "av1g_framing_error": (C.c_int32, []),
    "av1g_leb128": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64), C.POINTER(C.c_int32)]),
    "av1g_parse_obu": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(Obu), C.POINTER(C.c_uint64)]),
    "av1g_ivf_parse_header": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(IvfHeader)]),
    "av1g_ivf_next_frame": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64), C.POINTER(IvfFrame),
                                      C.POINTER(C.c_int32)]),
    "av1g_annexb_split": (C.c_int, [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64), C.c_int32,
                                    C.POINTER(C.c_int32), C.POINTER(C.c_uint64)]),
    "av1g_annexb_build": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.c_int32, C.c_void_p, C.c_size_t,
                                    C.POINTER(C.c_uint64)]),
    "av1g_parse_sequence_header": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(SequenceHeader)]),
    "av1g_seq_info_from_header": (C.c_int, [C.POINTER(SequenceHeader), C.POINTER(SeqInfo)]),
    "av1g_temporal_unit_obus": (C.c_int, [C.c_void_p, C.c_size_t, C.c_int32, C.POINTER(C.c_uint16),
                                          C.POINTER(SequenceHeader), C.POINTER(C.c_int32), C.POINTER(Obu), C.c_int32,
                                          C.POINTER(C.c_int32)]),
    "av1g_frame_header_prefix": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(SequenceHeader),
                                           C.POINTER(FramePrefix)]),
    "av1g_run_tile_list_output": (C.c_int, [C.POINTER(TileListJob), C.c_int32, C.c_void_p]),
    "av1g_parse_tile_list": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(TileListHeader),
                                       C.POINTER(TileListObuEntry), C.c_int32]),
    "av1g_write_tile_list": (C.c_int, [C.POINTER(TileListHeader), C.POINTER(TileListObuEntry), C.c_int32,
                                       C.c_void_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_uint64)]),
    "av1g_symbol_init": (C.c_int, [C.POINTER(SymbolDecoder), C.c_void_p, C.c_size_t, C.c_int32]),
    "av1g_symbol_read": (C.c_int, [C.POINTER(SymbolDecoder), C.POINTER(C.c_uint16), C.c_int32,
                                   C.POINTER(C.c_uint32)]),
    "av1g_symbol_read_bool": (C.c_int, [C.POINTER(SymbolDecoder), C.POINTER(C.c_uint32)]),
    "av1g_symbol_read_literal": (C.c_int, [C.POINTER(SymbolDecoder), C.c_int32, C.POINTER(C.c_uint32)]),
    "av1g_symbol_read_ns": (C.c_int, [C.POINTER(SymbolDecoder), C.c_uint32, C.POINTER(C.c_uint32)]),
    "av1g_symbol_read_signed_subexp": (C.c_int, [C.POINTER(SymbolDecoder), C.c_int64, C.c_int64, C.c_uint32,
                                                 C.c_int64, C.POINTER(C.c_int64)]),
    "av1g_symbol_exit": (C.c_int, [C.POINTER(SymbolDecoder), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "av1g_update_cdf": (None, [C.POINTER(C.c_uint16), C.c_uint32, C.c_int32]),
    "av1g_ref_state_init": (None, [C.POINTER(RefState)]),
    "av1g_parse_frame_header": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(SequenceHeader), C.POINTER(RefState),
                                          C.c_int32, C.c_int32, C.POINTER(ParsedFrameHeader)]),
    "av1g_ref_state_update": (C.c_int, [C.POINTER(RefState), C.POINTER(ParsedFrameHeader)]),
    "av1g_parse_tile_group": (C.c_int, [C.c_void_p, C.c_size_t, C.POINTER(ParsedFrameHeader),
                                        C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(TileSpan),
                                        C.c_int32]),
    "av1g_engine_create": (C.c_int, [C.POINTER(Config), C.POINTER(C.c_void_p)]),
    "av1g_engine_destroy": (None, [C.c_void_p]),
    "av1g_engine_get_stats": (C.c_int, [C.c_void_p, C.POINTER(EngineStats)]),
    "av1g_stream_open": (C.c_int, [C.c_void_p, C.POINTER(SeqInfo), C.POINTER(C.c_void_p)]),
    "av1g_stream_close": (C.c_int, [C.c_void_p]),
    "av1g_stream_reset_refs": (C.c_int, [C.c_void_p]),
    "av1g_submit_frame": (C.c_int, [C.c_void_p, C.POINTER(FrameDesc), C.POINTER(C.c_uint64)]),
    "av1g_poll": (C.c_int, [C.c_void_p, C.c_uint64, C.c_int64, C.POINTER(C.c_int)]),
    "av1g_fetch_output": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(FrameOut)]),
    "av1g_release_output": (C.c_int, [C.c_void_p, C.c_uint64]),
    "av1g_warp_estimation": (C.c_int, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                       C.c_int16, C.c_int16, C.POINTER(C.c_int32), C.POINTER(C.c_uint8)]),
    "av1g_decoder_create": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)]),
    "av1g_decoder_destroy": (None, [C.c_void_p]),
    "av1g_decoder_send_packet": (C.c_int, [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int64]),
    "av1g_decoder_receive_frame": (C.c_int, [C.c_void_p, C.POINTER(FrameOut), C.POINTER(C.c_int64)]),
    "av1g_decoder_flush": (C.c_int, [C.c_void_p]),
    "av1g_decoder_reset": (C.c_int, [C.c_void_p]),
    "av1g_decoder_parsed_count": (C.c_int32, [C.c_void_p]),
    "av1g_decoder_parsed_frame": (C.c_int, [C.c_void_p, C.c_int32, C.POINTER(FrameDesc),
                                            C.POINTER(ParsedFrameHeader)]),
    "av1g_decoder_sequence": (C.c_int, [C.c_void_p, C.POINTER(SequenceHeader)]),
    "av1g_decoder_host_ms": (C.c_double, [C.c_void_p]),
    "av1g_decoder_frames_out_of_sync": (C.c_int32, [C.c_void_p]),
    "av1g_test_intra_wait_fault": (C.c_int, [C.c_int64, C.c_int32]),
    "av1g_intra_plan_stats_get": (C.c_int, [C.POINTER(IntraJob), C.c_int32, C.POINTER(IntraPlanStats)]),
}

NOALLOC_MAX_FRAMES = 16
NOALLOC_SCRATCH_BYTES = 2 * 1024 * 1024

_lib = None


class Av1gError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def load(path=None):
    """Load the CUDA library once; raises if it is absent or inconsistent."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"CUDA library {p} is not built; run build.py (no CPU fallback exists)")
    lib = C.CDLL(str(p))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if lib.av1g_abi_version() != 1:
        raise RuntimeError("ABI version mismatch")
    for cname, cls in _STRUCTS.items():
        n = lib.av1g_struct_size(cname.encode())
        if n != C.sizeof(cls):
            raise RuntimeError(f"struct {cname}: library {n} bytes, ctypes {C.sizeof(cls)} bytes")
    _lib = lib
    return lib


def check(status):
    if status != AV1G_OK:
        raise Av1gError(status, _lib.av1g_last_error().decode(errors="replace"))


def exported_symbols():
    return list(_SIGS)


def warp_estimation(cands, mi_row, mi_col, bw4, bh4, mv_row, mv_col):
    """av1g_warp_estimation: cands = sequence of (sy, sx, dy, dx); returns (valid, params)."""
    lib = load()
    arr = (WarpSample * max(len(cands), 1))(*[WarpSample(*c) for c in cands])
    params = (C.c_int32 * 6)()
    valid = C.c_uint8()
    check(lib.av1g_warp_estimation(C.cast(arr, C.c_void_p), len(cands), mi_row, mi_col, bw4, bh4, mv_row, mv_col,
                                   params, C.byref(valid)))
    return bool(valid.value), list(params)
