// walker.h — host tile walker: the §5.11 tile / partition / block syntax,
// the §8.3 symbol contexts and the §7.10 motion vector prediction, turning
// one frame's tile data into the frame descriptor the engine reconstructs
// (av1g_frame_desc: mode-info grids, transform units with their quantized
// levels, inter prediction calls, intra transform units in decode order,
// CDEF indices and loop-restoration units).
//
// It replaces the parse half of the reference's PartitionWalker
// (src/cdf.rs:15391, decode_tile_syntax_with_lr cdf.rs:33430) in parse-only
// mode: where the reference predicts and reconstructs each transform block
// while it parses (transform_block_emit, cdf.rs:32482), this walker records
// the block's prediction inputs and levels and leaves every sample to the
// GPU kernels.  AV1 parsing never reads a sample value, so the split is
// exact.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "av1g.h"

namespace av1w {

// One CDF row of an n-symbol alphabet: n cumulative values and the counter.
// Every member below is an array of such rows (TileCdfContext,
// src/cdf.rs:9199).
struct Cdfs {
    uint16_t intra_frame_y_mode[5][5][14];
    uint16_t y_mode[4][14];
    uint16_t uv_mode_cfl_not_allowed[13][14];
    uint16_t uv_mode_cfl_allowed[13][15];
    uint16_t angle_delta[8][8];
    uint16_t intrabc[3];
    uint16_t partition_w8[4][5];
    uint16_t partition_w16[4][11];
    uint16_t partition_w32[4][11];
    uint16_t partition_w64[4][11];
    uint16_t partition_w128[4][9];
    uint16_t skip[3][3];
    uint16_t skip_mode[3][3];
    uint16_t segment_id[3][9];
    uint16_t segment_id_predicted[3][3];
    uint16_t delta_q[5];
    uint16_t delta_lf[5];
    uint16_t delta_lf_multi[4][5];
    uint16_t is_inter[4][3];
    uint16_t comp_mode[5][3];
    uint16_t comp_ref_type[5][3];
    uint16_t uni_comp_ref[3][3][3];
    uint16_t comp_ref[3][3][3];
    uint16_t comp_bwd_ref[3][2][3];
    uint16_t single_ref[3][6][3];
    uint16_t compound_mode[8][9];
    uint16_t new_mv[6][3];
    uint16_t zero_mv[2][3];
    uint16_t ref_mv[6][3];
    uint16_t drl_mode[3][3];
    // [MvCtx][comp]: MvCtx 1 is intra block copy (§8.3.2 MvCtx)
    uint16_t mv_joint[2][5];
    uint16_t mv_class[2][2][12];
    uint16_t mv_class0_bit[2][2][3];
    uint16_t mv_class0_fr[2][2][2][5];
    uint16_t mv_class0_hp[2][2][3];
    uint16_t mv_sign[2][2][3];
    uint16_t mv_bit[2][2][10][3];
    uint16_t mv_fr[2][2][5];
    uint16_t mv_hp[2][2][3];
    uint16_t interp_filter[16][4];
    uint16_t motion_mode[22][4];
    uint16_t use_obmc[22][3];
    uint16_t inter_intra[3][3];
    uint16_t inter_intra_mode[3][5];
    uint16_t wedge_inter_intra[22][3];
    uint16_t wedge_index[22][17];
    uint16_t compound_idx[6][3];
    uint16_t comp_group_idx[6][3];
    uint16_t compound_type[22][3];
    uint16_t filter_intra_mode[6];
    uint16_t filter_intra[22][3];
    uint16_t palette_y_mode[7][3][3];
    uint16_t palette_uv_mode[2][3];
    uint16_t palette_y_size[7][8];
    uint16_t palette_uv_size[7][8];
    // [n - 2][ctx][n + 1 used of 9]
    uint16_t palette_y_color[7][5][9];
    uint16_t palette_uv_color[7][5][9];
    uint16_t cfl_sign[9];
    uint16_t cfl_alpha[6][17];
    uint16_t tx_8x8[3][3];
    uint16_t tx_16x16[3][4];
    uint16_t tx_32x32[3][4];
    uint16_t tx_64x64[3][4];
    uint16_t txfm_split[21][3];
    uint16_t inter_tx_type_set1[2][17];
    uint16_t inter_tx_type_set2[13];
    uint16_t inter_tx_type_set3[4][3];
    uint16_t intra_tx_type_set1[2][13][8];
    uint16_t intra_tx_type_set2[3][13][6];
    uint16_t use_wiener[3];
    uint16_t use_sgrproj[3];
    uint16_t restoration_type[4];
    // coefficient CDFs (chosen by the base_q_idx context at init)
    uint16_t txb_skip[5][13][3];
    uint16_t eob_pt_16[2][2][6];
    uint16_t eob_pt_32[2][2][7];
    uint16_t eob_pt_64[2][2][8];
    uint16_t eob_pt_128[2][2][9];
    uint16_t eob_pt_256[2][2][10];
    uint16_t eob_pt_512[2][11];
    uint16_t eob_pt_1024[2][12];
    uint16_t eob_extra[5][2][9][3];
    uint16_t dc_sign[2][3][3];
    uint16_t coeff_base_eob[5][2][4][4];
    uint16_t coeff_base[5][2][42][5];
    uint16_t coeff_br[5][2][21][5];
};

// §8.3.1 init_non_coeff_cdfs + init_coeff_cdfs(base_q_idx).
void cdfs_init(Cdfs& c, int base_q_idx);
// §8.3.1 load_cdfs: every counter restarts at 0.
void cdfs_zero_counts(Cdfs& c);

// Per-slot state the syntax of later frames reads (§7.20): the frame-end
// CDFs, the segmentation map, the motion-field candidates (§7.19) and the
// frame's mi extent and type.
struct SlotParse {
    bool valid = false;
    Cdfs cdfs;
    int mi_rows = 0, mi_cols = 0;
    bool frame_is_intra = true;
    std::vector<uint8_t> segment_ids;
    std::vector<int8_t> mf_ref_frames;   // per mi cell
    std::vector<int16_t> mf_mvs;         // per mi cell, [row, col]
    int saved_order_hints[8] = {0};
};

// Everything the walk produced for one frame, owned until the next frame.
struct FrameOut {
    av1g_frame_header hdr;
    av1g_quant_params quant;
    std::vector<uint8_t> mi_size, skip, is_inter, y_mode, tx_size, inter_tx_size;
    std::vector<int8_t> ref_frame0, segment_id, delta_lf;
    std::vector<int8_t> cdef_idx;
    std::vector<av1g_lr_unit> lr_units[3];
    std::vector<av1g_inter_pred> inter_preds;
    std::vector<av1g_obmc_neighbour> neighbours;
    std::vector<av1g_warp_ctx> warps;
    std::vector<av1g_tu> inter_tus;
    std::vector<av1g_intra_tu> intra_tus;
    std::vector<uint8_t> palette_maps;
    std::vector<int32_t> coeffs;
    // grids later frames read (§7.19 storage input, §7.20 segment map)
    std::vector<int8_t> ref_frames;      // [cell][2]
    std::vector<int16_t> mvs;            // [cell][2][2]
    std::vector<uint8_t> segment_map;
    Cdfs end_cdfs;
    bool have_end_cdfs = false;
    // every tile's symbol data ended at its trailing bit (§8.2.4)
    bool tiles_in_sync = true;
    void fill_desc(av1g_frame_desc& d) const;
};

// Walks every tile of one frame.  `slots` is the decoder's per-slot parse
// state; `fh` the parsed header; `tiles` the tile payloads in tile order.
struct TileData {
    const uint8_t* data;
    size_t size;
};
av1g_status walk_frame(const av1g_sequence_header& seq, const av1g_parsed_frame_header& fh,
                       const av1g_ref_state& refs, const SlotParse* slots, const std::vector<TileData>& tiles,
                       FrameOut& out, std::string& err);

// §7.9 motion field estimation on the host (the walker's temporal
// candidates read it): MotionFieldMvs[ref - LAST][y8][x8][2] with
// MFMV_INVALID where nothing projects.
void motion_field_estimation(const av1g_parsed_frame_header& fh, const av1g_sequence_header& seq,
                             const av1g_ref_state& refs, const SlotParse* slots, std::vector<int16_t>& out);

}  // namespace av1w
