// walker_cdf.cpp — §8.3.1 CDF initialisation for the tile walker: the §9.4
// defaults (TileCdfContext::new_from_defaults, src/cdf.rs:9726), the
// coefficient CDFs of the base_q_idx context (init_coeff_cdfs, cdf.rs:10550;
// coeff_cdf_q_ctx, cdf.rs:10925) and the counter reset of load_cdfs.
#include <cstring>

#include "av1_cdf_tables.h"
#include "walker.h"

namespace av1w {

namespace {

template <typename T, typename U>
void cp(T& dst, const U& src) {
    static_assert(sizeof(T) == sizeof(U), "CDF shape mismatch");
    std::memcpy(&dst, &src, sizeof(T));
}

// Rows of width w: the counter is the last entry of each row.
void zero_rows(uint16_t* p, size_t total, size_t w) {
    for (size_t i = w - 1; i < total; i += w) p[i] = 0;
}

template <typename T>
void zr(T& a, size_t w) {
    zero_rows(reinterpret_cast<uint16_t*>(&a), sizeof(T) / sizeof(uint16_t), w);
}

void copy_palette(uint16_t dst[7][5][9], int n, const uint16_t* src) {
    for (int ctx = 0; ctx < 5; ctx++)
        for (int i = 0; i <= n; i++) dst[n - 2][ctx][i] = src[ctx * (n + 1) + i];
}

}  // namespace

void cdfs_init(Cdfs& c, int base_q_idx) {
    std::memset(&c, 0, sizeof(c));
    cp(c.intra_frame_y_mode, Default_Intra_Frame_Y_Mode_Cdf);
    cp(c.y_mode, Default_Y_Mode_Cdf);
    cp(c.uv_mode_cfl_not_allowed, Default_Uv_Mode_Cfl_Not_Allowed_Cdf);
    cp(c.uv_mode_cfl_allowed, Default_Uv_Mode_Cfl_Allowed_Cdf);
    cp(c.angle_delta, Default_Angle_Delta_Cdf);
    cp(c.intrabc, Default_Intrabc_Cdf);
    cp(c.partition_w8, Default_Partition_W8_Cdf);
    cp(c.partition_w16, Default_Partition_W16_Cdf);
    cp(c.partition_w32, Default_Partition_W32_Cdf);
    cp(c.partition_w64, Default_Partition_W64_Cdf);
    cp(c.partition_w128, Default_Partition_W128_Cdf);
    cp(c.skip, Default_Skip_Cdf);
    cp(c.skip_mode, Default_Skip_Mode_Cdf);
    cp(c.segment_id, Default_Segment_Id_Cdf);
    cp(c.segment_id_predicted, Default_Segment_Id_Predicted_Cdf);
    cp(c.delta_q, Default_Delta_Q_Cdf);
    cp(c.delta_lf, Default_Delta_Lf_Cdf);
    for (int i = 0; i < 4; i++) cp(c.delta_lf_multi[i], Default_Delta_Lf_Cdf);
    cp(c.is_inter, Default_Is_Inter_Cdf);
    cp(c.comp_mode, Default_Comp_Mode_Cdf);
    cp(c.comp_ref_type, Default_Comp_Ref_Type_Cdf);
    cp(c.uni_comp_ref, Default_Uni_Comp_Ref_Cdf);
    cp(c.comp_ref, Default_Comp_Ref_Cdf);
    cp(c.comp_bwd_ref, Default_Comp_Bwd_Ref_Cdf);
    cp(c.single_ref, Default_Single_Ref_Cdf);
    cp(c.compound_mode, Default_Compound_Mode_Cdf);
    cp(c.new_mv, Default_New_Mv_Cdf);
    cp(c.zero_mv, Default_Zero_Mv_Cdf);
    cp(c.ref_mv, Default_Ref_Mv_Cdf);
    cp(c.drl_mode, Default_Drl_Mode_Cdf);
    for (int ctx = 0; ctx < 2; ctx++) {
        cp(c.mv_joint[ctx], Default_Mv_Joint_Cdf);
        cp(c.mv_class[ctx], Default_Mv_Class_Cdf);
        cp(c.mv_class0_fr[ctx], Default_Mv_Class0_Fr_Cdf);
        cp(c.mv_fr[ctx], Default_Mv_Fr_Cdf);
        for (int comp = 0; comp < 2; comp++) {
            cp(c.mv_class0_bit[ctx][comp], Default_Mv_Class0_Bit_Cdf);
            cp(c.mv_class0_hp[ctx][comp], Default_Mv_Class0_Hp_Cdf);
            cp(c.mv_sign[ctx][comp], Default_Mv_Sign_Cdf);
            cp(c.mv_bit[ctx][comp], Default_Mv_Bit_Cdf);
            cp(c.mv_hp[ctx][comp], Default_Mv_Hp_Cdf);
        }
    }
    cp(c.interp_filter, Default_Interp_Filter_Cdf);
    cp(c.motion_mode, Default_Motion_Mode_Cdf);
    cp(c.use_obmc, Default_Use_Obmc_Cdf);
    cp(c.inter_intra, Default_Inter_Intra_Cdf);
    cp(c.inter_intra_mode, Default_Inter_Intra_Mode_Cdf);
    cp(c.wedge_inter_intra, Default_Wedge_Inter_Intra_Cdf);
    cp(c.wedge_index, Default_Wedge_Index_Cdf);
    cp(c.compound_idx, Default_Compound_Idx_Cdf);
    cp(c.comp_group_idx, Default_Comp_Group_Idx_Cdf);
    cp(c.compound_type, Default_Compound_Type_Cdf);
    cp(c.filter_intra_mode, Default_Filter_Intra_Mode_Cdf);
    cp(c.filter_intra, Default_Filter_Intra_Cdf);
    cp(c.palette_y_mode, Default_Palette_Y_Mode_Cdf);
    cp(c.palette_uv_mode, Default_Palette_Uv_Mode_Cdf);
    cp(c.palette_y_size, Default_Palette_Y_Size_Cdf);
    cp(c.palette_uv_size, Default_Palette_Uv_Size_Cdf);
    copy_palette(c.palette_y_color, 2, &Default_Palette_Size_2_Y_Color_Cdf[0][0]);
    copy_palette(c.palette_y_color, 3, &Default_Palette_Size_3_Y_Color_Cdf[0][0]);
    copy_palette(c.palette_y_color, 4, &Default_Palette_Size_4_Y_Color_Cdf[0][0]);
    copy_palette(c.palette_y_color, 5, &Default_Palette_Size_5_Y_Color_Cdf[0][0]);
    copy_palette(c.palette_y_color, 6, &Default_Palette_Size_6_Y_Color_Cdf[0][0]);
    copy_palette(c.palette_y_color, 7, &Default_Palette_Size_7_Y_Color_Cdf[0][0]);
    copy_palette(c.palette_y_color, 8, &Default_Palette_Size_8_Y_Color_Cdf[0][0]);
    copy_palette(c.palette_uv_color, 2, &Default_Palette_Size_2_Uv_Color_Cdf[0][0]);
    copy_palette(c.palette_uv_color, 3, &Default_Palette_Size_3_Uv_Color_Cdf[0][0]);
    copy_palette(c.palette_uv_color, 4, &Default_Palette_Size_4_Uv_Color_Cdf[0][0]);
    copy_palette(c.palette_uv_color, 5, &Default_Palette_Size_5_Uv_Color_Cdf[0][0]);
    copy_palette(c.palette_uv_color, 6, &Default_Palette_Size_6_Uv_Color_Cdf[0][0]);
    copy_palette(c.palette_uv_color, 7, &Default_Palette_Size_7_Uv_Color_Cdf[0][0]);
    copy_palette(c.palette_uv_color, 8, &Default_Palette_Size_8_Uv_Color_Cdf[0][0]);
    cp(c.cfl_sign, Default_Cfl_Sign_Cdf);
    cp(c.cfl_alpha, Default_Cfl_Alpha_Cdf);
    cp(c.tx_8x8, Default_Tx_8x8_Cdf);
    cp(c.tx_16x16, Default_Tx_16x16_Cdf);
    cp(c.tx_32x32, Default_Tx_32x32_Cdf);
    cp(c.tx_64x64, Default_Tx_64x64_Cdf);
    cp(c.txfm_split, Default_Txfm_Split_Cdf);
    cp(c.inter_tx_type_set1, Default_Inter_Tx_Type_Set1_Cdf);
    cp(c.inter_tx_type_set2, Default_Inter_Tx_Type_Set2_Cdf);
    cp(c.inter_tx_type_set3, Default_Inter_Tx_Type_Set3_Cdf);
    cp(c.intra_tx_type_set1, Default_Intra_Tx_Type_Set1_Cdf);
    cp(c.intra_tx_type_set2, Default_Intra_Tx_Type_Set2_Cdf);
    cp(c.use_wiener, Default_Use_Wiener_Cdf);
    cp(c.use_sgrproj, Default_Use_Sgrproj_Cdf);
    cp(c.restoration_type, Default_Restoration_Type_Cdf);
    int q = base_q_idx <= 20 ? 0 : base_q_idx <= 60 ? 1 : base_q_idx <= 120 ? 2 : 3;
    cp(c.txb_skip, Default_Txb_Skip_Cdf[q]);
    cp(c.eob_pt_16, Default_Eob_Pt_16_Cdf[q]);
    cp(c.eob_pt_32, Default_Eob_Pt_32_Cdf[q]);
    cp(c.eob_pt_64, Default_Eob_Pt_64_Cdf[q]);
    cp(c.eob_pt_128, Default_Eob_Pt_128_Cdf[q]);
    cp(c.eob_pt_256, Default_Eob_Pt_256_Cdf[q]);
    cp(c.eob_pt_512, Default_Eob_Pt_512_Cdf[q]);
    cp(c.eob_pt_1024, Default_Eob_Pt_1024_Cdf[q]);
    cp(c.eob_extra, Default_Eob_Extra_Cdf[q]);
    cp(c.dc_sign, Default_Dc_Sign_Cdf[q]);
    cp(c.coeff_base_eob, Default_Coeff_Base_Eob_Cdf[q]);
    cp(c.coeff_base, Default_Coeff_Base_Cdf[q]);
    cp(c.coeff_br, Default_Coeff_Br_Cdf[q]);
}

void cdfs_zero_counts(Cdfs& c) {
    zr(c.intra_frame_y_mode, 14);
    zr(c.y_mode, 14);
    zr(c.uv_mode_cfl_not_allowed, 14);
    zr(c.uv_mode_cfl_allowed, 15);
    zr(c.angle_delta, 8);
    zr(c.intrabc, 3);
    zr(c.partition_w8, 5);
    zr(c.partition_w16, 11);
    zr(c.partition_w32, 11);
    zr(c.partition_w64, 11);
    zr(c.partition_w128, 9);
    zr(c.skip, 3);
    zr(c.skip_mode, 3);
    zr(c.segment_id, 9);
    zr(c.segment_id_predicted, 3);
    zr(c.delta_q, 5);
    zr(c.delta_lf, 5);
    zr(c.delta_lf_multi, 5);
    zr(c.is_inter, 3);
    zr(c.comp_mode, 3);
    zr(c.comp_ref_type, 3);
    zr(c.uni_comp_ref, 3);
    zr(c.comp_ref, 3);
    zr(c.comp_bwd_ref, 3);
    zr(c.single_ref, 3);
    zr(c.compound_mode, 9);
    zr(c.new_mv, 3);
    zr(c.zero_mv, 3);
    zr(c.ref_mv, 3);
    zr(c.drl_mode, 3);
    zr(c.mv_joint, 5);
    zr(c.mv_class, 12);
    zr(c.mv_class0_bit, 3);
    zr(c.mv_class0_fr, 5);
    zr(c.mv_class0_hp, 3);
    zr(c.mv_sign, 3);
    zr(c.mv_bit, 3);
    zr(c.mv_fr, 5);
    zr(c.mv_hp, 3);
    zr(c.interp_filter, 4);
    zr(c.motion_mode, 4);
    zr(c.use_obmc, 3);
    zr(c.inter_intra, 3);
    zr(c.inter_intra_mode, 5);
    zr(c.wedge_inter_intra, 3);
    zr(c.wedge_index, 17);
    zr(c.compound_idx, 3);
    zr(c.comp_group_idx, 3);
    zr(c.compound_type, 3);
    zr(c.filter_intra_mode, 6);
    zr(c.filter_intra, 3);
    zr(c.palette_y_mode, 3);
    zr(c.palette_uv_mode, 3);
    zr(c.palette_y_size, 8);
    zr(c.palette_uv_size, 8);
    for (int n = 2; n <= 8; n++)
        for (int ctx = 0; ctx < 5; ctx++) {
            c.palette_y_color[n - 2][ctx][n] = 0;
            c.palette_uv_color[n - 2][ctx][n] = 0;
        }
    zr(c.cfl_sign, 9);
    zr(c.cfl_alpha, 17);
    zr(c.tx_8x8, 3);
    zr(c.tx_16x16, 4);
    zr(c.tx_32x32, 4);
    zr(c.tx_64x64, 4);
    zr(c.txfm_split, 3);
    zr(c.inter_tx_type_set1, 17);
    zr(c.inter_tx_type_set2, 13);
    zr(c.inter_tx_type_set3, 3);
    zr(c.intra_tx_type_set1, 8);
    zr(c.intra_tx_type_set2, 6);
    zr(c.use_wiener, 3);
    zr(c.use_sgrproj, 3);
    zr(c.restoration_type, 4);
    zr(c.txb_skip, 3);
    zr(c.eob_pt_16, 6);
    zr(c.eob_pt_32, 7);
    zr(c.eob_pt_64, 8);
    zr(c.eob_pt_128, 9);
    zr(c.eob_pt_256, 10);
    zr(c.eob_pt_512, 11);
    zr(c.eob_pt_1024, 12);
    zr(c.eob_extra, 3);
    zr(c.dc_sign, 3);
    zr(c.coeff_base_eob, 4);
    zr(c.coeff_base, 5);
    zr(c.coeff_br, 5);
}

}  // namespace av1w
