// walker.cpp — the §5.11 tile syntax walk of one frame (host, serial).
//
// Follows the reference's PartitionWalker in parse-only mode:
//   decode_tile_syntax_with_lr (src/cdf.rs:33430) -> read_lr (cdf.rs:20142)
//   -> decode_partition_syntax (cdf.rs:32995) -> decode_block_syntax
//   (cdf.rs:29840: mode info cdf.rs:23734-28172, palette cdf.rs:29592,
//   transform sizes cdf.rs:28302-28930) -> residual (cdf.rs:32000,
//   residual_transform_tree 32212, coefficients 29062, the §8.3.2 contexts
//   cdf.rs:21650-21860), and the §7.10.2 motion vector prediction
//   find_mv_stack (cdf.rs:33718-35430) with the §7.10.4 warp samples
//   (cdf.rs:26425).
// Where the reference reconstructs (transform_block_emit, cdf.rs:32482; the
// inter leaf, cdf.rs:19001; intra block copy, cdf.rs:19235) this walker
// records the inputs as engine descriptors instead.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

#include "av1_cdf_tables.h"
#include "walker.h"

namespace av1w {

namespace {

// ---------------------------------------------------------------------------
// constants (the reference's numbering: inter modes follow UV_CFL_PRED)
// ---------------------------------------------------------------------------
enum { INTRA_FRAME = 0, LAST_FRAME = 1, LAST2_FRAME, LAST3_FRAME, GOLDEN_FRAME, BWDREF_FRAME, ALTREF2_FRAME,
       ALTREF_FRAME };
constexpr int NONE_REF = -1;
enum { DC_PRED = 0, V_PRED, H_PRED, D45_PRED, D135_PRED, D113_PRED, D157_PRED, D203_PRED, D67_PRED, SMOOTH_PRED,
       SMOOTH_V_PRED, SMOOTH_H_PRED, PAETH_PRED, UV_CFL_PRED };
enum { NEARESTMV = 14, NEARMV, GLOBALMV, NEWMV, NEAREST_NEARESTMV, NEAR_NEARMV, NEAREST_NEWMV, NEW_NEARESTMV,
       NEAR_NEWMV, NEW_NEARMV, GLOBAL_GLOBALMV, NEW_NEWMV };
enum { BLOCK_4X4 = 0, BLOCK_4X8, BLOCK_8X4, BLOCK_8X8, BLOCK_8X16, BLOCK_16X8, BLOCK_16X16, BLOCK_16X32,
       BLOCK_32X16, BLOCK_32X32, BLOCK_32X64, BLOCK_64X32, BLOCK_64X64, BLOCK_64X128, BLOCK_128X64,
       BLOCK_128X128, BLOCK_4X16, BLOCK_16X4, BLOCK_8X32, BLOCK_32X8, BLOCK_16X64, BLOCK_64X16,
       BLOCK_INVALID };
enum { TX_4X4 = 0, TX_8X8, TX_16X16, TX_32X32, TX_64X64, TX_4X8, TX_8X4, TX_8X16, TX_16X8, TX_16X32, TX_32X16,
       TX_32X64, TX_64X32, TX_4X16, TX_16X4, TX_8X32, TX_32X8, TX_16X64, TX_64X16 };
enum { PARTITION_NONE = 0, PARTITION_HORZ, PARTITION_VERT, PARTITION_SPLIT, PARTITION_HORZ_A, PARTITION_HORZ_B,
       PARTITION_VERT_A, PARTITION_VERT_B, PARTITION_HORZ_4, PARTITION_VERT_4 };
enum { SEG_LVL_ALT_Q = 0, SEG_LVL_REF_FRAME = 5, SEG_LVL_SKIP = 6, SEG_LVL_GLOBALMV = 7 };
enum { DCT_DCT = 0, IDTX = 9, V_DCT = 10, H_DCT = 11, V_ADST = 12, H_ADST = 13, V_FLIPADST = 14,
       H_FLIPADST = 15 };
enum { TX_SET_DCTONLY = 0, TX_SET_INTER_1 = 1, TX_SET_INTER_2, TX_SET_INTER_3 };
enum { TX_SET_INTRA_1 = 1, TX_SET_INTRA_2 };
enum { SIMPLE = 0, OBMC = 1, LOCALWARP = 2 };
enum { COMPOUND_WEDGE = 0, COMPOUND_DIFFWTD = 1, COMPOUND_AVERAGE = 2, COMPOUND_INTRA = 3, COMPOUND_DISTANCE = 4 };
enum { IDENTITY = 0, TRANSLATION = 1, ROTZOOM = 2, AFFINE = 3 };
constexpr int REF_CAT_LEVEL = 640;
constexpr int MV_BORDER = 128;
constexpr int16_t MFMV_INVALID = -32768;
constexpr int WARPEDMODEL_PREC_BITS = 16;
constexpr int BILINEAR = 3;
constexpr int SWITCHABLE = 4;

inline int bw_of(int b) { return Num_4x4_Blocks_Wide[b] * 4; }
inline int bh_of(int b) { return Num_4x4_Blocks_High[b] * 4; }
inline int tx_sqr(int t) {
    int m = std::min(Tx_Width[t], Tx_Height[t]);
    return m == 4 ? 0 : m == 8 ? 1 : m == 16 ? 2 : m == 32 ? 3 : 4;
}
inline int clip3(int lo, int hi, int v) { return v < lo ? lo : v > hi ? hi : v; }
inline int64_t round2signed(int64_t x, int n) {
    if (n == 0) return x;
    return x >= 0 ? (x + ((int64_t)1 << (n - 1))) >> n : -((-x + ((int64_t)1 << (n - 1))) >> n);
}
inline int ceil_log2(int x) {
    if (x < 2) return 0;
    int i = 1, p = 2;
    while (p < x) {
        i++;
        p <<= 1;
    }
    return i;
}
int find_tx_size(int w, int h) {
    for (int t = 0; t < 19; t++)
        if (Tx_Width[t] == w && Tx_Height[t] == h) return t;
    return -1;
}
int get_relative_dist(int a, int b, int bits) {
    if (!bits) return 0;
    int diff = a - b;
    int m = 1 << (bits - 1);
    diff = (diff & (m - 1)) - (diff & m);
    return diff;
}

const int16_t Wiener_Taps_Min[3] = {-5, -23, -17};
const int16_t Wiener_Taps_Max[3] = {10, 8, 46};
const int16_t Wiener_Taps_K[3] = {1, 2, 3};
const int16_t Wiener_Taps_Mid[3] = {3, -7, 15};
const int16_t Sgrproj_Xqd_Min[2] = {-96, -32};
const int16_t Sgrproj_Xqd_Max[2] = {31, 95};
const int16_t Sgrproj_Xqd_Mid[2] = {-32, 31};
// radii r0, r1 of the 16 self-guided parameter sets (Sgr_Params[.][0], [.][2])
const uint8_t Sgr_Radius[16][2] = {{2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1}, {2, 1},
                                   {2, 1}, {2, 1}, {0, 1}, {0, 1}, {0, 1}, {0, 1}, {2, 0}, {2, 0}};
const uint8_t Filter_Intra_Mode_To_Intra_Dir[5] = {DC_PRED, V_PRED, H_PRED, D157_PRED, DC_PRED};

struct WalkError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// ---------------------------------------------------------------------------
// the walker
// ---------------------------------------------------------------------------
struct Walker {
    // inputs
    const av1g_sequence_header& seq;
    const av1g_parsed_frame_header& fh;
    const av1g_ref_state& refs;
    const SlotParse* slots;
    FrameOut& out;

    // frame constants
    int MiRows = 0, MiCols = 0, NumPlanes = 3, ssx = 1, ssy = 1, BitDepth = 8;
    bool FrameIsIntra = true, sb128 = false;
    int SegIdPreSkip = 0, LastActiveSegId = 0;
    bool CodedLossless = false;
    int OrderHintBits = 0;
    int RefFrameSignBias[8] = {0};
    bool IsScaled[8] = {false};
    std::vector<int16_t> MotionFieldMvs;   // [7][MiRows/2][MiCols/2][2]
    const uint8_t* PrevSegmentIds = nullptr;

    // tile state
    int MiRowStart = 0, MiRowEnd = 0, MiColStart = 0, MiColEnd = 0;
    av1g_symbol_decoder sd{};
    Cdfs cdf;
    int CurrentQIndex = 0;
    int DeltaLF[4] = {0};
    int RefSgrXqd[3][2];
    int RefLrWiener[3][2][3];
    bool ReadDeltas = false;
    std::vector<uint8_t> AboveLevelContext[3], AboveDcContext[3], LeftLevelContext[3], LeftDcContext[3];
    std::vector<uint8_t> AboveSegPredContext, LeftSegPredContext;

    // frame grids (per mi cell)
    std::vector<uint8_t> MiSizes, YModes, UVModes, IsInters, SkipModes, Skips, TxSizes, InterTxSizes, SegmentIds;
    std::vector<uint8_t> PaletteSizes[2];
    std::vector<uint16_t> PaletteColors[2];  // [cell][8]
    std::vector<uint8_t> CompGroupIdxs, CompoundIdxs, InterpFilters;  // InterpFilters [cell][2]
    std::vector<int8_t> RefFrames;   // [cell][2]
    std::vector<int16_t> Mvs;        // [cell][2][2]
    std::vector<uint8_t> TxTypes;    // per luma 4x4
    std::vector<int8_t> DeltaLFs;    // [cell][4]
    // BlockDecoded[plane][-1 .. 32][-1 .. 32]
    uint8_t BlockDecoded[3][34][34];

    // block state
    int MiRow = 0, MiCol = 0, MiSize = 0, bw4 = 0, bh4 = 0;
    bool HasChroma = false, AvailU = false, AvailL = false, AvailUChroma = false, AvailLChroma = false;
    int segment_id = 0, skip = 0, skip_mode = 0, is_inter = 0, use_intrabc = 0, Lossless = 0;
    int YMode = 0, UVMode = 0, AngleDeltaY = 0, AngleDeltaUV = 0, CflAlphaU = 0, CflAlphaV = 0;
    int use_filter_intra = 0, filter_intra_mode = 0;
    int PaletteSizeY = 0, PaletteSizeUV = 0;
    uint16_t palette_colors_y[8], palette_colors_u[8], palette_colors_v[8];
    std::vector<uint8_t> ColorMapY, ColorMapUV;
    int ColorMapYStride = 0, ColorMapUVStride = 0;
    int TxSize = 0;
    int RefFrame[2] = {0, -1};
    int Mv[2][2] = {{0, 0}, {0, 0}};
    int PredMv[2][2];
    int interp_filter[2] = {0, 0};
    int motion_mode = 0, interintra = 0, interintra_mode = 0, wedge_interintra = 0, wedge_index = 0,
        wedge_sign = 0, mask_type = 0, compound_type = COMPOUND_AVERAGE, comp_group_idx = 0, compound_idx = 1;
    int RefMvIdx = 0;
    int MaxLumaW = 0, MaxLumaH = 0;
    // neighbour references
    int LeftRefFrame[2], AboveRefFrame[2];
    bool LeftIntra = false, AboveIntra = false, LeftSingle = false, AboveSingle = false;
    // MV stack
    int NumMvFound = 0, NewMvCount = 0;
    int RefStackMv[9][2][2];
    int WeightStack[9];
    int GlobalMvs[2][2];
    int FoundMatch = 0, CloseMatches = 0, TotalMatches = 0, NewMvContext = 0, RefMvContext = 0, ZeroMvContext = 0;
    int DrlCtxStack[9];
    int RefIdCount[2], RefDiffCount[2], RefIdMvs[2][2][2], RefDiffMvs[2][2][2];
    // warp samples
    int NumSamples = 0, NumSamplesScanned = 0;
    av1g_warp_sample CandList[8];
    int32_t LocalWarpParams[6];
    int LocalValid = 0;
    // block's palette map offset in the output pool
    uint32_t palette_map_off[2] = {0, 0};
    // descriptor index where this block's prediction records start
    size_t block_first_intra_tu = 0;

    Walker(const av1g_sequence_header& s, const av1g_parsed_frame_header& f, const av1g_ref_state& r,
           const SlotParse* sl, FrameOut& o)
        : seq(s), fh(f), refs(r), slots(sl), out(o) {}

    // ---------------- symbol reading ----------------
    int S(uint16_t* c, int n) {
        uint32_t v;
        if (av1g_symbol_read(&sd, c, n, &v) != AV1G_OK) throw WalkError(av1g_last_error());
        return (int)v;
    }
    int L(int n) {
        uint32_t v;
        if (av1g_symbol_read_literal(&sd, n, &v) != AV1G_OK) throw WalkError(av1g_last_error());
        return (int)v;
    }
    int NS(int n) {
        uint32_t v;
        if (av1g_symbol_read_ns(&sd, (uint32_t)n, &v) != AV1G_OK) throw WalkError(av1g_last_error());
        return (int)v;
    }
    int subexp(int low, int high, int k, int r) {
        int64_t v;
        if (av1g_symbol_read_signed_subexp(&sd, low, high, (uint32_t)k, r, &v) != AV1G_OK)
            throw WalkError(av1g_last_error());
        return (int)v;
    }

    // ---------------- helpers ----------------
    size_t cell(int r, int c) const { return (size_t)r * MiCols + c; }
    bool is_inside(int r, int c) const {
        return c >= MiColStart && c < MiColEnd && r >= MiRowStart && r < MiRowEnd;
    }
    bool seg_feature_active_idx(int seg, int feature) const {
        return fh.segmentation_enabled && fh.seg_feature_enabled[seg][feature];
    }
    bool seg_feature_active(int feature) const { return seg_feature_active_idx(segment_id, feature); }
    int get_qidx(int ignoreDeltaQ, int seg) const {
        if (seg_feature_active_idx(seg, SEG_LVL_ALT_Q)) {
            int data = fh.seg_feature_data[seg][SEG_LVL_ALT_Q];
            int q = fh.base_q_idx + data;
            if (!ignoreDeltaQ && fh.delta_q_present) q = CurrentQIndex + data;
            return clip3(0, 255, q);
        }
        if (!ignoreDeltaQ && fh.delta_q_present) return CurrentQIndex;
        return fh.base_q_idx;
    }
    int plane_residual_size(int sz, int plane) const {
        if (plane == 0) return sz;
        return Subsampled_Size[sz][ssx][ssy];
    }
    int get_tx_size(int plane, int txSz) const {
        if (plane == 0) return txSz;
        int uvTx = Max_Tx_Size_Rect[plane_residual_size(MiSize, plane)];
        if (Tx_Width[uvTx] == 64 || Tx_Height[uvTx] == 64) {
            if (Tx_Width[uvTx] == 16) return TX_16X32;
            if (Tx_Height[uvTx] == 16) return TX_32X16;
            return TX_32X32;
        }
        return uvTx;
    }
    uint8_t& block_decoded(int plane, int y, int x) { return BlockDecoded[plane][y + 1][x + 1]; }

    // ---------------- frame set-up ----------------
    void setup_frame();
    void decode_tile(int tileRow, int tileCol, const TileData& td);
    void clear_block_decoded_flags(int r, int c, int sbSize4);
    void read_lr(int r, int c, int bSize);
    void read_lr_unit(int plane, int unitRow, int unitCol);
    void decode_partition(int r, int c, int bSize);
    void decode_block(int r, int c, int subSize);
    // mode info
    void intra_frame_mode_info();
    void inter_frame_mode_info();
    void intra_segment_id();
    void inter_segment_id(int preSkip);
    void read_segment_id();
    int get_segment_id();
    void read_skip_mode();
    void read_skip();
    void read_cdef();
    void read_delta_qindex();
    void read_delta_lf();
    void read_is_inter();
    void intra_block_mode_info();
    void inter_block_mode_info();
    void intra_angle_info_y();
    void intra_angle_info_uv();
    void read_uv_mode();
    void read_cfl_alphas();
    void palette_mode_info();
    int get_palette_cache(int plane, uint16_t* cache);
    void filter_intra_mode_info();
    void read_ref_frames();
    int count_refs(int frameType);
    void assign_mv(int isCompound);
    void read_mv(int ref);
    int read_mv_component(int ctx, int comp);
    void read_motion_mode(int isCompound);
    bool has_overlappable_candidates();
    void read_interintra_mode(int isCompound);
    void read_compound_type(int isCompound);
    bool needs_interp_filter();
    int interp_filter_ctx(int dir);
    int get_mode(int refList);
    // MV prediction
    void find_mv_stack(int isCompound);
    void setup_global_mv(int refList, int mv[2]);
    void lower_mv_precision(int mv[2]);
    void scan_row(int deltaRow, int isCompound);
    void scan_col(int deltaCol, int isCompound);
    void scan_point(int deltaRow, int deltaCol, int isCompound);
    void add_ref_mv_candidate(int mvRow, int mvCol, int isCompound, int weight);
    void search_stack(int mvRow, int mvCol, int candList, int weight);
    void compound_search_stack(int mvRow, int mvCol, int weight);
    void temporal_scan(int isCompound);
    void add_tpl_ref_mv(int deltaRow, int deltaCol, int isCompound);
    void sorting(int start, int end);
    void extra_search(int isCompound);
    void add_extra_mv_candidate(int mvRow, int mvCol, int isCompound);
    void context_and_clamping(int isCompound, int numNew);
    void find_warp_samples();
    void add_sample(int deltaRow, int deltaCol);
    // tx size / palette tokens / residual
    void read_block_tx_size();
    void read_var_tx_size(int row, int col, int txSz, int depth);
    void read_tx_size(int allowSelect);
    int get_above_tx_width(int row, int col);
    int get_left_tx_height(int row, int col);
    void palette_tokens();
    void get_palette_color_context(const uint8_t* map, int stride, int r, int c, int n, int* order, int* ctx);
    void reset_block_context();
    void residual();
    void transform_tree(int startX, int startY, int w, int h);
    void transform_block(int plane, int baseX, int baseY, int txSz, int x, int y);
    int coeffs(int plane, int startX, int startY, int txSz, int* planeTxType, uint32_t* coeffOff);
    void transform_type(int x4, int y4, int txSz);
    int get_tx_set(int txSz);
    int compute_tx_type(int plane, int txSz, int blockX, int blockY);
    int get_filter_type(int plane);
    bool is_smooth(int row, int col, int plane);
    // descriptors
    void emit_inter_block();
    void distance_weights(int* fwd, int* bck);
    void store_block_grids();
};

// ===========================================================================
// frame / tile
// ===========================================================================

void Walker::setup_frame() {
    const av1g_frame_header& pf = fh.pf;
    MiRows = pf.mi_rows;
    MiCols = pf.mi_cols;
    NumPlanes = pf.num_planes;
    ssx = pf.subsampling_x;
    ssy = pf.subsampling_y;
    BitDepth = pf.bit_depth;
    FrameIsIntra = fh.frame_type == 0 || fh.frame_type == 2;
    sb128 = seq.use_128x128_superblock;
    OrderHintBits = seq.enable_order_hint ? seq.order_hint_bits : 0;
    CodedLossless = pf.coded_lossless;
    if (fh.segmentation_enabled) {
        for (int i = 0; i < 8; i++)
            for (int j = 0; j < 8; j++)
                if (fh.seg_feature_enabled[i][j]) {
                    LastActiveSegId = i;
                    if (j >= SEG_LVL_REF_FRAME) SegIdPreSkip = 1;
                }
    }
    size_t cells = (size_t)MiRows * MiCols;
    MiSizes.assign(cells, BLOCK_INVALID);
    YModes.assign(cells, 0);
    UVModes.assign(cells, 0);
    IsInters.assign(cells, 0);
    SkipModes.assign(cells, 0);
    Skips.assign(cells, 0);
    TxSizes.assign(cells, 0);
    InterTxSizes.assign(cells, 0);
    SegmentIds.assign(cells, 0);
    CompGroupIdxs.assign(cells, 0);
    CompoundIdxs.assign(cells, 0);
    InterpFilters.assign(cells * 2, 0);
    RefFrames.assign(cells * 2, NONE_REF);
    for (size_t i = 0; i < cells; i++) RefFrames[i * 2] = INTRA_FRAME;
    Mvs.assign(cells * 4, 0);
    TxTypes.assign(cells, DCT_DCT);
    DeltaLFs.assign(cells * 4, 0);
    for (int p = 0; p < 2; p++) {
        PaletteSizes[p].assign(cells, 0);
        if (fh.allow_screen_content_tools) PaletteColors[p].assign(cells * 8, 0);
    }
    for (int p = 0; p < 3; p++) {
        AboveLevelContext[p].assign(MiCols + 32, 0);
        AboveDcContext[p].assign(MiCols + 32, 0);
        LeftLevelContext[p].assign(MiRows + 32, 0);
        LeftDcContext[p].assign(MiRows + 32, 0);
    }
    AboveSegPredContext.assign(MiCols + 32, 0);
    LeftSegPredContext.assign(MiRows + 32, 0);

    // reference frame properties (§7.8 sign bias, §5.11.27 is_scaled)
    if (!FrameIsIntra) {
        for (int i = 0; i < 7; i++) {
            int slot = fh.ref_frame_idx[i];
            int hint = refs.order_hint[slot];
            RefFrameSignBias[LAST_FRAME + i] =
                seq.enable_order_hint ? (get_relative_dist(hint, fh.order_hint, OrderHintBits) > 0) : 0;
            int64_t fw = std::max(1, pf.frame_width), fhh = std::max(1, pf.frame_height);
            int64_t xs = (((int64_t)refs.upscaled_width[slot] << 14) + fw / 2) / fw;
            int64_t ys = (((int64_t)refs.frame_height[slot] << 14) + fhh / 2) / fhh;
            IsScaled[LAST_FRAME + i] = xs != (1 << 14) || ys != (1 << 14);
        }
        if (fh.use_ref_frame_mvs) motion_field_estimation(fh, seq, refs, slots, MotionFieldMvs);
        if (fh.segmentation_enabled) {
            PrevSegmentIds = nullptr;
            if (fh.primary_ref_frame != 7) {
                const SlotParse& sp = slots[fh.ref_frame_idx[fh.primary_ref_frame]];
                if (sp.valid && sp.mi_rows == MiRows && sp.mi_cols == MiCols &&
                    sp.segment_ids.size() == cells)
                    PrevSegmentIds = sp.segment_ids.data();
            }
        }
    }

    // outputs
    out.hdr = pf;
    av1g_quant_params& q = out.quant;
    std::memset(&q, 0, sizeof q);
    q.base_q_idx = (uint8_t)fh.base_q_idx;
    q.delta_q_y_dc = (int8_t)fh.delta_q_y_dc;
    q.delta_q_u_dc = (int8_t)fh.delta_q_u_dc;
    q.delta_q_u_ac = (int8_t)fh.delta_q_u_ac;
    q.delta_q_v_dc = (int8_t)fh.delta_q_v_dc;
    q.delta_q_v_ac = (int8_t)fh.delta_q_v_ac;
    q.using_qmatrix = (uint8_t)fh.using_qmatrix;
    q.delta_q_present = (uint8_t)fh.delta_q_present;
    q.segmentation_enabled = (uint8_t)fh.segmentation_enabled;
    for (int s = 0; s < 8; s++) {
        q.seg_alt_q_active[s] = fh.segmentation_enabled && fh.seg_feature_enabled[s][SEG_LVL_ALT_Q];
        q.seg_alt_q_data[s] = fh.seg_feature_data[s][SEG_LVL_ALT_Q];
        q.lossless[s] = (uint8_t)fh.lossless[s];
        for (int p = 0; p < 3; p++) {
            int lvl = 15;
            if (fh.using_qmatrix && !fh.lossless[s]) lvl = p == 0 ? fh.qm_y : p == 1 ? fh.qm_u : fh.qm_v;
            q.seg_qm_level[p][s] = (uint8_t)lvl;
        }
    }
    int c64r = (MiRows + 15) >> 4, c64c = (MiCols + 15) >> 4;
    out.cdef_idx.assign((size_t)c64r * c64c, -1);
    for (int p = 0; p < 3; p++) {
        out.lr_units[p].clear();
        if (p < NumPlanes && pf.lr_type[p] != 0) {
            int sx = p ? ssx : 0, sy = p ? ssy : 0;
            int us = pf.lr_unit_size[p];
            int rows = av1g_lr_units_in_frame(us, (pf.frame_height + sy) >> sy);
            int cols = av1g_lr_units_in_frame(us, (pf.upscaled_width + sx) >> sx);
            out.lr_units[p].assign((size_t)rows * cols, av1g_lr_unit{});
        }
    }
    out.inter_preds.clear();
    out.neighbours.clear();
    out.warps.clear();
    out.inter_tus.clear();
    out.intra_tus.clear();
    out.palette_maps.clear();
    out.coeffs.clear();
}

void Walker::decode_tile(int tileRow, int tileCol, const TileData& td) {
    MiRowStart = fh.mi_row_starts[tileRow];
    MiRowEnd = fh.mi_row_starts[tileRow + 1];
    MiColStart = fh.mi_col_starts[tileCol];
    MiColEnd = fh.mi_col_starts[tileCol + 1];
    CurrentQIndex = fh.base_q_idx;
    if (av1g_symbol_init(&sd, td.data, td.size, fh.disable_cdf_update) != AV1G_OK)
        throw WalkError(av1g_last_error());
    // clear_above_context
    for (int p = 0; p < 3; p++) {
        std::fill(AboveLevelContext[p].begin(), AboveLevelContext[p].end(), 0);
        std::fill(AboveDcContext[p].begin(), AboveDcContext[p].end(), 0);
    }
    std::fill(AboveSegPredContext.begin(), AboveSegPredContext.end(), 0);
    for (int i = 0; i < 4; i++) DeltaLF[i] = 0;
    for (int p = 0; p < NumPlanes; p++)
        for (int pass = 0; pass < 2; pass++) {
            RefSgrXqd[p][pass] = Sgrproj_Xqd_Mid[pass];
            for (int i = 0; i < 3; i++) RefLrWiener[p][pass][i] = Wiener_Taps_Mid[i];
        }
    int sbSize = sb128 ? BLOCK_128X128 : BLOCK_64X64;
    int sbSize4 = Num_4x4_Blocks_Wide[sbSize];
    for (int r = MiRowStart; r < MiRowEnd; r += sbSize4) {
        // clear_left_context
        for (int p = 0; p < 3; p++) {
            std::fill(LeftLevelContext[p].begin(), LeftLevelContext[p].end(), 0);
            std::fill(LeftDcContext[p].begin(), LeftDcContext[p].end(), 0);
        }
        std::fill(LeftSegPredContext.begin(), LeftSegPredContext.end(), 0);
        for (int c = MiColStart; c < MiColEnd; c += sbSize4) {
            ReadDeltas = fh.delta_q_present;
            // clear_cdef
            int c64c = (MiCols + 15) >> 4;
            auto clr = [&](int rr, int cc) {
                if (rr < MiRows && cc < MiCols) out.cdef_idx[(size_t)(rr >> 4) * c64c + (cc >> 4)] = -1;
            };
            clr(r, c);
            if (sb128) {
                clr(r, c + 16);
                clr(r + 16, c);
                clr(r + 16, c + 16);
            }
            clear_block_decoded_flags(r, c, sbSize4);
            read_lr(r, c, sbSize);
            decode_partition(r, c, sbSize);
        }
    }
}

void Walker::clear_block_decoded_flags(int r, int c, int sbSize4) {
    for (int plane = 0; plane < NumPlanes; plane++) {
        int subX = plane ? ssx : 0, subY = plane ? ssy : 0;
        int sbWidth4 = (MiColEnd - c) >> subX;
        int sbHeight4 = (MiRowEnd - r) >> subY;
        for (int y = -1; y <= (sbSize4 >> subY); y++)
            for (int x = -1; x <= (sbSize4 >> subX); x++) {
                uint8_t v = (y < 0 && x < sbWidth4) || (x < 0 && y < sbHeight4);
                block_decoded(plane, y, x) = v;
            }
        block_decoded(plane, sbSize4 >> subY, -1) = 0;
    }
}

void Walker::read_lr(int r, int c, int bSize) {
    if (fh.pf.allow_intrabc) return;
    int w = Num_4x4_Blocks_Wide[bSize], h = Num_4x4_Blocks_High[bSize];
    const av1g_frame_header& pf = fh.pf;
    for (int plane = 0; plane < NumPlanes; plane++) {
        if (pf.lr_type[plane] == 0) continue;
        int subX = plane ? ssx : 0, subY = plane ? ssy : 0;
        int unitSize = pf.lr_unit_size[plane];
        int unitRows = av1g_lr_units_in_frame(unitSize, (pf.frame_height + subY) >> subY);
        int unitCols = av1g_lr_units_in_frame(unitSize, (pf.upscaled_width + subX) >> subX);
        int unitRowStart = (r * (4 >> subY) + unitSize - 1) / unitSize;
        int unitRowEnd = std::min(unitRows, ((r + h) * (4 >> subY) + unitSize - 1) / unitSize);
        int numerator, denominator;
        if (pf.use_superres) {
            numerator = (4 >> subX) * fh.superres_denom;
            denominator = unitSize * 8;
        } else {
            numerator = 4 >> subX;
            denominator = unitSize;
        }
        int unitColStart = (c * numerator + denominator - 1) / denominator;
        int unitColEnd = std::min(unitCols, ((c + w) * numerator + denominator - 1) / denominator);
        for (int ur = unitRowStart; ur < unitRowEnd; ur++)
            for (int uc = unitColStart; uc < unitColEnd; uc++) {
                read_lr_unit(plane, ur, uc);
                (void)unitCols;
            }
    }
}

void Walker::read_lr_unit(int plane, int unitRow, int unitCol) {
    const av1g_frame_header& pf = fh.pf;
    int subX = plane ? ssx : 0;
    int unitCols = av1g_lr_units_in_frame(pf.lr_unit_size[plane], (pf.upscaled_width + subX) >> subX);
    av1g_lr_unit& u = out.lr_units[plane][(size_t)unitRow * unitCols + unitCol];
    int rtype;
    if (pf.lr_type[plane] == 1) rtype = S(cdf.use_wiener, 2) ? 1 : 0;
    else if (pf.lr_type[plane] == 2) rtype = S(cdf.use_sgrproj, 2) ? 2 : 0;
    else rtype = S(cdf.restoration_type, 3);
    u = av1g_lr_unit{};
    u.type = (uint8_t)rtype;
    if (rtype == 1) {
        for (int pass = 0; pass < 2; pass++) {
            int first = 0;
            if (plane) {
                first = 1;
                u.wiener[pass][0] = 0;
            }
            for (int j = first; j < 3; j++) {
                int v = subexp(Wiener_Taps_Min[j], Wiener_Taps_Max[j] + 1, Wiener_Taps_K[j], RefLrWiener[plane][pass][j]);
                u.wiener[pass][j] = (int8_t)v;
                RefLrWiener[plane][pass][j] = v;
            }
        }
    } else if (rtype == 2) {
        int set = L(4);
        u.sgr_set = (uint8_t)set;
        for (int i = 0; i < 2; i++) {
            int radius = Sgr_Radius[set][i];
            int mn = Sgrproj_Xqd_Min[i], mx = Sgrproj_Xqd_Max[i];
            int v;
            if (radius) {
                v = subexp(mn, mx + 1, 4, RefSgrXqd[plane][i]);
            } else {
                v = 0;
                if (i == 1) v = clip3(mn, mx, (1 << 7) - RefSgrXqd[plane][0]);
            }
            u.sgr_xqd[i] = (int16_t)v;
            RefSgrXqd[plane][i] = v;
        }
    }
}

void Walker::decode_partition(int r, int c, int bSize) {
    if (r >= MiRows || c >= MiCols) return;
    bool availU = is_inside(r - 1, c), availL = is_inside(r, c - 1);
    int num4x4 = Num_4x4_Blocks_Wide[bSize];
    int half = num4x4 >> 1, quarter = half >> 1;
    bool hasRows = (r + half) < MiRows, hasCols = (c + half) < MiCols;
    int partition;
    if (bSize < BLOCK_8X8) {
        partition = PARTITION_NONE;
    } else {
        int bsl = Mi_Width_Log2[bSize];
        int above = availU && (Mi_Width_Log2[MiSizes[cell(r - 1, c)]] < bsl);
        int left = availL && (Mi_Height_Log2[MiSizes[cell(r, c - 1)]] < bsl);
        int ctx = left * 2 + above;
        uint16_t* pc;
        int n;
        switch (bsl) {
            case 1: pc = cdf.partition_w8[ctx]; n = 4; break;
            case 2: pc = cdf.partition_w16[ctx]; n = 10; break;
            case 3: pc = cdf.partition_w32[ctx]; n = 10; break;
            case 4: pc = cdf.partition_w64[ctx]; n = 10; break;
            default: pc = cdf.partition_w128[ctx]; n = 8; break;
        }
        if (hasRows && hasCols) {
            partition = S(pc, n);
        } else if (hasCols) {
            // split_or_horz (cdf.rs:10950)
            int psum = pc[PARTITION_VERT] - pc[PARTITION_VERT - 1] + pc[PARTITION_SPLIT] - pc[PARTITION_SPLIT - 1] +
                       pc[PARTITION_HORZ_A] - pc[PARTITION_HORZ_A - 1] + pc[PARTITION_VERT_A] -
                       pc[PARTITION_VERT_A - 1] + pc[PARTITION_VERT_B] - pc[PARTITION_VERT_B - 1];
            if (bSize != BLOCK_128X128) psum += pc[PARTITION_VERT_4] - pc[PARTITION_VERT_4 - 1];
            psum = clip3(0, 32768, psum);
            uint16_t tmp[3] = {(uint16_t)(32768 - psum), 32768, 0};
            partition = S(tmp, 2) ? PARTITION_SPLIT : PARTITION_HORZ;
        } else if (hasRows) {
            int psum = pc[PARTITION_HORZ] - pc[PARTITION_HORZ - 1] + pc[PARTITION_SPLIT] - pc[PARTITION_SPLIT - 1] +
                       pc[PARTITION_HORZ_A] - pc[PARTITION_HORZ_A - 1] + pc[PARTITION_HORZ_B] -
                       pc[PARTITION_HORZ_B - 1] + pc[PARTITION_VERT_A] - pc[PARTITION_VERT_A - 1];
            if (bSize != BLOCK_128X128) psum += pc[PARTITION_HORZ_4] - pc[PARTITION_HORZ_4 - 1];
            psum = clip3(0, 32768, psum);
            uint16_t tmp[3] = {(uint16_t)(32768 - psum), 32768, 0};
            partition = S(tmp, 2) ? PARTITION_SPLIT : PARTITION_VERT;
        } else {
            partition = PARTITION_SPLIT;
        }
    }
    int subSize = Partition_Subsize[partition][bSize];
    int splitSize = Partition_Subsize[PARTITION_SPLIT][bSize];
    switch (partition) {
        case PARTITION_NONE: decode_block(r, c, subSize); break;
        case PARTITION_HORZ:
            decode_block(r, c, subSize);
            if (hasRows) decode_block(r + half, c, subSize);
            break;
        case PARTITION_VERT:
            decode_block(r, c, subSize);
            if (hasCols) decode_block(r, c + half, subSize);
            break;
        case PARTITION_SPLIT:
            decode_partition(r, c, subSize);
            decode_partition(r, c + half, subSize);
            decode_partition(r + half, c, subSize);
            decode_partition(r + half, c + half, subSize);
            break;
        case PARTITION_HORZ_A:
            decode_block(r, c, splitSize);
            decode_block(r, c + half, splitSize);
            decode_block(r + half, c, subSize);
            break;
        case PARTITION_HORZ_B:
            decode_block(r, c, subSize);
            decode_block(r + half, c, splitSize);
            decode_block(r + half, c + half, splitSize);
            break;
        case PARTITION_VERT_A:
            decode_block(r, c, splitSize);
            decode_block(r + half, c, splitSize);
            decode_block(r, c + half, subSize);
            break;
        case PARTITION_VERT_B:
            decode_block(r, c, subSize);
            decode_block(r, c + half, splitSize);
            decode_block(r + half, c + half, splitSize);
            break;
        case PARTITION_HORZ_4:
            for (int i = 0; i < 4; i++)
                if (i < 3 || r + quarter * 3 < MiRows) decode_block(r + quarter * i, c, subSize);
            break;
        default:
            for (int i = 0; i < 4; i++)
                if (i < 3 || c + quarter * 3 < MiCols) decode_block(r, c + quarter * i, subSize);
            break;
    }
}

// ===========================================================================
// decode_block
// ===========================================================================

void Walker::decode_block(int r, int c, int subSize) {
    if (subSize >= BLOCK_INVALID) throw WalkError("walker: invalid block size");
    MiRow = r;
    MiCol = c;
    MiSize = subSize;
    bw4 = Num_4x4_Blocks_Wide[subSize];
    bh4 = Num_4x4_Blocks_High[subSize];
    if (bh4 == 1 && ssy && (MiRow & 1) == 0) HasChroma = false;
    else if (bw4 == 1 && ssx && (MiCol & 1) == 0) HasChroma = false;
    else HasChroma = NumPlanes > 1;
    AvailU = is_inside(r - 1, c);
    AvailL = is_inside(r, c - 1);
    AvailUChroma = AvailU;
    AvailLChroma = AvailL;
    if (HasChroma) {
        if (ssy && bh4 == 1) AvailUChroma = is_inside(r - 2, c);
        if (ssx && bw4 == 1) AvailLChroma = is_inside(r, c - 2);
    } else {
        AvailUChroma = AvailLChroma = false;
    }
    // block defaults
    use_intrabc = 0;
    is_inter = 0;
    skip_mode = 0;
    skip = 0;
    motion_mode = SIMPLE;
    interintra = 0;
    compound_type = COMPOUND_AVERAGE;
    comp_group_idx = 0;
    compound_idx = 1;
    use_filter_intra = 0;
    AngleDeltaY = AngleDeltaUV = 0;
    CflAlphaU = CflAlphaV = 0;
    PaletteSizeY = PaletteSizeUV = 0;
    RefFrame[0] = INTRA_FRAME;
    RefFrame[1] = NONE_REF;
    Mv[0][0] = Mv[0][1] = Mv[1][0] = Mv[1][1] = 0;
    interp_filter[0] = interp_filter[1] = 0;
    LocalValid = 0;
    YMode = DC_PRED;
    UVMode = DC_PRED;

    if (FrameIsIntra) intra_frame_mode_info();
    else inter_frame_mode_info();
    palette_tokens();
    read_block_tx_size();
    if (skip) reset_block_context();
    store_block_grids();
    block_first_intra_tu = out.intra_tus.size();
    if (is_inter && !use_intrabc) emit_inter_block();
    residual();
}

void Walker::store_block_grids() {
    int isCompound = RefFrame[1] > INTRA_FRAME;
    int rEnd = std::min(MiRows, MiRow + bh4), cEnd = std::min(MiCols, MiCol + bw4);
    for (int y = MiRow; y < rEnd; y++)
        for (int x = MiCol; x < cEnd; x++) {
            size_t i = cell(y, x);
            YModes[i] = (uint8_t)YMode;
            if (RefFrame[0] == INTRA_FRAME && HasChroma) UVModes[i] = (uint8_t)UVMode;
            RefFrames[i * 2] = (int8_t)RefFrame[0];
            RefFrames[i * 2 + 1] = (int8_t)RefFrame[1];
            if (is_inter) {
                for (int l = 0; l < 1 + isCompound; l++) {
                    Mvs[i * 4 + l * 2] = (int16_t)Mv[l][0];
                    Mvs[i * 4 + l * 2 + 1] = (int16_t)Mv[l][1];
                }
            }
            InterpFilters[i * 2] = (uint8_t)interp_filter[0];
            InterpFilters[i * 2 + 1] = (uint8_t)interp_filter[1];
            IsInters[i] = (uint8_t)is_inter;
            SkipModes[i] = (uint8_t)skip_mode;
            Skips[i] = (uint8_t)skip;
            TxSizes[i] = (uint8_t)TxSize;
            MiSizes[i] = (uint8_t)MiSize;
            SegmentIds[i] = (uint8_t)segment_id;
            CompGroupIdxs[i] = (uint8_t)comp_group_idx;
            CompoundIdxs[i] = (uint8_t)compound_idx;
            PaletteSizes[0][i] = (uint8_t)PaletteSizeY;
            PaletteSizes[1][i] = (uint8_t)PaletteSizeUV;
            if (!PaletteColors[0].empty()) {
                for (int k = 0; k < PaletteSizeY; k++) PaletteColors[0][i * 8 + k] = palette_colors_y[k];
                for (int k = 0; k < PaletteSizeUV; k++) PaletteColors[1][i * 8 + k] = palette_colors_u[k];
            }
            for (int k = 0; k < 4; k++) DeltaLFs[i * 4 + k] = (int8_t)DeltaLF[k];
        }
}

// ---------------- intra frame mode info ----------------

void Walker::intra_frame_mode_info() {
    skip = 0;
    if (SegIdPreSkip) intra_segment_id();
    skip_mode = 0;
    read_skip();
    if (!SegIdPreSkip) intra_segment_id();
    read_cdef();
    read_delta_qindex();
    read_delta_lf();
    ReadDeltas = false;
    RefFrame[0] = INTRA_FRAME;
    RefFrame[1] = NONE_REF;
    use_intrabc = fh.pf.allow_intrabc ? S(cdf.intrabc, 2) : 0;
    if (use_intrabc) {
        is_inter = 1;
        motion_mode = SIMPLE;
        compound_type = COMPOUND_AVERAGE;
        PaletteSizeY = PaletteSizeUV = 0;
        interp_filter[0] = interp_filter[1] = BILINEAR;
        YMode = DC_PRED;
        UVMode = DC_PRED;
        find_mv_stack(0);
        assign_mv(0);
    } else {
        is_inter = 0;
        int above = AvailU ? (int)YModes[cell(MiRow - 1, MiCol)] : (int)DC_PRED;
        int left = AvailL ? (int)YModes[cell(MiRow, MiCol - 1)] : (int)DC_PRED;
        YMode = S(cdf.intra_frame_y_mode[Intra_Mode_Context[above]][Intra_Mode_Context[left]], 13);
        intra_angle_info_y();
        if (HasChroma) {
            read_uv_mode();
            if (UVMode == UV_CFL_PRED) read_cfl_alphas();
            intra_angle_info_uv();
        }
        PaletteSizeY = PaletteSizeUV = 0;
        if (MiSize >= BLOCK_8X8 && bw_of(MiSize) <= 64 && bh_of(MiSize) <= 64 && fh.allow_screen_content_tools)
            palette_mode_info();
        filter_intra_mode_info();
    }
}

void Walker::intra_segment_id() {
    if (fh.segmentation_enabled) read_segment_id();
    else segment_id = 0;
    Lossless = fh.lossless[segment_id];
}

void Walker::read_segment_id() {
    int prevUL = (AvailU && AvailL) ? SegmentIds[cell(MiRow - 1, MiCol - 1)] : -1;
    int prevU = AvailU ? SegmentIds[cell(MiRow - 1, MiCol)] : -1;
    int prevL = AvailL ? SegmentIds[cell(MiRow, MiCol - 1)] : -1;
    int pred;
    if (prevU == -1) pred = prevL == -1 ? 0 : prevL;
    else if (prevL == -1) pred = prevU;
    else pred = prevUL == prevU ? prevU : prevL;
    if (skip) {
        segment_id = pred;
        return;
    }
    int ctx;
    if (prevUL < 0) ctx = 0;
    else if (prevUL == prevU && prevUL == prevL) ctx = 2;
    else if (prevUL == prevU || prevUL == prevL || prevU == prevL) ctx = 1;
    else ctx = 0;
    int v = S(cdf.segment_id[ctx], 8);
    // neg_deinterleave(diff, ref, max)
    int max = LastActiveSegId + 1, ref = pred, diff = v, res;
    if (!ref) res = diff;
    else if (ref >= max - 1) res = max - diff - 1;
    else if (2 * ref < max) {
        if (diff <= 2 * ref) res = (diff & 1) ? ref + ((diff + 1) >> 1) : ref - (diff >> 1);
        else res = diff;
    } else {
        if (diff <= 2 * (max - ref - 1)) res = (diff & 1) ? ref + ((diff + 1) >> 1) : ref - (diff >> 1);
        else res = max - (diff + 1);
    }
    segment_id = clip3(0, LastActiveSegId, res);
}

int Walker::get_segment_id() {
    int xMis = std::min(MiCols - MiCol, bw4), yMis = std::min(MiRows - MiRow, bh4);
    int seg = 7;
    for (int y = 0; y < yMis; y++)
        for (int x = 0; x < xMis; x++) {
            int p = PrevSegmentIds ? PrevSegmentIds[cell(MiRow + y, MiCol + x)] : 0;
            seg = std::min(seg, p);
        }
    return seg;
}

void Walker::inter_segment_id(int preSkip) {
    if (!fh.segmentation_enabled) {
        segment_id = 0;
        return;
    }
    int predictedSegmentId = get_segment_id();
    if (fh.segmentation_update_map) {
        if (preSkip && !SegIdPreSkip) {
            segment_id = 0;
            return;
        }
        if (!preSkip) {
            if (skip) {
                for (int i = 0; i < bw4; i++) AboveSegPredContext[MiCol + i] = 0;
                for (int i = 0; i < bh4; i++) LeftSegPredContext[MiRow + i] = 0;
                read_segment_id();
                return;
            }
        }
        if (fh.segmentation_temporal_update == 1) {
            int ctx = LeftSegPredContext[MiRow] + AboveSegPredContext[MiCol];
            int pred = S(cdf.segment_id_predicted[ctx], 2);
            if (pred) segment_id = predictedSegmentId;
            else read_segment_id();
            for (int i = 0; i < bw4; i++) AboveSegPredContext[MiCol + i] = (uint8_t)pred;
            for (int i = 0; i < bh4; i++) LeftSegPredContext[MiRow + i] = (uint8_t)pred;
        } else {
            read_segment_id();
        }
    } else {
        segment_id = predictedSegmentId;
    }
}

void Walker::read_skip_mode() {
    if (seg_feature_active(SEG_LVL_SKIP) || seg_feature_active(SEG_LVL_REF_FRAME) ||
        seg_feature_active(SEG_LVL_GLOBALMV) || !fh.skip_mode_present || bw_of(MiSize) < 8 || bh_of(MiSize) < 8) {
        skip_mode = 0;
        return;
    }
    int ctx = (AvailU ? SkipModes[cell(MiRow - 1, MiCol)] : 0) + (AvailL ? SkipModes[cell(MiRow, MiCol - 1)] : 0);
    skip_mode = S(cdf.skip_mode[ctx], 2);
}

void Walker::read_skip() {
    if (SegIdPreSkip && seg_feature_active(SEG_LVL_SKIP)) {
        skip = 1;
        return;
    }
    int ctx = (AvailU ? Skips[cell(MiRow - 1, MiCol)] : 0) + (AvailL ? Skips[cell(MiRow, MiCol - 1)] : 0);
    skip = S(cdf.skip[ctx], 2);
}

void Walker::read_cdef() {
    if (skip || CodedLossless || !seq.enable_cdef || fh.pf.allow_intrabc) return;
    int r = MiRow & ~15, c = MiCol & ~15;
    int c64c = (MiCols + 15) >> 4;
    int8_t& idx = out.cdef_idx[(size_t)(r >> 4) * c64c + (c >> 4)];
    if (idx == -1) {
        int v = L(fh.pf.cdef_bits);
        int w4 = bw4, h4 = bh4;
        for (int y = r; y < r + h4; y += 16)
            for (int x = c; x < c + w4; x += 16)
                if (y < MiRows && x < MiCols) out.cdef_idx[(size_t)(y >> 4) * c64c + (x >> 4)] = (int8_t)v;
    }
}

void Walker::read_delta_qindex() {
    int sbSize = sb128 ? BLOCK_128X128 : BLOCK_64X64;
    if (MiSize == sbSize && skip) return;
    if (!ReadDeltas) return;
    int a = S(cdf.delta_q, 4);
    if (a == 3) {
        int rem = L(3) + 1;
        int bits = L(rem);
        a = bits + (1 << rem) + 1;
    }
    if (a) {
        int sign = L(1);
        int red = sign ? -a : a;
        CurrentQIndex = clip3(1, 255, CurrentQIndex + red * (1 << fh.delta_q_res));
    }
}

void Walker::read_delta_lf() {
    int sbSize = sb128 ? BLOCK_128X128 : BLOCK_64X64;
    if (MiSize == sbSize && skip) return;
    if (!ReadDeltas || !fh.delta_lf_present) return;
    int cnt = 1;
    if (fh.pf.delta_lf_multi) cnt = NumPlanes > 1 ? 4 : 2;
    for (int i = 0; i < cnt; i++) {
        uint16_t* c = fh.pf.delta_lf_multi ? cdf.delta_lf_multi[i] : cdf.delta_lf;
        int a = S(c, 4);
        if (a == 3) {
            int n = L(3) + 1;
            int bits = L(n);
            a = bits + (1 << n) + 1;
        }
        if (a) {
            int sign = L(1);
            int red = sign ? -a : a;
            DeltaLF[i] = clip3(-63, 63, DeltaLF[i] + red * (1 << fh.delta_lf_res));
        }
    }
}

void Walker::intra_angle_info_y() {
    AngleDeltaY = 0;
    if (MiSize >= BLOCK_8X8 && YMode >= V_PRED && YMode <= D67_PRED)
        AngleDeltaY = S(cdf.angle_delta[YMode - V_PRED], 7) - 3;
}

void Walker::intra_angle_info_uv() {
    AngleDeltaUV = 0;
    if (MiSize >= BLOCK_8X8 && UVMode >= V_PRED && UVMode <= D67_PRED)
        AngleDeltaUV = S(cdf.angle_delta[UVMode - V_PRED], 7) - 3;
}

void Walker::read_uv_mode() {
    bool cflAllowed;
    if (Lossless && plane_residual_size(MiSize, 1) == BLOCK_4X4) cflAllowed = true;
    else if (!Lossless && std::max(bw_of(MiSize), bh_of(MiSize)) <= 32) cflAllowed = true;
    else cflAllowed = false;
    if (cflAllowed) UVMode = S(cdf.uv_mode_cfl_allowed[YMode], 14);
    else UVMode = S(cdf.uv_mode_cfl_not_allowed[YMode], 13);
}

void Walker::read_cfl_alphas() {
    int signs = S(cdf.cfl_sign, 8);
    int signU = (signs + 1) / 3, signV = (signs + 1) % 3;
    if (signU) {
        int a = S(cdf.cfl_alpha[(signU - 1) * 3 + signV], 16);
        CflAlphaU = 1 + a;
        if (signU == 1) CflAlphaU = -CflAlphaU;
    } else {
        CflAlphaU = 0;
    }
    if (signV) {
        int a = S(cdf.cfl_alpha[(signV - 1) * 3 + signU], 16);
        CflAlphaV = 1 + a;
        if (signV == 1) CflAlphaV = -CflAlphaV;
    } else {
        CflAlphaV = 0;
    }
}

int Walker::get_palette_cache(int plane, uint16_t* cache) {
    int aboveN = 0, leftN = 0;
    if (((MiRow * 4) % 64) && AvailU) aboveN = PaletteSizes[plane][cell(MiRow - 1, MiCol)];
    if (AvailL) leftN = PaletteSizes[plane][cell(MiRow, MiCol - 1)];
    const uint16_t* ac = aboveN ? &PaletteColors[plane][cell(MiRow - 1, MiCol) * 8] : nullptr;
    const uint16_t* lc = leftN ? &PaletteColors[plane][cell(MiRow, MiCol - 1) * 8] : nullptr;
    int ai = 0, li = 0, n = 0;
    while (ai < aboveN && li < leftN) {
        int aboveC = ac[ai], leftC = lc[li];
        if (leftC < aboveC) {
            if (n == 0 || leftC != cache[n - 1]) cache[n++] = (uint16_t)leftC;
            li++;
        } else {
            if (n == 0 || aboveC != cache[n - 1]) cache[n++] = (uint16_t)aboveC;
            ai++;
            if (leftC == aboveC) li++;
        }
    }
    while (ai < aboveN) {
        int v = ac[ai++];
        if (n == 0 || v != cache[n - 1]) cache[n++] = (uint16_t)v;
    }
    while (li < leftN) {
        int v = lc[li++];
        if (n == 0 || v != cache[n - 1]) cache[n++] = (uint16_t)v;
    }
    return n;
}

void Walker::palette_mode_info() {
    int bsizeCtx = Mi_Width_Log2[MiSize] + Mi_Height_Log2[MiSize] - 2;
    int maxv = (1 << BitDepth) - 1;
    if (YMode == DC_PRED) {
        int ctx = 0;
        if (AvailU && PaletteSizes[0][cell(MiRow - 1, MiCol)] > 0) ctx++;
        if (AvailL && PaletteSizes[0][cell(MiRow, MiCol - 1)] > 0) ctx++;
        if (S(cdf.palette_y_mode[bsizeCtx][ctx], 2)) {
            PaletteSizeY = S(cdf.palette_y_size[bsizeCtx], 7) + 2;
            uint16_t cache[16];
            int cacheN = get_palette_cache(0, cache);
            int idx = 0;
            for (int i = 0; i < cacheN && idx < PaletteSizeY; i++)
                if (L(1)) palette_colors_y[idx++] = cache[i];
            if (idx < PaletteSizeY) palette_colors_y[idx++] = (uint16_t)L(BitDepth);
            int paletteBits = 0;
            if (idx < PaletteSizeY) paletteBits = BitDepth - 3 + L(2);
            while (idx < PaletteSizeY) {
                int d = L(paletteBits) + 1;
                palette_colors_y[idx] = (uint16_t)std::min(maxv, palette_colors_y[idx - 1] + d);
                int range = (1 << BitDepth) - palette_colors_y[idx] - 1;
                paletteBits = std::min(paletteBits, ceil_log2(range));
                idx++;
            }
            std::sort(palette_colors_y, palette_colors_y + PaletteSizeY);
        }
    }
    if (HasChroma && UVMode == DC_PRED) {
        int ctx = PaletteSizeY > 0 ? 1 : 0;
        if (S(cdf.palette_uv_mode[ctx], 2)) {
            PaletteSizeUV = S(cdf.palette_uv_size[bsizeCtx], 7) + 2;
            uint16_t cache[16];
            int cacheN = get_palette_cache(1, cache);
            int idx = 0;
            for (int i = 0; i < cacheN && idx < PaletteSizeUV; i++)
                if (L(1)) palette_colors_u[idx++] = cache[i];
            if (idx < PaletteSizeUV) palette_colors_u[idx++] = (uint16_t)L(BitDepth);
            int paletteBits = 0;
            if (idx < PaletteSizeUV) paletteBits = BitDepth - 3 + L(2);
            while (idx < PaletteSizeUV) {
                int d = L(paletteBits);
                palette_colors_u[idx] = (uint16_t)std::min(maxv, palette_colors_u[idx - 1] + d);
                int range = (1 << BitDepth) - palette_colors_u[idx];
                paletteBits = std::min(paletteBits, ceil_log2(range));
                idx++;
            }
            std::sort(palette_colors_u, palette_colors_u + PaletteSizeUV);
            if (L(1)) {
                int minBits = BitDepth - 4;
                int maxVal = 1 << BitDepth;
                int bits = minBits + L(2);
                palette_colors_v[0] = (uint16_t)L(BitDepth);
                for (int i = 1; i < PaletteSizeUV; i++) {
                    int d = L(bits);
                    if (d && L(1)) d = -d;
                    int val = palette_colors_v[i - 1] + d;
                    if (val < 0) val += maxVal;
                    if (val >= maxVal) val -= maxVal;
                    palette_colors_v[i] = (uint16_t)clip3(0, maxv, val);
                }
            } else {
                for (int i = 0; i < PaletteSizeUV; i++) palette_colors_v[i] = (uint16_t)L(BitDepth);
            }
        }
    }
}

void Walker::filter_intra_mode_info() {
    use_filter_intra = 0;
    if (seq.enable_filter_intra && YMode == DC_PRED && PaletteSizeY == 0 &&
        std::max(bw_of(MiSize), bh_of(MiSize)) <= 32) {
        use_filter_intra = S(cdf.filter_intra[MiSize], 2);
        if (use_filter_intra) filter_intra_mode = S(cdf.filter_intra_mode, 5);
    }
}

// ---------------- inter frame mode info ----------------

void Walker::inter_frame_mode_info() {
    use_intrabc = 0;
    LeftRefFrame[0] = AvailL ? (int)RefFrames[cell(MiRow, MiCol - 1) * 2] : (int)INTRA_FRAME;
    AboveRefFrame[0] = AvailU ? (int)RefFrames[cell(MiRow - 1, MiCol) * 2] : (int)INTRA_FRAME;
    LeftRefFrame[1] = AvailL ? RefFrames[cell(MiRow, MiCol - 1) * 2 + 1] : NONE_REF;
    AboveRefFrame[1] = AvailU ? RefFrames[cell(MiRow - 1, MiCol) * 2 + 1] : NONE_REF;
    LeftIntra = LeftRefFrame[0] <= INTRA_FRAME;
    AboveIntra = AboveRefFrame[0] <= INTRA_FRAME;
    LeftSingle = LeftRefFrame[1] <= INTRA_FRAME;
    AboveSingle = AboveRefFrame[1] <= INTRA_FRAME;
    skip = 0;
    inter_segment_id(1);
    read_skip_mode();
    if (skip_mode) skip = 1;
    else read_skip();
    if (!SegIdPreSkip) inter_segment_id(0);
    Lossless = fh.lossless[segment_id];
    read_cdef();
    read_delta_qindex();
    read_delta_lf();
    ReadDeltas = false;
    read_is_inter();
    if (is_inter) inter_block_mode_info();
    else intra_block_mode_info();
}

void Walker::read_is_inter() {
    if (skip_mode) is_inter = 1;
    else if (seg_feature_active(SEG_LVL_REF_FRAME))
        is_inter = fh.seg_feature_data[segment_id][SEG_LVL_REF_FRAME] != INTRA_FRAME;
    else if (seg_feature_active(SEG_LVL_GLOBALMV)) is_inter = 1;
    else {
        int ctx;
        if (AvailU && AvailL) ctx = (LeftIntra && AboveIntra) ? 3 : (LeftIntra || AboveIntra);
        else if (AvailU || AvailL) ctx = 2 * (AvailU ? AboveIntra : LeftIntra);
        else ctx = 0;
        is_inter = S(cdf.is_inter[ctx], 2);
    }
}

void Walker::intra_block_mode_info() {
    RefFrame[0] = INTRA_FRAME;
    RefFrame[1] = NONE_REF;
    YMode = S(cdf.y_mode[Size_Group[MiSize]], 13);
    intra_angle_info_y();
    if (HasChroma) {
        read_uv_mode();
        if (UVMode == UV_CFL_PRED) read_cfl_alphas();
        intra_angle_info_uv();
    }
    PaletteSizeY = PaletteSizeUV = 0;
    if (MiSize >= BLOCK_8X8 && bw_of(MiSize) <= 64 && bh_of(MiSize) <= 64 && fh.allow_screen_content_tools)
        palette_mode_info();
    filter_intra_mode_info();
}

int Walker::count_refs(int frameType) {
    int c = 0;
    if (AvailU) {
        if (AboveRefFrame[0] == frameType) c++;
        if (AboveRefFrame[1] == frameType) c++;
    }
    if (AvailL) {
        if (LeftRefFrame[0] == frameType) c++;
        if (LeftRefFrame[1] == frameType) c++;
    }
    return c;
}

static int ref_count_ctx(int c0, int c1) { return c0 < c1 ? 0 : c0 == c1 ? 1 : 2; }
static bool check_backward(int r) { return r >= BWDREF_FRAME && r <= ALTREF_FRAME; }

void Walker::read_ref_frames() {
    if (skip_mode) {
        RefFrame[0] = fh.skip_mode_frame[0];
        RefFrame[1] = fh.skip_mode_frame[1];
        return;
    }
    if (seg_feature_active(SEG_LVL_REF_FRAME)) {
        RefFrame[0] = fh.seg_feature_data[segment_id][SEG_LVL_REF_FRAME];
        RefFrame[1] = NONE_REF;
        return;
    }
    if (seg_feature_active(SEG_LVL_SKIP) || seg_feature_active(SEG_LVL_GLOBALMV)) {
        RefFrame[0] = LAST_FRAME;
        RefFrame[1] = NONE_REF;
        return;
    }
    int comp_mode = 0;
    if (fh.reference_select && std::min(bw4, bh4) >= 2) {
        int ctx;
        if (AvailU && AvailL) {
            if (AboveSingle && LeftSingle) ctx = check_backward(AboveRefFrame[0]) ^ check_backward(LeftRefFrame[0]);
            else if (AboveSingle) ctx = 2 + (check_backward(AboveRefFrame[0]) || AboveIntra);
            else if (LeftSingle) ctx = 2 + (check_backward(LeftRefFrame[0]) || LeftIntra);
            else ctx = 4;
        } else if (AvailU) {
            ctx = AboveSingle ? check_backward(AboveRefFrame[0]) : 3;
        } else if (AvailL) {
            ctx = LeftSingle ? check_backward(LeftRefFrame[0]) : 3;
        } else {
            ctx = 1;
        }
        comp_mode = S(cdf.comp_mode[ctx], 2);
    }
    int fwdCount = count_refs(LAST_FRAME) + count_refs(LAST2_FRAME) + count_refs(LAST3_FRAME) +
                   count_refs(GOLDEN_FRAME);
    int bwdCount = count_refs(BWDREF_FRAME) + count_refs(ALTREF2_FRAME) + count_refs(ALTREF_FRAME);
    int ctxLast12vs3G = ref_count_ctx(count_refs(LAST_FRAME) + count_refs(LAST2_FRAME),
                                      count_refs(LAST3_FRAME) + count_refs(GOLDEN_FRAME));
    int ctxLastVsLast2 = ref_count_ctx(count_refs(LAST_FRAME), count_refs(LAST2_FRAME));
    int ctxLast3VsGold = ref_count_ctx(count_refs(LAST3_FRAME), count_refs(GOLDEN_FRAME));
    int ctxBrfArf2VsArf = ref_count_ctx(count_refs(BWDREF_FRAME) + count_refs(ALTREF2_FRAME),
                                        count_refs(ALTREF_FRAME));
    int ctxBrfVsArf2 = ref_count_ctx(count_refs(BWDREF_FRAME), count_refs(ALTREF2_FRAME));
    if (comp_mode) {
        // comp_ref_type context (§8.3.2)
        int above0 = AboveRefFrame[0], above1 = AboveRefFrame[1], left0 = LeftRefFrame[0], left1 = LeftRefFrame[1];
        auto samedir = [](int a, int b) { return (a >= BWDREF_FRAME) == (b >= BWDREF_FRAME); };
        bool aboveCompInter = AvailU && !AboveIntra && !AboveSingle;
        bool leftCompInter = AvailL && !LeftIntra && !LeftSingle;
        bool aboveUniComp = aboveCompInter && samedir(above0, above1);
        bool leftUniComp = leftCompInter && samedir(left0, left1);
        int ctx;
        if (AvailU && !AboveIntra && AvailL && !LeftIntra) {
            int sd = samedir(above0, left0);
            if (!aboveCompInter && !leftCompInter) ctx = 1 + 2 * sd;
            else if (!aboveCompInter) ctx = !leftUniComp ? 1 : 3 + sd;
            else if (!leftCompInter) ctx = !aboveUniComp ? 1 : 3 + sd;
            else {
                if (!aboveUniComp && !leftUniComp) ctx = 0;
                else if (!aboveUniComp || !leftUniComp) ctx = 2;
                else ctx = 3 + ((above0 == BWDREF_FRAME) == (left0 == BWDREF_FRAME));
            }
        } else if (AvailU && AvailL) {
            if (aboveCompInter) ctx = 1 + 2 * aboveUniComp;
            else if (leftCompInter) ctx = 1 + 2 * leftUniComp;
            else ctx = 2;
        } else if (aboveCompInter) {
            ctx = 4 * aboveUniComp;
        } else if (leftCompInter) {
            ctx = 4 * leftUniComp;
        } else {
            ctx = 2;
        }
        int comp_ref_type = S(cdf.comp_ref_type[ctx], 2);
        if (comp_ref_type == 0) {  // UNIDIR_COMP_REFERENCE
            int c0 = ref_count_ctx(fwdCount, bwdCount);
            if (S(cdf.uni_comp_ref[c0][0], 2)) {
                RefFrame[0] = BWDREF_FRAME;
                RefFrame[1] = ALTREF_FRAME;
            } else {
                int c1 = ref_count_ctx(count_refs(LAST2_FRAME), count_refs(LAST3_FRAME) + count_refs(GOLDEN_FRAME));
                if (S(cdf.uni_comp_ref[c1][1], 2)) {
                    int c2 = ctxLast3VsGold;
                    RefFrame[0] = LAST_FRAME;
                    RefFrame[1] = S(cdf.uni_comp_ref[c2][2], 2) ? GOLDEN_FRAME : LAST3_FRAME;
                } else {
                    RefFrame[0] = LAST_FRAME;
                    RefFrame[1] = LAST2_FRAME;
                }
            }
        } else {
            if (S(cdf.comp_ref[ctxLast12vs3G][0], 2) == 0)
                RefFrame[0] = S(cdf.comp_ref[ctxLastVsLast2][1], 2) ? LAST2_FRAME : LAST_FRAME;
            else
                RefFrame[0] = S(cdf.comp_ref[ctxLast3VsGold][2], 2) ? GOLDEN_FRAME : LAST3_FRAME;
            if (S(cdf.comp_bwd_ref[ctxBrfArf2VsArf][0], 2) == 0)
                RefFrame[1] = S(cdf.comp_bwd_ref[ctxBrfVsArf2][1], 2) ? ALTREF2_FRAME : BWDREF_FRAME;
            else
                RefFrame[1] = ALTREF_FRAME;
        }
    } else {
        if (S(cdf.single_ref[ref_count_ctx(fwdCount, bwdCount)][0], 2)) {
            if (S(cdf.single_ref[ctxBrfArf2VsArf][1], 2) == 0)
                RefFrame[0] = S(cdf.single_ref[ctxBrfVsArf2][5], 2) ? ALTREF2_FRAME : BWDREF_FRAME;
            else
                RefFrame[0] = ALTREF_FRAME;
        } else {
            if (S(cdf.single_ref[ctxLast12vs3G][2], 2))
                RefFrame[0] = S(cdf.single_ref[ctxLast3VsGold][4], 2) ? GOLDEN_FRAME : LAST3_FRAME;
            else
                RefFrame[0] = S(cdf.single_ref[ctxLastVsLast2][3], 2) ? LAST2_FRAME : LAST_FRAME;
        }
        RefFrame[1] = NONE_REF;
    }
}

int Walker::get_mode(int refList) {
    int compMode;
    if (refList == 0) {
        if (YMode < NEAREST_NEARESTMV) compMode = YMode;
        else if (YMode == NEW_NEWMV || YMode == NEW_NEARESTMV || YMode == NEW_NEARMV) compMode = NEWMV;
        else if (YMode == NEAREST_NEARESTMV || YMode == NEAREST_NEWMV) compMode = NEARESTMV;
        else if (YMode == NEAR_NEARMV || YMode == NEAR_NEWMV) compMode = NEARMV;
        else compMode = GLOBALMV;
    } else {
        if (YMode == NEW_NEWMV || YMode == NEAREST_NEWMV || YMode == NEAR_NEWMV) compMode = NEWMV;
        else if (YMode == NEAREST_NEARESTMV || YMode == NEW_NEARESTMV) compMode = NEARESTMV;
        else if (YMode == NEAR_NEARMV || YMode == NEW_NEARMV) compMode = NEARMV;
        else compMode = GLOBALMV;
    }
    return compMode;
}

void Walker::inter_block_mode_info() {
    PaletteSizeY = PaletteSizeUV = 0;
    read_ref_frames();
    int isCompound = RefFrame[1] > INTRA_FRAME;
    find_mv_stack(isCompound);
    if (skip_mode) {
        YMode = NEAREST_NEARESTMV;
    } else if (seg_feature_active(SEG_LVL_SKIP) || seg_feature_active(SEG_LVL_GLOBALMV)) {
        YMode = GLOBALMV;
    } else if (isCompound) {
        int ctx = Compound_Mode_Ctx_Map[RefMvContext >> 1][std::min(NewMvContext, 4)];
        YMode = NEAREST_NEARESTMV + S(cdf.compound_mode[ctx], 8);
    } else {
        if (S(cdf.new_mv[NewMvContext], 2) == 0) {
            YMode = NEWMV;
        } else if (S(cdf.zero_mv[ZeroMvContext], 2) == 0) {
            YMode = GLOBALMV;
        } else {
            YMode = S(cdf.ref_mv[RefMvContext], 2) == 0 ? NEARESTMV : NEARMV;
        }
    }
    RefMvIdx = 0;
    bool hasNear = YMode == NEARMV || YMode == NEAR_NEARMV || YMode == NEAR_NEWMV || YMode == NEW_NEARMV;
    if (YMode == NEWMV || YMode == NEW_NEWMV) {
        for (int idx = 0; idx < 2; idx++) {
            if (NumMvFound > idx + 1) {
                int d = S(cdf.drl_mode[DrlCtxStack[idx]], 2);
                if (d == 0) {
                    RefMvIdx = idx;
                    break;
                }
                RefMvIdx = idx + 1;
            }
        }
    } else if (hasNear) {
        RefMvIdx = 1;
        for (int idx = 1; idx < 3; idx++) {
            if (NumMvFound > idx + 1) {
                int d = S(cdf.drl_mode[DrlCtxStack[idx]], 2);
                if (d == 0) {
                    RefMvIdx = idx;
                    break;
                }
                RefMvIdx = idx + 1;
            }
        }
    }
    assign_mv(isCompound);
    read_interintra_mode(isCompound);
    read_motion_mode(isCompound);
    read_compound_type(isCompound);
    if (fh.interpolation_filter == SWITCHABLE) {
        for (int dir = 0; dir < (seq.enable_dual_filter ? 2 : 1); dir++) {
            if (needs_interp_filter()) interp_filter[dir] = S(cdf.interp_filter[interp_filter_ctx(dir)], 3);
            else interp_filter[dir] = 0;
        }
        if (!seq.enable_dual_filter) interp_filter[1] = interp_filter[0];
    } else {
        interp_filter[0] = interp_filter[1] = fh.interpolation_filter;
    }
}

bool Walker::needs_interp_filter() {
    bool large = std::min(bw_of(MiSize), bh_of(MiSize)) >= 8;
    if (skip_mode || motion_mode == LOCALWARP) return false;
    if (large && YMode == GLOBALMV) return fh.gm_type[RefFrame[0]] == TRANSLATION;
    if (large && YMode == GLOBAL_GLOBALMV)
        return fh.gm_type[RefFrame[0]] == TRANSLATION || fh.gm_type[RefFrame[1]] == TRANSLATION;
    return true;
}

int Walker::interp_filter_ctx(int dir) {
    int ctx = ((dir & 1) * 2 + (RefFrame[1] > INTRA_FRAME)) * 4;
    int leftType = 3, aboveType = 3;
    if (AvailL) {
        size_t i = cell(MiRow, MiCol - 1);
        if (RefFrames[i * 2] == RefFrame[0] || RefFrames[i * 2 + 1] == RefFrame[0])
            leftType = InterpFilters[i * 2 + dir];
    }
    if (AvailU) {
        size_t i = cell(MiRow - 1, MiCol);
        if (RefFrames[i * 2] == RefFrame[0] || RefFrames[i * 2 + 1] == RefFrame[0])
            aboveType = InterpFilters[i * 2 + dir];
    }
    if (leftType == aboveType) ctx += leftType;
    else if (leftType == 3) ctx += aboveType;
    else if (aboveType == 3) ctx += leftType;
    else ctx += 3;
    return ctx;
}

void Walker::assign_mv(int isCompound) {
    for (int i = 0; i < 1 + isCompound; i++) {
        int compMode = use_intrabc ? NEWMV : get_mode(i);
        if (use_intrabc) {
            PredMv[0][0] = RefStackMv[0][0][0];
            PredMv[0][1] = RefStackMv[0][0][1];
            if (PredMv[0][0] == 0 && PredMv[0][1] == 0) {
                PredMv[0][0] = RefStackMv[1][0][0];
                PredMv[0][1] = RefStackMv[1][0][1];
            }
            if (PredMv[0][0] == 0 && PredMv[0][1] == 0) {
                int sbSize4 = sb128 ? 32 : 16;
                if (MiRow - sbSize4 < MiRowStart) {
                    PredMv[0][0] = 0;
                    PredMv[0][1] = -(sbSize4 * 4 + 256) * 8;
                } else {
                    PredMv[0][0] = -(sbSize4 * 4 * 8);
                    PredMv[0][1] = 0;
                }
            }
        } else if (compMode == GLOBALMV) {
            PredMv[i][0] = GlobalMvs[i][0];
            PredMv[i][1] = GlobalMvs[i][1];
        } else {
            int pos = compMode == NEARESTMV ? 0 : RefMvIdx;
            if (compMode == NEWMV && NumMvFound <= 1) pos = 0;
            PredMv[i][0] = RefStackMv[pos][i][0];
            PredMv[i][1] = RefStackMv[pos][i][1];
        }
        if (compMode == NEWMV) {
            read_mv(i);
        } else {
            Mv[i][0] = PredMv[i][0];
            Mv[i][1] = PredMv[i][1];
        }
    }
}

void Walker::read_mv(int ref) {
    int diff[2] = {0, 0};
    int ctx = use_intrabc ? 1 : 0;
    int joint = S(cdf.mv_joint[ctx], 4);
    if (joint == 2 || joint == 3) diff[0] = read_mv_component(ctx, 0);
    if (joint == 1 || joint == 3) diff[1] = read_mv_component(ctx, 1);
    Mv[ref][0] = PredMv[ref][0] + diff[0];
    Mv[ref][1] = PredMv[ref][1] + diff[1];
}

int Walker::read_mv_component(int ctx, int comp) {
    int sign = S(cdf.mv_sign[ctx][comp], 2);
    int cls = S(cdf.mv_class[ctx][comp], 11);
    int mag;
    if (cls == 0) {
        int b = S(cdf.mv_class0_bit[ctx][comp], 2);
        int fr = fh.force_integer_mv ? 3 : S(cdf.mv_class0_fr[ctx][comp][b], 4);
        int hp = fh.allow_high_precision_mv ? S(cdf.mv_class0_hp[ctx][comp], 2) : 1;
        mag = ((b << 3) | (fr << 1) | hp) + 1;
    } else {
        int d = 0;
        for (int i = 0; i < cls; i++) d |= S(cdf.mv_bit[ctx][comp][i], 2) << i;
        mag = 2 << (cls + 2);
        int fr = fh.force_integer_mv ? 3 : S(cdf.mv_fr[ctx][comp], 4);
        int hp = fh.allow_high_precision_mv ? S(cdf.mv_hp[ctx][comp], 2) : 1;
        mag += ((d << 3) | (fr << 1) | hp) + 1;
    }
    return sign ? -mag : mag;
}

bool Walker::has_overlappable_candidates() {
    if (AvailU) {
        for (int x4 = MiCol; x4 < std::min(MiCols, MiCol + bw4); x4 += 2) {
            int x5 = x4 | 1;
            if (x5 >= MiCols) x5 = MiCols - 1;
            if (RefFrames[cell(MiRow - 1, x5) * 2] > INTRA_FRAME) return true;
        }
    }
    if (AvailL) {
        for (int y4 = MiRow; y4 < std::min(MiRows, MiRow + bh4); y4 += 2) {
            int y5 = y4 | 1;
            if (y5 >= MiRows) y5 = MiRows - 1;
            if (RefFrames[cell(y5, MiCol - 1) * 2] > INTRA_FRAME) return true;
        }
    }
    return false;
}

void Walker::read_motion_mode(int isCompound) {
    motion_mode = SIMPLE;
    if (skip_mode) return;
    if (!fh.is_motion_mode_switchable) return;
    if (std::min(bw_of(MiSize), bh_of(MiSize)) < 8) return;
    if (!fh.force_integer_mv && (YMode == GLOBALMV || YMode == GLOBAL_GLOBALMV)) {
        if (fh.gm_type[RefFrame[0]] > TRANSLATION) return;
    }
    if (isCompound || RefFrame[1] == INTRA_FRAME || !has_overlappable_candidates()) return;
    find_warp_samples();
    if (fh.force_integer_mv || NumSamples == 0 || !fh.allow_warped_motion || IsScaled[RefFrame[0]]) {
        motion_mode = S(cdf.use_obmc[MiSize], 2) ? OBMC : SIMPLE;
    } else {
        motion_mode = S(cdf.motion_mode[MiSize], 3);
    }
    if (motion_mode == LOCALWARP) {
        uint8_t valid = 0;
        if (av1g_warp_estimation(CandList, NumSamples, MiRow, MiCol, bw4, bh4, (int16_t)Mv[0][0],
                                 (int16_t)Mv[0][1], LocalWarpParams, &valid) != AV1G_OK)
            throw WalkError("walker: warp estimation rejected its samples");
        LocalValid = valid;
    }
}

void Walker::read_interintra_mode(int isCompound) {
    interintra = 0;
    if (!skip_mode && seq.enable_interintra_compound && !isCompound && MiSize >= BLOCK_8X8 &&
        MiSize <= BLOCK_32X32) {
        int ctx = Size_Group[MiSize] - 1;
        interintra = S(cdf.inter_intra[ctx], 2);
        if (interintra) {
            interintra_mode = S(cdf.inter_intra_mode[ctx], 4);
            RefFrame[1] = INTRA_FRAME;
            AngleDeltaY = AngleDeltaUV = 0;
            use_filter_intra = 0;
            wedge_interintra = S(cdf.wedge_inter_intra[MiSize], 2);
            if (wedge_interintra) {
                wedge_index = S(cdf.wedge_index[MiSize], 16);
                wedge_sign = 0;
            }
        }
    }
}

void Walker::read_compound_type(int isCompound) {
    comp_group_idx = 0;
    compound_idx = 1;
    if (skip_mode) {
        compound_type = COMPOUND_AVERAGE;
        return;
    }
    if (isCompound) {
        int n = Wedge_Bits[MiSize];
        if (seq.enable_masked_compound) {
            int ctx = 0;
            if (AvailU) {
                if (!AboveSingle) ctx += CompGroupIdxs[cell(MiRow - 1, MiCol)];
                else if (AboveRefFrame[0] == ALTREF_FRAME) ctx += 3;
            }
            if (AvailL) {
                if (!LeftSingle) ctx += CompGroupIdxs[cell(MiRow, MiCol - 1)];
                else if (LeftRefFrame[0] == ALTREF_FRAME) ctx += 3;
            }
            comp_group_idx = S(cdf.comp_group_idx[std::min(5, ctx)], 2);
        }
        if (comp_group_idx == 0) {
            if (seq.enable_jnt_comp) {
                int fwd = std::abs(get_relative_dist(fh.order_hints[RefFrame[0]], fh.order_hint, OrderHintBits));
                int bck = std::abs(get_relative_dist(fh.order_hints[RefFrame[1]], fh.order_hint, OrderHintBits));
                int ctx = fwd == bck ? 3 : 0;
                if (AvailU) {
                    if (!AboveSingle) ctx += CompoundIdxs[cell(MiRow - 1, MiCol)];
                    else if (AboveRefFrame[0] == ALTREF_FRAME) ctx++;
                }
                if (AvailL) {
                    if (!LeftSingle) ctx += CompoundIdxs[cell(MiRow, MiCol - 1)];
                    else if (LeftRefFrame[0] == ALTREF_FRAME) ctx++;
                }
                compound_idx = S(cdf.compound_idx[ctx], 2);
                compound_type = compound_idx ? COMPOUND_AVERAGE : COMPOUND_DISTANCE;
            } else {
                compound_type = COMPOUND_AVERAGE;
            }
        } else {
            if (n == 0) compound_type = COMPOUND_DIFFWTD;
            else compound_type = S(cdf.compound_type[MiSize], 2);
        }
        if (compound_type == COMPOUND_WEDGE) {
            wedge_index = S(cdf.wedge_index[MiSize], 16);
            wedge_sign = L(1);
        } else if (compound_type == COMPOUND_DIFFWTD) {
            mask_type = L(1);
        }
    } else {
        if (interintra) compound_type = wedge_interintra ? COMPOUND_WEDGE : COMPOUND_INTRA;
        else compound_type = COMPOUND_AVERAGE;
    }
}

// ===========================================================================
// §7.10.2 motion vector prediction
// ===========================================================================

void Walker::lower_mv_precision(int mv[2]) {
    if (fh.allow_high_precision_mv) return;
    for (int i = 0; i < 2; i++) {
        if (fh.force_integer_mv) {
            int a = std::abs(mv[i]);
            int aInt = (a + 3) >> 3;
            mv[i] = mv[i] > 0 ? (aInt << 3) : -(aInt << 3);
        } else if (mv[i] & 1) {
            mv[i] += mv[i] > 0 ? -1 : 1;
        }
    }
}

void Walker::setup_global_mv(int refList, int mv[2]) {
    int ref = RefFrame[refList];
    int typ = ref != INTRA_FRAME && ref > 0 ? fh.gm_type[ref] : IDENTITY;
    if (ref <= INTRA_FRAME || typ == IDENTITY) {
        mv[0] = mv[1] = 0;
    } else if (typ == TRANSLATION) {
        mv[0] = fh.gm_params[ref][0] >> (WARPEDMODEL_PREC_BITS - 3);
        mv[1] = fh.gm_params[ref][1] >> (WARPEDMODEL_PREC_BITS - 3);
    } else {
        const int32_t* gm = fh.gm_params[ref];
        int64_t x = MiCol * 4 + bw_of(MiSize) / 2 - 1;
        int64_t y = MiRow * 4 + bh_of(MiSize) / 2 - 1;
        int64_t xc = (int64_t)(gm[2] - (1 << WARPEDMODEL_PREC_BITS)) * x + (int64_t)gm[3] * y + gm[0];
        int64_t yc = (int64_t)gm[4] * x + (int64_t)(gm[5] - (1 << WARPEDMODEL_PREC_BITS)) * y + gm[1];
        if (fh.allow_high_precision_mv) {
            mv[0] = (int)round2signed(yc, WARPEDMODEL_PREC_BITS - 3);
            mv[1] = (int)round2signed(xc, WARPEDMODEL_PREC_BITS - 3);
        } else {
            mv[0] = (int)round2signed(yc, WARPEDMODEL_PREC_BITS - 2) * 2;
            mv[1] = (int)round2signed(xc, WARPEDMODEL_PREC_BITS - 2) * 2;
        }
    }
    lower_mv_precision(mv);
}

void Walker::find_mv_stack(int isCompound) {
    NumMvFound = 0;
    NewMvCount = 0;
    std::memset(RefStackMv, 0, sizeof RefStackMv);
    std::memset(WeightStack, 0, sizeof WeightStack);
    GlobalMvs[1][0] = GlobalMvs[1][1] = 0;
    setup_global_mv(0, GlobalMvs[0]);
    if (isCompound) setup_global_mv(1, GlobalMvs[1]);
    FoundMatch = 0;
    scan_row(-1, isCompound);
    int foundAboveMatch = FoundMatch;
    FoundMatch = 0;
    scan_col(-1, isCompound);
    int foundLeftMatch = FoundMatch;
    FoundMatch = 0;
    if (std::max(bw4, bh4) <= 16) scan_point(-1, bw4, isCompound);
    if (FoundMatch == 1) foundAboveMatch = 1;
    CloseMatches = foundAboveMatch + foundLeftMatch;
    int numNearest = NumMvFound, numNew = NewMvCount;
    for (int idx = 0; idx < numNearest; idx++) WeightStack[idx] += REF_CAT_LEVEL;
    ZeroMvContext = 0;
    if (fh.use_ref_frame_mvs) temporal_scan(isCompound);
    FoundMatch = 0;
    scan_point(-1, -1, isCompound);
    if (FoundMatch == 1) foundAboveMatch = 1;
    FoundMatch = 0;
    scan_row(-3, isCompound);
    if (FoundMatch == 1) foundAboveMatch = 1;
    FoundMatch = 0;
    scan_col(-3, isCompound);
    if (FoundMatch == 1) foundLeftMatch = 1;
    FoundMatch = 0;
    if (bh4 > 1) scan_row(-5, isCompound);
    if (FoundMatch == 1) foundAboveMatch = 1;
    FoundMatch = 0;
    if (bw4 > 1) scan_col(-5, isCompound);
    if (FoundMatch == 1) foundLeftMatch = 1;
    TotalMatches = foundAboveMatch + foundLeftMatch;
    sorting(0, numNearest);
    sorting(numNearest, NumMvFound);
    if (NumMvFound < 2) extra_search(isCompound);
    context_and_clamping(isCompound, numNew);
}

void Walker::scan_row(int deltaRow, int isCompound) {
    int end4 = std::min(std::min(bw4, MiCols - MiCol), 16);
    int deltaCol = 0;
    bool useStep16 = bw4 >= 16;
    if (std::abs(deltaRow) > 1) {
        deltaRow += MiRow & 1;
        deltaCol = 1 - (MiCol & 1);
    }
    int i = 0;
    while (i < end4) {
        int mvRow = MiRow + deltaRow, mvCol = MiCol + deltaCol + i;
        if (!is_inside(mvRow, mvCol)) break;
        int len = std::min(bw4, (int)Num_4x4_Blocks_Wide[MiSizes[cell(mvRow, mvCol)]]);
        if (std::abs(deltaRow) > 1) len = std::max(2, len);
        if (useStep16) len = std::max(4, len);
        add_ref_mv_candidate(mvRow, mvCol, isCompound, len * 2);
        i += len;
    }
}

void Walker::scan_col(int deltaCol, int isCompound) {
    int end4 = std::min(std::min(bh4, MiRows - MiRow), 16);
    int deltaRow = 0;
    bool useStep16 = bh4 >= 16;
    if (std::abs(deltaCol) > 1) {
        deltaRow = 1 - (MiRow & 1);
        deltaCol += MiCol & 1;
    }
    int i = 0;
    while (i < end4) {
        int mvRow = MiRow + deltaRow + i, mvCol = MiCol + deltaCol;
        if (!is_inside(mvRow, mvCol)) break;
        int len = std::min(bh4, (int)Num_4x4_Blocks_High[MiSizes[cell(mvRow, mvCol)]]);
        if (std::abs(deltaCol) > 1) len = std::max(2, len);
        if (useStep16) len = std::max(4, len);
        add_ref_mv_candidate(mvRow, mvCol, isCompound, len * 2);
        i += len;
    }
}

void Walker::scan_point(int deltaRow, int deltaCol, int isCompound) {
    int mvRow = MiRow + deltaRow, mvCol = MiCol + deltaCol;
    if (!is_inside(mvRow, mvCol)) return;
    if (mvRow >= MiRows || mvCol >= MiCols) return;
    if (MiSizes[cell(mvRow, mvCol)] == BLOCK_INVALID) return;  // not decoded yet in this frame
    add_ref_mv_candidate(mvRow, mvCol, isCompound, 4);
}

void Walker::add_ref_mv_candidate(int mvRow, int mvCol, int isCompound, int weight) {
    size_t i = cell(mvRow, mvCol);
    if (!IsInters[i]) return;
    if (!isCompound) {
        for (int candList = 0; candList < 2; candList++)
            if (RefFrames[i * 2 + candList] == RefFrame[0]) search_stack(mvRow, mvCol, candList, weight);
    } else {
        if (RefFrames[i * 2] == RefFrame[0] && RefFrames[i * 2 + 1] == RefFrame[1])
            compound_search_stack(mvRow, mvCol, weight);
    }
}

static bool has_newmv(int m) {
    return m == NEWMV || m == NEW_NEWMV || m == NEAR_NEWMV || m == NEW_NEARMV || m == NEAREST_NEWMV ||
           m == NEW_NEARESTMV;
}

void Walker::search_stack(int mvRow, int mvCol, int candList, int weight) {
    size_t i = cell(mvRow, mvCol);
    int candMode = YModes[i];
    int candSize = MiSizes[i];
    bool large = std::min(Num_4x4_Blocks_Wide[candSize], Num_4x4_Blocks_High[candSize]) >= 2;
    int candMv[2];
    if ((candMode == GLOBALMV || candMode == GLOBAL_GLOBALMV) && RefFrame[0] > 0 &&
        fh.gm_type[RefFrame[0]] > TRANSLATION && large) {
        candMv[0] = GlobalMvs[0][0];
        candMv[1] = GlobalMvs[0][1];
    } else {
        candMv[0] = Mvs[i * 4 + candList * 2];
        candMv[1] = Mvs[i * 4 + candList * 2 + 1];
    }
    lower_mv_precision(candMv);
    if (has_newmv(candMode)) NewMvCount++;
    FoundMatch = 1;
    for (int idx = 0; idx < NumMvFound; idx++)
        if (RefStackMv[idx][0][0] == candMv[0] && RefStackMv[idx][0][1] == candMv[1]) {
            WeightStack[idx] += weight;
            return;
        }
    if (NumMvFound < 8) {
        RefStackMv[NumMvFound][0][0] = candMv[0];
        RefStackMv[NumMvFound][0][1] = candMv[1];
        WeightStack[NumMvFound] = weight;
        NumMvFound++;
    }
}

void Walker::compound_search_stack(int mvRow, int mvCol, int weight) {
    size_t i = cell(mvRow, mvCol);
    int candMvs[2][2] = {{Mvs[i * 4], Mvs[i * 4 + 1]}, {Mvs[i * 4 + 2], Mvs[i * 4 + 3]}};
    int candMode = YModes[i];
    if (candMode == GLOBAL_GLOBALMV) {
        for (int l = 0; l < 2; l++) {
            candMvs[l][0] = GlobalMvs[l][0];
            candMvs[l][1] = GlobalMvs[l][1];
        }
    }
    lower_mv_precision(candMvs[0]);
    lower_mv_precision(candMvs[1]);
    FoundMatch = 1;
    if (has_newmv(candMode)) NewMvCount++;
    for (int idx = 0; idx < NumMvFound; idx++)
        if (RefStackMv[idx][0][0] == candMvs[0][0] && RefStackMv[idx][0][1] == candMvs[0][1] &&
            RefStackMv[idx][1][0] == candMvs[1][0] && RefStackMv[idx][1][1] == candMvs[1][1]) {
            WeightStack[idx] += weight;
            return;
        }
    if (NumMvFound < 8) {
        std::memcpy(RefStackMv[NumMvFound], candMvs, sizeof candMvs);
        WeightStack[NumMvFound] = weight;
        NumMvFound++;
    }
}

void Walker::temporal_scan(int isCompound) {
    int stepW4 = bw4 >= 16 ? 4 : 2, stepH4 = bh4 >= 16 ? 4 : 2;
    for (int dr = 0; dr < std::min(bh4, 16); dr += stepH4)
        for (int dc = 0; dc < std::min(bw4, 16); dc += stepW4) add_tpl_ref_mv(dr, dc, isCompound);
    bool allowExtension = bh4 >= 2 && bh4 < 16 && bw4 >= 2 && bw4 < 16;
    if (allowExtension) {
        const int pos[3][2] = {{bh4, -2}, {bh4, bw4}, {bh4 - 2, bw4}};
        for (int k = 0; k < 3; k++) {
            int row = (MiRow & 15) + pos[k][0], col = (MiCol & 15) + pos[k][1];
            if (row >= 0 && row < 16 && col >= 0 && col < 16) add_tpl_ref_mv(pos[k][0], pos[k][1], isCompound);
        }
    }
}

void Walker::add_tpl_ref_mv(int deltaRow, int deltaCol, int isCompound) {
    int mvRow = (MiRow + deltaRow) | 1, mvCol = (MiCol + deltaCol) | 1;
    if (!is_inside(mvRow, mvCol)) return;
    int x8 = mvCol >> 1, y8 = mvRow >> 1;
    int h8 = MiRows >> 1, w8 = MiCols >> 1;
    if (y8 >= h8 || x8 >= w8) return;
    if (deltaRow == 0 && deltaCol == 0) ZeroMvContext = 1;
    auto mf = [&](int ref, int comp) -> int {
        return MotionFieldMvs[(((size_t)(ref - LAST_FRAME) * h8 + y8) * w8 + x8) * 2 + comp];
    };
    if (!isCompound) {
        if (mf(RefFrame[0], 0) == MFMV_INVALID) return;
        int candMv[2] = {mf(RefFrame[0], 0), mf(RefFrame[0], 1)};
        lower_mv_precision(candMv);
        if (deltaRow == 0 && deltaCol == 0) {
            ZeroMvContext = (std::abs(candMv[0] - GlobalMvs[0][0]) >= 16 || std::abs(candMv[1] - GlobalMvs[0][1]) >= 16);
        }
        for (int idx = 0; idx < NumMvFound; idx++)
            if (RefStackMv[idx][0][0] == candMv[0] && RefStackMv[idx][0][1] == candMv[1]) {
                WeightStack[idx] += 2;
                return;
            }
        if (NumMvFound < 8) {
            RefStackMv[NumMvFound][0][0] = candMv[0];
            RefStackMv[NumMvFound][0][1] = candMv[1];
            WeightStack[NumMvFound] = 2;
            NumMvFound++;
        }
    } else {
        if (mf(RefFrame[0], 0) == MFMV_INVALID) return;
        if (mf(RefFrame[1], 0) == MFMV_INVALID) return;
        int c0[2] = {mf(RefFrame[0], 0), mf(RefFrame[0], 1)};
        int c1[2] = {mf(RefFrame[1], 0), mf(RefFrame[1], 1)};
        lower_mv_precision(c0);
        lower_mv_precision(c1);
        if (deltaRow == 0 && deltaCol == 0) {
            ZeroMvContext = (std::abs(c0[0] - GlobalMvs[0][0]) >= 16 || std::abs(c0[1] - GlobalMvs[0][1]) >= 16 ||
                             std::abs(c1[0] - GlobalMvs[1][0]) >= 16 || std::abs(c1[1] - GlobalMvs[1][1]) >= 16);
        }
        for (int idx = 0; idx < NumMvFound; idx++)
            if (RefStackMv[idx][0][0] == c0[0] && RefStackMv[idx][0][1] == c0[1] && RefStackMv[idx][1][0] == c1[0] &&
                RefStackMv[idx][1][1] == c1[1]) {
                WeightStack[idx] += 2;
                return;
            }
        if (NumMvFound < 8) {
            RefStackMv[NumMvFound][0][0] = c0[0];
            RefStackMv[NumMvFound][0][1] = c0[1];
            RefStackMv[NumMvFound][1][0] = c1[0];
            RefStackMv[NumMvFound][1][1] = c1[1];
            WeightStack[NumMvFound] = 2;
            NumMvFound++;
        }
    }
}

void Walker::sorting(int start, int end) {
    while (end > start) {
        int newEnd = start;
        for (int idx = start + 1; idx < end; idx++) {
            if (WeightStack[idx - 1] < WeightStack[idx]) {
                std::swap(WeightStack[idx - 1], WeightStack[idx]);
                int tmp[2][2];
                std::memcpy(tmp, RefStackMv[idx - 1], sizeof tmp);
                std::memcpy(RefStackMv[idx - 1], RefStackMv[idx], sizeof tmp);
                std::memcpy(RefStackMv[idx], tmp, sizeof tmp);
                newEnd = idx;
            }
        }
        end = newEnd;
    }
}

void Walker::extra_search(int isCompound) {
    RefIdCount[0] = RefIdCount[1] = RefDiffCount[0] = RefDiffCount[1] = 0;
    int w4 = std::min(std::min(16, bw4), MiCols - MiCol);
    int h4 = std::min(std::min(16, bh4), MiRows - MiRow);
    int num4x4 = std::min(w4, h4);
    for (int pass = 0; pass < 2 && NumMvFound < 2; pass++) {
        int idx = 0;
        while (idx < num4x4 && NumMvFound < 2) {
            int mvRow, mvCol;
            if (pass == 0) {
                mvRow = MiRow - 1;
                mvCol = MiCol + idx;
            } else {
                mvRow = MiRow + idx;
                mvCol = MiCol - 1;
            }
            if (!is_inside(mvRow, mvCol)) break;
            add_extra_mv_candidate(mvRow, mvCol, isCompound);
            int sz = MiSizes[cell(mvRow, mvCol)];
            idx += pass == 0 ? Num_4x4_Blocks_Wide[sz] : Num_4x4_Blocks_High[sz];
        }
    }
    if (isCompound) {
        int combined[2][2][2];
        for (int list = 0; list < 2; list++) {
            int compCount = 0;
            for (int idx = 0; idx < RefIdCount[list]; idx++) {
                combined[compCount][list][0] = RefIdMvs[list][idx][0];
                combined[compCount][list][1] = RefIdMvs[list][idx][1];
                compCount++;
            }
            for (int idx = 0; idx < RefDiffCount[list] && compCount < 2; idx++) {
                combined[compCount][list][0] = RefDiffMvs[list][idx][0];
                combined[compCount][list][1] = RefDiffMvs[list][idx][1];
                compCount++;
            }
            while (compCount < 2) {
                combined[compCount][list][0] = GlobalMvs[list][0];
                combined[compCount][list][1] = GlobalMvs[list][1];
                compCount++;
            }
        }
        if (NumMvFound == 1) {
            if (combined[0][0][0] == RefStackMv[0][0][0] && combined[0][0][1] == RefStackMv[0][0][1] &&
                combined[0][1][0] == RefStackMv[0][1][0] && combined[0][1][1] == RefStackMv[0][1][1])
                std::memcpy(RefStackMv[NumMvFound], combined[1], sizeof combined[1]);
            else
                std::memcpy(RefStackMv[NumMvFound], combined[0], sizeof combined[0]);
            WeightStack[NumMvFound] = 2;
            NumMvFound++;
        } else {
            for (int idx = 0; idx < 2; idx++) {
                std::memcpy(RefStackMv[NumMvFound], combined[idx], sizeof combined[idx]);
                WeightStack[NumMvFound] = 2;
                NumMvFound++;
            }
        }
    } else {
        for (int idx = NumMvFound; idx < 2; idx++) {
            RefStackMv[idx][0][0] = GlobalMvs[0][0];
            RefStackMv[idx][0][1] = GlobalMvs[0][1];
        }
    }
}

void Walker::add_extra_mv_candidate(int mvRow, int mvCol, int isCompound) {
    size_t i = cell(mvRow, mvCol);
    if (isCompound) {
        for (int candList = 0; candList < 2; candList++) {
            int candRef = RefFrames[i * 2 + candList];
            if (candRef > INTRA_FRAME) {
                for (int list = 0; list < 2; list++) {
                    int candMv[2] = {Mvs[i * 4 + candList * 2], Mvs[i * 4 + candList * 2 + 1]};
                    if (candRef == RefFrame[list] && RefIdCount[list] < 2) {
                        RefIdMvs[list][RefIdCount[list]][0] = candMv[0];
                        RefIdMvs[list][RefIdCount[list]][1] = candMv[1];
                        RefIdCount[list]++;
                    } else if (RefDiffCount[list] < 2) {
                        if (RefFrameSignBias[candRef] != RefFrameSignBias[RefFrame[list]]) {
                            candMv[0] = -candMv[0];
                            candMv[1] = -candMv[1];
                        }
                        RefDiffMvs[list][RefDiffCount[list]][0] = candMv[0];
                        RefDiffMvs[list][RefDiffCount[list]][1] = candMv[1];
                        RefDiffCount[list]++;
                    }
                }
            }
        }
    } else {
        for (int candList = 0; candList < 2; candList++) {
            int candRef = RefFrames[i * 2 + candList];
            if (candRef > INTRA_FRAME) {
                int candMv[2] = {Mvs[i * 4 + candList * 2], Mvs[i * 4 + candList * 2 + 1]};
                if (RefFrameSignBias[candRef] != RefFrameSignBias[RefFrame[0]]) {
                    candMv[0] = -candMv[0];
                    candMv[1] = -candMv[1];
                }
                int idx;
                for (idx = 0; idx < NumMvFound; idx++)
                    if (candMv[0] == RefStackMv[idx][0][0] && candMv[1] == RefStackMv[idx][0][1]) break;
                if (idx == NumMvFound && NumMvFound < 8) {
                    RefStackMv[idx][0][0] = candMv[0];
                    RefStackMv[idx][0][1] = candMv[1];
                    WeightStack[idx] = 2;
                    NumMvFound++;
                }
            }
        }
    }
}

void Walker::context_and_clamping(int isCompound, int numNew) {
    for (int idx = 0; idx < NumMvFound; idx++) {
        int z = 0;
        if (idx + 1 < NumMvFound) {
            int w0 = WeightStack[idx], w1 = WeightStack[idx + 1];
            if (w0 >= REF_CAT_LEVEL) {
                if (w1 < REF_CAT_LEVEL) z = 1;
            } else {
                z = 2;
            }
        }
        DrlCtxStack[idx] = z;
    }
    for (int list = 0; list < 1 + isCompound; list++)
        for (int idx = 0; idx < NumMvFound; idx++) {
            int* mv = RefStackMv[idx][list];
            int borderR = MV_BORDER + bh4 * 4 * 8, borderC = MV_BORDER + bw4 * 4 * 8;
            int top = -((MiRow * 4) * 8), bottom = ((MiRows - bh4 - MiRow) * 4) * 8;
            int left = -((MiCol * 4) * 8), right = ((MiCols - bw4 - MiCol) * 4) * 8;
            mv[0] = clip3(top - borderR, bottom + borderR, mv[0]);
            mv[1] = clip3(left - borderC, right + borderC, mv[1]);
        }
    if (CloseMatches == 0) {
        NewMvContext = std::min(TotalMatches, 1);
        RefMvContext = TotalMatches;
    } else if (CloseMatches == 1) {
        NewMvContext = 3 - std::min(numNew, 1);
        RefMvContext = 2 + TotalMatches;
    } else {
        NewMvContext = 5 - std::min(numNew, 1);
        RefMvContext = 5;
    }
}

// §7.10.4 warp samples
void Walker::find_warp_samples() {
    NumSamples = 0;
    NumSamplesScanned = 0;
    bool doTopLeft = true, doTopRight = true;
    if (AvailU) {
        int srcSize = MiSizes[cell(MiRow - 1, MiCol)];
        int srcW = Num_4x4_Blocks_Wide[srcSize];
        if (bw4 <= srcW) {
            int colOffset = -(MiCol & (srcW - 1));
            if (colOffset < 0) doTopLeft = false;
            if (colOffset + srcW > bw4) doTopRight = false;
            add_sample(-1, 0);
        } else {
            int step;
            for (int i = 0; i < std::min(bw4, MiCols - MiCol); i += step) {
                srcSize = MiSizes[cell(MiRow - 1, MiCol + i)];
                srcW = Num_4x4_Blocks_Wide[srcSize];
                step = std::min(bw4, srcW);
                add_sample(-1, i);
            }
        }
    }
    if (AvailL) {
        int srcSize = MiSizes[cell(MiRow, MiCol - 1)];
        int srcH = Num_4x4_Blocks_High[srcSize];
        if (bh4 <= srcH) {
            int rowOffset = -(MiRow & (srcH - 1));
            if (rowOffset < 0) doTopLeft = false;
            add_sample(0, -1);
        } else {
            int step;
            for (int i = 0; i < std::min(bh4, MiRows - MiRow); i += step) {
                srcSize = MiSizes[cell(MiRow + i, MiCol - 1)];
                srcH = Num_4x4_Blocks_High[srcSize];
                step = std::min(bh4, srcH);
                add_sample(i, -1);
            }
        }
    }
    if (doTopLeft) add_sample(-1, -1);
    if (doTopRight && std::max(bw4, bh4) <= 16) add_sample(-1, bw4);
    if (NumSamples == 0 && NumSamplesScanned > 0) NumSamples = 1;
}

void Walker::add_sample(int deltaRow, int deltaCol) {
    if (NumSamplesScanned >= 8) return;
    int mvRow = MiRow + deltaRow, mvCol = MiCol + deltaCol;
    if (!is_inside(mvRow, mvCol)) return;
    if (mvRow >= MiRows || mvCol >= MiCols) return;
    size_t i = cell(mvRow, mvCol);
    if (MiSizes[i] == BLOCK_INVALID) return;  // not decoded yet in this frame
    if (RefFrames[i * 2] != RefFrame[0]) return;
    if (RefFrames[i * 2 + 1] != NONE_REF) return;
    int candSz = MiSizes[i];
    int candW4 = Num_4x4_Blocks_Wide[candSz], candH4 = Num_4x4_Blocks_High[candSz];
    int candRow = mvRow & ~(candH4 - 1), candCol = mvCol & ~(candW4 - 1);
    int midY = candRow * 4 + candH4 * 2 - 1, midX = candCol * 4 + candW4 * 2 - 1;
    int threshold = clip3(16, 112, std::max(bw_of(MiSize), bh_of(MiSize)));
    int mvDiffRow = std::abs(Mvs[i * 4] - Mv[0][0]), mvDiffCol = std::abs(Mvs[i * 4 + 1] - Mv[0][1]);
    bool valid = mvDiffRow + mvDiffCol <= threshold;
    av1g_warp_sample cand{midY * 8, midX * 8, midY * 8 + Mvs[i * 4], midX * 8 + Mvs[i * 4 + 1]};
    NumSamplesScanned++;
    if (!valid && NumSamplesScanned > 1) return;
    CandList[NumSamples] = cand;
    if (valid) NumSamples++;
}

// ===========================================================================
// transform sizes, palette tokens
// ===========================================================================

int Walker::get_above_tx_width(int row, int col) {
    if (row == MiRow) {
        if (!AvailU) return 64;
        size_t i = cell(row - 1, col);
        if (Skips[i] && IsInters[i]) return bw_of(MiSizes[i]);
    }
    return Tx_Width[InterTxSizes[cell(row - 1, col)]];
}

int Walker::get_left_tx_height(int row, int col) {
    if (col == MiCol) {
        if (!AvailL) return 64;
        size_t i = cell(row, col - 1);
        if (Skips[i] && IsInters[i]) return bh_of(MiSizes[i]);
    }
    return Tx_Height[InterTxSizes[cell(row, col - 1)]];
}

void Walker::read_block_tx_size() {
    if (fh.tx_mode == 2 && MiSize > BLOCK_4X4 && is_inter && !skip && !Lossless) {
        int maxTxSz = Max_Tx_Size_Rect[MiSize];
        int txW4 = Tx_Width[maxTxSz] / 4, txH4 = Tx_Height[maxTxSz] / 4;
        for (int row = MiRow; row < MiRow + bh4; row += txH4)
            for (int col = MiCol; col < MiCol + bw4; col += txW4) read_var_tx_size(row, col, maxTxSz, 0);
    } else {
        read_tx_size(!skip || !is_inter);
        for (int row = MiRow; row < std::min(MiRows, MiRow + bh4); row++)
            for (int col = MiCol; col < std::min(MiCols, MiCol + bw4); col++) InterTxSizes[cell(row, col)] = (uint8_t)TxSize;
    }
}

void Walker::read_var_tx_size(int row, int col, int txSz, int depth) {
    if (row >= MiRows || col >= MiCols) return;
    int split;
    if (txSz == TX_4X4 || depth == 2) {
        split = 0;
    } else {
        int above = get_above_tx_width(row, col) < Tx_Width[txSz];
        int left = get_left_tx_height(row, col) < Tx_Height[txSz];
        int size = std::min(64, std::max(bw_of(MiSize), bh_of(MiSize)));
        int maxTxSz = find_tx_size(size, size);
        int txSzSqrUp = Tx_Size_Sqr_Up[txSz];
        int ctx = (txSzSqrUp != maxTxSz) * 3 + (4 - maxTxSz) * 6 + above + left;
        split = S(cdf.txfm_split[ctx], 2);
    }
    int w4 = Tx_Width[txSz] / 4, h4 = Tx_Height[txSz] / 4;
    if (split) {
        int sub = Split_Tx_Size[txSz];
        int stepW = Tx_Width[sub] / 4, stepH = Tx_Height[sub] / 4;
        for (int i = 0; i < h4; i += stepH)
            for (int j = 0; j < w4; j += stepW) read_var_tx_size(row + i, col + j, sub, depth + 1);
    } else {
        for (int i = 0; i < h4; i++)
            for (int j = 0; j < w4; j++)
                if (row + i < MiRows && col + j < MiCols) InterTxSizes[cell(row + i, col + j)] = (uint8_t)txSz;
        TxSize = txSz;
    }
}

void Walker::read_tx_size(int allowSelect) {
    if (Lossless) {
        TxSize = TX_4X4;
        return;
    }
    int maxRect = Max_Tx_Size_Rect[MiSize];
    int maxDepth = Max_Tx_Depth_Table[MiSize];
    TxSize = maxRect;
    if (MiSize > BLOCK_4X4 && allowSelect && fh.tx_mode == 2) {
        int maxW = Tx_Width[maxRect], maxH = Tx_Height[maxRect];
        int aboveW = 0, leftH = 0;
        if (AvailU) {
            size_t i = cell(MiRow - 1, MiCol);
            aboveW = IsInters[i] ? bw_of(MiSizes[i]) : get_above_tx_width(MiRow, MiCol);
        }
        if (AvailL) {
            size_t i = cell(MiRow, MiCol - 1);
            leftH = IsInters[i] ? bh_of(MiSizes[i]) : get_left_tx_height(MiRow, MiCol);
        }
        int ctx = (aboveW >= maxW) + (leftH >= maxH);
        int depth;
        if (maxDepth == 4) depth = S(cdf.tx_64x64[ctx], 3);
        else if (maxDepth == 3) depth = S(cdf.tx_32x32[ctx], 3);
        else if (maxDepth == 2) depth = S(cdf.tx_16x16[ctx], 3);
        else depth = S(cdf.tx_8x8[ctx], 2);
        for (int i = 0; i < depth; i++) TxSize = Split_Tx_Size[TxSize];
    }
}

void Walker::get_palette_color_context(const uint8_t* map, int stride, int r, int c, int n, int* order, int* ctx) {
    int scores[8];
    for (int i = 0; i < 8; i++) {
        scores[i] = 0;
        order[i] = i;
    }
    if (c > 0) scores[map[r * stride + c - 1]] += 2;
    if (r > 0 && c > 0) scores[map[(r - 1) * stride + c - 1]] += 1;
    if (r > 0) scores[map[(r - 1) * stride + c]] += 2;
    for (int i = 0; i < 3; i++) {
        int maxScore = scores[i], maxIdx = i;
        for (int j = i + 1; j < n; j++)
            if (scores[j] > maxScore) {
                maxScore = scores[j];
                maxIdx = j;
            }
        if (maxIdx != i) {
            maxScore = scores[maxIdx];
            int maxOrder = order[maxIdx];
            for (int k = maxIdx; k > i; k--) {
                scores[k] = scores[k - 1];
                order[k] = order[k - 1];
            }
            scores[i] = maxScore;
            order[i] = maxOrder;
        }
    }
    int hash = 0;
    for (int i = 0; i < 3; i++) hash += scores[i] * Palette_Color_Hash_Multipliers[i];
    *ctx = Palette_Color_Context[hash];
}

void Walker::palette_tokens() {
    int blockHeight = bh_of(MiSize), blockWidth = bw_of(MiSize);
    int onscreenHeight = std::min(blockHeight, (MiRows - MiRow) * 4);
    int onscreenWidth = std::min(blockWidth, (MiCols - MiCol) * 4);
    for (int pl = 0; pl < 2; pl++) {
        int n = pl == 0 ? PaletteSizeY : PaletteSizeUV;
        if (!n) continue;
        int bh = blockHeight, bw = blockWidth, oh = onscreenHeight, ow = onscreenWidth;
        if (pl == 1) {
            bh >>= ssy;
            bw >>= ssx;
            oh >>= ssy;
            ow >>= ssx;
            if (bw < 4) {
                bw += 2;
                ow += 2;
            }
            if (bh < 4) {
                bh += 2;
                oh += 2;
            }
        }
        std::vector<uint8_t>& map = pl == 0 ? ColorMapY : ColorMapUV;
        map.assign((size_t)bw * bh, 0);
        map[0] = (uint8_t)NS(n);
        for (int i = 1; i < oh + ow - 1; i++)
            for (int j = std::min(i, ow - 1); j >= std::max(0, i - oh + 1); j--) {
                int order[8], ctx;
                get_palette_color_context(map.data(), bw, i - j, j, n, order, &ctx);
                int idx = S(pl == 0 ? cdf.palette_y_color[n - 2][ctx] : cdf.palette_uv_color[n - 2][ctx], n);
                map[(size_t)(i - j) * bw + j] = (uint8_t)order[idx];
            }
        for (int i = 0; i < oh; i++)
            for (int j = ow; j < bw; j++) map[(size_t)i * bw + j] = map[(size_t)i * bw + ow - 1];
        for (int i = oh; i < bh; i++)
            for (int j = 0; j < bw; j++) map[(size_t)i * bw + j] = map[(size_t)(oh - 1) * bw + j];
        palette_map_off[pl] = (uint32_t)out.palette_maps.size();
        out.palette_maps.insert(out.palette_maps.end(), map.begin(), map.end());
        (pl == 0 ? ColorMapYStride : ColorMapUVStride) = bw;
    }
}

void Walker::reset_block_context() {
    for (int plane = 0; plane < 1 + 2 * HasChroma; plane++) {
        int subX = plane ? ssx : 0, subY = plane ? ssy : 0;
        for (int i = MiCol >> subX; i < ((MiCol + bw4) >> subX); i++) {
            AboveLevelContext[plane][i] = 0;
            AboveDcContext[plane][i] = 0;
        }
        for (int i = MiRow >> subY; i < ((MiRow + bh4) >> subY); i++) {
            LeftLevelContext[plane][i] = 0;
            LeftDcContext[plane][i] = 0;
        }
    }
}

// ===========================================================================
// residual
// ===========================================================================

void Walker::residual() {
    int sbMask = sb128 ? 31 : 15;
    (void)sbMask;
    int widthChunks = std::max(1, bw_of(MiSize) >> 6), heightChunks = std::max(1, bh_of(MiSize) >> 6);
    int sizeChunk = (widthChunks > 1 || heightChunks > 1) ? BLOCK_64X64 : MiSize;
    for (int chunkY = 0; chunkY < heightChunks; chunkY++)
        for (int chunkX = 0; chunkX < widthChunks; chunkX++) {
            int miRowChunk = MiRow + (chunkY << 4), miColChunk = MiCol + (chunkX << 4);
            for (int plane = 0; plane < 1 + HasChroma * 2; plane++) {
                int txSz = Lossless ? TX_4X4 : get_tx_size(plane, TxSize);
                int stepX = Tx_Width[txSz] >> 2, stepY = Tx_Height[txSz] >> 2;
                int planeSz = plane_residual_size(sizeChunk, plane);
                if (planeSz >= BLOCK_INVALID) continue;
                int num4x4W = Num_4x4_Blocks_Wide[planeSz], num4x4H = Num_4x4_Blocks_High[planeSz];
                int subX = plane ? ssx : 0, subY = plane ? ssy : 0;
                if (is_inter && !Lossless && !plane) {
                    transform_tree((miColChunk >> subX) * 4, (miRowChunk >> subY) * 4, num4x4W * 4, num4x4H * 4);
                } else {
                    int baseXBlock = (MiCol >> subX) * 4, baseYBlock = (MiRow >> subY) * 4;
                    for (int y = 0; y < num4x4H; y += stepY)
                        for (int x = 0; x < num4x4W; x += stepX)
                            transform_block(plane, baseXBlock, baseYBlock, txSz, x + ((chunkX << 4) >> subX),
                                            y + ((chunkY << 4) >> subY));
                }
            }
        }
}

void Walker::transform_tree(int startX, int startY, int w, int h) {
    int maxX = MiCols * 4, maxY = MiRows * 4;
    if (startX >= maxX || startY >= maxY) return;
    int row = startY >> 2, col = startX >> 2;
    int lumaTx = InterTxSizes[cell(row, col)];
    int lumaW = Tx_Width[lumaTx], lumaH = Tx_Height[lumaTx];
    if (w <= lumaW && h <= lumaH) {
        int txSz = find_tx_size(w, h);
        if (txSz < 0) throw WalkError("walker: transform tree reached an unknown size");
        transform_block(0, startX, startY, txSz, 0, 0);
    } else if (w > h) {
        transform_tree(startX, startY, w / 2, h);
        transform_tree(startX + w / 2, startY, w / 2, h);
    } else if (w < h) {
        transform_tree(startX, startY, w, h / 2);
        transform_tree(startX, startY + h / 2, w, h / 2);
    } else {
        transform_tree(startX, startY, w / 2, h / 2);
        transform_tree(startX + w / 2, startY, w / 2, h / 2);
        transform_tree(startX, startY + h / 2, w / 2, h / 2);
        transform_tree(startX + w / 2, startY + h / 2, w / 2, h / 2);
    }
}

bool Walker::is_smooth(int row, int col, int plane) {
    size_t i = cell(row, col);
    int mode;
    if (plane == 0) {
        mode = YModes[i];
    } else {
        if (RefFrames[i * 2] > INTRA_FRAME) return false;
        mode = UVModes[i];
    }
    return mode == SMOOTH_PRED || mode == SMOOTH_V_PRED || mode == SMOOTH_H_PRED;
}

int Walker::get_filter_type(int plane) {
    bool aboveSmooth = false, leftSmooth = false;
    if (plane == 0 ? AvailU : AvailUChroma) {
        int r = MiRow - 1, c = MiCol;
        if (plane > 0) {
            if (ssx && !(MiCol & 1)) c++;
            if (ssy && (MiRow & 1)) r--;
        }
        aboveSmooth = is_smooth(r, c, plane);
    }
    if (plane == 0 ? AvailL : AvailLChroma) {
        int r = MiRow, c = MiCol - 1;
        if (plane > 0) {
            if (ssx && (MiCol & 1)) c--;
            if (ssy && !(MiRow & 1)) r++;
        }
        leftSmooth = is_smooth(r, c, plane);
    }
    return aboveSmooth || leftSmooth;
}

void Walker::transform_block(int plane, int baseX, int baseY, int txSz, int x, int y) {
    int startX = baseX + 4 * x, startY = baseY + 4 * y;
    int subX = plane ? ssx : 0, subY = plane ? ssy : 0;
    int row = (startY << subY) >> 2, col = (startX << subX) >> 2;
    int sbMask = sb128 ? 31 : 15;
    int subBlockMiRow = row & sbMask, subBlockMiCol = col & sbMask;
    int stepX = Tx_Width[txSz] >> 2, stepY = Tx_Height[txSz] >> 2;
    int maxX = MiCols * 4 - 1, maxY = MiRows * 4 - 1;
    if (startX >= (maxX >> subX) || startY >= (maxY >> subY)) return;
    av1g_intra_tu t{};
    bool emitIntra = false;
    if (!is_inter || use_intrabc) {
        t.x = (uint16_t)startX;
        t.y = (uint16_t)startY;
        t.plane = (uint8_t)plane;
        t.tx_size = (uint8_t)txSz;
        t.filter_intra_mode = 255;
        emitIntra = true;
        if (use_intrabc) {
            t.mode = AV1G_INTRA_MODE_INTRABC;
            t.mv[0] = (int16_t)Mv[0][0];
            t.mv[1] = (int16_t)Mv[0][1];
        } else if ((plane == 0 && PaletteSizeY) || (plane != 0 && PaletteSizeUV)) {
            int pl = plane ? 1 : 0;
            int stride = pl ? ColorMapUVStride : ColorMapYStride;
            // the TU's map origin inside the block's map
            int bx = (MiCol >> subX) * 4, by = (MiRow >> subY) * 4;
            if (pl && bw4 == 1 && ssx) bx = ((MiCol - 1) >> subX) * 4;
            if (pl && bh4 == 1 && ssy) by = ((MiRow - 1) >> subY) * 4;
            t.mode = AV1G_INTRA_MODE_PALETTE;
            t.palette_map = palette_map_off[pl] + (uint32_t)((startY - by) * stride + (startX - bx));
            t.palette_stride = (uint16_t)stride;
            int n = pl ? PaletteSizeUV : PaletteSizeY;
            t.palette_size = (uint8_t)n;
            const uint16_t* cols = plane == 0 ? palette_colors_y : plane == 1 ? palette_colors_u : palette_colors_v;
            for (int k = 0; k < n; k++) t.palette_colors[k] = cols[k];
        } else {
            bool isCfl = plane > 0 && UVMode == UV_CFL_PRED;
            int mode = plane == 0 ? YMode : (isCfl ? DC_PRED : UVMode);
            t.mode = (uint8_t)mode;
            bool haveLeft = (plane == 0 ? AvailL : AvailLChroma) || x > 0;
            bool haveAbove = (plane == 0 ? AvailU : AvailUChroma) || y > 0;
            if (haveAbove) t.flags |= AV1G_INTRA_HAVE_ABOVE;
            if (haveLeft) t.flags |= AV1G_INTRA_HAVE_LEFT;
            if (block_decoded(plane, (subBlockMiRow >> subY) - 1, (subBlockMiCol >> subX) + stepX))
                t.flags |= AV1G_INTRA_HAVE_ABOVE_RIGHT;
            if (block_decoded(plane, (subBlockMiRow >> subY) + stepY, (subBlockMiCol >> subX) - 1))
                t.flags |= AV1G_INTRA_HAVE_BELOW_LEFT;
            if (seq.enable_intra_edge_filter) t.flags |= AV1G_INTRA_EDGE_FILTER;
            if (get_filter_type(plane)) t.flags |= AV1G_INTRA_FILTER_TYPE;
            t.angle_delta = (int8_t)(plane == 0 ? AngleDeltaY : AngleDeltaUV);
            if (plane == 0 && use_filter_intra) t.filter_intra_mode = (uint8_t)filter_intra_mode;
            if (isCfl) {
                t.flags |= AV1G_INTRA_CFL;
                t.cfl_alpha = (int8_t)(plane == 1 ? CflAlphaU : CflAlphaV);
                t.max_luma_w = (uint16_t)MaxLumaW;
                t.max_luma_h = (uint16_t)MaxLumaH;
            }
        }
        if (plane == 0) {
            MaxLumaW = startX + stepX * 4;
            MaxLumaH = startY + stepY * 4;
        }
    }
    av1g_tu tu{};
    tu.x = (uint16_t)startX;
    tu.y = (uint16_t)startY;
    tu.plane = (uint8_t)plane;
    tu.tx_size = (uint8_t)txSz;
    tu.segment_id = (uint8_t)segment_id;
    tu.current_q_index = (uint8_t)CurrentQIndex;
    int eob = 0;
    if (!skip) {
        int ptt;
        uint32_t off;
        eob = coeffs(plane, startX, startY, txSz, &ptt, &off);
        if (eob > 0) {
            tu.tx_type = (uint8_t)ptt;
            tu.coeff_offset = off;
        }
    }
    if (emitIntra) {
        t.res = tu;
        if (eob > 0) t.flags |= AV1G_INTRA_RESIDUAL;
        out.intra_tus.push_back(t);
    } else if (eob > 0) {
        if (interintra) {
            av1g_intra_tu r{};
            r.x = tu.x;
            r.y = tu.y;
            r.plane = tu.plane;
            r.tx_size = tu.tx_size;
            r.mode = AV1G_INTRA_MODE_NONE;
            r.flags = AV1G_INTRA_RESIDUAL;
            r.filter_intra_mode = 255;
            r.res = tu;
            out.intra_tus.push_back(r);
        } else {
            out.inter_tus.push_back(tu);
        }
    }
    for (int i = 0; i < stepY; i++)
        for (int j = 0; j < stepX; j++) {
            int by = (subBlockMiRow >> subY) + i, bx = (subBlockMiCol >> subX) + j;
            if (by <= 32 && bx <= 32) block_decoded(plane, by, bx) = 1;
        }
}

int Walker::get_tx_set(int txSz) {
    int sqr = tx_sqr(txSz), sqrUp = Tx_Size_Sqr_Up[txSz];
    if (sqrUp > TX_32X32) return TX_SET_DCTONLY;
    if (is_inter) {
        if (fh.reduced_tx_set || sqrUp == TX_32X32) return TX_SET_INTER_3;
        if (sqr == TX_16X16) return TX_SET_INTER_2;
        return TX_SET_INTER_1;
    }
    if (sqrUp == TX_32X32) return TX_SET_DCTONLY;
    if (fh.reduced_tx_set) return TX_SET_INTRA_2;
    if (sqr == TX_16X16) return TX_SET_INTRA_2;
    return TX_SET_INTRA_1;
}

void Walker::transform_type(int x4, int y4, int txSz) {
    int set = get_tx_set(txSz);
    int txType = DCT_DCT;
    int qidx = fh.segmentation_enabled ? get_qidx(1, segment_id) : fh.base_q_idx;
    if (set > 0 && qidx > 0) {
        int sqr = tx_sqr(txSz);
        if (is_inter) {
            if (set == TX_SET_INTER_1) txType = Tx_Type_Inter_Inv_Set1[S(cdf.inter_tx_type_set1[sqr], 16)];
            else if (set == TX_SET_INTER_2) txType = Tx_Type_Inter_Inv_Set2[S(cdf.inter_tx_type_set2, 12)];
            else txType = Tx_Type_Inter_Inv_Set3[S(cdf.inter_tx_type_set3[sqr], 2)];
        } else {
            int intraDir = use_filter_intra ? Filter_Intra_Mode_To_Intra_Dir[filter_intra_mode] : YMode;
            if (set == TX_SET_INTRA_1) txType = Tx_Type_Intra_Inv_Set1[S(cdf.intra_tx_type_set1[sqr][intraDir], 7)];
            else txType = Tx_Type_Intra_Inv_Set2[S(cdf.intra_tx_type_set2[sqr][intraDir], 5)];
        }
    }
    for (int i = 0; i < (Tx_Width[txSz] >> 2); i++)
        for (int j = 0; j < (Tx_Height[txSz] >> 2); j++)
            if (y4 + j < MiRows && x4 + i < MiCols) TxTypes[cell(y4 + j, x4 + i)] = (uint8_t)txType;
}

int Walker::compute_tx_type(int plane, int txSz, int blockX, int blockY) {
    int sqrUp = Tx_Size_Sqr_Up[txSz];
    if (Lossless || sqrUp > TX_32X32) return DCT_DCT;
    int txSet = get_tx_set(txSz);
    if (plane == 0) return TxTypes[cell(blockY, blockX)];
    int txType;
    if (is_inter) {
        int x4 = std::max(MiCol, blockX << ssx), y4 = std::max(MiRow, blockY << ssy);
        txType = TxTypes[cell(y4, x4)];
        if (!Tx_Type_In_Set_Inter[txSet][txType]) return DCT_DCT;
        return txType;
    }
    txType = Mode_To_Txfm[UVMode];
    if (!Tx_Type_In_Set_Intra[txSet][txType]) return DCT_DCT;
    return txType;
}

int Walker::coeffs(int plane, int startX, int startY, int txSz, int* planeTxType, uint32_t* coeffOff) {
    int x4 = startX >> 2, y4 = startY >> 2;
    int w4 = Tx_Width[txSz] >> 2, h4 = Tx_Height[txSz] >> 2;
    int txSzCtx = (tx_sqr(txSz) + Tx_Size_Sqr_Up[txSz] + 1) >> 1;
    int ptype = plane > 0;
    int segEob = (txSz == TX_16X64 || txSz == TX_64X16) ? 512 : std::min(1024, Tx_Width[txSz] * Tx_Height[txSz]);
    int32_t Quant[1024];
    std::memset(Quant, 0, sizeof(int32_t) * segEob);
    int eob = 0, culLevel = 0, dcCategory = 0;
    // all_zero context (txb_skip_ctx, cdf.rs:21650)
    int maxX4 = MiCols, maxY4 = MiRows;
    if (plane > 0) {
        maxX4 >>= ssx;
        maxY4 >>= ssy;
    }
    int w = Tx_Width[txSz], h = Tx_Height[txSz];
    int ctx;
    {
        int bsize = plane_residual_size(MiSize, plane);
        int bw = bw_of(bsize), bh = bh_of(bsize);
        if (plane == 0) {
            int top = 0, left = 0;
            for (int k = 0; k < w4; k++)
                if (x4 + k < maxX4) top = std::max(top, (int)AboveLevelContext[plane][x4 + k]);
            for (int k = 0; k < h4; k++)
                if (y4 + k < maxY4) left = std::max(left, (int)LeftLevelContext[plane][y4 + k]);
            top = std::min(top, 255);
            left = std::min(left, 255);
            if (bw == w && bh == h) ctx = 0;
            else if (top == 0 && left == 0) ctx = 1;
            else if (top == 0 || left == 0) ctx = 2 + (std::max(top, left) > 3);
            else if (std::max(top, left) <= 3) ctx = 4;
            else if (std::min(top, left) <= 3) ctx = 5;
            else ctx = 6;
        } else {
            int above = 0, left = 0;
            for (int i = 0; i < w4; i++)
                if (x4 + i < maxX4) above |= AboveLevelContext[plane][x4 + i] | AboveDcContext[plane][x4 + i];
            for (int i = 0; i < h4; i++)
                if (y4 + i < maxY4) left |= LeftLevelContext[plane][y4 + i] | LeftDcContext[plane][y4 + i];
            ctx = (above != 0) + (left != 0) + 7;
            if (bw * bh > w * h) ctx += 3;
        }
    }
    int allZero = S(cdf.txb_skip[txSzCtx][ctx], 2);
    if (allZero) {
        if (plane == 0)
            for (int i = 0; i < w4; i++)
                for (int j = 0; j < h4; j++)
                    if (y4 + j < MiRows && x4 + i < MiCols) TxTypes[cell(y4 + j, x4 + i)] = DCT_DCT;
        *planeTxType = DCT_DCT;
    } else {
        if (plane == 0) transform_type(x4, y4, txSz);
        int ptt = compute_tx_type(plane, txSz, x4, y4);
        *planeTxType = ptt;
        // scan (get_scan, src/scan.rs:563)
        const uint16_t* scan;
        {
            int adj = txSz;
            if (txSz == TX_16X64) scan = Default_Scan_16x32;
            else if (txSz == TX_64X16) scan = Default_Scan_32x16;
            else if (Tx_Size_Sqr_Up[txSz] == TX_64X64) scan = Default_Scan_32x32;
            else {
                bool preferRow = ptt == V_DCT || ptt == V_ADST || ptt == V_FLIPADST;
                bool preferCol = ptt == H_DCT || ptt == H_ADST || ptt == H_FLIPADST;
                if (ptt == IDTX) preferRow = preferCol = false;
                switch (adj) {
                    case TX_4X4: scan = preferRow ? Mrow_Scan_4x4 : preferCol ? Mcol_Scan_4x4 : Default_Scan_4x4; break;
                    case TX_4X8: scan = preferRow ? Mrow_Scan_4x8 : preferCol ? Mcol_Scan_4x8 : Default_Scan_4x8; break;
                    case TX_8X4: scan = preferRow ? Mrow_Scan_8x4 : preferCol ? Mcol_Scan_8x4 : Default_Scan_8x4; break;
                    case TX_8X8: scan = preferRow ? Mrow_Scan_8x8 : preferCol ? Mcol_Scan_8x8 : Default_Scan_8x8; break;
                    case TX_8X16: scan = preferRow ? Mrow_Scan_8x16 : preferCol ? Mcol_Scan_8x16 : Default_Scan_8x16; break;
                    case TX_16X8: scan = preferRow ? Mrow_Scan_16x8 : preferCol ? Mcol_Scan_16x8 : Default_Scan_16x8; break;
                    case TX_16X16:
                        scan = preferRow ? Mrow_Scan_16x16 : preferCol ? Mcol_Scan_16x16 : Default_Scan_16x16;
                        break;
                    case TX_4X16: scan = preferRow ? Mrow_Scan_4x16 : preferCol ? Mcol_Scan_4x16 : Default_Scan_4x16; break;
                    case TX_16X4: scan = preferRow ? Mrow_Scan_16x4 : preferCol ? Mcol_Scan_16x4 : Default_Scan_16x4; break;
                    case TX_8X32: scan = Default_Scan_8x32; break;
                    case TX_32X8: scan = Default_Scan_32x8; break;
                    case TX_16X32: scan = Default_Scan_16x32; break;
                    case TX_32X16: scan = Default_Scan_32x16; break;
                    default: scan = Default_Scan_32x32; break;
                }
            }
        }
        int eobMultisize = std::min((int)Tx_Width_Log2[txSz], 5) + std::min(ceil_log2(Tx_Height[txSz]), 5) - 4;
        int txClass = (ptt == V_DCT || ptt == V_ADST || ptt == V_FLIPADST) ? 2
                      : (ptt == H_DCT || ptt == H_ADST || ptt == H_FLIPADST) ? 1 : 0;
        int ectx = txClass == 0 ? 0 : 1;
        int eobPt;
        switch (eobMultisize) {
            case 0: eobPt = S(cdf.eob_pt_16[ptype][ectx], 5) + 1; break;
            case 1: eobPt = S(cdf.eob_pt_32[ptype][ectx], 6) + 1; break;
            case 2: eobPt = S(cdf.eob_pt_64[ptype][ectx], 7) + 1; break;
            case 3: eobPt = S(cdf.eob_pt_128[ptype][ectx], 8) + 1; break;
            case 4: eobPt = S(cdf.eob_pt_256[ptype][ectx], 9) + 1; break;
            case 5: eobPt = S(cdf.eob_pt_512[ptype], 10) + 1; break;
            default: eobPt = S(cdf.eob_pt_1024[ptype], 11) + 1; break;
        }
        eob = eobPt < 2 ? eobPt : ((1 << (eobPt - 2)) + 1);
        int eobShift = eobPt - 3;
        if (eobShift >= 0) {
            if (S(cdf.eob_extra[txSzCtx][ptype][eobPt - 3], 2)) eob += 1 << eobShift;
            for (int i = 1; i < std::max(0, eobPt - 2); i++) {
                eobShift = std::max(0, eobPt - 2) - 1 - i;
                if (L(1)) eob += 1 << eobShift;
            }
        }
        int adj = Adjusted_Tx_Size[txSz];
        int bwl = Tx_Width_Log2[adj];
        int txh = Tx_Height[adj];
        for (int c = eob - 1; c >= 0; c--) {
            int pos = scan[c];
            int row = pos >> bwl, col = pos - (row << bwl);
            int level;
            if (c == eob - 1) {
                int cctx;
                if (c == 0) cctx = 0;
                else if (c <= (txh << bwl) / 8) cctx = 1;
                else if (c <= (txh << bwl) / 4) cctx = 2;
                else cctx = 3;
                level = S(cdf.coeff_base_eob[txSzCtx][ptype][cctx], 3) + 1;
            } else {
                int mag = 0;
                for (int idx = 0; idx < 5; idx++) {
                    int rr = row + Sig_Ref_Diff_Offset[txClass][idx][0];
                    int cc = col + Sig_Ref_Diff_Offset[txClass][idx][1];
                    if (rr >= 0 && cc >= 0 && rr < txh && cc < (1 << bwl))
                        mag += std::min(std::abs(Quant[(rr << bwl) + cc]), 3);
                }
                int cctx = std::min((mag + 1) >> 1, 4);
                if (txClass == 0) {
                    if (row == 0 && col == 0) cctx = 0;
                    else cctx += Coeff_Base_Ctx_Offset[txSz][std::min(row, 4)][std::min(col, 4)];
                } else {
                    int idx = txClass == 2 ? row : col;
                    cctx += Coeff_Base_Pos_Ctx_Offset[std::min(idx, 2)];
                }
                level = S(cdf.coeff_base[txSzCtx][ptype][cctx], 4);
            }
            if (level > 2) {
                int mag = 0;
                for (int idx = 0; idx < 3; idx++) {
                    int rr = row + Mag_Ref_Offset_With_Tx_Class[txClass][idx][0];
                    int cc = col + Mag_Ref_Offset_With_Tx_Class[txClass][idx][1];
                    if (rr >= 0 && cc >= 0 && rr < txh && cc < (1 << bwl))
                        mag += std::min(Quant[rr * (1 << bwl) + cc], 15);
                }
                mag = std::min((mag + 1) >> 1, 6);
                int bctx;
                if (pos == 0) bctx = mag;
                else if (txClass == 0) bctx = (row < 2 && col < 2) ? mag + 7 : mag + 14;
                else if (txClass == 1) bctx = col == 0 ? mag + 7 : mag + 14;
                else bctx = row == 0 ? mag + 7 : mag + 14;
                for (int idx = 0; idx < 4; idx++) {
                    int br = S(cdf.coeff_br[std::min(txSzCtx, 3)][ptype][bctx], 4);
                    level += br;
                    if (br < 3) break;
                }
            }
            Quant[pos] = level;
        }
        for (int c = 0; c < eob; c++) {
            int pos = scan[c];
            int sign = 0;
            if (Quant[pos] != 0) {
                if (c == 0) {
                    int dc = 0;
                    for (int k = 0; k < w4; k++)
                        if (x4 + k < maxX4) {
                            int v = AboveDcContext[plane][x4 + k];
                            dc += v == 1 ? -1 : v == 2 ? 1 : 0;
                        }
                    for (int k = 0; k < h4; k++)
                        if (y4 + k < maxY4) {
                            int v = LeftDcContext[plane][y4 + k];
                            dc += v == 1 ? -1 : v == 2 ? 1 : 0;
                        }
                    int dctx = dc < 0 ? 1 : dc > 0 ? 2 : 0;
                    sign = S(cdf.dc_sign[ptype][dctx], 2);
                } else {
                    sign = L(1);
                }
            }
            if (Quant[pos] > 14) {
                int length = 0, bit;
                do {
                    length++;
                    bit = L(1);
                    if (length > 32) throw WalkError("walker: golomb length overflow");
                } while (!bit);
                int64_t xg = 1;
                for (int i = length - 2; i >= 0; i--) xg = (xg << 1) | L(1);
                Quant[pos] = (int32_t)(xg + 14);
            }
            if (pos == 0 && Quant[pos] > 0) dcCategory = sign ? 1 : 2;
            Quant[pos] &= 0xFFFFF;
            culLevel += Quant[pos];
            if (sign) Quant[pos] = -Quant[pos];
        }
        culLevel = std::min(63, culLevel);
    }
    for (int i = 0; i < w4; i++) {
        AboveLevelContext[plane][x4 + i] = (uint8_t)culLevel;
        AboveDcContext[plane][x4 + i] = (uint8_t)dcCategory;
    }
    for (int i = 0; i < h4; i++) {
        LeftLevelContext[plane][y4 + i] = (uint8_t)culLevel;
        LeftDcContext[plane][y4 + i] = (uint8_t)dcCategory;
    }
    if (eob > 0) {
        int tw = std::min(32, w), th = std::min(32, h);
        *coeffOff = (uint32_t)out.coeffs.size();
        out.coeffs.insert(out.coeffs.end(), Quant, Quant + tw * th);
    }
    return eob;
}

// ===========================================================================
// inter prediction descriptors (compute_prediction, §5.11.33)
// ===========================================================================

void Walker::distance_weights(int* fwd, int* bck) {
    static const int8_t Quant_Dist_Weight[4][2] = {{2, 3}, {2, 5}, {2, 7}, {1, 31}};
    static const int8_t Quant_Dist_Lookup[4][2] = {{9, 7}, {11, 5}, {12, 4}, {13, 3}};
    int dist[2];
    for (int l = 0; l < 2; l++) {
        int h = fh.order_hints[RefFrame[l]];
        dist[l] = clip3(0, 31, std::abs(get_relative_dist(h, fh.order_hint, OrderHintBits)));
    }
    int d0 = dist[1], d1 = dist[0];
    int order = d0 <= d1;
    if (d0 == 0 || d1 == 0) {
        *fwd = Quant_Dist_Lookup[3][order];
        *bck = Quant_Dist_Lookup[3][1 - order];
        return;
    }
    int i;
    for (i = 0; i < 3; i++) {
        int c0 = Quant_Dist_Weight[i][order], c1 = Quant_Dist_Weight[i][1 - order];
        if (order) {
            if (d0 * c0 > d1 * c1) break;
        } else {
            if (d0 * c0 < d1 * c1) break;
        }
    }
    *fwd = Quant_Dist_Lookup[i][order];
    *bck = Quant_Dist_Lookup[i][1 - order];
}

void Walker::emit_inter_block() {
    int isCompound = RefFrame[1] > INTRA_FRAME;
    int isII = RefFrame[1] == INTRA_FRAME;
    // warp context: local warp, or a GLOBALMV-class block of a non-translational model
    int warp = -1;
    bool yGlobal = YMode == GLOBALMV || YMode == GLOBAL_GLOBALMV;
    bool gmWarp = fh.gm_type[RefFrame[0]] > TRANSLATION || (isCompound && fh.gm_type[RefFrame[1]] > TRANSLATION);
    if (motion_mode == LOCALWARP || (yGlobal && gmWarp)) {
        av1g_warp_ctx w{};
        for (int l = 0; l < 2; l++) {
            int ref = (l == 0 || isCompound) ? RefFrame[l] : RefFrame[0];
            if (l == 1 && !isCompound) ref = RefFrame[0];
            for (int k = 0; k < 6; k++) w.gm_params[l][k] = fh.gm_params[ref][k];
            w.gm_type[l] = (uint8_t)fh.gm_type[ref];
            w.y_mode[l] = (uint8_t)YMode;
            w.ref_is_scaled[l] = IsScaled[ref];
        }
        if (!isCompound) {
            w.gm_type[1] = w.gm_type[0];
            w.ref_is_scaled[1] = 0;
        }
        if (motion_mode == LOCALWARP) {
            for (int k = 0; k < 6; k++) w.local_warp_params[k] = LocalWarpParams[k];
            w.local_valid = (uint8_t)LocalValid;
        } else {
            w.local_warp_params[2] = w.local_warp_params[5] = 1 << 16;
            w.local_valid = 0;
        }
        w.force_integer_mv = (uint8_t)fh.force_integer_mv;
        warp = (int)out.warps.size();
        out.warps.push_back(w);
    }
    // OBMC neighbours (§7.11.3.10): the above row, then the left column
    uint32_t obmcFirst = (uint32_t)out.neighbours.size();
    int nAbove = 0, nLeft = 0;
    if (motion_mode == OBMC) {
        if (AvailU) {
            int n = 0, nLimit = std::min(4, (int)Mi_Width_Log2[MiSize]);
            for (int x4 = MiCol; n < nLimit && x4 < std::min(MiCols, MiCol + bw4);) {
                int candRow = MiRow - 1, candCol = x4 | 1;
                size_t i = cell(candRow, candCol);
                int candSz = MiSizes[i];
                int step4 = clip3(2, 16, Num_4x4_Blocks_Wide[candSz]);
                if (RefFrames[i * 2] > INTRA_FRAME) {
                    n++;
                    av1g_obmc_neighbour nb{};
                    nb.mv[0] = Mvs[i * 4];
                    nb.mv[1] = Mvs[i * 4 + 1];
                    nb.axis_pos4 = (uint16_t)x4;
                    nb.ref = (uint8_t)(RefFrames[i * 2] - 1);
                    nb.step4 = (uint8_t)step4;
                    nb.filter_x = InterpFilters[i * 2 + 1];
                    nb.filter_y = InterpFilters[i * 2];
                    out.neighbours.push_back(nb);
                    nAbove++;
                }
                x4 += step4;
            }
        }
        if (AvailL) {
            int n = 0, nLimit = std::min(4, (int)Mi_Height_Log2[MiSize]);
            for (int y4 = MiRow; n < nLimit && y4 < std::min(MiRows, MiRow + bh4);) {
                int candCol = MiCol - 1, candRow = y4 | 1;
                size_t i = cell(candRow, candCol);
                int candSz = MiSizes[i];
                int step4 = clip3(2, 16, Num_4x4_Blocks_High[candSz]);
                if (RefFrames[i * 2] > INTRA_FRAME) {
                    n++;
                    av1g_obmc_neighbour nb{};
                    nb.mv[0] = Mvs[i * 4];
                    nb.mv[1] = Mvs[i * 4 + 1];
                    nb.axis_pos4 = (uint16_t)y4;
                    nb.ref = (uint8_t)(RefFrames[i * 2] - 1);
                    nb.step4 = (uint8_t)step4;
                    nb.filter_x = InterpFilters[i * 2 + 1];
                    nb.filter_y = InterpFilters[i * 2];
                    out.neighbours.push_back(nb);
                    nLeft++;
                }
                y4 += step4;
            }
        }
    }
    int fwd = 0, bck = 0;
    if (isCompound && compound_type == COMPOUND_DISTANCE) distance_weights(&fwd, &bck);
    int sbMask = sb128 ? 31 : 15;
    int subBlockMiRow = MiRow & sbMask, subBlockMiCol = MiCol & sbMask;
    for (int plane = 0; plane < 1 + HasChroma * 2; plane++) {
        int planeSz = plane_residual_size(MiSize, plane);
        if (planeSz >= BLOCK_INVALID) continue;
        int num4x4W = Num_4x4_Blocks_Wide[planeSz], num4x4H = Num_4x4_Blocks_High[planeSz];
        int subX = plane ? ssx : 0, subY = plane ? ssy : 0;
        int baseX = (MiCol >> subX) * 4, baseY = (MiRow >> subY) * 4;
        int candRow = (MiRow >> subY) << subY, candCol = (MiCol >> subX) << subX;
        if (isII) {
            // the intra half (drawn by the intra pass, then blended with the inter half)
            static const uint8_t ii_to_intra[4] = {DC_PRED, V_PRED, H_PRED, SMOOTH_PRED};
            av1g_intra_tu t{};
            t.x = (uint16_t)baseX;
            t.y = (uint16_t)baseY;
            t.plane = (uint8_t)plane;
            t.tx_size = (uint8_t)find_tx_size(num4x4W * 4, num4x4H * 4);
            t.mode = ii_to_intra[interintra_mode];
            t.filter_intra_mode = 255;
            if (plane == 0 ? AvailU : AvailUChroma) t.flags |= AV1G_INTRA_HAVE_ABOVE;
            if (plane == 0 ? AvailL : AvailLChroma) t.flags |= AV1G_INTRA_HAVE_LEFT;
            if (block_decoded(plane, (subBlockMiRow >> subY) - 1, (subBlockMiCol >> subX) + num4x4W))
                t.flags |= AV1G_INTRA_HAVE_ABOVE_RIGHT;
            if (block_decoded(plane, (subBlockMiRow >> subY) + num4x4H, (subBlockMiCol >> subX) - 1))
                t.flags |= AV1G_INTRA_HAVE_BELOW_LEFT;
            if (seq.enable_intra_edge_filter) t.flags |= AV1G_INTRA_EDGE_FILTER;
            if (get_filter_type(plane)) t.flags |= AV1G_INTRA_FILTER_TYPE;
            t.interintra = wedge_interintra ? 2 : 1;
            t.interintra_mode = (uint8_t)interintra_mode;
            t.wedge_index = (uint8_t)wedge_index;
            t.mi_size = (uint8_t)MiSize;
            t.res.x = t.x;
            t.res.y = t.y;
            t.res.plane = t.plane;
            t.res.tx_size = t.tx_size;
            out.intra_tus.push_back(t);
        }
        int predW = bw_of(MiSize) >> subX, predH = bh_of(MiSize) >> subY;
        bool someUseIntra = false;
        for (int r = 0; r < (num4x4H << subY); r++)
            for (int c = 0; c < (num4x4W << subX); c++) {
                int rr = candRow + r, cc = candCol + c;
                if (rr < MiRows && cc < MiCols && RefFrames[cell(rr, cc) * 2] == INTRA_FRAME) someUseIntra = true;
            }
        if (someUseIntra) {
            predW = num4x4W * 4;
            predH = num4x4H * 4;
            candRow = MiRow;
            candCol = MiCol;
        }
        int r = 0;
        for (int y = 0; y < num4x4H * 4; y += predH, r++) {
            int c = 0;
            for (int x = 0; x < num4x4W * 4; x += predW, c++) {
                size_t ci = cell(std::min(MiRows - 1, candRow + r), std::min(MiCols - 1, candCol + c));
                int cRef0 = RefFrames[ci * 2], cRef1 = RefFrames[ci * 2 + 1];
                av1g_inter_pred p{};
                p.x = (uint16_t)(baseX + x);
                p.y = (uint16_t)(baseY + y);
                p.w = (uint16_t)predW;
                p.h = (uint16_t)predH;
                p.plane = (uint8_t)plane;
                bool own = (int)ci == (int)cell(MiRow, MiCol) || someUseIntra;
                bool cComp = cRef1 > INTRA_FRAME;
                p.kind = isII && own ? AV1G_INTER_INTRA : (cComp ? AV1G_INTER_COMPOUND : AV1G_INTER_SINGLE);
                p.motion_mode = (uint8_t)motion_mode;
                p.filter_x = InterpFilters[ci * 2 + 1];
                p.filter_y = InterpFilters[ci * 2];
                p.ref[0] = (uint8_t)(cRef0 - 1);
                p.ref[1] = (uint8_t)(cComp ? cRef1 - 1 : 0);
                p.compound_type = (uint8_t)(cComp ? compound_type : COMPOUND_AVERAGE);
                p.mv[0][0] = Mvs[ci * 4];
                p.mv[0][1] = Mvs[ci * 4 + 1];
                p.mv[1][0] = cComp ? Mvs[ci * 4 + 2] : 0;
                p.mv[1][1] = cComp ? Mvs[ci * 4 + 3] : 0;
                p.mi_size = (uint8_t)MiSize;
                p.wedge_index = (uint8_t)wedge_index;
                p.wedge_sign = (uint8_t)(isII ? 0 : wedge_sign);
                p.mask_type = (uint8_t)mask_type;
                p.interintra_mode = (uint8_t)interintra_mode;
                p.wedge_interintra = (uint8_t)wedge_interintra;
                p.fwd_weight = (uint8_t)fwd;
                p.bck_weight = (uint8_t)bck;
                p.warp = own ? warp : -1;
                p.obmc_first = obmcFirst;
                p.obmc_above = (uint8_t)nAbove;
                p.obmc_left = (uint8_t)nLeft;
                p.avail_u = AvailU;
                p.avail_l = AvailL;
                p.plane_residual_ge_8x8 = planeSz >= BLOCK_8X8;  // block-size ordinal, as the specification compares
                p.mi_width_log2 = (uint8_t)Mi_Width_Log2[MiSize];
                p.mi_height_log2 = (uint8_t)Mi_Height_Log2[MiSize];
                p.mi_row = (uint16_t)MiRow;
                p.mi_col = (uint16_t)MiCol;
                if (!own) p.motion_mode = SIMPLE;
                out.inter_preds.push_back(p);
            }
        }
    }
}

}  // namespace

// ===========================================================================
// entry
// ===========================================================================

av1g_status walk_frame(const av1g_sequence_header& seq, const av1g_parsed_frame_header& fh,
                       const av1g_ref_state& refs, const SlotParse* slots, const std::vector<TileData>& tiles,
                       FrameOut& out, std::string& err) {
    Walker w(seq, fh, refs, slots, out);
    try {
        w.setup_frame();
        // §8.3.1 frame-start CDFs
        Cdfs start;
        if (fh.primary_ref_frame != 7) {
            const SlotParse& sp = slots[fh.ref_frame_idx[fh.primary_ref_frame]];
            if (!sp.valid) throw WalkError("walker: primary reference slot holds no frame");
            start = sp.cdfs;
            cdfs_zero_counts(start);
        } else {
            cdfs_init(start, fh.base_q_idx);
        }
        int numTiles = fh.tile_cols * fh.tile_rows;
        if ((int)tiles.size() != numTiles) throw WalkError("walker: tile count does not match the header");
        out.have_end_cdfs = false;
        out.tiles_in_sync = true;
        for (int t = 0; t < numTiles; t++) {
            w.cdf = start;
            w.decode_tile(t / fh.tile_cols, t % fh.tile_cols, tiles[t]);
            // §8.2.4 exit_symbol: the tile's data ends with a 1 bit at the
            // trailing position and zeros after it; a walk that consumed a
            // different number of symbols lands elsewhere.
            uint64_t tb = 0, pe = 0;
            av1g_symbol_decoder sd = w.sd;
            if (av1g_symbol_exit(&sd, &tb, &pe) != AV1G_OK) {
                out.tiles_in_sync = false;
            } else {
                const uint8_t* p = tiles[t].data;
                bool okb = tb < tiles[t].size * 8 && ((p[tb >> 3] >> (7 - (tb & 7))) & 1);
                for (uint64_t b = tb + 1; okb && b < tiles[t].size * 8; b++)
                    if ((p[b >> 3] >> (7 - (b & 7))) & 1) okb = false;
                if (!okb) out.tiles_in_sync = false;
            }
            if (!fh.disable_frame_end_update_cdf && t == fh.context_update_tile_id) {
                out.end_cdfs = w.cdf;
                out.have_end_cdfs = true;
            }
        }
        if (!out.have_end_cdfs) {
            out.end_cdfs = start;
            out.have_end_cdfs = true;
        }
    } catch (const std::exception& e) {
        err = e.what();
        return AV1G_EINVAL;
    }
    // grids the engine and later frames read
    size_t cells = (size_t)w.MiRows * w.MiCols;
    out.mi_size.resize(cells);
    for (size_t i = 0; i < cells; i++) out.mi_size[i] = w.MiSizes[i] >= BLOCK_INVALID ? 0 : w.MiSizes[i];
    out.skip = w.Skips;
    out.is_inter = w.IsInters;
    out.y_mode = w.YModes;
    out.tx_size = w.TxSizes;
    out.inter_tx_size = w.InterTxSizes;
    out.ref_frame0.resize(cells);
    out.segment_id.resize(cells);
    for (size_t i = 0; i < cells; i++) {
        out.ref_frame0[i] = w.RefFrames[i * 2];
        out.segment_id[i] = (int8_t)w.SegmentIds[i];
    }
    out.delta_lf = w.DeltaLFs;
    out.ref_frames = w.RefFrames;
    out.mvs = w.Mvs;
    out.segment_map = w.SegmentIds;
    return AV1G_OK;
}

void FrameOut::fill_desc(av1g_frame_desc& d) const {
    std::memset(&d, 0, sizeof d);
    d.hdr = &hdr;
    d.quant = &quant;
    d.grid.mi_size = mi_size.data();
    d.grid.skip = skip.data();
    d.grid.is_inter = is_inter.data();
    d.grid.ref_frame0 = ref_frame0.data();
    d.grid.y_mode = y_mode.data();
    d.grid.segment_id = segment_id.data();
    d.grid.delta_lf = delta_lf.data();
    d.grid.tx_size = tx_size.data();
    d.grid.inter_tx_size = inter_tx_size.data();
    d.cdef_idx = cdef_idx.data();
    for (int p = 0; p < 3; p++) d.lr_units[p] = lr_units[p].empty() ? nullptr : lr_units[p].data();
    d.inter_preds = inter_preds.data();
    d.num_inter_preds = (int32_t)inter_preds.size();
    d.neighbours = neighbours.data();
    d.num_neighbours = (int32_t)neighbours.size();
    d.warps = warps.data();
    d.num_warps = (int32_t)warps.size();
    d.inter_tus = inter_tus.data();
    d.num_inter_tus = (int32_t)inter_tus.size();
    d.intra_tus = intra_tus.data();
    d.num_intra_tus = (int32_t)intra_tus.size();
    d.palette_maps = palette_maps.data();
    d.palette_map_bytes = (int64_t)palette_maps.size();
    d.coeffs = coeffs.data();
    d.num_coeffs = (int64_t)coeffs.size();
}

}  // namespace av1w
