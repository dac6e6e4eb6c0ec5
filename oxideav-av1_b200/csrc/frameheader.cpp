// frameheader.cpp — the §5.9 uncompressed header, the §7.20 header state of
// the reference slots and the §5.11.1 tile group layout (host code).
//
// Follows parse_frame_header_with_refs (src/frame_header.rs:726-1520) and the
// parameter readers it calls: frame size / superres / render size
// (frame_header.rs:1692-2110), tile_info (src/tile_info.rs:359), quantization,
// segmentation, delta q / lf, loop filter, CDEF, loop restoration, tx mode,
// skip mode, global motion and film grain (src/uncompressed_header_tail.rs).
// Accepted inputs and rejections are the reference's: a decoder model in the
// sequence header is rejected as the reference does (temporal_point_info),
// and so are frame ids longer than 16 bits.  The syntax itself is the AV1
// specification's; pf (the post-filter header the kernels take) is filled
// from the parsed values, film grain resolved through the reference slots
// when update_grain is 0 (frame_driver.rs:1060-1075).
#include <algorithm>
#include <cstring>

#include "av1g.h"

namespace av1g {
void set_framing_error(int code, const char* text);
}

namespace {

enum { INTRA = 0, LAST = 1, LAST2 = 2, LAST3 = 3, GOLDEN = 4, BWDREF = 5, ALTREF2 = 6, ALTREF = 7 };
enum { KEY_FRAME = 0, INTER_FRAME = 1, INTRA_ONLY_FRAME = 2, SWITCH_FRAME = 3 };
constexpr int kPrimaryRefNone = 7;
constexpr int kWarpPrec = 16;  // WARPEDMODEL_PREC_BITS

struct Fail {
    int code;
    const char* what;
};

struct Reader {
    const uint8_t* p;
    size_t n;
    size_t pos = 0;
    uint32_t f(int k) {
        uint32_t v = 0;
        for (int i = 0; i < k; i++) {
            if (pos >= n * 8) throw Fail{AV1G_FE_UNEXPECTED_END, "frame header: unexpected end of data"};
            v = (v << 1) | ((p[pos >> 3] >> (7 - (pos & 7))) & 1);
            pos++;
        }
        return v;
    }
    bool b() { return f(1) != 0; }
    int su(int k) {
        int v = (int)f(k);
        const int sign = 1 << (k - 1);
        return (v & sign) ? v - 2 * sign : v;
    }
    uint32_t ns(uint32_t n_) {
        int w = 0;
        for (uint32_t x = n_; x; x >>= 1) w++;
        const uint32_t m = (1u << w) - n_;
        const uint32_t v = f(w - 1);
        return v < m ? v : (v << 1) - m + f(1);
    }
};

int relative_dist(const av1g_sequence_header& s, int a, int b) {
    if (!s.enable_order_hint) return 0;
    const int d = a - b, m = 1 << (s.order_hint_bits - 1);
    return (d & (m - 1)) - (d & m);
}

int tile_log2(int blk, int target) {
    int k = 0;
    while ((blk << k) < target) k++;
    return k;
}

// §5.9.5-§5.9.8 frame size, superres, MiCols / MiRows; §5.9.6 render size
void superres_and_image_size(Reader& r, const av1g_sequence_header& s, av1g_parsed_frame_header& h) {
    av1g_frame_header& pf = h.pf;
    pf.use_superres = s.enable_superres ? r.b() : 0;
    h.superres_denom = pf.use_superres ? (int)r.f(3) + 9 : 8;
    pf.upscaled_width = pf.frame_width;
    pf.frame_width = (pf.upscaled_width * 8 + h.superres_denom / 2) / h.superres_denom;
    pf.mi_cols = 2 * ((pf.frame_width + 7) >> 3);
    pf.mi_rows = 2 * ((pf.frame_height + 7) >> 3);
}

void frame_size(Reader& r, const av1g_sequence_header& s, av1g_parsed_frame_header& h) {
    if (h.frame_size_override_flag) {
        h.pf.frame_width = (int)r.f(s.frame_width_bits_minus_1 + 1) + 1;
        h.pf.frame_height = (int)r.f(s.frame_height_bits_minus_1 + 1) + 1;
    } else {
        h.pf.frame_width = (int)s.max_frame_width_minus_1 + 1;
        h.pf.frame_height = (int)s.max_frame_height_minus_1 + 1;
    }
    superres_and_image_size(r, s, h);
}

void render_size(Reader& r, av1g_parsed_frame_header& h) {
    if (r.b()) {
        h.render_width = (int)r.f(16) + 1;
        h.render_height = (int)r.f(16) + 1;
    } else {
        h.render_width = h.pf.upscaled_width;
        h.render_height = h.pf.frame_height;
    }
}

void frame_size_with_refs(Reader& r, const av1g_sequence_header& s, const av1g_ref_state& st,
                          av1g_parsed_frame_header& h) {
    for (int i = 0; i < 7; i++) {
        if (r.b()) {  // found_ref
            const int k = h.ref_frame_idx[i];
            h.pf.upscaled_width = st.upscaled_width[k];
            h.pf.frame_width = h.pf.upscaled_width;
            h.pf.frame_height = st.frame_height[k];
            h.render_width = st.render_width[k];
            h.render_height = st.render_height[k];
            superres_and_image_size(r, s, h);
            return;
        }
    }
    frame_size(r, s, h);
    render_size(r, h);
}

// §5.9.15 tile_info
void tile_info(Reader& r, const av1g_sequence_header& s, av1g_parsed_frame_header& h) {
    const int mi_cols = h.pf.mi_cols, mi_rows = h.pf.mi_rows;
    // a size taken from a reference slot that never held a frame
    if (mi_cols <= 0 || mi_rows <= 0) throw Fail{AV1G_FE_FRAME_HEADER_INVALID, "frame header: empty frame size"};
    const bool sb128 = s.use_128x128_superblock;
    const int sb_cols = sb128 ? (mi_cols + 31) >> 5 : (mi_cols + 15) >> 4;
    const int sb_rows = sb128 ? (mi_rows + 31) >> 5 : (mi_rows + 15) >> 4;
    const int sb_shift = sb128 ? 5 : 4, sb_size = sb_shift + 2;
    const int max_tile_width_sb = 4096 >> sb_size;
    int max_tile_area_sb = (4096 * 2304) >> (2 * sb_size);
    const int min_log2_tile_cols = tile_log2(max_tile_width_sb, sb_cols);
    const int max_log2_tile_cols = tile_log2(1, std::min(sb_cols, 64));
    const int max_log2_tile_rows = tile_log2(1, std::min(sb_rows, 64));
    const int min_log2_tiles = std::max(min_log2_tile_cols, tile_log2(max_tile_area_sb, sb_rows * sb_cols));
    int i;
    if (r.b()) {  // uniform_tile_spacing_flag
        h.tile_cols_log2 = min_log2_tile_cols;
        while (h.tile_cols_log2 < max_log2_tile_cols && r.b()) h.tile_cols_log2++;
        const int tw = (sb_cols + (1 << h.tile_cols_log2) - 1) >> h.tile_cols_log2;
        i = 0;
        for (int start = 0; start < sb_cols; start += tw) h.mi_col_starts[i++] = start << sb_shift;
        h.mi_col_starts[i] = mi_cols;
        h.tile_cols = i;
        const int min_log2_tile_rows = std::max(min_log2_tiles - h.tile_cols_log2, 0);
        h.tile_rows_log2 = min_log2_tile_rows;
        while (h.tile_rows_log2 < max_log2_tile_rows && r.b()) h.tile_rows_log2++;
        const int th = (sb_rows + (1 << h.tile_rows_log2) - 1) >> h.tile_rows_log2;
        i = 0;
        for (int start = 0; start < sb_rows; start += th) h.mi_row_starts[i++] = start << sb_shift;
        h.mi_row_starts[i] = mi_rows;
        h.tile_rows = i;
    } else {
        int widest = 0, start = 0;
        for (i = 0; start < sb_cols; i++) {
            if (i >= 64) throw Fail{AV1G_FE_FRAME_HEADER_INVALID, "frame header: more than 64 tile columns"};
            h.mi_col_starts[i] = start << sb_shift;
            const int size = (int)r.ns((uint32_t)std::min(sb_cols - start, max_tile_width_sb)) + 1;
            widest = std::max(size, widest);
            start += size;
        }
        h.mi_col_starts[i] = mi_cols;
        h.tile_cols = i;
        h.tile_cols_log2 = tile_log2(1, h.tile_cols);
        max_tile_area_sb = min_log2_tiles > 0 ? (sb_rows * sb_cols) >> (min_log2_tiles + 1) : sb_rows * sb_cols;
        const int max_tile_height_sb = std::max(max_tile_area_sb / widest, 1);
        start = 0;
        for (i = 0; start < sb_rows; i++) {
            if (i >= 64) throw Fail{AV1G_FE_FRAME_HEADER_INVALID, "frame header: more than 64 tile rows"};
            h.mi_row_starts[i] = start << sb_shift;
            start += (int)r.ns((uint32_t)std::min(sb_rows - start, max_tile_height_sb)) + 1;
        }
        h.mi_row_starts[i] = mi_rows;
        h.tile_rows = i;
        h.tile_rows_log2 = tile_log2(1, h.tile_rows);
    }
    if (h.tile_cols_log2 > 0 || h.tile_rows_log2 > 0) {
        h.context_update_tile_id = (int)r.f(h.tile_rows_log2 + h.tile_cols_log2);
        h.tile_size_bytes = (int)r.f(2) + 1;
    } else {
        h.context_update_tile_id = 0;
        h.tile_size_bytes = 4;
    }
}

int read_delta_q(Reader& r) { return r.b() ? r.su(7) : 0; }

void quantization(Reader& r, const av1g_sequence_header& s, av1g_parsed_frame_header& h) {
    h.base_q_idx = (int)r.f(8);
    h.delta_q_y_dc = read_delta_q(r);
    if (s.num_planes > 1) {
        const bool diff_uv = s.separate_uv_delta_q ? r.b() : false;
        h.delta_q_u_dc = read_delta_q(r);
        h.delta_q_u_ac = read_delta_q(r);
        if (diff_uv) {
            h.delta_q_v_dc = read_delta_q(r);
            h.delta_q_v_ac = read_delta_q(r);
        } else {
            h.delta_q_v_dc = h.delta_q_u_dc;
            h.delta_q_v_ac = h.delta_q_u_ac;
        }
    }
    h.using_qmatrix = r.b();
    if (h.using_qmatrix) {
        h.qm_y = (int)r.f(4);
        h.qm_u = (int)r.f(4);
        h.qm_v = s.separate_uv_delta_q ? (int)r.f(4) : h.qm_u;
    }
}

void segmentation(Reader& r, const av1g_ref_state& st, av1g_parsed_frame_header& h) {
    static const int bits[8] = {8, 6, 6, 6, 6, 3, 0, 0};
    static const int sgn[8] = {1, 1, 1, 1, 1, 0, 0, 0};
    static const int mx[8] = {255, 63, 63, 63, 63, 7, 0, 0};
    memset(h.seg_feature_enabled, 0, sizeof h.seg_feature_enabled);
    memset(h.seg_feature_data, 0, sizeof h.seg_feature_data);
    h.segmentation_enabled = r.b();
    if (!h.segmentation_enabled) return;
    if (h.primary_ref_frame == kPrimaryRefNone) {
        h.segmentation_update_map = 1;
        h.segmentation_temporal_update = 0;
        h.segmentation_update_data = 1;
    } else {
        h.segmentation_update_map = r.b();
        if (h.segmentation_update_map) h.segmentation_temporal_update = r.b();
        h.segmentation_update_data = r.b();
    }
    if (h.segmentation_update_data) {
        for (int i = 0; i < 8; i++)
            for (int j = 0; j < 8; j++) {
                int v = 0;
                h.seg_feature_enabled[i][j] = r.b();
                if (h.seg_feature_enabled[i][j]) {
                    v = sgn[j] ? r.su(1 + bits[j]) : (int)r.f(bits[j]);
                    v = std::min(std::max(v, sgn[j] ? -mx[j] : 0), mx[j]);
                }
                h.seg_feature_data[i][j] = (int16_t)v;
            }
    } else {  // load_previous(): the primary reference frame's features
        const int k = h.ref_frame_idx[h.primary_ref_frame];
        memcpy(h.seg_feature_enabled, st.seg_feature_enabled[k], sizeof h.seg_feature_enabled);
        memcpy(h.seg_feature_data, st.seg_feature_data[k], sizeof h.seg_feature_data);
    }
}

void loop_filter(Reader& r, const av1g_sequence_header& s, const av1g_ref_state& st, av1g_parsed_frame_header& h) {
    av1g_frame_header& pf = h.pf;
    static const int8_t def_ref[8] = {1, 0, 0, 0, -1, 0, -1, -1};
    if (h.primary_ref_frame == kPrimaryRefNone) {
        memcpy(pf.lf_ref_deltas, def_ref, 8);
        memset(pf.lf_mode_deltas, 0, 2);
    } else {
        const int k = h.ref_frame_idx[h.primary_ref_frame];
        memcpy(pf.lf_ref_deltas, st.lf_ref_deltas[k], 8);
        memcpy(pf.lf_mode_deltas, st.lf_mode_deltas[k], 2);
    }
    if (pf.coded_lossless || pf.allow_intrabc) {
        memcpy(pf.lf_ref_deltas, def_ref, 8);
        memset(pf.lf_mode_deltas, 0, 2);
        return;
    }
    pf.lf_level[0] = (uint8_t)r.f(6);
    pf.lf_level[1] = (uint8_t)r.f(6);
    if (s.num_planes > 1 && (pf.lf_level[0] || pf.lf_level[1])) {
        pf.lf_level[2] = (uint8_t)r.f(6);
        pf.lf_level[3] = (uint8_t)r.f(6);
    }
    pf.lf_sharpness = (uint8_t)r.f(3);
    pf.lf_delta_enabled = r.b();
    if (pf.lf_delta_enabled && r.b()) {  // loop_filter_delta_update
        for (int i = 0; i < 8; i++)
            if (r.b()) pf.lf_ref_deltas[i] = (int8_t)r.su(7);
        for (int i = 0; i < 2; i++)
            if (r.b()) pf.lf_mode_deltas[i] = (int8_t)r.su(7);
    }
}

void cdef(Reader& r, const av1g_sequence_header& s, av1g_parsed_frame_header& h) {
    av1g_frame_header& pf = h.pf;
    if (pf.coded_lossless || pf.allow_intrabc || !s.enable_cdef) {
        pf.cdef_short_circuited = 1;
        pf.cdef_damping = 3;
        return;
    }
    pf.cdef_damping = (uint8_t)(r.f(2) + 3);
    pf.cdef_bits = (uint8_t)r.f(2);
    for (int i = 0; i < (1 << pf.cdef_bits); i++) {
        pf.cdef_y_pri[i] = (uint8_t)r.f(4);
        pf.cdef_y_sec[i] = (uint8_t)r.f(2);
        if (pf.cdef_y_sec[i] == 3) pf.cdef_y_sec[i]++;
        if (s.num_planes > 1) {
            pf.cdef_uv_pri[i] = (uint8_t)r.f(4);
            pf.cdef_uv_sec[i] = (uint8_t)r.f(2);
            if (pf.cdef_uv_sec[i] == 3) pf.cdef_uv_sec[i]++;
        }
    }
}

void restoration(Reader& r, const av1g_sequence_header& s, av1g_parsed_frame_header& h) {
    av1g_frame_header& pf = h.pf;
    if (h.all_lossless || pf.allow_intrabc || !s.enable_restoration) return;
    static const uint8_t remap[4] = {0, 3, 1, 2};  // Remap_Lr_Type: NONE, SWITCHABLE, WIENER, SGRPROJ
    bool chroma = false;
    for (int i = 0; i < s.num_planes; i++) {
        pf.lr_type[i] = remap[r.f(2)];
        if (pf.lr_type[i]) {
            pf.uses_lr = 1;
            if (i > 0) chroma = true;
        }
    }
    if (!pf.uses_lr) return;
    if (s.use_128x128_superblock) {
        h.lr_unit_shift = (int)r.f(1) + 1;
    } else {
        h.lr_unit_shift = (int)r.f(1);
        if (h.lr_unit_shift) h.lr_unit_shift += (int)r.f(1);
    }
    pf.lr_unit_size[0] = 256 >> (2 - h.lr_unit_shift);
    h.lr_uv_shift = (s.subsampling_x && s.subsampling_y && chroma) ? (int)r.f(1) : 0;
    pf.lr_unit_size[1] = pf.lr_unit_size[2] = pf.lr_unit_size[0] >> h.lr_uv_shift;
}

// §5.9.22 skip_mode_params
void skip_mode(Reader& r, const av1g_sequence_header& s, const av1g_ref_state& st, av1g_parsed_frame_header& h) {
    bool allowed = false;
    if (!(h.frame_type == KEY_FRAME || h.frame_type == INTRA_ONLY_FRAME) && h.reference_select && s.enable_order_hint) {
        int fwd = -1, bwd = -1, fwd_hint = 0, bwd_hint = 0;
        for (int i = 0; i < 7; i++) {
            const int hint = st.order_hint[h.ref_frame_idx[i]];
            if (relative_dist(s, hint, h.order_hint) < 0) {
                if (fwd < 0 || relative_dist(s, hint, fwd_hint) > 0) {
                    fwd = i;
                    fwd_hint = hint;
                }
            } else if (relative_dist(s, hint, h.order_hint) > 0) {
                if (bwd < 0 || relative_dist(s, hint, bwd_hint) < 0) {
                    bwd = i;
                    bwd_hint = hint;
                }
            }
        }
        if (fwd >= 0 && bwd >= 0) {
            allowed = true;
            h.skip_mode_frame[0] = LAST + std::min(fwd, bwd);
            h.skip_mode_frame[1] = LAST + std::max(fwd, bwd);
        } else if (fwd >= 0) {
            int fwd2 = -1, fwd2_hint = 0;
            for (int i = 0; i < 7; i++) {
                const int hint = st.order_hint[h.ref_frame_idx[i]];
                if (relative_dist(s, hint, fwd_hint) < 0 && (fwd2 < 0 || relative_dist(s, hint, fwd2_hint) > 0)) {
                    fwd2 = i;
                    fwd2_hint = hint;
                }
            }
            if (fwd2 >= 0) {
                allowed = true;
                h.skip_mode_frame[0] = LAST + std::min(fwd, fwd2);
                h.skip_mode_frame[1] = LAST + std::max(fwd, fwd2);
            }
        }
    }
    h.skip_mode_present = allowed ? r.b() : 0;
    if (!h.skip_mode_present) h.skip_mode_frame[0] = h.skip_mode_frame[1] = 0;
}

int inverse_recenter(int r, int v) {
    if (v > 2 * r) return v;
    return (v & 1) ? r - ((v + 1) >> 1) : r + (v >> 1);
}

int decode_subexp(Reader& r, int num_syms) {
    int i = 0, mk = 0;
    const int k = 3;
    for (;;) {
        const int b2 = i ? k + i - 1 : k, a = 1 << b2;
        if (num_syms <= mk + 3 * a) return (int)r.ns((uint32_t)(num_syms - mk)) + mk;
        if (r.b()) {
            i++;
            mk += a;
        } else {
            return (int)r.f(b2) + mk;
        }
    }
}

int decode_signed_subexp_with_ref(Reader& r, int low, int high, int ref) {
    const int mx = high - low;
    ref -= low;
    const int v = decode_subexp(r, mx);
    const int x = (ref << 1) <= mx ? inverse_recenter(ref, v) : mx - 1 - inverse_recenter(mx - 1 - ref, v);
    return x + low;
}

// §5.9.24 global_motion_params
void global_motion(Reader& r, const av1g_ref_state& st, av1g_parsed_frame_header& h) {
    enum { IDENTITY = 0, TRANSLATION = 1, ROTZOOM = 2, AFFINE = 3 };
    int prev[8][6];
    for (int ref = LAST; ref <= ALTREF; ref++) {
        h.gm_type[ref] = IDENTITY;
        for (int i = 0; i < 6; i++) {
            h.gm_params[ref][i] = (i % 3 == 2) ? 1 << kWarpPrec : 0;
            prev[ref][i] = h.primary_ref_frame == kPrimaryRefNone
                               ? h.gm_params[ref][i]
                               : st.gm_params[h.ref_frame_idx[h.primary_ref_frame]][ref][i];
        }
    }
    if (h.frame_type == KEY_FRAME || h.frame_type == INTRA_ONLY_FRAME) return;
    auto param = [&](int type, int ref, int idx) {
        int abs_bits = 12, prec_bits = 15;  // GM_ABS_ALPHA_BITS, GM_ALPHA_PREC_BITS
        if (idx < 2) {
            if (type == TRANSLATION) {
                abs_bits = 9 - !h.allow_high_precision_mv;   // GM_ABS_TRANS_ONLY_BITS
                prec_bits = 3 - !h.allow_high_precision_mv;  // GM_TRANS_ONLY_PREC_BITS
            } else {
                abs_bits = 12;  // GM_ABS_TRANS_BITS
                prec_bits = 6;  // GM_TRANS_PREC_BITS
            }
        }
        const int prec_diff = kWarpPrec - prec_bits;
        const int round = (idx % 3) == 2 ? 1 << kWarpPrec : 0;
        const int sub = (idx % 3) == 2 ? 1 << prec_bits : 0;
        const int mx = 1 << abs_bits;
        const int rr = (prev[ref][idx] >> prec_diff) - sub;
        h.gm_params[ref][idx] = decode_signed_subexp_with_ref(r, -mx, mx + 1, rr) * (1 << prec_diff) + round;
    };
    for (int ref = LAST; ref <= ALTREF; ref++) {
        int type = IDENTITY;
        if (r.b()) {  // is_global
            if (r.b()) type = ROTZOOM;
            else type = r.b() ? TRANSLATION : AFFINE;
        }
        h.gm_type[ref] = type;
        if (type >= ROTZOOM) {
            param(type, ref, 2);
            param(type, ref, 3);
            if (type == AFFINE) {
                param(type, ref, 4);
                param(type, ref, 5);
            } else {
                h.gm_params[ref][4] = -h.gm_params[ref][3];
                h.gm_params[ref][5] = h.gm_params[ref][2];
            }
        }
        if (type >= TRANSLATION) {
            param(type, ref, 0);
            param(type, ref, 1);
        }
    }
}

// §5.9.30 film_grain_params (into pf.film_grain; update_grain == 0 loads the
// named reference slot's parameters with the new seed)
void film_grain(Reader& r, const av1g_sequence_header& s, const av1g_ref_state& st, av1g_parsed_frame_header& h) {
    av1g_film_grain& g = h.pf.film_grain;
    memset(&g, 0, sizeof g);
    if (!s.film_grain_params_present || (!h.show_frame && !h.showable_frame)) return;
    g.apply_grain = r.b();
    if (!g.apply_grain) return;
    const uint16_t seed = (uint16_t)r.f(16);
    h.update_grain = h.frame_type == INTER_FRAME ? r.b() : 1;
    if (!h.update_grain) {
        h.film_grain_params_ref_idx = (int)r.f(3);
        g = st.film_grain[h.film_grain_params_ref_idx];
        g.grain_seed = seed;
        g.apply_grain = 1;
        return;
    }
    g.grain_seed = seed;
    g.num_y_points = (uint8_t)r.f(4);
    if (g.num_y_points > 14) throw Fail{AV1G_FE_FRAME_HEADER_INVALID, "frame header: num_y_points above 14"};
    for (int i = 0; i < g.num_y_points; i++) {
        g.point_y_value[i] = (uint8_t)r.f(8);
        g.point_y_scaling[i] = (uint8_t)r.f(8);
    }
    g.chroma_scaling_from_luma = s.mono_chrome ? 0 : r.b();
    if (s.mono_chrome || g.chroma_scaling_from_luma || (s.subsampling_x == 1 && s.subsampling_y == 1 &&
                                                        g.num_y_points == 0)) {
        g.num_cb_points = g.num_cr_points = 0;
    } else {
        g.num_cb_points = (uint8_t)r.f(4);
        if (g.num_cb_points > 10) throw Fail{AV1G_FE_FRAME_HEADER_INVALID, "frame header: num_cb_points above 10"};
        for (int i = 0; i < g.num_cb_points; i++) {
            g.point_cb_value[i] = (uint8_t)r.f(8);
            g.point_cb_scaling[i] = (uint8_t)r.f(8);
        }
        g.num_cr_points = (uint8_t)r.f(4);
        if (g.num_cr_points > 10) throw Fail{AV1G_FE_FRAME_HEADER_INVALID, "frame header: num_cr_points above 10"};
        for (int i = 0; i < g.num_cr_points; i++) {
            g.point_cr_value[i] = (uint8_t)r.f(8);
            g.point_cr_scaling[i] = (uint8_t)r.f(8);
        }
    }
    g.grain_scaling = (uint8_t)(r.f(2) + 8);
    g.ar_coeff_lag = (uint8_t)r.f(2);
    const int npos_luma = 2 * g.ar_coeff_lag * (g.ar_coeff_lag + 1);
    int npos_chroma = npos_luma;
    if (g.num_y_points) {
        npos_chroma = npos_luma + 1;
        for (int i = 0; i < npos_luma; i++) g.ar_coeffs_y_plus_128[i] = (uint8_t)r.f(8);
    }
    if (g.chroma_scaling_from_luma || g.num_cb_points)
        for (int i = 0; i < npos_chroma; i++) g.ar_coeffs_cb_plus_128[i] = (uint8_t)r.f(8);
    if (g.chroma_scaling_from_luma || g.num_cr_points)
        for (int i = 0; i < npos_chroma; i++) g.ar_coeffs_cr_plus_128[i] = (uint8_t)r.f(8);
    g.ar_coeff_shift = (uint8_t)(r.f(2) + 6);
    g.grain_scale_shift = (uint8_t)r.f(2);
    if (g.num_cb_points) {
        g.cb_mult = (uint8_t)r.f(8);
        g.cb_luma_mult = (uint8_t)r.f(8);
        g.cb_offset = (uint16_t)r.f(9);
    }
    if (g.num_cr_points) {
        g.cr_mult = (uint8_t)r.f(8);
        g.cr_luma_mult = (uint8_t)r.f(8);
        g.cr_offset = (uint16_t)r.f(9);
    }
    g.overlap_flag = r.b();
    g.clip_to_restricted_range = r.b();
}

// §7.8 set_frame_refs: ref_frame_idx from last / golden and the order hints
void set_frame_refs(const av1g_sequence_header& s, const av1g_ref_state& st, int last_idx, int gold_idx,
                    int order_hint, int ref_frame_idx[7]) {
    for (int i = 0; i < 7; i++) ref_frame_idx[i] = -1;
    ref_frame_idx[LAST - LAST] = last_idx;
    ref_frame_idx[GOLDEN - LAST] = gold_idx;
    bool used[8] = {};
    used[last_idx] = used[gold_idx] = true;
    const int cur = 1 << (s.order_hint_bits - 1);
    int shifted[8];
    for (int i = 0; i < 8; i++) shifted[i] = cur + relative_dist(s, st.order_hint[i], order_hint);
    auto find_latest_backward = [&]() {
        int ref = -1, latest = 0;
        for (int i = 0; i < 8; i++) {
            const int hint = shifted[i];
            if (!used[i] && hint >= cur && (ref < 0 || hint >= latest)) {
                ref = i;
                latest = hint;
            }
        }
        return ref;
    };
    auto find_earliest_backward = [&]() {
        int ref = -1, earliest = 0;
        for (int i = 0; i < 8; i++) {
            const int hint = shifted[i];
            if (!used[i] && hint >= cur && (ref < 0 || hint < earliest)) {
                ref = i;
                earliest = hint;
            }
        }
        return ref;
    };
    auto find_latest_forward = [&]() {
        int ref = -1, latest = 0;
        for (int i = 0; i < 8; i++) {
            const int hint = shifted[i];
            if (!used[i] && hint < cur && (ref < 0 || hint >= latest)) {
                ref = i;
                latest = hint;
            }
        }
        return ref;
    };
    int ref = find_latest_backward();
    if (ref >= 0) {
        ref_frame_idx[ALTREF - LAST] = ref;
        used[ref] = true;
    }
    ref = find_earliest_backward();
    if (ref >= 0) {
        ref_frame_idx[BWDREF - LAST] = ref;
        used[ref] = true;
    }
    ref = find_earliest_backward();
    if (ref >= 0) {
        ref_frame_idx[ALTREF2 - LAST] = ref;
        used[ref] = true;
    }
    static const int order[5] = {LAST2, LAST3, BWDREF, ALTREF2, ALTREF};
    for (int k = 0; k < 5; k++) {
        const int rf = order[k];
        if (ref_frame_idx[rf - LAST] < 0) {
            ref = find_latest_forward();
            if (ref >= 0) {
                ref_frame_idx[rf - LAST] = ref;
                used[ref] = true;
            }
        }
    }
    // Finally, any remaining references are set to the reference frame with
    // the smallest output order
    ref = -1;
    int earliest = 0;
    for (int i = 0; i < 8; i++) {
        const int hint = shifted[i];
        if (ref < 0 || hint < earliest) {
            ref = i;
            earliest = hint;
        }
    }
    for (int i = 0; i < 7; i++)
        if (ref_frame_idx[i] < 0) ref_frame_idx[i] = ref;
}

void parse(const uint8_t* p, size_t n, const av1g_sequence_header& s, const av1g_ref_state& st,
           av1g_parsed_frame_header& h) {
    Reader r{p, n};
    av1g_frame_header& pf = h.pf;
    pf.bit_depth = s.bit_depth;
    pf.subsampling_x = s.subsampling_x;
    pf.subsampling_y = s.subsampling_y;
    pf.num_planes = s.num_planes;
    pf.matrix_coefficients = s.matrix_coefficients;
    pf.enable_cdef = s.enable_cdef;
    h.frame_to_show_map_idx = -1;
    h.primary_ref_frame = kPrimaryRefNone;
    const int id_len = s.frame_id_numbers_present_flag
                           ? s.additional_frame_id_length_minus_1 + s.delta_frame_id_length_minus_2 + 3
                           : 0;
    if (id_len > 16) throw Fail{AV1G_FE_FRAME_HEADER_INVALID, "frame header: frame id length above 16"};
    bool intra;
    if (s.reduced_still_picture_header) {
        h.frame_type = KEY_FRAME;
        h.show_frame = 1;
        h.showable_frame = 0;
        h.error_resilient_mode = 1;
        intra = true;
    } else {
        h.show_existing_frame = r.b();
        if (h.show_existing_frame) {
            h.frame_to_show_map_idx = (int)r.f(3);
            if (s.decoder_model_info_present_flag && !s.equal_picture_interval)
                throw Fail{AV1G_FE_TEMPORAL_POINT_INFO_UNSUPPORTED, "frame header: temporal_point_info"};
            if (s.frame_id_numbers_present_flag) h.current_frame_id = (int)r.f(id_len);  // display_frame_id
            h.frame_type = st.frame_type[h.frame_to_show_map_idx];
            h.show_frame = 1;
            h.refresh_frame_flags = h.frame_type == KEY_FRAME ? 0xff : 0;
            h.header_bits = (uint32_t)r.pos;
            return;
        }
        h.frame_type = (int)r.f(2);
        intra = h.frame_type == INTRA_ONLY_FRAME || h.frame_type == KEY_FRAME;
        h.show_frame = r.b();
        if (h.show_frame && s.decoder_model_info_present_flag && !s.equal_picture_interval)
            throw Fail{AV1G_FE_TEMPORAL_POINT_INFO_UNSUPPORTED, "frame header: temporal_point_info"};
        h.showable_frame = h.show_frame ? h.frame_type != KEY_FRAME : r.b();
        h.error_resilient_mode =
            (h.frame_type == SWITCH_FRAME || (h.frame_type == KEY_FRAME && h.show_frame)) ? 1 : r.b();
    }
    h.disable_cdf_update = r.b();
    h.allow_screen_content_tools = s.seq_force_screen_content_tools == 2 ? r.b() : s.seq_force_screen_content_tools;
    if (h.allow_screen_content_tools)
        h.force_integer_mv = s.seq_force_integer_mv == 2 ? r.b() : s.seq_force_integer_mv;
    if (intra) h.force_integer_mv = 1;
    if (s.frame_id_numbers_present_flag) h.current_frame_id = (int)r.f(id_len);
    h.frame_size_override_flag =
        h.frame_type == SWITCH_FRAME ? 1 : (s.reduced_still_picture_header ? 0 : r.b());
    h.order_hint = s.order_hint_bits ? (int)r.f(s.order_hint_bits) : 0;
    if (!intra && !h.error_resilient_mode) h.primary_ref_frame = (int)r.f(3);
    if (s.decoder_model_info_present_flag)  // buffer_removal_time: not handled, as in the reference
        throw Fail{AV1G_FE_TEMPORAL_POINT_INFO_UNSUPPORTED, "frame header: decoder model timing is not supported"};
    h.refresh_frame_flags = (h.frame_type == SWITCH_FRAME || (h.frame_type == KEY_FRAME && h.show_frame))
                                ? 0xff
                                : (int)r.f(8);
    if ((!intra || h.refresh_frame_flags != 0xff) && h.error_resilient_mode && s.enable_order_hint)
        for (int i = 0; i < 8; i++) r.f(s.order_hint_bits);  // ref_order_hint[i]
    if (intra) {
        frame_size(r, s, h);
        render_size(r, h);
        if (h.allow_screen_content_tools && pf.upscaled_width == pf.frame_width) pf.allow_intrabc = r.b();
    } else {
        h.frame_refs_short_signaling = s.enable_order_hint ? r.b() : 0;
        if (h.frame_refs_short_signaling) {
            const int last = (int)r.f(3), gold = (int)r.f(3);
            set_frame_refs(s, st, last, gold, h.order_hint, h.ref_frame_idx);
        }
        for (int i = 0; i < 7; i++) {
            if (!h.frame_refs_short_signaling) h.ref_frame_idx[i] = (int)r.f(3);
            if (s.frame_id_numbers_present_flag) r.f(s.delta_frame_id_length_minus_2 + 2);  // delta_frame_id_minus_1
        }
        if (h.frame_size_override_flag && !h.error_resilient_mode) {
            frame_size_with_refs(r, s, st, h);
        } else {
            frame_size(r, s, h);
            render_size(r, h);
        }
        h.allow_high_precision_mv = h.force_integer_mv ? 0 : r.b();
        h.interpolation_filter = r.b() ? 4 : (int)r.f(2);  // is_filter_switchable: SWITCHABLE
        h.is_motion_mode_switchable = r.b();
        h.use_ref_frame_mvs = (h.error_resilient_mode || !s.enable_ref_frame_mvs) ? 0 : r.b();
        for (int i = 0; i < 7; i++) h.order_hints[LAST + i] = st.order_hint[h.ref_frame_idx[i]];
    }
    h.disable_frame_end_update_cdf =
        (s.reduced_still_picture_header || h.disable_cdf_update) ? 1 : r.b();
    tile_info(r, s, h);
    quantization(r, s, h);
    segmentation(r, st, h);
    h.delta_q_present = h.base_q_idx > 0 ? r.b() : 0;
    if (h.delta_q_present) h.delta_q_res = (int)r.f(2);
    if (h.delta_q_present) {
        if (!pf.allow_intrabc) h.delta_lf_present = r.b();
        if (h.delta_lf_present) {
            h.delta_lf_res = (int)r.f(2);
            pf.delta_lf_multi = r.b();
        }
    }
    // CodedLossless / LosslessArray (§5.9.2 with get_qindex(1, segment))
    bool coded_lossless = true;
    for (int seg = 0; seg < 8; seg++) {
        int q = h.base_q_idx;
        if (h.segmentation_enabled && h.seg_feature_enabled[seg][0])
            q = std::min(std::max(h.base_q_idx + h.seg_feature_data[seg][0], 0), 255);
        h.lossless[seg] = q == 0 && !h.delta_q_y_dc && !h.delta_q_u_ac && !h.delta_q_u_dc && !h.delta_q_v_ac &&
                          !h.delta_q_v_dc;
        coded_lossless &= h.lossless[seg] != 0;
    }
    pf.coded_lossless = coded_lossless;
    h.all_lossless = coded_lossless && pf.frame_width == pf.upscaled_width;
    for (int seg = 0; seg < 8; seg++)
        for (int i = 0; i < 4; i++) {  // SEG_LVL_ALT_LF_Y_V .. SEG_LVL_ALT_LF_V
            pf.seg_lf_active[seg][i] = h.segmentation_enabled && h.seg_feature_enabled[seg][1 + i];
            pf.seg_lf_data[seg][i] = pf.seg_lf_active[seg][i] ? h.seg_feature_data[seg][1 + i] : 0;
        }
    loop_filter(r, s, st, h);
    cdef(r, s, h);
    restoration(r, s, h);
    h.tx_mode = coded_lossless ? 0 : (r.b() ? 2 : 1);  // ONLY_4X4, TX_MODE_LARGEST, TX_MODE_SELECT
    h.reference_select = intra ? 0 : r.b();
    skip_mode(r, s, st, h);
    h.allow_warped_motion = (intra || h.error_resilient_mode || !s.enable_warped_motion) ? 0 : r.b();
    h.reduced_tx_set = r.b();
    global_motion(r, st, h);
    film_grain(r, s, st, h);
    h.header_bits = (uint32_t)r.pos;
}

av1g_status fail(int code, const char* what) {
    av1g::set_framing_error(code, what);
    return AV1G_EINVAL;
}

}  // namespace

extern "C" {

void av1g_ref_state_init(av1g_ref_state* st) {
    if (!st) return;
    memset(st, 0, sizeof *st);
    for (int k = 0; k < 8; k++) {
        static const int8_t def_ref[8] = {1, 0, 0, 0, -1, 0, -1, -1};
        memcpy(st->lf_ref_deltas[k], def_ref, 8);
        for (int ref = 0; ref < 8; ref++)
            for (int i = 0; i < 6; i++) st->gm_params[k][ref][i] = (i % 3 == 2) ? 1 << kWarpPrec : 0;
    }
}

av1g_status av1g_parse_frame_header(const uint8_t* payload, size_t n, const av1g_sequence_header* sh,
                                    const av1g_ref_state* st, int32_t temporal_id, int32_t spatial_id,
                                    av1g_parsed_frame_header* out) {
    if (!sh || !st || !out || (!payload && n)) return fail(AV1G_FE_UNEXPECTED_END, "frame header: null argument");
    av1g_parsed_frame_header h;
    memset(&h, 0, sizeof h);
    h.temporal_id = temporal_id;
    h.spatial_id = spatial_id;
    try {
        parse(payload, n, *sh, *st, h);
    } catch (const Fail& f) {
        return fail(f.code, f.what);
    }
    *out = h;
    return AV1G_OK;
}

av1g_status av1g_ref_state_update(av1g_ref_state* st, const av1g_parsed_frame_header* fh) {
    if (!st || !fh) return fail(AV1G_FE_UNEXPECTED_END, "frame header: null argument");
    if (fh->show_existing_frame) {
        if (fh->frame_type != KEY_FRAME) return AV1G_OK;
        // §7.21: a shown key frame is loaded and stored into every slot
        const int k = fh->frame_to_show_map_idx;
        av1g_ref_state src = *st;
        for (int i = 0; i < 8; i++) {
            st->valid[i] = 1;
            st->frame_id[i] = src.frame_id[k];
            st->frame_type[i] = src.frame_type[k];
            st->order_hint[i] = src.order_hint[k];
            memcpy(st->saved_order_hints[i], src.saved_order_hints[k], sizeof st->saved_order_hints[i]);
            st->upscaled_width[i] = src.upscaled_width[k];
            st->frame_width[i] = src.frame_width[k];
            st->frame_height[i] = src.frame_height[k];
            st->render_width[i] = src.render_width[k];
            st->render_height[i] = src.render_height[k];
            st->mi_cols[i] = src.mi_cols[k];
            st->mi_rows[i] = src.mi_rows[k];
            memcpy(st->gm_params[i], src.gm_params[k], sizeof st->gm_params[i]);
            memcpy(st->lf_ref_deltas[i], src.lf_ref_deltas[k], 8);
            memcpy(st->lf_mode_deltas[i], src.lf_mode_deltas[k], 2);
            memcpy(st->seg_feature_enabled[i], src.seg_feature_enabled[k], sizeof st->seg_feature_enabled[i]);
            memcpy(st->seg_feature_data[i], src.seg_feature_data[k], sizeof st->seg_feature_data[i]);
            st->film_grain[i] = src.film_grain[k];
        }
        return AV1G_OK;
    }
    for (int i = 0; i < 8; i++) {
        if (!((fh->refresh_frame_flags >> i) & 1)) continue;
        st->valid[i] = 1;
        st->frame_id[i] = fh->current_frame_id;
        st->frame_type[i] = fh->frame_type;
        st->order_hint[i] = fh->order_hint;
        memcpy(st->saved_order_hints[i], fh->order_hints, sizeof st->saved_order_hints[i]);
        st->upscaled_width[i] = fh->pf.upscaled_width;
        st->frame_width[i] = fh->pf.frame_width;
        st->frame_height[i] = fh->pf.frame_height;
        st->render_width[i] = fh->render_width;
        st->render_height[i] = fh->render_height;
        st->mi_cols[i] = fh->pf.mi_cols;
        st->mi_rows[i] = fh->pf.mi_rows;
        memcpy(st->gm_params[i], fh->gm_params, sizeof st->gm_params[i]);
        memcpy(st->lf_ref_deltas[i], fh->pf.lf_ref_deltas, 8);
        memcpy(st->lf_mode_deltas[i], fh->pf.lf_mode_deltas, 2);
        memcpy(st->seg_feature_enabled[i], fh->seg_feature_enabled, sizeof st->seg_feature_enabled[i]);
        memcpy(st->seg_feature_data[i], fh->seg_feature_data, sizeof st->seg_feature_data[i]);
        st->film_grain[i] = fh->pf.film_grain;
    }
    return AV1G_OK;
}

av1g_status av1g_parse_tile_group(const uint8_t* payload, size_t n, const av1g_parsed_frame_header* fh,
                                  int32_t* tg_start, int32_t* tg_end, av1g_tile_span* tiles, int32_t cap) {
    if (!fh || !tg_start || !tg_end || (!payload && n) || cap < 0 || (cap > 0 && !tiles))
        return fail(AV1G_FE_UNEXPECTED_END, "tile group: null argument");
    try {
        Reader r{payload, n};
        const int num_tiles = fh->tile_cols * fh->tile_rows;
        bool flag = false;
        if (num_tiles > 1) flag = r.b();
        int start = 0, end = num_tiles - 1;
        if (num_tiles > 1 && flag) {
            const int bits = fh->tile_cols_log2 + fh->tile_rows_log2;
            start = (int)r.f(bits);
            end = (int)r.f(bits);
        }
        if (end < start || end >= num_tiles)
            return fail(AV1G_FE_FRAME_HEADER_INVALID, "tile group: tile range outside the frame");
        size_t at = (r.pos + 7) >> 3;  // byte_alignment
        for (int t = start; t <= end; t++) {
            size_t size;
            if (t == end) {
                if (at >= n) return fail(AV1G_FE_UNEXPECTED_END, "tile group: no bytes for the last tile");
                size = n - at;
            } else {
                if (n - at < (size_t)fh->tile_size_bytes) return fail(AV1G_FE_UNEXPECTED_END, "tile group: tile size");
                uint64_t v = 0;
                for (int i = 0; i < fh->tile_size_bytes; i++) v |= (uint64_t)payload[at + i] << (8 * i);
                at += fh->tile_size_bytes;
                size = (size_t)v + 1;
                if (size > n - at) return fail(AV1G_FE_UNEXPECTED_END, "tile group: tile runs past the OBU");
            }
            if (t - start < cap) tiles[t - start] = av1g_tile_span{t, 0, (uint64_t)at, (uint64_t)size};
            at += size;
        }
        *tg_start = start;
        *tg_end = end;
        if (end - start + 1 > cap) return fail(AV1G_FE_OUTPUT_TOO_SMALL, "tile group: more tiles than the output holds");
    } catch (const Fail& f) {
        return fail(f.code, f.what);
    }
    return AV1G_OK;
}

}  // extern "C"
