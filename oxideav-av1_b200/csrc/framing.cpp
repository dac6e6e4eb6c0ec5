// framing.cpp — host-side framing of AV1 streams: IVF records, §5.3 OBU
// headers and leb128, Annex B length-delimited units, the §5.5 sequence
// header, the §7.5 temporal-unit OBU walk with operating-point selection and
// the leading fields of §5.9.2 frame headers.
//
// Behaviour (accepted inputs, error variants) follows the reference:
//   leb128 / OBU header        src/obu.rs (parse_leb128, parse_obu)
//   IVF                        src/encoder/ivf.rs:242-352
//   Annex B                    src/annexb.rs:66-230
//   sequence header            src/sequence_header.rs, bit reader src/bitreader.rs
//   temporal-unit walk         src/decoder/frame_driver.rs:1590-1650
//   frame header prefix        src/frame_header.rs:920-1008
// The syntax is the AV1 specification's; the code is written for this
// library: spans over caller memory, no allocation in the parsers, and one
// thread-local error record shared with the rest of the C ABI.
#include <cstring>
#include <string>
#include <vector>

#include "av1g.h"

namespace av1g {
void set_framing_error(int code, const char* text);  // defined below
}

namespace {

thread_local int g_code = AV1G_FE_NONE;

av1g_status fe(int code, const char* what) {
    av1g::set_framing_error(code, what);
    return AV1G_EINVAL;
}

// ---------------------------------------------------------------------------
// bit reader (§4.10: f(n) MSB first, uvlc)

struct Bits {
    const uint8_t* p;
    size_t n;
    size_t pos = 0;  // bits
    bool bad = false;

    uint64_t f(int k) {
        uint64_t v = 0;
        for (int i = 0; i < k; i++) {
            if (pos >= n * 8) {
                bad = true;
                return 0;
            }
            v = (v << 1) | ((p[pos >> 3] >> (7 - (pos & 7))) & 1);
            pos++;
        }
        return v;
    }
    bool flag() { return f(1) != 0; }
    uint32_t uvlc() {
        int lz = 0;
        while (!bad && f(1) == 0) {
            if (++lz >= 32) return 0xffffffffu;
        }
        if (bad) return 0;
        const uint64_t v = f(lz) + ((uint64_t)1 << lz) - 1;
        return v > 0xffffffffull ? 0xffffffffu : (uint32_t)v;
    }
};

// ---------------------------------------------------------------------------
// leb128 and OBU headers

// §4.10.5: at most 8 bytes, the last with bit 7 clear; value < 2^32.
int leb128(const uint8_t* p, size_t n, uint64_t& value, int& len) {
    value = 0;
    for (int i = 0; i < 8; i++) {
        if ((size_t)i >= n) return AV1G_FE_UNEXPECTED_END;
        value |= (uint64_t)(p[i] & 0x7f) << (7 * i);
        if (!(p[i] & 0x80)) {
            len = i + 1;
            return value > 0xffffffffull ? AV1G_FE_LEB128_OVERFLOW : AV1G_FE_NONE;
        }
    }
    return AV1G_FE_LEB128_TOO_LONG;
}

const char* fe_text(int code) {
    switch (code) {
        case AV1G_FE_UNEXPECTED_END: return "unexpected end of data";
        case AV1G_FE_FORBIDDEN_BIT_SET: return "obu_forbidden_bit is set";
        case AV1G_FE_MISSING_SIZE_FIELD: return "OBU without obu_size in a low-overhead stream";
        case AV1G_FE_LEB128_OVERFLOW: return "leb128 value above 2^32 - 1";
        case AV1G_FE_LEB128_TOO_LONG: return "leb128 longer than 8 bytes";
        case AV1G_FE_SIZE_OVERFLOW: return "size overflow";
        case AV1G_FE_ANNEXB_INVALID: return "malformed Annex B unit";
        case AV1G_FE_IVF_BAD_MAGIC: return "IVF: no DKIF magic";
        case AV1G_FE_IVF_UNSUPPORTED_VERSION: return "IVF: version is not 0";
        case AV1G_FE_IVF_UNSUPPORTED_HEADER_LENGTH: return "IVF: header length is not 32";
        case AV1G_FE_RESERVED_PROFILE: return "seq_profile above 2";
        case AV1G_FE_REDUCED_STILL_REQUIRES_STILL: return "reduced_still_picture_header without still_picture";
        case AV1G_FE_OPERATING_POINT_OUT_OF_RANGE: return "chosen operating point beyond operating_points_cnt";
        case AV1G_FE_OUTPUT_TOO_SMALL: return "output buffer too small";
        case AV1G_FE_UNSUPPORTED_OBU: return "reserved OBU type in a temporal unit";
        case AV1G_FE_TEMPORAL_POINT_INFO_UNSUPPORTED: return "temporal_point_info is not supported";
        case AV1G_FE_TILE_LIST_INVALID: return "tile list outside the conformance bounds";
        default: return "framing error";
    }
}

// parse_obu: header byte, optional extension, mandatory leb128 obu_size.
int parse_obu(const uint8_t* p, size_t n, av1g_obu& o, uint64_t& consumed) {
    if (n < 1) return AV1G_FE_UNEXPECTED_END;
    const uint8_t h = p[0];
    if (h >> 7) return AV1G_FE_FORBIDDEN_BIT_SET;
    memset(&o, 0, sizeof o);
    o.obu_type = (h >> 3) & 15;
    o.extension_flag = (h >> 2) & 1;
    o.has_size_field = (h >> 1) & 1;
    size_t at = 1;
    if (o.extension_flag) {
        if (n < 2) return AV1G_FE_UNEXPECTED_END;
        o.temporal_id = (p[1] >> 5) & 7;
        o.spatial_id = (p[1] >> 3) & 3;
        at = 2;
    }
    if (!o.has_size_field) return AV1G_FE_MISSING_SIZE_FIELD;
    uint64_t size;
    int len;
    if (int c = leb128(p + at, n - at, size, len)) return c;
    at += len;
    if (size > n - at) return AV1G_FE_UNEXPECTED_END;
    o.header_len = (int32_t)at;
    o.payload_offset = at;
    o.payload_len = size;
    consumed = at + size;
    return AV1G_FE_NONE;
}

void put_leb128(std::vector<uint8_t>& out, uint64_t v) {
    do {
        uint8_t b = v & 0x7f;
        v >>= 7;
        out.push_back(b | (v ? 0x80 : 0));
    } while (v);
}

// ---------------------------------------------------------------------------
// sequence header (§5.5)

int parse_seq(const uint8_t* p, size_t n, av1g_sequence_header& s) {
    memset(&s, 0, sizeof s);
    Bits b{p, n};
    s.seq_profile = (uint8_t)b.f(3);
    if (b.bad) return AV1G_FE_UNEXPECTED_END;
    if (s.seq_profile > 2) return AV1G_FE_RESERVED_PROFILE;
    s.still_picture = b.flag();
    s.reduced_still_picture_header = b.flag();
    if (s.reduced_still_picture_header && !s.still_picture) return AV1G_FE_REDUCED_STILL_REQUIRES_STILL;
    if (s.reduced_still_picture_header) {
        s.operating_points[0].seq_level_idx = (uint8_t)b.f(5);
    } else {
        s.timing_info_present_flag = b.flag();
        if (s.timing_info_present_flag) {
            s.num_units_in_display_tick = (uint32_t)b.f(32);
            s.time_scale = (uint32_t)b.f(32);
            s.equal_picture_interval = b.flag();
            if (s.equal_picture_interval) s.num_ticks_per_picture_minus_1 = b.uvlc();
            s.decoder_model_info_present_flag = b.flag();
            if (s.decoder_model_info_present_flag) {
                s.buffer_delay_length_minus_1 = (uint8_t)b.f(5);
                s.num_units_in_decoding_tick = (uint32_t)b.f(32);
                s.buffer_removal_time_length_minus_1 = (uint8_t)b.f(5);
                s.frame_presentation_time_length_minus_1 = (uint8_t)b.f(5);
            }
        }
        s.initial_display_delay_present_flag = b.flag();
        s.operating_points_cnt_minus_1 = (uint8_t)b.f(5);
        for (int i = 0; i <= s.operating_points_cnt_minus_1 && !b.bad; i++) {
            av1g_operating_point& op = s.operating_points[i];
            op.idc = (uint16_t)b.f(12);
            op.seq_level_idx = (uint8_t)b.f(5);
            op.seq_tier = op.seq_level_idx > 7 ? (uint8_t)b.f(1) : 0;
            if (s.decoder_model_info_present_flag) {
                op.decoder_model_present = b.flag();
                if (op.decoder_model_present) {
                    const int k = s.buffer_delay_length_minus_1 + 1;
                    op.decoder_buffer_delay = b.f(k);
                    op.encoder_buffer_delay = b.f(k);
                    op.low_delay_mode_flag = b.flag();
                }
            }
            if (s.initial_display_delay_present_flag) {
                op.initial_display_delay_present = b.flag();
                if (op.initial_display_delay_present) op.initial_display_delay_minus_1 = (uint8_t)b.f(4);
            }
        }
    }
    s.frame_width_bits_minus_1 = (uint8_t)b.f(4);
    s.frame_height_bits_minus_1 = (uint8_t)b.f(4);
    s.max_frame_width_minus_1 = (uint32_t)b.f(s.frame_width_bits_minus_1 + 1);
    s.max_frame_height_minus_1 = (uint32_t)b.f(s.frame_height_bits_minus_1 + 1);
    if (!s.reduced_still_picture_header) s.frame_id_numbers_present_flag = b.flag();
    if (s.frame_id_numbers_present_flag) {
        s.delta_frame_id_length_minus_2 = (uint8_t)b.f(4);
        s.additional_frame_id_length_minus_1 = (uint8_t)b.f(3);
    }
    s.use_128x128_superblock = b.flag();
    s.enable_filter_intra = b.flag();
    s.enable_intra_edge_filter = b.flag();
    if (s.reduced_still_picture_header) {
        s.seq_force_screen_content_tools = 2;  // SELECT_SCREEN_CONTENT_TOOLS
        s.seq_force_integer_mv = 2;            // SELECT_INTEGER_MV
    } else {
        s.enable_interintra_compound = b.flag();
        s.enable_masked_compound = b.flag();
        s.enable_warped_motion = b.flag();
        s.enable_dual_filter = b.flag();
        s.enable_order_hint = b.flag();
        if (s.enable_order_hint) {
            s.enable_jnt_comp = b.flag();
            s.enable_ref_frame_mvs = b.flag();
        }
        const bool choose_sct = b.flag();
        s.seq_force_screen_content_tools = choose_sct ? 2 : (uint8_t)b.f(1);
        if (s.seq_force_screen_content_tools > 0) {
            const bool choose_imv = b.flag();
            s.seq_force_integer_mv = choose_imv ? 2 : (uint8_t)b.f(1);
        } else {
            s.seq_force_integer_mv = 2;
        }
        if (s.enable_order_hint) s.order_hint_bits = (uint8_t)(b.f(3) + 1);
    }
    s.enable_superres = b.flag();
    s.enable_cdef = b.flag();
    s.enable_restoration = b.flag();
    // §5.5.2 color_config
    s.high_bitdepth = b.flag();
    if (s.seq_profile == 2 && s.high_bitdepth) {
        s.twelve_bit = b.flag();
        s.bit_depth = s.twelve_bit ? 12 : 10;
    } else {
        s.bit_depth = s.high_bitdepth ? 10 : 8;
    }
    s.mono_chrome = s.seq_profile == 1 ? 0 : b.flag();
    s.num_planes = s.mono_chrome ? 1 : 3;
    s.color_description_present_flag = b.flag();
    if (s.color_description_present_flag) {
        s.color_primaries = (uint8_t)b.f(8);
        s.transfer_characteristics = (uint8_t)b.f(8);
        s.matrix_coefficients = (uint8_t)b.f(8);
    } else {
        s.color_primaries = s.transfer_characteristics = s.matrix_coefficients = 2;  // unspecified
    }
    if (s.mono_chrome) {
        s.color_range = b.flag();
        s.subsampling_x = s.subsampling_y = 1;
        s.chroma_sample_position = 0;
        s.separate_uv_delta_q = 0;
    } else {
        if (s.color_primaries == 1 && s.transfer_characteristics == 13 && s.matrix_coefficients == 0) {
            s.color_range = 1;  // sRGB: 4:4:4, full range
        } else {
            s.color_range = b.flag();
            if (s.seq_profile == 0) {
                s.subsampling_x = s.subsampling_y = 1;
            } else if (s.seq_profile == 2) {
                if (s.bit_depth == 12) {
                    s.subsampling_x = b.flag();
                    s.subsampling_y = s.subsampling_x ? b.flag() : 0;
                } else {
                    s.subsampling_x = 1;
                }
            }
            if (s.subsampling_x && s.subsampling_y) s.chroma_sample_position = (uint8_t)b.f(2);
        }
        s.separate_uv_delta_q = b.flag();
    }
    s.film_grain_params_present = b.flag();
    if (b.bad) return AV1G_FE_UNEXPECTED_END;
    s.bits_consumed = (uint32_t)b.pos;
    return AV1G_FE_NONE;
}

// Frame-header prefix (§5.9.2 up to error_resilient_mode).
int parse_prefix(const uint8_t* p, size_t n, const av1g_sequence_header& s, av1g_frame_prefix& o) {
    memset(&o, 0, sizeof o);
    o.frame_to_show_map_idx = -1;
    if (s.reduced_still_picture_header) {
        o.frame_type = 0;
        o.show_frame = 1;
        o.error_resilient_mode = 1;
        return AV1G_FE_NONE;
    }
    Bits b{p, n};
    const bool temporal_point = s.decoder_model_info_present_flag && !s.equal_picture_interval;
    o.show_existing_frame = b.flag();
    if (o.show_existing_frame) {
        o.frame_to_show_map_idx = (int32_t)b.f(3);
        if (b.bad) return AV1G_FE_UNEXPECTED_END;
        if (temporal_point) return AV1G_FE_TEMPORAL_POINT_INFO_UNSUPPORTED;
        if (s.frame_id_numbers_present_flag)  // display_frame_id
            b.f(s.additional_frame_id_length_minus_1 + s.delta_frame_id_length_minus_2 + 3);
        if (b.bad) return AV1G_FE_UNEXPECTED_END;
        o.frame_type = -1;  // RefFrameType[frame_to_show_map_idx]: reference state
        o.show_frame = 1;
        return AV1G_FE_NONE;
    }
    o.frame_type = (int32_t)b.f(2);
    o.show_frame = b.flag();
    if (b.bad) return AV1G_FE_UNEXPECTED_END;
    if (o.show_frame && temporal_point) return AV1G_FE_TEMPORAL_POINT_INFO_UNSUPPORTED;
    o.showable_frame = o.show_frame ? o.frame_type != 0 : b.flag();
    o.error_resilient_mode = (o.frame_type == 3 || (o.frame_type == 0 && o.show_frame)) ? 1 : b.flag();
    return b.bad ? AV1G_FE_UNEXPECTED_END : AV1G_FE_NONE;
}

av1g_status done(int code) { return code ? fe(code, fe_text(code)) : AV1G_OK; }

}  // namespace

namespace av1g {

// The text goes to the C ABI's thread-local error string (api.cu).
void set_last_error_text(const std::string& s);

void set_framing_error(int code, const char* text) {
    g_code = code;
    set_last_error_text(std::string("framing: ") + text);
}

}  // namespace av1g

extern "C" {

int32_t av1g_framing_error(void) { return g_code; }

av1g_status av1g_leb128(const uint8_t* p, size_t n, uint64_t* value, int32_t* len) {
    g_code = AV1G_FE_NONE;
    if ((!p && n) || !value || !len) return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    int l = 0;
    uint64_t v = 0;
    const int c = leb128(p, n, v, l);
    if (c) return done(c);
    *value = v;
    *len = l;
    return AV1G_OK;
}

av1g_status av1g_parse_obu(const uint8_t* p, size_t n, av1g_obu* out, uint64_t* consumed) {
    g_code = AV1G_FE_NONE;
    if ((!p && n) || !out || !consumed) return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    av1g_obu o;
    uint64_t c = 0;
    const int code = parse_obu(p, n, o, c);
    if (code) return done(code);
    *out = o;
    *consumed = c;
    return AV1G_OK;
}

av1g_status av1g_ivf_parse_header(const uint8_t* p, size_t n, av1g_ivf_header* out) {
    g_code = AV1G_FE_NONE;
    if (!out || !p || n < 32) return done(AV1G_FE_UNEXPECTED_END);
    if (memcmp(p, "DKIF", 4)) return done(AV1G_FE_IVF_BAD_MAGIC);
    auto u16 = [&](int at) { return (uint16_t)(p[at] | p[at + 1] << 8); };
    auto u32 = [&](int at) { return (uint32_t)p[at] | (uint32_t)p[at + 1] << 8 | (uint32_t)p[at + 2] << 16 |
                                    (uint32_t)p[at + 3] << 24; };
    av1g_ivf_header h;
    h.version = u16(4);
    if (h.version != 0) return done(AV1G_FE_IVF_UNSUPPORTED_VERSION);
    h.header_length = u16(6);
    if (h.header_length != 32) return done(AV1G_FE_IVF_UNSUPPORTED_HEADER_LENGTH);
    memcpy(h.fourcc, p + 8, 4);
    h.width = u16(12);
    h.height = u16(14);
    h.fps_num = u32(16);
    h.fps_den = u32(20);
    h.frame_count = u32(24);
    *out = h;
    return AV1G_OK;
}

av1g_status av1g_ivf_next_frame(const uint8_t* p, size_t n, uint64_t* cursor, av1g_ivf_frame* out, int32_t* got) {
    g_code = AV1G_FE_NONE;
    if (!cursor || !out || !got || (!p && n)) return done(AV1G_FE_UNEXPECTED_END);
    *got = 0;
    const uint64_t c = *cursor;
    if (c >= n) return AV1G_OK;
    if (n - c < 12) return done(AV1G_FE_UNEXPECTED_END);
    uint64_t size = 0, pts = 0;
    for (int i = 3; i >= 0; i--) size = size << 8 | p[c + i];
    for (int i = 7; i >= 0; i--) pts = pts << 8 | p[c + 4 + i];
    if (size > n - c - 12) return done(AV1G_FE_UNEXPECTED_END);
    out->pts = pts;
    out->offset = c + 12;
    out->size = size;
    *cursor = c + 12 + size;
    *got = 1;
    return AV1G_OK;
}

av1g_status av1g_annexb_split(const uint8_t* p, size_t n, uint8_t* out, size_t cap, uint64_t* tu_end, int32_t tu_cap,
                              int32_t* n_tu, uint64_t* out_len) {
    g_code = AV1G_FE_NONE;
    if ((!p && n) || (!out && cap) || !n_tu || !out_len || (tu_cap > 0 && !tu_end) || tu_cap < 0)
        return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    size_t pos = 0, w = 0;
    int units = 0;
    auto emit = [&](const uint8_t* src, size_t k) {
        if (w + k > cap) return false;
        memcpy(out + w, src, k);
        w += k;
        return true;
    };
    while (pos < n) {
        uint64_t tu_size;
        int len;
        if (int c = leb128(p + pos, n - pos, tu_size, len)) return done(c);
        pos += len;
        if (tu_size > n - pos) return done(AV1G_FE_UNEXPECTED_END);
        const size_t tu_stop = pos + tu_size;
        bool first_fu = true;
        while (pos < tu_stop) {
            uint64_t fu_size;
            if (int c = leb128(p + pos, tu_stop - pos, fu_size, len)) return done(c);
            pos += len;
            if (fu_size > tu_stop - pos) return done(AV1G_FE_ANNEXB_INVALID);
            const size_t fu_stop = pos + fu_size;
            bool first_obu = true;
            while (pos < fu_stop) {
                uint64_t obu_len;
                if (int c = leb128(p + pos, fu_stop - pos, obu_len, len)) return done(c);
                pos += len;
                if (obu_len > fu_stop - pos) return done(AV1G_FE_ANNEXB_INVALID);
                const uint8_t* ob = p + pos;
                // one OBU of the unit in low-overhead form
                if (obu_len < 1) return done(AV1G_FE_ANNEXB_INVALID);
                const uint8_t h = ob[0];
                if (h >> 7) return done(AV1G_FE_FORBIDDEN_BIT_SET);
                const int type = (h >> 3) & 15, ext = (h >> 2) & 1, has_size = (h >> 1) & 1;
                if ((first_fu && first_obu) != (type == AV1G_OBU_TEMPORAL_DELIMITER))
                    return done(AV1G_FE_ANNEXB_INVALID);
                const size_t hl = 1 + ext;
                if (obu_len < hl) return done(AV1G_FE_UNEXPECTED_END);
                if (has_size) {
                    av1g_obu o;
                    uint64_t used;
                    if (int c = parse_obu(ob, obu_len, o, used)) return done(c);
                    if (used != obu_len) return done(AV1G_FE_ANNEXB_INVALID);
                    if (!emit(ob, obu_len)) return done(AV1G_FE_OUTPUT_TOO_SMALL);
                } else {
                    uint8_t hdr[2 + 8];
                    size_t k = 0;
                    hdr[k++] = h | 2;
                    if (ext) hdr[k++] = ob[1];
                    uint64_t pl = obu_len - hl;
                    do {
                        uint8_t byte = pl & 0x7f;
                        pl >>= 7;
                        hdr[k++] = byte | (pl ? 0x80 : 0);
                    } while (pl);
                    if (!emit(hdr, k) || !emit(ob + hl, obu_len - hl)) return done(AV1G_FE_OUTPUT_TOO_SMALL);
                }
                pos += obu_len;
                first_obu = false;
            }
            first_fu = false;
        }
        if (units >= tu_cap) return done(AV1G_FE_OUTPUT_TOO_SMALL);
        tu_end[units++] = w;
    }
    *n_tu = units;
    *out_len = w;
    return AV1G_OK;
}

av1g_status av1g_annexb_build(const uint8_t* tus, const uint64_t* tu_end, int32_t n_tu, uint8_t* out, size_t cap,
                              uint64_t* out_len) {
    g_code = AV1G_FE_NONE;
    if (n_tu < 0 || (n_tu > 0 && (!tu_end || !tus)) || !out_len) return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    std::vector<uint8_t> stream, body, fu;
    uint64_t start = 0;
    for (int t = 0; t < n_tu; t++) {
        const uint64_t stop = tu_end[t];
        if (stop < start) return fe(AV1G_FE_SIZE_OVERFLOW, "temporal unit ends out of order");
        const uint8_t* tu = tus + start;
        const size_t len = stop - start;
        body.clear();
        fu.clear();
        bool fu_has_frame = false, first = true;
        size_t pos = 0;
        while (pos < len) {
            av1g_obu o;
            uint64_t used;
            if (int c = parse_obu(tu + pos, len - pos, o, used)) return done(c);
            if (first && o.obu_type != AV1G_OBU_TEMPORAL_DELIMITER) return done(AV1G_FE_ANNEXB_INVALID);
            first = false;
            const bool starts_frame = o.obu_type == AV1G_OBU_FRAME || o.obu_type == AV1G_OBU_FRAME_HEADER;
            if (starts_frame && fu_has_frame) {  // a new frame unit
                put_leb128(body, fu.size());
                body.insert(body.end(), fu.begin(), fu.end());
                fu.clear();
                fu_has_frame = false;
            }
            put_leb128(fu, used);
            fu.insert(fu.end(), tu + pos, tu + pos + used);
            fu_has_frame |= starts_frame;
            pos += used;
        }
        if (!fu.empty()) {
            put_leb128(body, fu.size());
            body.insert(body.end(), fu.begin(), fu.end());
        }
        put_leb128(stream, body.size());
        stream.insert(stream.end(), body.begin(), body.end());
        start = stop;
    }
    *out_len = stream.size();
    if (!out) return AV1G_OK;
    if (stream.size() > cap) return done(AV1G_FE_OUTPUT_TOO_SMALL);
    memcpy(out, stream.data(), stream.size());
    return AV1G_OK;
}

av1g_status av1g_parse_sequence_header(const uint8_t* payload, size_t n, av1g_sequence_header* out) {
    g_code = AV1G_FE_NONE;
    if (!out || (!payload && n)) return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    av1g_sequence_header s;
    const int c = parse_seq(payload, n, s);
    if (c) return done(c);
    *out = s;
    return AV1G_OK;
}

av1g_status av1g_seq_info_from_header(const av1g_sequence_header* sh, av1g_seq_info* out) {
    g_code = AV1G_FE_NONE;
    if (!sh || !out) return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    out->max_width = (int32_t)sh->max_frame_width_minus_1 + 1;
    out->max_height = (int32_t)sh->max_frame_height_minus_1 + 1;
    out->bit_depth = sh->bit_depth;
    out->subsampling_x = sh->subsampling_x;
    out->subsampling_y = sh->subsampling_y;
    out->num_planes = sh->num_planes;
    out->sb_size = sh->use_128x128_superblock ? 128 : 64;
    return AV1G_OK;
}

av1g_status av1g_temporal_unit_obus(const uint8_t* tu, size_t n, int32_t chosen_op, uint16_t* op_idc,
                                    av1g_sequence_header* seq, int32_t* have_seq, av1g_obu* obus, int32_t cap,
                                    int32_t* count) {
    g_code = AV1G_FE_NONE;
    if ((!tu && n) || !op_idc || !seq || !have_seq || !count || cap < 0 || (cap > 0 && !obus) || chosen_op < 0)
        return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    int k = 0;
    size_t pos = 0;
    while (pos < n) {
        av1g_obu o;
        uint64_t used;
        if (int c = parse_obu(tu + pos, n - pos, o, used)) {
            *count = k;
            return done(c);
        }
        o.payload_offset += pos;
        pos += used;
        const int t = o.obu_type;
        if (*op_idc != 0 && o.extension_flag && t != AV1G_OBU_SEQUENCE_HEADER && t != AV1G_OBU_TEMPORAL_DELIMITER) {
            const bool in_t = (*op_idc >> o.temporal_id) & 1, in_s = (*op_idc >> (o.spatial_id + 8)) & 1;
            if (!in_t || !in_s) continue;
        }
        switch (t) {
            case AV1G_OBU_TEMPORAL_DELIMITER:
            case AV1G_OBU_PADDING:
            case AV1G_OBU_METADATA:
            case AV1G_OBU_TILE_LIST:
                continue;
            case AV1G_OBU_SEQUENCE_HEADER: {
                av1g_sequence_header s;
                if (int c = parse_seq(tu + o.payload_offset, o.payload_len, s)) {
                    *count = k;
                    return done(c);
                }
                if (chosen_op > s.operating_points_cnt_minus_1) {
                    *count = k;
                    return done(AV1G_FE_OPERATING_POINT_OUT_OF_RANGE);
                }
                *op_idc = s.operating_points[chosen_op].idc;
                *seq = s;
                *have_seq = 1;
                break;
            }
            case AV1G_OBU_FRAME_HEADER:
            case AV1G_OBU_REDUNDANT_FRAME_HEADER:
            case AV1G_OBU_TILE_GROUP:
            case AV1G_OBU_FRAME:
                break;
            default:
                *count = k;
                return done(AV1G_FE_UNSUPPORTED_OBU);
        }
        if (k >= cap) {
            *count = k;
            return done(AV1G_FE_OUTPUT_TOO_SMALL);
        }
        obus[k++] = o;
    }
    *count = k;
    return AV1G_OK;
}

av1g_status av1g_frame_header_prefix(const uint8_t* payload, size_t n, const av1g_sequence_header* sh,
                                     av1g_frame_prefix* out) {
    g_code = AV1G_FE_NONE;
    if (!sh || !out || (!payload && n)) return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    av1g_frame_prefix o;
    const int c = parse_prefix(payload, n, *sh, o);
    if (c) return done(c);
    *out = o;
    return AV1G_OK;
}

av1g_status av1g_parse_tile_list(const uint8_t* payload, size_t n, av1g_tile_list_header* hdr,
                                 av1g_tile_list_obu_entry* entries, int32_t cap) {
    g_code = AV1G_FE_NONE;
    if (!hdr || (!payload && n) || cap < 0 || (cap > 0 && !entries)) return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    if (n < 4) return done(AV1G_FE_UNEXPECTED_END);
    av1g_tile_list_header h;
    memset(&h, 0, sizeof h);
    h.output_frame_width_in_tiles_minus_1 = payload[0];
    h.output_frame_height_in_tiles_minus_1 = payload[1];
    h.tile_count_minus_1 = payload[2] << 8 | payload[3];
    if (h.tile_count_minus_1 > 511) return done(AV1G_FE_TILE_LIST_INVALID);
    size_t at = 4;
    for (int k = 0; k <= h.tile_count_minus_1; k++) {
        if (n - at < 5) return done(AV1G_FE_UNEXPECTED_END);
        av1g_tile_list_obu_entry e;
        memset(&e, 0, sizeof e);
        e.anchor_frame_idx = payload[at];
        if (e.anchor_frame_idx > 127) return done(AV1G_FE_TILE_LIST_INVALID);
        e.anchor_tile_row = payload[at + 1];
        e.anchor_tile_col = payload[at + 2];
        e.data_size = (uint64_t)(payload[at + 3] << 8 | payload[at + 4]) + 1;
        at += 5;
        if (e.data_size > n - at) return done(AV1G_FE_UNEXPECTED_END);
        e.data_offset = at;
        at += e.data_size;
        if (k < cap) entries[k] = e;
    }
    if (at != n) return done(AV1G_FE_TILE_LIST_INVALID);
    if (h.tile_count_minus_1 + 1 > cap) return done(AV1G_FE_OUTPUT_TOO_SMALL);
    *hdr = h;
    return AV1G_OK;
}

av1g_status av1g_write_tile_list(const av1g_tile_list_header* hdr, const av1g_tile_list_obu_entry* entries,
                                 int32_t count, const uint8_t* data, uint8_t* out, size_t cap, uint64_t* out_len) {
    g_code = AV1G_FE_NONE;
    if (!hdr || !out_len || count < 0 || (count > 0 && (!entries || !data)))
        return fe(AV1G_FE_UNEXPECTED_END, "null argument");
    if (count < 1 || count > 512) return done(AV1G_FE_TILE_LIST_INVALID);
    std::vector<uint8_t> b;
    b.push_back((uint8_t)hdr->output_frame_width_in_tiles_minus_1);
    b.push_back((uint8_t)hdr->output_frame_height_in_tiles_minus_1);
    b.push_back((uint8_t)((count - 1) >> 8));
    b.push_back((uint8_t)(count - 1));
    for (int k = 0; k < count; k++) {
        const av1g_tile_list_obu_entry& e = entries[k];
        if (e.anchor_frame_idx < 0 || e.anchor_frame_idx > 127 || e.data_size < 1 || e.data_size > 65536)
            return done(AV1G_FE_TILE_LIST_INVALID);
        b.push_back((uint8_t)e.anchor_frame_idx);
        b.push_back((uint8_t)e.anchor_tile_row);
        b.push_back((uint8_t)e.anchor_tile_col);
        b.push_back((uint8_t)((e.data_size - 1) >> 8));
        b.push_back((uint8_t)(e.data_size - 1));
        b.insert(b.end(), data + e.data_offset, data + e.data_offset + e.data_size);
    }
    *out_len = b.size();
    if (!out) return AV1G_OK;
    if (b.size() > cap) return done(AV1G_FE_OUTPUT_TOO_SMALL);
    memcpy(out, b.data(), b.size());
    return AV1G_OK;
}

}  // extern "C"
