// decoder.cpp — the stream decoder behind the reference's registry Decoder
// API (src/registry.rs: send_packet 132, receive_frame 168, flush 181,
// reset 186; the session is SpecDecodeSession, src/decoder/frame_driver.rs:
// 1295-1400, and its temporal-unit walk decode_temporal_unit_spec,
// frame_driver.rs:1590-1813).
//
// Host work per frame: the §7.5 OBU walk (framing.cpp), the §5.9 header
// (frameheader.cpp), the §5.11 tile walk (walker.cpp) with the §7.9 motion
// field it reads, then one av1g_submit_frame to the serving engine, which
// runs every pixel stage on the GPU.  The per-slot parse state the syntax of
// later frames reads (frame-end CDFs, segmentation map, §7.19 motion-field
// candidates) is kept here, as the reference keeps it in SpecRefSlot
// (frame_driver.rs:84-139, reference_frame_update 1409).
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "av1g.h"
#include "walker.h"

namespace av1g {
void set_framing_error(int code, const char* text);
}

namespace {

thread_local std::string t_dec_err;

av1g_status dfail(av1g_status st, const std::string& msg) {
    av1g::set_framing_error(AV1G_FE_FRAME_HEADER_INVALID, msg.c_str());
    return st;
}

int rel_dist(int a, int b, int bits) {
    if (!bits) return 0;
    int diff = a - b, m = 1 << (bits - 1);
    return (diff & (m - 1)) - (diff & m);
}

// A shown frame waiting for receive_frame: its engine ticket, or the planes
// already copied out.
struct Pending {
    uint64_t ticket = 0;
    bool has_ticket = false;
    int64_t pts = 0;
};

}  // namespace

namespace av1w {

// §7.9 motion field estimation (motion_field_estimation_core,
// src/inter_pred.rs:7592): up to five projection passes of the stored §7.19
// candidates of the reference slots onto the current frame's 8x8 grid; a
// later writer of a position overwrites an earlier one.
void motion_field_estimation(const av1g_parsed_frame_header& fh, const av1g_sequence_header& seq,
                             const av1g_ref_state& refs, const SlotParse* slots, std::vector<int16_t>& out) {
    static const int Div_Mult[32] = {0,    16384, 8192, 5461, 4096, 3276, 2730, 2340, 2048, 1820, 1638,
                                     1489, 1365,  1260, 1170, 1092, 1024, 963,  910,  862,  819,  780,
                                     744,  712,   682,  655,  630,  606,  585,  564,  546,  528};
    const int MiRows = fh.pf.mi_rows, MiCols = fh.pf.mi_cols;
    const int h8 = MiRows >> 1, w8 = MiCols >> 1;
    const int bits = seq.enable_order_hint ? seq.order_hint_bits : 0;
    out.assign((size_t)7 * h8 * w8 * 2, 0);
    for (size_t i = 0; i < out.size(); i += 2) out[i] = -32768;
    int order_hints[8] = {0};
    for (int i = 0; i < 7; i++) order_hints[1 + i] = refs.order_hint[fh.ref_frame_idx[i]];
    auto proj = [](int mv, int num, int den) {
        int cden = den < 31 ? den : 31;
        int cnum = num < -31 ? -31 : num > 31 ? 31 : num;
        int64_t v = (int64_t)mv * cnum * Div_Mult[cden];
        int64_t s = v >= 0 ? (v + (1 << 13)) >> 14 : -((-v + (1 << 13)) >> 14);
        if (s < -(1 << 14) + 1) s = -(1 << 14) + 1;
        if (s > (1 << 14) - 1) s = (1 << 14) - 1;
        return (int)s;
    };
    auto project_ref = [&](int src, int dstSign) -> bool {
        int srcIdx = fh.ref_frame_idx[src - 1];
        const SlotParse& sl = slots[srcIdx];
        if (!sl.valid || sl.mi_rows != MiRows || sl.mi_cols != MiCols || sl.frame_is_intra) return false;
        for (int y8 = 0; y8 < h8; y8++)
            for (int x8 = 0; x8 < w8; x8++) {
                size_t c = (size_t)(2 * y8 + 1) * MiCols + (2 * x8 + 1);
                int srcRef = sl.mf_ref_frames[c];
                if (srcRef <= 0) continue;
                int refToCur = rel_dist(order_hints[src], fh.order_hint, bits);
                int refOffset = rel_dist(order_hints[src], sl.saved_order_hints[srcRef], bits);
                if (!(std::abs(refToCur) <= 31 && std::abs(refOffset) <= 31 && refOffset > 0)) continue;
                int mv[2] = {sl.mf_mvs[c * 2], sl.mf_mvs[c * 2 + 1]};
                int pm[2] = {proj(mv[0], refToCur * dstSign, refOffset), proj(mv[1], refToCur * dstSign, refOffset)};
                auto axis = [&](int v8, int delta, int max8, int maxOff8, int& pos) {
                    int base8 = (v8 >> 3) << 3;
                    int off8 = delta >= 0 ? delta >> 6 : -((-delta) >> 6);
                    pos = v8 + dstSign * off8;
                    return !(pos < 0 || pos >= max8 || pos < base8 - maxOff8 || pos >= base8 + 8 + maxOff8);
                };
                int py, px;
                if (!axis(y8, pm[0], h8, 0, py) || !axis(x8, pm[1], w8, 8, px)) continue;
                for (int dst = 1; dst <= 7; dst++) {
                    int refToDst = rel_dist(fh.order_hint, order_hints[dst], bits);
                    size_t o = (((size_t)(dst - 1) * h8 + py) * w8 + px) * 2;
                    out[o] = (int16_t)proj(mv[0], refToDst, refOffset);
                    out[o + 1] = (int16_t)proj(mv[1], refToDst, refOffset);
                }
            }
        return true;
    };
    int lastIdx = fh.ref_frame_idx[0];
    int lastAlt = slots[lastIdx].valid ? slots[lastIdx].saved_order_hints[7] : 0;
    if (lastAlt != order_hints[4]) project_ref(1, -1);
    int stamp = 3 - 2;
    if (rel_dist(order_hints[5], fh.order_hint, bits) > 0 && project_ref(5, 1)) stamp--;
    if (rel_dist(order_hints[6], fh.order_hint, bits) > 0 && project_ref(6, 1)) stamp--;
    if (rel_dist(order_hints[7], fh.order_hint, bits) > 0 && stamp >= 0 && project_ref(7, 1)) stamp--;
    if (stamp >= 0) project_ref(2, -1);
}

}  // namespace av1w

struct av1g_decoder {
    av1g_engine* engine = nullptr;
    av1g_stream* stream = nullptr;
    av1g_seq_info stream_seq{};
    int32_t chosen_op = 0;
    uint16_t op_idc = 0;
    av1g_sequence_header seq{};
    int32_t have_seq = 0;
    av1g_ref_state refs{};
    av1w::SlotParse slots[8];
    // the frame whose tile groups are still arriving
    bool pending_frame = false;
    av1g_parsed_frame_header pending_fh{};
    std::vector<uint8_t> pending_tiles;           // concatenated tile bytes
    std::vector<std::pair<size_t, size_t>> pending_spans;
    int next_tg_start = 0;
    // parse-only record of every frame (engine == NULL)
    std::vector<std::unique_ptr<av1w::FrameOut>> parsed;
    std::vector<av1g_parsed_frame_header> parsed_hdr;
    av1w::FrameOut work;
    // outputs
    std::deque<Pending> queue;
    bool eof = false;
    std::vector<uint8_t> out_buf;
    double host_ms = 0.0;
    int32_t frames_out_of_sync = 0;
};

namespace {

av1g_status open_stream(av1g_decoder* d) {
    if (!d->engine) return AV1G_OK;
    av1g_seq_info si;
    if (av1g_status st = av1g_seq_info_from_header(&d->seq, &si)) return st;
    if (d->stream && std::memcmp(&si, &d->stream_seq, sizeof si) == 0) return AV1G_OK;
    if (d->stream) {
        av1g_stream_close(d->stream);
        d->stream = nullptr;
    }
    if (av1g_status st = av1g_stream_open(d->engine, &si, &d->stream)) return st;
    d->stream_seq = si;
    return AV1G_OK;
}

// §7.20 reference_frame_update of the parse state (and §7.21 for a shown key frame).
void update_slots(av1g_decoder* d, const av1g_parsed_frame_header& fh, const av1w::FrameOut* fo) {
    if (fh.show_existing_frame) {
        if (!fh.refresh_frame_flags) return;
        av1w::SlotParse src = d->slots[fh.frame_to_show_map_idx];
        for (int i = 0; i < 8; i++)
            if ((fh.refresh_frame_flags >> i) & 1) d->slots[i] = src;
        return;
    }
    if (!fh.refresh_frame_flags || !fo) return;
    av1w::SlotParse s;
    s.valid = true;
    s.cdfs = fo->end_cdfs;
    s.mi_rows = fh.pf.mi_rows;
    s.mi_cols = fh.pf.mi_cols;
    s.frame_is_intra = fh.frame_type == 0 || fh.frame_type == 2;
    s.segment_ids = fo->segment_map;
    size_t cells = (size_t)s.mi_rows * s.mi_cols;
    s.mf_ref_frames.assign(cells, -1);
    s.mf_mvs.assign(cells * 2, 0);
    for (int i = 0; i < 8; i++) s.saved_order_hints[i] = fh.order_hints[i];
    if (!s.frame_is_intra) {
        // §7.19 motion field motion vector storage (frame_driver.rs:1119-1160)
        const int bits = d->seq.enable_order_hint ? d->seq.order_hint_bits : 0;
        for (size_t c = 0; c < cells; c++)
            for (int list = 0; list < 2; list++) {
                int r = fo->ref_frames[c * 2 + list];
                if (r <= 0) continue;
                int hint = d->refs.order_hint[fh.ref_frame_idx[r - 1]];
                if (rel_dist(hint, fh.order_hint, bits) >= 0) continue;
                int mr = fo->mvs[c * 4 + list * 2], mc = fo->mvs[c * 4 + list * 2 + 1];
                if (std::abs(mr) > 4095 || std::abs(mc) > 4095) continue;
                s.mf_ref_frames[c] = (int8_t)r;
                s.mf_mvs[c * 2] = (int16_t)mr;
                s.mf_mvs[c * 2 + 1] = (int16_t)mc;
            }
    }
    for (int i = 0; i < 8; i++)
        if ((fh.refresh_frame_flags >> i) & 1) d->slots[i] = s;
}

av1g_status submit(av1g_decoder* d, const av1g_parsed_frame_header& fh, const av1w::FrameOut* fo, int64_t pts) {
    if (!d->engine) return AV1G_OK;
    if (av1g_status st = open_stream(d)) return st;
    av1g_frame_desc desc;
    av1g_frame_header hdr_copy;
    if (fo) {
        fo->fill_desc(desc);
    } else {
        std::memset(&desc, 0, sizeof desc);
        hdr_copy = fh.pf;
        desc.hdr = &hdr_copy;
    }
    for (int i = 0; i < 7; i++) desc.ref_frame_idx[i] = (uint8_t)fh.ref_frame_idx[i];
    desc.refresh_frame_flags = (uint8_t)fh.refresh_frame_flags;
    desc.show_frame = (uint8_t)(fh.show_existing_frame ? 1 : fh.show_frame);
    desc.show_existing_frame = (uint8_t)fh.show_existing_frame;
    desc.frame_to_show_map_idx = (uint8_t)(fh.show_existing_frame ? fh.frame_to_show_map_idx : 0);
    uint64_t ticket = 0;
    for (int tries = 0;; tries++) {
        av1g_status st = av1g_submit_frame(d->stream, &desc, &ticket);
        if (st == AV1G_OK) break;
        if (st != AV1G_EBUSY || tries > 20000) return st;
        // no free slot: wait for the oldest queued frame before retrying
        if (!d->queue.empty() && d->queue.front().has_ticket) {
            av1g_status res;
            av1g_poll(d->engine, d->queue.front().ticket, 1000000, &res);
        } else {
            std::this_thread::sleep_for(std::chrono::microseconds(100));
        }
    }
    if (desc.show_frame) {
        Pending p;
        p.ticket = ticket;
        p.has_ticket = true;
        p.pts = pts;
        d->queue.push_back(p);
    } else {
        // hidden frames still own a ticket: free it once finished
        av1g_status res;
        if (av1g_poll(d->engine, ticket, 60000000000LL, &res) == AV1G_OK) av1g_release_output(d->stream, ticket);
    }
    return AV1G_OK;
}

av1g_status decode_frame(av1g_decoder* d, const av1g_parsed_frame_header& fh, const uint8_t* tile_base,
                         const std::vector<std::pair<size_t, size_t>>& spans, int64_t pts) {
    std::vector<av1w::TileData> tiles;
    for (auto& s : spans) tiles.push_back({tile_base + s.first, s.second});
    av1w::FrameOut* fo = &d->work;
    std::unique_ptr<av1w::FrameOut> keep;
    if (!d->engine) {
        keep.reset(new av1w::FrameOut());
        fo = keep.get();
    }
    std::string err;
    nvtxRangePushA("av1g tile walk");
    av1g_status st = av1w::walk_frame(d->seq, fh, d->refs, d->slots, tiles, *fo, err);
    nvtxRangePop();
    if (st != AV1G_OK) return dfail(st, err);
    if (!fo->tiles_in_sync) d->frames_out_of_sync++;
    if (av1g_status s2 = submit(d, fh, fo, pts)) return s2;
    update_slots(d, fh, fo);
    if (av1g_status s3 = av1g_ref_state_update(&d->refs, &fh)) return s3;
    if (!d->engine) {
        d->parsed.push_back(std::move(keep));
        d->parsed_hdr.push_back(fh);
    }
    return AV1G_OK;
}

av1g_status temporal_unit(av1g_decoder* d, const uint8_t* tu, size_t n, int64_t pts) {
    std::vector<av1g_obu> obus(256);
    int32_t count = 0;
    av1g_sequence_header seq_after = d->seq;
    int32_t have_after = d->have_seq;
    uint16_t op_after = d->op_idc;
    for (;;) {
        av1g_status st = av1g_temporal_unit_obus(tu, n, d->chosen_op, &op_after, &seq_after, &have_after,
                                                 obus.data(), (int32_t)obus.size(), &count);
        if (st == AV1G_OK) break;
        if (av1g_framing_error() == AV1G_FE_OUTPUT_TOO_SMALL && obus.size() < (1u << 16)) {
            obus.resize(obus.size() * 4);
            op_after = d->op_idc;
            continue;
        }
        return st;
    }
    for (int k = 0; k < count; k++) {
        const av1g_obu& o = obus[k];
        const uint8_t* pl = tu + o.payload_offset;
        size_t len = o.payload_len;
        switch (o.obu_type) {
            case AV1G_OBU_SEQUENCE_HEADER: {
                if (av1g_status st = av1g_parse_sequence_header(pl, len, &d->seq)) return st;
                d->have_seq = 1;
                d->op_idc = d->seq.operating_points[d->chosen_op].idc;
                break;
            }
            case AV1G_OBU_FRAME_HEADER:
            case AV1G_OBU_FRAME: {
                if (d->pending_frame && !d->pending_spans.empty())
                    return dfail(AV1G_EINVAL, "a frame header arrived before the previous frame's last tile group");
                d->pending_frame = false;
                if (!d->have_seq) return dfail(AV1G_EINVAL, "frame before any sequence header");
                av1g_parsed_frame_header fh;
                if (av1g_status st = av1g_parse_frame_header(pl, len, &d->seq, &d->refs, o.temporal_id,
                                                             o.spatial_id, &fh))
                    return st;
                if (fh.show_existing_frame) {
                    if (d->engine) {
                        if (av1g_status st = submit(d, fh, nullptr, pts)) return st;
                    } else {
                        d->parsed.push_back(nullptr);
                        d->parsed_hdr.push_back(fh);
                    }
                    update_slots(d, fh, nullptr);
                    if (av1g_status st = av1g_ref_state_update(&d->refs, &fh)) return st;
                    break;
                }
                d->pending_frame = true;
                d->pending_fh = fh;
                d->pending_tiles.clear();
                d->pending_spans.clear();
                d->next_tg_start = 0;
                if (o.obu_type == AV1G_OBU_FRAME_HEADER) break;
                size_t start = (fh.header_bits + 7) >> 3;
                if (start > len) return dfail(AV1G_EINVAL, "frame OBU shorter than its header");
                pl += start;
                len -= start;
            }
                [[fallthrough]];  // the tile group of a frame OBU
            case AV1G_OBU_TILE_GROUP: {
                if (!d->pending_frame) return dfail(AV1G_EINVAL, "tile group without a frame header");
                const av1g_parsed_frame_header& fh = d->pending_fh;
                int numTiles = fh.tile_cols * fh.tile_rows;
                std::vector<av1g_tile_span> spans(numTiles);
                int32_t a = 0, b = 0;
                if (av1g_status st = av1g_parse_tile_group(pl, len, &fh, &a, &b, spans.data(), numTiles)) return st;
                if (a != d->next_tg_start) return dfail(AV1G_EINVAL, "tile groups out of order");
                d->next_tg_start = b + 1;
                for (int i = 0; i <= b - a; i++) {
                    size_t off = d->pending_tiles.size();
                    d->pending_tiles.insert(d->pending_tiles.end(), pl + spans[i].offset,
                                            pl + spans[i].offset + spans[i].size);
                    d->pending_spans.push_back({off, (size_t)spans[i].size});
                }
                if (b + 1 == numTiles) {
                    d->pending_frame = false;
                    auto sp = d->pending_spans;
                    d->pending_spans.clear();
                    if (av1g_status st = decode_frame(d, fh, d->pending_tiles.data(), sp, pts)) return st;
                }
                break;
            }
            case AV1G_OBU_REDUNDANT_FRAME_HEADER:
            default:
                break;
        }
    }
    if (d->pending_frame && !d->pending_spans.empty())
        return dfail(AV1G_EINVAL, "temporal unit ended inside a frame's tile groups");
    return AV1G_OK;
}

}  // namespace

extern "C" {

av1g_status av1g_decoder_create(av1g_engine* engine, int32_t operating_point, av1g_decoder** out) {
    if (!out || operating_point < 0 || operating_point > 31) return dfail(AV1G_EINVAL, "bad argument");
    av1g_decoder* d = new (std::nothrow) av1g_decoder();
    if (!d) return AV1G_EDEVICE;
    d->engine = engine;
    d->chosen_op = operating_point;
    av1g_ref_state_init(&d->refs);
    *out = d;
    return AV1G_OK;
}

void av1g_decoder_destroy(av1g_decoder* d) {
    if (!d) return;
    if (d->stream) {
        for (auto& p : d->queue)
            if (p.has_ticket) {
                av1g_status r;
                av1g_poll(d->engine, p.ticket, 60000000000LL, &r);
                av1g_release_output(d->stream, p.ticket);
            }
        av1g_stream_close(d->stream);
    }
    delete d;
}

av1g_status av1g_decoder_send_packet(av1g_decoder* d, const uint8_t* data, size_t n, int64_t pts) {
    if (!d || (!data && n)) return dfail(AV1G_EINVAL, "bad argument");
    if (d->eof) return dfail(AV1G_EINVAL, "packet after flush");
    auto t0 = std::chrono::steady_clock::now();
    av1g_status st = AV1G_OK;
    if (n >= 4 && std::memcmp(data, "DKIF", 4) == 0) {
        av1g_ivf_header h;
        if ((st = av1g_ivf_parse_header(data, n, &h)) != AV1G_OK) return st;
        uint64_t cur = 32;
        for (;;) {
            av1g_ivf_frame f;
            int32_t got = 0;
            if ((st = av1g_ivf_next_frame(data, n, &cur, &f, &got)) != AV1G_OK) return st;
            if (!got) break;
            if ((st = temporal_unit(d, data + f.offset, f.size, (int64_t)f.pts)) != AV1G_OK) return st;
        }
    } else {
        st = temporal_unit(d, data, n, pts);
    }
    d->host_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return st;
}

av1g_status av1g_decoder_receive_frame(av1g_decoder* d, av1g_frame_out* out, int64_t* pts) {
    if (!d || !out) return dfail(AV1G_EINVAL, "bad argument");
    if (d->queue.empty()) return d->eof ? AV1G_EOF : AV1G_ENOTREADY;
    Pending p = d->queue.front();
    av1g_status res = AV1G_OK;
    av1g_status st = av1g_poll(d->engine, p.ticket, 60000000000LL, &res);
    if (st != AV1G_OK) return st;
    d->queue.pop_front();
    av1g_frame_out fo;
    st = av1g_fetch_output(d->stream, p.ticket, &fo);
    if (st != AV1G_OK) {
        av1g_release_output(d->stream, p.ticket);
        return st;
    }
    size_t total = 0;
    for (int i = 0; i < fo.num_planes; i++) total += (size_t)fo.planes[i].stride * fo.planes[i].height;
    d->out_buf.resize(total);
    size_t off = 0;
    *out = fo;
    for (int i = 0; i < fo.num_planes; i++) {
        size_t b = (size_t)fo.planes[i].stride * fo.planes[i].height;
        std::memcpy(d->out_buf.data() + off, fo.planes[i].data, b);
        out->planes[i].data = d->out_buf.data() + off;
        off += b;
    }
    av1g_release_output(d->stream, p.ticket);
    if (pts) *pts = p.pts;
    return AV1G_OK;
}

av1g_status av1g_decoder_flush(av1g_decoder* d) {
    if (!d) return dfail(AV1G_EINVAL, "bad argument");
    d->eof = true;
    return AV1G_OK;
}

av1g_status av1g_decoder_reset(av1g_decoder* d) {
    if (!d) return dfail(AV1G_EINVAL, "bad argument");
    if (d->stream) {
        for (auto& p : d->queue)
            if (p.has_ticket) {
                av1g_status r;
                av1g_poll(d->engine, p.ticket, 60000000000LL, &r);
                av1g_release_output(d->stream, p.ticket);
            }
        av1g_stream_reset_refs(d->stream);
    }
    d->queue.clear();
    d->eof = false;
    d->pending_frame = false;
    d->pending_spans.clear();
    av1g_ref_state_init(&d->refs);
    for (auto& s : d->slots) s = av1w::SlotParse();
    d->parsed.clear();
    d->parsed_hdr.clear();
    return AV1G_OK;
}

int32_t av1g_decoder_parsed_count(const av1g_decoder* d) { return d ? (int32_t)d->parsed.size() : 0; }

av1g_status av1g_decoder_parsed_frame(const av1g_decoder* d, int32_t i, av1g_frame_desc* out,
                                      av1g_parsed_frame_header* fh) {
    if (!d || !out || i < 0 || i >= (int32_t)d->parsed.size()) return dfail(AV1G_EINVAL, "bad argument");
    const av1g_parsed_frame_header& h = d->parsed_hdr[i];
    if (d->parsed[i]) {
        d->parsed[i]->fill_desc(*out);
    } else {
        std::memset(out, 0, sizeof *out);
        out->hdr = &d->parsed_hdr[i].pf;
    }
    for (int k = 0; k < 7; k++) out->ref_frame_idx[k] = (uint8_t)h.ref_frame_idx[k];
    out->refresh_frame_flags = (uint8_t)h.refresh_frame_flags;
    out->show_frame = (uint8_t)(h.show_existing_frame ? 1 : h.show_frame);
    out->show_existing_frame = (uint8_t)h.show_existing_frame;
    out->frame_to_show_map_idx = (uint8_t)(h.show_existing_frame ? h.frame_to_show_map_idx : 0);
    if (fh) *fh = h;
    return AV1G_OK;
}

av1g_status av1g_decoder_sequence(const av1g_decoder* d, av1g_sequence_header* out) {
    if (!d || !out || !d->have_seq) return dfail(AV1G_EINVAL, "no sequence header yet");
    *out = d->seq;
    return AV1G_OK;
}

double av1g_decoder_host_ms(const av1g_decoder* d) { return d ? d->host_ms : 0.0; }

int32_t av1g_decoder_frames_out_of_sync(const av1g_decoder* d) { return d ? d->frames_out_of_sync : 0; }

}  // extern "C"
