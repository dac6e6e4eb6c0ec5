"""Stream framing (row f3) through the C ABI, pinned by the reference's tests.

Host code only (framing.cpp): these run without a GPU.
  * unit tests of src/obu.rs (leb128, OBU headers), src/annexb.rs (split /
    build, temporal-delimiter placement, size nesting, truncations) and
    src/encoder/ivf.rs (header fields, frame records) restated;
  * tests/sequence_header_fixtures.rs: the 16 SEQUENCE_HEADER payloads and
    every field value the reference test expects;
  * tests/fixture_conformance.rs: all 110 embedded IVF streams — the IVF
    walk, the temporal-unit OBU walk and the frame-header prefix must give
    the shown-frame count each reference test asserts, and every stream must
    survive an Annex B round trip unit for unit;
  * tests/annexb_conformance.rs: the external Annex B stream splits into 4
    temporal units showing 4 frames, and its malformed-input cases fail;
  * operating-point selection (frame_driver.rs:1620-1644, the scenario of
    tests/scalability_op.rs) on units built here: a two-point sequence
    header, layer-1 OBUs dropped under point 1, an out-of-range point
    rejected.
The golden vectors come from tests/golden/make_framing_fixtures.py.
"""
import base64
import gzip
import json
from pathlib import Path

import pytest

from oxideav_av1_b200 import abi, framing
from oxideav_av1_b200.framing import FramingError

GOLDEN = json.load(gzip.open(Path(__file__).parent / "golden" / "framing_fixtures.json.gz", "rt"))


def _variant(fn, *a):
    with pytest.raises(FramingError) as e:
        fn(*a)
    return e.value.variant


def leb(v):
    out = bytearray()
    while True:
        b = v & 0x7F
        v >>= 7
        out.append(b | (0x80 if v else 0))
        if not v:
            return bytes(out)


def obu_header_byte(obu_type, ext, has_size):
    return (obu_type << 3) | (int(ext) << 2) | (int(has_size) << 1)


# --- src/obu.rs unit tests ---

def test_leb128_pins():
    assert framing.parse_leb128([0x00]) == (0, 1)
    assert framing.parse_leb128([0x81, 0x01]) == (129, 2)
    assert framing.parse_leb128([0x80, 0x00]) == (0, 2)
    assert _variant(framing.parse_leb128, [0x80, 0x80, 0x80, 0x80, 0x10]) == "Leb128Overflow"
    assert _variant(framing.parse_leb128, [0x80] * 9) == "Leb128TooLong"
    assert _variant(framing.parse_leb128, [0x80]) == "UnexpectedEnd"


def test_obu_header_pins():
    d, used = framing.parse_obu([obu_header_byte(2, False, True), 0x00])
    assert (d.type_name, d.extension_flag, d.has_size_field, d.temporal_id, d.spatial_id) == \
        ("TemporalDelimiter", False, True, 0, 0)
    assert (d.payload_len, d.header_len, d.payload, used) == (0, 2, b"", 2)
    ext = (3 << 5) | (2 << 3)
    d, used = framing.parse_obu([obu_header_byte(6, True, True), ext, 0x05, 0xA1, 0xA2, 0xA3, 0xA4, 0xA5])
    assert (d.type_name, d.extension_flag, d.temporal_id, d.spatial_id) == ("Frame", True, 3, 2)
    assert (d.payload_len, d.header_len, d.payload, used) == (5, 3, bytes([0xA1, 0xA2, 0xA3, 0xA4, 0xA5]), 8)
    stream = bytes([obu_header_byte(1, False, True), 2, 0x11, 0x22, obu_header_byte(6, False, True), 3, 0x33, 0x44,
                    0x55, obu_header_byte(2, False, True), 0])
    got = [(d.type_name, d.payload) for d in framing.obu_iter(stream)]
    assert got == [("SequenceHeader", b"\x11\x22"), ("Frame", b"\x33\x44\x55"), ("TemporalDelimiter", b"")]
    assert _variant(framing.parse_obu, [0x80 | obu_header_byte(2, False, True), 0]) == "ForbiddenBitSet"
    assert _variant(framing.parse_obu, [obu_header_byte(6, False, True), 4, 0xAA, 0xBB]) == "UnexpectedEnd"
    assert _variant(framing.parse_obu, [obu_header_byte(6, False, False)]) == "MissingSizeField"
    d, _ = framing.parse_obu([obu_header_byte(9, False, True), 1, 0xDE])
    assert (d.obu_type, d.type_name, d.payload) == (9, "Reserved(9)", b"\xde")


# --- src/annexb.rs unit tests ---

def test_annexb_pins():
    tu = bytes([0x12, 0x00, 0x32, 0x03, 1, 2, 3])
    annexb = framing.build_from_temporal_units([tu])
    assert framing.split_temporal_units(annexb) == [tu]
    fu = bytes([0x01, 0x10, 0x04, 0x30, 7, 8, 9])  # size-less OBUs gain obu_size
    assert framing.split_temporal_units(leb(len(fu) + 1) + leb(len(fu)) + fu) == \
        [bytes([0x12, 0x00, 0x32, 0x03, 7, 8, 9])]
    for fu in (bytes([0x04, 0x30, 7, 8, 9]), bytes([0x01, 0x10, 0x01, 0x10])):  # TD placement
        assert _variant(framing.split_temporal_units, leb(len(fu)) + fu) == "AnnexBInvalid"
    fu = bytes([0x02, 0x12, 0x00, 0x06, 0x32, 0x03, 1, 2, 3, 0])  # obu_size disagrees with obu_length
    assert _variant(framing.split_temporal_units, leb(len(fu)) + fu) == "AnnexBInvalid"
    for cut in range(1, len(annexb)):
        with pytest.raises(FramingError):
            framing.split_temporal_units(annexb[:cut])


# --- src/encoder/ivf.rs ---

def _ivf(frames, w=320, h=240, fourcc=b"AV01"):
    head = b"DKIF" + (0).to_bytes(2, "little") + (32).to_bytes(2, "little") + fourcc + w.to_bytes(2, "little") + \
        h.to_bytes(2, "little") + (30).to_bytes(4, "little") + (1).to_bytes(4, "little") + \
        len(frames).to_bytes(4, "little") + bytes(4)
    return head + b"".join(len(p).to_bytes(4, "little") + pts.to_bytes(8, "little") + p for pts, p in frames)


def test_ivf_reader():
    frames = [(0, b"\x12\x00"), (1, b"abc"), (7, b"")]
    r = framing.IvfReader(_ivf(frames))
    assert (bytes(r.header.fourcc), r.header.width, r.header.height, r.header.fps_num, r.header.fps_den,
            r.header.frame_count) == (b"AV01", 320, 240, 30, 1, 3)
    assert [(f.pts, f.payload) for f in r.read_all()] == frames
    good = _ivf(frames)
    assert _variant(framing.IvfReader, good[:31]) == "UnexpectedEnd"
    assert _variant(framing.IvfReader, b"XKIF" + good[4:]) == "BadMagic"
    assert _variant(framing.IvfReader, good[:4] + b"\x01\x00" + good[6:]) == "UnsupportedVersion"
    assert _variant(framing.IvfReader, good[:6] + b"\x20\x01" + good[8:]) == "UnsupportedHeaderLength"
    assert _variant(framing.IvfReader(good[:-2]).read_all) == "UnexpectedEnd"
    assert _variant(framing.IvfReader(good[:40]).read_all) == "UnexpectedEnd"


# --- tests/sequence_header_fixtures.rs ---

FIELDS = {"profile": "seq_profile", "still_picture": "still_picture", "reduced_still": "reduced_still_picture_header",
          "use_128sb": "use_128x128_superblock", "enable_filter_intra": "enable_filter_intra",
          "enable_intra_edge_filter": "enable_intra_edge_filter", "enable_interintra": "enable_interintra_compound",
          "enable_masked": "enable_masked_compound", "enable_warped": "enable_warped_motion",
          "enable_dual_filter": "enable_dual_filter", "enable_order_hint": "enable_order_hint",
          "order_hint_bits": "order_hint_bits", "enable_jnt_comp": "enable_jnt_comp",
          "enable_ref_mvs": "enable_ref_frame_mvs", "enable_superres": "enable_superres",
          "enable_cdef": "enable_cdef", "enable_restoration": "enable_restoration", "monochrome": "mono_chrome",
          "high_bitdepth": "high_bitdepth", "twelve_bit": "twelve_bit", "color_range": "color_range",
          "subsampling_x": "subsampling_x", "subsampling_y": "subsampling_y",
          "film_grain_present": "film_grain_params_present"}


@pytest.mark.parametrize("fx", GOLDEN["sequence_headers"], ids=lambda f: f["name"])
def test_sequence_header_fixture(fx):
    sh = framing.parse_sequence_header(bytes.fromhex(fx["payload"]))
    e = fx["expected"]
    got = {k: getattr(sh, f) for k, f in FIELDS.items()}
    got.update(max_w=sh.max_frame_width_minus_1 + 1, max_h=sh.max_frame_height_minus_1 + 1,
               level0=sh.operating_points[0].seq_level_idx, tier0=sh.operating_points[0].seq_tier,
               num_ops=sh.operating_points_cnt_minus_1 + 1)
    diff = {k: (got[k], v) for k, v in e.items() if int(got[k]) != int(v)}
    assert not diff, diff
    si = framing.seq_info(sh)
    assert (si.max_width, si.max_height, si.bit_depth, si.num_planes, si.sb_size) == \
        (e["max_w"], e["max_h"], 12 if e["twelve_bit"] else (10 if e["high_bitdepth"] else 8),
         1 if e["monochrome"] else 3, 128 if e["use_128sb"] else 64)


def test_sequence_header_errors():
    assert _variant(framing.parse_sequence_header, b"") == "UnexpectedEnd"
    assert _variant(framing.parse_sequence_header, bytes([0b01100000, 0])) == "ReservedProfile"
    assert _variant(framing.parse_sequence_header, bytes([0b00001000, 0])) == "ReducedStillRequiresStill"
    payload = bytes.fromhex(GOLDEN["sequence_headers"][0]["payload"])
    for cut in range(len(payload) - 1):
        with pytest.raises(FramingError):
            framing.parse_sequence_header(payload[:cut])


# --- tests/fixture_conformance.rs streams ---

@pytest.mark.parametrize("st", GOLDEN["ivf_streams"], ids=lambda s: s["name"])
def test_fixture_stream_shown_frames_and_annexb_round_trip(st):
    ivf = base64.b64decode(st["ivf"])
    assert framing.ivf_shown_frames(ivf) == st["shown_frames"]
    tus = [f.payload for f in framing.IvfReader(ivf).read_all()]
    assert framing.split_temporal_units(framing.build_from_temporal_units(tus)) == tus


def test_fixture_streams_open_engine_streams():
    """Each fixture's first sequence header gives the engine's stream
    parameters; they agree with the IVF header's frame size bound."""
    for st in GOLDEN["ivf_streams"]:
        ivf = base64.b64decode(st["ivf"])
        r = framing.IvfReader(ivf)
        w = framing.TemporalUnitWalker()
        w.walk(r.read_next_frame().payload)
        assert w.have_seq.value, st["name"]
        si = framing.seq_info(w.seq)
        assert si.max_width >= 1 and si.max_height >= 1 and si.bit_depth in (8, 10, 12) and si.sb_size in (64, 128)


# --- tests/annexb_conformance.rs ---

def test_external_annexb_stream():
    a = GOLDEN["annexb"]
    data = base64.b64decode(a["annexb"])
    tus = framing.split_temporal_units(data)
    w = framing.TemporalUnitWalker()
    assert sum(w.shown_frames(t) for t in tus) == a["shown_frames"] == 4
    assert framing.split_temporal_units(framing.build_from_temporal_units(tus)) == tus
    with pytest.raises(FramingError):
        framing.split_temporal_units(bytes([0x05, 1, 2]))  # truncated TU
    for cut in range(1, min(len(data), 64)):
        try:
            units = framing.split_temporal_units(data[:cut])
        except FramingError:
            continue
        assert len(units) < len(tus)  # a cut on a unit boundary keeps the whole units before it
    ivf = base64.b64decode(GOLDEN["ivf_streams"][0]["ivf"])
    with pytest.raises(FramingError):
        framing.split_temporal_units(ivf)


# --- operating points (frame_driver.rs:1620-1644) ---

class BitWriter:
    def __init__(self):
        self.bits = []

    def f(self, n, v):
        self.bits += [(v >> (n - 1 - i)) & 1 for i in range(n)]

    def bytes(self):
        b = self.bits + [1] + [0] * ((8 - (len(self.bits) + 1) % 8) % 8)  # trailing bits
        return bytes(int("".join(map(str, b[i: i + 8])), 2) for i in range(0, len(b), 8))


def seq_header(ops, timing=False):
    """A §5.5 sequence header: 64x64 profile 0 8-bit 4:2:0, order hints on,
    the given operating_point_idc values; with timing, decoder-model info and
    per-point operating parameters."""
    w = BitWriter()
    w.f(3, 0), w.f(1, 0), w.f(1, 0)
    w.f(1, int(timing))
    if timing:
        w.f(32, 1001), w.f(32, 60000), w.f(1, 1), w.f(3, 0b010)  # uvlc(1)
        w.f(1, 1), w.f(5, 9), w.f(32, 90000), w.f(5, 20), w.f(5, 7)
    w.f(1, 0)  # initial_display_delay_present_flag
    w.f(5, len(ops) - 1)
    for idc in ops:
        w.f(12, idc), w.f(5, 9), w.f(1, 1)  # level 9 carries seq_tier
        if timing:
            w.f(1, 1), w.f(10, 300), w.f(10, 200), w.f(1, 0)
    w.f(4, 5), w.f(4, 5), w.f(6, 63), w.f(6, 63)  # 64 x 64
    w.f(1, 0)  # frame ids
    w.f(3, 0b011)  # 64 sb, filter intra, edge filter
    w.f(5, 0b00001)  # interintra, masked, warped, dual: 0, order hint: 1
    w.f(2, 0b11), w.f(1, 1), w.f(1, 1), w.f(3, 6)  # jnt, ref mvs, choose sct, choose imv, 7 bits
    w.f(3, 0b011)  # superres 0, cdef 1, restoration 1
    w.f(1, 0), w.f(1, 0), w.f(1, 0), w.f(1, 0), w.f(2, 0), w.f(1, 0)  # color config
    w.f(1, 0)  # film grain
    return w.bytes()


def obu(t, payload, tid=None, sid=0):
    if tid is None:
        return bytes([obu_header_byte(t, False, True)]) + leb(len(payload)) + payload
    return bytes([obu_header_byte(t, True, True), (tid << 5) | (sid << 3)]) + leb(len(payload)) + payload


def frame_payload(show):
    w = BitWriter()
    w.f(1, 0), w.f(2, 1), w.f(1, int(show)), w.f(1, 1), w.f(1, 0)  # INTER, show, (showable), error_res 0
    return w.bytes()


def test_sequence_header_with_timing_and_operating_points():
    sh = framing.parse_sequence_header(seq_header([0x103, 0x101], timing=True))
    assert (sh.timing_info_present_flag, sh.num_units_in_display_tick, sh.time_scale, sh.equal_picture_interval,
            sh.num_ticks_per_picture_minus_1) == (1, 1001, 60000, 1, 1)
    assert (sh.decoder_model_info_present_flag, sh.buffer_delay_length_minus_1, sh.num_units_in_decoding_tick,
            sh.buffer_removal_time_length_minus_1, sh.frame_presentation_time_length_minus_1) == (1, 9, 90000, 20, 7)
    assert sh.operating_points_cnt_minus_1 == 1
    for k, idc in enumerate((0x103, 0x101)):
        op = sh.operating_points[k]
        assert (op.idc, op.seq_level_idx, op.seq_tier, op.decoder_model_present, op.decoder_buffer_delay,
                op.encoder_buffer_delay, op.low_delay_mode_flag) == (idc, 9, 1, 1, 300, 200, 0)
    assert (sh.max_frame_width_minus_1, sh.order_hint_bits, sh.enable_jnt_comp, sh.enable_cdef) == (63, 7, 1, 1)
    assert (sh.seq_force_screen_content_tools, sh.seq_force_integer_mv, sh.bit_depth) == (2, 2, 8)


def test_operating_point_selection_drops_other_layers():
    sh = seq_header([0x103, 0x101])
    tus = [obu(2, b"") + obu(1, sh) + obu(6, frame_payload(True), tid=0)]
    tus += [obu(2, b"") + obu(6, frame_payload(True), tid=k % 2) + obu(5, b"\x01", tid=1) for k in range(1, 6)]
    tus += [obu(2, b"") + obu(15, b"\x00\x00") + obu(6, frame_payload(False), tid=0)]
    full = framing.TemporalUnitWalker(0)
    base = framing.TemporalUnitWalker(1)
    assert sum(full.shown_frames(t) for t in tus) == 6
    assert full.op_idc.value == 0x103
    assert sum(base.shown_frames(t) for t in tus) == 3  # the temporal_id 1 frames are dropped
    assert base.op_idc.value == 0x101
    assert [d.type_name for d in base.walk(tus[1])] == []
    assert [d.type_name for d in full.walk(tus[1])] == ["Frame"]
    assert _variant(framing.TemporalUnitWalker(2).walk, tus[0]) == "OperatingPointOutOfRange"
    assert _variant(framing.TemporalUnitWalker(0).walk, obu(2, b"") + obu(9, b"\x00")) == "UnsupportedObu"


# --- src/tile_list.rs unit tests (§5.12 tile list OBU) ---

def _sample_tl():
    E = framing.TileListEntry
    return framing.TileListObu(1, 0, [E(0, 0, 0, bytes([0xAA, 0xBB, 0xCC])), E(3, 0, 1, bytes([0x11]))])


def test_tile_list_round_trips_byte_exact():
    tl = _sample_tl()
    b = framing.write_tile_list_obu(tl)
    assert len(b) == 4 + 5 + 3 + 5 + 1
    assert b[:4] == bytes([1, 0, 0x00, 0x01])
    assert framing.parse_tile_list_obu(b) == tl


def test_tile_list_rejects_truncated_and_overlong_payloads():
    b = framing.write_tile_list_obu(_sample_tl())
    assert _variant(framing.parse_tile_list_obu, b[:-1]) == "UnexpectedEnd"
    assert _variant(framing.parse_tile_list_obu, b + b"\x00") == "TileListInvalid"
    assert _variant(framing.parse_tile_list_obu, b[:3]) == "UnexpectedEnd"


def test_tile_list_conformance_bounds():
    assert _variant(framing.parse_tile_list_obu, bytes([0, 0, 0x02, 0x00])) == "TileListInvalid"
    assert _variant(framing.parse_tile_list_obu, bytes([0, 0, 0, 0, 128, 0, 0, 0, 0, 0xAA])) == "TileListInvalid"
    tl = _sample_tl()
    tl.entries[0].anchor_frame_idx = 128
    assert _variant(framing.write_tile_list_obu, tl) == "TileListInvalid"
    tl = _sample_tl()
    tl.entries[0].coded_tile_data = b""
    assert _variant(framing.write_tile_list_obu, tl) == "TileListInvalid"
    assert _variant(framing.write_tile_list_obu, framing.TileListObu(0, 0, [])) == "TileListInvalid"
    big = framing.TileListObu(31, 15, [framing.TileListEntry(k % 128, k % 4, k % 8, bytes([k & 255]) * (1 + k % 3))
                                       for k in range(512)])
    assert framing.parse_tile_list_obu(framing.write_tile_list_obu(big)) == big
