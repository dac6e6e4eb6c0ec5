"""Stream framing through the C ABI: IVF, OBUs, Annex B, sequence headers.

Names and behaviour mirror the reference's framing layer — ``parse_leb128`` /
``parse_obu`` / ``ObuIter`` (src/obu.rs), ``IvfReader`` (src/encoder/ivf.rs),
``split_temporal_units`` / ``build_from_temporal_units`` (src/annexb.rs),
``parse_sequence_header`` (src/sequence_header.rs), ``parse_tile_list_obu`` /
``write_tile_list_obu`` (src/tile_list.rs) — and the OBU walk of a
temporal unit (decode_temporal_unit_spec, src/decoder/frame_driver.rs:1590).
Errors raise ``FramingError`` whose ``variant`` is the reference's error
variant name.  The work happens in the library's host code (framing.cpp).
"""
import ctypes as C
from dataclasses import dataclass

from . import abi

VARIANTS = {abi.FE_UNEXPECTED_END: "UnexpectedEnd", abi.FE_FORBIDDEN_BIT_SET: "ForbiddenBitSet",
            abi.FE_MISSING_SIZE_FIELD: "MissingSizeField", abi.FE_LEB128_OVERFLOW: "Leb128Overflow",
            abi.FE_LEB128_TOO_LONG: "Leb128TooLong", abi.FE_SIZE_OVERFLOW: "SizeOverflow",
            abi.FE_ANNEXB_INVALID: "AnnexBInvalid", abi.FE_IVF_BAD_MAGIC: "BadMagic",
            abi.FE_IVF_UNSUPPORTED_VERSION: "UnsupportedVersion",
            abi.FE_IVF_UNSUPPORTED_HEADER_LENGTH: "UnsupportedHeaderLength",
            abi.FE_RESERVED_PROFILE: "ReservedProfile",
            abi.FE_REDUCED_STILL_REQUIRES_STILL: "ReducedStillRequiresStill",
            abi.FE_OPERATING_POINT_OUT_OF_RANGE: "OperatingPointOutOfRange",
            abi.FE_OUTPUT_TOO_SMALL: "OutputTooSmall", abi.FE_UNSUPPORTED_OBU: "UnsupportedObu",
            abi.FE_TEMPORAL_POINT_INFO_UNSUPPORTED: "TemporalPointInfoUnsupported",
            abi.FE_TILE_LIST_INVALID: "TileListInvalid",
            abi.FE_SYMBOL_STATE_INVARIANT: "SymbolStateInvariantBroken",
            abi.FE_SYMBOL_EXIT_UNDERFLOW: "SymbolExitUnderflow",
            abi.FE_FRAME_HEADER_INVALID: "FrameHeaderInvalid"}

OBU_NAMES = {1: "SequenceHeader", 2: "TemporalDelimiter", 3: "FrameHeader", 4: "TileGroup", 5: "Metadata",
             6: "Frame", 7: "RedundantFrameHeader", 8: "TileList", 15: "Padding"}


class FramingError(ValueError):
    def __init__(self, code, text):
        self.code = code
        self.variant = VARIANTS.get(code, str(code))
        super().__init__(f"{self.variant}: {text}")


def _check(lib, status):
    if status != abi.AV1G_OK:
        raise FramingError(lib.av1g_framing_error(), lib.av1g_last_error().decode(errors="replace"))


def _buf(data):
    data = bytes(data)
    return data, C.cast(C.c_char_p(data), C.c_void_p) if data else None


def parse_leb128(data):
    """(value, bytes used)."""
    lib = abi.load()
    data, p = _buf(data)
    v, n = C.c_uint64(), C.c_int32()
    _check(lib, lib.av1g_leb128(p, len(data), C.byref(v), C.byref(n)))
    return v.value, n.value


@dataclass
class ObuDescriptor:
    obu_type: int
    extension_flag: bool
    has_size_field: bool
    temporal_id: int
    spatial_id: int
    payload_len: int
    header_len: int
    payload: bytes

    @property
    def type_name(self):
        return OBU_NAMES.get(self.obu_type, f"Reserved({self.obu_type})")


def _desc(o, data, base=0):
    off = o.payload_offset - base
    return ObuDescriptor(o.obu_type, bool(o.extension_flag), bool(o.has_size_field), o.temporal_id, o.spatial_id,
                         o.payload_len, o.header_len, bytes(data[off: off + o.payload_len]))


def parse_obu(data):
    """(ObuDescriptor, bytes consumed) of the OBU at the start of data."""
    lib = abi.load()
    data, p = _buf(data)
    o, used = abi.Obu(), C.c_uint64()
    _check(lib, lib.av1g_parse_obu(p, len(data), C.byref(o), C.byref(used)))
    return _desc(o, data), used.value


def obu_iter(data):
    """Yields the OBUs of a low-overhead byte stream; a malformed OBU raises."""
    pos = 0
    data = bytes(data)
    while pos < len(data):
        d, used = parse_obu(data[pos:])
        pos += used
        yield d


@dataclass
class IvfFrame:
    pts: int
    payload: bytes


class IvfReader:
    """IvfReader (src/encoder/ivf.rs:284): header, read_next_frame, read_all."""

    def __init__(self, data):
        self._lib = abi.load()
        self._data, self._p = _buf(data)
        self.header = abi.IvfHeader()
        _check(self._lib, self._lib.av1g_ivf_parse_header(self._p, len(self._data), C.byref(self.header)))
        self._cursor = C.c_uint64(32)

    def read_next_frame(self):
        f, got = abi.IvfFrame(), C.c_int32()
        _check(self._lib, self._lib.av1g_ivf_next_frame(self._p, len(self._data), C.byref(self._cursor), C.byref(f),
                                                        C.byref(got)))
        if not got.value:
            return None
        return IvfFrame(f.pts, self._data[f.offset: f.offset + f.size])

    def read_all(self):
        out = []
        while (f := self.read_next_frame()) is not None:
            out.append(f)
        return out


def split_temporal_units(data):
    """Annex B stream -> list of low-overhead temporal units (bytes)."""
    lib = abi.load()
    data, p = _buf(data)
    cap_units = max(1, len(data))
    out = (C.c_uint8 * max(1, len(data)))()
    ends = (C.c_uint64 * cap_units)()
    n_tu, out_len = C.c_int32(), C.c_uint64()
    _check(lib, lib.av1g_annexb_split(p, len(data), out, len(data), ends, cap_units, C.byref(n_tu),
                                      C.byref(out_len)))
    raw = bytes(out)[: out_len.value]
    units, start = [], 0
    for i in range(n_tu.value):
        units.append(raw[start: ends[i]])
        start = ends[i]
    return units


def build_from_temporal_units(units):
    """Low-overhead temporal units -> one Annex B stream."""
    lib = abi.load()
    joined = b"".join(bytes(u) for u in units)
    ends, acc = (C.c_uint64 * max(1, len(units)))(), 0
    for i, u in enumerate(units):
        acc += len(u)
        ends[i] = acc
    joined, p = _buf(joined)
    need = C.c_uint64()
    _check(lib, lib.av1g_annexb_build(p, ends, len(units), None, 0, C.byref(need)))
    out = (C.c_uint8 * max(1, need.value))()
    _check(lib, lib.av1g_annexb_build(p, ends, len(units), out, need.value, C.byref(need)))
    return bytes(out)[: need.value]


def parse_sequence_header(payload):
    """The §5.5 sequence header of an OBU payload (av1g_sequence_header)."""
    lib = abi.load()
    data, p = _buf(payload)
    sh = abi.SequenceHeader()
    _check(lib, lib.av1g_parse_sequence_header(p, len(data), C.byref(sh)))
    return sh


def seq_info(sh):
    """The engine's stream parameters (av1g_seq_info) of a sequence header."""
    lib = abi.load()
    out = abi.SeqInfo()
    _check(lib, lib.av1g_seq_info_from_header(C.byref(sh), C.byref(out)))
    return out


def frame_header_prefix(payload, sh):
    lib = abi.load()
    data, p = _buf(payload)
    out = abi.FramePrefix()
    _check(lib, lib.av1g_frame_header_prefix(p, len(data), C.byref(sh), C.byref(out)))
    return out


class TemporalUnitWalker:
    """The per-stream state of the §7.5 OBU walk: the chosen operating point,
    its idc and the latest sequence header, carried from unit to unit."""

    def __init__(self, chosen_op=0):
        self._lib = abi.load()
        self.chosen_op = chosen_op
        self.op_idc = C.c_uint16(0)
        self.seq = abi.SequenceHeader()
        self.have_seq = C.c_int32(0)

    def walk(self, tu):
        """The OBUs of one temporal unit that the frame decode acts on."""
        data, p = _buf(tu)
        cap = max(1, len(data) // 2 + 1)
        obus, count = (abi.Obu * cap)(), C.c_int32()
        _check(self._lib, self._lib.av1g_temporal_unit_obus(p, len(data), self.chosen_op, C.byref(self.op_idc),
                                                            C.byref(self.seq), C.byref(self.have_seq), obus, cap,
                                                            C.byref(count)))
        return [_desc(obus[i], data) for i in range(count.value)]

    def shown_frames(self, tu):
        """Frames this temporal unit outputs: every frame header that shows an
        existing frame and every frame whose show_frame is set."""
        n = 0
        for d in self.walk(tu):
            if d.obu_type in (3, 6):
                pre = frame_header_prefix(d.payload, self.seq)
                n += 1 if (pre.show_existing_frame or pre.show_frame) else 0
        return n


def ivf_shown_frames(data, chosen_op=0):
    """Frames a whole IVF stream outputs under operating point chosen_op."""
    w = TemporalUnitWalker(chosen_op)
    return sum(w.shown_frames(f.payload) for f in IvfReader(data).read_all())


@dataclass
class TileListEntry:
    anchor_frame_idx: int
    anchor_tile_row: int
    anchor_tile_col: int
    coded_tile_data: bytes


@dataclass
class TileListObu:
    output_frame_width_in_tiles_minus_1: int
    output_frame_height_in_tiles_minus_1: int
    entries: list


def parse_tile_list_obu(payload):
    """parse_tile_list_obu (src/tile_list.rs:102)."""
    lib = abi.load()
    data, p = _buf(payload)
    hdr = abi.TileListHeader()
    ents = (abi.TileListObuEntry * 512)()
    _check(lib, lib.av1g_parse_tile_list(p, len(data), C.byref(hdr), ents, 512))
    out = [TileListEntry(e.anchor_frame_idx, e.anchor_tile_row, e.anchor_tile_col,
                         data[e.data_offset: e.data_offset + e.data_size])
           for e in ents[: hdr.tile_count_minus_1 + 1]]
    return TileListObu(hdr.output_frame_width_in_tiles_minus_1, hdr.output_frame_height_in_tiles_minus_1, out)


def write_tile_list_obu(tl):
    """write_tile_list_obu (src/tile_list.rs:156)."""
    lib = abi.load()
    hdr = abi.TileListHeader(tl.output_frame_width_in_tiles_minus_1, tl.output_frame_height_in_tiles_minus_1,
                             max(len(tl.entries) - 1, 0), 0)
    data = b"".join(bytes(e.coded_tile_data) for e in tl.entries)
    ents = (abi.TileListObuEntry * max(1, len(tl.entries)))()
    off = 0
    for i, e in enumerate(tl.entries):
        ents[i] = abi.TileListObuEntry(e.anchor_frame_idx, e.anchor_tile_row, e.anchor_tile_col, 0, off,
                                       len(e.coded_tile_data))
        off += len(e.coded_tile_data)
    data, p = _buf(data if data else b"\0")
    need = C.c_uint64()
    _check(lib, lib.av1g_write_tile_list(C.byref(hdr), ents, len(tl.entries), p, None, 0, C.byref(need)))
    out = (C.c_uint8 * max(1, need.value))()
    _check(lib, lib.av1g_write_tile_list(C.byref(hdr), ents, len(tl.entries), p, out, need.value, C.byref(need)))
    return bytes(out)[: need.value]


class SymbolDecoder:
    """SymbolDecoder (src/symbol_decoder.rs) over the library's §8.2 decoder:
    init_symbol, read_symbol (a CDF is a list of n values plus the counter,
    adapted in place), read_bool, read_literal, read_ns,
    decode_signed_subexp_with_ref_bool and exit_symbol."""

    def __init__(self, data, sz, disable_cdf_update):
        self._lib = abi.load()
        self._data, p = _buf(data)
        self.s = abi.SymbolDecoder()
        _check(self._lib, self._lib.av1g_symbol_init(C.byref(self.s), p, sz, int(disable_cdf_update)))

    @property
    def position(self):
        return self.s.pos

    def read_symbol(self, cdf):
        arr = (C.c_uint16 * len(cdf))(*cdf)
        out = C.c_uint32()
        _check(self._lib, self._lib.av1g_symbol_read(C.byref(self.s), arr, len(cdf) - 1, C.byref(out)))
        cdf[:] = list(arr)
        return out.value

    def read_bool(self):
        out = C.c_uint32()
        _check(self._lib, self._lib.av1g_symbol_read_bool(C.byref(self.s), C.byref(out)))
        return out.value

    def read_literal(self, n):
        out = C.c_uint32()
        _check(self._lib, self._lib.av1g_symbol_read_literal(C.byref(self.s), n, C.byref(out)))
        return out.value

    def read_ns(self, n):
        out = C.c_uint32()
        _check(self._lib, self._lib.av1g_symbol_read_ns(C.byref(self.s), n, C.byref(out)))
        return out.value

    def decode_signed_subexp_with_ref_bool(self, low, high, k, r):
        out = C.c_int64()
        _check(self._lib, self._lib.av1g_symbol_read_signed_subexp(C.byref(self.s), low, high, k, r, C.byref(out)))
        return out.value

    def exit_symbol(self):
        t, e = C.c_uint64(), C.c_uint64()
        _check(self._lib, self._lib.av1g_symbol_exit(C.byref(self.s), C.byref(t), C.byref(e)))
        return t.value, e.value


def update_cdf(cdf, symbol, n):
    arr = (C.c_uint16 * len(cdf))(*cdf)
    abi.load().av1g_update_cdf(arr, symbol, n)
    cdf[:] = list(arr)


def new_ref_state():
    st = abi.RefState()
    abi.load().av1g_ref_state_init(C.byref(st))
    return st


def parse_frame_header(payload, seq, state, temporal_id=0, spatial_id=0):
    """The §5.9 uncompressed header (av1g_parsed_frame_header) of a frame
    header or frame OBU payload against the reference state."""
    lib = abi.load()
    data, p = _buf(payload)
    out = abi.ParsedFrameHeader()
    _check(lib, lib.av1g_parse_frame_header(p, len(data), C.byref(seq), C.byref(state), temporal_id, spatial_id,
                                            C.byref(out)))
    return out


def parse_tile_group(payload, fh):
    """(tg_start, tg_end, [(tile_num, offset, size)]) of a tile group."""
    lib = abi.load()
    data, p = _buf(payload)
    cap = max(1, fh.tile_cols * fh.tile_rows)
    spans = (abi.TileSpan * cap)()
    a, b = C.c_int32(), C.c_int32()
    _check(lib, lib.av1g_parse_tile_group(p, len(data), C.byref(fh), C.byref(a), C.byref(b), spans, cap))
    return a.value, b.value, [(spans[i].tile_num, spans[i].offset, spans[i].size) for i in range(b.value - a.value + 1)]


def stream_frame_headers(temporal_units, chosen_op=0):
    """Walks a stream's temporal units as the reference's
    decode_temporal_unit_spec does (frame_driver.rs:1618-1700): every frame
    header is parsed against the reference state, the tile groups of each
    frame are laid out until the frame's last tile, and the state is updated
    per decoded (or shown existing) frame.  Returns a list of
    (parsed header, [tile spans]) in decode order."""
    lib = abi.load()
    walker = TemporalUnitWalker(chosen_op)
    state = new_ref_state()
    out = []
    for tu in temporal_units:
        pending = None
        for d in walker.walk(tu):
            if d.obu_type in (3, 6):  # frame header, frame
                fh = parse_frame_header(d.payload, walker.seq, state, d.temporal_id, d.spatial_id)
                if fh.show_existing_frame:
                    _check(lib, lib.av1g_ref_state_update(C.byref(state), C.byref(fh)))
                    out.append((fh, []))
                    continue
                if d.obu_type == 3:
                    pending = (fh, [])
                    continue
                start = (fh.header_bits + 7) >> 3
                a, b, spans = parse_tile_group(d.payload[start:], fh)
                assert a == 0 and b == fh.tile_cols * fh.tile_rows - 1
                _check(lib, lib.av1g_ref_state_update(C.byref(state), C.byref(fh)))
                out.append((fh, spans))
            elif d.obu_type == 4 and pending is not None:  # tile group
                fh, spans = pending
                a, b, more = parse_tile_group(d.payload, fh)
                assert a == (spans[-1][0] + 1 if spans else 0)
                spans = spans + more
                pending = (fh, spans)
                if b == fh.tile_cols * fh.tile_rows - 1:
                    _check(lib, lib.av1g_ref_state_update(C.byref(state), C.byref(fh)))
                    out.append((fh, spans))
                    pending = None
    return out
