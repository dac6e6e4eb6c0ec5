"""The registry Decoder API over the whole decode path.

`Av1Decoder` mirrors the reference's `Av1Decoder` (src/registry.rs:103-195):
`send_packet` takes a whole IVF file or one temporal unit, `receive_frame`
returns the next shown frame (raising `NeedMore` when none is queued and
`Eof` after `flush`), `reset` drops the reference state.  Host work (OBU walk,
frame headers, the tile walk) runs in the C++ library, every pixel stage in the
GPU engine; there is no CPU path.

`parse_stream` runs the same host walk without an engine and returns each
frame's descriptor as a `synth.StreamFrame`, the form the test suite's
checkers take.
"""
import ctypes as C
import hashlib

import numpy as np

from . import abi, synth


class NeedMore(Exception):
    """receive_frame: no frame is queued (send another packet)."""


class Eof(Exception):
    """receive_frame after flush: every frame has been returned."""


class Frame:
    """A decoded frame: planes as numpy arrays (uint8, or uint16 for 10/12-bit
    content), pts, bit depth."""

    def __init__(self, planes, bit_depth, pts):
        self.planes, self.bit_depth, self.pts = planes, bit_depth, pts

    def tobytes(self):
        """The SpecFrame byte layout: planes back to back, u8 or little-endian u16."""
        return b"".join(p.astype("<u2").tobytes() if self.bit_depth > 8 else p.tobytes() for p in self.planes)


class Av1Decoder:
    def __init__(self, engine, operating_point=0):
        self.lib = abi.load()
        self.engine = engine
        h = C.c_void_p()
        abi.check(self.lib.av1g_decoder_create(engine.h if engine is not None else None, operating_point,
                                               C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.av1g_decoder_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def send_packet(self, data, pts=0):
        data = bytes(data)
        buf = (C.c_uint8 * max(len(data), 1)).from_buffer_copy(data or b"\0")
        abi.check(self.lib.av1g_decoder_send_packet(self.h, buf, len(data), pts))

    def receive_frame(self):
        o = abi.FrameOut()
        pts = C.c_int64()
        st = self.lib.av1g_decoder_receive_frame(self.h, C.byref(o), C.byref(pts))
        if st == abi.AV1G_ENOTREADY:
            raise NeedMore()
        if st == abi.AV1G_EOF:
            raise Eof()
        abi.check(st)
        dt = np.uint16 if o.bit_depth > 8 else np.uint8
        planes = []
        for p in range(o.num_planes):
            pl = o.planes[p]
            n = pl.stride * pl.height
            raw = (C.c_uint8 * n).from_address(pl.data)
            planes.append(np.frombuffer(raw, np.uint8).copy().view(dt).reshape(pl.height, pl.width))
        return Frame(planes, o.bit_depth, pts.value)

    def flush(self):
        abi.check(self.lib.av1g_decoder_flush(self.h))

    def reset(self):
        abi.check(self.lib.av1g_decoder_reset(self.h))

    def host_ms(self):
        return self.lib.av1g_decoder_host_ms(self.h)

    def drain(self):
        out = []
        while True:
            try:
                out.append(self.receive_frame())
            except (NeedMore, Eof):
                return out


def decode(data, engine, operating_point=0):
    """Every shown frame of an IVF file (or one temporal unit), in order."""
    dec = Av1Decoder(engine, operating_point)
    try:
        dec.send_packet(data)
        dec.flush()
        return dec.drain()
    finally:
        dec.close()


def digest(frames):
    """SHA-256 of the frames' planes back to back (the conformance tests' digest)."""
    h = hashlib.sha256()
    for f in frames:
        h.update(f.tobytes())
    return h.hexdigest()


# ---------------------------------------------------------------------------
# parse-only: the descriptors the host walk produces
# ---------------------------------------------------------------------------

def _copy(ptr, dtype, count, shape=None):
    if not ptr or count == 0:
        return np.zeros(0 if shape is None else shape, dtype)
    n = np.dtype(dtype).itemsize * count
    raw = (C.c_uint8 * n).from_address(ptr)
    a = np.frombuffer(raw, np.uint8).copy().view(dtype)
    return a.reshape(shape) if shape is not None else a


def _stream_frame(desc, fh):
    fr = synth.StreamFrame()
    fr.hdr = abi.FrameHeader.from_buffer_copy(desc.hdr.contents)
    h = fr.hdr
    fr.ref_frame_idx = list(desc.ref_frame_idx)
    fr.refresh = desc.refresh_frame_flags
    fr.show = desc.show_frame
    fr.show_existing = desc.show_existing_frame
    fr.show_idx = desc.frame_to_show_map_idx
    if fr.show_existing:
        return fr
    fr.quant = abi.QuantParams.from_buffer_copy(desc.quant.contents)
    cells = h.mi_rows * h.mi_cols
    g = desc.grid
    fr.grid = {}
    for k, dt in [("mi_size", np.uint8), ("skip", np.uint8), ("is_inter", np.uint8), ("ref_frame0", np.int8),
                  ("y_mode", np.uint8), ("segment_id", np.int8), ("tx_size", np.uint8), ("inter_tx_size", np.uint8)]:
        fr.grid[k] = _copy(getattr(g, k), dt, cells, (h.mi_rows, h.mi_cols))
    fr.grid["delta_lf"] = _copy(g.delta_lf, np.int8, cells * 4, (h.mi_rows, h.mi_cols, 4))
    fr.cdef_idx = _copy(desc.cdef_idx, np.int8, ((h.mi_rows + 15) >> 4) * ((h.mi_cols + 15) >> 4),
                        ((h.mi_rows + 15) >> 4, (h.mi_cols + 15) >> 4))
    lib = abi.load()
    for p in range(3):
        fr.lr_units[p] = None
        if p < h.num_planes and h.lr_type[p] and desc.lr_units[p]:
            sx, sy = (h.subsampling_x, h.subsampling_y) if p else (0, 0)
            rows = lib.av1g_lr_units_in_frame(h.lr_unit_size[p], (h.frame_height + sy) >> sy)
            cols = lib.av1g_lr_units_in_frame(h.lr_unit_size[p], (h.upscaled_width + sx) >> sx)
            fr.lr_units[p] = _copy(desc.lr_units[p], synth.LR_DTYPE, rows * cols, (rows, cols))
    fr.preds = _copy(desc.inter_preds, synth.INTER_DTYPE, desc.num_inter_preds)
    fr.neighbours = _copy(desc.neighbours, synth.NB_DTYPE, desc.num_neighbours)
    fr.warps = _copy(desc.warps, synth.WARP_DTYPE, desc.num_warps)
    fr.inter_tus = _copy(desc.inter_tus, synth.TU_DTYPE, desc.num_inter_tus)
    fr.intra_tus = _copy(desc.intra_tus, synth.INTRA_TU_DTYPE, desc.num_intra_tus)
    fr.palette_maps = _copy(desc.palette_maps, np.uint8, desc.palette_map_bytes)
    fr.coeffs = _copy(desc.coeffs, np.int32, desc.num_coeffs)
    return fr


def parse_stream(data, operating_point=0):
    """(sequence header, [synth.StreamFrame per frame in decode order]) of an
    IVF file, from the host walk alone (no engine, no pixels)."""
    lib = abi.load()
    h = C.c_void_p()
    abi.check(lib.av1g_decoder_create(None, operating_point, C.byref(h)))
    try:
        data = bytes(data)
        buf = (C.c_uint8 * max(len(data), 1)).from_buffer_copy(data or b"\0")
        abi.check(lib.av1g_decoder_send_packet(h, buf, len(data), 0))
        frames = []
        for i in range(lib.av1g_decoder_parsed_count(h)):
            d = abi.FrameDesc()
            fh = abi.ParsedFrameHeader()
            abi.check(lib.av1g_decoder_parsed_frame(h, i, C.byref(d), C.byref(fh)))
            frames.append(_stream_frame(d, fh))
        seq = abi.SequenceHeader()
        abi.check(lib.av1g_decoder_sequence(h, C.byref(seq)))
        parse_stream.frames_out_of_sync = lib.av1g_decoder_frames_out_of_sync(h)
        return seq, frames
    finally:
        lib.av1g_decoder_destroy(h)
