"""Python side of the serving engine (av1g_engine_* / av1g_stream_* /
av1g_submit_frame / av1g_poll / av1g_fetch_output in include/av1g.h).

A FrameDesc is built from host numpy arrays that stay referenced until the
submit call returns (the engine copies what it needs)."""
import ctypes as C

import numpy as np

from . import abi


def _p(a):
    return a.ctypes.data if a is not None and len(a) else None


class Engine:
    def __init__(self, device=0, max_batch=0, budget_bytes=0, max_inflight_steps=0, lanes=0, max_step_samples=0):
        self.lib = abi.load()
        cfg = abi.Config(device, max_batch, budget_bytes, max_inflight_steps, lanes, None, max_step_samples)
        h = C.c_void_p()
        abi.check(self.lib.av1g_engine_create(C.byref(cfg), C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            self.lib.av1g_engine_destroy(self.h)
            self.h = None

    def stats(self):
        s = abi.EngineStats()
        abi.check(self.lib.av1g_engine_get_stats(self.h, C.byref(s)))
        return s

    def open_stream(self, seq):
        info = abi.SeqInfo(seq["max_width"], seq["max_height"], seq["bit_depth"], seq["subsampling_x"],
                           seq["subsampling_y"], seq["num_planes"], seq["sb_size"])
        h = C.c_void_p()
        st = self.lib.av1g_stream_open(self.h, C.byref(info), C.byref(h))
        if st == abi.AV1G_ENOMEM_BUDGET:
            return None
        abi.check(st)
        return Stream(self, h)

    def poll(self, ticket, timeout_s=10.0):
        res = C.c_int(0)
        st = self.lib.av1g_poll(self.h, ticket, int(timeout_s * 1e9), C.byref(res))
        if st != abi.AV1G_OK:
            return None
        return res.value


class Stream:
    def __init__(self, engine, h):
        self.e, self.h = engine, h

    def close(self):
        if self.h:
            abi.check(self.e.lib.av1g_stream_close(self.h))
            self.h = None

    def reset_refs(self):
        abi.check(self.e.lib.av1g_stream_reset_refs(self.h))

    def submit(self, fr):
        """fr: a synth.StreamFrame."""
        d = abi.FrameDesc()
        keep = []
        d.hdr = C.pointer(fr.hdr)
        if fr.quant is not None:
            d.quant = C.pointer(fr.quant)
        if fr.grid is not None:
            for k in ["mi_size", "skip", "is_inter", "ref_frame0", "y_mode", "segment_id", "delta_lf", "tx_size",
                      "inter_tx_size"]:
                a = np.ascontiguousarray(fr.grid[k])
                keep.append(a)
                setattr(d.grid, k, a.ctypes.data)
        if fr.cdef_idx is not None:
            a = np.ascontiguousarray(fr.cdef_idx)
            keep.append(a)
            d.cdef_idx = a.ctypes.data
        for p in range(3):
            u = fr.lr_units[p] if fr.lr_units else None
            if u is not None:
                a = np.ascontiguousarray(u)
                keep.append(a)
                d.lr_units[p] = a.ctypes.data
        for name, cnt, arr in [("inter_preds", "num_inter_preds", fr.preds), ("neighbours", "num_neighbours",
                                                                              fr.neighbours),
                               ("warps", "num_warps", fr.warps), ("inter_tus", "num_inter_tus", fr.inter_tus),
                               ("intra_tus", "num_intra_tus", fr.intra_tus)]:
            if arr is not None and len(arr):
                a = np.ascontiguousarray(arr)
                keep.append(a)
                setattr(d, name, a.ctypes.data)
                setattr(d, cnt, len(a))
        if fr.palette_maps is not None and len(fr.palette_maps):
            a = np.ascontiguousarray(fr.palette_maps, np.uint8)
            keep.append(a)
            d.palette_maps, d.palette_map_bytes = a.ctypes.data, len(a)
        if fr.coeffs is not None and len(fr.coeffs):
            a = np.ascontiguousarray(fr.coeffs, np.int32)
            keep.append(a)
            d.coeffs, d.num_coeffs = a.ctypes.data, len(a)
        for i in range(7):
            d.ref_frame_idx[i] = fr.ref_frame_idx[i]
        d.refresh_frame_flags = fr.refresh
        d.show_frame = fr.show
        d.show_existing_frame = fr.show_existing
        d.frame_to_show_map_idx = fr.show_idx
        t = C.c_uint64(0)
        abi.check(self.e.lib.av1g_submit_frame(self.h, C.byref(d), C.byref(t)))
        return t.value

    def fetch(self, ticket, release=True):
        """(status, planes or None, latency_ms); planes are numpy copies."""
        o = abi.FrameOut()
        st = self.e.lib.av1g_fetch_output(self.h, ticket, C.byref(o))
        planes = None
        if st == abi.AV1G_OK and o.shown:
            dt = np.uint16 if o.bit_depth > 8 else np.uint8
            planes = []
            for p in range(o.num_planes):
                pl = o.planes[p]
                n = pl.stride * pl.height
                buf = (C.c_uint8 * n).from_address(pl.data)
                planes.append(np.frombuffer(buf, np.uint8).copy().view(dt).reshape(pl.height, pl.width))
        lat = o.latency_ms
        if release:
            self.e.lib.av1g_release_output(self.h, ticket)
        return st, planes, lat
