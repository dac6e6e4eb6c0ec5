"""Device-resident post-filter frames and the calls into the CUDA library.

``DeviceFrame`` uploads a frame's grids, CDEF indices, restoration units and
reconstructed planes to HBM once and allocates the chain's intermediate planes
(deblocked, CDEF, upscaled, restored, output) with 64-byte aligned rows.  The
``run_*`` functions fill ``av1g_frame_job`` records for a batch and call the
library; PyTorch is used only to own device memory and streams.
"""
import ctypes as C

import numpy as np
import torch

from . import abi

ALIGN = 64


def _pitch(width, bps):
    return (width * bps + ALIGN - 1) // ALIGN * ALIGN


class DevPlane:
    """A byte tensor of rows x pitch holding u8 or u16 samples."""

    def __init__(self, height, width, hbd, device, fill=None):
        self.h, self.w, self.hbd = height, width, hbd
        self.bps = 2 if hbd else 1
        self.pitch = _pitch(width, self.bps)
        self.t = torch.zeros((height, self.pitch), dtype=torch.uint8, device=device)
        if fill is not None:
            self.upload(fill)

    def upload(self, arr):
        a = np.ascontiguousarray(arr)
        assert a.shape == (self.h, self.w)
        raw = a.view(np.uint8).reshape(self.h, self.w * self.bps)
        self.t[:, : self.w * self.bps].copy_(torch.from_numpy(raw))

    def download(self, height=None, width=None):
        h = self.h if height is None else height
        w = self.w if width is None else width
        raw = self.t[:h, : w * self.bps].cpu().numpy()
        return raw.view(np.uint16 if self.hbd else np.uint8).reshape(h, w)

    def cplane(self, width=None, height=None):
        return abi.Plane(self.t.data_ptr(), self.pitch, self.w if width is None else width,
                         self.h if height is None else height)


class DeviceFrame:
    """One frame's inputs and work buffers on the GPU."""

    GRID_KEYS = ["mi_size", "skip", "is_inter", "ref_frame0", "y_mode", "segment_id", "delta_lf", "tx_size",
                 "inter_tx_size"]

    def __init__(self, frame, device="cuda"):
        self.frame = frame
        self.hdr = frame.hdr
        h = frame.hdr
        hbd = frame.hbd
        self.grid = {k: torch.from_numpy(np.ascontiguousarray(frame.grid[k])).to(device) for k in self.GRID_KEYS}
        self.cdef_idx = torch.from_numpy(np.ascontiguousarray(frame.cdef_idx)).to(device)
        self.lr_units = []
        for p in range(3):
            u = frame.lr_units[p]
            self.lr_units.append(None if u is None else
                                 torch.from_numpy(np.ascontiguousarray(u).view(np.uint8).reshape(-1)).to(device))
        np_ = h.num_planes
        self.recon = [DevPlane(*frame.plane_dims(p), hbd, device, fill=frame.recon[p]) for p in range(np_)]
        self.deblocked = [DevPlane(*frame.plane_dims(p), hbd, device) for p in range(np_)]
        self.cdef = [DevPlane(*frame.plane_dims(p), hbd, device) for p in range(np_)]
        sr = h.use_superres and h.upscaled_width > h.frame_width
        self.up_cdef = [DevPlane(*frame.out_dims(p), hbd, device) for p in range(np_)] if sr else []
        self.up_deblocked = [DevPlane(*frame.out_dims(p), hbd, device) for p in range(np_)] if sr else []
        # the restored planes share the padded or upscaled extent of their input
        lr_dims = [frame.out_dims(p) if sr else frame.plane_dims(p) for p in range(np_)]
        self.lr = [DevPlane(*lr_dims[p], hbd, device) for p in range(np_)]
        self.out = [DevPlane(*frame.out_dims(p), hbd, device) for p in range(np_)]
        self._hdr_ref = h

    def job(self):
        j = abi.FrameJob()
        j.hdr = C.pointer(self._hdr_ref)
        for k in self.GRID_KEYS:
            setattr(j.grid, k, self.grid[k].data_ptr())
        j.cdef_idx = self.cdef_idx.data_ptr()
        for p in range(3):
            j.lr_units[p] = self.lr_units[p].data_ptr() if self.lr_units[p] is not None else None
        for p in range(self.hdr.num_planes):
            j.recon[p] = self.recon[p].cplane()
            j.deblocked[p] = self.deblocked[p].cplane()
            j.cdef[p] = self.cdef[p].cplane()
            if self.up_cdef:
                j.up_cdef[p] = self.up_cdef[p].cplane()
                j.up_deblocked[p] = self.up_deblocked[p].cplane()
            j.lr[p] = self.lr[p].cplane()
            j.out[p] = self.out[p].cplane()
        return j

    # which buffer holds each stage's result after gating (mirrors api.cu)
    def stage_planes(self):
        h = self.hdr
        res = {}
        do_deb = (h.lf_level[0] or h.lf_level[1]) and not h.coded_lossless and not h.allow_intrabc
        do_cdef = not h.coded_lossless and not h.allow_intrabc and h.enable_cdef and not h.cdef_short_circuited
        do_sr = h.use_superres and h.upscaled_width > h.frame_width
        deb, cdef, lr, out = [], [], [], []
        for p in range(h.num_planes):
            d = self.deblocked[p] if do_deb and (p == 0 or h.lf_level[1 + p]) else self.recon[p]
            c = self.cdef[p] if do_cdef else d
            uc = self.up_cdef[p] if do_sr else c
            ud = self.up_deblocked[p] if do_sr and h.uses_lr else d
            l_ = self.lr[p] if h.uses_lr and h.lr_type[p] else uc
            o = self.out[p] if h.film_grain.apply_grain else l_
            deb.append(d)
            cdef.append(c)
            lr.append(l_)
            out.append(o)
            res.setdefault("up_cdef", []).append(uc)
            res.setdefault("up_deblocked", []).append(ud)
        res.update(deblocked=deb, cdef=cdef, lr=lr, out=out)
        return res

    def download(self, stage):
        """Host copy of a stage's result planes (the cropped view for lr/out)."""
        planes = self.stage_planes()[stage]
        res = []
        for p, pl in enumerate(planes):
            if stage in ("lr", "out"):
                oh, ow = self.frame.out_dims(p)
                res.append(pl.download(oh, ow))
            else:
                res.append(pl.download())
        return res


def jobs_array(frames):
    arr = (abi.FrameJob * len(frames))()
    for i, f in enumerate(frames):
        arr[i] = f.job()
    return arr


def _stream_ptr(stream):
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def run_stage(name, frames, stream=None):
    lib = abi.load()
    jobs = jobs_array(frames)
    fn = getattr(lib, "av1g_run_" + name)
    abi.check(fn(jobs, len(frames), _stream_ptr(stream)))
    return jobs


def run_postfilter(frames, mode=abi.MODE_BATCHED, stream=None, jobs=None):
    """Runs the whole chain for the frames; returns the kernel launch count."""
    lib = abi.load()
    if jobs is None:
        jobs = jobs_array(frames)
    n = C.c_int32(0)
    abi.check(lib.av1g_run_postfilter(jobs, len(frames), mode, _stream_ptr(stream), C.byref(n)))
    return n.value


class DeviceRecon:
    """A reconstruction frame on the GPU: prediction planes (updated in place) + coefficient pool."""

    def __init__(self, rframe, device="cuda"):
        self.frame = rframe
        hbd = rframe.hbd
        self.planes = [DevPlane(*rframe.plane_dims(p), hbd, device, fill=rframe.planes[p])
                       for p in range(rframe.hdr.num_planes)]
        self.coeffs = torch.from_numpy(np.ascontiguousarray(rframe.coeffs)).to(device)
        self.tus = np.ascontiguousarray(rframe.tus)   # host array: the library buckets and uploads it

    def job(self):
        j = abi.ReconJob()
        j.hdr = C.pointer(self.frame.hdr)
        j.quant = C.pointer(self.frame.quant)
        j.tus = self.tus.ctypes.data
        j.num_tus = len(self.tus)
        j.coeffs = self.coeffs.data_ptr()
        for p, pl in enumerate(self.planes):
            j.planes[p] = pl.cplane()
        return j

    def download(self):
        return [pl.download() for pl in self.planes]


def run_recon(frames, stream=None):
    lib = abi.load()
    arr = (abi.ReconJob * len(frames))()
    for i, f in enumerate(frames):
        arr[i] = f.job()
    abi.check(lib.av1g_run_recon(arr, len(frames), _stream_ptr(stream)))
    return arr


class DeviceIntra(DeviceRecon):
    """An intra frame on the GPU: planes (reconstructed in place) + coefficient pool + TU list."""

    def job(self):
        j = abi.IntraJob()
        j.hdr = C.pointer(self.frame.hdr)
        j.quant = C.pointer(self.frame.quant)
        j.tus = self.tus.ctypes.data
        j.num_tus = len(self.tus)
        j.sb_size = self.frame.sb_size
        j.coeffs = self.coeffs.data_ptr()
        for p, pl in enumerate(self.planes):
            j.planes[p] = pl.cplane()
        self._maps = np.ascontiguousarray(getattr(self.frame, "palette_maps", np.zeros(0, np.uint8)), np.uint8)
        j.palette_maps = self._maps.ctypes.data if len(self._maps) else None
        j.palette_map_bytes = len(self._maps)
        for p, sp in enumerate(getattr(self, "side", None) or []):
            j.interintra_in[p] = sp.cplane()
        return j


def run_intra(frames, stream=None):
    lib = abi.load()
    arr = (abi.IntraJob * len(frames))()
    for i, f in enumerate(frames):
        arr[i] = f.job()
    abi.check(lib.av1g_run_intra(arr, len(frames), _stream_ptr(stream)))
    return arr


class DeviceInter:
    """An inter frame on the GPU: CurrFrame planes (written in place), the 7
    reference planes, and the host call / neighbour / warp lists."""

    def __init__(self, frame, device="cuda", side=False):
        self.frame = frame
        h = frame.hdr
        hbd = h.bit_depth > 8
        self.planes = [DevPlane(*frame.plane_dims(p), hbd, device, frame.planes[p]) for p in range(h.num_planes)]
        # inter halves of inter-intra calls, when their blend is left to av1g_run_intra
        self.side = [DevPlane(*frame.plane_dims(p), hbd, device) for p in range(h.num_planes)] if side else None
        self.refs = (abi.RefFrame * 7)()
        self.ref_planes = []
        for r, ref in enumerate(frame.refs):
            self.refs[r].upscaled_width = ref["upscaled_width"]
            self.refs[r].frame_height = ref["frame_height"]
            for p in range(h.num_planes):
                a = ref["planes"][p]
                dp = DevPlane(a.shape[0], a.shape[1], hbd, device, a)
                self.ref_planes.append(dp)
                self.refs[r].planes[p] = dp.cplane()
        self.preds = np.ascontiguousarray(frame.preds)
        self.neighbours = np.ascontiguousarray(frame.neighbours)
        self.warps = np.ascontiguousarray(frame.warps)

    def job(self):
        j = abi.InterJob()
        j.hdr = C.pointer(self.frame.hdr)
        j.refs = C.cast(self.refs, C.POINTER(abi.RefFrame))
        j.preds = self.preds.ctypes.data if len(self.preds) else None
        j.num_preds = len(self.preds)
        j.neighbours = self.neighbours.ctypes.data if len(self.neighbours) else None
        j.num_neighbours = len(self.neighbours)
        j.warps = self.warps.ctypes.data if len(self.warps) else None
        j.num_warps = len(self.warps)
        for p, pl in enumerate(self.planes):
            j.planes[p] = pl.cplane()
            if self.side:
                j.interintra_out[p] = self.side[p].cplane()
        return j

    def download(self):
        return [pl.download() for pl in self.planes]


def run_inter(frames, stream=None):
    lib = abi.load()
    arr = (abi.InterJob * len(frames))()
    for i, f in enumerate(frames):
        arr[i] = f.job()
    abi.check(lib.av1g_run_inter(arr, len(frames), _stream_ptr(stream)))
    return arr
