"""CPU parity oracle — TEST INFRASTRUCTURE ONLY.

A C restatement of the reference decoder's pixel path (see oracle.h), built
with gcc into ``liboxav1_oracle.so`` and driven through ctypes.  Only the test
suite, the smoke check and the bench's CPU-baseline / reference arms use it;
the engine never imports it.
"""
import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent
LIB = HERE / "liboxav1_oracle.so"
SOURCES = sorted(HERE.glob("*.c"))
HEADERS = [HERE / "oracle.h", REPO / "include" / "av1g.h",
           REPO / "oxideav-av1_b200" / "csrc" / "av1_spec_tables.h"]

_lib = None


def build(force=False):
    srcs = sorted(HERE.glob("*.c"))
    newest = max(p.stat().st_mtime for p in srcs + HEADERS)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = ["gcc", "-O2", "-fPIC", "-shared", "-Wall", "-Wno-missing-braces", "-std=gnu11",
               "-I" + str(REPO / "include"), "-I" + str(REPO / "oxideav-av1_b200" / "csrc"),
               *map(str, srcs), "-o", str(LIB), "-lm"]
        subprocess.run(cmd, check=True)
    return LIB


class OraPlane(C.Structure):
    _fields_ = [("s", C.POINTER(C.c_int32)), ("rows", C.c_int32), ("cols", C.c_int32)]


def load():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(str(LIB))
        _lib.ora_postfilter_frame.restype = C.c_int
        _lib.ora_random_next.restype = C.c_uint32
        _lib.ora_random_next.argtypes = [C.POINTER(C.c_uint16), C.c_int]
    return _lib


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _ptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _grid_struct(frame, keep):
    from_abi = _abi_module()
    g = from_abi.MiGrid()
    for k in ["mi_size", "skip", "is_inter", "ref_frame0", "y_mode", "segment_id", "delta_lf", "tx_size",
              "inter_tx_size"]:
        a = np.ascontiguousarray(frame.grid[k])
        keep.append(a)
        setattr(g, k, a.ctypes.data)
    return g


def _abi_module():
    import sys
    return sys.modules["oxideav_av1_b200.abi"]


def _units(frame, keep):
    arr = (C.c_void_p * 3)()
    for p in range(3):
        u = frame.lr_units[p]
        if u is not None:
            a = np.ascontiguousarray(u)
            keep.append(a)
            arr[p] = a.ctypes.data
    return arr


def postfilter_frame(frame):
    """Full §7.4 chain on the CPU; returns (ref_planes, out_planes) as int32 arrays."""
    lib = load()
    keep = []
    h = frame.hdr
    grid = _grid_struct(frame, keep)
    idx = np.ascontiguousarray(frame.cdef_idx)
    units = _units(frame, keep)
    recon = [_i32(frame.recon[p]) for p in range(h.num_planes)]
    rec_p = (C.POINTER(C.c_int32) * 3)(*[_ptr(r) for r in recon])
    refs, outs = [], []
    for p in range(h.num_planes):
        oh, ow = frame.out_dims(p)
        refs.append(np.zeros((oh, ow), np.int32))
        outs.append(np.zeros((oh, ow), np.int32))
    ref_p = (C.POINTER(C.c_int32) * 3)(*[_ptr(r) for r in refs])
    out_p = (C.POINTER(C.c_int32) * 3)(*[_ptr(r) for r in outs])
    rc = lib.ora_postfilter_frame(C.byref(h), C.byref(grid), idx.ctypes.data_as(C.c_void_p), units, rec_p,
                                  ref_p, out_p)
    if rc != 0:
        raise RuntimeError(f"oracle rejected the frame ({rc})")
    return refs, outs


def _planes(arrs):
    ps = (OraPlane * 3)()
    for i, a in enumerate(arrs):
        ps[i] = OraPlane(_ptr(a), a.shape[0], a.shape[1])
    return ps


def loop_filter(frame, planes):
    """§7.14 on int32 planes (modified in place)."""
    lib = load()
    keep = []
    grid = _grid_struct(frame, keep)
    lib.ora_loop_filter_frame(C.byref(frame.hdr), C.byref(grid), _planes(planes))
    return planes


def cdef(frame, src):
    lib = load()
    keep = []
    grid = _grid_struct(frame, keep)
    dst = [np.zeros_like(s) for s in src]
    idx = np.ascontiguousarray(frame.cdef_idx)
    lib.ora_cdef_frame(C.byref(frame.hdr), C.byref(grid), idx.ctypes.data_as(C.c_void_p), _planes(src),
                       _planes(dst))
    return dst


def upscale(frame, src):
    lib = load()
    dst = [np.zeros(frame.out_dims(p), np.int32) for p in range(frame.hdr.num_planes)]
    rc = lib.ora_upscale_frame(C.byref(frame.hdr), _planes(src), _planes(dst))
    if rc:
        raise RuntimeError("oracle upscale rejected the frame")
    return dst


def loop_restoration(frame, curr, cdef_planes):
    lib = load()
    keep = []
    units = _units(frame, keep)
    rows = (C.c_int32 * 3)()
    cols = (C.c_int32 * 3)()
    for p in range(frame.hdr.num_planes):
        rows[p], cols[p] = frame.lr_grid(p)
    lr = [np.zeros_like(c) for c in cdef_planes]
    lib.ora_lr_frame(C.byref(frame.hdr), units, rows, cols, _planes(curr), _planes(cdef_planes), _planes(lr))
    return lr


def film_grain(frame, planes):
    lib = load()
    h = frame.hdr
    lib.ora_film_grain(C.byref(h.film_grain), h.bit_depth, h.num_planes, h.subsampling_x, h.subsampling_y,
                       h.matrix_coefficients, _planes(planes))
    return planes


def generate_grain(fg, bit_depth, ssx, ssy):
    lib = load()
    luma = np.zeros((73, 82), np.int32)
    cw, ch = (44 if ssx else 82), (38 if ssy else 73)
    cb = np.zeros((ch, cw), np.int32)
    cr = np.zeros((ch, cw), np.int32)
    lib.ora_generate_grain(C.byref(fg), bit_depth, ssx, ssy, _ptr(luma), _ptr(cb), _ptr(cr))
    return luma, cb, cr


def scaling_lut(fg, num_planes):
    lib = load()
    lut = np.zeros((3, 256), np.uint8)
    lib.ora_scaling_lookup_init(C.byref(fg), num_planes, lut.ctypes.data_as(C.c_void_p))
    return lut


def random_draws(seed, bits, count):
    lib = load()
    st = C.c_uint16(seed)
    return [lib.ora_random_next(C.byref(st), bits) for _ in range(count)]


def recon(frame):
    """Dequant + inverse transform + merge of every TU onto the prediction planes (int32 copies)."""
    lib = load()
    planes = [np.ascontiguousarray(p, dtype=np.int32) for p in frame.planes]
    tus = np.ascontiguousarray(frame.tus)
    coeffs = np.ascontiguousarray(frame.coeffs, dtype=np.int32)
    lib.ora_recon_frame(C.byref(frame.hdr), C.byref(frame.quant), tus.ctypes.data_as(C.c_void_p), len(tus),
                        _ptr(coeffs), _planes(planes))
    return planes


def dequantize(quant, bit_depth, levels, tx, plane, segment_id, current_q_index, tx_type):
    lib = load()
    w = [4, 8, 16, 32, 64, 4, 8, 8, 16, 16, 32, 32, 64, 4, 16, 8, 32, 16, 64][tx]
    h = [4, 8, 16, 32, 64, 8, 4, 16, 8, 32, 16, 64, 32, 16, 4, 32, 8, 64, 16][tx]
    lv = np.ascontiguousarray(levels, dtype=np.int32)
    out = np.zeros(w * h, np.int64)
    lib.ora_dequantize(C.byref(quant), bit_depth, _ptr(lv), tx, plane, segment_id, current_q_index, tx_type,
                       out.ctypes.data_as(C.c_void_p))
    return out.reshape(h, w)


def inverse_transform(dequant, tx, tx_type, bit_depth, lossless=False):
    lib = load()
    d = np.ascontiguousarray(dequant, dtype=np.int64)
    res = np.zeros_like(d)
    lib.ora_inverse_transform_2d(d.ctypes.data_as(C.c_void_p), tx, tx_type, bit_depth, int(lossless),
                                 res.ctypes.data_as(C.c_void_p))
    return res


def intra_rc(frame):
    """Every intra TU in decode order (prediction, CfL, residual) on int32 copies
    of the planes; returns (planes, rc) with rc = 0 or 1 + the first rejected TU."""
    lib = load()
    planes = [np.ascontiguousarray(p, dtype=np.int32) for p in frame.planes]
    tus = np.ascontiguousarray(frame.tus)
    coeffs = np.ascontiguousarray(frame.coeffs, dtype=np.int32)
    maps = np.ascontiguousarray(getattr(frame, "palette_maps", np.zeros(1, np.uint8)), dtype=np.uint8)
    side = getattr(frame, "interintra_side", None)
    side = None if side is None else [None if a is None else np.ascontiguousarray(a, dtype=np.int32) for a in side]
    rc = lib.ora_intra_frame(C.byref(frame.hdr), C.byref(frame.quant), tus.ctypes.data_as(C.c_void_p), len(tus),
                             _ptr(coeffs), _planes(planes), maps.ctypes.data_as(C.c_void_p),
                             C.c_int64(len(getattr(frame, "palette_maps", []))), _side_planes(side))
    return planes, rc


def intra(frame):
    planes, rc = intra_rc(frame)
    if rc:
        raise RuntimeError(f"oracle rejected intra TU {rc - 1}")
    return planes


def intrabc_predict(plane_arr, plane, ssx, ssy, mi_cols, mi_rows, x, y, w, h, mv_row, mv_col, bd):
    lib = load()
    a = np.ascontiguousarray(plane_arr, dtype=np.int32)
    p = OraPlane(_ptr(a), a.shape[0], a.shape[1])
    out = np.zeros((h, w), np.uint16)
    rc = lib.ora_intrabc_predict(C.byref(p), plane, ssx, ssy, mi_cols, mi_rows, x, y, w, h, mv_row, mv_col, bd,
                                 out.ctypes.data_as(C.c_void_p))
    return None if rc else out


def _struct_ptr(a):
    return a.ctypes.data_as(C.c_void_p) if len(a) else None


def _side_planes(side):
    """OraPlane[3] over int32 arrays (None entries: no side plane), or None."""
    if side is None:
        return None
    arr = (OraPlane * 3)()
    for p, a in enumerate(side):
        if a is not None:
            arr[p] = OraPlane(_ptr(a), a.shape[0], a.shape[1])
    return arr


def inter(frame, side=None):
    """Every inter prediction call in list order on int32 copies of the planes.
    side: None, or a list of int32 arrays (CurrFrame shape) that receive the
    inter halves of inter-intra calls instead of the blend.

    Returns (planes, rc): rc is 0, or 1 + the index of the first call the
    reference rejects."""
    lib = load()
    abi = _abi_module()
    planes = [np.ascontiguousarray(p, dtype=np.int32) for p in frame.planes]
    refs = (abi.RefFrame * 7)()
    ref_planes = (OraPlane * 21)()
    keep = []
    for r in range(7):
        refs[r].upscaled_width = frame.refs[r]["upscaled_width"]
        refs[r].frame_height = frame.refs[r]["frame_height"]
        for p in range(3):
            a = np.ascontiguousarray(frame.refs[r]["planes"][p], dtype=np.int32)
            keep.append(a)
            ref_planes[r * 3 + p] = OraPlane(_ptr(a), a.shape[0], a.shape[1])
    preds = np.ascontiguousarray(frame.preds)
    nb = np.ascontiguousarray(frame.neighbours)
    warps = np.ascontiguousarray(frame.warps)
    rc = lib.ora_inter_frame(C.byref(frame.hdr), refs, ref_planes, _struct_ptr(preds), len(preds),
                             _struct_ptr(nb), len(nb), _struct_ptr(warps), len(warps), _planes(planes),
                             _side_planes(side))
    return planes, rc


def mv_scaling(plane, ssx, ssy, fw, fh, ruw, rh, x, y, mv_row, mv_col):
    lib = load()
    out = (C.c_int32 * 4)()
    rc = lib.ora_mv_scaling(plane, ssx, ssy, fw, fh, ruw, rh, x, y, mv_row, mv_col, out)
    return None if rc else tuple(out)


def setup_shear(params):
    lib = load()
    p = (C.c_int32 * 6)(*params)
    out = (C.c_int32 * 5)()
    rc = lib.ora_setup_shear(p, out)
    return None if rc else tuple(out)


def wedge_mask(mi_size, wedge_index, wedge_sign):
    lib = load()
    w = [4, 4, 8, 8, 8, 16, 16, 16, 32, 32, 32, 64, 64, 64, 128, 128, 4, 16, 8, 32, 16, 64][mi_size]
    h = [4, 8, 4, 8, 16, 8, 16, 32, 16, 32, 64, 32, 64, 128, 64, 128, 16, 4, 32, 8, 64, 16][mi_size]
    m = np.zeros((h, w), np.uint8)
    rc = lib.ora_wedge_mask(mi_size, wedge_index, wedge_sign, m.ctypes.data_as(C.c_void_p))
    return None if rc else m


def warp_estimation(cands, mi_row, mi_col, bw4, bh4, mv_row, mv_col):
    """cands: sequence of (sy, sx, dy, dx).  Returns (valid, params)."""
    lib = load()
    arr = np.ascontiguousarray(np.array(cands, np.int32).reshape(-1, 4))
    params = (C.c_int32 * 6)()
    v = lib.ora_warp_estimation(arr.ctypes.data_as(C.c_void_p), len(arr), mi_row, mi_col, bw4, bh4, mv_row, mv_col,
                                params)
    return bool(v), list(params)



class _Obj:
    pass


def decode_stream(frames):
    """Sequential CPU decode of synth.StreamFrame objects: inter calls, inter
    residuals, intra TUs, the §7.4 chain, slot refresh with the pre-grain
    frame, output (show_existing_frame: the slot with its grain).  Returns the
    shown frames' int32 planes in order (None for frames not shown)."""
    import copy
    from oxideav_av1_b200 import synth
    slots = [None] * 8
    outs = []
    for fr in frames:
        if fr.show_existing:
            sl = slots[fr.show_idx]
            planes = [p.copy() for p in sl["planes"]]
            if sl["hdr"].film_grain.apply_grain:
                o = _Obj()
                o.hdr = sl["hdr"]
                film_grain(o, planes)
            for i in range(8):
                if (fr.refresh >> i) & 1:
                    slots[i] = sl
            outs.append(planes)
            continue
        h = fr.hdr
        ph = lambda p: ((h.mi_rows * 4) >> (h.subsampling_y if p else 0), (h.mi_cols * 4) >> (h.subsampling_x if p else 0))
        planes = [np.zeros(ph(p), np.int32) for p in range(h.num_planes)]
        side = None
        if fr.preds is not None and (fr.preds["kind"] == 2).any():
            # inter halves of inter-intra blocks wait for their intra halves
            # (the reference's per-block order; see tests/test_oracle_interintra_split.py)
            side = [np.zeros(ph(p), np.int32) for p in range(h.num_planes)]
        if fr.preds is not None and len(fr.preds):
            o = _Obj()
            o.hdr, o.preds, o.neighbours, o.warps, o.planes = h, fr.preds, fr.neighbours, fr.warps, planes
            o.refs = []
            for r in range(7):
                sl = slots[fr.ref_frame_idx[r]]
                pls = list(sl["planes"]) + [np.zeros((1, 1), np.int32)] * (3 - len(sl["planes"]))
                o.refs.append({"planes": pls, "upscaled_width": sl["uw"], "frame_height": sl["fh"]})
            planes, rc = inter(o, side=side)
            if rc:
                raise RuntimeError(f"oracle rejected inter call {rc - 1}")
        if fr.inter_tus is not None and len(fr.inter_tus):
            o = _Obj()
            o.hdr, o.quant, o.tus, o.coeffs, o.planes = h, fr.quant, fr.inter_tus, fr.coeffs, planes
            planes = recon(o)
        if fr.intra_tus is not None and len(fr.intra_tus):
            o = _Obj()
            o.hdr, o.quant, o.tus, o.coeffs, o.planes = h, fr.quant, fr.intra_tus, fr.coeffs, planes
            o.palette_maps = fr.palette_maps if fr.palette_maps is not None else np.zeros(0, np.uint8)
            o.interintra_side = side
            planes = intra(o)
        sf = synth.SyntheticFrame()
        sf.hdr, sf.grid, sf.cdef_idx, sf.lr_units, sf.recon = h, fr.grid, fr.cdef_idx, fr.lr_units, planes
        ref, out = postfilter_frame(sf)
        if fr.refresh:
            sl = {"planes": ref, "uw": h.upscaled_width, "fh": h.frame_height, "hdr": copy.copy(h)}
            for i in range(8):
                if (fr.refresh >> i) & 1:
                    slots[i] = sl
        outs.append(out if fr.show else None)
    return outs


def relative_dist(a, b, bits):
    """get_relative_dist (inter_pred.rs:3383)."""
    return load().ora_relative_dist(int(a), int(b), int(bits))


def mv_projection(mv, numerator, denominator):
    """§7.9.3 get_mv_projection (cdf.rs:35101) of mv = (row, col)."""
    lib = load()
    src = (C.c_int * 2)(int(mv[0]), int(mv[1]))
    out = (C.c_int * 2)()
    lib.ora_mv_projection(src, int(numerator), int(denominator), out)
    return [out[0], out[1]]


def block_position(x8, y8, sign, proj_mv, mi_rows, mi_cols):
    """§7.9.4 get_block_position (cdf.rs:35141): (pos_y8, pos_x8) or None."""
    py, px = C.c_int(), C.c_int()
    ok = load().ora_block_position(x8, y8, sign, int(proj_mv[0]), int(proj_mv[1]), mi_rows, mi_cols, C.byref(py),
                                   C.byref(px))
    return (py.value, px.value) if ok else None


def mf_store(mi_rows, mi_cols, is_inter, order_hint, hint_bits, ref_order_hint, ref_frames, mvs):
    """§7.19 storage of one frame (frame_driver.rs:1119-1160).

    ref_frames: int8 [cells, 2]; mvs: int16 [cells, 2, 2].  Returns
    (mf_ref_frames int8 [cells], mf_mvs int16 [cells, 2])."""
    abi = _abi_module()
    cells = mi_rows * mi_cols
    rf = np.ascontiguousarray(ref_frames, dtype=np.int8).reshape(-1)
    mv = np.ascontiguousarray(mvs, dtype=np.int16).reshape(-1)
    assert rf.size == 2 * cells and mv.size == 4 * cells
    out_r = np.empty(cells, np.int8)
    out_m = np.empty((cells, 2), np.int16)
    j = abi.MfStoreJob(mi_rows, mi_cols, int(is_inter), order_hint, hint_bits, (C.c_int32 * 7)(*ref_order_hint),
                       rf.ctypes.data, mv.ctypes.data, out_r.ctypes.data, out_m.ctypes.data)
    load().ora_mf_store(C.byref(j))
    return out_r, out_m


def mf_project(slots, ref_frame_idx, order_hints, order_hint, hint_bits, mi_rows, mi_cols):
    """§7.9 motion_field_estimation_core (inter_pred.rs:7592) for one frame.

    slots: 8 entries, None or dict(mf_mvs int16 [cells, 2], mf_ref_frames
    int8 [cells], saved_order_hints (8), mi_rows, mi_cols, frame_is_intra).
    Returns the MotionFieldMvs grid, int16 [7, mi_rows >> 1, mi_cols >> 1, 2]."""
    abi = _abi_module()
    j = abi.MfProjectJob()
    keep = []
    for i, sl in enumerate(slots):
        if sl is None:
            continue
        m = np.ascontiguousarray(sl["mf_mvs"], dtype=np.int16)
        r = np.ascontiguousarray(sl["mf_ref_frames"], dtype=np.int8)
        keep += [m, r]
        j.slots[i] = abi.MfSlot(m.ctypes.data, r.ctypes.data, (C.c_int32 * 8)(*sl["saved_order_hints"]),
                                sl["mi_rows"], sl["mi_cols"], int(sl["frame_is_intra"]), 0)
    for k in range(7):
        j.ref_frame_idx[k] = ref_frame_idx[k]
    for k in range(8):
        j.order_hints[k] = order_hints[k]
    j.order_hint, j.hint_bits, j.mi_rows, j.mi_cols = order_hint, hint_bits, mi_rows, mi_cols
    out = np.empty((7, mi_rows >> 1, mi_cols >> 1, 2), np.int16)
    j.out = out.ctypes.data
    load().ora_mf_project(C.byref(j))
    return out


def tile_list_output(tile_w, tile_h, width_in_tiles, height_in_tiles, ssx, ssy, bit_depth, tiles):
    """The §7.3.1 placement of decode_tile_list (src/tile_list.rs:665-740):
    tiles = list of (camera frame planes, x0, y0) in list order; tile k goes
    to (tile_w * (k % width_in_tiles), tile_h * (k // width_in_tiles)), chroma
    shifted by the subsampling; the rest of the output stays 0; samples are
    clamped to the bit depth."""
    np_ = len(tiles[0][0])
    ow, oh = width_in_tiles * tile_w, height_in_tiles * tile_h
    dims = [(oh, ow) if p == 0 else (oh >> ssy, ow >> ssx) for p in range(np_)]
    out = [np.zeros(d, np.int32) for d in dims]
    for k, (planes, x0, y0) in enumerate(tiles):
        dx, dy = tile_w * (k % width_in_tiles), tile_h * (k // width_in_tiles)
        for p in range(np_):
            sx, sy = (ssx, ssy) if p else (0, 0)
            tw, th = (tile_w + sx) >> sx, (tile_h + sy) >> sy
            src = np.asarray(planes[p], np.int32)[y0 >> sy: (y0 >> sy) + th, x0 >> sx: (x0 >> sx) + tw]
            out[p][dy >> sy: (dy >> sy) + th, dx >> sx: (dx >> sx) + tw] = src
    return [np.clip(o, 0, (1 << bit_depth) - 1) for o in out]
