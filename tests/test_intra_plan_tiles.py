"""Tiles run side by side in the intra wavefront (host plan, no GPU).

The intra launch's plan (av1g_intra_plan_stats_get reports it without
running anything) gives each superblock waits only on the superblocks whose
samples its TUs read, as the TUs' availability flags name them.  The tile
walker bounds those flags by the tile (§5.11 AvailU / AvailL stop at the tile
edge), so with a 2 x 2 tile grid the longest chain of waits runs through one
tile only: the critical path shrinks and more superblocks share a depth.
"""
import ctypes as C

import numpy as np
import pytest

from oxideav_av1_b200 import abi, synth


def _stats(f, sb):
    lib = abi.load()
    coeffs = np.ascontiguousarray(f.coeffs, np.int32)  # never read by the planner
    j = abi.IntraJob()
    j.hdr = C.pointer(f.hdr)
    j.quant = C.pointer(f.quant)
    tus = np.ascontiguousarray(f.tus)
    j.tus, j.num_tus, j.sb_size = tus.ctypes.data, len(tus), sb
    j.coeffs = coeffs.ctypes.data
    maps = np.ascontiguousarray(f.palette_maps, np.uint8)
    if len(maps):
        j.palette_maps, j.palette_map_bytes = maps.ctypes.data, len(maps)
    for p in range(f.hdr.num_planes):
        ph, pw = f.plane_dims(p)
        j.planes[p] = abi.Plane(1 << 20, pw * (2 if f.hdr.bit_depth > 8 else 1), pw, ph)  # not dereferenced
    st = abi.IntraPlanStats()
    abi.check(lib.av1g_intra_plan_stats_get(C.byref(j), 1, C.byref(st)))
    return st, tus


@pytest.mark.parametrize("w,h,sb", [(1280, 720, 64), (1920, 1088, 128)])
def test_tiles_shorten_the_critical_path(w, h, sb):
    one, tus1 = _stats(synth.make_intra_frame(41, w, h, sb_size=sb, split=0.6), sb)
    four, tus4 = _stats(synth.make_intra_frame(41, w, h, sb_size=sb, split=0.6, tiles=(1, 1)), sb)
    assert one.superblocks == four.superblocks
    sb_cols, sb_rows = -(-w // sb), -(-h // sb)
    # one tile: a wavefront over the whole frame; 2 x 2: over a quarter
    assert one.depth >= sb_cols + sb_rows - 1
    assert four.depth < one.depth
    assert four.depth <= (-(-sb_cols // 2)) * 2 + (-(-sb_rows // 2)) * 2
    assert four.width >= 2 * one.width - 2


def test_tile_edges_bound_availability():
    f = synth.make_intra_frame(43, 512, 256, sb_size=64, tiles=(1, 1), ssx=0, ssy=0)
    tcols, trows = synth.tile_grid(f.hdr.mi_rows, f.hdr.mi_cols, 64, 1, 1)
    xs = {a for a, _ in tcols}
    ys = {a for a, _ in trows}
    t = f.tus
    on_left = np.isin(t["x"], list(xs))
    on_top = np.isin(t["y"], list(ys))
    assert on_left.any() and on_top.any()
    assert not (t["flags"][on_left] & (abi.INTRA_HAVE_LEFT | abi.INTRA_HAVE_BELOW_LEFT)).any()
    assert not (t["flags"][on_top] & (abi.INTRA_HAVE_ABOVE | abi.INTRA_HAVE_ABOVE_RIGHT)).any()
