"""Intra prediction + reconstruction on the GPU (superblock wavefront) against the oracle.

Every mode (DC, V, H, the six directional modes with angle deltas, edge filter
and upsampling, SMOOTH/_V/_H, PAETH), recursive filter intra, chroma from luma,
palette prediction, intra block copy (reading within the level-2 wavefront,
further right so that a steeper wavefront is needed, and from not yet decoded
superblocks so that only decode order reproduces the reference) and residuals,
with availability flags derived from decode order, at 8/10/12 bits, 4:2:0,
4:4:4 and monochrome, 64x64 and 128x128 superblocks.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = [
    dict(seed=81, width=176, height=144),
    dict(seed=82, width=176, height=144, bit_depth=10),
    dict(seed=83, width=200, height=120, bit_depth=12, edge_filter=False),
    dict(seed=84, width=130, height=70, ssx=0, ssy=0),
    dict(seed=85, width=96, height=96, mono=True),
    dict(seed=86, width=352, height=288, sb_size=128),
    dict(seed=87, width=640, height=360),
    dict(seed=90, width=176, height=144, palette=0.3),
    dict(seed=91, width=352, height=288, intrabc=0.4),
    dict(seed=92, width=640, height=360, intrabc=0.4, intrabc_order="steep"),
    dict(seed=93, width=1280, height=128, intrabc=0.5, intrabc_order="raster"),
    dict(seed=94, width=352, height=288, bit_depth=10, palette=0.2, intrabc=0.2, ssx=0, ssy=0),
    # 128x128 superblocks of 4:4:4 4x4 TUs (thousands per superblock: the TU window slides)
    dict(seed=96, width=256, height=192, sb_size=128, ssx=0, ssy=0, split=0.97),
    # palette blocks read no neighbours: a superblock's tiny TUs share one level wider than the TU window
    dict(seed=97, width=256, height=128, palette=1.0, split=0.95),
]


def _check(f, d):
    exp = oracle.intra(f)
    for p, (g, e) in enumerate(zip(d.download(), exp)):
        diff = np.argwhere(g.astype(np.int64) != e)
        assert len(diff) == 0, f"plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"


@pytest.mark.parametrize("case", CASES, ids=[f"c{c['seed']}" for c in CASES])
def test_intra_parity(case):
    abi.load()
    f = synth.make_intra_frame(**case)
    d = postfilter.DeviceIntra(f)
    postfilter.run_intra([d])
    torch.cuda.synchronize()
    _check(f, d)


def test_intra_batch_of_frames_shares_levels():
    abi.load()
    frames = [synth.make_intra_frame(**c) for c in CASES[:5]]
    devs = [postfilter.DeviceIntra(f) for f in frames]
    postfilter.run_intra(devs)
    torch.cuda.synchronize()
    for f, d in zip(frames, devs):
        _check(f, d)


def test_intra_rejects_split_superblock():
    abi.load()
    f = synth.make_intra_frame(seed=88, width=128, height=64)
    tus = f.tus.copy()
    # move the first luma TU of the second superblock to the front: that superblock's
    # TUs are no longer contiguous in decode order
    k = int(np.argmax((tus["plane"] == 0) & (tus["x"] >= 64)))
    f.tus = np.concatenate([tus[k:k + 1], tus[:k], tus[k + 1:]])
    d = postfilter.DeviceIntra(f)
    with pytest.raises(abi.Av1gError):
        postfilter.run_intra([d])


def test_intra_rejects_palette_index_out_of_range():
    abi.load()
    f = synth.make_intra_frame(seed=95, width=128, height=64, palette=1.0)
    k = int(np.argmax(f.tus["mode"] == abi.INTRA_MODE_PALETTE))
    t = f.tus[k]
    f.palette_maps = f.palette_maps.copy()
    f.palette_maps[int(t["palette_map"])] = int(t["palette_size"])
    assert oracle.intra_rc(f)[1] == k + 1
    d = postfilter.DeviceIntra(f)
    with pytest.raises(abi.Av1gError):
        postfilter.run_intra([d])


def test_concurrent_launches_with_different_shared_memory_sizes():
    """Two host threads (as engine lanes do) run av1g_run_intra on their own
    streams at the same time, one with 64x64 4:2:0 superblocks (a small
    shared-memory copy) and one with 128x128 4:4:4 superblocks (the largest):
    the kernel's shared-memory limit is a per-device attribute, so neither
    thread's launches may fail because of the other's, and both frames come
    out equal to the oracle."""
    import ctypes as C
    import threading

    lib = abi.load()
    fa = synth.make_intra_frame(seed=98, width=176, height=144)
    fb = synth.make_intra_frame(seed=99, width=256, height=192, sb_size=128, ssx=0, ssy=0, bit_depth=10)
    da, db = postfilter.DeviceIntra(fa), postfilter.DeviceIntra(fb)
    torch.cuda.synchronize()
    errors = []

    def worker(d):
        torch.cuda.set_device(0)
        s = torch.cuda.Stream()
        jobs = (abi.IntraJob * 1)(d.job())
        for _ in range(40):  # a frame re-run from its inputs gives the same samples
            rc = lib.av1g_run_intra(jobs, 1, C.c_void_p(s.cuda_stream))
            if rc != abi.AV1G_OK:
                errors.append((rc, lib.av1g_last_error()))
                break
        s.synchronize()

    ts = [threading.Thread(target=worker, args=(d,)) for d in (da, db)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors
    _check(fa, da)
    _check(fb, db)
