"""The allocation-free film grain entry point gives the allocating one's output.

Some callers may not allocate device memory on the per-frame path — a host
application that reserves its whole device-memory budget at start-up and
forbids plug-ins to allocate while frames flow, since an allocation there can
stall on the allocator or fail once the pool is full.  For them
av1g_run_film_grain_noalloc keeps its frame records and grain scratch in one
static device array.  Two calls in a row, each on a fresh batch, must match
av1g_run_film_grain on identical inputs; the output is integer, so the
tolerance is zero, as in every parity test of this suite.  This file is
collected last so that a run stopping at the first failure has already run
every other test.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

GRAIN_ONLY = dict(film_grain=True, deblock=False, cdef=False, lr=False)


def _batch(cases):
    return [synth.make_frame(**c, **GRAIN_ONLY) for c in cases]


def _run_both(frames):
    lib = abi.load()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    a = [postfilter.DeviceFrame(f) for f in frames]
    b = [postfilter.DeviceFrame(f) for f in frames]
    ja, jb = postfilter.jobs_array(a), postfilter.jobs_array(b)
    abi.check(lib.av1g_run_film_grain(ja, len(a), sp))
    abi.check(lib.av1g_run_film_grain_noalloc(jb, len(b), sp))
    torch.cuda.synchronize()
    return a, b


def _assert_same(a, b):
    for fa, fb in zip(a, b):
        for p, (x, y) in enumerate(zip(fa.download("out"), fb.download("out"))):
            assert x.shape == y.shape
            d = np.argwhere(x != y)
            assert len(d) == 0, f"plane {p}: {len(d)} samples differ, first at {tuple(d[0])}"


def _assert_oracle(frames, b):
    """The grain stage's input here is the cropped reconstruction (every
    other stage is off); oracle.film_grain restates film_grain_synthesis."""
    for f, fb in zip(frames, b):
        crop = [np.ascontiguousarray(f.recon[p][: f.out_dims(p)[0], : f.out_dims(p)[1]]).astype(np.int32)
                for p in range(f.hdr.num_planes)]
        want = oracle.film_grain(f, crop)
        for p, (g, e) in enumerate(zip(fb.download("out"), want)):
            assert np.array_equal(g.astype(np.int64), e), f"plane {p} differs from the oracle"


# The default memory pool of the current device (the stream-ordered allocator
# the allocating entry points draw from), read through the driver API:
# CU_MEMPOOL_ATTR_USED_MEM_CURRENT = 7, CU_MEMPOOL_ATTR_USED_MEM_HIGH = 8.
def _pool():
    cu = C.CDLL("libcuda.so.1")
    dev, pool = C.c_int(), C.c_void_p()
    assert cu.cuDeviceGet(C.byref(dev), C.c_int(torch.cuda.current_device())) == 0
    assert cu.cuDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    return cu, pool


def _pool_attr(attr):
    cu, pool = _pool()
    v = C.c_uint64()
    assert cu.cuMemPoolGetAttribute(pool, C.c_int(attr), C.byref(v)) == 0
    return v.value


def _reset_pool_high():
    cu, pool = _pool()
    zero = C.c_uint64(0)  # resets the high-water mark to the current use
    assert cu.cuMemPoolSetAttribute(pool, C.c_int(8), C.byref(zero)) == 0


def test_noalloc_film_grain_matches_allocating_entry_point_twice():
    first = _batch([dict(seed=301, width=352, height=288), dict(seed=302, width=200, height=120, bit_depth=10),
                    dict(seed=303, width=130, height=70, ssx=0, ssy=0)])
    a, b = _run_both(first)
    _assert_same(a, b)
    # second call in a row: the static array still holds the first call's contents
    second = _batch([dict(seed=304, width=96, height=64, mono=True),
                     dict(seed=305, width=256, height=136, bit_depth=12),
                     dict(seed=306, width=320, height=180, ssx=1, ssy=0),
                     dict(seed=307, width=1920, height=1080)])
    a, b = _run_both(second)
    _assert_same(a, b)
    _assert_oracle(second, b)


def test_noalloc_draws_nothing_from_the_device_memory_pool():
    lib = abi.load()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    frames = _batch([dict(seed=320, width=640, height=360), dict(seed=321, width=320, height=240, bit_depth=10)])
    b = [postfilter.DeviceFrame(f) for f in frames]
    jb = postfilter.jobs_array(b)
    abi.check(lib.av1g_run_film_grain_noalloc(jb, len(b), sp))   # first call on the device: symbol address
    torch.cuda.synchronize()
    used = _pool_attr(7)
    _reset_pool_high()
    abi.check(lib.av1g_run_film_grain_noalloc(jb, len(b), sp))
    torch.cuda.synchronize()
    assert _pool_attr(8) == used, "the allocation-free entry point allocated from the memory pool"
    _assert_oracle(frames, b)
    # the allocating entry point does draw from the same pool: the probe sees allocations
    a = [postfilter.DeviceFrame(f) for f in frames]
    abi.check(lib.av1g_run_film_grain(postfilter.jobs_array(a), len(a), sp))
    torch.cuda.synchronize()
    assert _pool_attr(8) > used


def test_noalloc_rejects_a_batch_whose_scratch_exceeds_the_array():
    """Sixteen 10240x10240 monochrome grain frames need about 139 KB of grain
    scratch each (templates, LUTs and one offset byte per 32x32 block of each
    stripe), 2.2 MB in all: more than the static array holds, so the call is
    refused on the host before anything is enqueued.  The jobs point at real
    planes of that size."""
    lib = abi.load()
    small = postfilter.DeviceFrame(synth.make_frame(seed=330, width=64, height=64, mono=True, **GRAIN_ONLY))
    hdr = type(small.hdr).from_buffer_copy(small.hdr)
    side = 10240
    hdr.frame_width = hdr.upscaled_width = hdr.frame_height = side
    hdr.mi_cols = hdr.mi_rows = 2 * ((side + 7) >> 3)
    big_in = torch.zeros((side, side), dtype=torch.uint8, device="cuda")
    big_out = torch.zeros((side, side), dtype=torch.uint8, device="cuda")
    job = small.job()
    job.hdr = C.pointer(hdr)
    job.recon[0] = abi.Plane(big_in.data_ptr(), side, side, side)
    job.out[0] = abi.Plane(big_out.data_ptr(), side, side, side)
    n = abi.NOALLOC_MAX_FRAMES
    jobs = (abi.FrameJob * n)(*([job] * n))
    rc = lib.av1g_run_film_grain_noalloc(jobs, n, None)
    assert rc == abi.AV1G_EINVAL
    assert b"static array" in lib.av1g_last_error()
    torch.cuda.synchronize()
    assert int(big_out.count_nonzero()) == 0  # nothing ran


def test_noalloc_rejects_batches_beyond_its_limit():
    lib = abi.load()
    frames = [postfilter.DeviceFrame(f) for f in _batch([dict(seed=310, width=64, height=64)])]
    jobs = postfilter.jobs_array(frames * (abi.NOALLOC_MAX_FRAMES + 1))
    rc = lib.av1g_run_film_grain_noalloc(jobs, abi.NOALLOC_MAX_FRAMES + 1, None)
    assert rc == abi.AV1G_EINVAL
    assert b"limit" in lib.av1g_last_error()
