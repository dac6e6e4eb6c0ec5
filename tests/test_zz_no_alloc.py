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


def test_noalloc_rejects_batches_beyond_its_limit():
    lib = abi.load()
    frames = [postfilter.DeviceFrame(f) for f in _batch([dict(seed=310, width=64, height=64)])]
    jobs = postfilter.jobs_array(frames * (abi.NOALLOC_MAX_FRAMES + 1))
    rc = lib.av1g_run_film_grain_noalloc(jobs, abi.NOALLOC_MAX_FRAMES + 1, None)
    assert rc == abi.AV1G_EINVAL
    assert b"limit" in lib.av1g_last_error()
