"""Launch-shape autotuner (av1g_autotune_*) and the shapes it can pick.

The tuner times every candidate shape of every post-filter stage on a real
batch and keeps the fastest; whatever it picks, the chain's output must stay
the oracle's.  Every superres tile width and a spread of grid sizes are also
forced through a cache file and checked against the oracle, and malformed
cache lines are rejected.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

FRAMES = [
    dict(seed=61, width=352, height=288, superres_denom=11),
    dict(seed=62, width=200, height=120, superres_denom=16, film_grain=True),
    dict(seed=63, width=130, height=70, ssx=0, ssy=0, film_grain=True),
]


def _run_and_check(frames):
    dframes = [postfilter.DeviceFrame(f) for f in frames]
    postfilter.run_postfilter(dframes)
    torch.cuda.synchronize()
    for f, d in zip(frames, dframes):
        _, out = oracle.postfilter_frame(f)
        for p, (g, r) in enumerate(zip(d.download("out"), out)):
            diff = np.argwhere(g.astype(np.int64) != r)
            assert len(diff) == 0, f"plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"


def _get(lib, stage, hbd):
    c, t = C.c_int32(), C.c_int32()
    abi.check(lib.av1g_autotune_get(stage, hbd, C.byref(c), C.byref(t)))
    return c.value, t.value


def test_autotune_picks_valid_shapes_and_keeps_parity(tmp_path):
    lib = abi.load()
    frames = [synth.make_frame(**c) for c in FRAMES]
    dframes = [postfilter.DeviceFrame(f) for f in frames]
    jobs = postfilter.jobs_array(dframes)
    cache = tmp_path / "shapes.txt"
    stream = torch.cuda.Stream()
    abi.check(lib.av1g_autotune_postfilter(jobs, len(dframes), C.c_void_p(stream.cuda_stream),
                                           str(cache).encode()))
    for stage in range(5):
        c, t = _get(lib, stage, 0)
        assert 1 <= c <= 64
        if stage == 2:
            assert t in (256, 512, 1024)
    lines = [l for l in cache.read_text().splitlines() if not l.startswith("#")]
    assert len(lines) == 10
    abi.check(lib.av1g_autotune_load(str(cache).encode()))
    _run_and_check(frames)


@pytest.mark.parametrize("tile,ctas", [(256, 1), (512, 5), (1024, 33)])
def test_forced_shapes_keep_parity(tmp_path, tile, ctas):
    lib = abi.load()
    cache = tmp_path / "forced.txt"
    cache.write_text("".join(f"{st} {h} {ctas} {tile if st == 2 else 0}\n" for st in range(5) for h in range(2)))
    abi.check(lib.av1g_autotune_load(str(cache).encode()))
    try:
        assert _get(lib, 2, 1) == (ctas, tile)
        _run_and_check([synth.make_frame(**c) for c in FRAMES])
    finally:  # back to the defaults for the tests that follow
        cache.write_text("".join(f"{st} {h} {c} {t}\n" for st, c, t in
                                 [(0, 16, 0), (1, 16, 0), (2, 16, 512), (3, 8, 0), (4, 8, 0)] for h in range(2)))
        abi.check(lib.av1g_autotune_load(str(cache).encode()))


def test_malformed_cache_is_rejected(tmp_path):
    lib = abi.load()
    cache = tmp_path / "bad.txt"
    cache.write_text("2 0 16 300\n9 0 4 0\nnot a line\n")
    assert lib.av1g_autotune_load(str(cache).encode()) == abi.AV1G_EINVAL
    assert lib.av1g_autotune_load(str(tmp_path / "missing.txt").encode()) == abi.AV1G_EINVAL
    assert _get(lib, 2, 0)[1] in (256, 512, 1024)
