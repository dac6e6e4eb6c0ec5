"""The §7.4 chain captured as a CUDA graph (av1g_chain_graph_*) against the oracle.

A graph is captured once over a fixed batch of frames (every stage, the
reference's gating, superres and film grain included, mixed bit depths and
chroma formats) and replayed: each replay must give the oracle's output, in
the batched and the per-frame launch mode, and a replay after the frames'
input samples are rewritten in place must give the oracle's output for the
new samples (the graph bakes in pointers, not data).
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

FRAMES = [
    dict(seed=41, width=352, height=288),
    dict(seed=42, width=200, height=120, bit_depth=10, film_grain=True),
    dict(seed=43, width=176, height=144, superres_denom=12, film_grain=True),
    dict(seed=44, width=130, height=70, ssx=0, ssy=0),
]


def _check(frames, dframes):
    for f, d in zip(frames, dframes):
        ref_out, out = oracle.postfilter_frame(f)
        got = d.download("out")
        for p, (g, r) in enumerate(zip(got, out)):
            diff = np.argwhere(g.astype(np.int64) != r)
            assert len(diff) == 0, f"plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"


def _graph(lib, jobs, n, mode, stream):
    g = C.c_void_p()
    abi.check(lib.av1g_chain_graph_create(jobs, n, (1 << 5) - 1, mode, C.c_void_p(stream.cuda_stream), C.byref(g)))
    return g


@pytest.mark.parametrize("mode", [abi.MODE_BATCHED, abi.MODE_PER_FRAME], ids=["batched", "per_frame"])
def test_graph_replay_matches_oracle(mode):
    lib = abi.load()
    frames = [synth.make_frame(**c) for c in FRAMES]
    dframes = [postfilter.DeviceFrame(f) for f in frames]
    jobs = postfilter.jobs_array(dframes)
    stream = torch.cuda.Stream()
    g = _graph(lib, jobs, len(dframes), mode, stream)
    try:
        assert lib.av1g_chain_graph_launches(g) > 0
        for d in dframes:  # clear the outputs the capture run wrote
            for pl in d.out + d.lr:
                pl.t.zero_()
        torch.cuda.synchronize()
        for _ in range(2):
            abi.check(lib.av1g_chain_graph_launch(g, C.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize()
        _check(frames, dframes)
    finally:
        abi.check(lib.av1g_chain_graph_destroy(g))


def test_graph_replay_follows_new_samples():
    lib = abi.load()
    frames = [synth.make_frame(**c) for c in FRAMES[:2]]
    dframes = [postfilter.DeviceFrame(f) for f in frames]
    jobs = postfilter.jobs_array(dframes)
    stream = torch.cuda.Stream()
    g = _graph(lib, jobs, len(dframes), abi.MODE_BATCHED, stream)
    try:
        rng = np.random.default_rng(5)
        for f, d in zip(frames, dframes):  # new reconstructed samples, same buffers
            maxv = (1 << f.hdr.bit_depth) - 1
            for p in range(len(f.recon)):
                f.recon[p] = np.clip(f.recon[p].astype(np.int64) + rng.integers(-9, 10, f.recon[p].shape), 0,
                                     maxv).astype(f.recon[p].dtype)
                d.recon[p].upload(f.recon[p])
        torch.cuda.synchronize()
        abi.check(lib.av1g_chain_graph_launch(g, C.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize()
        _check(frames, dframes)
    finally:
        abi.check(lib.av1g_chain_graph_destroy(g))


def test_graph_rejects_bad_arguments():
    lib = abi.load()
    g = C.c_void_p()
    assert lib.av1g_chain_graph_create(None, 0, 31, abi.MODE_BATCHED, None, C.byref(g)) == abi.AV1G_EINVAL
    f = synth.make_frame(seed=45, width=64, height=64)
    d = postfilter.DeviceFrame(f)
    jobs = postfilter.jobs_array([d])
    assert lib.av1g_chain_graph_create(jobs, 1, 1 << 7, abi.MODE_BATCHED, None, C.byref(g)) == abi.AV1G_EINVAL
    assert lib.av1g_chain_graph_launch(None, None) == abi.AV1G_EINVAL
    assert lib.av1g_chain_graph_destroy(None) == abi.AV1G_OK
