"""Dequant + inverse transform + merge on the GPU against the oracle (bit-exact).

Covers every transform size (4x4 .. 64x64, the 4:1 and 2:1 rectangles), every
type a size admits (16 types up to 16 samples, DCT/IDTX at 32, DCT at 64),
FLIPADST merges, lossless WHT segments, quantizer matrices, segmentation
alt-q and delta-q, coefficient clamping, 8/10/12-bit and 4:2:0/4:4:4/4:2:2/mono.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = [
    dict(seed=61, width=352, height=288),
    dict(seed=62, width=352, height=288, bit_depth=10),
    dict(seed=63, width=200, height=136, bit_depth=12),
    dict(seed=64, width=130, height=70, ssx=0, ssy=0),
    dict(seed=65, width=256, height=128, ssx=1, ssy=0),
    dict(seed=66, width=96, height=96, mono=True),
    dict(seed=67, width=1920, height=1080),
]


@pytest.mark.parametrize("case", CASES, ids=[f"c{c['seed']}" for c in CASES])
def test_recon_parity(case):
    abi.load()
    f = synth.make_recon_frame(**case)
    d = postfilter.DeviceRecon(f)
    postfilter.run_recon([d])
    torch.cuda.synchronize()
    exp = oracle.recon(f)
    for p, (g, e) in enumerate(zip(d.download(), exp)):
        diff = np.argwhere(g.astype(np.int64) != e)
        assert len(diff) == 0, f"plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"


def test_recon_batch_of_mixed_frames():
    abi.load()
    frames = [synth.make_recon_frame(**c) for c in CASES[:6]]
    devs = [postfilter.DeviceRecon(f) for f in frames]
    postfilter.run_recon(devs)
    torch.cuda.synchronize()
    for f, d in zip(frames, devs):
        for g, e in zip(d.download(), oracle.recon(f)):
            assert np.array_equal(g.astype(np.int64), e)


def test_recon_rejects_bad_tu():
    abi.load()
    f = synth.make_recon_frame(seed=70, width=64, height=64)
    f.tus["tx_size"][0] = 19
    d = postfilter.DeviceRecon(f)
    with pytest.raises(abi.Av1gError) as e:
        postfilter.run_recon([d])
    assert e.value.status == abi.AV1G_EINVAL
