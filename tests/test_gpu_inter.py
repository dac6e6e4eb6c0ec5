"""Inter prediction on the GPU against the oracle.

Single reference, compound average / distance / wedge / difference weight,
inter-intra (smooth and wedge masks), OBMC with above and left neighbours,
local and global warp, references at other sizes (2x, 1/2, 1.5x, and 3x past
the spec's 2x limit), the 4-tap small-block filters, edge clamping and calls
clipped at the plane edge, at 8/10/12 bits in 4:2:0, 4:2:2, 4:4:4 and mono.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = [
    dict(seed=101, width=176, height=144),
    dict(seed=102, width=176, height=144, bit_depth=10),
    dict(seed=103, width=200, height=120, bit_depth=12),
    dict(seed=104, width=130, height=70, ssx=0, ssy=0),
    dict(seed=105, width=160, height=96, ssx=1, ssy=0),
    dict(seed=106, width=96, height=96, mono=True),
    dict(seed=107, width=352, height=288, sb_size=128),
    dict(seed=108, width=640, height=360, p_intra=0.0),
    dict(seed=109, width=176, height=144, scaled=False),
]


def _check(f, d):
    exp, rc = oracle.inter(f)
    assert rc == 0, f"oracle rejected call {rc - 1}"
    for p, (g, e) in enumerate(zip(d.download(), exp)):
        diff = np.argwhere(g.astype(np.int64) != e)
        assert len(diff) == 0, f"plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"


@pytest.mark.parametrize("case", CASES, ids=[f"c{c['seed']}" for c in CASES])
def test_inter_parity(case):
    abi.load()
    f = synth.make_inter_frame(**case)
    d = postfilter.DeviceInter(f)
    postfilter.run_inter([d])
    torch.cuda.synchronize()
    _check(f, d)


def test_inter_batch_of_frames():
    abi.load()
    frames = [synth.make_inter_frame(**c) for c in CASES[:6]]
    devs = [postfilter.DeviceInter(f) for f in frames]
    postfilter.run_inter(devs)
    torch.cuda.synchronize()
    for f, d in zip(frames, devs):
        _check(f, d)


def _ramp():
    return (np.arange(16)[:, None] * 16 + np.arange(16)[None, :]).astype(np.uint8)


def test_inter_half_sample_golden():
    # the reference's r291 hand-built golden vector, on the GPU
    abi.load()
    f = synth.custom_inter_frame(16, 16, [(16, 16, [_ramp()])], [dict(x=4, y=4, w=4, h=4, mv=[[0, 4], [0, 0]])])
    d = postfilter.DeviceInter(f)
    postfilter.run_inter([d])
    torch.cuda.synchronize()
    got = d.download()[0]
    assert got[4:8, 4:8].tolist() == [[69, 70, 71, 72], [85, 86, 87, 88], [101, 102, 103, 104],
                                      [117, 118, 119, 120]]


def test_inter_rejects_caller_bugs():
    abi.load()
    for c in [dict(x=0, y=0, w=4, h=4, ref=[7, 0]), dict(x=0, y=0, w=8, h=8, motion_mode=2),
              dict(x=0, y=0, w=4, h=4, filter_x=6), dict(x=16, y=0, w=4, h=4)]:
        f = synth.custom_inter_frame(16, 16, [(16, 16, [_ramp()])], [c])
        d = postfilter.DeviceInter(f)
        with pytest.raises(abi.Av1gError):
            postfilter.run_inter([d])


II_CASES = [dict(seed=311), dict(seed=312, bit_depth=10), dict(seed=313, ssx=0, ssy=0), dict(seed=314, mono=True),
            dict(seed=315, width=200, height=120, bit_depth=12)]


@pytest.mark.parametrize("case", II_CASES, ids=[f"s{c['seed']}" for c in II_CASES])
def test_interintra_two_pass_on_gpu(case):
    # the inter pass leaves inter-intra blocks' inter halves in side planes;
    # the intra wavefront blends them with the intra halves, as in
    # tests/test_oracle_interintra_split.py
    from test_oracle_interintra_split import ii_case, split_order
    abi.load()
    f, quant, tus, coeffs = ii_case(**case)
    want = split_order(f, quant, tus, coeffs)
    d = postfilter.DeviceInter(f, side=True)
    postfilter.run_inter([d])
    it = synth.IntraFrame()
    it.hdr, it.quant, it.tus, it.coeffs, it.planes = f.hdr, quant, tus, coeffs, f.planes
    di = postfilter.DeviceIntra(it)
    di.planes, di.side = d.planes, d.side
    postfilter.run_intra([di])
    torch.cuda.synchronize()
    for p, (g, e) in enumerate(zip(di.download(), want)):
        diff = np.argwhere(g.astype(np.int64) != e)
        assert len(diff) == 0, f"plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"
