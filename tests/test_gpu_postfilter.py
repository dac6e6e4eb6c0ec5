"""Per-stage and whole-chain parity of the CUDA post-filter path with the oracle.

Modelled on the reference's conformance A/B harnesses (tests/cdef_ab.rs,
tests/lr_ab.rs, tests/film_grain_ab.rs, tests/superres_ab.rs): the same seeded
frame goes through the CPU oracle and the GPU engine, and every stage's output
planes must be byte-identical.  Integer path: the tolerance is zero.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = [
    dict(seed=11, width=352, height=288),                                   # 4:2:0 8-bit, CIF
    dict(seed=12, width=200, height=120, bit_depth=10),                     # 10-bit
    dict(seed=13, width=130, height=70, ssx=0, ssy=0),                      # 4:4:4, non-mi-aligned
    dict(seed=14, width=96, height=64, mono=True),                          # monochrome
    dict(seed=15, width=176, height=144, superres_denom=13),                # superres
    dict(seed=16, width=176, height=144, film_grain=True),                  # film grain
    dict(seed=17, width=178, height=146, bit_depth=10, film_grain=True, superres_denom=10),
    dict(seed=18, width=256, height=136, bit_depth=12, film_grain=True),    # 12-bit
    dict(seed=19, width=320, height=180, lr_unit=128, lr_uv_shift=1, lr_none_frac=0.3),
    dict(seed=20, width=320, height=180, ssx=1, ssy=0, film_grain=True),    # 4:2:2
    dict(seed=21, width=64, height=64, lr_unit=256, deblock=False),         # deblock off
    dict(seed=22, width=150, height=98, cdef=False, lr_types=(1, 0, 2)),    # cdef off, per-plane LR types
    dict(seed=23, width=1920, height=1080),                                 # full-size 1080p
    dict(seed=24, width=1920, height=1080, bit_depth=10),                   # full-size 10-bit
    dict(seed=25, width=130, height=70, ssx=0, ssy=0, film_grain=True),     # 4:4:4 grain, odd width / 4
    dict(seed=26, width=98, height=66, mono=True, film_grain=True),         # monochrome grain
    dict(seed=27, width=177, height=143, film_grain=True),                  # odd sizes, grain
    dict(seed=28, width=322, height=182, bit_depth=10, ssx=1, ssy=0, film_grain=True),  # 4:2:2 10-bit grain
    # 32-sample chroma restoration units: LR tiles half as wide as the four-output runs assume
    dict(seed=29, width=200, height=120, lr_unit=64, lr_uv_shift=1),
    dict(seed=30, width=210, height=100, bit_depth=10, lr_unit=64, lr_uv_shift=1, lr_none_frac=0.2),
]


def _ids(c):
    return "-".join(f"{k}{v}" for k, v in c.items() if k != "seed") or "default"


def _first_diff(a, b):
    d = np.argwhere(a != b)
    if len(d) == 0:
        return None
    y, x = d[0]
    return f"{len(d)} samples differ; first at (y={y}, x={x}): gpu={a[y, x]} oracle={b[y, x]}"


def _assert_planes(stage, gpu, ref):
    for p, (g, r) in enumerate(zip(gpu, ref)):
        assert g.shape == r.shape, f"{stage} plane {p}: shape {g.shape} vs {r.shape}"
        msg = _first_diff(g.astype(np.int64), r.astype(np.int64))
        assert msg is None, f"{stage} plane {p}: {msg}"


def oracle_stages(f):
    """Each stage's expected planes, following frame_driver.rs:830-1096."""
    h = f.hdr
    rec = [r.astype(np.int32) for r in f.recon]
    do_deb = (h.lf_level[0] or h.lf_level[1]) and not h.coded_lossless and not h.allow_intrabc
    deb = oracle.loop_filter(f, [r.copy() for r in rec]) if do_deb else rec
    do_cdef = not h.coded_lossless and not h.allow_intrabc and h.enable_cdef and not h.cdef_short_circuited
    cd = oracle.cdef(f, deb) if do_cdef else deb
    if h.use_superres and h.upscaled_width > h.frame_width:
        up_c = oracle.upscale(f, cd)
        up_d = oracle.upscale(f, deb) if h.uses_lr else None
    else:
        up_c, up_d = cd, deb
    lr = oracle.loop_restoration(f, up_d, up_c) if h.uses_lr else up_c
    crop = [np.ascontiguousarray(lr[p][: f.out_dims(p)[0], : f.out_dims(p)[1]]) for p in range(h.num_planes)]
    out = oracle.film_grain(f, [c.copy() for c in crop]) if h.film_grain.apply_grain else crop
    return dict(deblocked=deb, cdef=cd, up_cdef=up_c, lr=crop, out=out)


@pytest.fixture(scope="module")
def lib():
    return abi.load()


@pytest.mark.parametrize("case", CASES, ids=[_ids(c) for c in CASES])
def test_stage_parity(lib, case):
    f = synth.make_frame(**case)
    df = postfilter.DeviceFrame(f)
    postfilter.run_postfilter([df])
    torch.cuda.synchronize()
    exp = oracle_stages(f)
    _assert_planes("deblock", df.download("deblocked"), exp["deblocked"])
    _assert_planes("cdef", df.download("cdef"), exp["cdef"])
    if f.hdr.use_superres:
        got = [p.download() for p in df.stage_planes()["up_cdef"]]
        _assert_planes("superres", got, exp["up_cdef"])
    _assert_planes("loop restoration", df.download("lr"), exp["lr"])
    _assert_planes("film grain", df.download("out"), exp["out"])


@pytest.mark.parametrize("case", CASES[:12], ids=[_ids(c) for c in CASES[:12]])
def test_chain_matches_oracle_chain(lib, case):
    """Whole chain against the oracle's frame-driver restatement (ref payload and output)."""
    f = synth.make_frame(**case)
    df = postfilter.DeviceFrame(f)
    postfilter.run_postfilter([df], mode=abi.MODE_PER_FRAME)
    torch.cuda.synchronize()
    refs, outs = oracle.postfilter_frame(f)
    _assert_planes("reference payload", df.download("lr"), refs)
    _assert_planes("output", df.download("out"), outs)


def test_mixed_batch_equals_single(lib):
    """One launch per stage over frames of mixed size / depth / format gives
    each frame's solo result (8- and 10-bit frames take CDEF's half-precision
    path and the 12-bit one its integer path, in the same launch)."""
    cases = [CASES[0], CASES[1], CASES[2], CASES[3], CASES[5], CASES[6], CASES[7], CASES[9]]
    frames = [synth.make_frame(**c) for c in cases]
    batch = [postfilter.DeviceFrame(f) for f in frames]
    launches = postfilter.run_postfilter(batch, mode=abi.MODE_BATCHED)
    solo = [postfilter.DeviceFrame(f) for f in frames]
    for d in solo:
        postfilter.run_postfilter([d], mode=abi.MODE_BATCHED)
    torch.cuda.synchronize()
    assert launches <= 7  # deblock prep + filter, cdef, superres, lr, grain template + blend
    for b, s in zip(batch, solo):
        for stage in ("deblocked", "cdef", "lr", "out"):
            _assert_planes(stage, b.download(stage), s.download(stage))


def test_per_frame_mode_equals_batched(lib):
    frames = [synth.make_frame(seed=40 + i, width=240, height=136, film_grain=(i % 2 == 0)) for i in range(4)]
    a = [postfilter.DeviceFrame(f) for f in frames]
    b = [postfilter.DeviceFrame(f) for f in frames]
    na = postfilter.run_postfilter(a, mode=abi.MODE_BATCHED)
    nb = postfilter.run_postfilter(b, mode=abi.MODE_PER_FRAME)
    torch.cuda.synchronize()
    assert nb > na
    for x, y in zip(a, b):
        _assert_planes("out", x.download("out"), y.download("out"))


def test_invalid_descriptor_is_typed_error(lib):
    f = synth.make_frame(seed=50, width=64, height=64)
    df = postfilter.DeviceFrame(f)
    f.hdr.mi_cols += 2  # inconsistent with FrameWidth
    with pytest.raises(abi.Av1gError) as e:
        postfilter.run_postfilter([df])
    assert e.value.status == abi.AV1G_EINVAL
    f.hdr.mi_cols -= 2
    f.hdr.bit_depth = 9
    with pytest.raises(abi.Av1gError):
        postfilter.run_postfilter([df])
