"""No kernel writes outside its planes (GPU, guard zones).

Every device plane these tests create is carved out of a larger buffer: the
bytes before and after the plane, and each row's padding past its last
sample, hold 0xA5.  After every call they must still hold 0xA5, and the
stage outputs must equal the oracle's.  The guard bytes lie inside the
allocation, so a stray write changes them instead of faulting the GPU; this
stands in for a bounds-checked device build (compute-sanitizer is closed on
this pool).  It covers the writes of every pixel kernel that takes caller
planes: the post-filter chain (deblock, CDEF, superres, loop restoration,
film grain), the inter-block residual pass, the intra wavefront and its
residual pre-pass, and inter prediction (with the inter-intra side planes).
Collected late (zz) so a stop at the first failure has run the rest.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

GUARD = 4096
PATTERN = 0xA5


@pytest.fixture
def guarded(monkeypatch):
    """Every DevPlane built while the fixture is active sits inside a guard
    buffer; yields the list of (plane, buffer) pairs to check."""
    made = []
    orig_init = postfilter.DevPlane.__init__

    def init(self, height, width, hbd, device, fill=None):
        orig_init(self, height, width, hbd, device, fill=None)
        rows, pitch = self.t.shape
        buf = torch.full((2 * GUARD + rows * pitch,), PATTERN, dtype=torch.uint8, device=self.t.device)
        t = buf[GUARD:GUARD + rows * pitch].view(rows, pitch)
        t[:, : self.w * self.bps].zero_()
        self.t = t
        if fill is not None:
            self.upload(fill)
        made.append((self, buf))

    monkeypatch.setattr(postfilter.DevPlane, "__init__", init)
    yield made


def _intact(made):
    torch.cuda.synchronize()
    bad = []
    for pl, buf in made:
        head, tail = buf[:GUARD], buf[-GUARD:]
        pad = pl.t[:, pl.w * pl.bps:]
        for what, part in (("before", head), ("after", tail), ("row padding", pad)):
            if part.numel() and not bool((part == PATTERN).all()):
                bad.append(f"{pl.h}x{pl.w} plane: bytes {what} it changed")
    return bad


def _same(got, want, tag):
    for p, (g, e) in enumerate(zip(got, want)):
        d = np.argwhere(g.astype(np.int64) != e)
        assert len(d) == 0, f"{tag} plane {p}: {len(d)} samples differ, first {tuple(d[0])}"


POSTFILTER = [
    dict(seed=501, width=178, height=146, bit_depth=10, film_grain=True, superres_denom=10),
    dict(seed=502, width=130, height=70, ssx=0, ssy=0, film_grain=True),
    dict(seed=503, width=98, height=66, mono=True, film_grain=True),
    dict(seed=504, width=322, height=182, bit_depth=12, ssx=1, ssy=0, film_grain=True),
    dict(seed=505, width=210, height=100, lr_unit=64, lr_uv_shift=1, lr_none_frac=0.2, superres_denom=13),
]


def test_postfilter_chain_stays_inside_its_planes(guarded):
    frames = [synth.make_frame(**c) for c in POSTFILTER]
    dfs = [postfilter.DeviceFrame(f) for f in frames]
    postfilter.run_postfilter(dfs)
    assert _intact(guarded) == []
    for f, d in zip(frames, dfs):
        refs, outs = oracle.postfilter_frame(f)
        _same(d.download("lr"), refs, "reference payload")
        _same(d.download("out"), outs, "output")


@pytest.mark.parametrize("case", [dict(seed=511, width=200, height=120, bit_depth=10),
                                  dict(seed=512, width=130, height=70, ssx=0, ssy=0),
                                  dict(seed=513, width=98, height=66, mono=True)])
def test_residual_pass_stays_inside_its_planes(guarded, case):
    f = synth.make_recon_frame(**case)
    d = postfilter.DeviceRecon(f)
    postfilter.run_recon([d])
    assert _intact(guarded) == []
    _same(d.download(), oracle.recon(f), "recon")


@pytest.mark.parametrize("case", [dict(seed=521, width=178, height=146, palette=0.2, intrabc=0.1),
                                  dict(seed=522, width=264, height=136, bit_depth=10, sb_size=128, palette=0.1),
                                  dict(seed=523, width=200, height=120, ssx=0, ssy=0, tiles=(1, 1)),
                                  dict(seed=524, width=98, height=66, mono=True)])
def test_intra_wavefront_stays_inside_its_planes(guarded, case):
    f = synth.make_intra_frame(**case)
    d = postfilter.DeviceIntra(f)
    postfilter.run_intra([d])
    assert _intact(guarded) == []
    _same(d.download(), oracle.intra(f), "intra")


@pytest.mark.parametrize("case", [dict(seed=531, width=176, height=144),
                                  dict(seed=532, width=200, height=120, bit_depth=12),
                                  dict(seed=533, width=130, height=70, ssx=0, ssy=0),
                                  dict(seed=534, width=96, height=96, mono=True)])
def test_inter_prediction_stays_inside_its_planes(guarded, case):
    f = synth.make_inter_frame(**case)
    d = postfilter.DeviceInter(f)
    postfilter.run_inter([d])
    assert _intact(guarded) == []
    exp, rc = oracle.inter(f)
    assert rc == 0
    _same(d.download(), exp, "inter")


def test_guard_check_sees_a_stray_write(guarded):
    """The check itself: a byte written past a plane's last row is reported."""
    pl = postfilter.DevPlane(8, 10, False, "cuda")
    assert _intact(guarded) == []
    _, buf = guarded[-1]
    buf[-1] = 0
    assert _intact(guarded) == ["8x10 plane: bytes after it changed"]


def test_two_pass_inter_intra_stays_inside_its_planes(guarded):
    """Inter pass into CurrFrame and the side planes, then the intra wavefront
    blending the side planes (tests/test_oracle_interintra_split.py's split)."""
    from test_oracle_interintra_split import ii_case, split_order
    f, quant, tus, coeffs = ii_case(seed=541, width=176, height=144)
    want = split_order(f, quant, tus, coeffs)
    d = postfilter.DeviceInter(f, side=True)
    postfilter.run_inter([d])
    it = synth.IntraFrame()
    it.hdr, it.quant, it.tus, it.coeffs, it.planes = f.hdr, quant, tus, coeffs, f.planes
    di = postfilter.DeviceIntra(it)
    di.planes, di.side = d.planes, d.side
    postfilter.run_intra([di])
    assert _intact(guarded) == []
    _same(di.download(), want, "inter-intra")
