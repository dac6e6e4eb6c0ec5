"""Inter-intra blocks decoded in two passes equal the reference's per-block order.

The reference predicts an inter-intra block by writing its intra prediction
into CurrFrame and then calling predict_inter, which blends its inter
prediction with it (inter_pred.rs:2230-2290, mask_blend_interintra at 3272),
then adds the residual.  A whole frame on the GPU runs the inter pass for
every block first and the intra wavefront after it, so an inter-intra block
leaves its clipped inter prediction in a side plane during the inter pass and
the intra pass blends it with the intra half.  This file checks, on the
oracle, that the two orders give identical frames.
"""
import copy

import numpy as np
import pytest

import oracle
from oxideav_av1_b200 import abi, synth


class _Obj:
    pass


def ii_case(seed, width=176, height=144, bit_depth=8, ssx=1, ssy=1, mono=False):
    f = synth.make_inter_frame(seed, width, height, bit_depth, ssx, ssy, mono, scaled=False, p_intra=0.0, p_ii=0.6)
    rec = synth.make_recon_frame(seed + 1, width, height, bit_depth, ssx, ssy, mono)
    tus, coeffs = synth.interintra_tus(f, seed + 2, quant=rec.quant)
    coeffs = np.concatenate(coeffs).astype(np.int32) if coeffs else np.zeros(1, np.int32)
    return f, rec.quant, tus, coeffs


def split_order(f, quant, tus, coeffs):
    """Inter pass (inter halves to side planes), then the intra pass."""
    side = [np.zeros(f.plane_dims(p), np.int32) for p in range(f.hdr.num_planes)]
    planes, rc = oracle.inter(f, side=side)
    assert rc == 0
    o = _Obj()
    o.hdr, o.quant, o.tus, o.coeffs, o.planes, o.interintra_side = f.hdr, quant, tus, coeffs, planes, side
    return oracle.intra(o)


def reference_order(f, quant, tus, coeffs):
    """Plain inter blocks, then each inter-intra call in decode order: its
    intra prediction into CurrFrame, predict_inter blending in place, its
    residual."""
    g = copy.copy(f)
    g.preds = f.preds[f.preds["kind"] != abi.INTER_INTRA]
    planes, rc = oracle.inter(g)
    assert rc == 0
    ii_calls = f.preds[f.preds["kind"] == abi.INTER_INTRA]
    k = 0
    for call in ii_calls:
        t = tus[k:k + 1].copy()
        if (int(t["x"][0]), int(t["y"][0]), int(t["plane"][0])) != (int(call["x"]), int(call["y"]), int(call["plane"])):
            continue  # a call without a transform size of its own shape gets no TU
        t["interintra"] = 0                    # the intra half alone, written to CurrFrame
        o = _Obj()
        o.hdr, o.quant, o.tus, o.coeffs, o.planes = f.hdr, quant, t, coeffs, planes
        planes = oracle.intra(o)
        g.preds = call.reshape(1)
        g.planes = planes
        planes, rc = oracle.inter(g)           # predict_inter's in-place blend
        assert rc == 0
        k += 1
        if k < len(tus) and tus[k]["mode"] == abi.INTRA_MODE_NONE:
            o.tus, o.planes = tus[k:k + 1], planes
            planes = oracle.intra(o)
            k += 1
    return planes


CASES = [dict(seed=301), dict(seed=302, bit_depth=10), dict(seed=303, ssx=0, ssy=0), dict(seed=304, mono=True),
         dict(seed=305, width=200, height=120, bit_depth=12)]


@pytest.mark.parametrize("case", CASES, ids=[f"s{c['seed']}" for c in CASES])
def test_split_passes_equal_reference_order(case):
    f, quant, tus, coeffs = ii_case(**case)
    assert (f.preds["kind"] == abi.INTER_INTRA).sum() > 0 and (tus["interintra"] == 2).sum() > 0
    a = reference_order(f, quant, tus, coeffs)
    b = split_order(f, quant, tus, coeffs)
    for p, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"plane {p} differs"


def test_intra_half_rejects_inconsistent_mode():
    f, quant, tus, coeffs = ii_case(306)
    tus = tus.copy()
    k = int(np.argmax(tus["interintra"] > 0))
    tus["mode"][k] = 5   # not the intra mode of its inter-intra mode
    side = [np.zeros(f.plane_dims(p), np.int32) for p in range(f.hdr.num_planes)]
    o = _Obj()
    o.hdr, o.quant, o.tus, o.coeffs, o.planes, o.interintra_side = f.hdr, quant, tus, coeffs, f.planes, side
    assert oracle.intra_rc(o)[1] == k + 1
