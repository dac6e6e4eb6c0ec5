"""Full inter reconstruction at 3840x2160 10-bit 4:2:0 through the engine.

The full-reconstruction configuration's shape: 128x128 superblocks, a 2 x 2
tile grid on the key frame (its intra wavefront runs the four tiles side by
side), inter frames with compound prediction (average, distance, wedge,
difference-weighted), OBMC, global and local warp, inter-intra, and film
grain; every frame through inter prediction, residuals, the intra
wavefront, deblock, CDEF, loop restoration, grain and the slot refresh.
Each output plane must equal the oracle's sequential decode sample for
sample.  A second stream at 1920x1080 4:4:4 10-bit with the same grid runs
in the same engine steps (two shapes batched together).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, engine, synth  # noqa: E402

pytestmark = pytest.mark.gpu


def _same(got, exp, tag):
    assert len(got) == len(exp)
    for k, (g, e) in enumerate(zip(got, exp)):
        if e is None:
            assert g is None, f"{tag} frame {k}: output for a frame not shown"
            continue
        for p, (gp, ep) in enumerate(zip(g, e)):
            diff = np.argwhere(gp.astype(np.int64) != ep)
            assert len(diff) == 0, f"{tag} frame {k} plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"


def test_uhd_10bit_stream_with_every_tool_matches_oracle():
    uhd = synth.make_stream(331, n_frames=3, width=3840, height=2160, bit_depth=10, film_grain=True, sb_size=128,
                            tiles=(1, 1))
    fhd = synth.make_stream(332, n_frames=3, width=1920, height=1080, bit_depth=10, ssx=0, ssy=0, sb_size=128,
                            tiles=(1, 1))
    preds = np.concatenate([f.preds for f in uhd[1:]])
    assert (preds["kind"] == abi.INTER_COMPOUND).any() and (preds["kind"] == abi.INTER_INTRA).any()
    assert (preds["motion_mode"] == 1).any() and (preds["warp"] >= 0).any()
    assert uhd[1].hdr.film_grain.apply_grain
    want_uhd, want_fhd = oracle.decode_stream(uhd), oracle.decode_stream(fhd)
    eng = engine.Engine(device=0)
    try:
        su = eng.open_stream(synth.stream_seq(uhd, 128))
        sf = eng.open_stream(synth.stream_seq(fhd, 128))
        assert su is not None and sf is not None
        tickets = []
        for a, b in zip(uhd, fhd):   # both streams' frames in flight together
            tickets.append((su.submit(a), sf.submit(b)))
        got_u, got_f = [], []
        for tu, tf in tickets:
            assert eng.poll(tu, 120.0) == abi.AV1G_OK and eng.poll(tf, 120.0) == abi.AV1G_OK
            st, planes, _ = su.fetch(tu)
            assert st == abi.AV1G_OK
            got_u.append(planes)
            st, planes, _ = sf.fetch(tf)
            assert st == abi.AV1G_OK
            got_f.append(planes)
        su.close()
        sf.close()
    finally:
        eng.close()
    _same(got_u, want_uhd, "3840x2160")
    _same(got_f, want_fhd, "1920x1080 4:4:4")
