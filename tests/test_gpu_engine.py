"""The serving engine: streams of whole frames (prediction, residuals, intra
wavefront, post-filter chain, reference slots, show_existing_frame) decoded
byte-identical to the oracle's sequential decode, alone and batched with
other streams of other shapes; budget admission; reset; per-frame errors."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, engine, synth  # noqa: E402

pytestmark = pytest.mark.gpu

STREAMS = [
    dict(seed=201, n_frames=5, width=176, height=144, show_existing_at=(3,)),
    dict(seed=202, n_frames=4, width=200, height=120, bit_depth=10, film_grain=True, show_existing_at=(2,)),
    dict(seed=203, n_frames=4, width=130, height=70, ssx=0, ssy=0),
    dict(seed=204, n_frames=3, width=96, height=96, mono=True),
    dict(seed=205, n_frames=4, width=256, height=128, superres_denom=12),
]


def _decode(eng, frames, sb=64):
    st = eng.open_stream(synth.stream_seq(frames, sb))
    assert st is not None
    tickets = [st.submit(fr) for fr in frames]
    outs = []
    for t in tickets:
        assert eng.poll(t, 60.0) == abi.AV1G_OK
        status, planes, lat = st.fetch(t)
        assert status == abi.AV1G_OK
        outs.append(planes)
    st.close()
    return outs


def _same(got, exp, tag):
    assert len(got) == len(exp)
    for k, (g, e) in enumerate(zip(got, exp)):
        if e is None:
            assert g is None, f"{tag} frame {k}: output for a frame not shown"
            continue
        for p, (gp, ep) in enumerate(zip(g, e)):
            diff = np.argwhere(gp.astype(np.int64) != ep)
            assert len(diff) == 0, f"{tag} frame {k} plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"


@pytest.fixture(scope="module")
def eng():
    e = engine.Engine(device=0)
    yield e
    e.close()


@pytest.mark.parametrize("case", STREAMS, ids=[f"s{c['seed']}" for c in STREAMS])
def test_stream_alone_matches_oracle(eng, case):
    frames = synth.make_stream(**case)
    _same(_decode(eng, frames), oracle.decode_stream(frames), f"seed {case['seed']}")


def test_streams_mixed_equal_alone_and_oracle(eng):
    streams = [synth.make_stream(**c) for c in STREAMS]
    alone = [_decode(eng, fr) for fr in streams]
    before = eng.stats()
    handles = [eng.open_stream(synth.stream_seq(fr)) for fr in streams]
    tickets = [[] for _ in streams]
    # interleave submissions so steps batch frames of every stream
    for k in range(max(len(f) for f in streams)):
        for i, fr in enumerate(streams):
            if k < len(fr):
                tickets[i].append(handles[i].submit(fr[k]))
    for i, (h, ts) in enumerate(zip(handles, tickets)):
        outs = []
        for t in ts:
            assert eng.poll(t, 60.0) == abi.AV1G_OK
            status, planes, _ = h.fetch(t)
            assert status == abi.AV1G_OK
            outs.append(planes)
        h.close()
        _same(outs, alone[i], f"stream {i} mixed vs alone")
        _same(outs, oracle.decode_stream(streams[i]), f"stream {i} mixed vs oracle")
    s = eng.stats()
    # frames of several streams shared steps
    assert s.steps_done - before.steps_done < s.frames_done - before.frames_done


def test_budget_admission():
    frames = synth.make_stream(seed=210, n_frames=2)
    seq = synth.stream_seq(frames)
    # eight slots plus one payload of 176x144 8-bit 4:2:0 with 64-byte row
    # pitch: 9 * (192 * 144 + 2 * 128 * 72) = 414720 bytes
    e = engine.Engine(device=0, budget_bytes=600_000)
    try:
        a = e.open_stream(seq)
        assert a is not None
        assert e.open_stream(seq) is None          # a second stream's slots do not fit
        a.close()
        b = e.open_stream(seq)                     # admitted once the first leaves
        assert b is not None
        b.close()
    finally:
        e.close()


def test_reset_refs_and_bad_frame_fail_alone(eng):
    good = synth.make_stream(seed=211, n_frames=3)
    bad = synth.make_stream(seed=212, n_frames=3)
    bad[1].preds = bad[1].preds.copy()
    bad[1].preds["ref"][0, 0] = 9                  # not a reference index: EINVAL for that frame only
    hg, hb = eng.open_stream(synth.stream_seq(good)), eng.open_stream(synth.stream_seq(bad))
    tg = [hg.submit(f) for f in good]
    tb = [hb.submit(f) for f in bad]
    for t in tg:
        assert eng.poll(t, 60.0) == abi.AV1G_OK
    assert [eng.poll(t, 60.0) for t in tb] == [abi.AV1G_OK, abi.AV1G_EINVAL, abi.AV1G_OK]
    outs = [hg.fetch(t)[1] for t in tg]
    _same(outs, oracle.decode_stream(good), "good stream beside a failing one")
    # after a reset, showing a slot is an error
    hg.reset_refs()
    fr = synth.StreamFrame()
    fr.hdr, fr.show_existing, fr.show_idx = good[0].hdr, 1, 0
    t = hg.submit(fr)
    assert eng.poll(t, 60.0) == abi.AV1G_EINVAL
    hg.close()
    hb.close()
