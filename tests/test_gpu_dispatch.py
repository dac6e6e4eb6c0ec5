"""The stream dispatcher over real serving engines (GPU).

Two engines stand for two GPUs (both on device 0 here: every GPU call of
this suite has one GPU, and the engines share nothing, so the placement and
decode logic is the same).  Streams of different shapes are placed by free
HBM budget, decoded through whichever engine took them, and every frame
must equal the oracle's decode; a stream that fits no engine is refused.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, engine, synth  # noqa: E402
from oxideav_av1_b200.dispatch import Dispatcher, required_slot_bytes  # noqa: E402

pytestmark = pytest.mark.gpu

STREAMS = [dict(seed=601, n_frames=3, width=176, height=144),
           dict(seed=602, n_frames=3, width=200, height=120, bit_depth=10, film_grain=True),
           dict(seed=603, n_frames=2, width=130, height=70, ssx=0, ssy=0),
           dict(seed=604, n_frames=3, width=256, height=128)]


def test_dispatcher_places_and_decodes_on_real_engines():
    frames = [synth.make_stream(**c) for c in STREAMS]
    seqs = [synth.stream_seq(f) for f in frames]
    # equal budgets: the first stream goes to engine 0 (ties go to the lower
    # index), the next to engine 1, which then has more room
    budget = 512 << 20
    assert all(required_slot_bytes(q) < budget // 8 for q in seqs)
    engines = [engine.Engine(device=0, budget_bytes=budget), engine.Engine(device=0, budget_bytes=budget)]
    d = Dispatcher(engines)
    try:
        placed = []
        for q in seqs:
            r = d.open_stream(q)
            assert r is not None
            placed.append(r)
        assert [i for i, _ in placed[:2]] == [0, 1]
        # each engine reserved exactly what the dispatcher's estimate says
        for k, e in enumerate(engines):
            mine = [required_slot_bytes(q) for (i, _), q in zip(placed, seqs) if i == k]
            assert e.stats().bytes_reserved == sum(mine)
        tickets = [[st.submit(fr) for fr in f] for (i, st), f in zip(placed, frames)]
        for (i, st), ts, f in zip(placed, tickets, frames):
            want = oracle.decode_stream(f)
            for t, w in zip(ts, want):
                assert engines[i].poll(t, 60.0) == abi.AV1G_OK
                status, planes, _ = st.fetch(t)
                assert status == abi.AV1G_OK
                for g, e in zip(planes, w):
                    assert np.array_equal(g.astype(np.int64), e)
        for _, st in placed:
            st.close()
        # a stream larger than both budgets fits nowhere
        huge = dict(seqs[0], max_width=16384, max_height=16384, bit_depth=10)
        assert d.open_stream(huge) is None
    finally:
        d.close()
