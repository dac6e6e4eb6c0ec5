"""The intra wavefront's bounded dependency waits report on the frame they hit.

Every wait of the persistent intra launch is bounded; when one runs out the
launch marks that frame, the frame's superblocks skip their remaining work
(still publishing their levels, so no other wait is left hanging) and the
host reports that frame as AV1G_EDEVICE — in av1g_run_intra's own return
value and, in the serving engine, on that frame's ticket only.  The test
hook av1g_test_intra_wait_fault shortens the bound to 1 ms and plans, into
the frames of a chosen width, a wait that nothing satisfies.  No GPU fault is
involved: the wait ends by its time bound and the kernel returns normally.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, engine, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu

ONE_MS = 1_000_000


@pytest.fixture
def hook():
    lib = abi.load()
    yield lib
    abi.check(lib.av1g_test_intra_wait_fault(0, 0))


def _same_as_oracle(f, d):
    exp = oracle.intra(f)
    for p, (g, e) in enumerate(zip(d.download(), exp)):
        assert np.array_equal(g.astype(np.int64), e), f"plane {p} differs from the oracle"


def test_run_intra_reports_the_timed_out_job_and_recovers(hook):
    lib = hook
    a = synth.make_intra_frame(seed=301, width=176, height=144)
    b = synth.make_intra_frame(seed=302, width=128, height=96)
    abi.check(lib.av1g_test_intra_wait_fault(ONE_MS, 176))
    da, db = postfilter.DeviceIntra(a), postfilter.DeviceIntra(b)
    with pytest.raises(abi.Av1gError) as ei:
        postfilter.run_intra([da, db])
    assert ei.value.status == abi.AV1G_EDEVICE
    assert b"job 0" in lib.av1g_last_error()
    torch.cuda.synchronize()
    _same_as_oracle(b, db)   # the other frame of the launch is complete
    # the next call on the same device succeeds, bit-exact
    abi.check(lib.av1g_test_intra_wait_fault(0, 0))
    da2 = postfilter.DeviceIntra(a)
    postfilter.run_intra([da2])
    torch.cuda.synchronize()
    _same_as_oracle(a, da2)


def test_engine_fails_only_the_timed_out_frame(hook):
    lib = hook
    frames_a = synth.make_stream(311, n_frames=2, width=176, height=144)
    frames_b = synth.make_stream(312, n_frames=2, width=128, height=96)
    want_b = oracle.decode_stream(frames_b)
    abi.check(lib.av1g_test_intra_wait_fault(ONE_MS, 176))
    eng = engine.Engine(device=0)
    try:
        sa = eng.open_stream(synth.stream_seq(frames_a))
        sb = eng.open_stream(synth.stream_seq(frames_b))
        ta = [sa.submit(fr) for fr in frames_a]
        tb = [sb.submit(fr) for fr in frames_b]
        results_a = [eng.poll(t, 60.0) for t in ta]
        results_b = [eng.poll(t, 60.0) for t in tb]
        # stream a's key frame has intra work and times out; stream b decodes bit-exact
        assert results_a[0] == abi.AV1G_EDEVICE
        assert results_b == [abi.AV1G_OK, abi.AV1G_OK]
        for t, w in zip(tb, want_b):
            st, planes, _ = sb.fetch(t)
            assert st == abi.AV1G_OK
            for g, e in zip(planes, w):
                assert np.array_equal(g.astype(np.int64), e)
        st, _, _ = sa.fetch(ta[0])
        assert st == abi.AV1G_EDEVICE
        assert b"dependency wait ran out of time" in lib.av1g_last_error()  # the failed frame's reason
        for t in ta[1:]:
            sa.fetch(t)
        sa.close()
        sb.close()
        # with the hook off the same device decodes stream a bit-exact
        abi.check(lib.av1g_test_intra_wait_fault(0, 0))
        sa = eng.open_stream(synth.stream_seq(frames_a))
        want_a = oracle.decode_stream(frames_a)
        for fr, w in zip(frames_a, want_a):
            t = sa.submit(fr)
            assert eng.poll(t, 60.0) == abi.AV1G_OK
            st, planes, _ = sa.fetch(t)
            for g, e in zip(planes, w):
                assert np.array_equal(g.astype(np.int64), e)
        sa.close()
    finally:
        eng.close()
