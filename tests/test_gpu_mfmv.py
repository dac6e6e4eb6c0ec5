"""Motion-field storage and projection on the device against the oracle, bit-exact.

av1g_run_mf_store (§7.19, src/decoder/frame_driver.rs:1119-1160) and
av1g_run_mf_project (§7.9 motion_field_estimation_core,
src/inter_pred.rs:7592-7742) are called through the C ABI on batches that mix
frame sizes (1080p, odd mi extents, a 1x1 frame, an empty frame), order-hint
widths (0, 3, 7, 8 bits), empty / intra / mismatched reference slots, and
dense stored fields where many cells land on one position, so the
last-writer order of the reference decides the result.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, mfmv, synth  # noqa: E402

pytestmark = pytest.mark.gpu

STORE_CASES = [(270, 480, 7, True), (7, 9, 4, True), (1, 1, 8, True), (36, 64, 0, True), (36, 64, 7, False),
               (0, 12, 7, True), (33, 17, 3, True)]


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _dev_slots(slots):
    out = []
    for sl in slots:
        if sl is None:
            out.append(None)
            continue
        d = dict(sl)
        d["mf_mvs"], d["mf_ref_frames"] = _dev(sl["mf_mvs"]), _dev(sl["mf_ref_frames"])
        out.append(d)
    return out


def _oracle_project(sc):
    return oracle.mf_project(sc["slots"], sc["ref_frame_idx"], sc["order_hints"], sc["order_hint"],
                             sc["hint_bits"], sc["mi_rows"], sc["mi_cols"])


def test_store_matches_oracle():
    jobs, outs, want, keep = [], [], [], []
    for seed, (rows, cols, bits, inter) in enumerate(STORE_CASES):
        s = synth.make_mf_store_inputs(10 + seed, rows, cols, bits, inter)
        ins = (_dev(s["ref_frames"]), _dev(s["mvs"]))  # alive until the batch has run
        keep.append(ins)
        j, r, m = mfmv.store_job(rows, cols, inter, s["order_hint"], bits, s["ref_order_hint"], *ins)
        r.fill_(99)
        m.fill_(1234)
        jobs.append(j)
        outs.append((r, m))
        want.append(oracle.mf_store(rows, cols, inter, s["order_hint"], bits, s["ref_order_hint"], s["ref_frames"],
                                    s["mvs"]))
    mfmv.run_store(jobs)
    torch.cuda.synchronize()
    kept = 0
    for k, ((r, m), (wr, wm)) in enumerate(zip(outs, want)):
        assert np.array_equal(r.cpu().numpy(), wr), f"case {k}: mf_ref_frames differ"
        assert np.array_equal(m.cpu().numpy(), wm), f"case {k}: mf_mvs differ"
        kept += int((wr > 0).sum())
    assert kept > 0


SCENES = [dict(seed=1, mi_rows=270, mi_cols=480), dict(seed=2, mi_rows=68, mi_cols=120, empty=(0, 4)),
          dict(seed=3, mi_rows=68, mi_cols=120, intra=(1, 2, 3)), dict(seed=4, mi_rows=45, mi_cols=80,
                                                                        mismatched=(0, 5, 7)),
          dict(seed=5, mi_rows=45, mi_cols=81, hint_bits=3), dict(seed=6, mi_rows=40, mi_cols=40, hint_bits=0),
          dict(seed=7, mi_rows=135, mi_cols=240, fill=1.0), dict(seed=8, mi_rows=3, mi_cols=5, hint_bits=8),
          dict(seed=9, mi_rows=1, mi_cols=30), dict(seed=10, mi_rows=33, mi_cols=47, empty=tuple(range(8)))]


def _scene(kw):
    kw = dict(kw)
    return synth.make_mf_scene(kw.pop("seed"), kw.pop("mi_rows"), kw.pop("mi_cols"), **kw)


def test_project_matches_oracle():
    scenes = [_scene(kw) for kw in SCENES]
    jobs, outs, keep = [], [], []
    for sc in scenes:
        slots = _dev_slots(sc["slots"])
        keep.append(slots)
        j, out = mfmv.project_job(slots, sc["ref_frame_idx"], sc["order_hints"], sc["order_hint"], sc["hint_bits"],
                                  sc["mi_rows"], sc["mi_cols"])
        out.fill_(77)  # every entry must be written
        jobs.append(j)
        outs.append(out)
    mfmv.run_project(jobs)
    torch.cuda.synchronize()
    projected = 0
    for k, (sc, out) in enumerate(zip(scenes, outs)):
        want = _oracle_project(sc)
        got = out.cpu().numpy()
        diff = np.argwhere(got != want)
        assert len(diff) == 0, f"scene {k}: {len(diff)} entries differ, first {tuple(diff[0])}"
        projected += int((want != abi.MFMV_INVALID).sum())
    assert projected > 0


def test_projection_is_repeatable():
    sc = _scene(dict(seed=11, mi_rows=135, mi_cols=240, fill=1.0))
    slots = _dev_slots(sc["slots"])
    first = mfmv.motion_field_estimation(slots, sc["ref_frame_idx"], sc["order_hints"], sc["order_hint"],
                                         sc["hint_bits"], sc["mi_rows"], sc["mi_cols"])
    for _ in range(3):
        again = mfmv.motion_field_estimation(slots, sc["ref_frame_idx"], sc["order_hints"], sc["order_hint"],
                                             sc["hint_bits"], sc["mi_rows"], sc["mi_cols"])
        assert torch.equal(first, again)
    assert np.array_equal(first.cpu().numpy(), _oracle_project(sc))


def test_store_then_project_on_device():
    """Four decoded 1080p frames store their fields on the device; the next
    frame projects from those device-resident slots."""
    rows, cols, bits = 270, 480, 7
    slots_dev, slots_host = [None] * 8, [None] * 8
    hints = [10, 12, 14, 18]
    for k, h in enumerate(hints):
        s = synth.make_mf_store_inputs(40 + k, rows, cols, bits, True)
        s["order_hint"] = h
        s["ref_order_hint"] = [(h - d) % 128 for d in (1, 2, 3, 4, 6, 8, 2)]
        r, m = mfmv.motion_vector_storage(rows, cols, True, h, bits, s["ref_order_hint"], _dev(s["ref_frames"]),
                                          _dev(s["mvs"]))
        wr, wm = oracle.mf_store(rows, cols, True, h, bits, s["ref_order_hint"], s["ref_frames"], s["mvs"])
        saved = [h] + list(s["ref_order_hint"])
        common = dict(saved_order_hints=saved, mi_rows=rows, mi_cols=cols, frame_is_intra=False)
        slots_dev[k] = dict(mf_mvs=m, mf_ref_frames=r, **common)
        slots_host[k] = dict(mf_mvs=wm, mf_ref_frames=wr, **common)
    ref_frame_idx = [2, 1, 0, 0, 3, 3, 3]
    cur = 16
    order_hints = [0] + [hints[i] for i in ref_frame_idx]
    got = mfmv.motion_field_estimation(slots_dev, ref_frame_idx, order_hints, cur, bits, rows, cols)
    want = oracle.mf_project(slots_host, ref_frame_idx, order_hints, cur, bits, rows, cols)
    torch.cuda.synchronize()
    assert np.array_equal(got.cpu().numpy(), want)
    assert (want != abi.MFMV_INVALID).any()
