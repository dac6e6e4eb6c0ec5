"""Motion-field oracle pins and host-side checks (no GPU).

The C oracle (oracle/mfmv.c) is pinned to the reference's own unit tests of
the pieces it restates:
  get_relative_dist_sign_extends            src/frame_header.rs:3271-3280
  get_mv_projection_identity / _clamps      src/cdf.rs:55252-55275
  get_block_position_valid / _invalid       src/cdf.rs:55278-55297
  motion_field_mvs_new_invalid_sizes        src/cdf.rs:55200-55211
and cross-checked against a direct pure-Python statement of §7.19 and of
motion_field_estimation_core (src/inter_pred.rs:7592-7742) on small seeded
scenes, including ones where several cells land on one position (the last
writer in the reference's order must win).  The C ABI's argument checks run
without a device: every malformed descriptor is rejected before any CUDA
call.
"""
import ctypes as C

import numpy as np

import oracle
from oxideav_av1_b200 import abi, synth

DIV_MULT = [0, 16384, 8192, 5461, 4096, 3276, 2730, 2340, 2048, 1820, 1638, 1489, 1365, 1260, 1170, 1092, 1024,
            963, 910, 862, 819, 780, 744, 712, 682, 655, 630, 606, 585, 564, 546, 528]


def test_relative_dist_pins():
    assert oracle.relative_dist(2, 1, 7) == 1
    assert oracle.relative_dist(1, 2, 7) == -1
    assert oracle.relative_dist(0, 127, 7) == 1
    assert oracle.relative_dist(50, 1, 0) == 0


def test_mv_projection_pins():
    assert oracle.mv_projection([100, -100], 4, 4) == [100, -100]
    assert oracle.mv_projection([42, 17], 1, 1) == [42, 17]
    assert oracle.mv_projection([30000, -30000], 8, 1) == [16383, -16383]


def test_block_position_pins():
    assert oracle.block_position(4, 4, 1, [0, 0], 16, 16) == (4, 4)
    assert oracle.block_position(4, 7, 1, [16384, 0], 16, 16) is None


def test_new_invalid_sizing():
    out = oracle.mf_project([None] * 8, [0] * 7, [0] * 8, 0, 7, 16, 8)
    assert out.shape == (7, 8, 4, 2)
    assert (out == abi.MFMV_INVALID).all()


# --- direct statement of the reference, pure Python (small cases only) ---

def _rd(a, b, bits):
    if bits == 0:
        return 0
    d, m = a - b, 1 << (bits - 1)
    return (d & (m - 1)) - (d & m)


def _proj(mv, num, den):
    den = min(den, 31)
    num = max(-31, min(31, num))
    out = []
    for v in mv:
        v = v * num * DIV_MULT[den]
        s = (v + 8192) >> 14 if v >= 0 else -((-v + 8192) >> 14)
        out.append(max(-16383, min(16383, s)))
    return out


def _py_store(s):
    cells = s["mi_rows"] * s["mi_cols"]
    r_out = np.full(cells, -1, np.int8)
    m_out = np.zeros((cells, 2), np.int16)
    if s["is_inter"]:
        for c in range(cells):
            for lst in range(2):
                r = int(s["ref_frames"][c, lst])
                if 0 < r <= 7 and _rd(s["ref_order_hint"][r - 1], s["order_hint"], s["hint_bits"]) < 0:
                    mr, mc = (int(v) for v in s["mvs"][c, lst])
                    if abs(mr) <= 4095 and abs(mc) <= 4095:
                        r_out[c], m_out[c] = r, (mr, mc)
    return r_out, m_out


def _py_project(sc):
    mi_rows, mi_cols, bits = sc["mi_rows"], sc["mi_cols"], sc["hint_bits"]
    oh, cur = sc["order_hints"], sc["order_hint"]
    h8, w8 = mi_rows >> 1, mi_cols >> 1
    out = np.full((7, h8, w8, 2), abi.MFMV_INVALID, np.int16)
    writes = [0]

    def project_ref(src, sign):
        sl = sc["slots"][sc["ref_frame_idx"][src - 1]]
        if sl is None or sl["mi_rows"] != mi_rows or sl["mi_cols"] != mi_cols or sl["frame_is_intra"]:
            return False
        for y8 in range(h8):
            for x8 in range(w8):
                cell = (2 * y8 + 1) * mi_cols + 2 * x8 + 1
                sref = int(sl["mf_ref_frames"][cell])
                if sref <= 0:
                    continue
                to_cur = _rd(oh[src], cur, bits)
                off = _rd(oh[src], sl["saved_order_hints"][sref], bits)
                if not (abs(to_cur) <= 31 and abs(off) <= 31 and off > 0):
                    continue
                mv = [int(v) for v in sl["mf_mvs"][cell]]
                p = _proj(mv, to_cur * sign, off)
                pos = []
                for v8, d, mx, mo in ((y8, p[0], h8, 0), (x8, p[1], w8, 8)):
                    base = (v8 >> 3) << 3
                    o8 = d >> 6 if d >= 0 else -((-d) >> 6)
                    v = v8 + sign * o8
                    pos.append(v if 0 <= v < mx and base - mo <= v < base + 8 + mo else None)
                if None in pos:
                    continue
                writes[0] += 1
                for dst in range(1, 8):
                    out[dst - 1, pos[0], pos[1]] = _proj(mv, _rd(cur, oh[dst], bits), off)
        return True

    last = sc["slots"][sc["ref_frame_idx"][0]]
    if (last["saved_order_hints"][7] if last is not None else 0) != oh[4]:
        project_ref(1, -1)
    stamp = 1
    if _rd(oh[5], cur, bits) > 0 and project_ref(5, 1):
        stamp -= 1
    if _rd(oh[6], cur, bits) > 0 and project_ref(6, 1):
        stamp -= 1
    if _rd(oh[7], cur, bits) > 0 and stamp >= 0 and project_ref(7, 1):
        stamp -= 1
    if stamp >= 0:
        project_ref(2, -1)
    return out, writes[0]


def _ora_project(sc):
    return oracle.mf_project(sc["slots"], sc["ref_frame_idx"], sc["order_hints"], sc["order_hint"],
                             sc["hint_bits"], sc["mi_rows"], sc["mi_cols"])


def test_store_matches_direct_statement():
    for seed, (rows, cols, bits, inter) in enumerate([(12, 20, 7, True), (7, 9, 4, True), (10, 10, 0, True),
                                                      (6, 8, 7, False), (1, 1, 8, True)]):
        s = synth.make_mf_store_inputs(100 + seed, rows, cols, bits, inter)
        got = oracle.mf_store(rows, cols, inter, s["order_hint"], bits, s["ref_order_hint"], s["ref_frames"],
                              s["mvs"])
        want = _py_store(s)
        assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1]), seed


def test_project_matches_direct_statement_with_collisions():
    total_writes = 0
    cases = [dict(), dict(empty=(1, 3)), dict(intra=(0, 2, 5)), dict(mismatched=(4, 6)), dict(hint_bits=3),
             dict(hint_bits=0), dict(fill=1.0)]
    for seed, kw in enumerate(cases):
        for rows, cols in ((24, 40), (17, 23)):
            sc = synth.make_mf_scene(200 + seed, rows, cols, **kw)
            want, writes = _py_project(sc)
            total_writes += writes
            got = _ora_project(sc)
            assert np.array_equal(got, want), (seed, kw, rows, cols)
    sc = synth.make_mf_scene(300, 24, 40, fill=1.0)
    want, writes = _py_project(sc)
    written = int((want[0, :, :, 0] != abi.MFMV_INVALID).sum())
    assert writes > written > 0, "the scene must have positions that several cells reach"
    assert total_writes > 0


def _store_job(**kw):
    j = abi.MfStoreJob(4, 4, 1, 0, 7, (C.c_int32 * 7)(), 16, 16, 16, 16)
    for k, v in kw.items():
        setattr(j, k, v)
    return j


def test_store_rejects_bad_descriptors_without_a_device():
    lib = abi.load()
    for kw in (dict(mi_rows=-1), dict(hint_bits=9), dict(mf_mvs=None), dict(mf_mvs=18), dict(mvs=20),
               dict(ref_frames=17), dict(ref_frames=None)):
        arr = (abi.MfStoreJob * 1)(_store_job(**kw))
        assert lib.av1g_run_mf_store(arr, 1, None) == abi.AV1G_EINVAL, kw
    assert lib.av1g_run_mf_store(None, 1, None) == abi.AV1G_EINVAL
    assert lib.av1g_run_mf_store(None, 0, None) == abi.AV1G_OK


def test_project_rejects_bad_descriptors_without_a_device():
    lib = abi.load()

    def job(**kw):
        j = abi.MfProjectJob()
        j.mi_rows, j.mi_cols, j.hint_bits, j.out = 8, 8, 7, 64
        for k, v in kw.items():
            setattr(j, k, v)
        return j

    bad_idx = job()
    bad_idx.ref_frame_idx[3] = 8
    slot_unaligned = job()
    slot_unaligned.slots[2] = abi.MfSlot(66, 64, (C.c_int32 * 8)(), 8, 8, 0, 0)
    for j in (job(hint_bits=-1), job(hint_bits=9), job(mi_cols=-2), job(out=None), job(out=66), bad_idx,
              slot_unaligned):
        arr = (abi.MfProjectJob * 1)(j)
        assert lib.av1g_run_mf_project(arr, 1, None) == abi.AV1G_EINVAL
    # a frame without a whole 8x8 position has nothing to write and needs no output array
    fine_but_empty = job(mi_rows=1, mi_cols=1, out=None)
    assert lib.av1g_run_mf_project((abi.MfProjectJob * 1)(fine_but_empty), 1, None) == abi.AV1G_OK
