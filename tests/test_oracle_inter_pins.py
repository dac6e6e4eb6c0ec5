"""Pins of the inter-prediction oracle against the reference's own unit tests.

Each case restates a known answer or property from the `#[cfg(test)]` module
of src/inter_pred.rs (test names cited), run through the oracle's exported
helpers or through a hand-built frame of predict_inter calls.
"""
import numpy as np
import pytest

import oracle
from oxideav_av1_b200 import abi, synth


def _ramp():
    return (np.arange(16)[:, None] * 16 + np.arange(16)[None, :]).astype(np.uint8)


def test_mv_scaling_identity_and_integer_shift():
    # motion_vector_scaling_identity_yields_unit_scale / _integer_mv_shifts_origin
    s = oracle.mv_scaling(0, 0, 0, 640, 360, 640, 360, 16, 8, 0, 0)
    assert s == ((16 << 10) + 32, (8 << 10) + 32, 1024, 1024)
    base = oracle.mv_scaling(0, 0, 0, 640, 360, 640, 360, 0, 0, 0, 0)
    sh = oracle.mv_scaling(0, 0, 0, 640, 360, 640, 360, 0, 0, 8, 0)
    assert sh[1] - base[1] == 1 << 10 and sh[0] == base[0]


@pytest.mark.parametrize("dims", [(0, 8, 8, 8), (8, 0, 8, 8), (8, 8, 0, 8), (8, 8, 8, 0)])
def test_mv_scaling_rejects_zero_extents(dims):
    # motion_vector_scaling_rejects_invalid_inputs
    assert oracle.mv_scaling(0, 0, 0, *dims, 0, 0, 0, 0) is None


def test_setup_shear_known_answers():
    one = 1 << 16
    # r192_setup_shear_identity_is_zero
    assert oracle.setup_shear([0, 0, one, 0, 0, one]) == (0, 0, 0, 0, 1)
    # r192_setup_shear_zero_diag_is_caller_bug
    assert oracle.setup_shear([0, 0, 0, 0, 0, one]) is None
    # r192_setup_shear_small_horizontal_shear
    assert oracle.setup_shear([0, 0, one + 64, 0, 0, one]) == (64, 0, 0, 0, 1)
    # r192_setup_shear_rejects_unstable_factorisation
    s = oracle.setup_shear([0, 0, one + 16384, 0, 0, one])
    assert s[0] == 16384 and s[4] == 0


def test_wedge_mask_range_sign_and_rejections():
    # r191_wedge_mask_block_8x8_values_within_0_64
    for idx in range(16):
        for sign in range(2):
            m = oracle.wedge_mask(3, idx, sign)
            assert m.max() <= 64
    # r191_wedge_mask_sign_flip_inverts (BLOCK_16X16, index 5)
    m0, m1 = oracle.wedge_mask(6, 5, 0), oracle.wedge_mask(6, 5, 1)
    assert np.all(m0.astype(int) + m1 == 64)
    # r191_wedge_mask_rejects_invalid_inputs
    assert oracle.wedge_mask(3, 16, 0) is None
    assert oracle.wedge_mask(3, 0, 2) is None
    assert oracle.wedge_mask(0, 0, 0) is None       # BLOCK_4X4 has no wedges
    assert oracle.wedge_mask(12, 0, 0) is None      # BLOCK_64X64 has no wedges


def test_half_sample_mv_matches_hand_built_reference():
    # r291_predict_inter_half_sample_mv_matches_hand_built_reference
    f = synth.custom_inter_frame(16, 16, [(16, 16, [_ramp()])], [dict(x=4, y=4, w=4, h=4, mv=[[0, 4], [0, 0]])])
    planes, rc = oracle.inter(f)
    assert rc == 0
    expected = [[69, 70, 71, 72], [85, 86, 87, 88], [101, 102, 103, 104], [117, 118, 119, 120]]
    assert planes[0][4:8, 4:8].tolist() == expected
    # the rest of CurrFrame is untouched (r292_reconstruct_inter_block_drives_modeinfo_through_predict_inter)
    mask = np.ones((16, 16), bool)
    mask[4:8, 4:8] = False
    assert np.all(planes[0][mask] == 0)


@pytest.mark.parametrize("bd", [8, 10, 12])
@pytest.mark.parametrize("filt", [0, 1, 2, 3])
def test_zero_mv_copies_reference(bd, filt):
    # block_inter_prediction_zero_mv_copies_reference
    rng = np.random.default_rng(bd * 10 + filt)
    ref = rng.integers(0, 1 << bd, size=(32, 32))
    f = synth.custom_inter_frame(32, 32, [(32, 32, [ref])],
                                 [dict(x=8, y=8, w=16, h=8, filter_x=filt, filter_y=filt)], bit_depth=bd)
    planes, rc = oracle.inter(f)
    assert rc == 0
    assert np.array_equal(planes[0][8:16, 8:24], ref[8:16, 8:24])


def test_negative_start_clamps_to_edge():
    # block_inter_prediction_clamps_at_negative_start: a constant reference
    # read far outside its left / top edges predicts the constant
    ref = np.full((8, 8), 42)
    f = synth.custom_inter_frame(8, 8, [(8, 8, [ref])], [dict(x=0, y=0, w=4, h=4, mv=[[-100, -300], [0, 0]])])
    planes, rc = oracle.inter(f)
    assert rc == 0 and np.all(planes[0][:4, :4] == 42)


def _two_const_refs(a, b, size=32):
    return [(size, size, [np.full((size, size), a)]), (size, size, [np.full((size, size), b)])]


def test_obmc_above_hand_computed():
    # r193_overlap_blending_above_hand_computed_8tap: curr 200, neighbour 40,
    # mask of length 8: row 0 -> 130, row 7 -> 200 (a 16-high block has an
    # 8-row overlap)
    f = synth.custom_inter_frame(
        32, 32, _two_const_refs(200, 40),
        [dict(x=0, y=16, w=16, h=16, motion_mode=1, ref=[0, 0], avail_u=1, plane_residual_ge_8x8=1,
              obmc_first=0, obmc_above=1, obmc_left=0, mi_width_log2=2, mi_height_log2=2, mi_row=4, mi_col=0)],
        neighbours=[dict(axis_pos4=0, ref=1, step4=4)])
    planes, rc = oracle.inter(f)
    assert rc == 0
    blk = planes[0][16:32, 0:16]
    assert np.all(blk[0] == 130) and np.all(blk[7:] == 200)
    assert np.all(np.diff(blk[:8, 0]) >= 0)


def test_obmc_neighbour_outside_the_edge_is_rejected():
    # r193_overlap_blending_rejects_caller_bugs / obmc_walk_axis axis range
    f = synth.custom_inter_frame(
        32, 32, _two_const_refs(200, 40),
        [dict(x=0, y=16, w=16, h=16, motion_mode=1, avail_u=1, plane_residual_ge_8x8=1, obmc_above=1,
              mi_width_log2=2, mi_height_log2=2, mi_row=4, mi_col=0)],
        neighbours=[dict(axis_pos4=5, ref=1, step4=4)])
    assert oracle.inter(f)[1] == 1


def test_difference_weight_mask_values():
    # r191_difference_weight_mask_equal_preds_yields_38 / _saturates_at_64:
    # constant predictions 16a and 16b (compound rounding at 8 bits) give
    # m = 38 + |a - b| / 16, blended as Round2(m*16a + (64-m)*16b, 10)
    for a, b, mt in [(200, 40, 0), (200, 40, 1), (90, 90, 0), (255, 0, 0)]:
        f = synth.custom_inter_frame(32, 32, _two_const_refs(a, b),
                                     [dict(x=0, y=0, w=16, h=16, kind=abi.INTER_COMPOUND, ref=[0, 1],
                                           compound_type=1, mask_type=mt, mi_size=6)])
        planes, rc = oracle.inter(f)
        assert rc == 0
        m = min(38 + abs(a - b) // 16, 64)
        if mt:
            m = 64 - m
        want = (m * 16 * a + (64 - m) * 16 * b + 512) >> 10
        assert np.all(planes[0][:16, :16] == want), (a, b, mt)


def test_compound_average_and_distance_blends():
    # r201_predict_inter_compound_average_matches_hand_blend /
    # r201_predict_inter_compound_distance_matches_hand_blend
    f = synth.custom_inter_frame(32, 32, _two_const_refs(100, 50),
                                 [dict(x=0, y=0, w=8, h=8, kind=abi.INTER_COMPOUND, ref=[0, 1], compound_type=2),
                                  dict(x=8, y=0, w=8, h=8, kind=abi.INTER_COMPOUND, ref=[0, 1], compound_type=4,
                                       fwd_weight=9, bck_weight=7)])
    planes, rc = oracle.inter(f)
    assert rc == 0
    assert np.all(planes[0][:8, :8] == 75)
    assert np.all(planes[0][:8, 8:16] == (9 * 1600 + 7 * 800 + 128) >> 8)


def test_interintra_dc_mask_is_even_split():
    # r191_intra_mode_variant_mask_dc_yields_32 through mask_blend_interintra
    f = synth.custom_inter_frame(32, 32, _two_const_refs(100, 0),
                                 [dict(x=0, y=0, w=16, h=16, kind=abi.INTER_INTRA, interintra_mode=0)], fill=31)
    planes, rc = oracle.inter(f)
    assert rc == 0 and np.all(planes[0][:16, :16] == (32 * 31 + 32 * 100 + 32) >> 6)


def test_identity_warp_on_constant_reference():
    # r192_block_warp_identity_on_constant_ref
    one = 1 << 16
    f = synth.custom_inter_frame(32, 32, [(32, 32, [np.full((32, 32), 77)])],
                                 [dict(x=8, y=8, w=16, h=16, motion_mode=2, warp=0)],
                                 warps=[dict(local_warp_params=[0, 0, one, 0, 0, one], local_valid=1)])
    planes, rc = oracle.inter(f)
    assert rc == 0 and np.all(planes[0][8:24, 8:24] == 77)


def test_caller_bugs_are_rejected():
    # r194_predict_inter_rejects_caller_bugs / r201_..._rejects_caller_bugs
    ref = [(16, 16, [_ramp()])]
    bad = [dict(x=0, y=0, w=0, h=4), dict(x=0, y=0, w=4, h=4, plane=3), dict(x=0, y=0, w=4, h=4, ref=[7, 0]),
           dict(x=0, y=0, w=8, h=8, kind=1, ref=[0, 0], compound_type=3),
           dict(x=0, y=0, w=8, h=8, kind=2, interintra_mode=4), dict(x=0, y=0, w=8, h=8, motion_mode=2),
           dict(x=0, y=0, w=4, h=4, filter_x=6), dict(x=16, y=0, w=4, h=4)]
    for c in bad:
        f = synth.custom_inter_frame(16, 16, ref, [c])
        assert oracle.inter(f)[1] == 1, c


def test_intrabc_pieces_equal_the_whole_block():
    # predict_intrabc_leaf_into_curr_frame predicts the whole block at unit
    # scale; transform-sized pieces at their own origins give the same samples
    rng = np.random.default_rng(0)
    pl = rng.integers(0, 1024, size=(64, 128))
    for mv in [(-56, -72), (-64, 8), (-120, -4)]:
        a = oracle.intrabc_predict(pl, 1, 1, 1, 64, 32, 40, 20, 16, 16, *mv, 10)
        b = np.block([[oracle.intrabc_predict(pl, 1, 1, 1, 64, 32, 40 + dx, 20 + dy, 8, 8, *mv, 10)
                       for dx in (0, 8)] for dy in (0, 8)])
        assert np.array_equal(a, b)


def test_intrabc_integer_mv_copies_and_rejects_out_of_range():
    rng = np.random.default_rng(1)
    pl = rng.integers(0, 256, size=(64, 64))
    got = oracle.intrabc_predict(pl, 0, 1, 1, 16, 16, 32, 32, 8, 8, -8 * 16, -8 * 24, 8)
    assert np.array_equal(got, pl[16:24, 8:16])
    assert oracle.intrabc_predict(pl, 0, 1, 1, 16, 16, 32, 32, 8, 8, 1 << 14, 0, 8) is None


def test_palette_prediction_and_index_check():
    # predict_palette: CurrFrame = palette[map]; an index >= PaletteSize is rejected
    f = synth.make_intra_frame(seed=5, width=64, height=64, palette=1.0, mono=True)
    planes, rc = oracle.intra_rc(f)
    assert rc == 0
    t = f.tus[0]
    assert t["mode"] == abi.INTRA_MODE_PALETTE
    f.palette_maps = f.palette_maps.copy()
    f.palette_maps[int(t["palette_map"])] = 9
    assert oracle.intra_rc(f)[1] == 1
