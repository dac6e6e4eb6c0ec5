"""Pin the CPU oracle to the reference's own module unit tests.

Each test restates an assertion of the reference crate's `#[cfg(test)]`
modules (src/loop_filter.rs, src/cdef.rs, src/superres.rs,
src/loop_restoration.rs, src/film_grain.rs) against the oracle's C
restatement, so the oracle the CUDA kernels are compared with is itself checked
against the reference's known answers.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from oxideav_av1_b200 import abi, synth


@pytest.fixture(scope="module")
def lib():
    return oracle.load()


def _plane(a):
    a = np.ascontiguousarray(a, dtype=np.int32)
    return oracle.OraPlane(a.ctypes.data_as(C.POINTER(C.c_int32)), a.shape[0], a.shape[1]), a


def _uniform_grid(mi_rows, mi_cols, **vals):
    g = {k: np.full((mi_rows, mi_cols), v, dt) for k, (v, dt) in dict(
        mi_size=(0, np.uint8), skip=(0, np.uint8), is_inter=(0, np.uint8), ref_frame0=(0, np.int8),
        y_mode=(0, np.uint8), segment_id=(0, np.int8), tx_size=(0, np.uint8), inter_tx_size=(0, np.uint8)).items()}
    g["delta_lf"] = np.zeros((mi_rows, mi_cols, 4), np.int8)
    for k, v in vals.items():
        g[k][...] = v
    s = abi.MiGrid()
    for k, a in g.items():
        setattr(s, k, a.ctypes.data)
    return s, g


def _hdr(mi_rows=4, mi_cols=4, levels=(0, 0, 0, 0), bd=8):
    h = abi.FrameHeader()
    h.mi_rows, h.mi_cols = mi_rows, mi_cols
    h.frame_width, h.frame_height, h.upscaled_width = mi_cols * 4, mi_rows * 4, mi_cols * 4
    h.num_planes, h.bit_depth, h.subsampling_x, h.subsampling_y = 3, bd, 1, 1
    for i, v in enumerate(levels):
        h.lf_level[i] = v
    return h


def _strength(lib, h, grid, row=0, col=0, plane=0, passno=0):
    out = (C.c_int32 * 4)()
    lib.ora_lf_strength(C.byref(h), C.byref(grid), row, col, plane, passno, out)
    return list(out)


# --- loop_filter.rs tests -------------------------------------------------------

def test_strength_zero_level(lib):
    g, keep = _uniform_grid(4, 4)
    assert _strength(lib, _hdr(), g)[0] == 0


def test_strength_basic_table_lvl_32_sharp_0(lib):
    g, keep = _uniform_grid(4, 4)
    assert _strength(lib, _hdr(levels=(32, 32, 32, 32)), g) == [32, 32, 100, 2]


def test_strength_intra_ref_delta_lifts_lvl(lib):
    g, keep = _uniform_grid(4, 4)
    h = _hdr(levels=(10, 10, 10, 10))
    h.lf_delta_enabled = 1
    h.lf_ref_deltas[0] = 5
    assert _strength(lib, h, g)[0] == 15


def test_strength_clipped_at_max_loop_filter(lib):
    g, keep = _uniform_grid(4, 4)
    h = _hdr(levels=(60, 60, 60, 60))
    h.lf_delta_enabled = 1
    h.lf_ref_deltas[0] = 40
    assert _strength(lib, h, g)[0] == 63


def test_filter_size_caps(lib):
    TX_64X64, TX_32X32, TX_4X4 = 4, 3, 0
    assert lib.ora_lf_filter_size(TX_64X64, TX_64X64, 0, 0) == 16
    assert lib.ora_lf_filter_size(TX_32X32, TX_32X32, 0, 1) == 8
    assert lib.ora_lf_filter_size(TX_4X4, TX_4X4, 0, 0) == 4


def test_narrow_filter_idempotent_and_softens_step(lib):
    p, a = _plane(np.full((8, 8), 100))
    lib.ora_lf_narrow(C.byref(p), 4, 0, 1, 0, 0, 8)
    assert (a == 100).all()
    step = np.tile(np.array([100, 100, 100, 100, 156, 156, 156, 156]), (8, 1))
    p, a = _plane(step)
    lib.ora_lf_narrow(C.byref(p), 4, 0, 1, 0, 0, 8)
    p0, q0 = a[0, 3], a[0, 4]
    assert p0 > 100 and q0 < 156 and q0 - 128 == 128 - p0


@pytest.mark.parametrize("log2", [3, 4])
def test_wide_filter_preserves_uniform(lib, log2):
    p, a = _plane(np.full((32, 32), 77))
    lib.ora_lf_wide(C.byref(p), 16, 4, 0, 1, 0, log2)
    assert (a == 77).all()


# --- cdef.rs tests ---------------------------------------------------------------

def test_constrain(lib):
    assert lib.ora_cdef_constrain(5, 0, 3) == 0
    assert lib.ora_cdef_constrain(-7, 0, 3) == 0
    assert lib.ora_cdef_constrain(5, 16, 8) == 5
    assert lib.ora_cdef_constrain(-5, 16, 8) == -5
    assert lib.ora_cdef_constrain(20, 8, 4) == 0


def _direction(lib, img):
    h = _hdr()
    p, a = _plane(img)
    out = (C.c_int32 * 2)()
    lib.ora_cdef_direction(C.byref(h), C.byref(p), 0, 0, out)
    return list(out)


def test_direction_uniform_block(lib):
    assert _direction(lib, np.full((16, 16), 100)) == [0, 0]


def test_direction_horizontal_stripes_is_2(lib):
    img = 128 + 10 * np.arange(16)[:, None] * np.ones((1, 16), int)
    assert _direction(lib, img)[0] == 2


def test_direction_vertical_stripes_is_6(lib):
    img = 128 + 10 * np.arange(16)[None, :] * np.ones((16, 1), int)
    assert _direction(lib, img)[0] == 6


# --- loop_restoration.rs tests ---------------------------------------------------

def test_count_units_in_frame(lib):
    assert lib.ora_lr_count_units(64, 256) == 4
    assert lib.ora_lr_count_units(64, 100) == 2
    assert lib.ora_lr_count_units(64, 0) == 1
    assert lib.ora_lr_count_units(256, 240) == 1


def test_block_geometry_luma_top_left(lib):
    h = _hdr(16, 16)
    h.lr_unit_size[0] = 64
    out = (C.c_int32 * 10)()
    lib.ora_lr_geometry(C.byref(h), 0, 0, 0, out)
    unit_row, unit_col, x, y, w, hh, ss, se, pex, pey = list(out)
    assert (unit_row, unit_col, x, y, w, hh) == (0, 0, 0, 0, 4, 4)
    assert (pex, pey, ss, se) == (63, 63, -8, 55)


def test_source_sample_routing(lib):
    h = _hdr(32, 16)
    h.lr_unit_size[0] = 64
    curr, ca = _plane(np.arange(128 * 64).reshape(128, 64) % 251)
    cdef, cda = _plane(np.full((128, 64), 99))
    # inside the stripe of row 0: CDEF frame
    assert lib.ora_lr_source_sample(C.byref(h), 0, 0, 0, C.byref(curr), C.byref(cdef), 5, 10) == 99
    # stripe 1 (luma rows 56..119) reading above its start: deblocked frame, clamped to start-2
    v = lib.ora_lr_source_sample(C.byref(h), 0, 16, 0, C.byref(curr), C.byref(cdef), 5, 50)
    assert v == ca[54, 5]
    # stripe 0 reading below its end: deblocked frame rows 56, 57 then clamped
    assert lib.ora_lr_source_sample(C.byref(h), 0, 0, 0, C.byref(curr), C.byref(cdef), 3, 56) == ca[56, 3]
    assert lib.ora_lr_source_sample(C.byref(h), 0, 0, 0, C.byref(curr), C.byref(cdef), 3, 60) == ca[57, 3]


def _lr_frame(lib, unit, fill_cdef=175, fill_curr=10, size=64):
    f = synth.make_frame(seed=3, width=size, height=size, mono=True, deblock=False, cdef=False)
    f.hdr.lr_type[0] = unit["type"] if unit["type"] else 1
    u = np.zeros(f.lr_grid(0), synth.LR_DTYPE)
    u["type"] = unit["type"]
    u["sgr_set"] = unit.get("sgr_set", 0)
    u["wiener"] = unit.get("wiener", 0)
    u["sgr_xqd"] = unit.get("sgr_xqd", (0, 0))
    f.lr_units[0] = u
    curr = [np.full(f.plane_dims(0), fill_curr, np.int32)]
    cdef = [np.full(f.plane_dims(0), fill_cdef, np.int32)]
    return oracle.loop_restoration(f, curr, cdef)[0]


def test_restore_none_keeps_cdef_copy(lib):
    assert (_lr_frame(lib, {"type": 0}) == 175).all()


def test_wiener_identity_filter_recovers_source(lib):
    assert (_lr_frame(lib, {"type": 1}, fill_cdef=100, fill_curr=100) == 100).all()


def test_self_guided_w2_zero_recovers_source(lib):
    # w0 = 0, w1 = 128 => w2 = 0: v = 128 * u => the CDEF sample itself
    out = _lr_frame(lib, {"type": 2, "sgr_set": 0, "sgr_xqd": (0, 128)}, fill_cdef=137, fill_curr=137)
    assert (out == 137).all()


@pytest.mark.parametrize("sgr_set", [10, 14])
def test_self_guided_single_radius_sets(lib, sgr_set):
    out = _lr_frame(lib, {"type": 2, "sgr_set": sgr_set, "sgr_xqd": (0, 64)}, fill_cdef=200, fill_curr=200)
    assert (out == 200).all()


# --- superres.rs tests -----------------------------------------------------------

def _sr_frame(w_up=128, denom=16, bd=8, mono=False):
    return synth.make_frame(seed=5, width=w_up, height=32, bit_depth=bd, superres_denom=denom, mono=mono)


def test_flat_input_yields_flat_output():
    f = _sr_frame()
    src = [np.full(f.plane_dims(p), v, np.int32) for p, v in zip(range(3), (80, 80, 80))]
    out = oracle.upscale(f, src)
    assert all((o == 80).all() for o in out)


def test_chroma_subsampling_halves_widths():
    f = _sr_frame()
    src = [np.full(f.plane_dims(p), v, np.int32) for p, v in zip(range(3), (64, 128, 192))]
    out = oracle.upscale(f, src)
    assert out[1].shape[1] == (f.hdr.upscaled_width + 1) // 2
    assert [(o == v).all() for o, v in zip(out, (64, 128, 192))] == [True] * 3


def test_upscale_clips_to_bit_depth():
    f = _sr_frame()
    rng = np.random.default_rng(0)
    src = [np.where(rng.random(f.plane_dims(p)) < 0.5, 0, 255).astype(np.int32) for p in range(3)]
    out = oracle.upscale(f, src)
    assert all(((o >= 0) & (o <= 255)).all() for o in out)


def test_upscale_rejects_smaller_target():
    f = _sr_frame()
    f.hdr.upscaled_width = f.hdr.frame_width - 8
    src = [np.zeros(f.plane_dims(p), np.int32) for p in range(3)]
    with pytest.raises(RuntimeError):
        oracle.upscale(f, src)


# --- film_grain.rs tests ---------------------------------------------------------

def test_lfsr_known_draws():
    assert oracle.random_draws(1, 11, 2) == [0x400, 0x200]
    assert oracle.random_draws(0xFF00, 8, 1) == [0xFF]


def _fg(**kw):
    fg = abi.FilmGrain()
    fg.apply_grain = 1
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            arr = getattr(fg, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(fg, k, v)
    return fg


def test_scaling_lookup_zero_points_is_zero_table():
    assert (oracle.scaling_lut(_fg(), 3) == 0).all()


def test_scaling_lookup_two_point_ramp():
    lut = oracle.scaling_lut(_fg(num_y_points=2, point_y_value=[0, 255], point_y_scaling=[0, 255]), 1)
    assert lut[0, 0] == 0 and abs(int(lut[0, 128]) - 128) <= 1 and lut[0, 255] == 255


def test_scaling_lookup_left_plateau():
    lut = oracle.scaling_lut(_fg(num_y_points=2, point_y_value=[32, 255], point_y_scaling=[64, 200]), 1)
    assert (lut[0, :32] == 64).all() and lut[0, 255] == 200


def test_generate_grain_zero_without_points():
    luma, cb, cr = oracle.generate_grain(_fg(grain_seed=12345), 8, 1, 1)
    assert not luma.any() and not cb.any() and not cr.any()
    assert cb.shape == (38, 44)


def test_generate_grain_first_sample_is_round2_of_first_draw():
    from oxideav_av1_b200 import tables
    fg = _fg(grain_seed=1, num_y_points=2, point_y_value=[0, 255], point_y_scaling=[0, 255], ar_coeff_lag=0,
             ar_coeff_shift=6)
    luma, _, _ = oracle.generate_grain(fg, 8, 1, 1)
    g = tables.GAUSSIAN_SEQUENCE[oracle.random_draws(1, 11, 1)[0]]
    assert luma[0, 0] == (g + 8) >> 4


def test_film_grain_no_apply_is_noop():
    f = synth.make_frame(seed=9, width=64, height=32)
    planes = [np.full(f.out_dims(p), 100, np.int32) for p in range(3)]
    f.hdr.film_grain.apply_grain = 0
    out = oracle.film_grain(f, [p.copy() for p in planes])
    assert all((o == 100).all() for o in out)


def test_film_grain_zero_y_points_leaves_luma():
    f = synth.make_frame(seed=9, width=64, height=32, film_grain=True)
    f.hdr.film_grain.num_y_points = 0
    planes = [np.full(f.out_dims(p), 100, np.int32) for p in range(3)]
    out = oracle.film_grain(f, [p.copy() for p in planes])
    assert (out[0] == 100).all()
