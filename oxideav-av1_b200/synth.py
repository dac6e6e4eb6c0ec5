"""Seeded synthetic post-filter frames (the decoder's pre-parsed symbol state).

The reference measures its post-filter path on encoder-produced streams that
cannot be produced in this environment (its Rust encoder does not build here),
so the workload is generated directly at the seam the engine consumes: a
frame's reconstructed planes at the padded mi extent plus the per-mi decode
grids and the frame header fields the §7.14-§7.18 stages read.

Shapes and value distributions follow the post-filter micro-benchmark
configuration (1920x1080 4:2:0, 8-bit and a 10-bit variant):
  * planes: a 16x16 uniform random field, bilinearly upsampled, plus uniform
    noise in [-12, 12] (scaled by 2^(bitdepth-8)), clipped to the sample range;
  * a random legal partition of every 64x64 superblock (NONE / HORZ / VERT /
    SPLIT / HORZ_4 / VERT_4), per block a transform size from the legal set
    (Max_Tx_Size_Rect split 0..2 times), intra/inter, skip, modes, references,
    segment ids and delta-LF values;
  * deblock levels uniform 0..63 with sharpness 0..7; per-64x64 CDEF indices
    uniform over 1 << cdef_bits = 8 strength sets with primary 0..15,
    secondary {0,1,2,4}, damping 3..6;
  * 64x64 restoration units, each Wiener (taps uniform within the spec
    coefficient bounds, chroma tap 0 = 0) or self-guided (set 0..15, projection
    weights within the spec bounds).
Superres and film grain are off in that configuration; the generator can turn
them on for parity cases.
"""
import ctypes as C

import numpy as np

from . import abi

# (w4, h4) in 4x4 units -> BLOCK_* ordinal (spec §3 block size order)
BLOCK_OF = {(1, 1): 0, (1, 2): 1, (2, 1): 2, (2, 2): 3, (2, 4): 4, (4, 2): 5, (4, 4): 6, (4, 8): 7, (8, 4): 8,
            (8, 8): 9, (8, 16): 10, (16, 8): 11, (16, 16): 12, (16, 32): 13, (32, 16): 14, (32, 32): 15,
            (1, 4): 16, (4, 1): 17, (2, 8): 18, (8, 2): 19, (4, 16): 20, (16, 4): 21}
# Max_Tx_Size_Rect[BLOCK_*] and Split_Tx_Size[TX_*] (spec additional tables)
MAX_TX_RECT = [0, 5, 6, 1, 7, 8, 2, 9, 10, 3, 11, 12, 4, 4, 4, 4, 13, 14, 15, 16, 17, 18]
SPLIT_TX = [0, 0, 1, 2, 3, 0, 0, 1, 1, 2, 2, 3, 3, 5, 6, 7, 8, 9, 10]

WIENER_MIN = [-5, -23, -17]
WIENER_MAX = [10, 8, 46]
SGR_R = [(2, 1), (2, 1), (2, 1), (2, 1), (2, 1), (2, 1), (2, 1), (2, 1), (2, 1), (2, 1), (0, 1), (0, 1), (0, 1),
         (0, 1), (2, 0), (2, 0)]

LR_DTYPE = np.dtype([("type", np.uint8), ("sgr_set", np.uint8), ("wiener", np.int8, (2, 3)),
                     ("sgr_xqd", np.int16, (2,))], align=True)
assert LR_DTYPE.itemsize == C.sizeof(abi.LrUnit)


def _lerp_weights(n):
    pos = np.linspace(0, 15, n)
    i0 = np.minimum(pos.astype(np.int64), 14)
    return i0, pos - i0


def _field(rng, h, w, maxv):
    """16x16 uniform field bilinearly upsampled to h x w."""
    f = rng.uniform(0, maxv, size=(16, 16))
    xi, xf = _lerp_weights(w)
    rows = f[:, xi] * (1 - xf) + f[:, xi + 1] * xf
    yi, yf = _lerp_weights(h)
    return rows[yi] * (1 - yf)[:, None] + rows[yi + 1] * yf[:, None]


def _plane(rng, h, w, bd):
    maxv = (1 << bd) - 1
    base = _field(rng, h, w, maxv)
    noise = rng.integers(-12, 13, size=(h, w)) * (1 << (bd - 8))
    v = np.clip(np.rint(base) + noise, 0, maxv)
    return v.astype(np.uint8 if bd == 8 else np.uint16)


class SyntheticFrame:
    """One frame's post-filter inputs: header, mi grids, CDEF indices, LR units, planes."""

    def __init__(self):
        self.hdr = abi.FrameHeader()
        self.grid = {}
        self.cdef_idx = None
        self.lr_units = [None, None, None]
        self.recon = []

    @property
    def hbd(self):
        return self.hdr.bit_depth > 8

    def plane_dims(self, p):
        """padded (height, width) of plane p."""
        h = self.hdr
        sx = h.subsampling_x if p else 0
        sy = h.subsampling_y if p else 0
        return (h.mi_rows * 4) >> sy, (h.mi_cols * 4) >> sx

    def out_dims(self, p):
        """cropped (height, width) of output plane p."""
        h = self.hdr
        sx = h.subsampling_x if p else 0
        sy = h.subsampling_y if p else 0
        return (h.frame_height + sy) >> sy, (h.upscaled_width + sx) >> sx

    def lr_grid(self, p):
        h = self.hdr
        sx = h.subsampling_x if p else 0
        sy = h.subsampling_y if p else 0
        us = h.lr_unit_size[p]
        rows = _count_units(us, (h.frame_height + (1 << sy >> 1)) >> sy)
        cols = _count_units(us, (h.upscaled_width + (1 << sx >> 1)) >> sx)
        return rows, cols


def _count_units(us, size):
    return max((size + (us >> 1)) // us, 1)


def _partition(rng, grid, r, c, n4, mi_rows, mi_cols, depth_bias):
    """Random legal partition of a square block of n4 x n4 4x4 units at (r, c)."""
    if r >= mi_rows or c >= mi_cols:
        return
    opts = ["NONE"]
    if n4 > 1:
        opts += ["HORZ", "VERT", "SPLIT"]
        if n4 >= 4:
            opts += ["HORZ_4", "VERT_4"]
    w = np.array([1.0 if o == "NONE" else (depth_bias if o == "SPLIT" else 0.5) for o in opts])
    # blocks crossing the frame edge split like the spec's forced partitions
    if r + n4 > mi_rows or c + n4 > mi_cols:
        if n4 > 1:
            opts, w = ["SPLIT"], np.array([1.0])
    o = opts[rng.choice(len(opts), p=w / w.sum())]
    if o == "NONE":
        _leaf(rng, grid, r, c, n4, n4)
    elif o == "HORZ":
        _leaf(rng, grid, r, c, n4, n4 // 2)
        _leaf(rng, grid, r + n4 // 2, c, n4, n4 // 2)
    elif o == "VERT":
        _leaf(rng, grid, r, c, n4 // 2, n4)
        _leaf(rng, grid, r, c + n4 // 2, n4 // 2, n4)
    elif o == "HORZ_4":
        for k in range(4):
            _leaf(rng, grid, r + k * n4 // 4, c, n4, n4 // 4)
    elif o == "VERT_4":
        for k in range(4):
            _leaf(rng, grid, r, c + k * n4 // 4, n4 // 4, n4)
    else:
        h = n4 // 2
        for dr in (0, h):
            for dc in (0, h):
                _partition(rng, grid, r + dr, c + dc, h, mi_rows, mi_cols, depth_bias * 0.85)


def _leaf(rng, grid, r, c, w4, h4):
    bs = BLOCK_OF[(w4, h4)]
    tx = MAX_TX_RECT[bs]
    for _ in range(rng.integers(0, 3)):
        tx = SPLIT_TX[tx]
    inter = rng.random() < 0.5
    sl = (slice(r, r + h4), slice(c, c + w4))
    g = grid
    g["mi_size"][sl] = bs
    g["skip"][sl] = rng.random() < 0.3
    g["is_inter"][sl] = inter
    g["ref_frame0"][sl] = rng.integers(1, 8) if inter else 0
    g["y_mode"][sl] = rng.integers(14, 26) if inter else rng.integers(0, 13)
    g["segment_id"][sl] = rng.integers(0, 8) if g["_seg"] else 0
    g["delta_lf"][sl] = rng.integers(-6, 7, size=4) if g["_dlf"] else 0
    g["tx_size"][sl] = tx
    g["inter_tx_size"][sl] = tx


def make_frame(seed, width=1920, height=1080, bit_depth=8, ssx=1, ssy=1, mono=False, superres_denom=8,
               film_grain=False, lr_unit=64, lr_uv_shift=0, lr_types=(3, 3, 3), lr_none_frac=0.0, deblock=True,
               cdef=True, lr=True, segmentation=True, delta_lf=True):
    rng = np.random.default_rng(seed)
    f = SyntheticFrame()
    h = f.hdr
    up_w = width
    fw = (up_w * 8 + superres_denom // 2) // superres_denom if superres_denom != 8 else up_w
    h.frame_width, h.frame_height, h.upscaled_width = fw, height, up_w
    h.mi_cols = 2 * ((fw + 7) >> 3)
    h.mi_rows = 2 * ((height + 7) >> 3)
    h.bit_depth = bit_depth
    h.num_planes = 1 if mono else 3
    h.subsampling_x, h.subsampling_y = (1, 1) if mono else (ssx, ssy)
    h.matrix_coefficients = int(rng.integers(0, 3))
    h.use_superres = 1 if superres_denom != 8 else 0
    h.enable_cdef = 1 if cdef else 0
    # §5.9.11 loop filter
    if deblock:
        for i in range(4):
            h.lf_level[i] = int(rng.integers(0, 64))
        h.lf_level[0] = max(h.lf_level[0], 1)
    h.lf_sharpness = int(rng.integers(0, 8))
    h.lf_delta_enabled = int(rng.random() < 0.7)
    h.delta_lf_multi = int(rng.random() < 0.5)
    for i, d in enumerate([1, 0, 0, 0, -1, 0, -1, -1]):
        h.lf_ref_deltas[i] = int(np.clip(d + rng.integers(-3, 4), -63, 63))
    h.lf_mode_deltas[0] = int(rng.integers(-3, 4))
    h.lf_mode_deltas[1] = int(rng.integers(-3, 4))
    if segmentation:
        for s in range(8):
            for i in range(4):
                if rng.random() < 0.3:
                    h.seg_lf_active[s][i] = 1
                    h.seg_lf_data[s][i] = int(rng.integers(-20, 21))
    # §5.9.19 cdef
    h.cdef_short_circuited = 0
    h.cdef_damping = int(rng.integers(3, 7))
    h.cdef_bits = 3
    for i in range(8):
        h.cdef_y_pri[i] = int(rng.integers(0, 16))
        h.cdef_y_sec[i] = int(rng.choice([0, 1, 2, 4]))
        h.cdef_uv_pri[i] = int(rng.integers(0, 16))
        h.cdef_uv_sec[i] = int(rng.choice([0, 1, 2, 4]))
    # §5.9.20 restoration
    h.uses_lr = 1 if lr else 0
    for p in range(3):
        h.lr_type[p] = lr_types[p] if lr else 0
        h.lr_unit_size[p] = lr_unit if p == 0 else lr_unit >> lr_uv_shift
    # grids
    mr, mc = h.mi_rows, h.mi_cols
    g = {
        "mi_size": np.zeros((mr, mc), np.uint8), "skip": np.zeros((mr, mc), np.uint8),
        "is_inter": np.zeros((mr, mc), np.uint8), "ref_frame0": np.zeros((mr, mc), np.int8),
        "y_mode": np.zeros((mr, mc), np.uint8), "segment_id": np.zeros((mr, mc), np.int8),
        "delta_lf": np.zeros((mr, mc, 4), np.int8), "tx_size": np.zeros((mr, mc), np.uint8),
        "inter_tx_size": np.zeros((mr, mc), np.uint8), "_seg": segmentation, "_dlf": delta_lf,
    }
    for r in range(0, mr, 16):
        for c in range(0, mc, 16):
            _partition(rng, g, r, c, 16, mr, mc, 1.6)
    del g["_seg"], g["_dlf"]
    f.grid = g
    cr, cc = (mr + 15) // 16, (mc + 15) // 16
    idx = rng.integers(0, 8, size=(cr, cc)).astype(np.int8)
    idx[rng.random((cr, cc)) < 0.05] = -1
    f.cdef_idx = idx
    for p in range(h.num_planes):
        rows, cols = f.lr_grid(p)
        u = np.zeros((rows, cols), LR_DTYPE)
        kinds = rng.random((rows, cols))
        for i in range(rows):
            for j in range(cols):
                k = kinds[i, j]
                if k < lr_none_frac:
                    continue
                if k < lr_none_frac + (1 - lr_none_frac) / 2:
                    u[i, j]["type"] = 1
                    for ps in range(2):
                        for t in range(3):
                            v = int(rng.integers(WIENER_MIN[t], WIENER_MAX[t] + 1))
                            u[i, j]["wiener"][ps, t] = 0 if (p > 0 and t == 0) else v
                else:
                    u[i, j]["type"] = 2
                    s = int(rng.integers(0, 16))
                    u[i, j]["sgr_set"] = s
                    r0, r1 = SGR_R[s]
                    w0 = int(rng.integers(-96, 32)) if r0 else 0
                    w1 = int(rng.integers(-32, 96))
                    if r1 == 0:
                        w1 = int(np.clip(128 - w0, -32, 95))
                    u[i, j]["sgr_xqd"] = (w0, w1)
        f.lr_units[p] = u
    for p in range(h.num_planes):
        ph, pw = f.plane_dims(p)
        f.recon.append(_plane(rng, ph, pw, bit_depth))
    if film_grain:
        _film_grain(rng, h.film_grain, bit_depth, mono)
    return f


def _points(rng, n, maxn):
    n = min(n, maxn)
    xs = np.sort(rng.choice(np.arange(256), size=n, replace=False)) if n else np.array([], int)
    ys = rng.integers(0, 256, size=n)
    return xs, ys


def _film_grain(rng, fg, bd, mono):
    fg.apply_grain = 1
    fg.grain_seed = int(rng.integers(0, 65536))
    ny = int(rng.integers(1, 15))
    xs, ys = _points(rng, ny, 14)
    fg.num_y_points = len(xs)
    for i in range(len(xs)):
        fg.point_y_value[i], fg.point_y_scaling[i] = int(xs[i]), int(ys[i])
    fg.chroma_scaling_from_luma = 0 if mono else int(rng.random() < 0.25)
    if not mono and not fg.chroma_scaling_from_luma:
        for name in ("cb", "cr"):
            n = int(rng.integers(0, 11))
            xs, ys = _points(rng, n, 10)
            setattr(fg, f"num_{name}_points", len(xs))
            vals, scs = getattr(fg, f"point_{name}_value"), getattr(fg, f"point_{name}_scaling")
            for i in range(len(xs)):
                vals[i], scs[i] = int(xs[i]), int(ys[i])
    fg.grain_scaling = int(rng.integers(8, 12))
    fg.ar_coeff_lag = int(rng.integers(0, 4))
    for i in range(24):
        fg.ar_coeffs_y_plus_128[i] = int(128 + rng.integers(-24, 25))
    for i in range(25):
        fg.ar_coeffs_cb_plus_128[i] = int(128 + rng.integers(-24, 25))
        fg.ar_coeffs_cr_plus_128[i] = int(128 + rng.integers(-24, 25))
    fg.ar_coeff_shift = int(rng.integers(6, 10))
    fg.grain_scale_shift = int(rng.integers(0, 4))
    fg.cb_mult, fg.cb_luma_mult = int(rng.integers(0, 256)), int(rng.integers(0, 256))
    fg.cr_mult, fg.cr_luma_mult = int(rng.integers(0, 256)), int(rng.integers(0, 256))
    fg.cb_offset, fg.cr_offset = int(rng.integers(0, 512)), int(rng.integers(0, 512))
    fg.overlap_flag = int(rng.random() < 0.7)
    fg.clip_to_restricted_range = int(rng.random() < 0.5)


# ---------------------------------------------------------------------------
# Reconstruction workloads: predictions + TU lists with coefficients
# ---------------------------------------------------------------------------

TU_DTYPE = np.dtype([("x", np.uint16), ("y", np.uint16), ("plane", np.uint8), ("tx_size", np.uint8),
                     ("tx_type", np.uint8), ("segment_id", np.uint8), ("current_q_index", np.uint8),
                     ("pad", np.uint8, (3,)), ("coeff_offset", np.uint32)])
assert TU_DTYPE.itemsize == C.sizeof(abi.Tu)
TX_W = [4, 8, 16, 32, 64, 4, 8, 8, 16, 16, 32, 32, 64, 4, 16, 8, 32, 16, 64]
TX_H = [4, 8, 16, 32, 64, 8, 4, 16, 8, 32, 16, 64, 32, 16, 4, 32, 8, 64, 16]
TX_OF = {(w, h): i for i, (w, h) in enumerate(zip(TX_W, TX_H))}


class ReconFrame:
    """Prediction planes + the TUs (with levels) the reference would reconstruct."""

    def __init__(self):
        self.hdr = abi.FrameHeader()
        self.quant = abi.QuantParams()
        self.tus = None
        self.coeffs = None
        self.planes = []

    @property
    def hbd(self):
        return self.hdr.bit_depth > 8

    def plane_dims(self, p):
        h = self.hdr
        return (h.mi_rows * 4) >> (h.subsampling_y if p else 0), (h.mi_cols * 4) >> (h.subsampling_x if p else 0)


def _tx_type_for(rng, w, h):
    m = max(w, h)
    if m == 64:
        return 0                                   # TX_SET_DCTONLY
    if m == 32:
        return int(rng.choice([0, 9]))             # DCT_DCT or IDTX
    return int(rng.integers(0, 16))


def _levels(rng, tw, th, big):
    n = tw * th
    lv = np.zeros(n, np.int32)
    k = int(min(n, 1 + rng.geometric(0.15)))       # roughly an end-of-block position
    mags = rng.geometric(0.35, size=k).astype(np.int64)
    sign = np.where(rng.random(k) < 0.5, -1, 1)
    lv[:k] = (mags * sign).astype(np.int32)
    if big and rng.random() < 0.2:
        lv[int(rng.integers(0, k))] = int(rng.choice([-1, 1]) * rng.integers(2000, 200000))
    return lv


def make_recon_frame(seed, width=352, height=288, bit_depth=8, ssx=1, ssy=1, mono=False, qmatrix=True,
                     lossless_segments=True, big_levels=True):
    rng = np.random.default_rng(seed)
    f = ReconFrame()
    h = f.hdr
    h.frame_width = h.upscaled_width = width
    h.frame_height = height
    h.mi_cols, h.mi_rows = 2 * ((width + 7) >> 3), 2 * ((height + 7) >> 3)
    h.bit_depth = bit_depth
    h.num_planes = 1 if mono else 3
    h.subsampling_x, h.subsampling_y = (1, 1) if mono else (ssx, ssy)
    q = f.quant
    q.base_q_idx = int(rng.integers(0, 256))
    for name in ("delta_q_y_dc", "delta_q_u_dc", "delta_q_u_ac", "delta_q_v_dc", "delta_q_v_ac"):
        setattr(q, name, int(rng.integers(-15, 16)))
    q.using_qmatrix = int(qmatrix and rng.random() < 0.7)
    q.delta_q_present = int(rng.random() < 0.5)
    q.segmentation_enabled = 1
    for s in range(8):
        q.seg_alt_q_active[s] = int(rng.random() < 0.4)
        q.seg_alt_q_data[s] = int(rng.integers(-60, 61))
        for p in range(3):
            q.seg_qm_level[p][s] = int(rng.integers(0, 16))
        q.lossless[s] = int(lossless_segments and s == 7)
    maxv = (1 << bit_depth) - 1
    for p in range(h.num_planes):
        ph, pw = f.plane_dims(p)
        f.planes.append(rng.integers(0, maxv + 1, size=(ph, pw)).astype(np.uint8 if bit_depth == 8 else np.uint16))
    tus, coeffs, off = [], [], 0
    for p in range(h.num_planes):
        ph, pw = f.plane_dims(p)
        # tile the plane with 64x64 areas, each split into TUs of one random legal size
        for y0 in range(0, ph, 64):
            for x0 in range(0, pw, 64):
                seg = int(rng.integers(0, 8))
                if q.lossless[seg]:
                    w = hh = 4
                else:
                    w, hh = [(TX_W[i], TX_H[i]) for i in range(19)][int(rng.integers(0, 19))]
                tx = TX_OF[(w, hh)]
                cq = int(rng.integers(1, 256))
                for y in range(y0, min(y0 + 64, ph), hh):
                    for x in range(x0, min(x0 + 64, pw), w):
                        if rng.random() < 0.3:
                            continue                      # no coefficients (eob == 0): not listed
                        tw, th = min(32, w), min(32, hh)
                        tt = 0 if q.lossless[seg] else _tx_type_for(rng, w, hh)
                        tus.append((x, y, p, tx, tt, seg, cq, (0, 0, 0), off))
                        coeffs.append(_levels(rng, tw, th, big_levels))
                        off += tw * th
    f.tus = np.array(tus, dtype=TU_DTYPE)
    f.coeffs = np.concatenate(coeffs).astype(np.int32) if coeffs else np.zeros(1, np.int32)
    return f


# ---------------------------------------------------------------------------
# Intra workloads: TU lists in decode order with prediction parameters
# ---------------------------------------------------------------------------

INTRA_TU_DTYPE = np.dtype([("x", np.uint16), ("y", np.uint16), ("plane", np.uint8), ("tx_size", np.uint8),
                           ("mode", np.uint8), ("flags", np.uint8), ("angle_delta", np.int8), ("cfl_alpha", np.int8),
                           ("filter_intra_mode", np.uint8), ("pad", np.uint8), ("max_luma_w", np.uint16),
                           ("max_luma_h", np.uint16), ("res", TU_DTYPE), ("mv", np.int16, (2,)),
                           ("palette_map", np.uint32), ("palette_stride", np.uint16), ("palette_size", np.uint8),
                           ("pad2", np.uint8), ("palette_colors", np.uint16, (8,)), ("interintra", np.uint8),
                           ("interintra_mode", np.uint8), ("wedge_index", np.uint8), ("mi_size", np.uint8)])
assert INTRA_TU_DTYPE.itemsize == C.sizeof(abi.IntraTu)


class IntraFrame(ReconFrame):
    """Planes (left as garbage: intra TUs overwrite every sample) + intra TUs in decode order."""

    def __init__(self):
        super().__init__()
        self.sb_size = 64


def _blocks(rng, x0, y0, n, pw, ph, out, split=0.55):
    """Recursive square/rect partition of an n x n area (samples) into blocks,
    in decode order; `split` is the probability of a quad split."""
    if x0 >= pw or y0 >= ph:
        return
    if n > 4 and (rng.random() < split or x0 + n > pw or y0 + n > ph):
        h = n // 2
        for dy in (0, h):
            for dx in (0, h):
                _blocks(rng, x0 + dx, y0 + dy, h, pw, ph, out, split)
        return
    r = rng.random()
    if n >= 8 and r < 0.2:
        out.append((x0, y0, n, n // 2))
        out.append((x0, y0 + n // 2, n, n // 2))
    elif n >= 8 and r < 0.4:
        out.append((x0, y0, n // 2, n))
        out.append((x0 + n // 2, y0, n // 2, n))
    else:
        out.append((x0, y0, n, n))


def tile_grid(mi_rows, mi_cols, sb_size, tile_cols_log2=0, tile_rows_log2=0):
    """Uniformly spaced tiles (§5.9.15 with uniform_tile_spacing_flag): the
    luma-sample edges [x0, x1) and [y0, y1) of the tile columns and rows."""
    sb_cols = -(-mi_cols * 4 // sb_size)
    sb_rows = -(-mi_rows * 4 // sb_size)

    def edges(n_sb, log2, limit):
        step = (n_sb + (1 << log2) - 1) >> log2
        xs = list(range(0, n_sb, step)) + [n_sb]
        return [(a * sb_size, min(b * sb_size, limit)) for a, b in zip(xs[:-1], xs[1:])]
    return edges(sb_cols, tile_cols_log2, mi_cols * 4), edges(sb_rows, tile_rows_log2, mi_rows * 4)


def make_intra_frame(seed, width=176, height=144, bit_depth=8, ssx=1, ssy=1, mono=False, sb_size=64,
                     edge_filter=True, palette=0.0, intrabc=0.0, intrabc_order="wavefront", split=0.55, tiles=(0, 0)):
    """Intra TUs in decode order.  palette / intrabc: probability that a block
    is a palette block / an intra-block-copy block; split: probability of a
    quad split in the block partition.  intrabc_order picks where
    copies read from: "wavefront" (the superblock row above, within reach of
    the level-2 wavefront), "steep" (further right in the row above, which
    needs a steeper wavefront) or "raster" (the row below, not yet decoded,
    which only decode order reproduces).  tiles = (tile_cols_log2,
    tile_rows_log2): superblocks in tile order, and the edge availability of
    every TU bounded by its tile as the tile walker sets it (AvailU / AvailL
    and the above-right / below-left tests stop at the tile edge); intra
    block copies then stay off."""
    rng = np.random.default_rng(seed)
    base = make_recon_frame(seed + 1000, width, height, bit_depth, ssx, ssy, mono)
    f = IntraFrame()
    f.hdr, f.quant, f.sb_size = base.hdr, base.quant, sb_size
    h = f.hdr
    maxv = (1 << bit_depth) - 1
    f.planes = [rng.integers(0, maxv + 1, size=f.plane_dims(p)).astype(np.uint8 if bit_depth == 8 else np.uint16)
                for p in range(h.num_planes)]
    tus, coeffs, off = [], [], 0
    maps, map_off = [], 0
    decoded = [np.zeros(((f.plane_dims(p)[0] + 3) // 4, (f.plane_dims(p)[1] + 3) // 4), bool)
               for p in range(h.num_planes)]
    lossless_seg = [s for s in range(8) if f.quant.lossless[s]]
    tcols, trows = tile_grid(h.mi_rows, h.mi_cols, sb_size, *tiles)
    if tiles != (0, 0):
        intrabc = 0.0
    order = [(ty0, ty1, tx0, tx1, sby, sbx) for (ty0, ty1) in trows for (tx0, tx1) in tcols
             for sby in range(ty0, ty1, sb_size) for sbx in range(tx0, tx1, sb_size)]
    for (ty0, ty1, tx0, tx1, sby, sbx) in order:
        if True:
            for p in range(h.num_planes):
                sx_, sy_ = (h.subsampling_x, h.subsampling_y) if p else (0, 0)
                ph, pw = f.plane_dims(p)
                # the tile in this plane's samples
                tpx0, tpx1, tpy0, tpy1 = tx0 >> sx_, min(tx1 >> sx_, pw), ty0 >> sy_, min(ty1 >> sy_, ph)
                blocks = []
                _blocks(rng, sbx >> sx_, sby >> sy_, sb_size >> max(sx_, sy_), pw, ph, blocks, split)
                for (bx, by, bw, bh) in blocks:
                    # a legal TU size for the block (Max_Tx_Size_Rect, optionally split once)
                    bw_, bh_ = min(bw, 64), min(bh, 64)
                    tw, th = bw_, bh_
                    if rng.random() < 0.3 and tw >= 8 and th >= 8:
                        tw, th = tw // 2, th // 2
                    if (tw, th) not in TX_OF:
                        tw, th = min(tw, th), min(tw, th)
                    tx = TX_OF[(tw, th)]
                    mode = int(rng.integers(0, 13))
                    ad = int(rng.integers(-3, 4)) if 1 <= mode <= 8 else 0
                    fim = 255
                    cfl = False
                    if p == 0 and tw <= 32 and th <= 32 and rng.random() < 0.15:
                        mode, ad, fim = 0, 0, int(rng.integers(0, 5))
                    if p > 0 and rng.random() < 0.25:
                        mode, ad, cfl = 0, 0, True
                    kind = rng.random()
                    pal, bc_mv = None, None
                    if kind < palette:
                        n_col = int(rng.integers(1, 9))
                        colors = [int(v) for v in rng.integers(0, maxv + 1, size=n_col)] + [0] * (8 - n_col)
                        idx = rng.integers(0, n_col, size=(bh, bw)).astype(np.uint8)
                        pal = (map_off, bw, n_col, colors)
                        maps.append(idx.ravel())
                        map_off += idx.size
                        mode, ad, fim, cfl = abi.INTRA_MODE_PALETTE, 0, 255, False
                    elif kind < palette + intrabc:
                        sbp_x, sbp_y = sb_size >> sx_, sb_size >> sy_
                        spx, spy = sbx >> sx_, sby >> sy_
                        src = None
                        if intrabc_order in ("wavefront", "steep") and spy >= sbp_y and spy - bh - 5 >= 0:
                            reach = 2 if intrabc_order == "wavefront" else 5
                            xs_max = min(spx + reach * sbp_x - bw - 6, pw - bw)
                            xs_min = spx + 2 * sbp_x if intrabc_order == "steep" else 0
                            if xs_max >= max(xs_min, 0):
                                src = (int(rng.integers(max(xs_min, 0), xs_max + 1)),
                                       int(rng.integers(0, spy - bh - 5 + 1)))
                        elif intrabc_order == "raster" and spy + sbp_y + bh + 5 <= ph and spx >= 3 * sbp_x:
                            src = (int(rng.integers(0, spx - 2 * sbp_x)),
                                   int(rng.integers(spy + sbp_y, ph - bh - 5 + 1)))
                        if src is not None:
                            odd = int(rng.integers(0, 2))
                            bc_mv = (((src[1] - by) << sy_) * 8, (((src[0] - bx) << sx_) + odd) * 8)
                            mode, ad, fim, cfl = abi.INTRA_MODE_INTRABC, 0, 255, False
                    seg = int(rng.integers(0, 8))
                    if seg in lossless_seg and tx != 0:
                        seg = 0 if 0 not in lossless_seg else 1
                    for ty in range(by, by + bh, th):
                        for tx_ in range(bx, bx + bw, tw):
                            if ty >= ph or tx_ >= pw:
                                continue
                            flags = 0
                            if ty > tpy0:
                                flags |= abi.INTRA_HAVE_ABOVE
                            if tx_ > tpx0:
                                flags |= abi.INTRA_HAVE_LEFT
                            cy, cx = ty // 4, tx_ // 4
                            if ty > tpy0 and tx_ + tw < tpx1 and (tx_ + tw) // 4 < decoded[p].shape[1] and \
                                    decoded[p][cy - 1, (tx_ + tw) // 4]:
                                flags |= abi.INTRA_HAVE_ABOVE_RIGHT
                            if tx_ > tpx0 and ty + th < tpy1 and (ty + th) // 4 < decoded[p].shape[0] and \
                                    decoded[p][(ty + th) // 4, cx - 1]:
                                flags |= abi.INTRA_HAVE_BELOW_LEFT
                            if edge_filter:
                                flags |= abi.INTRA_EDGE_FILTER
                            if rng.random() < 0.3:
                                flags |= abi.INTRA_FILTER_TYPE
                            if cfl:
                                flags |= abi.INTRA_CFL
                            res = (tx_, ty, p, tx, 0, seg, int(rng.integers(1, 256)), (0, 0, 0), 0)
                            if rng.random() < 0.7 and (seg not in lossless_seg or tx == 0):
                                flags |= abi.INTRA_RESIDUAL
                                tt = 0 if seg in lossless_seg else _tx_type_for(rng, tw, th)
                                res = (tx_, ty, p, tx, tt, seg, res[6], (0, 0, 0), off)
                                lv = _levels(rng, min(32, tw), min(32, th), True)
                                coeffs.append(lv)
                                off += len(lv)
                            mlw = min((bx + bw) << sx_, 65535)
                            mlh = min((by + bh) << sy_, 65535)
                            pm, ps, pn, pc = (0, 0, 0, [0] * 8) if pal is None else pal
                            if pal is not None:
                                pm += (ty - by) * bw + (tx_ - bx)
                            tus.append((tx_, ty, p, tx, mode, flags, ad, int(rng.integers(-16, 17)) if cfl else 0,
                                        fim, 0, mlw, mlh, res, bc_mv if bc_mv else (0, 0), pm, ps, pn, 0, pc,
                                        0, 0, 0, 0))
                            decoded[p][cy:cy + (th + 3) // 4, cx:cx + (tw + 3) // 4] = True
    f.tus = np.array(tus, dtype=INTRA_TU_DTYPE)
    f.coeffs = np.concatenate(coeffs).astype(np.int32) if coeffs else np.zeros(1, np.int32)
    f.palette_maps = np.concatenate(maps).astype(np.uint8) if maps else np.zeros(0, np.uint8)
    return f


# ---------------------------------------------------------------------------
# Inter prediction calls
# ---------------------------------------------------------------------------

INTER_DTYPE = np.dtype([("x", np.uint16), ("y", np.uint16), ("w", np.uint16), ("h", np.uint16),
                        ("plane", np.uint8), ("kind", np.uint8), ("motion_mode", np.uint8),
                        ("filter_x", np.uint8), ("filter_y", np.uint8), ("ref", np.uint8, (2,)),
                        ("compound_type", np.uint8), ("mv", np.int16, (2, 2)), ("mi_size", np.uint8),
                        ("wedge_index", np.uint8), ("wedge_sign", np.uint8), ("mask_type", np.uint8),
                        ("interintra_mode", np.uint8), ("wedge_interintra", np.uint8), ("fwd_weight", np.uint8),
                        ("bck_weight", np.uint8), ("warp", np.int32), ("obmc_first", np.uint32),
                        ("obmc_above", np.uint8), ("obmc_left", np.uint8), ("avail_u", np.uint8),
                        ("avail_l", np.uint8), ("plane_residual_ge_8x8", np.uint8), ("mi_width_log2", np.uint8),
                        ("mi_height_log2", np.uint8), ("pad", np.uint8), ("mi_row", np.uint16),
                        ("mi_col", np.uint16)], align=True)
assert INTER_DTYPE.itemsize == C.sizeof(abi.InterPred)
NB_DTYPE = np.dtype([("mv", np.int16, (2,)), ("axis_pos4", np.uint16), ("ref", np.uint8), ("step4", np.uint8),
                     ("filter_x", np.uint8), ("filter_y", np.uint8), ("pad", np.uint8, (2,))], align=True)
assert NB_DTYPE.itemsize == C.sizeof(abi.ObmcNeighbour)
WARP_DTYPE = np.dtype([("gm_params", np.int32, (2, 6)), ("local_warp_params", np.int32, (6,)),
                       ("y_mode", np.uint8, (2,)), ("gm_type", np.uint8, (2,)), ("local_valid", np.uint8),
                       ("ref_is_scaled", np.uint8, (2,)), ("force_integer_mv", np.uint8)], align=True)
assert WARP_DTYPE.itemsize == C.sizeof(abi.WarpCtx)

BLOCK_W = [4, 4, 8, 8, 8, 16, 16, 16, 32, 32, 32, 64, 64, 64, 128, 128, 4, 16, 8, 32, 16, 64]
BLOCK_H = [4, 8, 4, 8, 16, 8, 16, 32, 16, 32, 64, 32, 64, 128, 64, 128, 16, 4, 32, 8, 64, 16]
WEDGE_OK = {3, 4, 5, 6, 7, 8, 9, 18, 19}        # blocks with WEDGE_BITS > 0
DIST_WEIGHTS = [(9, 7), (11, 5), (12, 4), (13, 3), (7, 9), (5, 11), (4, 12), (3, 13)]
SUBSAMPLED = None


class InterFrame(ReconFrame):
    """CurrFrame planes on entry, the 7 references and the predict_inter calls."""

    def __init__(self):
        super().__init__()
        self.refs = []
        self.preds = None
        self.neighbours = None
        self.warps = None


def _warp_params(rng, valid=True, tx=0, ty=0):
    spread = 1500 if valid else 30000
    a, b, c, d = (int(v) for v in rng.integers(-spread, spread + 1, size=4))
    return [int(tx * 65536 + rng.integers(-20000, 20000)), int(ty * 65536 + rng.integers(-20000, 20000)),
            65536 + a, b, c, 65536 + d]


def _subsampled(mi_size, ssx, ssy):
    global SUBSAMPLED
    if SUBSAMPLED is None:
        from . import tables
        SUBSAMPLED = tables.SUBSAMPLED_SIZE
    return int(SUBSAMPLED[mi_size][ssx][ssy])


def make_inter_frame(seed, width=176, height=144, bit_depth=8, ssx=1, ssy=1, mono=False, scaled=True,
                     sb_size=64, overhang=True, p_intra=0.12, ref_dims=None, p_ii=0.10):
    """A frame of inter blocks over a random partition: single, compound
    (average / distance / wedge / difference weight), inter-intra (smooth and
    wedge), OBMC with neighbour lists walked like obmc_dispatch_leaf
    (src/inter_pred.rs:6519), local and global warp; references of other sizes
    (2x, 1/2, 1.5x and a 3x one past the spec's 2x limit) when `scaled`."""
    rng = np.random.default_rng(seed)
    f = InterFrame()
    h = f.hdr
    h.frame_width = h.upscaled_width = width
    h.frame_height = height
    h.mi_cols, h.mi_rows = 2 * ((width + 7) >> 3), 2 * ((height + 7) >> 3)
    h.bit_depth = bit_depth
    h.num_planes = 1 if mono else 3
    h.subsampling_x, h.subsampling_y = (1, 1) if mono else (ssx, ssy)
    maxv = (1 << bit_depth) - 1
    dt = np.uint8 if bit_depth == 8 else np.uint16
    if ref_dims is None:
        ref_dims = [(width, height)] * 7
        if scaled:
            ref_dims[3] = (2 * width, 2 * height)
            ref_dims[4] = ((width + 1) // 2, (height + 1) // 2)
            ref_dims[5] = (width * 3 // 2 + 3, height * 3 // 2 - 1)
            ref_dims[6] = (3 * width, 3 * height)
    for r in range(7):
        uw, rh = ref_dims[r]
        planes = []
        for p in range(3):
            sx_, sy_ = (h.subsampling_x, h.subsampling_y) if p else (0, 0)
            if p < h.num_planes:
                planes.append(_plane(rng, (rh + sy_) >> sy_, (uw + sx_) >> sx_, bit_depth))
            else:
                planes.append(np.zeros((1, 1), dt))
        f.refs.append({"planes": planes, "upscaled_width": uw, "frame_height": rh})
    f.planes = [rng.integers(0, maxv + 1, size=f.plane_dims(p)).astype(dt) for p in range(h.num_planes)]
    scaled_ref = [ref_dims[r] != (width, height) for r in range(7)]

    pw, ph = h.mi_cols * 4, h.mi_rows * 4
    blocks = []
    ext = 16 if overhang else 0   # edge blocks may run past the plane (the write is clipped)
    for sby in range(0, ph, sb_size):
        for sbx in range(0, pw, sb_size):
            if overhang and sb_size == 128 and rng.random() < 0.3 and sbx + 128 <= pw + 64:
                blocks.append((sbx, sby, 128, 128))
                continue
            _blocks(rng, sbx, sby, sb_size, pw + ext, ph + ext, blocks)
    blocks = [b for b in blocks if b[0] < pw and b[1] < ph]
    mi_map = -np.ones((h.mi_rows, h.mi_cols), np.int64)
    info = []
    for bi, (x0, y0, bw, bh) in enumerate(blocks):
        mi_size = BLOCK_OF[(bw // 4, bh // 4)]
        intra = rng.random() < p_intra
        mvs = rng.integers(-160, 161, size=(2, 2))
        if rng.random() < 0.1:
            mvs = rng.integers(-2400, 2401, size=(2, 2))   # far outside the reference
        info.append({"mi_size": mi_size, "intra": intra, "ref": [int(rng.integers(0, 7)), int(rng.integers(0, 7))],
                     "mv": mvs, "fx": int(rng.integers(0, 4)), "fy": int(rng.integers(0, 4))})
        if rng.random() < 0.03:
            info[-1]["fx"] = int(rng.integers(4, 6))
        r0, c0 = y0 // 4, x0 // 4
        mi_map[r0:r0 + bh // 4, c0:c0 + bw // 4] = bi

    preds, nbs, warps = [], [], []
    f.intra_blocks = [blk for bi, blk in enumerate(blocks) if info[bi]["intra"]]
    f.block_list = list(blocks)                                  # decode order
    f.block_intra = [bool(info[bi]["intra"]) for bi in range(len(blocks))]
    pred_block = []                                              # block of each call
    for bi, (x0, y0, bw, bh) in enumerate(blocks):
        b = info[bi]
        if b["intra"]:
            continue
        mi_size, mi_row, mi_col = b["mi_size"], y0 // 4, x0 // 4
        big = min(bw, bh) >= 8
        r = rng.random()
        kind, ctype, mmode, ii_mode, wii = abi.INTER_SINGLE, 2, 0, 0, 0
        warp = -1
        if big and r < 0.35:
            kind = abi.INTER_COMPOUND
            choices = [2, 4, 1] + ([0] if mi_size in WEDGE_OK else [])
            ctype = int(rng.choice(choices))
        elif big and r < 0.35 + p_ii and bw <= 32 and bh <= 32:
            kind = abi.INTER_INTRA
            ii_mode = int(rng.integers(0, 4))
            wii = int(mi_size in WEDGE_OK and rng.random() < 0.5)
        elif big and r < 0.65:
            mmode = 1
        elif big and r < 0.78:
            mmode = 2
        w = {}
        if mmode == 2 or (big and rng.random() < 0.25):
            wc = np.zeros((), WARP_DTYPE)
            glob = rng.random() < 0.6
            wc["y_mode"][:] = (24 if kind == abi.INTER_COMPOUND else 16) if glob else 13
            wc["gm_type"][:] = rng.integers(1, 4, size=2)
            for l in range(2):
                wc["gm_params"][l] = _warp_params(rng, rng.random() < 0.9, b["mv"][l][1] / 8, b["mv"][l][0] / 8)
            wc["local_warp_params"] = _warp_params(rng, rng.random() < 0.85, b["mv"][0][1] / 8, b["mv"][0][0] / 8)
            wc["local_valid"] = int(rng.random() < 0.9)
            wc["ref_is_scaled"] = [scaled_ref[b["ref"][0]], scaled_ref[b["ref"][1]]]
            wc["force_integer_mv"] = int(rng.random() < 0.05)
            warp = len(warps)
            warps.append(wc)
        obmc_first, n_above, n_left = len(nbs), 0, 0
        avail_u, avail_l = int(mi_row > 0), int(mi_col > 0)
        if mmode == 1:
            w4, h4 = bw // 4, bh // 4
            wl2, hl2 = w4.bit_length() - 1, h4.bit_length() - 1
            if avail_u:
                x4, n = mi_col, 0
                while n < min(4, wl2) and x4 < min(h.mi_cols, mi_col + w4):
                    cc = min(x4 | 1, h.mi_cols - 1)
                    cand = mi_map[mi_row - 1, cc]
                    ci = info[cand]
                    step4 = min(max(BLOCK_W[ci["mi_size"]] // 4, 2), 16)
                    if not ci["intra"]:
                        n += 1
                        nbs.append((ci["mv"][0], x4, ci["ref"][0], step4, ci["fx"], ci["fy"]))
                        n_above += 1
                    x4 += step4
            if avail_l:
                y4, n = mi_row, 0
                while n < min(4, hl2) and y4 < min(h.mi_rows, mi_row + h4):
                    cr = min(y4 | 1, h.mi_rows - 1)
                    cand = mi_map[cr, mi_col - 1]
                    ci = info[cand]
                    step4 = min(max(BLOCK_H[ci["mi_size"]] // 4, 2), 16)
                    if not ci["intra"]:
                        n += 1
                        nbs.append((ci["mv"][0], y4, ci["ref"][0], step4, ci["fx"], ci["fy"]))
                        n_left += 1
                    y4 += step4
        wedge_index, wedge_sign = int(rng.integers(0, 16)), int(rng.integers(0, 2))
        mask_type = int(rng.integers(0, 2))
        fwd, bck = DIST_WEIGHTS[int(rng.integers(0, len(DIST_WEIGHTS)))]
        for p in range(h.num_planes):
            sx_, sy_ = (h.subsampling_x, h.subsampling_y) if p else (0, 0)
            cw, chh = bw >> sx_, bh >> sy_
            if cw < 2 or chh < 2:
                continue
            ge8 = _subsampled(mi_size, sx_, sy_) >= 3
            pred_block.append(bi)
            preds.append(((x0 >> sx_), (y0 >> sy_), cw, chh, p, kind, mmode, b["fx"], b["fy"], b["ref"], ctype,
                          b["mv"], mi_size, wedge_index, wedge_sign, mask_type, ii_mode, wii, fwd, bck, warp,
                          obmc_first, n_above, n_left, avail_u, avail_l, int(ge8), (bw // 4).bit_length() - 1,
                          (bh // 4).bit_length() - 1, 0, mi_row, mi_col))
    f.preds = np.zeros(len(preds), INTER_DTYPE)
    for i, t in enumerate(preds):
        f.preds[i] = t
    f.pred_block = np.array(pred_block, np.int64)
    f.neighbours = np.zeros(len(nbs), NB_DTYPE)
    for i, (mv, pos, ref, step4, fx, fy) in enumerate(nbs):
        f.neighbours[i] = (mv, pos, ref, step4, fx, fy, (0, 0))
    f.warps = np.array(warps, WARP_DTYPE) if warps else np.zeros(0, WARP_DTYPE)
    return f


def custom_inter_frame(width, height, refs, calls, neighbours=(), warps=(), bit_depth=8, ssx=1, ssy=1,
                       mono=True, fill=0):
    """A hand-built inter frame: refs = list of (upscaled_width, frame_height,
    [plane arrays]) (padded to 7 with copies of the first), calls = dicts of
    av1g_inter_pred fields (missing ones zero, warp -1)."""
    f = InterFrame()
    h = f.hdr
    h.frame_width = h.upscaled_width = width
    h.frame_height = height
    h.mi_cols, h.mi_rows = 2 * ((width + 7) >> 3), 2 * ((height + 7) >> 3)
    h.bit_depth = bit_depth
    h.num_planes = 1 if mono else 3
    h.subsampling_x, h.subsampling_y = (1, 1) if mono else (ssx, ssy)
    dt = np.uint8 if bit_depth == 8 else np.uint16
    refs = list(refs) + [refs[0]] * (7 - len(refs))
    for uw, rh, planes in refs:
        ps = [np.asarray(p, dt) for p in planes] + [np.zeros((1, 1), dt)] * (3 - len(planes))
        f.refs.append({"planes": ps, "upscaled_width": uw, "frame_height": rh})
    f.planes = [np.full(f.plane_dims(p), fill, dt) for p in range(h.num_planes)]
    f.preds = np.zeros(len(calls), INTER_DTYPE)
    for i, c in enumerate(calls):
        f.preds[i]["warp"] = -1
        for k, v in c.items():
            f.preds[i][k] = v
    f.neighbours = np.zeros(len(neighbours), NB_DTYPE)
    for i, c in enumerate(neighbours):
        for k, v in c.items():
            f.neighbours[i][k] = v
    f.warps = np.zeros(len(warps), WARP_DTYPE)
    for i, c in enumerate(warps):
        for k, v in c.items():
            f.warps[i][k] = v
    return f



# ---------------------------------------------------------------------------
# Streams of whole frames for the serving engine
# ---------------------------------------------------------------------------

class StreamFrame:
    """One av1g_frame_desc: header, quantizer, post-filter side data, the
    prediction and residual lists, and the reference / refresh / show fields."""

    def __init__(self):
        self.hdr = None
        self.quant = None
        self.grid = None
        self.cdef_idx = None
        self.lr_units = [None, None, None]
        self.preds = self.neighbours = self.warps = None
        self.inter_tus = self.intra_tus = None
        self.palette_maps = None
        self.coeffs = None
        self.ref_frame_idx = [0] * 7
        self.refresh = 0
        self.show = 1
        self.show_existing = 0
        self.show_idx = 0


def _intra_tus_for_blocks(rng, h, quant, blocks, sb_size, coeff_base):
    """Intra TUs (modes, residuals) for the intra blocks of an inter frame, in
    decode order (superblocks in raster order, blocks in partition order,
    planes per block).  Above-right / below-left stay off so that every edge
    sample read was decoded earlier in block order."""
    tus, coeffs, off = [], [], coeff_base
    ok_segs = [s for s in range(8) if not quant.lossless[s]]
    sbs = {}
    for b in blocks:
        sbs.setdefault((b[1] // sb_size, b[0] // sb_size), []).append(b)
    for key in sorted(sbs):
        for (x0, y0, bw, bh) in sbs[key]:
            for p in range(h.num_planes):
                sx_, sy_ = (h.subsampling_x, h.subsampling_y) if p else (0, 0)
                bx, by, w, hh = x0 >> sx_, y0 >> sy_, bw >> sx_, bh >> sy_
                if w < 4 or hh < 4:
                    continue
                tw, th = min(w, 32), min(hh, 32)
                if (tw, th) not in TX_OF:
                    tw = th = min(tw, th)
                tx = TX_OF[(tw, th)]
                mode = int(rng.integers(0, 13))
                ad = int(rng.integers(-3, 4)) if 1 <= mode <= 8 else 0
                pw = (h.mi_cols * 4) >> sx_
                ph = (h.mi_rows * 4) >> sy_
                for ty in range(by, by + hh, th):
                    for tx_ in range(bx, bx + w, tw):
                        if ty >= ph or tx_ >= pw:
                            continue
                        flags = abi.INTRA_EDGE_FILTER
                        if ty > 0:
                            flags |= abi.INTRA_HAVE_ABOVE
                        if tx_ > 0:
                            flags |= abi.INTRA_HAVE_LEFT
                        res = (tx_, ty, p, tx, 0, 0, 0, (0, 0, 0), 0)
                        if ok_segs and rng.random() < 0.7:
                            seg = int(rng.choice(ok_segs))
                            flags |= abi.INTRA_RESIDUAL
                            lv = _levels(rng, min(32, tw), min(32, th), False)
                            res = (tx_, ty, p, tx, _tx_type_for(rng, tw, th), seg, int(rng.integers(1, 256)),
                                   (0, 0, 0), off)
                            coeffs.append(lv)
                            off += len(lv)
                        tus.append((tx_, ty, p, tx, mode, flags, ad, 0, 255, 0, 0, 0, res, (0, 0), 0, 0, 0, 0,
                                    [0] * 8, 0, 0, 0, 0))
    return np.array(tus, dtype=INTRA_TU_DTYPE) if tus else np.zeros(0, INTRA_TU_DTYPE), coeffs


def make_stream(seed, n_frames=4, width=176, height=144, bit_depth=8, ssx=1, ssy=1, mono=False, superres_denom=8,
                film_grain=False, sb_size=64, show_existing_at=(), palette=0.1, tiles=(0, 0)):
    """A key frame (intra TUs, palette blocks) then inter frames (inter calls
    over a random partition with some intra blocks, residual TUs), each with
    the post-filter side data of make_frame, random references among the
    eight slots and random refresh flags.  Frames listed in show_existing_at
    are show_existing_frame outputs of a random slot instead.  tiles: the
    key frame's tile grid (make_intra_frame)."""
    rng = np.random.default_rng(seed)
    frames = []
    for k in range(n_frames):
        fs = seed * 1000 + k
        if k in show_existing_at:
            fr = StreamFrame()
            fr.hdr = frames[0].hdr
            fr.show_existing = 1
            fr.show_idx = int(rng.integers(0, 8))
            fr.refresh = 0
            frames.append(fr)
            continue
        base = make_frame(fs, width, height, bit_depth, ssx, ssy, mono, superres_denom, film_grain)
        h = base.hdr
        fw = h.frame_width
        fr = StreamFrame()
        fr.hdr, fr.grid, fr.cdef_idx, fr.lr_units = h, base.grid, base.cdef_idx, base.lr_units
        if k == 0:
            it = make_intra_frame(fs, fw, height, bit_depth, ssx, ssy, mono, sb_size, palette=palette, tiles=tiles)
            fr.quant, fr.intra_tus, fr.coeffs, fr.palette_maps = it.quant, it.tus, it.coeffs, it.palette_maps
            fr.refresh = 0xFF
        else:
            inter = make_inter_frame(fs, fw, height, bit_depth, ssx, ssy, mono, scaled=False, sb_size=sb_size,
                                     p_intra=0.1, ref_dims=[(h.upscaled_width, height)] * 7)
            fr.preds, fr.neighbours, fr.warps = inter.preds, inter.neighbours, inter.warps
            rec = make_recon_frame(fs + 500, fw, height, bit_depth, ssx, ssy, mono)
            fr.quant, fr.inter_tus = rec.quant, rec.tus
            # intra TUs in decode order: intra blocks, and the intra halves
            # (+ residuals) of inter-intra blocks
            parts, icoeffs, off = [], [], len(rec.coeffs)
            ii_calls = np.nonzero(inter.preds["kind"] == abi.INTER_INTRA)[0]
            for bi, blk in enumerate(inter.block_list):
                if inter.block_intra[bi]:
                    t, c = _intra_tus_for_blocks(rng, h, rec.quant, [blk], sb_size, off)
                else:
                    calls = ii_calls[inter.pred_block[ii_calls] == bi]
                    if not len(calls):
                        continue
                    t, c = interintra_tus(inter, 0, rec.quant, off, calls=calls, rng=rng)
                parts.append(t)
                icoeffs += c
                off += sum(len(x) for x in c)
            fr.intra_tus = np.concatenate(parts) if parts else np.zeros(0, INTRA_TU_DTYPE)
            fr.coeffs = np.concatenate([rec.coeffs] + icoeffs).astype(np.int32)
            fr.ref_frame_idx = [int(v) for v in rng.integers(0, 8, size=7)]
            fr.refresh = int(rng.integers(0, 256)) & int(rng.integers(0, 256))
        frames.append(fr)
    return frames


def with_film_grain(frames, seed):
    """The same stream with film grain on every frame: each frame a shallow
    copy sharing the descriptors, with its own header carrying seeded grain
    parameters (a new grain_seed per frame)."""
    import copy
    rng = np.random.default_rng(seed)
    out = []
    for fr in frames:
        g = copy.copy(fr)
        h = abi.FrameHeader()
        C.memmove(C.addressof(h), C.addressof(fr.hdr), C.sizeof(h))
        _film_grain(rng, h.film_grain, h.bit_depth, h.num_planes == 1)
        g.hdr = h
        out.append(g)
    return out


def stream_seq(frames, sb_size=64):
    h = frames[0].hdr
    return {"max_width": h.upscaled_width, "max_height": h.frame_height, "bit_depth": h.bit_depth,
            "subsampling_x": h.subsampling_x, "subsampling_y": h.subsampling_y, "num_planes": h.num_planes,
            "sb_size": sb_size}



II_TO_INTRA = [0, 1, 2, 9]   # II_DC/V/H/SMOOTH -> DC_PRED, V_PRED, H_PRED, SMOOTH_PRED


def interintra_tus(f, seed, quant=None, coeff_base=0, calls=None, rng=None):
    """For each inter-intra call of an InterFrame (or of the call indices
    `calls`), in list order (block decode order), the TU of its intra half
    (the block's intra prediction blended with the inter half) and a residual
    TU over the block.  Returns (tus, coeffs)."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    h = f.hdr
    q = quant if quant is not None else f.quant
    ok_segs = [s_ for s_ in range(8) if not q.lossless[s_]]
    tus, coeffs, off = [], [], coeff_base
    for d in (f.preds if calls is None else f.preds[calls]):
        if d["kind"] != abi.INTER_INTRA:
            continue
        x, y, w, hh, p = int(d["x"]), int(d["y"]), int(d["w"]), int(d["h"]), int(d["plane"])
        if (w, hh) not in TX_OF:
            continue
        tx = TX_OF[(w, hh)]
        flags = abi.INTRA_EDGE_FILTER
        if y > 0:
            flags |= abi.INTRA_HAVE_ABOVE
        if x > 0:
            flags |= abi.INTRA_HAVE_LEFT
        iim = int(d["interintra_mode"])
        kind = 2 if d["wedge_interintra"] else 1
        none_res = (x, y, p, tx, 0, 0, 0, (0, 0, 0), 0)
        tus.append((x, y, p, tx, II_TO_INTRA[iim], flags, 0, 0, 255, 0, 0, 0, none_res, (0, 0), 0, 0, 0, 0,
                    [0] * 8, kind, iim, int(d["wedge_index"]), int(d["mi_size"])))
        if ok_segs and rng.random() < 0.8:
            seg = int(rng.choice(ok_segs))
            lv = _levels(rng, min(32, w), min(32, hh), False)
            res = (x, y, p, tx, _tx_type_for(rng, w, hh), seg, int(rng.integers(1, 256)), (0, 0, 0), off)
            coeffs.append(lv)
            off += len(lv)
            tus.append((x, y, p, tx, abi.INTRA_MODE_NONE, abi.INTRA_RESIDUAL, 0, 0, 255, 0, 0, 0, res, (0, 0), 0,
                        0, 0, 0, [0] * 8, 0, 0, 0, 0))
    arr = np.array(tus, dtype=INTRA_TU_DTYPE) if tus else np.zeros(0, INTRA_TU_DTYPE)
    return arr, coeffs


def _mf_mvs(rng, shape, far=0.25):
    """MV components: mostly short (they project inside the §7.9.4 window),
    a share long enough to leave it, a few beyond the storage limit."""
    near = rng.integers(-160, 161, shape)
    long_ = rng.integers(-4095, 4096, shape)
    huge = rng.integers(-16384, 16385, shape)
    pick = rng.random(shape)
    return np.where(pick < 1 - far, near, np.where(pick < 1 - far / 8, long_, huge)).astype(np.int16)


def make_mf_store_inputs(seed, mi_rows, mi_cols, hint_bits=7, is_inter=True):
    """One frame's §7.19 storage inputs: per-cell RefFrames[2] in -1..7 and
    Mvs[2][2], with the order hints of the frame and of its seven references
    (some past, some future).  Returns a dict of the av1g_mf_store_job fields
    with host arrays."""
    rng = np.random.default_rng(seed)
    cells = mi_rows * mi_cols
    period = 1 << hint_bits if hint_bits else 256
    cur = int(rng.integers(0, period))
    ref_hints = [int((cur + d) % period) for d in rng.integers(-8, 9, 7)]
    refs = rng.choice(np.array([-1, 0, 1, 2, 3, 4, 5, 6, 7]), size=(cells, 2)).astype(np.int8)
    return dict(mi_rows=mi_rows, mi_cols=mi_cols, is_inter=is_inter, order_hint=cur, hint_bits=hint_bits,
                ref_order_hint=ref_hints, ref_frames=refs, mvs=_mf_mvs(rng, (cells, 2, 2)))


def make_mf_scene(seed, mi_rows, mi_cols, hint_bits=7, empty=(), intra=(), mismatched=(), fill=0.7):
    """The §7.9 projection inputs of one frame: eight stored slots (MfMvs,
    MfRefFrames, SavedOrderHints, extent, FrameIsIntra), ref_frame_idx,
    OrderHints, OrderHint and OrderHintBits.  Slots in `empty` are absent,
    those in `intra` are intra frames, those in `mismatched` have another mi
    extent.  Stored frames lie up to 7 order hints before or after the
    current frame and their own references up to 8 before them (a few after,
    which the projection rejects)."""
    rng = np.random.default_rng(seed)
    period = 1 << hint_bits if hint_bits else 256
    cur = int(rng.integers(0, period))
    slot_hints = [int((cur + d) % period) for d in rng.choice([-7, -5, -3, -2, -1, 1, 2, 3, 4, 6], 8)]
    slots = []
    for s in range(8):
        if s in empty:
            slots.append(None)
            continue
        rows, cols = (mi_rows + 2, mi_cols) if s in mismatched else (mi_rows, mi_cols)
        cells = rows * cols
        h = slot_hints[s]
        saved = [h] + [int((h - d) % period) for d in rng.choice([1, 2, 3, 4, 5, 8, -2], 7)]
        refs = np.where(rng.random(cells) < fill, rng.integers(1, 8, cells), -1).astype(np.int8)
        mvs = _mf_mvs(rng, (cells, 2), far=0.15)
        mvs[refs < 0] = 0
        slots.append(dict(mf_mvs=mvs, mf_ref_frames=refs, saved_order_hints=saved, mi_rows=rows, mi_cols=cols,
                          frame_is_intra=s in intra))
    ref_frame_idx = [int(v) for v in rng.integers(0, 8, 7)]
    order_hints = [0] + [slot_hints[ref_frame_idx[i]] for i in range(7)]
    return dict(slots=slots, ref_frame_idx=ref_frame_idx, order_hints=order_hints, order_hint=cur,
                hint_bits=hint_bits, mi_rows=mi_rows, mi_cols=mi_cols)
