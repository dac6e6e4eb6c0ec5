"""Large-scale-tile output assembly on the device against the oracle, bit-exact.

Each tile list entry is a camera tile decoded independently against its
anchor frame (the §7.3.2 camera-tile decode: inter prediction from the anchor
as reference, then residuals); the entries of all lists are decoded together
by av1g_run_inter / av1g_run_recon as one batch, and av1g_run_tile_list_output
places the tiles in the output frames (decode_tile_list,
src/tile_list.rs:651-740).  Cases after the reference's large_scale_tile.rs:
a 2x2 assembly, repeated anchors with partial coverage (uncovered output
tiles stay zero), a wide camera frame, 10-bit, 4:4:4, monochrome, and a batch
of several lists in one launch.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
from oxideav_av1_b200 import abi, postfilter, synth  # noqa: E402

pytestmark = pytest.mark.gpu


def _camera_tiles(seed, n, cam_w, cam_h, anchors, bit_depth, ssx, ssy, mono, with_residual):
    """n camera frames, each an inter frame predicted from one anchor (all
    seven references are that anchor), with residuals when asked."""
    out = []
    for k in range(n):
        a = anchors[k % len(anchors)]
        f = synth.make_inter_frame(seed + k, cam_w, cam_h, bit_depth=bit_depth, ssx=ssx, ssy=ssy, mono=mono,
                                   scaled=False, p_intra=0.0, p_ii=0.0)
        planes = list(a) + [np.zeros((1, 1), a[0].dtype)] * (3 - len(a))  # monochrome: unused chroma
        f.refs = [{"planes": planes, "upscaled_width": cam_w, "frame_height": cam_h} for _ in range(7)]
        out.append(f)
    recon = None
    if with_residual:
        recon = [synth.make_recon_frame(seed + 100 + k, cam_w, cam_h, bit_depth=bit_depth, ssx=ssx, ssy=ssy,
                                        mono=mono) for k in range(n)]
    return out, recon


def _oracle_tiles(frames, recon):
    tiles = []
    for k, f in enumerate(frames):
        planes, rc = oracle.inter(f)
        assert rc == 0
        if recon is not None:
            r = recon[k]
            r.planes = planes
            planes = oracle.recon(r)
        tiles.append(planes)
    return tiles


class _List:
    def __init__(self, tile_w, tile_h, wt, ht, frames, recon, origins, bit_depth, ssx, ssy, np_):
        self.tile_w, self.tile_h, self.wt, self.ht = tile_w, tile_h, wt, ht
        self.frames, self.recon, self.origins = frames, recon, origins
        self.bd, self.ssx, self.ssy, self.np = bit_depth, ssx, ssy, np_
        hbd = bit_depth > 8
        ow, oh = wt * tile_w, ht * tile_h
        self.out = [postfilter.DevPlane(oh if p == 0 else oh >> ssy, ow if p == 0 else ow >> ssx, hbd, "cuda")
                    for p in range(np_)]
        for pl in self.out:
            pl.t.fill_(0x5A)  # the kernel must write every output sample
        self.dev = [postfilter.DeviceInter(f) for f in frames]
        self.devr = None
        if recon is not None:
            self.devr = []
            for d, r in zip(self.dev, recon):
                dr = postfilter.DeviceRecon(r)
                dr.planes = d.planes  # residuals merge into the tile's CurrFrame
                self.devr.append(dr)

    def job(self):
        self.ents = (abi.TileListEntry * len(self.dev))()
        for k, d in enumerate(self.dev):
            for p in range(self.np):
                self.ents[k].src[p] = d.planes[p].cplane()
            self.ents[k].x0, self.ents[k].y0 = self.origins[k]
        j = abi.TileListJob(self.tile_w, self.tile_h, self.wt, self.ht, self.np, self.ssx, self.ssy, self.bd,
                            len(self.dev), 0, C.cast(self.ents, C.POINTER(abi.TileListEntry)))
        for p in range(self.np):
            j.out[p] = self.out[p].cplane()
        return j

    def expected(self):
        tiles = _oracle_tiles(self.frames, self.recon)
        return oracle.tile_list_output(self.tile_w, self.tile_h, self.wt, self.ht, self.ssx, self.ssy, self.bd,
                                       [(t, x0, y0) for t, (x0, y0) in zip(tiles, self.origins)])


def _anchors(seed, n, w, h, bit_depth, ssx, ssy, mono):
    rng = np.random.default_rng(seed)
    dt = np.uint8 if bit_depth == 8 else np.uint16
    out = []
    for _ in range(n):
        planes = [rng.integers(0, 1 << bit_depth, (h, w), dtype=np.int64).astype(dt)]
        if not mono:
            for _ in range(2):
                planes.append(rng.integers(0, 1 << bit_depth, (h >> ssy, w >> ssx), dtype=np.int64).astype(dt))
        out.append(planes)
    return out


CASES = [
    # (name, cam_w, cam_h, tile_w, tile_h, wt, ht, n_entries, bit_depth, ssx, ssy, mono, residual)
    ("2x2", 128, 128, 64, 64, 2, 2, 4, 8, 1, 1, False, True),
    ("partial_repeat", 128, 64, 64, 64, 2, 2, 3, 8, 1, 1, False, False),
    ("wide", 256, 64, 128, 64, 2, 1, 2, 8, 1, 1, False, True),
    ("10bit", 128, 128, 64, 64, 3, 1, 3, 10, 1, 1, False, True),
    ("444", 128, 64, 64, 64, 2, 2, 4, 8, 0, 0, False, False),
    ("mono", 128, 128, 64, 64, 1, 3, 2, 8, 1, 1, True, True),
]


def _make(case, seed):
    name, cw, ch, tw, th, wt, ht, n, bd, ssx, ssy, mono, res = case
    anchors = _anchors(seed, 3, cw, ch, bd, ssx, ssy, mono)
    frames, recon = _camera_tiles(seed * 10, n, cw, ch, anchors, bd, ssx, ssy, mono, res)
    rng = np.random.default_rng(seed)
    origins = [(int(rng.integers(0, cw // tw)) * tw, int(rng.integers(0, ch // th)) * th) for _ in range(n)]
    np_ = 1 if mono else 3
    return _List(tw, th, wt, ht, frames, recon, origins, bd, ssx, ssy, np_)


def _decode_and_assemble(lists):
    devs = [d for L in lists for d in L.dev]
    postfilter.run_inter(devs)
    recs = [d for L in lists if L.devr for d in L.devr]
    if recs:
        postfilter.run_recon(recs)
    arr = (abi.TileListJob * len(lists))(*[L.job() for L in lists])
    abi.check(abi.load().av1g_run_tile_list_output(arr, len(lists), None))
    torch.cuda.synchronize()


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_tile_list_output_matches_oracle(case):
    L = _make(case, 7)
    _decode_and_assemble([L])
    want = L.expected()
    for p, (pl, w) in enumerate(zip(L.out, want)):
        got = pl.download().astype(np.int64)
        assert got.shape == w.shape
        diff = np.argwhere(got != w)
        assert len(diff) == 0, f"plane {p}: {len(diff)} samples differ, first {tuple(diff[0])}"


def test_tile_lists_batched_in_one_launch():
    lists = [_make(c, 20 + i) for i, c in enumerate(CASES[:4])]
    _decode_and_assemble(lists)
    for L in lists:
        for pl, w in zip(L.out, L.expected()):
            assert np.array_equal(pl.download().astype(np.int64), w)


def test_tile_list_rejects_bad_jobs():
    lib = abi.load()
    L = _make(CASES[0], 3)
    j = L.job()
    bad = abi.TileListJob.from_buffer_copy(j)
    bad.num_entries = 5  # more entries than 2 x 2 output tiles
    assert lib.av1g_run_tile_list_output((abi.TileListJob * 1)(bad), 1, None) == abi.AV1G_EINVAL
    L.ents[1].x0 = 96  # tile reaches past the camera frame
    assert lib.av1g_run_tile_list_output((abi.TileListJob * 1)(j), 1, None) == abi.AV1G_EINVAL
