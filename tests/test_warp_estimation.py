"""The §7.11.3.8 local warp fit (av1g_warp_estimation, a host entry point of
the library) against the oracle and the reference's unit tests."""
import numpy as np
import pytest

import oracle
from oxideav_av1_b200 import abi


def test_pins_from_reference_tests():
    abi.load()
    # r192_warp_estimation_empty_cands_is_invalid
    assert abi.warp_estimation([], 0, 0, 4, 4, 0, 0)[0] is False
    assert oracle.warp_estimation([], 0, 0, 4, 4, 0, 0)[0] is False
    # r192_warp_estimation_single_cand_is_invalid (det = 48: valid)
    assert abi.warp_estimation([(0, 0, 0, 0)], 0, 0, 4, 4, 0, 0)[0] is True
    assert oracle.warp_estimation([(0, 0, 0, 0)], 0, 0, 4, 4, 0, 0)[0] is True


def test_pure_translation_fits_identity_shear():
    # neighbours moving with the block's own mv: the fitted matrix is close to
    # the identity (the fit's rounding bias terms keep it from being exact)
    mv = (-24, 40)
    cands = []
    for (r, c) in [(-4, 4), (4, -4), (-4, 20), (20, -4), (-4, 12)]:
        sy, sx = (64 + r) * 8, (128 + c) * 8
        cands.append((sy, sx, sy + mv[0], sx + mv[1]))
    ok, p = abi.warp_estimation(cands, 16, 32, 4, 4, *mv)
    assert ok and abs(p[2] - 65536) < 64 and abs(p[5] - 65536) < 64 and abs(p[3]) < 64 and abs(p[4]) < 64
    assert (ok, p) == tuple(oracle.warp_estimation(cands, 16, 32, 4, 4, *mv))


@pytest.mark.parametrize("seed", range(6))
def test_matches_oracle_on_random_samples(seed):
    abi.load()
    rng = np.random.default_rng(seed)
    for _ in range(300):
        n = int(rng.integers(0, 10))
        mi_row, mi_col = int(rng.integers(0, 300)), int(rng.integers(0, 500))
        bw4, bh4 = (int(v) for v in rng.choice([1, 2, 4, 8, 16, 32], size=2))
        mv = [int(v) for v in rng.integers(-600, 600, size=2)]
        my, mx = (mi_row * 4 + bh4 * 2 - 1) * 8, (mi_col * 4 + bw4 * 2 - 1) * 8
        spread = int(rng.choice([8, 64, 400, 1 << 20]))
        cands = []
        for _ in range(n):
            sy, sx = my + int(rng.integers(-spread, spread)), mx + int(rng.integers(-spread, spread))
            j = int(rng.choice([4, 64, 300]))
            cands.append((sy, sx, sy + mv[0] + int(rng.integers(-j, j)), sx + mv[1] + int(rng.integers(-j, j))))
        if rng.random() < 0.05:
            cands = [(2 ** 31 - 1, -2 ** 31, -2 ** 31, 2 ** 31 - 1)] * max(n, 1)
        got = abi.warp_estimation(cands, mi_row, mi_col, bw4, bh4, *mv)
        want = oracle.warp_estimation(cands, mi_row, mi_col, bw4, bh4, *mv)
        assert got == (want[0], want[1] if want[0] else [0] * 6), (cands, mi_row, mi_col, bw4, bh4, mv)
