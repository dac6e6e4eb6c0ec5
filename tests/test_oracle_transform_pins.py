"""Pin the oracle's dequant / inverse transform to the reference's unit tests
(src/transform.rs tests, src/qmatrix.rs tests, src/cdf.rs dequant helpers)."""
import numpy as np
import pytest

import oracle
from oxideav_av1_b200 import abi, tables

TX_4X4, TX_8X8, TX_16X16, TX_32X32, TX_64X64, TX_4X8 = 0, 1, 2, 3, 4, 5
DCT_DCT, ADST_ADST, FLIPADST_FLIPADST, IDTX = 0, 3, 6, 9


def _dc(tx, value):
    w = [4, 8, 16, 32, 64, 4][tx]
    h = [4, 8, 16, 32, 64, 8][tx]
    d = np.zeros((h, w), np.int64)
    d[0, 0] = value
    return d


def test_dct_dct_4x4_dc_only_is_flat_128():
    assert (oracle.inverse_transform(_dc(TX_4X4, 4096), TX_4X4, DCT_DCT, 8) == 128).all()


def test_idtx_4x4_dc_only():
    r = oracle.inverse_transform(_dc(TX_4X4, 4096), TX_4X4, IDTX, 8)
    exp = np.zeros((4, 4), np.int64)
    exp[0, 0] = 512
    assert (r == exp).all()


@pytest.mark.parametrize("tx,tt", [(TX_4X4, DCT_DCT), (TX_4X8, DCT_DCT), (TX_8X8, DCT_DCT),
                                   (TX_16X16, ADST_ADST), (TX_32X32, DCT_DCT), (TX_64X64, DCT_DCT),
                                   (TX_8X8, FLIPADST_FLIPADST)] + [(TX_8X8, t) for t in (10, 11, 12, 13, 14, 15)])
def test_zero_in_zero_out(tx, tt):
    assert not oracle.inverse_transform(_dc(tx, 0), tx, tt, 8).any()


def test_lossless_zero_in_zero_out():
    assert not oracle.inverse_transform(_dc(TX_4X4, 0), TX_4X4, DCT_DCT, 8, lossless=True).any()


def test_cos128_anchor_points():
    c = tables.COS128_LOOKUP
    assert c[0] == 4096 and c[64] == 0 and c[32] == 2896


def test_qmatrix_first_row_level0_luma_4x4():
    # src/qmatrix.rs tests: the first TX_4X4 luma row at level 0
    assert list(tables.QUANTIZER_MATRIX[0][0][:4]) == [32, 43, 73, 97]


def test_dequant_dc_ac_and_denominator():
    q = abi.QuantParams()
    q.base_q_idx = 100
    for s in range(8):
        for p in range(3):
            q.seg_qm_level[p][s] = 15
    lv = np.zeros(16, np.int32)
    lv[0], lv[1] = 3, -2
    d = oracle.dequantize(q, 8, lv, TX_4X4, 0, 0, 100, DCT_DCT)
    assert d[0, 0] == 3 * tables.DC_QLOOKUP[0][100]
    assert d[0, 1] == -2 * tables.AC_QLOOKUP[0][100]
    # TX_32X32 divides by 2 with truncation toward zero
    lv32 = np.zeros(32 * 32, np.int32)
    lv32[1] = -1
    d32 = oracle.dequantize(q, 8, lv32, TX_32X32, 0, 0, 100, DCT_DCT)
    assert d32[0, 1] == -(tables.AC_QLOOKUP[0][100] // 2)


def test_dequant_clamps_to_bitdepth_range():
    q = abi.QuantParams()
    q.base_q_idx = 255
    for s in range(8):
        for p in range(3):
            q.seg_qm_level[p][s] = 15
    lv = np.zeros(16, np.int32)
    lv[0] = 100000
    d = oracle.dequantize(q, 8, lv, TX_4X4, 0, 0, 255, DCT_DCT)
    assert d[0, 0] == (1 << 15) - 1
