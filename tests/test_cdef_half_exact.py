"""CDEF's half-precision filter path gives the reference's integers exactly.

For 8- and 10-bit frames cdef_kernel filters two adjacent samples per thread
in packed half-precision registers (one instruction per pair of samples).
Every quantity on that path is an integer below 2048 or a value with few
enough significant bits that each operation is exact, except two additions
whose rounding is the integer rounding the reference asks for:

* samples are held as 1024 + v (v < 1024), so the bit pattern is 0x6400 | v
  and differences of two samples are the integer differences;
* floor(|d| / 2^adj) (constrain, cdef.rs:592-606): v1 = |d| * 2^-adj -
  (2^adj - 1) / 2^(adj+1) is exact (an odd numerator below 2^11 over a power
  of two), and v1 + 1536 rounds to 1536 + floor(|d| / 2^adj) because the
  fraction of v1 lies strictly inside (-1/2, 1/2) and the sum lands in
  [1024, 2048), where half precision holds exactly the integers; where the
  floor is 512 or more the sum may round to an even neighbour, but the
  threshold (at most 60) is then far below it and the result is 0 either way;
* (8 + sum - (sum < 0)) >> 4: sum / 16 + copysign(1/32, sum) is exact and never
  a half-integer, so its round-to-nearest after adding 1536 is the
  reference's rounding (half away from zero); the tap sums stay within
  12 x (15 + 4) << (bitDepth - 8) = 912 at 10 bits.

This restates the kernel's sequence of half-precision operations in numpy
(each operation computed exactly in float64 and rounded once to float16, as
the hardware does) and compares it with the integer arithmetic over every
difference, threshold and damping shift the syntax allows at 8 and 10 bits,
and every tap sum.  Unavailable taps (outside the plane) are NaN: the
maximum with zero maps them to a zero contribution, and the min / max of the
clip range ignore them.
"""
import numpy as np

H = np.float16


def _r(x):
    """One rounding to half precision of an exactly computed value."""
    return np.asarray(x, dtype=np.float64).astype(np.float16)


def _floor_log2(v):
    return np.where(v > 0, np.floor(np.log2(np.maximum(v, 1))).astype(np.int64), 0)


def _constrain_int(diff, thr, adj):
    ad = np.abs(diff)
    v = np.minimum(ad, np.maximum(thr - (ad >> adj), 0))
    return np.where(diff < 0, -v, v)


def _constrain_half(xb, xvb, thr, adj, nan_aware):
    """The kernel's sequence: xb, xvb are biased samples (1024 + v) or NaN."""
    d = _r(xb.astype(np.float64) - xvb.astype(np.float64))
    ad = np.abs(d)
    ka = np.float64(2.0) ** -adj
    ca = -(np.float64(2.0) ** adj - 1) / np.float64(2.0) ** (adj + 1)
    v1 = _r(ad.astype(np.float64) * ka + ca)
    assert np.all(np.isnan(v1) | (v1.astype(np.float64) == ad.astype(np.float64) * ka + ca)), "v1 inexact"
    v2 = _r(v1.astype(np.float64) + 1536.0)
    tb = H(1536 + thr) if np.isscalar(thr) else (1536 + thr).astype(np.float16)
    if nan_aware:
        m = np.fmax(_r(tb.astype(np.float64) - v2.astype(np.float64)), H(0))
    else:
        m = np.maximum(_r(tb.astype(np.float64) - v2.astype(np.float64)), H(0))
    c = np.fmin(ad, m)
    return np.where(np.signbit(d), -c, c)  # the sign bit of d copied onto c


def test_constrain_is_exact_for_every_difference_threshold_and_shift():
    for bd in (8, 10):
        cs = bd - 8
        hi = (1 << bd) - 1
        d = np.arange(-hi, hi + 1)
        xv = np.full_like(d, hi // 2)
        x = xv + d
        ok = (x >= 0) & (x <= hi)
        # the full difference range: centre at 0 and at the maximum as well
        xs = np.concatenate([x[ok], np.arange(0, hi + 1), np.arange(0, hi + 1)])
        xvs = np.concatenate([xv[ok], np.zeros(hi + 1, np.int64), np.full(hi + 1, hi)])
        diff = xs - xvs
        xb, xvb = (xs + 1024).astype(np.float16), (xvs + 1024).astype(np.float16)
        assert np.all(xb.astype(np.int64) == xs + 1024)
        for thr in range(1, (15 << cs) + 1):
            for damping in range(3 + cs - 1, 6 + cs + 1):  # chroma damping is one lower
                adj = max(damping - int(_floor_log2(np.array(thr))), 0)
                want = _constrain_int(diff, thr, adj)
                for nan_aware in (False, True):
                    got = _constrain_half(xb, xvb, thr, adj, nan_aware)
                    assert np.array_equal(got.astype(np.int64), want), (bd, thr, damping)


def test_unavailable_taps_contribute_nothing():
    xvb = (np.arange(0, 1024) + 1024).astype(np.float16)
    nan = np.full_like(xvb, np.nan)
    for thr in (1, 4, 15, 60):
        for adj in range(0, 9):
            got = _constrain_half(nan, xvb, thr, adj, True)
            assert np.all(got == 0)
    # and the clip range ignores them
    assert np.fmax(H(1030), H(np.nan)) == H(1030)
    assert np.fmin(H(np.nan), H(1030)) == H(1030)


def test_rounding_of_the_tap_sum_is_the_reference_rounding():
    for bd in (8, 10):
        cs = bd - 8
        lim = 12 * (15 + 4) << cs
        s = np.arange(-lim, lim + 1)
        want = (8 + s - (s < 0)) >> 4
        sh = s.astype(np.float16)
        assert np.all(sh.astype(np.int64) == s)
        sign = np.where(np.signbit(sh), -1.0 / 32, 1.0 / 32)
        g = _r(sh.astype(np.float64) / 16 + sign)
        assert np.all(g.astype(np.float64) == s / 16 + sign), "g inexact"
        v = _r(g.astype(np.float64) + 1536.0)
        assert np.array_equal(v.astype(np.int64) - 1536, want)
        # the output: centre (biased) plus the offset, then the clip in the
        # biased domain; 1024 + y is exact and its low ten bits are y
        for xv in (0, 1, 100, (1 << bd) - 1):
            y = xv + want
            inside = (y >= 0) & (y <= (1 << bd) - 1)
            yb = _r(v.astype(np.float64) + np.float64(xv + 1024 - 1536))
            assert np.array_equal(yb[inside].astype(np.int64), 1024 + y[inside])
            bits = yb[inside].view(np.uint16)
            assert np.array_equal(bits & 0x3FF, y[inside])
            assert np.all(bits >> 10 == 0x19)  # 0x6400 >> 10


def test_partial_sums_stay_exact():
    """Each tap pair adds w * (c0 + c1), |c| <= threshold, into the sum; every
    partial sum is an integer within the bound, so each addition is exact."""
    rng = np.random.default_rng(5)
    for bd in (8, 10):
        cs = bd - 8
        n = 100_000
        tp, ts = 15 << cs, 4 << cs
        c = np.concatenate([rng.integers(-tp, tp + 1, (n, 4)), rng.integers(-ts, ts + 1, (n, 8))], axis=1)
        w = np.array([4, 4, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1])
        acc = np.zeros(n, np.float16)
        exact = np.zeros(n, np.int64)
        for k in range(0, 12, 2):
            pair = _r(c[:, k].astype(np.float64) + c[:, k + 1])
            acc = _r(pair.astype(np.float64) * w[k] + acc.astype(np.float64))
            exact += w[k] * (c[:, k] + c[:, k + 1])
            assert np.array_equal(acc.astype(np.int64), exact)
