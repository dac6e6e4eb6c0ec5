"""The CDEF kernel leaves out the clip when one strength is zero.

cdef_filter_block (cdef.rs:505-556) always clips the filtered sample to the
range of the tap samples it read.  cdef_kernel skips the taps of a zero
strength (constrain returns 0 at threshold 0, cdef.rs:592-606) and, when only
one strength is non-zero, the clip as well: the remaining taps' weights sum
to 12, every constrained difference has its tap's sign and at most its
magnitude, so the rounded offset never leaves [min, max].  This checks that
claim on random tap sets (availability, strengths, damping, 8 to 12 bits),
with the reference's arithmetic restated in numpy.
"""
import numpy as np

PRI_TAPS = np.array([[4, 2], [3, 3]])
SEC_TAPS = np.array([2, 1])


def _floor_log2(v):
    return np.where(v > 0, np.floor(np.log2(np.maximum(v, 1))).astype(np.int64), 0)


def _constrain(diff, thr, damping):
    """constrain (cdef.rs:592-606), vectorised."""
    adj = np.maximum(damping - _floor_log2(thr), 0)
    ad = np.abs(diff)
    inner = np.maximum(thr - (ad >> np.minimum(adj, 62)), 0)
    v = np.minimum(ad, inner)
    return np.where(thr == 0, 0, np.where(diff < 0, -v, v))


def _filter(x, pri_s, sec_s, avail_p, avail_s, pri, sec, damping, coeff_shift, clip):
    """One sample: primary taps pri_s[..., k, sign], secondary sec_s[..., k, sign, dir]."""
    row = (pri >> coeff_shift) & 1
    s = np.zeros_like(x)
    mn, mx = x.copy(), x.copy()
    for k in range(2):
        for g in range(2):
            a = avail_p[:, k, g]
            pv = pri_s[:, k, g]
            s += np.where(a, PRI_TAPS[row, k] * _constrain(pv - x, pri, damping), 0)
            mn = np.where(a, np.minimum(mn, pv), mn)
            mx = np.where(a, np.maximum(mx, pv), mx)
            for d in range(2):
                a2 = avail_s[:, k, g, d]
                sv = sec_s[:, k, g, d]
                s += np.where(a2, SEC_TAPS[k] * _constrain(sv - x, sec, damping), 0)
                mn = np.where(a2, np.minimum(mn, sv), mn)
                mx = np.where(a2, np.maximum(mx, sv), mx)
    y = x + ((8 + s - (s < 0)) >> 4)
    return np.clip(y, mn, mx) if clip else y


def test_unclipped_equals_clipped_when_one_strength_is_zero():
    rng = np.random.default_rng(2024)
    n = 200_000
    for bd in (8, 10, 12):
        cs = bd - 8
        hi = (1 << bd) - 1
        x = rng.integers(0, hi + 1, n)
        # taps near x (the interesting range) and anywhere in range
        near = lambda shape: np.clip(x.reshape((n,) + (1,) * (len(shape) - 1)) +
                                     rng.integers(-40 << cs, (40 << cs) + 1, shape), 0, hi)
        far = lambda shape: rng.integers(0, hi + 1, shape)
        for mk in (near, far):
            pri_s, sec_s = mk((n, 2, 2)), mk((n, 2, 2, 2))
            avail_p = rng.random((n, 2, 2)) < 0.9
            avail_s = rng.random((n, 2, 2, 2)) < 0.9
            damping = rng.integers(3, 7, n) + cs
            strength = rng.integers(1, 16, n) << cs     # primary strengths 1..15
            sec_strength = np.array([1, 2, 4])[rng.integers(0, 3, n)] << cs
            # only primary
            a = _filter(x, pri_s, sec_s, avail_p, avail_s, strength, 0 * strength, damping, cs, True)
            b = _filter(x, pri_s, sec_s, avail_p, avail_s, strength, 0 * strength, damping, cs, False)
            assert np.array_equal(a, b)
            # only secondary (the primary tap row still follows priStr = 0)
            a = _filter(x, pri_s, sec_s, avail_p, avail_s, 0 * strength, sec_strength, damping, cs, True)
            b = _filter(x, pri_s, sec_s, avail_p, avail_s, 0 * strength, sec_strength, damping, cs, False)
            assert np.array_equal(a, b)
            # both non-zero: the clip matters somewhere (the claim is not vacuous)
            a = _filter(x, pri_s, sec_s, avail_p, avail_s, strength, sec_strength, damping, cs, True)
            b = _filter(x, pri_s, sec_s, avail_p, avail_s, strength, sec_strength, damping, cs, False)
            if mk is near:
                assert not np.array_equal(a, b)
