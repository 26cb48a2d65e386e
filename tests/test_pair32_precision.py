"""The single-precision pair without a core, restated on the CPU (no GPU): why the mixed path takes FP64 within a
quarter of a segment's length of the segment (NOCORE_NEAR2 in csrc/bs_internal.cuh).

pair32 (csrc/bs_internal.cuh) works in units of the segment's length: a = (x - s)/L from the two-float difference
(rounded once to FP32), b = a - d, c = d x a, and the reference's pair (vortex_numba.pair_velocity) on a, b, c, with
the rationalised denominator where a.b < 0.  a carries about one ulp of |a|, and b = a - d inherits that absolute
error, so beside an end point (or the axis) the pair's relative error grows as eps / distance; the core models take
FP64 within three core radii, which covers that, but without a core (model 0) only the rule does.  Checked against the
oracle's FP64 pair (model 0, segments 0.05-0.5 m long at coordinates of tens of metres):

* targets 0.02-0.06 L beside an end point: the FP32 pair errs by more than 2e-6 relative for some of them;
* targets 0.25-3 L from the segment (beside an end point or its middle): within 1e-6 relative, every one.
"""
import numpy as np

from oracle import oracle as O


def pair32_no_core(x, s, d, length):
    """pair32 for model 0 in float32 (the velocity for unit circulation, as a float64 array)."""
    f = np.float32
    a = (x - s).astype(f) * f(1.0 / length)
    dd = d.astype(f)
    b = a - dd
    c = np.cross(dd, a).astype(f)
    na = np.sqrt((a * a).sum(dtype=f))
    nb = np.sqrt((b * b).sum(dtype=f))
    dot = (a * b).sum(dtype=f)
    h2 = (c * c).sum(dtype=f)
    p = na * nb
    k = (na + nb) * (p - dot) / (p * h2) if dot < 0 else (na + nb) / (p * (p + dot))
    return (k * c / f(length)).astype(np.float64) / (4.0 * np.pi)


def worst_error(rng, lo, hi, beside_end, trials=600):
    worst = 0.0
    for _ in range(trials):
        s = rng.normal(size=3) * 30.0
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        length = rng.uniform(0.05, 0.5)
        u = rng.normal(size=3)
        u -= u.dot(d) * d
        u /= np.linalg.norm(u)
        along = length if beside_end else length * rng.uniform(0.2, 0.8)
        x = s + d * along + u * rng.uniform(lo, hi) * length
        pairs, _ = O.pair_matrix(x[None, :], s[None, :], d[None, :], np.array([length]), np.array([0.0]), 0, False)
        ref = pairs[0, 0]
        worst = max(worst, np.linalg.norm(pair32_no_core(x, s, d, length) - ref) / np.linalg.norm(ref))
    return worst


def test_fp32_pair_beside_an_end_point_needs_fp64():
    assert worst_error(np.random.default_rng(1), 0.02, 0.06, True) > 2e-6


def test_fp32_pair_a_quarter_length_away_stays_within_1e6():
    rng = np.random.default_rng(2)
    assert worst_error(rng, 0.25, 3.0, True) <= 1e-6
    assert worst_error(rng, 0.25, 3.0, False) <= 1e-6
