"""The clear-leaf pair and its adjoint, restated on the CPU (no GPU).

The single-precision evaluation takes a shorter form for a target at least 1.5 bounding radii from a leaf's centre
O (csrc/bs_internal.cuh pair32x2_clear, csrc/bs_pair_vjp.cuh pair_vjp32_clear): leaf-relative FP32 offsets in physical
units, r1 = (x - O) + (O - s), r2 = r1 - l, c = l x r1 = r1 x r2, and

    u = Gamma/(4 pi) f (|r1| + |r2|) c / (|r1||r2| (|r1||r2| + r1.r2)),   f from (h / rc)^2 = |c|^2 / (L rc)^2,

the reference's pair (vortex_numba.pair_velocity) with numerator and denominator multiplied by L^3.  Checked here:

* the form in float32 against the oracle's FP64 pair for random clear targets, models 0, 1, 2: within 1e-6 of the
  largest pair (every segment is seen under less than 84 degrees, r1.r2 >= 0.1 |r1||r2|);
* the closed-form gradients the adjoint kernel uses (d(w.u)/dr1, d(w.u)/dr2, d(w.u)/dGamma, with the dependence of
  rho^2 on L = |B - A|) against central finite differences of the same pair in float64.
"""
import numpy as np
import pytest

from oracle import oracle as O

LAMB_A = 1.25643
LAMB_CUT2 = 10.0 / LAMB_A


def clear_leaf(rng, model):
    """A leaf of 8 segments around a centre O, a target 1.5-4.6 bounding radii out, circulations and cores."""
    centre = rng.normal(size=3) * 10.0
    starts = centre + rng.normal(size=(8, 3)) * 0.3
    d = rng.normal(size=(8, 3))
    d /= np.linalg.norm(d, axis=1)[:, None]
    lengths = rng.uniform(0.05, 0.4, 8)
    ends = starts + d * lengths[:, None]
    bound = max(np.linalg.norm(starts - centre, axis=1).max(), np.linalg.norm(ends - centre, axis=1).max())
    u = rng.normal(size=3)
    x = centre + u / np.linalg.norm(u) * bound * rng.uniform(1.5, 4.6)
    gamma = rng.normal(size=8)
    radius = np.full(8, 0.05 if model else 0.0)
    return x, centre, starts, d, lengths, gamma, radius


def clear_pair_f32(x, centre, starts, d, lengths, gamma, radius, model):
    """The clear-leaf form in float32, from the record fields the build writes (clear_half)."""
    f = np.float32
    rel = (x - centre).astype(f)
    nsr = (centre - starts).astype(f)
    gf = (gamma / (4.0 * np.pi)).astype(f)
    l = (d * lengths[:, None]).astype(f)
    with np.errstate(divide="ignore"):
        w = np.where(radius > 0, 1.0 / (lengths * radius) ** 2, np.inf).astype(f)
    r1 = rel[None, :] + nsr
    r2 = r1 - l
    c = np.cross(l, r1).astype(f)
    h2 = (c * c).sum(axis=1, dtype=f)
    n1 = np.sqrt((r1 * r1).sum(axis=1, dtype=f))
    n2 = np.sqrt((r2 * r2).sum(axis=1, dtype=f))
    dot = (r1 * r2).sum(axis=1, dtype=f)
    product = n1 * n2
    k = gf * (n1 + n2)
    with np.errstate(invalid="ignore", over="ignore"):
        if model == 1:
            k = k * np.fmin(h2 * w, f(1))
        elif model == 2:
            r2c = h2 * w
            k = k * np.where(r2c < f(LAMB_CUT2), f(1) - np.exp2(r2c * f(-LAMB_A * np.log2(np.e))), f(1))
    return (k / (product * (product + dot)))[:, None] * c


@pytest.mark.parametrize("model", [0, 1, 2])
def test_clear_pair_float32_against_the_oracle(model):
    rng = np.random.default_rng(3 + model)
    worst = 0.0
    for _ in range(100):
        x, centre, starts, d, lengths, gamma, radius = clear_leaf(rng, model)
        pairs, _ = O.pair_matrix(x[None, :], starts, d, lengths, radius, model, False)
        ref = pairs[0] * gamma[:, None]
        got = clear_pair_f32(x, centre, starts, d, lengths, gamma, radius, model)
        worst = max(worst, np.abs(got - ref).max() / np.linalg.norm(ref, axis=1).max())
    assert worst <= 1e-6, worst


def pair64(x, a, b, gamma, rc, model):
    """The pair in its two-endpoint form, float64."""
    r1, r2, l = x - a, x - b, b - a
    c = np.cross(r1, r2)
    n1, n2 = np.linalg.norm(r1), np.linalg.norm(r2)
    p = n1 * n2
    f = 1.0
    if model and rc > 0:
        rho2 = (c @ c) / ((l @ l) * rc * rc)
        if model == 1:
            f = min(rho2, 1.0)
        elif rho2 <= LAMB_CUT2:
            f = 1.0 - np.exp(-LAMB_A * rho2)
    return gamma / (4 * np.pi) * f * (n1 + n2) * c / (p * (p + r1 @ r2))


def clear_vjp(x, a, b, gamma, rc, model, w):
    """The gradients pair_vjp32_clear forms (in float64 here): d(w.u)/dr1, d(w.u)/dr2, d(w.u)/dGamma."""
    r1, r2 = x - a, x - b
    l = r1 - r2
    L2 = l @ l
    c = np.cross(r1, r2)
    cc = c @ c
    n1, n2 = np.linalg.norm(r1), np.linalg.norm(r2)
    p, dt = n1 * n2, r1 @ r2
    D, S = p * (p + dt), n1 + n2
    f, df, rho2, wr = 1.0, 0.0, 0.0, 0.0
    if model and rc > 0:
        wr = 1.0 / (L2 * rc * rc)
        rho2 = cc * wr
        if model == 1:
            if rho2 < 1.0:
                f, df = rho2, 1.0
        elif rho2 <= LAMB_CUT2:
            e = np.exp(-LAMB_A * rho2)
            f, df = 1.0 - e, LAMB_A * e
    gf = gamma / (4 * np.pi)
    wc = w @ c
    h = gf * wc / D
    gg = f * S * wc / (4 * np.pi * D)
    g_S, g_D = h * f, -h * f * S / D
    g_rho2 = h * S * df
    g_cc = g_rho2 * wr if df != 0.0 else 0.0
    g_P, g_dt = g_D * (2 * p + dt), g_D * p
    k = gf * f * S / D
    gc = k * w + 2 * c * g_cc
    s1, s2 = (g_S + g_P * n2) / n1, (g_S + g_P * n1) / n2
    bb = 2 * g_rho2 * rho2 / L2 if df != 0.0 else 0.0
    g1 = s1 * r1 + g_dt * r2 + np.cross(r2, gc) - bb * l
    g2 = s2 * r2 + g_dt * r1 + np.cross(gc, r1) + bb * l
    return g1, g2, gg


@pytest.mark.parametrize("model", [0, 1, 2])
def test_clear_vjp_against_finite_differences(model):
    rng = np.random.default_rng(11 + model)
    h = 1e-6
    for _ in range(100):
        a = rng.normal(size=3) * 0.3
        b = a + rng.normal(size=3) * 0.2
        x = rng.normal(size=3)
        x = x / np.linalg.norm(x) * rng.uniform(0.8, 3.0)
        gamma, rc, w = rng.normal(), (0.3 if model else 0.0), rng.normal(size=3)
        g1, g2, gg = clear_vjp(x, a, b, gamma, rc, model, w)
        e = np.eye(3)
        # r1 = x - A: d/dr1 = -d/dA; r2 = x - B: d/dr2 = -d/dB
        fd1 = np.array([(w @ pair64(x, a - h * e[i], b, gamma, rc, model)
                         - w @ pair64(x, a + h * e[i], b, gamma, rc, model)) / (2 * h) for i in range(3)])
        fd2 = np.array([(w @ pair64(x, a, b - h * e[i], gamma, rc, model)
                         - w @ pair64(x, a, b + h * e[i], gamma, rc, model)) / (2 * h) for i in range(3)])
        fdg = (w @ pair64(x, a, b, gamma + h, rc, model) - w @ pair64(x, a, b, gamma - h, rc, model)) / (2 * h)
        scale = max(np.abs(fd1).max(), np.abs(fd2).max(), 1e-12)
        assert np.abs(g1 - fd1).max() <= 1e-6 * scale and np.abs(g2 - fd2).max() <= 1e-6 * scale
        assert abs(gg - fdg) <= 1e-6 * max(abs(fdg), 1e-12)
