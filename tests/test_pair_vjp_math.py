"""The FP64 pair VJP of every core model, restated on the CPU (no GPU).

pair_vjp64 (csrc/bs_pair_vjp.cuh) differentiates the pair in its two-endpoint form by hand: the core factor f(rho^2)
of models 1-3 (Rankine, Lamb-Oseen, Vatistas n = 2), the offset core's rc^2 |B - A|^2 in the denominator (model 4)
and the Rosenhead-Moore core's augmented distances (model 5, with P^2 - d^2 = |c|^2 + rc^2 |B - A|^2 in the
rationalised branch).  Restated here line for line in float64 and checked against central differences (h = 1e-6) of
the oracle's pair (vortex_numba.pair_velocity restated) for random geometry: d/dx = g1 + g2, d/dA = -g1, d/dB = -g2
within 1e-7 of the gradient's scale, and d/dGamma equal to the unit-circulation pair.
"""
import numpy as np
import pytest

from oracle import oracle as O

LAMB_A = 1.25643
CUT2 = 10 / LAMB_A
INV_FOUR_PI = 1 / (4 * np.pi)


def fwd(x, a, b, G, rc, model):
    """The oracle's FP64 pair velocity of segment a -> b at x, circulation G."""
    length = np.linalg.norm(b - a)
    pairs, _ = O.pair_matrix(x[None], a[None], ((b - a) / length)[None], np.array([length]), np.array([rc]), model,
                             False)
    return G * pairs[0, 0]


def core_factor(rho2, model):
    """f(rho^2) and df/drho^2 of the core-factor models (1, 2, 3)."""
    if model == 1:
        return (rho2, 1.0) if rho2 < 1 else (1.0, 0.0)
    if model == 3:
        f = rho2 / np.hypot(1, rho2) if rho2 < 1 else 1 / np.hypot(1, 1 / rho2)
        g = 1 / np.hypot(1, rho2) if rho2 < 1 else (1 / rho2) / np.hypot(1, 1 / rho2)
        return f, g ** 3
    if rho2 <= CUT2:
        em1 = np.expm1(-LAMB_A * rho2)
        return -em1, LAMB_A * (1 + em1)
    return 1.0, 0.0


def vjp(x, a, b, G, rc, model, w):
    """pair_vjp64: d(w.u)/dr1, d(w.u)/dr2 (r1 = x - a, r2 = x - b) and d(w.u)/dG."""
    r1, r2 = x - a, x - b
    l = r1 - r2
    L2 = l @ l
    c = np.cross(r1, r2)
    cc = c @ c
    q1, q2 = r1 @ r1, r2 @ r2
    irc2L2 = 1 / (L2 * rc * rc) if (1 <= model <= 3 and rc > 0) else 0.0
    rc2 = rc * rc if (model >= 4 and rc > 0) else 0.0
    rm = model == 5 and rc2 > 0
    n1, n2 = (np.sqrt(q1 + rc2), np.sqrt(q2 + rc2)) if rm else (np.sqrt(q1), np.sqrt(q2))
    d = r1 @ r2 + (rc2 if rm else 0.0)
    P = n1 * n2
    Q = cc + rc2 * L2 if rm else cc  # P^2 - d^2
    dD_dL2 = 0.0
    if d >= 0:
        D, dD_dP, dD_dd, dD_dcc = P * (P + d), 2 * P + d, P, 0.0
    else:
        iq = 1 / (P - d)
        D, dD_dP, dD_dd, dD_dcc = P * Q * iq, -Q * d * iq * iq, P * Q * iq * iq, P * iq
        if rm:
            dD_dL2 = rc2 * P * iq
    if model == 4 and rc2 > 0:
        D += rc2 * L2
        dD_dL2 = rc2
    rho2 = cc * irc2L2
    f, df = core_factor(rho2, model) if irc2L2 > 0 else (1.0, 0.0)
    S = n1 + n2
    coef = INV_FOUR_PI * f * S / D
    wc = w @ c
    h = G * wc * INV_FOUR_PI / D
    g_S, g_D = h * f, -h * f * S / D
    g_rho2 = h * S * df
    g_cc = g_rho2 * irc2L2 + g_D * dD_dcc
    g_L2 = -g_rho2 * rho2 / L2 + g_D * dD_dL2
    g_P, g_d = g_D * dD_dP, g_D * dD_dd
    gc = G * coef * w + 2 * c * g_cc
    g1 = (g_S + g_P * n2) / n1 * r1 + g_d * r2 + np.cross(r2, gc) + 2 * g_L2 * l
    g2 = (g_S + g_P * n1) / n2 * r2 + g_d * r1 + np.cross(gc, r1) - 2 * g_L2 * l
    return g1, g2, coef * wc


@pytest.mark.parametrize("model", [0, 1, 2, 3, 4, 5])
def test_pair_vjp_against_central_differences(model):
    rng = np.random.default_rng(3 + model)
    checked = 0
    for _ in range(120):
        a = rng.normal(size=3) * 0.3
        b = a + rng.normal(size=3) * 0.3
        x = rng.normal(size=3) * 0.6
        G, rc, w = rng.normal(), 0.2, rng.normal(size=3)
        c = np.cross(x - a, x - b)
        rho2 = (c @ c) / (((b - a) @ (b - a)) * rc * rc)
        if (model == 2 and abs(rho2 - CUT2) < 0.3 * CUT2) or (model == 1 and abs(rho2 - 1) < 0.05):
            continue  # the factor's kinks: no derivative there
        g1, g2, gg = vjp(x, a, b, G, rc, model, w)
        h, e = 1e-6, np.eye(3)

        def fd(moved):
            return np.array([(w @ fwd(*moved(h * e[i]), G, rc, model) - w @ fwd(*moved(-h * e[i]), G, rc, model))
                             / (2 * h) for i in range(3)])
        fdx = fd(lambda s: (x + s, a, b))
        fda = fd(lambda s: (x, a + s, b))
        fdb = fd(lambda s: (x, a, b + s))
        scale = max(np.abs(fdx).max(), np.abs(fda).max(), np.abs(fdb).max(), 1e-12)
        assert np.abs(g1 + g2 - fdx).max() <= 1e-7 * scale
        assert np.abs(-g1 - fda).max() <= 1e-7 * scale and np.abs(-g2 - fdb).max() <= 1e-7 * scale
        unit = w @ fwd(x, a, b, 1.0, rc, model)
        assert abs(gg - unit) <= 1e-12 * max(abs(unit), 1e-12)
        checked += 1
    assert checked > 60
