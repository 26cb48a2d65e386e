"""The hand-written adjoint (bs_adjoint_direct behind torch.autograd) against central finite differences and against
the unit-circulation pair velocities of the reference's VSM operators.

* Finite differences: central, h = 1e-4 m, on the FP64 direct sum, for a random subset of target and endpoint
  coordinates, every core model (none, Rankine, Lamb-Oseen, Vatistas, offset, Rosenhead-Moore); geometry kept away
  from the Lamb-Oseen cut-off band (the core factor jumps there by e^-10).
* Circulation gradients: d(w.u)/dGamma_s = sum_p w_p . g_ps with g the unit-circulation pair velocity, which is what the
  reference's ``vortex_numba.pair_matrix`` (src/openfawe/aero/vortex_numba.py:271-287) computes for its VSM influence
  operators; checked on a 64-panel wing's rings assembled into panel columns the way ``assemble_columns`` (:290-308)
  assembles them, with the oracle's bit-exact pair matrix.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

LAMB_CUT2 = 10 / 1.25643


def network(seed, segments=40, points=30, core=0.1):
    """Random segments and targets whose pairs all stay clear of the Lamb-Oseen cut-off band."""
    rng = np.random.default_rng(seed)
    while True:
        starts = rng.uniform(-2, 2, (segments, 3))
        d = rng.normal(size=(segments, 3))
        ends = starts + 0.3 * d / np.linalg.norm(d, axis=1)[:, None] * rng.uniform(0.5, 1.5, (segments, 1))
        x = rng.uniform(-2, 2, (points, 3))
        r1 = x[:, None, :] - starts[None]
        r2 = x[:, None, :] - ends[None]
        lv = ends - starts
        h2 = np.sum(np.cross(r1, r2) ** 2, axis=2) / np.sum(lv * lv, axis=1)[None]
        rho2 = h2 / core ** 2
        if np.all(np.abs(rho2 - LAMB_CUT2) > 0.25 * LAMB_CUT2):
            return x, starts, ends, rng.uniform(0.5, 8.0, segments), np.full(segments, core)
        seed += 1000
        rng = np.random.default_rng(seed)


def direct_u(device, x, a, b, g, r, model=2):
    import torch
    from openfawe_b200 import adjoint, engine
    s, d, length = adjoint.segments_from_endpoints(torch.as_tensor(a, device=device), torch.as_tensor(b, device=device))
    src = engine.Sources(s, d, length, g, r, device)
    u, _ = engine.direct(src, engine.Targets(x, None, device), model, "zero", "fp64")
    return u.cpu().numpy()


@pytest.mark.parametrize("model", [0, 1, 2, 3, 4, 5])
def test_adjoint_against_central_differences(device, model):
    import torch
    from openfawe_b200 import adjoint
    x, a, b, g, r = network(5 + model)
    w = np.random.default_rng(5).normal(size=x.shape).astype(np.float32).astype(np.float64)
    gx, ga, gb, gg = [t.cpu().numpy() for t in adjoint.adjoint_direct(
        torch.as_tensor(x, device=device), a, b, g, r, model, w)]
    loss = lambda *args: float(np.sum(w * direct_u(device, *args, model=model)))  # noqa: E731
    h = 1e-4
    rng = np.random.default_rng(11)
    scale = max(np.abs(gx).max(), np.abs(ga).max(), np.abs(gb).max())
    for which, grad in ((0, gx), (1, ga), (2, gb)):
        for _ in range(21):
            i, k = rng.integers(grad.shape[0]), rng.integers(3)
            plus = [x.copy(), a.copy(), b.copy()]
            minus = [x.copy(), a.copy(), b.copy()]
            plus[which][i, k] += h
            minus[which][i, k] -= h
            fd = (loss(*plus, g, r) - loss(*minus, g, r)) / (2 * h)
            assert abs(fd - grad[i, k]) <= 1e-6 * scale, (model, which, i, k, fd, grad[i, k])
    # circulation: the sum is linear in Gamma, so the derivative is exact
    for s in rng.integers(len(g), size=8):
        gp = g.copy()
        gp[s] += 1.0
        assert abs((loss(x, a, b, gp, r) - loss(x, a, b, g, r)) - gg[s]) <= 1e-10 * max(1.0, abs(gg).max())


def test_autograd_function_matches_direct_adjoint(device):
    import torch
    from openfawe_b200 import adjoint
    x, a, b, g, r = network(21)
    tensors = [torch.tensor(v, device=device, requires_grad=True) for v in (x, a, b, g)]
    radius = torch.tensor(r, device=device)
    u = adjoint.induced_velocity(*tensors, radius, model=2, method="direct", precision="fp64", singularity="zero")
    w = torch.tensor(np.random.default_rng(3).normal(size=x.shape), device=device)
    (u * w).sum().backward()
    ref = adjoint.adjoint_direct(tensors[0].detach(), a, b, g, r, 2, w)
    for t, gref in zip(tensors, ref):
        assert torch.allclose(t.grad, gref, rtol=1e-12, atol=0)
    # the tree forward evaluates the same function to its truncation error
    ut = adjoint.induced_velocity(*[t.detach() for t in tensors], radius, model=2, method="tree", precision="mixed",
                                  theta=0.1, leaf_size=4, singularity="zero")
    assert torch.linalg.norm(ut - u.detach()) / torch.linalg.norm(u) < 1e-5


def wing_rings(panels=64, span=26.0, chord=2.0, wake=8.0):
    """Horseshoe-closed vortex rings of an elliptic wing: bound leg at the quarter chord, trailing legs to a far
    closing leg; returns the 4*panels edges (starts, ends), the panel of each edge and its sign, and the control
    points (three-quarter chord)."""
    y = np.linspace(-span / 2, span / 2, panels + 1)
    c = chord * np.sqrt(np.maximum(1 - (2 * y / span) ** 2, 0.05))
    quarter = np.column_stack((0.25 * c, y, np.zeros_like(y)))
    far = quarter + [wake, 0.0, 0.0]
    starts, ends, panel, sign = [], [], [], []
    for j in range(panels):
        corners = [quarter[j], quarter[j + 1], far[j + 1], far[j]]
        for k in range(4):
            starts.append(corners[k])
            ends.append(corners[(k + 1) % 4])
            panel.append(j)
            sign.append(1.0)
    yc = 0.5 * (y[:-1] + y[1:])
    cc = chord * np.sqrt(np.maximum(1 - (2 * yc / span) ** 2, 0.05))
    control = np.column_stack((0.75 * cc, yc, np.full(panels, 0.01)))
    return np.array(starts), np.array(ends), np.array(panel), np.array(sign), control


def test_circulation_gradient_is_the_vsm_influence_operator(device):
    import torch
    from openfawe_b200 import adjoint
    a, b, panel, sign, control = wing_rings()
    m, panels = len(a), panel.max() + 1
    radius = np.full(m, 0.05)
    lv = b - a
    length = np.hypot(np.hypot(lv[:, 0], lv[:, 1]), lv[:, 2])
    pairs, flags = O.pair_matrix(control, a, lv / length[:, None], length, radius, 2, False)
    # ring columns as assemble_columns builds them: column j = sum of its edges' signed unit velocities
    columns = np.zeros((len(control), panels, 3))
    for k in range(m):
        columns[:, panel[k]] += sign[k] * pairs[:, k]
    rng = np.random.default_rng(64)
    for _ in range(3):
        w = rng.normal(size=control.shape)
        gamma_panel = rng.uniform(0.5, 2.0, panels)
        _, _, _, gg = adjoint.adjoint_direct(torch.as_tensor(control, device=device), a, b, gamma_panel[panel] * sign,
                                             radius, 2, w)
        per_panel = np.zeros(panels)
        np.add.at(per_panel, panel, sign * gg.cpu().numpy())
        expected = np.einsum("pk,pjk->j", w, columns)
        np.testing.assert_allclose(per_panel, expected, rtol=1e-12, atol=1e-12 * np.abs(expected).max())
