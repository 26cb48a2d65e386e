"""The adjoint of the tree sum (bs_tree_adjoint) against the exact adjoint and against finite differences of the tree
forward it differentiates.

* No far field (theta 1e-9: every node is opened): the tree adjoint is the exact adjoint, so it equals
  bs_adjoint_direct (itself checked against central differences and the VSM columns) within 1e-12 relative in FP64
  and 1e-5 in mixed precision (FP32 pair terms).
* Central differences (h = 1e-4 m and h/2, Richardson-extrapolated, FP64 forward) of the tree sum at theta 0.3,
  orders 2 and 5: targets sit 0.011 m above the sheet, where a plain central difference at 1e-4 m still carries a
  truncation error of (h / 0.011 m)^2 ~ 1e-4, hence the extrapolation (error ~ h^4).  The tree adjoint holds node
  centres and acceptance decisions fixed, so coordinates are taken only where the forward's tree, accepted nodes and
  near pairs stay the same under the perturbations (identical counters at all of them) and where the perturbed
  endpoint is interior to every node box that holds it (a box's extreme endpoints move its centre); there the
  extrapolated quotient equals the adjoint to 1e-6 of the gradient's scale.  Circulations enter linearly: exact.
* The benchmark's setting (fifth-order Morton tree, theta 0.215, leaf 384, mixed) on the 468-row rotor wake (102k
  segments x 20,570 targets): every gradient within 2e-5 relative L2 of the exact adjoint.
* Excluded (target, segment) pairs: with no far field the mixed tree adjoint with exclusions is the exact adjoint
  with the same exclusions; so are the Vatistas, offset and Rosenhead-Moore cores' tree adjoints (FP64 near pairs).
* The autograd function's backward on a tree forward is the tree adjoint.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def small_wake(rows=14, targets=700, seed=9):
    from openfawe_b200 import wakes
    case = wakes.rotor_sheet(rows, seed=seed, targets=targets)
    a = case["starts"]
    b = case["nodes"][case["edges"][:, 1]]
    rng = np.random.default_rng(seed)
    w = rng.normal(size=case["points"].shape)
    return case["points"], a, b, case["gamma"], case["radius"], w


def tree_forward(device, x, a, b, g, r, theta, order, leaf, kind, precision="fp64", model=2):
    import torch
    from openfawe_b200 import adjoint, engine
    s, d, length = adjoint.segments_from_endpoints(torch.as_tensor(a, device=device), torch.as_tensor(b, device=device))
    src = engine.Sources(s, d, length, g, r, device)
    u, _, far = engine.tree_sum(src, engine.Targets(x, None, device), model, "zero", precision, 128, 3.0, theta, order,
                                leaf, 3.0, kind)
    st = engine.last_stats(device)
    return u.cpu().numpy(), (st["near_pairs"], st["far_evaluations"], st["nodes"], int(far.sum().item()))


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("kind", ["morton", "median"])
def test_tree_adjoint_without_far_field_is_the_exact_adjoint(device, kind):
    import torch
    from openfawe_b200 import adjoint
    x, a, b, g, r, w = small_wake()
    pts = torch.as_tensor(x, device=device)
    exact = [t.cpu().numpy() for t in adjoint.adjoint_direct(pts, a, b, g, r, 2, w)]
    for precision, tol in (("fp64", 1e-12), ("mixed", 1e-5)):
        got = [t.cpu().numpy() for t in adjoint.adjoint_tree(pts, a, b, g, r, 2, w, precision=precision, theta=1e-9,
                                                             order=2, leaf_size=32, kind=kind)]
        for name, u, v in zip(("points", "starts", "ends", "gamma"), got, exact):
            assert rel(u, v) <= tol, (kind, precision, name, rel(u, v))


@pytest.mark.parametrize("model", [3, 4, 5])
def test_tree_adjoint_of_the_other_core_models_is_the_exact_adjoint(device, model):
    """Vatistas, offset and Rosenhead-Moore cores (FP64 near pairs in either precision): with no far field the tree
    adjoint equals the exact adjoint."""
    import torch
    from openfawe_b200 import adjoint
    x, a, b, g, r, w = small_wake()
    pts = torch.as_tensor(x, device=device)
    exact = [t.cpu().numpy() for t in adjoint.adjoint_direct(pts, a, b, g, r, model, w)]
    for precision in ("fp64", "mixed"):
        got = [t.cpu().numpy() for t in adjoint.adjoint_tree(pts, a, b, g, r, model, w, precision=precision,
                                                             theta=1e-9, order=2, leaf_size=32, kind="morton")]
        for name, u, v in zip(("points", "starts", "ends", "gamma"), got, exact):
            assert rel(u, v) <= 1e-12, (model, precision, name, rel(u, v))


def test_tree_adjoint_with_exclusions_is_the_exact_adjoint(device):
    """Excluded (target, segment) pairs in the near pairs: with no far field the mixed tree adjoint equals the exact
    adjoint with the same exclusions.  The targets on one side of the wake exclude three segments each, spread over
    the wake, so that work items with excluding targets, without them, and with both occur (the near kernel's clear
    paths with and without the per-pair exclusion test); each also excludes the segment nearest to it."""
    import torch
    from openfawe_b200 import adjoint
    x, a, b, g, r, w = small_wake()
    n, m = len(x), len(a)
    left = x[:, 0] < np.median(x[:, 0])
    mid = 0.5 * (a + b)
    nearest = np.argmin(((x[:, None, :] - mid[None, :, :]) ** 2).sum(axis=2), axis=1)
    rows = [sorted({int(nearest[p]), p % m, (7 * p + 3) % m, (13 * p + 5) % m}) if left[p] else [] for p in range(n)]
    csr = (np.concatenate(([0], np.cumsum([len(q) for q in rows]))).astype(np.int64),
           np.array([s_ for q in rows for s_ in q], dtype=np.int64))
    pts = torch.as_tensor(x, device=device)
    exact = [t.cpu().numpy() for t in adjoint.adjoint_direct(pts, a, b, g, r, 2, w, csr=csr)]
    plain = [t.cpu().numpy() for t in adjoint.adjoint_direct(pts, a, b, g, r, 2, w)]
    assert min(rel(u, v) for u, v in zip(plain, exact)) > 1e-3  # the exclusions matter
    got = [t.cpu().numpy() for t in adjoint.adjoint_tree(pts, a, b, g, r, 2, w, csr=csr, precision="mixed",
                                                         theta=1e-9, order=2, leaf_size=32, kind="morton")]
    for name, u, v in zip(("points", "starts", "ends", "gamma"), got, exact):
        assert rel(u, v) <= 1e-5, (name, rel(u, v))


def interior_endpoints(x, a, b, g, r, leaf, kind, device):
    """(segment, end, axis) triples whose coordinate is strictly inside the endpoint box of every node holding the
    segment (moving it moves no node centre)."""
    import torch
    from openfawe_b200 import adjoint, engine
    s, d, length = adjoint.segments_from_endpoints(torch.as_tensor(a, device=device), torch.as_tensor(b, device=device))
    tree = engine.build_tree(engine.Sources(s, d, length, g, r, device), leaf_size=leaf, kind=kind, order=2)
    arr = tree.export()
    ends = np.stack((a, b), axis=1)  # [m, 2, 3]
    extreme = np.zeros((len(a), 2, 3), dtype=bool)
    for lo, hi in zip(arr["lo"], arr["hi"]):
        segs = arr["order"][lo:hi]
        e = ends[segs]
        for axis in range(3):
            vals = e[:, :, axis]
            extreme[segs, :, axis] |= (vals == vals.min()) | (vals == vals.max())
    return [(i, k, axis) for i in range(len(a)) for k in range(2) for axis in range(3) if not extreme[i, k, axis]]


@pytest.mark.parametrize("order,kind", [(2, "median"), (5, "morton")])
def test_tree_adjoint_against_central_differences(device, order, kind):
    import torch
    from openfawe_b200 import adjoint
    theta, leaf, h = 0.3, 16, 1e-4
    x, a, b, g, r, w = small_wake(rows=10, targets=400, seed=order)
    pts = torch.as_tensor(x, device=device)
    gx, ga, gb, gg = [t.cpu().numpy() for t in adjoint.adjoint_tree(pts, a, b, g, r, 2, w, precision="fp64",
                                                                    theta=theta, order=order, leaf_size=leaf,
                                                                    kind=kind)]
    base_u, base_c = tree_forward(device, x, a, b, g, r, theta, order, leaf, kind)
    assert base_c[1] > 0  # the far field takes part
    loss = lambda u: float(np.sum(w * u))  # noqa: E731
    scale = max(np.abs(gx).max(), np.abs(ga).max(), np.abs(gb).max())
    rng = np.random.default_rng(order)
    candidates = interior_endpoints(x, a, b, g, r, leaf, kind, device)
    checked = 0
    trials = [("point", int(i), 0, int(k)) for i, k in zip(rng.integers(len(x), size=24), rng.integers(3, size=24))]
    trials += [("end",) + candidates[int(j)] for j in rng.choice(len(candidates), size=48, replace=False)]
    for trial in trials:
        if trial[0] == "point":
            _, i, _, k = trial
            which, grad = 0, gx[i, k]
        else:
            _, i, end, k = trial
            which, grad = 1 + end, (ga if end == 0 else gb)[i, k]
        quotients, same = [], True
        for step in (h, h / 2):
            values = []
            for sign in (1.0, -1.0):
                moved = [x.copy(), a.copy(), b.copy()]
                moved[which][i, k] += sign * step
                u, c = tree_forward(device, *moved, g, r, theta, order, leaf, kind)
                same = same and c == base_c
                values.append(loss(u))
            quotients.append((values[0] - values[1]) / (2 * step))
        if not same:
            continue  # the tree or its decisions changed: the forward is not differentiable across that step
        fd = (4.0 * quotients[1] - quotients[0]) / 3.0
        assert abs(fd - grad) <= 1e-6 * scale, (order, kind, trial, fd, grad, quotients)
        checked += 1
    assert checked >= 40, checked
    # circulations enter linearly: the derivative is exact
    for s_ in rng.integers(len(g), size=6):
        gp = g.copy()
        gp[s_] += 1.0
        u1, _ = tree_forward(device, x, a, b, gp, r, theta, order, leaf, kind)
        assert abs(loss(u1) - loss(base_u) - gg[s_]) <= 1e-10 * max(1.0, np.abs(gg).max())


def test_tree_adjoint_at_the_bench_setting_matches_the_exact_gradient(device):
    import torch
    from openfawe_b200 import adjoint, wakes
    case = wakes.rotor_sheet(468, seed=468, targets=20570)
    x, a, g, r = case["points"], case["starts"], case["gamma"], case["radius"]
    b = case["nodes"][case["edges"][:, 1]]
    w = np.random.default_rng(5).standard_normal(x.shape).astype(np.float32).astype(np.float64)
    pts = torch.as_tensor(x, device=device)
    exact = [t.cpu().numpy() for t in adjoint.adjoint_direct(pts, a, b, g, r, 2, w)]
    got = [t.cpu().numpy() for t in adjoint.adjoint_tree(pts, a, b, g, r, 2, w, precision="mixed", theta=0.215,
                                                         order=5, leaf_size=384, kind="morton")]
    for name, u, v in zip(("points", "starts", "ends", "gamma"), got, exact):
        assert rel(u, v) <= 2e-5, (name, rel(u, v))


def test_autograd_backward_of_a_tree_forward_is_the_tree_adjoint(device):
    import torch
    from openfawe_b200 import adjoint
    x, a, b, g, r, w = small_wake(rows=8, targets=300, seed=4)
    tensors = [torch.tensor(v, device=device, requires_grad=True) for v in (x, a, b, g)]
    radius = torch.tensor(r, device=device)
    opts = dict(model=2, method="tree", precision="mixed", theta=0.3, order=5, leaf_size=16, kind="morton",
                singularity="zero")
    u = adjoint.induced_velocity(*tensors, radius, **opts)
    wt = torch.tensor(w, device=device)
    (u * wt).sum().backward()
    ref = adjoint.adjoint_tree(tensors[0].detach(), a, b, g, r, 2, wt, precision="mixed", theta=0.3, order=5,
                               leaf_size=16, kind="morton")
    for t, gref in zip(tensors, ref):
        assert rel(t.grad.cpu().numpy(), gref.cpu().numpy()) <= 1e-6
