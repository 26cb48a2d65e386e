"""Batched wakes: one forest over many wakes (bs_forest_build / bs_forest_eval / bs_forest_graph) against each wake's
exact direct sum from the CPU oracle (oracle/bs_oracle.c, pinned to the reference's numba direct sum).

* A forest at a vanishing opening angle accepts no cell: every wake's velocity equals that wake's own FP64 direct sum
  within 1e-12 * max|u| (no cross-wake interaction, far counts all zero).
* Mixed precision at a small opening angle: each wake within 1e-5 relative L2 of its FP64 direct sum.
* The captured graph replays to the same bits as a fresh evaluation, also after the targets moved in place.
* The autotuned batch and the one-call-per-wake path agree.
"""
import numpy as np
import pytest

from conftest import no_exclusions
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def small_cases():
    from openfawe_b200 import wakes
    cases = [wakes.rotor_sheet(rows, seed=rows, targets=t, wind=w) for rows, t, w in
             ((12, 700, 8.0), (30, 1500, 10.0), (5, 300, 13.0), (18, 900, 6.0))]
    tiny = wakes.rotor_sheet(2, seed=1, targets=7)
    for k in ("starts", "directions", "lengths", "gamma", "radius"):
        tiny[k] = tiny[k][:7]
    one = wakes.rotor_sheet(2, seed=2, targets=5)
    for k in ("starts", "directions", "lengths", "gamma", "radius"):
        one[k] = one[k][:1]
    return cases + [tiny, one]


def per_wake_direct(cases, device=None):
    """Each wake's FP64 direct sum from the CPU oracle."""
    from openfawe_b200 import wakes
    out = []
    for c in cases:
        u, flagged = O.direct_sum(*wakes.backend_args(c), no_exclusions(len(c["points"])), "raise")
        assert not flagged
        out.append(u)
    return out


def test_forest_roots_cover_exactly_each_wake(device):
    from openfawe_b200 import batch, engine
    cases = small_cases()
    b = batch.WakeBatch(cases, device)
    forest = b.build(16)
    roots = engine.forest_roots(forest)
    arrays = forest.export()
    lo, hi = arrays["lo"], arrays["hi"]
    # the sorted order keeps wakes contiguous, so each wake's root spans exactly its own segment range
    for w, r in enumerate(roots):
        assert (lo[r], hi[r]) == (b.wake_ptr[w], b.wake_ptr[w + 1]), w


def test_forest_at_zero_angle_equals_per_wake_direct(device):
    from openfawe_b200 import batch
    cases = small_cases()
    b = batch.WakeBatch(cases, device)
    u, flags, far = b.evaluate(theta=1e-9, precision="fp64")
    assert not flags.any() and int(far.sum()) == 0
    for got, ref in zip(b.split(u.cpu().numpy()), per_wake_direct(cases, device)):
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * max(np.abs(ref).max(), 1e-300))


def test_forest_mixed_and_graph_replay(device):
    from openfawe_b200 import batch
    cases = small_cases()
    b = batch.WakeBatch(cases, device)
    u, flags, far = b.evaluate(theta=0.05, precision="mixed")
    assert not flags.any() and int(far.sum()) > 0
    for got, ref in list(zip(b.split(u.cpu().numpy()), per_wake_direct(cases, device)))[:4]:
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5
    g = b.capture(theta=0.05, precision="mixed")
    for _ in range(2):
        gu, gflags, gfar = g.launch()
        assert g.status()["near_pairs"] > 0
        assert np.array_equal(gu.cpu().numpy(), u.cpu().numpy())
        assert np.array_equal(gfar.cpu().numpy(), far.cpu().numpy())
    # the graph reads the target buffer in place: moved targets give the fresh evaluation's answer
    b.targets.points.add_(0.05)
    gu, _, _ = g.launch()
    fresh, _, _ = b.evaluate(theta=0.05, precision="mixed")
    assert np.array_equal(gu.cpu().numpy(), fresh.cpu().numpy())


def test_autotune_and_sequential_agree(device):
    from openfawe_b200 import batch
    cases = small_cases()[:4]
    b = batch.WakeBatch(cases, device)
    tuned = batch.autotune(b, theta=0.05, leaves=(16, 32), blocks=(64, 128))
    assert tuned["choice"] in {(16, 64), (16, 128), (32, 64), (32, 128)} and len(tuned["table"]) == 4
    u, _, _ = b.evaluate(theta=0.05, block=tuned["choice"][1])
    times, outs = batch.sequential(cases, device, theta=0.05)
    assert len(times) == 4 and np.all(times > 0)
    for got, seq, ref in zip(b.split(u.cpu().numpy()), outs, per_wake_direct(cases)):
        seq = seq.cpu().numpy()
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5
        assert np.linalg.norm(seq - ref) / np.linalg.norm(ref) < 1e-5


def _scale(points, case):
    """sum_s |u_s| per point from the oracle's per-pair velocities."""
    pairs, _ = O.pair_matrix(points, case["starts"], case["directions"], case["lengths"], case["radius"],
                             case["model"], False)
    return (np.linalg.norm(pairs, axis=2) * np.abs(case["gamma"])[None, :]).sum(axis=1)


def test_control_points_summed_exactly_in_the_same_launch(device):
    """Each wake's wing control points ride in the batch marked exact: no far node is accepted for them (far count 0),
    so they equal the oracle's direct sum over their own wake (A1 bound in FP64, 1e-5 of sum |u_s| mixed), while the
    wake's own targets keep their tree result; the captured graph replays the same bits."""
    from openfawe_b200 import batch, wakes
    cases = small_cases()[:4]
    control = [wakes.ring_wing(64)["points"] + [0.1 * w, 0.0, 0.0] for w in range(len(cases))]
    with_control = batch.WakeBatch(cases, device, control=control)
    plain = batch.WakeBatch(cases, device)
    for precision, tol in (("fp64", 1e-12), ("mixed", 1e-5)):
        u, flags, far = with_control.evaluate(theta=0.3, precision=precision)
        u0, _, far0 = plain.evaluate(theta=0.3, precision=precision)
        assert not flags.any()
        u, far, u0 = u.cpu().numpy(), far.cpu().numpy(), u0.cpu().numpy()
        for w, (c, q) in enumerate(zip(cases, control)):
            got = with_control.split_control(u)[w]
            assert np.all(with_control.split_control(far)[w] == 0)
            ref, flagged = O.direct_sum(q, *wakes.backend_args(c)[1:], no_exclusions(len(q)), "raise")
            assert not flagged
            err = np.linalg.norm(got - ref, axis=1)
            assert np.all(err <= tol * _scale(q, c)), (precision, w, float(err.max()))
            own, own0 = with_control.split(u)[w], plain.split(u0)[w]
            assert np.linalg.norm(own - own0) / np.linalg.norm(own0) <= (1e-13 if precision == "fp64" else 1e-6)
        assert int(far.sum()) == int(far0.sum().item()) and int(far.sum()) > 0
    g = with_control.capture(theta=0.3, precision="mixed")
    gu, _, gfar = g.launch()
    fresh, _, ffar = with_control.evaluate(theta=0.3, precision="mixed")
    assert np.array_equal(gu.cpu().numpy(), fresh.cpu().numpy())
    assert np.array_equal(gfar.cpu().numpy(), ffar.cpu().numpy())
