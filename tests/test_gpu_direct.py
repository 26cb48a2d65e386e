"""GPU direct sum (libbs_b200 bs_direct through the drop-in ``cuda_sum``) against the reference's outputs.

Bounds: FP64 -- the reference's acceptance A1, |u_gpu - u_ref| <= 1e-12 * sum_s |u_s| per target
(tests/test_vortex_numba.py:3-5 of the reference); flags identical per target.  Mixed/FP32 -- 1e-5 * sum_s |u_s| per
target (the reference's single-precision bound, tests/test_cuda_moments.py:136-149, measured here per target).
"""
import numpy as np
import pytest

from conftest import golden, no_exclusions
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def settings(precision="fp64", block=128):
    from openfawe_b200.settings import CudaSettings
    return CudaSettings(precision, block)


def scale_of(points, starts, directions, lengths, gamma, radius, model, csr=None, chunk=256):
    """sum_s |u_s| per target from the oracle's per-pair velocities (excluded pairs left out)."""
    out = np.zeros(len(points))
    for a in range(0, len(points), chunk):
        pairs, _ = O.pair_matrix(points[a:a + chunk], starts, directions, lengths, radius, model, False)
        mag = np.linalg.norm(pairs, axis=2) * np.abs(gamma)[None, :]
        if csr is not None:
            for p in range(a, min(a + chunk, len(points))):
                mag[p - a, csr[1][csr[0][p]:csr[0][p + 1]]] = 0.0
        out[a:a + chunk] = mag.sum(axis=1)
    return out


def within(u, ref, scale, tol):
    err = np.linalg.norm(u - ref, axis=1)
    assert np.all(err <= tol * scale + 1e-300), float(np.max(err - tol * scale))


def test_random_networks_every_model(device):
    from openfawe_b200.vortex_cuda import cuda_sum
    g = golden("direct_random.npz")
    for seed in (3, 4):
        P = lambda k: g[f"s{seed}_{k}"]  # noqa: E731
        csr = no_exclusions(len(P("points")))
        for model in range(6):
            for ci, core in enumerate((0.0, 0.2, P("radius"))):
                r = np.broadcast_to(np.asarray(core, dtype=np.float64), (len(P("gamma")),)).copy()
                args = (P("points"), P("starts"), P("directions"), P("lengths"), P("gamma"), r, model)
                scale = scale_of(*args)
                for sing in ("zero", "raise"):
                    key = f"s{seed}_m{model}_c{ci}_{sing}"
                    _, ref_flags = O.direct_sum(*args, csr, sing, return_flags=True)
                    for precision in ("fp64", "mixed", "fp32"):
                        u, flag = cuda_sum(*args, csr, sing, settings(precision))
                        assert flag == bool(g[key + "_flag"]), (key, precision)
                        assert u.flags.owndata and u.shape == (len(P("points")), 3)
                        ok = ref_flags == 0
                        within(u[ok], g[key][ok], scale[ok], 1e-12 if precision == "fp64" else 1e-5)


def test_per_target_flags_and_values_of_failure_cases(device):
    from openfawe_b200 import engine
    g = golden("direct_flags.npz")
    names = sorted({k.rsplit("_", 1)[0] for k in g.files if k.endswith("_points")})
    for name in names:
        for sing in ("raise", "zero"):
            for precision in ("fp64", "mixed"):
                src = engine.Sources(g[f"{name}_starts"], g[f"{name}_directions"], g[f"{name}_lengths"],
                                     g[f"{name}_gamma"], g[f"{name}_radius"], device)
                tgt = engine.Targets(g[f"{name}_points"], None, device)
                u, flags = engine.direct(src, tgt, int(g[f"{name}_model"]), sing, precision)
                assert np.array_equal(flags.cpu().numpy(), g[f"{name}_{sing}_flags"]), (name, sing, precision)
                if g[f"{name}_{sing}_flags"][0] == 0:
                    np.testing.assert_allclose(u.cpu().numpy(), g[f"{name}_{sing}_u"], rtol=1e-12, atol=0)


def test_exclusions_at_own_nodes(device):
    from openfawe_b200.vortex_cuda import cuda_sum
    g = golden("direct_exclusions.npz")
    csr = (g["ptr"], g["seg"])
    for model in (0, 2, 5):
        args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], model)
        scale = scale_of(*args, csr=csr)
        for precision in ("fp64", "mixed"):
            u, flag = cuda_sum(*args, csr, "raise", settings(precision))
            assert flag == bool(g[f"m{model}_flag"])
            within(u, g[f"m{model}"], scale, 1e-12 if precision == "fp64" else 1e-5)


def test_lattice_config_and_chunking(device):
    from openfawe_b200 import wakes
    from openfawe_b200.vortex_cuda import cuda_sum
    g = golden("direct_lattice.npz")
    case = wakes.lattice()
    args = wakes.backend_args(case)
    scale = scale_of(*args)
    csr = no_exclusions(len(case["points"]))
    for block in (32, 128, 256):
        u, flag = cuda_sum(*args, csr, "raise", settings("fp64", block))
        assert not flag
        within(u, g["u"], scale, 1e-12)
    u, _ = cuda_sum(*args, csr, "raise", settings("mixed"))
    within(u, g["u"], scale, 1e-6)
    rel = np.linalg.norm(u - g["u"]) / np.linalg.norm(g["u"])
    assert rel < 1e-6, rel


def test_selftest_sheet_with_exclusions_many_chunks(device):
    from openfawe_b200.vortex_cuda import cuda_sum
    g = golden("tree_selftest.npz")
    args = (g["points"], g["starts"], g["directions"], g["lengths"], g["gamma"], g["radius"], 2)
    csr = (g["ptr"], g["seg"])
    u, flag = cuda_sum(*args, csr, "raise", settings("fp64"))
    assert not flag
    scale = scale_of(g["points"][:400], *args[1:], csr=(g["ptr"][:401], g["seg"]))
    within(u[:400], g["direct"][:400], scale, 1e-12)
    np.testing.assert_allclose(u, g["direct"], rtol=1e-11, atol=1e-12 * np.abs(g["direct"]).max())
    um, _ = cuda_sum(*args, csr, "raise", settings("mixed"))
    assert np.linalg.norm(um - g["direct"]) / np.linalg.norm(g["direct"]) < 1e-6


def test_empty_inputs(device):
    from openfawe_b200.vortex_cuda import cuda_sum
    u, flag = cuda_sum(np.zeros((0, 3)), np.zeros((1, 3)), np.array([[1.0, 0, 0]]), np.ones(1), np.ones(1),
                       np.zeros(1), 0, no_exclusions(0), "raise", settings())
    assert u.shape == (0, 3) and not flag
    u, flag = cuda_sum(np.ones((4, 3)), np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), np.zeros(0), np.zeros(0), 0,
                       no_exclusions(4), "raise", settings())
    assert np.all(u == 0) and not flag


def test_repeatable_bitwise(device):
    from openfawe_b200 import wakes
    from openfawe_b200.vortex_cuda import cuda_sum
    case = wakes.lattice()
    csr = no_exclusions(len(case["points"]))
    for precision in ("fp64", "mixed"):
        a, _ = cuda_sum(*wakes.backend_args(case), csr, "raise", settings(precision))
        b, _ = cuda_sum(*wakes.backend_args(case), csr, "raise", settings(precision))
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_mixed_pairs_at_any_length_scale_and_tiny_cores(device):
    """The mixed pair works in units of each segment's length, so the same network scaled from 1e-7 m to 1e10 m stays
    in FP32 within the mixed bound; a core below 1e-15 of its segment's length carries a NaN 1/L in its FP32 record
    and every pair of such a segment is evaluated in FP64 (counted in fp64_pairs)."""
    from openfawe_b200 import engine
    g = golden("direct_random.npz")
    P = lambda k: g[f"s3_{k}"]  # noqa: E731
    n, m = len(P("points")), len(P("gamma"))
    for scale_x, core, all_fp64 in ((1e-7, 0.2, False), (1e7, 0.2, False), (1e10, 0.2, False), (1.0, 1e-17, True)):
        args = (P("points") * scale_x, P("starts") * scale_x, P("directions"), P("lengths") * scale_x, P("gamma"),
                np.full(m, core * scale_x), 2)
        src = engine.Sources(*args[1:6], device)
        tgt = engine.Targets(args[0], None, device)
        u64, f64 = engine.direct(src, tgt, 2, "zero", "fp64")
        um, fm = engine.direct(src, tgt, 2, "zero", "mixed")
        stats = engine.last_stats(device)
        assert np.array_equal(f64.cpu().numpy(), fm.cpu().numpy())
        if all_fp64:
            assert stats["fp64_pairs"] == n * m, (scale_x, core, stats["fp64_pairs"])
            np.testing.assert_allclose(um.cpu().numpy(), u64.cpu().numpy(), rtol=1e-12,
                                       atol=1e-12 * float(np.abs(u64.cpu().numpy()).max()))
        else:
            assert stats["fp64_pairs"] < n * m // 10, (scale_x, stats["fp64_pairs"])
            within(um.cpu().numpy(), u64.cpu().numpy(), scale_of(*args), 1e-5)
