"""GPU Robin Hood solve (kemcu_robin_hood) against the reference's KRobinHood<double>
(tests/golden/robinhood.npz, made by tests/golden/make_golden.py from the reference build) and
against the direct solution of the reference's boundary-integral matrix."""

import numpy as np
import pytest

import kassiopeia_b200 as K
from oracle import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = K.CUDAElectrostaticContext(0)
    yield c
    c.close()


def rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("name,direct", [("icosphere_L2", "sigma_direct"), ("mixed_small", "x_direct")])
@pytest.mark.parametrize("tol", [1e-8, 1e-10])
def test_robin_hood_matches_reference(ctx, name, direct, tol):
    fx = golden.load(name)
    rh = golden.load("robinhood")
    key = f"{name}_{tol:.0e}"
    ctx.SetGeometry(golden.mesh_from(fx))
    x, st = ctx.SolveRobinHood(tol=tol)
    assert st["rel_residual"] <= tol
    # same method, same checks: the reference needs the same number of residual checks
    assert abs(st["iterations"] - int(rh[key + "_iterations"])) <= 1, (st["iterations"], int(rh[key + "_iterations"]))
    # both runs stop within the tolerance of the exact solution of the same matrix
    ref_err = rel(rh[key + "_sigma"], fx[direct])
    assert rel(x, fx[direct]) <= max(5 * ref_err, 100 * tol)
    assert rel(x, rh[key + "_sigma"]) <= max(5 * ref_err, 100 * tol)
    # the solution becomes the context's charge density
    np.testing.assert_array_equal(ctx.GetSigma(), x)


def test_robin_hood_assembled_columns_identical(ctx):
    fx = golden.load("icosphere_L2")
    ctx.SetGeometry(golden.mesh_from(fx))
    x1, s1 = ctx.SolveRobinHood(tol=1e-9)
    x2, s2 = ctx.SolveRobinHood(tol=1e-9, assembled=True)
    # the assembled FP64 operator holds the same entries the matrix-free pass computes
    assert s1["subiterations"] == s2["subiterations"]
    np.testing.assert_array_equal(x1, x2)


def test_robin_hood_initial_guess_and_limits(ctx):
    fx = golden.load("icosphere_L2")
    ctx.SetGeometry(golden.mesh_from(fx))
    xd = fx["sigma_direct"]
    rng = np.random.default_rng(5)
    x0 = xd * (1 + 1e-3 * rng.normal(size=xd.size))
    x, st = ctx.SolveRobinHood(tol=1e-8, x0=x0)
    cold = ctx.SolveRobinHood(tol=1e-8)[1]
    assert st["rel_residual"] <= 1e-8 and st["subiterations"] < cold["subiterations"]
    # a sub-iteration limit below what the solve needs ends it unconverged
    x, st = ctx.SolveRobinHood(tol=1e-8, max_subiterations=100, raise_on_failure=False)
    assert st["status"] == K._native.ENOTCONVERGED and st["subiterations"] == 100
    # a shorter residual-check interval checks more often
    x, st = ctx.SolveRobinHood(tol=1e-8, check_interval=32)
    assert st["rel_residual"] <= 1e-8 and st["iterations"] > cold["iterations"]


def test_robin_hood_callback_stops(ctx):
    fx = golden.load("icosphere_L2")
    ctx.SetGeometry(golden.mesh_from(fx))
    seen = []

    def cb(it, r):
        seen.append((it, r))
        return len(seen) >= 3

    ctx.SetIterationCallback(cb)
    try:
        x, st = ctx.SolveRobinHood(tol=1e-12, raise_on_failure=False)
    finally:
        ctx.SetIterationCallback(None)
    assert st["status"] == K._native.ENOTCONVERGED
    assert [s[0] for s in seen] == [1, 2, 3]


def test_robin_hood_c1_at_size_on_many_ctas(ctx):
    # configuration 1 (1,280 triangles): the rows are spread over several CTAs of one
    # cooperative launch; the reference's KRobinHood needs the same number of checks, and the
    # matrix-free and assembled columns give the same corrections bit for bit
    from kassiopeia_b200 import geometry as G

    fx = golden.load("c1_sphere")
    ctx.SetGeometry(G.icosphere(3))
    x, st = ctx.SolveRobinHood(tol=1e-8)
    assert st["rel_residual"] <= 1e-8
    assert abs(st["iterations"] - int(fx["robinhood_iterations"])) <= 1
    ref_err = rel(fx["robinhood_sigma"], fx["sigma_direct"])
    assert rel(x, fx["sigma_direct"]) <= max(5 * ref_err, 100 * 1e-8)
    xa, sa = ctx.SolveRobinHood(tol=1e-8, assembled=True)
    assert sa["subiterations"] == st["subiterations"]
    np.testing.assert_array_equal(xa, x)


def test_robin_hood_many_ctas_equals_gmres_solution(ctx):
    # 5,120 triangles: twenty CTAs exchange their residual maxima every correction
    from kassiopeia_b200 import geometry as G

    ctx.SetGeometry(G.icosphere(4))
    xg, _ = ctx.Solve(tol=1e-12, mode=K.SOLVE_ASSEMBLED)
    x, st = ctx.SolveRobinHood(tol=1e-9, assembled=True)
    assert st["rel_residual"] <= 1e-9
    assert rel(x, xg) < 1e-6
