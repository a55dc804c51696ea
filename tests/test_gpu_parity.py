"""GPU parity of the direct sum, the boundary-integral matrix and the GMRES solve against the
reference's own FP64 CPU results (golden fixtures from tests/golden/make_golden.py).

Tolerances: the FP64 form must agree with the reference to rounding (1e-12 relative to the
largest value of the quantity, 1e-11 at the near-singular RWG special points); the MIXED form
must stay within 1e-9 relative error of the FP64 results.
"""

import numpy as np
import pytest

import kassiopeia_b200 as K
from kassiopeia_b200 import geometry as G
from oracle import golden

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    """max |a - b| / max |b| per quantity (field vector, potential)"""
    a, b = np.asarray(a), np.asarray(b)
    ef = np.max(np.abs(a[..., :3] - b[..., :3])) / max(np.max(np.abs(b[..., :3])), 1e-300)
    ep = np.max(np.abs(a[..., 3] - b[..., 3])) / max(np.max(np.abs(b[..., 3])), 1e-300)
    return ef, ep


def pointwise(a, b):
    """per-point relative error of |E| and phi"""
    a, b = np.asarray(a), np.asarray(b)
    ef = np.linalg.norm(a[:, :3] - b[:, :3], axis=1) / np.maximum(np.linalg.norm(b[:, :3], axis=1), 1e-300)
    ep = np.abs(a[:, 3] - b[:, 3]) / np.maximum(np.abs(b[:, 3]), 1e-300)
    return ef, ep


@pytest.fixture(scope="module")
def ctx():
    c = K.CUDAElectrostaticContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("shape", ["rect", "tri"])
def test_single_element_special_points(ctx, shape):
    fx = golden.load("integrators")
    ctx.SetGeometry(golden.mesh_from(fx, shape + "_"))
    ctx.SetSigma(np.ones(1))
    P, ref = fx[shape + "_points"], fx[shape + "_field"]
    out = ctx.ElectricFieldAndPotential(P, precision=K.FP64)
    scale = np.max(np.abs(ref), axis=0)
    err = np.abs(out - ref) / scale
    assert np.max(err[:, :3]) < 1e-11, np.argmax(np.max(err[:, :3], axis=1))
    assert np.max(err[:, 3]) < 1e-12
    # the mixed form is FP64 in the near field and bounded by 1e-9 elsewhere
    outm = ctx.ElectricFieldAndPotential(P, precision=K.MIXED)
    errm = np.abs(outm - ref) / scale
    assert np.max(errm) < 1e-9


def _inside_any_wire(m, P):
    inside = np.zeros(len(P), bool)
    for g in m.geom:
        p0, p1, d = g[0:3], g[3:6], g[6]
        L = np.linalg.norm(p1 - p0)
        u = (p1 - p0) / L
        t = (P - p0) @ u
        perp = np.linalg.norm(P - p0 - t[:, None] * u, axis=1)
        inside |= (t >= -d / 2) & (t <= L + d / 2) & (perp < d / 2)
    return inside


def test_line_segments_all_bands(ctx):
    fx = golden.load("lines")
    m = golden.mesh_from(fx)
    ctx.SetGeometry(m)
    # Inside a wire the reference's analytic field divides by Da + Db - L, which is rounding
    # noise there (NaN or ~1e20: KElectrostaticAnalyticLineSegmentIntegrator.cc:63-82), so the
    # field is compared outside the wires and the (well-conditioned) potential everywhere.
    inside = _inside_any_wire(m, fx["points"])
    assert inside.sum() >= 2
    for k in range(m.n):
        s = np.zeros(m.n)
        s[k] = 1.0
        ctx.SetSigma(s)
        ref = fx["element_field"][k][~inside]
        out = ctx.ElectricFieldAndPotential(fx["points"][~inside], precision=K.FP64)
        scale = np.max(np.abs(ref), axis=0)
        assert np.max(np.abs(out - ref) / scale) < 1e-12
        pin = ctx.Potential(fx["points"][inside])
        np.testing.assert_allclose(pin, fx["element_field"][k][inside, 3], rtol=1e-12)
    # a field evaluation that produces NaN (a point on the axis of wire 0) is reported
    s = np.zeros(m.n)
    s[0] = 1.0
    ctx.SetSigma(s)
    with pytest.raises(K.KemcuError) as e:
        ctx.ElectricFieldAndPotential(np.array([[0.5, 0.0, 0.0]]))
    assert e.value.code == K._native.ENONFINITE


def test_sorted_and_unsorted_paths_agree(ctx):
    # >= 4096 points are evaluated in Morton order; the permutation must be invisible
    fx = golden.load("icosphere_L2")
    ctx.SetGeometry(golden.mesh_from(fx))
    ctx.SetSigma(fx["sigma"])
    P = G.shell_points(5000, seed=8)
    big = ctx.ElectricFieldAndPotential(P)
    small = np.concatenate([ctx.ElectricFieldAndPotential(P[i:i + 1000]) for i in range(0, 5000, 1000)])
    np.testing.assert_allclose(big, small, rtol=1e-13, atol=1e-13 * np.abs(big).max())


def test_icosphere_field_fp64_and_mixed(ctx):
    fx = golden.load("icosphere_L2")
    ctx.SetGeometry(golden.mesh_from(fx))
    ctx.SetSigma(fx["sigma"])
    out = ctx.ElectricFieldAndPotential(fx["points"], precision=K.FP64)
    ef, ep = pointwise(out, fx["field"])
    assert ef.max() < 1e-12 and ep.max() < 1e-12, (ef.max(), ep.max())
    outm = ctx.ElectricFieldAndPotential(fx["points"], precision=K.MIXED)
    ef, ep = pointwise(outm, fx["field"])
    assert ef.max() < 1e-9 and ep.max() < 1e-9, (ef.max(), ep.max())
    # potential-only and field-only variants agree with the combined evaluation
    np.testing.assert_allclose(ctx.Potential(fx["points"]), out[:, 3], rtol=1e-14)
    np.testing.assert_allclose(ctx.ElectricField(fx["points"]), out[:, :3], rtol=1e-13, atol=1e-12 * np.abs(out).max())


def test_coax_small_field(ctx):
    fx = golden.load("coax_small")
    ctx.SetGeometry(golden.mesh_from(fx))
    ctx.SetSigma(fx["sigma"])
    out = ctx.ElectricFieldAndPotential(fx["points"], precision=K.FP64)
    ef, ep = pointwise(out, fx["field"])
    assert ef.max() < 1e-11 and ep.max() < 1e-11, (ef.max(), ep.max())
    outm = ctx.ElectricFieldAndPotential(fx["points"], precision=K.MIXED)
    ef, ep = pointwise(outm, fx["field"])
    assert ef.max() < 1e-9 and ep.max() < 1e-9, (ef.max(), ep.max())


def test_matrix_entries_and_matvec(ctx):
    fx = golden.load("mixed_small")
    m = golden.mesh_from(fx)
    ctx.SetGeometry(m)
    A = np.stack([ctx.Multiply(np.eye(m.n)[j]) for j in range(m.n)], axis=1)
    scale = np.max(np.abs(fx["A"]), axis=1, keepdims=True)
    assert np.max(np.abs(A - fx["A"]) / scale) < 1e-12
    assert abs(ctx.MatrixElement(2, 5) - fx["A"][2, 5]) <= 1e-12 * scale[2, 0]
    np.testing.assert_allclose(ctx.RHS(), fx["b"], rtol=0, atol=0)
    y = ctx.Multiply(fx["xv"])
    assert np.max(np.abs(y - fx["Axv"])) < 1e-12 * np.max(np.abs(fx["Axv"]))
    ya = ctx.Multiply(fx["xv"], assembled=True)
    assert np.max(np.abs(ya - fx["Axv"])) < 1e-12 * np.max(np.abs(fx["Axv"]))
    # multi-RHS matvec equals column-by-column application
    X = np.stack([fx["xv"], np.eye(m.n)[3], -2 * fx["xv"]])
    Y = ctx.Multiply(X)
    for r in range(3):
        np.testing.assert_allclose(Y[r], ctx.Multiply(X[r]), rtol=1e-13, atol=1e-12 * np.abs(Y).max())


@pytest.mark.parametrize("nrhs", [2, 3, 8])
def test_assembled_multi_rhs_against_reference_matrix(ctx, nrhs):
    # the several-right-hand-side dense kernel (FP64 tensor cores) on an operator whose size is
    # not a multiple of its 64-row warp tiles or 4-column chunks, with 2, 3 or 8 right-hand sides
    fx = golden.load("mixed_small")
    m = golden.mesh_from(fx)
    ctx.SetGeometry(m)
    rng = np.random.default_rng(5)
    X = rng.standard_normal((nrhs, m.n))
    ref = X @ fx["A"].T
    scale = np.abs(X) @ np.abs(fx["A"]).T
    Y64 = ctx.Multiply(X, assembled=True)
    assert np.max(np.abs(Y64 - ref) / scale) < 1e-12
    for r in range(nrhs):
        np.testing.assert_allclose(Y64[r], ctx.Multiply(X[r], assembled=True), rtol=0,
                                   atol=1e-14 * scale[r].max())
    # FP32 operator copy: entries rounded to FP32 (2^-24 relative), products and sums in FP64
    Y32 = ctx.Multiply(X, precision=K.MIXED, assembled=True)
    assert np.max(np.abs(Y32 - ref) / scale) < 1e-7
    A32 = fx["A"].astype(np.float32).astype(np.float64)
    assert np.max(np.abs(Y32 - X @ A32.T) / scale) < 1e-13


def test_assembled_multi_rhs_ragged_coax(ctx):
    # 1,554 rectangles and triangles (1554 = 24 x 64 + 18 rows, column splits not multiples of
    # 4): the tensor-core dense product against the matrix-free FP64 matvec, 5 right-hand sides
    m = G.coax(n_phi=21, n_z=31, n_cap_rings=3)
    ctx.SetGeometry(m)
    rng = np.random.default_rng(9)
    X = rng.standard_normal((5, m.n))
    Yf = ctx.Multiply(X)
    Ya = ctx.Multiply(X, assembled=True)
    Y32 = ctx.Multiply(X, precision=K.MIXED, assembled=True)
    norm = np.abs(Yf).max(axis=1, keepdims=True)
    assert np.max(np.abs(Ya - Yf) / norm) < 1e-13
    assert np.max(np.abs(Y32 - Yf) / norm) < 1e-6


def test_gmres_plain_matches_reference(ctx):
    # oracle: the direct solution of the reference's own boundary-integral matrix. The
    # reference GMRES converges in the same number of iterations on its implicit estimate,
    # but its SVD least-squares step returns a sigma with true residual ~2e-5 here.
    fx = golden.load("icosphere_L2")
    ctx.SetGeometry(golden.mesh_from(fx))
    x, st = ctx.Solve(tol=1e-12, mode=K.SOLVE_PLAIN)
    assert np.max(np.abs(x - fx["sigma_direct"])) / np.max(np.abs(fx["sigma_direct"])) < 1e-9
    assert abs(st["iterations"] - int(fx["iterations"])) <= 1
    np.testing.assert_array_equal(ctx.GetSigma(), x)
    # the reference's own iterate is within its (larger) true-residual error of ours
    assert np.max(np.abs(x - fx["sigma"])) / np.max(np.abs(x)) < 50 * float(fx["gmres_true_residual"])


@pytest.mark.parametrize("mode", [K.SOLVE_MIXED, K.SOLVE_ASSEMBLED])
def test_gmres_refinement_modes(ctx, mode):
    fx = golden.load("icosphere_L2")
    ctx.SetGeometry(golden.mesh_from(fx))
    x, st = ctx.Solve(tol=1e-12, mode=mode)
    assert st["rel_residual"] <= 1e-12
    assert np.max(np.abs(x - fx["sigma_direct"])) / np.max(np.abs(fx["sigma_direct"])) < 1e-9
    assert st["outer"] >= 1 and st["fp64_matvecs"] == st["outer"]


def test_gmres_mixed_boundaries(ctx):
    fx = golden.load("mixed_small")
    ctx.SetGeometry(golden.mesh_from(fx))
    x, st = ctx.Solve(tol=1e-12, mode=K.SOLVE_PLAIN)
    assert np.max(np.abs(x - fx["x_direct"])) / np.max(np.abs(fx["x_direct"])) < 1e-9


def test_gmres_coax_small(ctx):
    fx = golden.load("coax_small")
    ctx.SetGeometry(golden.mesh_from(fx))
    x, st = ctx.Solve(tol=1e-12, mode=K.SOLVE_PLAIN)
    ref = fx["sigma_direct"]
    assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) < 1e-9
    xm, stm = ctx.Solve(tol=1e-12, mode=K.SOLVE_MIXED)
    assert np.max(np.abs(xm - ref)) / np.max(np.abs(ref)) < 1e-9
    xa, sta = ctx.Solve(tol=1e-12, mode=K.SOLVE_ASSEMBLED)
    assert np.max(np.abs(xa - ref)) / np.max(np.abs(ref)) < 1e-9


def test_multi_rhs_solve(ctx):
    m = G.icosphere(2)
    ctx.SetGeometry(m)
    rng = np.random.default_rng(3)
    B = np.stack([np.ones(m.n), rng.uniform(-1, 1, m.n), np.linspace(0, 2, m.n)])
    X, st = ctx.Solve(B, tol=1e-11, mode=K.SOLVE_PLAIN)
    for r in range(3):
        xr, _ = ctx.Solve(B[r], tol=1e-11, mode=K.SOLVE_PLAIN)
        assert np.max(np.abs(X[r] - xr)) <= 1e-9 * np.max(np.abs(xr))
    XA, _ = ctx.Solve(B, tol=1e-11, mode=K.SOLVE_ASSEMBLED)
    assert np.max(np.abs(XA - X)) <= 1e-9 * np.max(np.abs(X))


def test_iteration_callback_terminates(ctx):
    ctx.SetGeometry(G.icosphere(2))
    seen = []

    def cb(it, r):
        seen.append((it, r))
        return it >= 3

    ctx.SetIterationCallback(cb)
    try:
        x, st = ctx.Solve(tol=1e-14, mode=K.SOLVE_PLAIN, raise_on_failure=False)
    finally:
        ctx.SetIterationCallback(None)
    assert st["status"] == K._native.ENOTCONVERGED
    assert [s[0] for s in seen] == [1, 2, 3]
    assert seen[0][1] > seen[2][1]


def test_invalid_inputs_are_reported(ctx):
    m = G.icosphere(1)
    bad = G.Mesh(m.shape.copy(), m.boundary.copy(), m.geom.copy(), m.value.copy())
    bad.geom[3, 4] = np.nan
    with pytest.raises(K.KemcuError) as e:
        ctx.SetGeometry(bad)
    assert e.value.code == K._native.EINVAL
    fresh = K.CUDAElectrostaticContext(0)
    with pytest.raises(K.KemcuError) as e:
        fresh.ElectricFieldAndPotential(np.zeros((2, 3)))
    assert e.value.code == K._native.ESTATE
    fresh.close()


def test_empty_and_boundary_sized_point_sets(ctx):
    # n = 0 is a no-op; sizes around the Morton-ordering threshold (4,096) and a ragged last
    # CTA give the same values as evaluating the points one block at a time
    fx = golden.load("icosphere_L2")
    ctx.SetGeometry(golden.mesh_from(fx))
    ctx.SetSigma(fx["sigma"])
    assert ctx.ElectricFieldAndPotential(np.zeros((0, 3))).shape == (0, 4)
    P = G.shell_points(4097 + 129, seed=21)
    ref = np.concatenate([ctx.ElectricFieldAndPotential(P[i:i + 128]) for i in range(0, len(P), 128)])
    for n in (1, 127, 4095, 4096, 4097, 4097 + 129):
        out = ctx.ElectricFieldAndPotential(P[:n])
        np.testing.assert_allclose(out, ref[:n], rtol=1e-13, atol=1e-13 * np.abs(ref).max())


def test_cube_capacitance(ctx):
    # the reference's CubeCapacitanceTest box (384 rectangles, refined towards the edges):
    # device solves against the oracle's direct solution and the accepted 0.6606785 (tol 1e-2)
    from oracle import port

    m = G.cube()
    ctx.SetGeometry(m)
    A, b = port.PortProblem(m).matrix()
    ref = np.linalg.solve(A, b)
    for mode in (K.SOLVE_PLAIN, K.SOLVE_MIXED, K.SOLVE_ASSEMBLED):
        x, _ = ctx.Solve(tol=1e-12, mode=mode)
        assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) < 1e-9, mode
        c = float((x * m.areas()).sum()) / (4 * np.pi * 8.8541878128e-12)
        assert abs(c - 0.6606785) < 1e-2
