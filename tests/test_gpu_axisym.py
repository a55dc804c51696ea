"""Axisymmetric elements (conic sections and rings, KElectrostaticAnalyticConicSectionIntegrator
and ...RingIntegrator) on the device against the reference (golden fixture axisym): single
elements at points in every quadrature band of the conic-section integral, and two solved
problems (a conic-section sphere, a conic coax with rings): matrix, solves, field."""

import numpy as np
import pytest

import kassiopeia_b200 as K
from kassiopeia_b200 import geometry as G
from oracle import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = K.CUDAElectrostaticContext(0)
    yield c
    c.close()


def _rel(a, b):
    # per point: |E| error over |E| and phi error over |phi| (reference values as scale)
    e = np.linalg.norm(a[:, :3] - b[:, :3], axis=1) / np.maximum(np.linalg.norm(b[:, :3], axis=1), 1e-300)
    p = np.abs(a[:, 3] - b[:, 3]) / np.maximum(np.abs(b[:, 3]), 1e-300)
    return e, p


def _band_d(geom, pts):
    # the conic-section integrator's band variable D = |Da + Db - L| / L
    r0, z0, r1, z1 = geom[:4]
    r = np.hypot(pts[:, 0], pts[:, 1])
    L = np.hypot(r1 - r0, z1 - z0)
    return np.abs(np.hypot(z0 - pts[:, 2], r0 - r) + np.hypot(z1 - pts[:, 2], r1 - r) - L) / L


@pytest.mark.parametrize("name", ["cone", "ring"])
def test_single_element_every_band(ctx, name):
    fx = golden.load("axisym")
    ctx.SetGeometry(golden.mesh_from(fx, name + "_"))
    ctx.SetSigma(np.ones(1))
    pts = fx[name + "_points"]
    out = ctx.ElectricFieldAndPotential(pts)
    e, p = _rel(out, fx[name + "_field"])
    assert p.max() < 1e-12, p.max()
    if name == "cone":
        # D < 5e-4: the subdivided near branch. On and next to the generator its field is a
        # sum of terms of both signs far larger than the result (1 / eta near the foot point),
        # so one rounding apart in any term shows at ~1e-8 of the result there
        near = _band_d(fx["cone_geom"][0], pts) < 5e-4
        assert near.sum() >= 10 and (~near).sum() >= 60
        assert e[~near].max() < 1e-11 and e[near].max() < 1e-6, (e[~near].max(), e[near].max())
    else:
        assert e.max() < 1e-11, e.max()
    # precision MIXED evaluates axisymmetric elements in FP64 as well
    np.testing.assert_array_equal(ctx.ElectricFieldAndPotential(fx[name + "_points"], precision=K.MIXED), out)


@pytest.mark.parametrize("name", ["sphere", "coax"])
def test_matrix_solve_and_field(ctx, name):
    fx = golden.load("axisym")
    m = golden.mesh_from(fx, name + "_")
    ctx.SetGeometry(m)
    n = m.n
    A = np.stack([ctx.Multiply(np.eye(n)[j]) for j in range(n)], axis=1)
    scale = np.max(np.abs(fx[name + "_A"]), axis=1, keepdims=True)
    assert np.max(np.abs(A - fx[name + "_A"]) / scale) < 1e-12
    assert abs(ctx.MatrixElement(3, 7) - fx[name + "_A"][3, 7]) <= 1e-12 * scale[3, 0]
    np.testing.assert_array_equal(ctx.RHS(), fx[name + "_b"])
    ref = fx[name + "_sigma"]
    for mode in (K.SOLVE_PLAIN, K.SOLVE_ASSEMBLED):
        x, st = ctx.Solve(tol=1e-12, mode=mode)
        assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) < 1e-9, (mode, st)
    # the assembled operator (FP64 copy) against the reference matrix, 3 right-hand sides
    X = np.random.default_rng(3).standard_normal((3, n))
    Y = ctx.Multiply(X, assembled=True)
    assert np.max(np.abs(Y - X @ fx[name + "_A"].T) / (np.abs(X) @ np.abs(fx[name + "_A"]).T)) < 1e-12
    ctx.SetSigma(ref)
    e, p = _rel(ctx.ElectricFieldAndPotential(fx[name + "_points"]), fx[name + "_field"])
    assert e.max() < 1e-11 and p.max() < 1e-12, (e.max(), p.max())


def test_capacitance_of_a_finer_sphere(ctx):
    # 400 sections, solved on the device only: C / (4 pi eps0 R) closer to 1 than at 120
    m = G.conic_sphere(400)
    ctx.SetGeometry(m)
    x, _ = ctx.Solve(tol=1e-12, mode=K.SOLVE_ASSEMBLED)
    c = float((x * m.areas()).sum()) / (4 * np.pi * 8.8541878128e-12)
    assert abs(c - 1.0) < abs(float(golden.load("axisym")["sphere_capacitance"]) - 1.0)


def test_axisymmetric_limits(ctx):
    cone = G.axisymmetric(G.CONIC_SECTION, 0.5, 0.0, 0.6, 0.1)
    with pytest.raises(K.KemcuError):  # planar and axisymmetric elements in one context
        ctx.SetGeometry(cone.concat(G.icosphere(1)))
    ctx.SetGeometry(cone)
    ctx.SetSigma(np.ones(1))
    st = G.electrons(4, seed=3)
    with pytest.raises(K.KemcuError):
        ctx.TrackRK8(st, 1e-11, 4)
    with pytest.raises(K.KemcuError):  # matrix-free Robin Hood columns are planar-only
        ctx.SolveRobinHood()


def test_robin_hood_on_the_assembled_axisymmetric_operator(ctx):
    fx = golden.load("axisym")
    ctx.SetGeometry(golden.mesh_from(fx, "sphere_"))
    x, st = ctx.SolveRobinHood(tol=1e-10, assembled=True)
    assert st["rel_residual"] <= 1e-10 and st["subiterations"] > 0
    ref = fx["sphere_sigma"]
    assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) < 1e-7


def test_disk_capacitance(ctx):
    # the reference's DiskCapacitanceTest mesh (128 flat conic sections): coplanar neighbours
    # put every collocation point on the extension of the other generators, the near branch
    # with the foot point outside the generator; device solves against the oracle's direct
    # solution and the known answer C = 8 eps0 R (test tolerance 1e-2)
    from oracle import port

    m = G.conic_disk()
    ctx.SetGeometry(m)
    A, b = port.PortProblem(m).matrix()
    ref = np.linalg.solve(A, b)
    for mode in (K.SOLVE_PLAIN, K.SOLVE_ASSEMBLED):
        x, _ = ctx.Solve(tol=1e-12, mode=mode)
        assert np.max(np.abs(x - ref)) / np.max(np.abs(ref)) < 1e-9
        assert abs(float((x * m.areas()).sum()) / 8.8541878128e-12 - 8.0) < 1e-2
