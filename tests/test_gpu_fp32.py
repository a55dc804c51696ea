"""The FP32 far-field form (precision KEMCU_FP32): cubature nodes of triangles and rectangles in
FP32 relative to each element's FP64 centre distance, the analytic near field, wires and the
compensated element sums in FP64. It trades accuracy for speed: ~1e-7 relative per element, a
few 1e-8 of the largest value on whole fields. With FP64 iterative refinement (solve mode
KEMCU_SOLVE_FP32) the charge densities are FP64-accurate."""

import numpy as np
import pytest

import kassiopeia_b200 as K
from kassiopeia_b200 import _native as N
from kassiopeia_b200 import geometry as G
from oracle import golden

pytestmark = pytest.mark.gpu

# relative to the largest value of each quantity over the points
TOL_FP32 = 2e-7


def rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.fixture(scope="module")
def ctx():
    c = K.CUDAElectrostaticContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", ["icosphere_L2", "coax_small"])
def test_fp32_field_against_reference(ctx, name):
    fx = golden.load(name)
    ctx.SetGeometry(golden.mesh_from(fx))
    ctx.SetSigma(fx["sigma"])
    out = ctx.ElectricFieldAndPotential(fx["points"], precision=K.FP32)
    ref = fx["field"]
    e_f, e_p = rel(out[:, :3], ref[:, :3]), rel(out[:, 3], ref[:, 3])
    assert e_f < TOL_FP32 and e_p < TOL_FP32, (e_f, e_p)
    # a genuinely reduced form: not the FP64 result
    assert e_f > 1e-12 or e_p > 1e-12
    # the analytic near field stays FP64: at the IntegratorsTest special points (all in the RWG
    # band or next to it) FP32 equals FP64 where the analytic integral applies
    it = golden.load("integrators")
    ctx.SetGeometry(golden.mesh_from(it, "rect_"))
    ctx.SetSigma(np.ones(1))
    P = it["rect_points"][:16]
    a = ctx.ElectricFieldAndPotential(P, precision=K.FP32)
    b = ctx.ElectricFieldAndPotential(P, precision=K.FP64)
    assert rel(a, b) < TOL_FP32


def test_fp32_config2_field_and_matvec():
    fx = golden.load("c2_coax")
    m = G.coax()
    with K.CUDAElectrostaticContext(0) as c:
        c.SetGeometry(m)
        c.SetSigma(G.coax_density(m))
        out = c.ElectricFieldAndPotential(fx["points"], precision=K.FP32)
        assert rel(out[:, :3], fx["field"][:, :3]) < TOL_FP32
        assert rel(out[:, 3], fx["field"][:, 3]) < TOL_FP32
        x = np.random.default_rng(int(fx["x_seed"])).normal(size=m.n) * 1e-8
        assert rel(c.Multiply(x, precision=K.FP32)[fx["rows"]], fx["Ax"]) < TOL_FP32


@pytest.mark.parametrize("tol", [1e-10, 1e-12])
def test_fp32_refined_solve_is_fp64_accurate(ctx, tol):
    fx = golden.load("c1_sphere")
    ctx.SetGeometry(G.icosphere(3))
    x, st = ctx.Solve(tol=tol, mode=K.SOLVE_FP32)
    assert st["rel_residual"] <= tol and st["outer"] >= 2 and st["low_matvecs"] > st["fp64_matvecs"]
    r = ctx.Multiply(fx["sigma_direct"] - x, precision=K.FP64)
    assert np.linalg.norm(r) / np.linalg.norm(fx["b"]) <= 1.5 * tol
    if tol <= 1e-12:
        assert rel(x, fx["sigma_direct"]) < 1e-9


def test_fp32_is_refused_where_not_offered(ctx):
    ctx.SetGeometry(G.icosphere(2))
    ctx.SetSigma(np.full(320, 1e-11))
    P = G.shell_points(64, seed=1)
    with pytest.raises(K.KemcuError) as e:
        ctx.FieldVJP(P, np.ones((64, 4)), precision=K.FP32)
    assert e.value.code == N.EINVAL
    with pytest.raises(K.KemcuError) as e:
        ctx.TrackRK8(G.electrons(4, seed=1), 1e-11, 4, precision=K.FP32)
    assert e.value.code == N.EINVAL
