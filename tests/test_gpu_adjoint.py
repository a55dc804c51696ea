"""GPU adjoint kernels: dL/dsigma and dL/dvertices of L = sum_p w_p . (E, phi)(P_p) against the
reference's FP64 per-element integrals and central differences of the reference field solver
(golden fixture adjoint), against this library's own forward sum, and through torch.autograd."""

import numpy as np
import pytest
import torch

import kassiopeia_b200 as K
from kassiopeia_b200 import autograd as KA
from kassiopeia_b200 import geometry as G
from oracle import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = K.CUDAElectrostaticContext(0)
    yield c
    c.close()


@pytest.mark.parametrize("precision", [K.FP64, K.MIXED])
def test_vjp_matches_reference(ctx, precision):
    fx = golden.load("adjoint")
    ctx.SetGeometry(golden.mesh_from(fx))
    ctx.SetSigma(fx["sigma"])
    ds, dv = ctx.FieldVJP(fx["points"], fx["w"], precision=precision)
    tol_s = 1e-12 if precision == K.FP64 else 1e-9
    assert np.max(np.abs(ds - fx["dsigma"])) <= tol_s * np.max(np.abs(fx["dsigma"]))
    # vertex gradients vs central differences of the reference (h = 1e-6 m): 1e-6 relative
    fd = fx["dvert_fd"]
    mine = dv[fx["elems"]]
    assert np.max(np.abs(mine - fd)) <= 1e-6 * np.max(np.abs(fd)), np.max(np.abs(mine - fd)) / np.max(np.abs(fd))


def test_vjp_sigma_is_the_transpose_of_the_forward_sum(ctx):
    m = G.icosphere(2)
    ctx.SetGeometry(m)
    rng = np.random.default_rng(5)
    sigma = rng.normal(size=m.n) * 1e-11
    P = np.concatenate([G.shell_points(40, seed=9), G.shell_points(8, 1.01, 1.05, seed=10)])  # incl. RWG pairs
    w = rng.normal(size=(P.shape[0], 4))
    ctx.SetSigma(sigma)
    ds, _ = ctx.FieldVJP(P, w, want_vertices=False)
    for _ in range(3):
        d = rng.normal(size=m.n)
        ctx.SetSigma(d)
        L = np.sum(w * ctx.ElectricFieldAndPotential(P))
        assert abs(ds @ d - L) <= 1e-12 * np.sum(np.abs(w * ctx.ElectricFieldAndPotential(P)))


def test_vertex_gradient_near_field_pairs_by_finite_differences(ctx):
    # points within the RWG band exercise the device-side central differences of the
    # analytic integral; compare with differences of this library's own forward FP64 sum
    m = G.icosphere(1)
    rng = np.random.default_rng(6)
    sigma = 1e-11 * (1 + 0.1 * rng.normal(size=m.n))
    P = G.shell_points(12, 1.02, 1.3, seed=12)
    w = rng.normal(size=(P.shape[0], 4)) * np.array([0.1, 0.1, 0.1, 1.0])
    verts = KA.vertices_of(m)
    ctx.SetGeometry(m)
    ctx.SetSigma(sigma)
    _, dv = ctx.FieldVJP(P, w, want_sigma=False)

    def L(vv):
        ctx.SetGeometry(KA.mesh_with_vertices(m, vv))
        ctx.SetSigma(sigma)
        return np.sum(w * ctx.ElectricFieldAndPotential(P))

    h = 1e-6
    worst = 0.0
    for j in (0, 5, 33, 79):
        for c in range(9):
            vp, vm = verts.copy(), verts.copy()
            vp[j, c // 3, c % 3] += h
            vm[j, c // 3, c % 3] -= h
            fd = (L(vp) - L(vm)) / (2 * h)
            worst = max(worst, abs(dv[j, c] - fd) / np.max(np.abs(dv)))
    assert worst < 1e-6, worst


def test_torch_autograd_function(ctx):
    m = G.icosphere(1)
    rng = np.random.default_rng(8)
    sigma = torch.tensor(1e-11 * (1 + 0.1 * rng.normal(size=m.n)), dtype=torch.float64, requires_grad=True)
    verts = torch.tensor(KA.vertices_of(m), dtype=torch.float64, requires_grad=True)
    P = torch.tensor(G.shell_points(6, seed=13), dtype=torch.float64)
    out = KA.DirectSumField.apply(sigma, verts, P, ctx, m, K.FP64)
    wt = torch.tensor(rng.normal(size=tuple(out.shape)), dtype=torch.float64)
    (out * wt).sum().backward()
    ctx.SetGeometry(m)
    ctx.SetSigma(sigma.detach().numpy())
    ds, dv = ctx.FieldVJP(P.numpy(), wt.numpy())
    np.testing.assert_allclose(sigma.grad.numpy(), ds, rtol=1e-14, atol=0)
    np.testing.assert_allclose(verts.grad.numpy().reshape(-1, 9), dv, rtol=1e-14, atol=0)
    # torch's own finite-difference check on the charge densities (linear, so exact up to rounding)
    s_small = sigma.detach().clone().requires_grad_(True)
    f = lambda s: KA.DirectSumField.apply(s, verts.detach(), P, ctx, m, K.FP64)  # noqa: E731
    assert torch.autograd.gradcheck(f, (s_small,), eps=1e-13, atol=1e-9, rtol=1e-6)
