"""torch.autograd.Function around the direct sum and its adjoint (kemcu_field_vjp).

Used to check the hand-written adjoint kernels with torch's own machinery (gradcheck,
finite differences); the computation itself runs in libkemcu on the GPU. Tensors are CPU
float64 at this interface because the C ABI takes host buffers.

    out = DirectSumField.apply(sigma, vertices, points, kctx, template_mesh, precision)

sigma: [N]; vertices: [N, 3, 3] defining vertices (P0, P1, P2) of triangles (rectangles:
P0, P0 + A N1, P0 + B N2); points: [M, 3]; out: [M, 4] = (Ex, Ey, Ez, phi).
"""

from __future__ import annotations

import numpy as np
import torch

from . import FP64
from .geometry import RECTANGLE, TRIANGLE, Mesh


def mesh_with_vertices(template: Mesh, vertices: np.ndarray) -> Mesh:
    """Template mesh with triangle / rectangle geometry replaced by the given vertices."""
    g = template.geom.copy()
    v = np.asarray(vertices, np.float64).reshape(-1, 3, 3)
    planar = (template.shape == TRIANGLE) | (template.shape == RECTANGLE)
    a = v[planar, 1] - v[planar, 0]
    b = v[planar, 2] - v[planar, 0]
    A = np.linalg.norm(a, axis=1)
    B = np.linalg.norm(b, axis=1)
    g[planar, 0] = A
    g[planar, 1] = B
    g[planar, 2:5] = v[planar, 0]
    g[planar, 5:8] = a / A[:, None]
    g[planar, 8:11] = b / B[:, None]
    return Mesh(template.shape, template.boundary, g, template.value, template.name, template.meta)


def vertices_of(mesh: Mesh) -> np.ndarray:
    g = mesh.geom
    v = np.zeros((mesh.n, 3, 3))
    v[:, 0] = g[:, 2:5]
    v[:, 1] = g[:, 2:5] + g[:, 0:1] * g[:, 5:8]
    v[:, 2] = g[:, 2:5] + g[:, 1:2] * g[:, 8:11]
    return v


class DirectSumField(torch.autograd.Function):
    @staticmethod
    def forward(ctx, sigma, vertices, points, kctx, template, precision=FP64):
        mesh = mesh_with_vertices(template, vertices.detach().cpu().numpy())
        kctx.SetGeometry(mesh)
        kctx.SetSigma(sigma.detach().cpu().numpy())
        P = points.detach().cpu().numpy()
        out = kctx.ElectricFieldAndPotential(P, precision=precision)
        ctx.save_for_backward(sigma, vertices, points)
        ctx.kctx, ctx.template, ctx.precision = kctx, template, precision
        return torch.from_numpy(out)

    @staticmethod
    def backward(ctx, grad_out):
        sigma, vertices, points = ctx.saved_tensors
        kctx = ctx.kctx
        mesh = mesh_with_vertices(ctx.template, vertices.detach().cpu().numpy())
        kctx.SetGeometry(mesh)
        kctx.SetSigma(sigma.detach().cpu().numpy())
        ds, dv = kctx.FieldVJP(points.detach().cpu().numpy(), grad_out.detach().cpu().numpy(),
                               precision=ctx.precision)
        return (torch.from_numpy(ds), torch.from_numpy(dv.reshape(-1, 3, 3)), None, None, None, None)
