"""kemcu_field_dev_noalloc: the direct sum for callers that cannot call cudaMalloc while they
evaluate fields (for example a framework whose pool allocator owns all device memory, or a
loop that must not take the implicit device synchronisation of cudaMalloc / cudaFree). It
takes the caller's device buffers and keeps its partial sums in a fixed 8 MiB device array.

Collected last (file name) so that a stopped-at-first-failure run has already run every other
test; it also passes on its own in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    import kassiopeia_b200 as K
    from kassiopeia_b200 import _native as N
    from kassiopeia_b200 import geometry as G

    L = N.lib()
    ctx = K.CUDAElectrostaticContext(0)
    mesh = G.coax(n_phi=40, n_z=40, n_cap_rings=4)  # 3,200 rectangles + 640 cap triangles
    ctx.SetGeometry(mesh)
    rng = np.random.default_rng(3)
    ctx.SetSigma(np.where(mesh.value < -1.0, -1e-8, 1e-8) * (1 + 0.1 * rng.normal(size=mesh.n)))
    limit = N.header_constant("KEMCU_NOALLOC_MAX_POINTS")
    assert limit * 32 == N.header_constant("KEMCU_NOALLOC_SCRATCH_BYTES")
    # two calls in a row with different sizes: the second reuses (and must fully overwrite)
    # the scratch the first one left behind
    for n_pts, prec in ((3000, K.MIXED), (20000, K.FP64)):
        P = torch.from_numpy(G.gap_points(n_pts, seed=n_pts)).cuda()
        ref = torch.zeros((n_pts, 4), dtype=torch.float64, device="cuda")
        out = torch.full((n_pts, 4), float("nan"), dtype=torch.float64, device="cuda")
        assert L.kemcu_field_dev(ctx._h, C.c_void_p(P.data_ptr()), n_pts, C.c_void_p(ref.data_ptr()), prec,
                                 K.FIELD_AND_POTENTIAL) == 0
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        rc = L.kemcu_field_dev_noalloc(ctx._h, C.c_void_p(P.data_ptr()), n_pts, C.c_void_p(out.data_ptr()), prec,
                                       K.FIELD_AND_POTENTIAL)
        assert rc == 0, L.kemcu_last_error(ctx._h).decode()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free_before  # nothing was allocated
        r, o = ref.cpu().numpy(), out.cpu().numpy()
        # same kernels, same element splits up to the scratch cap: agreement to rounding
        assert np.max(np.abs(o - r) / np.abs(r).max(axis=0)) < 1e-12
    # the largest accepted call (one partial sum per point fills the scratch exactly) against
    # the allocating entry point, then one point more, refused with a clear error
    P = torch.from_numpy(G.gap_points(limit + 1, seed=5)).cuda()
    ref = torch.zeros((limit, 4), dtype=torch.float64, device="cuda")
    out = torch.full((limit + 1, 4), float("nan"), dtype=torch.float64, device="cuda")
    assert L.kemcu_field_dev(ctx._h, C.c_void_p(P.data_ptr()), limit, C.c_void_p(ref.data_ptr()), K.MIXED,
                             K.POTENTIAL) == 0
    rc = L.kemcu_field_dev_noalloc(ctx._h, C.c_void_p(P.data_ptr()), limit, C.c_void_p(out.data_ptr()), K.MIXED,
                                   K.POTENTIAL)
    assert rc == 0, L.kemcu_last_error(ctx._h).decode()
    r, o = ref.cpu().numpy()[:, 3], out.cpu().numpy()[:limit, 3]
    assert np.max(np.abs(o - r)) / np.abs(r).max() < 1e-12
    rc = L.kemcu_field_dev_noalloc(ctx._h, C.c_void_p(P.data_ptr()), limit + 1, C.c_void_p(out.data_ptr()),
                                   K.FP64, K.FIELD_AND_POTENTIAL)
    assert rc == N.EINVAL
    assert "at most" in L.kemcu_last_error(ctx._h).decode()
    ctx.close()


def test_noalloc_axisymmetric_elements():
    # conic sections and rings take the same no-allocation entry point (element range split
    # over the grid, partial sums in the fixed scratch)
    import torch

    import kassiopeia_b200 as K
    from kassiopeia_b200 import _native as N
    from kassiopeia_b200 import geometry as G

    L = N.lib()
    ctx = K.CUDAElectrostaticContext(0)
    mesh = G.conic_coax(n_z=40, n_cap=6, n_rings=4)
    ctx.SetGeometry(mesh)
    ctx.Solve(tol=1e-10, mode=K.SOLVE_ASSEMBLED)
    n_pts = 3000
    P = torch.from_numpy(G.gap_points(n_pts, seed=11)).cuda()
    ref = torch.zeros((n_pts, 4), dtype=torch.float64, device="cuda")
    out = torch.full((n_pts, 4), float("nan"), dtype=torch.float64, device="cuda")
    assert L.kemcu_field_dev(ctx._h, C.c_void_p(P.data_ptr()), n_pts, C.c_void_p(ref.data_ptr()), K.FP64,
                             K.FIELD_AND_POTENTIAL) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = L.kemcu_field_dev_noalloc(ctx._h, C.c_void_p(P.data_ptr()), n_pts, C.c_void_p(out.data_ptr()), K.FP64,
                                   K.FIELD_AND_POTENTIAL)
    assert rc == 0, L.kemcu_last_error(ctx._h).decode()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
    r, o = ref.cpu().numpy(), out.cpu().numpy()
    assert np.max(np.abs(o - r) / np.abs(r).max(axis=0)) < 1e-12
    ctx.close()
