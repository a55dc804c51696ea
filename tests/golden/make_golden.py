"""Generate the golden fixtures in this directory from the reference's own FP64 CPU code.

    make -C oracle ref          # builds oracle/_ref/libkemref.so from the reference tree
    python tests/golden/make_golden.py

Every array is produced by unmodified reference classes driven through oracle/ref_harness.cc
(KSurfaceContainer + KEBIFactory::MakeNumeric() + KIntegratingFieldSolver /
KBoundaryIntegralMatrix / KSimpleIterativeKrylovSolver<double, KGeneralizedMinimalResidual> /
KSMathRK8). Inputs are seeded; the seeds are fixed below.

Fixtures:
  rules          nodes and weights of the six cubature rules on canonical elements
  integrators    the IntegratorsTest.cc rectangle and triangle (UnitTest/KEMField/Fields/src/
                 IntegratorsTest.cc:28-60, 106-135) with their evaluation points (corner, on
                 surface, centroid, in-plane far, on side line, arbitrary) plus seeded near
                 points, vertices and edge midpoints: per-element normalised field and potential
  lines          wires: near (analytic, inside and outside the wire), 16-node and 4-node bands
  icosphere_L2   320-triangle sphere at 1 V: GMRES sigma (rel. tol 1e-12), field at shell and
                 near-surface points, capacitance
  mixed_small    triangles (Dirichlet), rectangles (Neumann, flux 0.4) and wires (Dirichlet):
                 full boundary-integral matrix, right-hand side, GMRES solution
  coax_small     reduced coax (960 rectangles + 288 cap triangles): sigma and gap field
  rk8            4 electrons x 40 RK8 steps of 1e-11 s in the icosphere_L2 field
  robinhood      KRobinHood<double> (default residual-check interval, tolerances 1e-8 and
                 1e-10) on the icosphere_L2 and mixed_small meshes: sigma, iterations, residual
  axisym         conic sections and rings (KElectrostaticAnalyticConicSectionIntegrator /
                 ...RingIntegrator): per-element field of one conic section and one ring at
                 points in every quadrature band of the conic section (20, 100, 500 intervals
                 and the subdivided near branch, on and beyond the generator, on the axis); a
                 120-section sphere and a conic coax with rings: matrix, right-hand side,
                 direct solution, field at seeded points
  c1_sphere      configuration 1 at its stated size: 1,280-triangle icosphere at 1 V, the
                 reference's matrix solved directly (and its GMRES at 1e-10 for the record), its
                 Robin Hood at 1e-8, the field of the direct density at the 10,000 seeded shell
                 points
  c2_coax        configuration 2 at its stated size (44,000 elements): the field of a fixed
                 density (geometry.coax_density) at 200 seeded gap points; 64 sampled rows of
                 the boundary-integral matrix: 64 entries each (diagonal, nearest neighbours,
                 seeded columns) and the rows of A x for a seeded x
  c3_tracks      configuration 3's tracking in the configuration-1 field: 16 electrons x up to
                 1,000 RK8 steps of 1e-11 s, stopping at the sphere (|x| <= 1 m); states every
                 50 steps, the steps taken and the final states
  c4_adjoint     configuration 4 at its stated size: 20,480-triangle sphere, perturbed density
                 (geometry.sphere_density, seed 4), 4,096 probes, L = sum_p (E_z + phi):
                 dL/dsigma for 512 seeded elements and central differences (h = 1e-6 m) of L
                 over the 9 vertex coordinates of 16 elements whose quadrature bands the
                 perturbation leaves unchanged at every probe
  c5_rings       configuration 5 at its stated size (100,000 jittered triangles): 64 sampled
                 matrix rows, 64 entries each, and the rows of A x for 8 seeded right-hand sides
  fftm           the reference's fast-multipole code (oracle/_ref/libkemref_fm.so, make -C oracle
                 fm): analytic multipole moments (degree 10) of the mixed_small elements about
                 seeded origins; a seeded degree-8 local expansion evaluated at 100 points; the
                 M2M, M2L and L2L response matrices (degree 6) between fixed origins; and the
                 FFTM field (KFMElectrostaticFastMultipoleFieldSolver, degree 8, divisions 2,
                 zeromask 1, depths 3 and 4) of the coax_small density at 300 gap points, with
                 the world cube it estimated; the fast-multipole matrix
                 (KFastMultipoleMatrixGenerator, degree 8, depth 3) times the coax_small density
                 and times a seeded vector on mixed_small (Neumann rows and wires), with the world
                 cubes of those trees
  c2_fftm        configuration 2's 44,000-element coax with its fixed density
                 (geometry.coax_density) under the reference's fast multipole code with region
                 estimation (degree 8, divisions 2, zeromask 1, depth 5): the world cube it
                 estimated, the field at 2,000 seeded gap points, and its matrix
                 (KFastMultipoleMatrixGenerator) times the density
  krylov         the reference's Krylov solvers on the coax_small system: the solver factory
                 (KBuildKrylovSolver, the path of KKrylovChargeDensitySolver) with gmres and
                 bicgstab, preconditioners none, jacobi and implicit_krylov (inner gmres on the
                 same matrix to 0.1, at most 10 iterations), no restart and a restart every 7
                 iterations, tolerance 1e-9: solution, iterations, residual norm, and the true
                 residual of the solution; and the fast-multipole boundary-value solver
                 (KFMElectrostaticFastMultipoleBoundaryValueSolver, the solver of krylov_bem_solver;
                 degree 8, depth 3) with every solver / preconditioner pair but gmres / none
                 (which does not initialise its tree and crashes), tolerance 1e-6, inner
                 tolerance 0.01 and 30 iterations, preconditioner degree 1 (implicit_krylov) or
                 the degree-2, depth-2 tree (independent_implicit_krylov): solution and residual

Usage: python tests/golden/make_golden.py [fixture ...]   (default: all)
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from kassiopeia_b200 import geometry as G  # noqa: E402
from oracle import ref  # noqa: E402


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    print(f"{name}: " + ", ".join(f"{k}{list(np.shape(v))}" for k, v in arrays.items()))


def mesh_arrays(m, prefix=""):
    return {prefix + "shape": m.shape, prefix + "boundary": m.boundary, prefix + "geom": m.geom,
            prefix + "value": m.value}


def rules():
    out = {}
    for i, name in enumerate(["tri7", "tri12", "tri33", "rect7", "rect12", "rect33"]):
        buf = np.zeros((33, 3))
        n = ref.lib().kemref_rule_nodes(i, buf.ctypes.data_as(ref._dp))
        out[name] = buf[:n].copy()
    save("rules", **out)


def integrators():
    rng = np.random.default_rng(11)
    rect = G.rectangles_from_corners([-2., -2., 0.], [2., -2., 0.], [-2., 2., 0.], 10.)
    tri = G.triangles_from_vertices([-1.75, 0.25, 0.], [1.75, 0.25, 0.], [0., 2.25, 0.], 10.)
    rect_pts = [[-2., -2., 0.], [0.1, -1.5, 0.], [0., 0., 0.], [10., 10., 0.], [0., -2., 0.], [10., -20.5, 33.58],
                [-1., -1., 0.]]
    tri_pts = [[-1.75, 0.25, 0.], [0.01, 0.5, 0.], list(tri.centroids()[0]), [10., 1., 0.], [0., 0.25, 0.],
               [10., -20.5, 33.58]]
    extra_r = [[2., 2., 0.], [2., 0., 0.], [-2., 0.5, 0.], [0., 0., 1e-3], [0., 0., -0.7], [3., 1., 0.2],
               [-2., -2., 0.5], [2.5, 2.5, 0.], [0.3, 0.4, 1e-9]]
    extra_t = [[1.75, 0.25, 0.], [0., 2.25, 0.], [0.875, 1.25, 0.], [-0.875, 1.25, 0.], [0., 1., 0.5],
               [0., 1., -2e-3], [3., 3., 1.], [0.2, 0.9, 1e-10]]
    near_r = rng.uniform(-6, 6, size=(40, 3)) * np.array([1, 1, 0.5])
    near_t = rng.uniform(-4, 4, size=(40, 3)) * np.array([1, 1, 0.5]) + np.array([0, 1, 0])
    far = rng.normal(size=(20, 3))
    far /= np.linalg.norm(far, axis=1)[:, None]
    far_r = far * rng.uniform(20, 1500, size=(20, 1))
    far_t = far * rng.uniform(15, 900, size=(20, 1))
    P_r = np.concatenate([rect_pts, extra_r, near_r, far_r])
    P_t = np.concatenate([tri_pts, extra_t, near_t, far_t])
    pr = ref.RefProblem(rect)
    pt = ref.RefProblem(tri)
    save("integrators", rect_points=P_r, rect_field=pr.element_field(0, P_r), tri_points=P_t,
         tri_field=pt.element_field(0, P_t), **mesh_arrays(rect, "rect_"), **mesh_arrays(tri, "tri_"))


def lines():
    rng = np.random.default_rng(12)
    p0 = np.array([[0., 0., 0.], [0.3, 0.1, -0.2], [1., 1., 1.]])
    p1 = np.array([[1., 0., 0.], [0.3, 0.6, 0.4], [1.2, 0.9, 1.5]])
    diam = 2e-3
    m = G.line_segments(p0, p1, diam, 5.0)
    pts = [[0.5, 0.0005, 0.], [0.5, 0.002, 0.], [0.5, 0., 0.], [-0.0005, 0.0002, 0.], [1.0003, 0., 0.0001],
           [0.5, 0.3, 0.], [2., 1., 1.], [40., 3., 2.], [0.3, 0.35, 0.1 + 1e-4]]
    pts = np.concatenate([np.array(pts), rng.uniform(-1.5, 2.5, size=(30, 3)),
                          rng.normal(size=(10, 3)) * rng.uniform(5, 80, size=(10, 1))])
    p = ref.RefProblem(m)
    fields = np.stack([p.element_field(k, pts) for k in range(m.n)])
    save("lines", points=pts, element_field=fields, **mesh_arrays(m))


def icosphere():
    m = G.icosphere(2)
    p = ref.RefProblem(m)
    x, it, r = p.gmres(1e-12)
    # the reference GMRES's SVD least-squares step (kfm_matrix_svd) is not accurate enough here:
    # its sigma has a true relative residual ~2e-5 although its implicit estimate reads ~6e-14;
    # the direct solution of the reference's own matrix is kept alongside as the solve oracle
    A = p.matrix()
    b = p.rhs()
    xd = np.linalg.solve(A, b)
    pts = np.concatenate([G.shell_points(64, seed=3), G.shell_points(16, 1.005, 1.1, seed=4)])
    p.set_sigma(x)
    f = p.field(pts)
    cap = float((x * m.areas()).sum() * ref.constant("one_over_four_pi_eps0"))
    save("icosphere_L2", sigma=x, sigma_direct=xd, gmres_true_residual=np.array(np.linalg.norm(b - A @ x) / np.linalg.norm(b)),
         iterations=np.array(it), residual=np.array(r), points=pts, field=f,
         capacitance=np.array(cap), **mesh_arrays(m))


def mixed_small():
    rng = np.random.default_rng(13)
    # a bent triangle strip (Dirichlet), a Neumann rectangle patch, and two wires
    v = np.array([[0, 0, 0], [0.2, 0, 0.02], [0, 0.2, 0.01], [0.2, 0.2, 0.05], [0.4, 0.05, 0.0], [0.4, 0.25, 0.04]],
                 float)
    tri = G.triangles_from_vertices(v[[0, 1, 3, 1]], v[[1, 3, 1, 4]], v[[2, 2, 4, 5]], 1.0)
    tri.value[:] = [1.0, 1.0, 0.5, 0.5]
    ro = np.array([[0., 0., 0.3], [0.15, 0., 0.3], [0., 0.12, 0.3], [0.15, 0.12, 0.3]])
    rect = G.rectangles_from_corners(ro, ro + [0.15, 0, 0.], ro + [0., 0.12, 0.], 0.4, boundary=G.NEUMANN)
    wire = G.line_segments([[-0.1, 0., 0.1], [-0.1, 0.1, 0.1]], [[-0.1, 0.1, 0.1], [-0.1, 0.2, 0.12]], 3e-3, -0.5)
    m = tri.concat(rect).concat(wire)
    p = ref.RefProblem(m)
    A = p.matrix()
    b = p.rhs()
    x, it, r = p.gmres(1e-12)
    xv = rng.normal(size=m.n)
    save("mixed_small", A=A, b=b, x=x, x_direct=np.linalg.solve(A, b), xv=xv, Axv=p.matvec(xv), **mesh_arrays(m))


def coax_small():
    m = G.coax(n_phi=24, n_z=20, n_cap_rings=3)
    p = ref.RefProblem(m)
    x, it, r = p.gmres(1e-10)
    A = p.matrix()
    b = p.rhs()
    pts = G.gap_points(200, seed=21)
    p.set_sigma(x)
    f = p.field(pts)
    save("coax_small", sigma=x, sigma_direct=np.linalg.solve(A, b),
         gmres_true_residual=np.array(np.linalg.norm(b - A @ x) / np.linalg.norm(b)), iterations=np.array(it),
         points=pts, field=f, **mesh_arrays(m))


def rk8():
    fx = dict(np.load(os.path.join(HERE, "icosphere_L2.npz")))
    from oracle.golden import mesh_from
    m = mesh_from(fx)
    p = ref.RefProblem(m)
    p.set_sigma(fx["sigma"] * 1e4)  # scale the charge so the 1-18.6 keV tracks bend visibly
    st0 = G.electrons(4, seed=5)
    trajs = []
    for k in range(4):
        _, n, tr = p.rk8_track(st0[k], 1e-11, 40, record=True)
        trajs.append(tr)
    save("rk8", state0=st0, traj=np.stack(trajs), sigma_scale=np.array(1e4), dt=np.array(1e-11),
         charge=np.array(-ref.constant("q")), mass=np.array(ref.constant("m_el")))


def adjoint():
    """icosphere L2 with sigma = solved sigma * (1 + 0.1 N(0,1)), 32 shell probes, seeded
    weights w on (E, phi); L = sum_p w_p . out_p. dL/dsigma from the per-element fields, and
    central differences (h = 1e-6 m) of L over the defining vertices of six elements."""
    fx = dict(np.load(os.path.join(HERE, "icosphere_L2.npz")))
    from oracle.golden import mesh_from
    m = mesh_from(fx)
    rng = np.random.default_rng(41)
    sigma = fx["sigma"] * (1.0 + 0.1 * rng.normal(size=m.n))
    P = G.shell_points(32, seed=42)
    w = rng.normal(size=(32, 4))
    w[:, :3] *= 1e-1  # E is ~10x phi here; keep both parts of L comparable
    p = ref.RefProblem(m)
    dsig = np.array([np.sum(w * p.element_field(k, P)) for k in range(m.n)])
    elems = np.array([0, 7, 55, 120, 211, 319])
    h = 1e-6
    verts = np.zeros((m.n, 3, 3))
    g = m.geom
    verts[:, 0] = g[:, 2:5]
    verts[:, 1] = g[:, 2:5] + g[:, 0:1] * g[:, 5:8]
    verts[:, 2] = g[:, 2:5] + g[:, 1:2] * g[:, 8:11]

    def L_of(vv):
        mm = G.triangles_from_vertices(vv[:, 0], vv[:, 1], vv[:, 2], 1.0)
        q = ref.RefProblem(mm)
        q.set_sigma(sigma)
        return float(np.sum(w * q.field(P)))

    fd = np.zeros((len(elems), 9))
    for a, j in enumerate(elems):
        for c in range(9):
            vp, vm = verts.copy(), verts.copy()
            vp[j, c // 3, c % 3] += h
            vm[j, c // 3, c % 3] -= h
            fd[a, c] = (L_of(vp) - L_of(vm)) / (2 * h)
    save("adjoint", sigma=sigma, points=P, w=w, dsigma=dsig, elems=elems, dvert_fd=fd, h=np.array(h),
         vertices=verts, **mesh_arrays(m))


def robinhood():
    from oracle import golden

    out = {}
    for name in ("icosphere_L2", "mixed_small"):
        m = golden.mesh_from(golden.load(name))
        p = ref.RefProblem(m)
        for tol in (1e-8, 1e-10):
            x, it, r = p.robinhood(tol)
            key = f"{name}_{tol:.0e}"
            out[key + "_sigma"] = x
            out[key + "_iterations"] = np.array(it)
            out[key + "_residual"] = np.array(r)
    save("robinhood", **out)


def _band_points(r0, z0, r1, z1, seed):
    # points at distance d = f L from the generator (both sides), at fractions t along it and
    # beyond its ends, each turned to a seeded azimuth; plus points on the axis
    rng = np.random.default_rng(seed)
    L = np.hypot(r1 - r0, z1 - z0)
    u = np.array([r1 - r0, z1 - z0]) / L
    nrm = np.array([-u[1], u[0]])
    pts = []
    for t in (-0.3, 0.0, 0.1, 0.5, 0.9, 1.0, 1.3):
        for f in (0.5, 0.2, 0.1, 0.05, 0.02, 0.01, 0.003, 0.001, 0.0003, 0.0):
            for side in ((1.0, -1.0) if f > 0 else (1.0,)):
                rz = np.array([r0, z0]) + t * L * u + side * f * L * nrm
                if rz[0] < 0:
                    continue
                phi = rng.uniform(0, 2 * np.pi)
                pts.append([rz[0] * np.cos(phi), rz[0] * np.sin(phi), rz[1]])
    for z in (-1.0, 0.0, 0.05, 0.7):
        pts.append([0.0, 0.0, z])
    return np.array(pts)


def axisym():
    out = {}
    # single elements at unit charge density
    cone = G.axisymmetric(G.CONIC_SECTION, 0.5, -0.2, 0.7, 0.3)
    ring = G.axisymmetric(G.RING, 0.6, 0.1)
    for name, m, pts in (("cone", cone, _band_points(0.5, -0.2, 0.7, 0.3, seed=41)),
                         ("ring", ring, _band_points(0.45, 0.1, 0.75, 0.1, seed=43))):
        p = ref.RefProblem(m)
        f = p.element_field(0, pts)
        keep = np.isfinite(f).all(axis=1)  # a point on the ring itself has no finite field
        out[name + "_points"] = pts[keep]
        out[name + "_field"] = f[keep]
        out.update(mesh_arrays(m, name + "_"))
    # whole problems
    for name, m, pts in (("sphere", G.conic_sphere(120), G.shell_points(64, seed=47)),
                         ("coax", G.conic_coax(n_z=40, n_cap=6, n_rings=4), G.gap_points(64, seed=53))):
        p = ref.RefProblem(m)
        A = p.matrix()
        b = p.rhs()
        x = np.linalg.solve(A, b)
        p.set_sigma(x)
        out[name + "_A"] = A
        out[name + "_b"] = b
        out[name + "_sigma"] = x
        out[name + "_points"] = pts
        out[name + "_field"] = p.field(pts)
        out.update(mesh_arrays(m, name + "_"))
    out["sphere_capacitance"] = np.array(float((out["sphere_sigma"] * G.conic_sphere(120).areas()).sum()) /
                                         (4 * np.pi * ref.constant("eps0")))
    save("axisym", **out)


# ----------------------------------------------------------------------------- configurations
# Fixtures at the benchmark configurations' stated sizes. Their meshes are regenerated by the
# tests with the same geometry functions; a checksum of each mesh is stored with it.
def mesh_checksum(m):
    return np.array([m.geom.sum(), np.abs(m.geom).sum(), m.value.sum(), float(m.n)])


def sampled_rows(p, m, n_rows, n_cols, seed):
    """n_rows seeded rows of the reference's matrix; per row the diagonal, the nearest
    neighbours by centroid (the analytic near-field band) and seeded columns, n_cols in all."""
    rng = np.random.default_rng(seed)
    rows = np.sort(rng.choice(m.n, n_rows, replace=False))
    A = p.matrix(rows)
    c = m.centroids()
    cols = np.zeros((n_rows, n_cols), np.int64)
    for k, i in enumerate(rows):
        near = np.argsort(np.linalg.norm(c - c[i], axis=1))[: n_cols // 4]
        rest = np.setdiff1d(np.arange(m.n), near)
        cols[k] = np.concatenate([near, rng.choice(rest, n_cols - len(near), replace=False)])
    return rows, cols, A


def c1_sphere():
    m = G.icosphere(3)
    p = ref.RefProblem(m)
    A = p.matrix()
    b = p.rhs()
    xd = np.linalg.solve(A, b)
    xg, it, r = p.gmres(1e-10)
    xr, itr, rr = p.robinhood(1e-8)
    pts = G.shell_points(10000, seed=2025)
    p.set_sigma(xd)
    f = p.field(pts)
    save("c1_sphere", sigma_direct=xd, b=b, gmres_sigma=xg, gmres_iterations=np.array(it),
         robinhood_sigma=xr, robinhood_iterations=np.array(itr), robinhood_residual=np.array(rr),
         gmres_true_residual=np.array(np.linalg.norm(b - A @ xg) / np.linalg.norm(b)), points=pts, field=f,
         checksum=mesh_checksum(m))


def c2_coax():
    m = G.coax()
    sigma = G.coax_density(m)
    p = ref.RefProblem(m)
    p.set_sigma(sigma)
    pts = G.gap_points(200, seed=2026)
    f = p.field(pts)
    rows, cols, A = sampled_rows(p, m, 64, 64, seed=2027)
    x = np.random.default_rng(2028).normal(size=m.n) * 1e-8
    save("c2_coax", points=pts, field=f, rows=rows, cols=cols, entries=np.take_along_axis(A, cols, axis=1),
         x_seed=np.array(2028), Ax=A @ x, checksum=mesh_checksum(m))


def _track_worker(args):
    geom_arrays, sigma, st, nsteps = args
    sys.path.insert(0, ROOT)
    from kassiopeia_b200.geometry import Mesh
    from oracle import ref as R

    q = R.RefProblem(Mesh(*geom_arrays))
    q.set_sigma(sigma)
    _, n, tr = q.rk8_track(st, 1e-11, nsteps, stop_radius=1.0, record=True)
    return n, tr


def c3_tracks():
    import multiprocessing as mp

    fx = dict(np.load(os.path.join(HERE, "c1_sphere.npz")))
    m = G.icosphere(3)
    # 8 electrons whose straight flight line meets the sphere between steps 100 and 900 and 8
    # that stay clear of it, from a seeded batch, so both ends of a track are covered
    cand = G.electrons(4096, seed=2029)
    x, p = cand[:, 2:5], cand[:, 5:8]
    mc = G.ELECTRON_MASS * G.SPEED_OF_LIGHT
    v = p / (G.ELECTRON_MASS * np.sqrt(1.0 + np.sum(p * p, axis=1) / mc ** 2))[:, None]
    b = np.sum(x * v, axis=1)
    vv = np.sum(v * v, axis=1)
    disc = b * b - vv * (np.sum(x * x, axis=1) - 1.0)
    t_hit = np.where((disc > 0) & (b < 0), (-b - np.sqrt(np.maximum(disc, 0))) / vv, np.inf) / 1e-11
    hit = np.flatnonzero((t_hit > 100) & (t_hit < 900))[:8]
    miss = np.flatnonzero(~np.isfinite(t_hit))[:8]
    idx = np.sort(np.concatenate([hit, miss]))
    st0 = cand[idx]
    arrays = (m.shape, m.boundary, m.geom, m.value)
    with mp.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
        res = pool.map(_track_worker, [(arrays, fx["sigma_direct"], st0[k], 1000) for k in range(16)])
    steps = np.array([r[0] for r in res], np.int32)
    every = 50
    snaps = np.full((16, 1000 // every, 8), np.nan)
    for k, (n, tr) in enumerate(res):
        for s in range(every, n + 1, every):
            snaps[k, s // every - 1] = tr[s - 1]
    final = np.stack([r[1][r[0] - 1] for r in res])
    save("c3_tracks", state0=st0, candidates_seed=np.array(2029), candidates_index=idx, steps=steps, every=np.array(every), snapshots=snaps, final=final,
         dt=np.array(1e-11), max_steps=np.array(1000), sphere_radius=np.array(1.0))


def _tri_bands(v0, v1, v2, P):
    """the reference's triangle rule band of every probe (0 RWG, 1 33-point, 2 12-point,
    3 7-point): ratio |P - centroid| / ((|P1-P0| + |P2-P0| + |P2-P1|) / 3)"""
    size = (np.linalg.norm(v1 - v0) + np.linalg.norm(v2 - v0) + np.linalg.norm(v2 - v1)) / 3.0
    ratio = np.linalg.norm(P - (v0 + v1 + v2) / 3.0, axis=1) / size
    return np.digitize(ratio, [3.42, 30.4, 131.4], right=True), ratio


def c4_adjoint():
    m = G.icosphere(5)
    sigma = G.sphere_density(m, seed=4)
    P = G.shell_points(4096, seed=44)
    w = np.zeros((4096, 4))
    w[:, 2] = 1.0
    w[:, 3] = 1.0
    rng = np.random.default_rng(2030)
    ds_elems = np.sort(rng.choice(m.n, 512, replace=False))
    p = ref.RefProblem(m)
    dsig = np.array([np.sum(w * p.element_field(k, P)) for k in ds_elems])
    g = m.geom
    verts = np.stack([g[:, 2:5], g[:, 2:5] + g[:, 0:1] * g[:, 5:8], g[:, 2:5] + g[:, 1:2] * g[:, 8:11]], axis=1)
    h = 1e-6
    chosen, fd = [], []
    for j in rng.permutation(m.n):
        if len(chosen) == 16:
            break
        base, ratio = _tri_bands(*verts[j], P)
        cuts = np.array([3.42, 30.4, 131.4])
        if np.min(np.abs(ratio[:, None] / cuts[None, :] - 1.0)) < 1e-4:
            continue  # a probe close to a band cut: the difference quotient would straddle rules
        ok = True
        rowfd = np.zeros(9)
        for c in range(9):
            vals = []
            for sgn in (1.0, -1.0):
                vv = verts[j].copy()
                vv[c // 3, c % 3] += sgn * h
                if not np.array_equal(_tri_bands(*vv, P)[0], base):
                    ok = False
                    break
                e = G.triangles_from_vertices(vv[0], vv[1], vv[2], 1.0)
                vals.append(sigma[j] * float(np.sum(w * ref.RefProblem(e).element_field(0, P))))
            if not ok:
                break
            rowfd[c] = (vals[0] - vals[1]) / (2 * h)
        if ok:
            chosen.append(j)
            fd.append(rowfd)
    order = np.argsort(chosen)
    save("c4_adjoint", sigma_seed=np.array(4), points=P, w=w, dsigma_elems=ds_elems, dsigma=dsig,
         fd_elems=np.array(chosen)[order], dvert_fd=np.array(fd)[order], h=np.array(h),
         fd_vertices=verts[np.array(chosen)[order]], checksum=mesh_checksum(m))


def c5_rings():
    m = G.stacked_rings()
    p = ref.RefProblem(m)
    rows, cols, A = sampled_rows(p, m, 64, 64, seed=2031)
    X = np.random.default_rng(2032).normal(size=(8, m.n)) * 1e-8
    save("c5_rings", rows=rows, cols=cols, entries=np.take_along_axis(A, cols, axis=1), x_seed=np.array(2032),
         Ax=(A @ X.T).T, checksum=mesh_checksum(m))


def element_vertices(m):
    """vertex lists of planar elements as the reference's point clouds (KFMElectrostaticSurfaceConverter):
    triangle P0, P0 + A N1, P0 + B N2; rectangle P0, P0 + A N1, P0 + A N1 + B N2, P0 + B N2; wire P0, P1"""
    out = []
    for k in range(m.n):
        g = m.geom[k]
        p0, n1, n2 = g[2:5], g[5:8], g[8:11]
        if m.shape[k] == G.TRIANGLE:
            out.append(np.array([p0, p0 + g[0] * n1, p0 + g[1] * n2]))
        elif m.shape[k] == G.RECTANGLE:
            out.append(np.array([p0, p0 + g[0] * n1, p0 + g[0] * n1 + g[1] * n2, p0 + g[1] * n2]))
        else:
            out.append(np.array([g[0:3], g[3:6]]))
    return out


def fftm():
    from oracle import ref_fm

    rng = np.random.default_rng(2040)
    mx = golden_mesh("mixed_small")
    origins = np.array([v.mean(axis=0) for v in element_vertices(mx)]) + rng.uniform(-0.1, 0.1, (mx.n, 3))
    moments = np.array([ref_fm.moments(v, o, 10) for v, o in zip(element_vertices(mx), origins)])
    deg = 8
    coeff = np.array([complex(rng.standard_normal(), rng.standard_normal() if mm else 0.) * 0.6 ** l
                      for l in range(deg + 1) for mm in range(l + 1)])
    l2p_origin = np.array([0.1, -0.2, 0.15])
    l2p_points = l2p_origin + rng.uniform(-0.7, 0.7, (100, 3))
    l2p = ref_fm.l2p(deg, l2p_origin, coeff, l2p_points)
    src, tgt, far = np.array([0.3, -0.2, 0.5]), np.array([-0.1, 0.4, 0.2]), np.array([2.1, 1.4, -1.7])
    resp = np.array([ref_fm.response(0, 6, src, tgt), ref_fm.response(1, 6, src, far), ref_fm.response(2, 6, src, tgt)])
    cx = golden_mesh("coax_small")
    sigma = np.load(os.path.join(HERE, "coax_small.npz"))["sigma"]
    pts = G.gap_points(300, seed=2041)
    fr = ref_fm.FmRefProblem(cx)
    fr.set_sigma(sigma)
    f3, w3 = fr.field(pts, degree=8, maximum_tree_depth=3)
    f4, w4 = fr.field(pts, degree=8, maximum_tree_depth=4)
    coax_Ax = fr.matvec(sigma, degree=8, maximum_tree_depth=3)
    fm = ref_fm.FmRefProblem(mx)
    xv = np.load(os.path.join(HERE, "mixed_small.npz"))["xv"]
    mixed_Ax = fm.matvec(xv, degree=8, maximum_tree_depth=3)
    _, mixed_world = fm.field(np.zeros((1, 3)), degree=8, maximum_tree_depth=3)
    save("fftm", mixed_origins=origins, mixed_moments=moments, l2p_degree=np.array(deg), l2p_coeff=coeff,
         l2p_origin=l2p_origin, l2p_points=l2p_points, l2p=l2p, resp_src=src, resp_tgt=tgt, resp_far=far,
         resp=resp, coax_points=pts, coax_field_d3=f3, coax_world_d3=w3, coax_field_d4=f4, coax_world_d4=w4,
         coax_Ax_d3=coax_Ax, mixed_Ax_d3=mixed_Ax, mixed_world_d3=mixed_world)


def c2_fftm():
    from oracle import ref_fm

    mesh = G.coax()
    sigma = G.coax_density(mesh)
    pts = G.gap_points(2000, seed=2049)
    fr = ref_fm.FmRefProblem(mesh)
    fr.set_sigma(sigma)
    field, world = fr.field(pts, degree=8, maximum_tree_depth=5)
    Ax = fr.matvec(sigma, degree=8, maximum_tree_depth=5)
    save("c2_fftm", points=pts, field=field, world=world, Ax=Ax)


def krylov():
    from oracle import ref_fm

    cx = golden_mesh("coax_small")
    p = ref.RefProblem(cx)
    A, b = p.matrix(), p.rhs()
    out = {"direct_sigma": np.linalg.solve(A, b)}
    for solver in ("gmres", "bicgstab"):
        for pc in ("none", "jacobi", "implicit_krylov"):
            for restart in (0, 7):
                x, it, r = p.krylov(solver, pc, tol=1e-9, max_iter=300, restart=restart, preconditioner_tol=0.1,
                                    max_preconditioner_iter=10)
                key = f"{solver}_{pc}_r{restart}"
                out[key + "_sigma"] = x
                out[key + "_iterations"] = np.array(it)
                out[key + "_residual"] = np.array(r)
                out[key + "_true_residual"] = np.array(np.linalg.norm(b - A @ x) / np.linalg.norm(b))
    fr = ref_fm.FmRefProblem(cx)
    for solver, pc in (("gmres", "jacobi"), ("gmres", "implicit_krylov"), ("gmres", "independent_implicit_krylov"),
                       ("bicgstab", "none"), ("bicgstab", "jacobi"), ("bicgstab", "implicit_krylov"),
                       ("bicgstab", "independent_implicit_krylov")):
        x, r = fr.solve(solver, pc, tol=1e-6, max_iter=200, preconditioner_tol=0.01, max_preconditioner_iter=30,
                        preconditioner_degree=1, preconditioner_params=dict(degree=2, maximum_tree_depth=2), degree=8,
                        maximum_tree_depth=3)
        out[f"fftm_{solver}_{pc}_sigma"] = x
        out[f"fftm_{solver}_{pc}_residual"] = np.array(r)
    save("krylov", **out)


def golden_mesh(name):
    from oracle.golden import mesh_from

    return mesh_from(dict(np.load(os.path.join(HERE, name + ".npz"))))


FIXTURES = {f.__name__: f for f in (rules, integrators, lines, icosphere, mixed_small, coax_small, rk8, adjoint,
                                     robinhood, axisym, c1_sphere, c2_coax, c3_tracks, c4_adjoint, c5_rings, fftm,
                                     krylov, c2_fftm)}

if __name__ == "__main__":
    for name in sys.argv[1:] or list(FIXTURES):
        FIXTURES[name]()
