"""Device fast-multipole method against the reference's own FFTM code: element moments, the
local-expansion field, and the whole FFTM field (KFMElectrostaticFastMultipoleFieldSolver on
the tree of KFMElectrostaticTreeConstructor, same parameters and world cube) on the
coax_small density (fixture) and the 1,280-triangle sphere (live, oracle/_ref/libkemref_fm.so);
points outside the world cube take the direct sum; the truncation error against the direct sum
shrinks with the degree."""

import numpy as np
import pytest

import kassiopeia_b200 as K
from kassiopeia_b200 import geometry as G
from oracle import golden, ref_fm
from oracle.golden import mesh_from

pytestmark = pytest.mark.gpu
needs_ref_fm = pytest.mark.skipif(not ref_fm.available(), reason="oracle/_ref/libkemref_fm.so not built")


def _vertices(m):
    out = []
    for k in range(m.n):
        g = m.geom[k]
        p0, n1, n2 = g[2:5], g[5:8], g[8:11]
        if m.shape[k] == 0:
            out.append(np.array([p0, p0 + g[0] * n1, p0 + g[1] * n2]))
        elif m.shape[k] == 1:
            out.append(np.array([p0, p0 + g[0] * n1, p0 + g[0] * n1 + g[1] * n2, p0 + g[1] * n2]))
        else:
            out.append(np.array([g[0:3], g[3:6]]))
    return out


def test_moments_equal_reference_fixture():
    fx = golden.load("fftm")
    m = mesh_from(golden.load("mixed_small"))
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(m)
    got = ctx.MultipoleMoments(10, fx["mixed_origins"])
    want = fx["mixed_moments"]
    for e in range(m.n):
        assert np.abs(got[e] - want[e]).max() <= 1e-13 * np.abs(want[e]).max(), e


@needs_ref_fm
@pytest.mark.parametrize("degree", [2, 8, 15])
def test_moments_equal_live_reference(degree):
    rng = np.random.default_rng(degree)
    m = G.icosphere(1).concat(mesh_from(golden.load("coax_small")))
    sel = np.r_[0:80, 80:m.n:23]
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(m)
    origins = m.centroids() + rng.uniform(-0.2, 0.2, (m.n, 3))
    got = ctx.MultipoleMoments(degree, origins)
    verts = _vertices(m)
    for e in sel:
        want = ref_fm.moments(verts[e], origins[e], degree)
        assert np.abs(got[e] - want).max() <= 2e-13 * np.abs(want).max(), e


def test_local_field_equals_reference_fixture():
    fx = golden.load("fftm")
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(G.icosphere(1))
    got = ctx.LocalExpansionField(int(fx["l2p_degree"]), fx["l2p_origin"], fx["l2p_coeff"], fx["l2p_points"])
    want = fx["l2p"]
    assert np.all(np.abs(got - want).max(axis=0) <= 1e-13 * np.abs(want).max(axis=0))


@pytest.mark.parametrize("depth", [3, 4])
def test_fftm_equals_reference_fftm_fixture(depth):
    # the coax_small density (960 rectangles, 288 triangles): same degree, divisions, zeromask,
    # depth, insertion ratio and world cube as the reference's tree
    fx = golden.load("fftm")
    cs = golden.load("coax_small")
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(mesh_from(cs))
    ctx.SetSigma(cs["sigma"])
    w = fx[f"coax_world_d{depth}"]
    ctx.ConfigureFFTM(degree=8, maximum_tree_depth=depth, world_center=w[:3], world_length=w[3])
    got = ctx.FFTMField(fx["coax_points"])
    want = fx[f"coax_field_d{depth}"]
    scale = np.abs(want).max(axis=0)
    err = np.abs(got - want).max(axis=0) / scale
    # the gap potential is the difference of the two cylinders' much larger contributions, so
    # rounding shows at ~6e-12 of the largest value (the field agrees to ~1e-13)
    assert np.all(err[:3] <= 1e-11) and err[3] <= 2e-11, err


@needs_ref_fm
@pytest.mark.parametrize("depth", [2, 3, 4])
def test_fftm_equals_live_reference_fftm_on_sphere(depth):
    fx = golden.load("c1_sphere")
    sph = G.icosphere(3)
    rng = np.random.default_rng(3)
    Q = rng.uniform(-1.0, 1.0, (6000, 3))
    P = Q[np.abs(np.linalg.norm(Q, axis=1) - 1) > 0.08][:300]
    fr = ref_fm.FmRefProblem(sph)
    fr.set_sigma(fx["sigma_direct"])
    want, world = fr.field(P, degree=8, maximum_tree_depth=depth)
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(sph)
    ctx.SetSigma(fx["sigma_direct"])
    ctx.ConfigureFFTM(degree=8, maximum_tree_depth=depth, world_center=world[:3], world_length=world[3])
    got = ctx.FFTMField(P)
    err = np.abs(got - want).max(axis=0) / np.abs(want).max(axis=0)
    assert np.all(err[:3] <= 1e-11) and err[3] <= 1e-13, err


def test_fftm_points_outside_world_take_direct_sum():
    fx = golden.load("c1_sphere")
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(G.icosphere(3))
    ctx.SetSigma(fx["sigma_direct"])
    ctx.ConfigureFFTM(degree=6, maximum_tree_depth=3)
    info = ctx.FFTMInfo(3)
    P = fx["points"]
    far = P[np.abs(P - info["world_center"]).max(axis=1) > 0.55 * info["world_length"]][:100]
    assert len(far) >= 50
    got = ctx.FFTMField(far)
    want = ctx.ElectricFieldAndPotential(far)
    assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()


def test_fftm_error_falls_with_degree():
    fx = golden.load("c1_sphere")
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(G.icosphere(3))
    ctx.SetSigma(fx["sigma_direct"])
    rng = np.random.default_rng(8)
    Q = rng.uniform(-1.0, 1.0, (4000, 3))
    P = Q[np.abs(np.linalg.norm(Q, axis=1) - 1) > 0.08][:400]
    direct = ctx.ElectricFieldAndPotential(P)
    errs = []
    for deg in (4, 8, 12):
        ctx.ConfigureFFTM(degree=deg, maximum_tree_depth=3)
        errs.append(np.abs(ctx.FFTMField(P) - direct).max() / np.abs(direct).max())
    assert errs[0] > errs[1] > errs[2]
    # on the reference's estimated world cube: 1.0e-2, 5.3e-4 and 2.4e-5 of the largest value
    assert errs[1] < 1e-3 and errs[2] < 1e-4, errs


def test_fftm_state_and_argument_errors():
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(G.icosphere(1))
    ctx.SetSigma(np.ones(80) * 1e-9)
    with pytest.raises(K.KemcuError):
        ctx.FFTMField(np.zeros((4, 3)))  # not configured
    for bad in ({"divisions": 1}, {"divisions": 9}, {"zeromask": 0}, {"zeromask": 4}, {"degree": -1}, {"degree": 16},
                {"maximum_tree_depth": 11}):
        with pytest.raises(K.KemcuError):
            ctx.ConfigureFFTM(**bad)
    ax = K.CUDAElectrostaticContext(0)
    ax.SetGeometry(G.conic_sphere(20))
    with pytest.raises(K.KemcuError):
        ax.ConfigureFFTM()


@pytest.mark.parametrize("case", ["coax_small", "mixed_small"])
def test_fftm_matvec_equals_reference_fixture(case):
    # KFastMultipoleMatrixGenerator's matrix (dense far part from the local expansions, sparse near
    # part by the numeric integrator) times a vector: Dirichlet rows (coax), Neumann rows and
    # wires (mixed)
    fx = golden.load("fftm")
    g = golden.load(case)
    x = g["sigma"] if case == "coax_small" else g["xv"]
    w = fx["coax_world_d3" if case == "coax_small" else "mixed_world_d3"]
    want = fx["coax_Ax_d3" if case == "coax_small" else "mixed_Ax_d3"]
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(mesh_from(g))
    ctx.ConfigureFFTM(degree=8, maximum_tree_depth=3, world_center=w[:3], world_length=w[3])
    got = ctx.FFTMMultiply(x)
    assert np.abs(got - want).max() <= 1e-11 * np.abs(want).max()


@pytest.mark.parametrize("case", ["coax_small", "mixed_small"])
def test_fftm_region_estimate_equals_reference(case):
    # use_region_estimation: the reference's minimal bounding ball over the element balls
    # (KFMElectrostaticRegionSizeEstimator) in its container's order, side 2 r x 1.1; the same
    # tree then gives the reference's operator without an explicit world cube
    fx = golden.load("fftm")
    g = golden.load(case)
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(mesh_from(g))
    ctx.ConfigureFFTM(degree=8, maximum_tree_depth=3)
    info = ctx.FFTMInfo(3)
    got = np.r_[info["world_center"], info["world_length"]]
    want = fx["coax_world_d3" if case == "coax_small" else "mixed_world_d3"]
    assert np.abs(got - want).max() <= 1e-9 * want[3]
    x = g["sigma"] if case == "coax_small" else g["xv"]
    Ax = fx["coax_Ax_d3" if case == "coax_small" else "mixed_Ax_d3"]
    assert np.abs(ctx.FFTMMultiply(x) - Ax).max() <= 1e-11 * np.abs(Ax).max()


@needs_ref_fm
def test_fftm_region_estimate_equals_live_reference_on_sphere():
    sph = G.icosphere(3)
    fr = ref_fm.FmRefProblem(sph)
    _, world = fr.field(np.zeros((1, 3)), degree=6, maximum_tree_depth=3)
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(sph)
    ctx.ConfigureFFTM(degree=6, maximum_tree_depth=3)
    info = ctx.FFTMInfo(3)
    got = np.r_[info["world_center"], info["world_length"]]
    assert np.abs(got - world).max() <= 1e-9 * world[3]
    x = np.random.default_rng(3).normal(size=sph.n) * 1e-9
    want = fr.matvec(x, degree=6, maximum_tree_depth=3)
    assert np.abs(ctx.FFTMMultiply(x) - want).max() <= 1e-11 * np.abs(want).max()


@needs_ref_fm
def test_fftm_matvec_equals_live_reference_on_sphere():
    fx = golden.load("c1_sphere")
    sph = G.icosphere(3)
    fr = ref_fm.FmRefProblem(sph)
    want = fr.matvec(fx["sigma_direct"], degree=8, maximum_tree_depth=3)
    _, world = fr.field(np.zeros((1, 3)), degree=8, maximum_tree_depth=3)
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(sph)
    ctx.ConfigureFFTM(degree=8, maximum_tree_depth=3, world_center=world[:3], world_length=world[3])
    got = ctx.FFTMMultiply(fx["sigma_direct"])
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    # and the FFTM operator is the direct one to its truncation error
    direct = ctx.Multiply(fx["sigma_direct"])
    assert np.abs(got - direct).max() <= 2e-5 * np.abs(direct).max()


def test_fftm_solve_reaches_direct_density():
    # GMRES on the fast-multipole operator (KKrylovChargeDensitySolver with
    # KFastMultipoleMatrixGenerator): its residual is the FFTM operator's; the density differs from
    # the direct solution by the operator's truncation error
    fx = golden.load("c1_sphere")
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(G.icosphere(3))
    ctx.ConfigureFFTM(degree=10, maximum_tree_depth=3)
    sigma, st = ctx.Solve(tol=1e-10, mode=K.SOLVE_FFTM)
    assert st["rel_residual"] <= 1e-10
    ref = fx["sigma_direct"]
    assert np.abs(sigma - ref).max() <= 1e-4 * np.abs(ref).max()


def test_fftm_matvec_several_rhs_equal_single_products():
    # the direct entries are evaluated once for all right-hand sides; every row equals the
    # product with that right-hand side alone
    cs = golden.load("coax_small")
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(mesh_from(cs))
    ctx.ConfigureFFTM(degree=6, maximum_tree_depth=3)
    X = np.random.default_rng(11).normal(size=(5, len(cs["sigma"]))) * 1e-9
    Y = ctx.FFTMMultiply(X)
    for r in range(len(X)):
        y1 = ctx.FFTMMultiply(X[r])
        assert np.abs(Y[r] - y1).max() <= 1e-14 * np.abs(y1).max()


@needs_ref_fm
@pytest.mark.parametrize("t,d,zm,depth", [(2, 3, 1, 3), (4, 4, 1, 2), (3, 4, 1, 3), (2, 2, 2, 3), (2, 4, 2, 2)])
def test_fftm_other_divisions_and_zeromask_equal_live_reference(t, d, zm, depth):
    # top-level divisions, division ratio and neighbour order of the reference's parameters
    fx = golden.load("c1_sphere")
    sph = G.icosphere(3)
    rng = np.random.default_rng(3)
    Q = rng.uniform(-1.0, 1.0, (4000, 3))
    P = Q[np.abs(np.linalg.norm(Q, axis=1) - 1) > 0.08][:200]
    fr = ref_fm.FmRefProblem(sph)
    fr.set_sigma(fx["sigma_direct"])
    want, world = fr.field(P, degree=8, top_level_divisions=t, divisions=d, zeromask=zm, maximum_tree_depth=depth)
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(sph)
    ctx.SetSigma(fx["sigma_direct"])
    ctx.ConfigureFFTM(degree=8, top_level_divisions=t, divisions=d, zeromask=zm, maximum_tree_depth=depth,
                      world_center=world[:3], world_length=world[3])
    got = ctx.FFTMField(P)
    err = np.abs(got - want).max(axis=0) / np.abs(want).max(axis=0)
    assert np.all(err[:3] <= 1e-11) and err[3] <= 1e-13, err


def test_fftm_full_coax_equals_reference_fixture():
    # configuration 2's coax at its stated size (44,000 elements) with its fixed density and the
    # reference's own region estimate (no world cube given on either side): the same cube, the
    # reference's field at 2,000 gap points and its matrix times the density
    fx = golden.load("c2_fftm")
    mesh = G.coax()
    sigma = G.coax_density(mesh)
    ctx = K.CUDAElectrostaticContext(0)
    ctx.SetGeometry(mesh)
    ctx.SetSigma(sigma)
    ctx.ConfigureFFTM(degree=8, maximum_tree_depth=5)
    info = ctx.FFTMInfo(5)
    got_world = np.r_[info["world_center"], info["world_length"]]
    assert np.abs(got_world - fx["world"]).max() <= 1e-9 * fx["world"][3]
    got = ctx.FFTMField(fx["points"])
    want = fx["field"]
    err = np.abs(got - want).max(axis=0) / np.abs(want).max(axis=0)
    # as on the reduced coax: the gap potential is a difference of much larger contributions
    assert np.all(err[:3] <= 1e-11) and err[3] <= 2e-11, err
    Ax = fx["Ax"]
    assert np.abs(ctx.FFTMMultiply(sigma) - Ax).max() <= 1e-11 * np.abs(Ax).max()
