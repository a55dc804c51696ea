"""CPU checks of the oracle itself: the golden fixtures are reproduced by the reference build
(when it is present) and satisfy the reference's own known answers."""

import numpy as np
import pytest

from kassiopeia_b200 import geometry as G
from oracle import golden, ref

needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (reference tree absent)")


def test_sphere_capacitance_known_answer():
    # SphereCapacitanceTest.cc:110-133: C = sum sigma_i A_i / (4 pi eps0 R) = 1 within 5e-2
    fx = golden.load("icosphere_L2")
    assert abs(float(fx["capacitance"]) - 1.0) < 5e-2
    # the discretisation bound of the analytic 1/r potential outside the sphere
    r = np.linalg.norm(fx["points"], axis=1)
    far = r > 1.2
    assert np.max(np.abs(fx["field"][far, 3] * r[far] - 1.0)) < 3e-2


def test_integrators_cross_agreement_shape():
    # IntegratorsTest.cc checks RWG vs analytic to 2.5 %; the fixture holds the numeric
    # policy's values, which must be finite at every special point (corners, edges, plane)
    fx = golden.load("integrators")
    assert np.all(np.isfinite(fx["rect_field"])) and np.all(np.isfinite(fx["tri_field"]))


@needs_ref
def test_reference_reproduces_fixtures():
    fx = golden.load("icosphere_L2")
    p = ref.RefProblem(golden.mesh_from(fx))
    p.set_sigma(fx["sigma"])
    np.testing.assert_array_equal(p.field(fx["points"][:10]), fx["field"][:10])
    mx = golden.load("mixed_small")
    q = ref.RefProblem(golden.mesh_from(mx))
    np.testing.assert_array_equal(q.matrix(), mx["A"])


@needs_ref
def test_reference_container_order_is_grouped_by_type():
    # KSurfaceContainer groups elements by (boundary, shape) type in first-seen order;
    # the harness maps caller order <-> container order explicitly
    mx = golden.load("mixed_small")
    m = golden.mesh_from(mx)
    perm = np.r_[m.n - 1, 0:m.n - 1]  # put a wire first
    m2 = G.Mesh(m.shape[perm], m.boundary[perm], m.geom[perm], m.value[perm])
    q = ref.RefProblem(m2)
    A2 = q.matrix()
    np.testing.assert_allclose(A2, mx["A"][np.ix_(perm, perm)], rtol=1e-15, atol=0)


# ---------------------------------------------------------------- the C restatement, pinned
from oracle import port  # noqa: E402

needs_port = pytest.mark.skipif(not port.available(), reason="oracle/libkemoracle.so not built")


@needs_port
@pytest.mark.parametrize("shape", ["rect", "tri"])
def test_port_single_element_special_points(shape):
    fx = golden.load("integrators")
    p = port.PortProblem(golden.mesh_from(fx, shape + "_"))
    out = p.element_field(0, fx[shape + "_points"])
    ref_ = fx[shape + "_field"]
    assert np.max(np.abs(out - ref_) / np.max(np.abs(ref_), axis=0)) < 1e-11


@needs_port
def test_port_lines():
    fx = golden.load("lines")
    m = golden.mesh_from(fx)
    p = port.PortProblem(m)
    for k in range(m.n):
        ref_ = fx["element_field"][k]
        ok = np.all(np.isfinite(ref_), axis=1) & (np.abs(ref_).max(axis=1) < 1e15)
        out = p.element_field(k, fx["points"][ok])
        assert np.max(np.abs(out - ref_[ok]) / np.max(np.abs(ref_[ok]), axis=0)) < 1e-12


@needs_port
def test_port_field_matrix_and_solve():
    fx = golden.load("icosphere_L2")
    p = port.PortProblem(golden.mesh_from(fx))
    p.set_sigma(fx["sigma"])
    out = p.field(fx["points"])
    assert np.max(np.abs(out - fx["field"]) / np.abs(fx["field"]).max(axis=0)) < 1e-13
    mx = golden.load("mixed_small")
    q = port.PortProblem(golden.mesh_from(mx))
    A, b = q.matrix()
    assert np.max(np.abs(A - mx["A"]) / np.abs(mx["A"]).max(axis=1, keepdims=True)) < 1e-13
    np.testing.assert_array_equal(b, mx["b"])
    x, it, r = q.gmres(1e-13)
    assert np.max(np.abs(x - mx["x_direct"])) / np.max(np.abs(mx["x_direct"])) < 1e-10


@needs_port
def test_port_rk8():
    fx = golden.load("icosphere_L2")
    rk = golden.load("rk8")
    p = port.PortProblem(golden.mesh_from(fx))
    p.set_sigma(fx["sigma"] * float(rk["sigma_scale"]))
    st, traj = p.rk8_track(rk["state0"][0], float(rk["dt"]), 10, float(rk["charge"]), float(rk["mass"]))
    ref_ = rk["traj"][0, :10]
    assert np.max(np.abs(traj[:, 2:8] - ref_[:, 2:8]) / np.abs(ref_[:, 2:8]).max(axis=0)) < 1e-12


def test_axisym_fixture_known_answers():
    # a sphere of conic sections at 1 V: C = 4 pi eps0 R as the sections shrink, and the
    # potential outside is 1/r (120 sections: within 1e-4)
    fx = golden.load("axisym")
    assert abs(float(fx["sphere_capacitance"]) - 1.0) < 1e-4
    r = np.linalg.norm(fx["sphere_points"], axis=1)
    assert np.max(np.abs(fx["sphere_field"][:, 3] * r - 1.0)) < 1e-4
    # on the axis the field of an axisymmetric charge is axial
    on_axis = np.hypot(fx["cone_points"][:, 0], fx["cone_points"][:, 1]) == 0.0
    assert on_axis.sum() == 4 and np.all(fx["cone_field"][on_axis, :2] == 0.0)


@needs_ref
def test_reference_reproduces_axisym_fixture():
    fx = golden.load("axisym")
    for name in ("cone", "ring"):
        p = ref.RefProblem(golden.mesh_from(fx, name + "_"))
        np.testing.assert_array_equal(p.element_field(0, fx[name + "_points"]), fx[name + "_field"])
    q = ref.RefProblem(golden.mesh_from(fx, "coax_"))
    np.testing.assert_array_equal(q.matrix(), fx["coax_A"])


def test_port_axisymmetric_elements_bit_exact():
    # the C restatement of the conic-section and ring integrators reproduces the reference's
    # values exactly: single elements in every band, the matrices and the fields of the
    # sphere and the coax with rings
    from oracle import port

    fx = golden.load("axisym")
    for name in ("cone", "ring"):
        p = port.PortProblem(golden.mesh_from(fx, name + "_"))
        np.testing.assert_array_equal(p.element_field(0, fx[name + "_points"]), fx[name + "_field"])
    for name in ("sphere", "coax"):
        p = port.PortProblem(golden.mesh_from(fx, name + "_"))
        A, b = p.matrix()
        np.testing.assert_array_equal(A, fx[name + "_A"])
        np.testing.assert_array_equal(b, fx[name + "_b"])
        p.set_sigma(fx[name + "_sigma"])
        np.testing.assert_array_equal(p.field(fx[name + "_points"]), fx[name + "_field"])


def test_disk_capacitance_known_answer():
    # DiskCapacitanceTest.cc:47-113: 128 conic sections clustered at the rim, C = Q / eps0 = 8 R
    # within 1e-2, on the C restatement (and its matrix equals the reference build's)
    from oracle import port

    m = G.conic_disk()
    p = port.PortProblem(m)
    A, b = p.matrix()
    x = np.linalg.solve(A, b)
    assert abs(float((x * m.areas()).sum()) / 8.8541878128e-12 - 8.0) < 1e-2
    if ref.available():
        np.testing.assert_array_equal(ref.RefProblem(m).matrix(), A)


def test_cube_capacitance_known_answer():
    # CubeCapacitanceTest.cc:43-113: unit cube, 8 x 8 rectangles per face on a power-1.5 grid,
    # C / (4 pi eps0) = 0.6606785 within 1e-2, on the C restatement
    from oracle import port

    m = G.cube()
    p = port.PortProblem(m)
    A, b = p.matrix()
    x = np.linalg.solve(A, b)
    assert abs(float((x * m.areas()).sum()) / (4 * np.pi * 8.8541878128e-12) - 0.6606785) < 1e-2
