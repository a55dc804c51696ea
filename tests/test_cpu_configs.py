"""CPU checks of the fixtures at the benchmark configurations' stated sizes (c1_sphere ...
c5_rings, made by tests/golden/make_golden.py from the reference's own code): the meshes the
tests regenerate are the ones the fixtures were made on, the fixtures satisfy the known
answers that exist (the analytic sphere), and the plain-C restatement reproduces samples of
them. The GPU comparisons at these sizes are in test_gpu_configs.py."""

import numpy as np
import pytest

from kassiopeia_b200 import geometry as G
from oracle import golden, port, ref

needs_port = pytest.mark.skipif(not port.available(), reason="oracle/libkemoracle.so not built")
needs_ref = pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built (reference tree absent)")

MESHES = {"c1_sphere": lambda: G.icosphere(3), "c2_coax": G.coax, "c4_adjoint": lambda: G.icosphere(5),
          "c5_rings": G.stacked_rings}


def checksum(m):
    return np.array([m.geom.sum(), np.abs(m.geom).sum(), m.value.sum(), float(m.n)])


@pytest.mark.parametrize("name", sorted(MESHES))
def test_regenerated_mesh_is_the_fixtures(name):
    fx = golden.load(name)
    np.testing.assert_allclose(checksum(MESHES[name]()), fx["checksum"], rtol=1e-12, atol=0)


def test_c1_known_answers():
    # a conducting sphere at 1 V: phi = 1 V * (1 m / r) outside, C = 4 pi eps0 R; a mesh of
    # 1,280 flat triangles meets both to its discretisation error (3.4e-3 in phi)
    fx = golden.load("c1_sphere")
    m = G.icosphere(3)
    r = np.linalg.norm(fx["points"], axis=1)
    assert np.max(np.abs(fx["field"][:, 3] * r - 1.0)) < 5e-3
    cap = float((fx["sigma_direct"] * m.areas()).sum() / (4 * np.pi * 8.8541878128e-12))
    assert abs(cap - 1.0) < 5e-2
    # E is radial and |E| = phi / r to the same bound
    E = fx["field"][:, :3]
    assert np.max(np.abs(np.linalg.norm(E, axis=1) * r * r - 1.0)) < 5e-3
    # the reference GMRES at 1e-10 (kept for the record): its SVD least-squares step leaves a
    # true residual above its own estimate, which is why the direct solution is the oracle
    assert float(fx["gmres_true_residual"]) < 1e-3


@needs_port
def test_c1_port_reproduces_field_sample():
    fx = golden.load("c1_sphere")
    p = port.PortProblem(G.icosphere(3))
    p.set_sigma(fx["sigma_direct"])
    sel = slice(0, 10000, 50)
    out = p.field(fx["points"][sel])
    ref_ = fx["field"][sel]
    assert np.max(np.abs(out - ref_) / np.abs(ref_).max(axis=0)) < 1e-13


def _port_entries(m, rows, cols):
    """A(i, j) of a Dirichlet row: the potential of element j at the centroid of element i
    (KElectrostaticBoundaryIntegrator.hh:260-280), from the restatement's element integrals"""
    p = port.PortProblem(m)
    c = m.centroids()
    out = np.zeros(cols.shape)
    for k, i in enumerate(rows):
        for q, j in enumerate(cols[k]):
            out[k, q] = p.element_field(int(j), c[i])[0, 3]
    return out


@needs_port
@pytest.mark.parametrize("name", ["c2_coax", "c5_rings"])
def test_port_reproduces_sampled_matrix_entries(name):
    fx = golden.load(name)
    m = MESHES[name]()
    rows, cols = fx["rows"][:16], fx["cols"][:16]
    out = _port_entries(m, rows, cols)
    assert np.max(np.abs(out - fx["entries"][:16]) / np.abs(fx["entries"][:16]).max(axis=1, keepdims=True)) < 1e-12


@needs_port
def test_c2_port_reproduces_field_sample():
    fx = golden.load("c2_coax")
    m = G.coax()
    p = port.PortProblem(m)
    p.set_sigma(G.coax_density(m))
    out = p.field(fx["points"][:20])
    ref_ = fx["field"][:20]
    assert np.max(np.abs(out - ref_) / np.abs(ref_).max(axis=0)) < 1e-12


def test_c3_tracks_fixture_shape():
    fx = golden.load("c3_tracks")
    steps = fx["steps"]
    assert steps.shape == (16,) and np.all((steps >= 1) & (steps <= int(fx["max_steps"])))
    r_end = np.linalg.norm(fx["final"][:, 2:5], axis=1)
    # a track that stopped early ended on the sphere (electrode hit), the others ran to the budget
    early = steps < int(fx["max_steps"])
    assert np.all(r_end[early] <= float(fx["sphere_radius"]))
    assert np.all(r_end[~early] > float(fx["sphere_radius"]))
    assert early.any() and (~early).any()  # both outcomes are covered


@needs_port
def test_c4_port_reproduces_dsigma_sample():
    fx = golden.load("c4_adjoint")
    m = G.icosphere(5)
    p = port.PortProblem(m)
    for a in range(0, 512, 64):
        j = int(fx["dsigma_elems"][a])
        v = float(np.sum(fx["w"] * p.element_field(j, fx["points"])))
        assert abs(v - fx["dsigma"][a]) <= 1e-12 * abs(fx["dsigma"][a])


@needs_ref
def test_reference_reproduces_config_fixtures():
    fx = golden.load("c2_coax")
    m = G.coax()
    p = ref.RefProblem(m)
    p.set_sigma(G.coax_density(m))
    np.testing.assert_array_equal(p.field(fx["points"][:2]), fx["field"][:2])
