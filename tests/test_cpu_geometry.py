"""CPU checks of the synthetic element lists: the encoding each shape uses and the geometric
facts the benchmark workloads rely on (areas, centroids, counts), planar and axisymmetric."""

import numpy as np

from kassiopeia_b200 import geometry as G


def test_conic_sphere_area_centroids_and_axis():
    m = G.conic_sphere(120)
    assert m.n == 120 and np.all(m.shape == G.CONIC_SECTION) and np.all(m.boundary == G.DIRICHLET)
    # the chords' surface of revolution approaches 4 pi R^2 from below
    a = m.areas().sum()
    assert 4 * np.pi * (1 - 1e-3) < a < 4 * np.pi
    # the first and last sections close the sphere on the axis; centroids lie in the x-z plane
    assert m.geom[0, 0] == 0.0 and m.geom[-1, 2] == 0.0
    c = m.centroids()
    assert np.all(c[:, 1] == 0.0) and np.allclose(np.hypot(c[:, 0], c[:, 2]), np.cos(np.pi / 240), atol=1e-12)


def test_conic_coax_composition():
    m = G.conic_coax(n_z=40, n_cap=6, n_rings=4)
    assert m.n == 2 * 40 + 2 * 6 + 4
    assert (m.shape == G.CONIC_SECTION).sum() == 92 and (m.shape == G.RING).sum() == 4
    rings = m.shape == G.RING
    # ring area = circumference (KRing::Area), radius at mid-gap
    assert np.allclose(m.areas()[rings], 2 * np.pi * 0.75)
    assert set(np.unique(m.value[:40])) == {-1000.0} and set(np.unique(m.value[40:80])) == {0.0}


def test_planar_meshes_unchanged_by_axisymmetric_encoding():
    # the icosphere is still triangles only, with the areas of its flat faces
    m = G.icosphere(2)
    assert np.all(m.shape == G.TRIANGLE) and m.n == 320
    assert 0.95 * 4 * np.pi < m.areas().sum() < 4 * np.pi
    mixed = m.concat(G.conic_sphere(10))
    assert (mixed.shape == G.CONIC_SECTION).sum() == 10 and np.isfinite(mixed.centroids()).all()
