"""Seeded synthetic meshes, field points and particle states for the benchmark configurations.

The reference builds its meshes with KGeoBag and converts them with KGBEMMeshConverter
(KEMField/Source/Interface/KGeoBag/src/KGBEMConverter.cc); that stack needs Boost and is
outside the hot path, so the configurations are synthesised here directly as element lists
in the reference's element encoding:

* triangle / rectangle: ``geom = (A, B, P0x, P0y, P0z, N1x, N1y, N1z, N2x, N2y, N2z)`` with
  ``P1 = P0 + A*N1`` and ``P2 = P0 + B*N2`` (KTriangle::SetValues(p0, p1, p2),
  KEMField/Source/Surfaces/src/KTriangle.cc:18-28; KRectangle.hh:132-137);
* line segment: ``geom = (P0x, P0y, P0z, P1x, P1y, P1z, diameter, 0, 0, 0, 0)``
  (KEMField/Source/Surfaces/include/KLineSegment.hh:74-76);
* conic section: ``geom = (r0, z0, r1, z1, 0, ...)``, the generator from (r0, z0) to (r1, z1)
  turned about the z axis (KEMField/Source/Surfaces/include/KConicSection.hh);
* ring: ``geom = (r, z, 0, ...)`` (KEMField/Source/Surfaces/include/KRing.hh).
  A mesh holds either planar elements or axisymmetric ones.

Every generator is deterministic for a given seed (numpy ``default_rng``).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

TRIANGLE, RECTANGLE, LINE_SEGMENT, CONIC_SECTION, RING = 0, 1, 2, 3, 4
DIRICHLET, NEUMANN = 0, 1


@dataclass
class Mesh:
    """Element list in container order (the matrix row/column order)."""

    shape: np.ndarray  # int32 [n]
    boundary: np.ndarray  # int32 [n]
    geom: np.ndarray  # float64 [n, 11]
    value: np.ndarray  # float64 [n] Dirichlet potential or Neumann flux ratio
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.shape.shape[0])

    def concat(self, other: "Mesh") -> "Mesh":
        return Mesh(
            np.concatenate([self.shape, other.shape]).astype(np.int32),
            np.concatenate([self.boundary, other.boundary]).astype(np.int32),
            np.concatenate([self.geom, other.geom]),
            np.concatenate([self.value, other.value]),
            name=self.name or other.name,
            meta={**other.meta, **self.meta},
        )

    def centroids(self) -> np.ndarray:
        g = self.geom
        c = np.empty((self.n, 3))
        tri = self.shape == TRIANGLE
        rect = self.shape == RECTANGLE
        line = self.shape == LINE_SEGMENT
        c[tri] = g[tri, 2:5] + (g[tri, 0:1] * g[tri, 5:8] + g[tri, 1:2] * g[tri, 8:11]) / 3.0
        c[rect] = g[rect, 2:5] + 0.5 * g[rect, 0:1] * g[rect, 5:8] + 0.5 * g[rect, 1:2] * g[rect, 8:11]
        c[line] = 0.5 * (g[line, 0:3] + g[line, 3:6])
        conic = self.shape == CONIC_SECTION
        ring = self.shape == RING
        c[conic] = np.stack([0.5 * (g[conic, 0] + g[conic, 2]), np.zeros(int(conic.sum())),
                             0.5 * (g[conic, 1] + g[conic, 3])], axis=1)
        c[ring] = np.stack([g[ring, 0], np.zeros(int(ring.sum())), g[ring, 1]], axis=1)
        return c

    def areas(self) -> np.ndarray:
        g = self.geom
        a = np.empty(self.n)
        tri = self.shape == TRIANGLE
        rect = self.shape == RECTANGLE
        line = self.shape == LINE_SEGMENT
        cr = np.cross(g[tri, 5:8], g[tri, 8:11])
        a[tri] = 0.5 * g[tri, 0] * g[tri, 1] * np.linalg.norm(cr, axis=1)
        a[rect] = g[rect, 0] * g[rect, 1]
        a[line] = np.pi * g[line, 6] * np.linalg.norm(g[line, 3:6] - g[line, 0:3], axis=1)
        conic = self.shape == CONIC_SECTION
        a[conic] = np.pi * (g[conic, 0] + g[conic, 2]) * np.hypot(g[conic, 0] - g[conic, 2], g[conic, 1] - g[conic, 3])
        a[self.shape == RING] = 2.0 * np.pi * g[self.shape == RING, 0]  # KRing::Area (KRing.cc:20-23)
        return a


def axisymmetric(shape, r0, z0, r1=None, z1=None, value=1.0, name: str = "") -> Mesh:
    """Conic sections (``r1``, ``z1`` given) or rings from per-element arrays, Dirichlet."""
    r0 = np.atleast_1d(np.asarray(r0, np.float64))
    n = r0.shape[0]
    geom = np.zeros((n, 11))
    geom[:, 0] = r0
    geom[:, 1] = np.broadcast_to(np.asarray(z0, np.float64), (n,))
    if r1 is not None:
        geom[:, 2] = np.broadcast_to(np.asarray(r1, np.float64), (n,))
        geom[:, 3] = np.broadcast_to(np.asarray(z1, np.float64), (n,))
    return Mesh(np.full(n, shape, np.int32), np.full(n, DIRICHLET, np.int32), geom,
                np.broadcast_to(np.asarray(value, np.float64), (n,)).copy(), name=name)


def conic_sphere(n_sections: int = 200, radius: float = 1.0, potential: float = 1.0) -> Mesh:
    """Sphere as ``n_sections`` conic sections between equally spaced polar angles (the
    generator a chord of the meridian; the first and last sections are cones meeting the
    axis). Its capacitance tends to 4 pi eps0 radius as the sections shrink."""
    th = np.linspace(0.0, np.pi, n_sections + 1)
    r, z = radius * np.sin(th), radius * np.cos(th)
    r[0] = r[-1] = 0.0
    m = axisymmetric(CONIC_SECTION, r[:-1], z[:-1], r[1:], z[1:], potential, name="conic-sphere")
    m.meta = {"n_sections": n_sections, "radius": radius}
    return m


def conic_disk(n_sections: int = 128, radius: float = 1.0, power: float = 1.5, potential: float = 1.0) -> Mesh:
    """Flat disk of ``n_sections`` annular conic sections at z = 0, from the rim inwards, their
    widths growing like a power law away from the rim: the mesh of the reference's disk
    capacitance test (UnitTest/KEMField/Fields/src/DiskCapacitanceTest.cc:47-69: the first half
    of :func:`power_interval` over the diameter in 2 n segments). Capacitance 8 eps0 R."""
    n = n_sections
    seg = power_interval(2.0 * radius, 2 * n, power)[:n]  # the rim-to-centre half of a diameter
    r_out, r_in = np.empty(n), np.empty(n)
    r0 = r1 = radius
    for i in range(n):  # r1 -= segment, in sequence, as the test builds its sections
        r1 -= seg[i]
        r_out[i], r_in[i] = r0, max(r1, 0.0)  # the last edge lands on the axis up to rounding
        r0 = r1
    m = axisymmetric(CONIC_SECTION, r_out, 0.0, r_in, 0.0, potential, name="conic-disk")
    m.meta = {"n_sections": n, "radius": radius, "power": power}
    return m


def conic_coax(n_z: int = 100, n_cap: int = 10, r_in: float = 0.5, r_out: float = 1.0, length: float = 4.0,
               v_in: float = -1000.0, v_out: float = 0.0, n_rings: int = 0) -> Mesh:
    """Axisymmetric counterpart of :func:`coax`: inner and outer cylinders of ``n_z``
    conic sections each, annular end caps of ``n_cap`` sections at z = +-length/2, plus
    ``n_rings`` rings (thin wires) at the inner potential spread over the gap's mid-radius."""
    z = np.linspace(-length / 2, length / 2, n_z + 1)
    parts = [axisymmetric(CONIC_SECTION, np.full(n_z, r_in), z[:-1], np.full(n_z, r_in), z[1:], v_in),
             axisymmetric(CONIC_SECTION, np.full(n_z, r_out), z[:-1], np.full(n_z, r_out), z[1:], v_out)]
    rr = np.linspace(r_in, r_out, n_cap + 1)
    for zc in (-length / 2, length / 2):
        parts.append(axisymmetric(CONIC_SECTION, rr[:-1], np.full(n_cap, zc), rr[1:], np.full(n_cap, zc),
                                  np.where(0.5 * (rr[:-1] + rr[1:]) < 0.5 * (r_in + r_out), v_in, v_out)))
    if n_rings:
        zr = np.linspace(-length / 4, length / 4, n_rings)
        parts.append(axisymmetric(RING, np.full(n_rings, 0.5 * (r_in + r_out)), zr, value=v_in))
    m = parts[0]
    for p in parts[1:]:
        m = m.concat(p)
    m.name = "conic-coax"
    m.meta = {"n_z": n_z, "n_cap": n_cap, "n_rings": n_rings}
    return m


def triangles_from_vertices(p0, p1, p2, value, boundary=DIRICHLET) -> Mesh:
    """Triangles from vertex triples, as KTriangle::SetValues(p0, p1, p2) stores them."""
    p0, p1, p2 = (np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in (p0, p1, p2))
    e1, e2 = p1 - p0, p2 - p0
    a, b = np.linalg.norm(e1, axis=1), np.linalg.norm(e2, axis=1)
    geom = np.concatenate([a[:, None], b[:, None], p0, e1 / a[:, None], e2 / b[:, None]], axis=1)
    n = p0.shape[0]
    return Mesh(
        np.full(n, TRIANGLE, np.int32),
        np.full(n, boundary, np.int32),
        geom,
        np.broadcast_to(np.asarray(value, np.float64), (n,)).copy(),
    )


def rectangles_from_corners(p0, p1, p3, value, boundary=DIRICHLET) -> Mesh:
    """Rectangles from the corner P0 and its two neighbours P1 = P0 + A*N1, P3 = P0 + B*N2."""
    p0, p1, p3 = (np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in (p0, p1, p3))
    e1, e2 = p1 - p0, p3 - p0
    a, b = np.linalg.norm(e1, axis=1), np.linalg.norm(e2, axis=1)
    geom = np.concatenate([a[:, None], b[:, None], p0, e1 / a[:, None], e2 / b[:, None]], axis=1)
    n = p0.shape[0]
    return Mesh(
        np.full(n, RECTANGLE, np.int32),
        np.full(n, boundary, np.int32),
        geom,
        np.broadcast_to(np.asarray(value, np.float64), (n,)).copy(),
    )


def line_segments(p0, p1, diameter, value, boundary=DIRICHLET) -> Mesh:
    p0, p1 = (np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in (p0, p1))
    n = p0.shape[0]
    geom = np.zeros((n, 11))
    geom[:, 0:3] = p0
    geom[:, 3:6] = p1
    geom[:, 6] = diameter
    return Mesh(
        np.full(n, LINE_SEGMENT, np.int32),
        np.full(n, boundary, np.int32),
        geom,
        np.broadcast_to(np.asarray(value, np.float64), (n,)).copy(),
    )


# --------------------------------------------------------------------------- icosphere
def power_interval(length: float, n: int, power: float) -> np.ndarray:
    """Segment lengths of an interval refined towards both ends: n segments symmetric about
    the middle, half-interval widths ((i+1)/(n/2))^p - (i/(n/2))^p, a middle segment of length /
    n when n is odd (the DiscretizeInterval of the reference's capacitance tests,
    UnitTest/KEMField/Fields/src/DiskCapacitanceTest.cc:117-141)."""
    seg = np.empty(n)
    if n == 1:
        seg[0] = length
        return seg
    mid = length * 0.5
    if n % 2 == 1:
        seg[n // 2] = length / n
        mid -= length / (2 * n)
    for i in range(n // 2):
        inc1 = (i / (n / 2.0)) ** power
        inc2 = ((i + 1) / (n / 2.0)) ** power
        seg[i] = seg[n - (i + 1)] = mid * (inc2 - inc1)
    return seg


def cube(scale: int = 8, power: float = 1.5, side: float = 1.0, potential: float = 1.0) -> Mesh:
    """Cube of ``side`` centred at the origin, each face ``scale`` x ``scale`` rectangles on the
    power-law grid of :func:`power_interval` (the box of the reference's cube capacitance test,
    UnitTest/KEMField/Fields/src/CubeCapacitanceTest.cc:43-60: mesh count 8, power 1.5).
    Capacitance 0.6606785 x 4 pi eps0 side."""
    edges = -side / 2 + np.concatenate([[0.0], np.cumsum(power_interval(side, scale, power))])
    edges[-1] = side / 2
    u0, v0 = np.meshgrid(edges[:-1], edges[:-1], indexing="ij")
    u1, v1 = np.meshgrid(edges[1:], edges[1:], indexing="ij")
    u0, v0, u1, v1 = u0.ravel(), v0.ravel(), u1.ravel(), v1.ravel()
    h = np.full(u0.shape, side / 2)
    parts = []
    for axis in range(3):
        for sgn in (-1.0, 1.0):
            def pt(u, v):
                c = [None, None, None]
                c[axis] = sgn * h
                others = [k for k in range(3) if k != axis]
                c[others[0]], c[others[1]] = u, v
                return np.stack(c, axis=1)
            parts.append(rectangles_from_corners(pt(u0, v0), pt(u1, v0), pt(u0, v1), potential))
    m = parts[0]
    for p in parts[1:]:
        m = m.concat(p)
    m.name = "cube"
    m.meta = {"scale": scale, "power": power, "side": side}
    return m


def icosphere_vertices(level: int, radius: float = 1.0):
    """Vertices and faces of a subdivided icosahedron (20 * 4**level faces, outward winding)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t),
         (0, -1, -t), (0, 1, -t), (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, float) / np.linalg.norm(p) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4),
             (11, 10, 2), (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8),
             (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(level):
        cache: dict = {}

        def mid(i, j):
            key = (min(i, j), max(i, j))
            if key not in cache:
                m = verts[i] + verts[j]
                verts.append(m / np.linalg.norm(m))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = nf
    return np.array(verts) * radius, np.array(faces, dtype=np.int64)


def icosphere(level: int = 3, radius: float = 1.0, potential: float = 1.0) -> Mesh:
    """Conducting sphere as a flat-triangle icosphere held at ``potential`` (configuration 1:
    level 3 = 1,280 triangles; configuration 4: level 5 = 20,480 triangles)."""
    v, f = icosphere_vertices(level, radius)
    p0, p1, p2 = v[f[:, 0]], v[f[:, 1]], v[f[:, 2]]
    # orient every face outwards (N1 x N2 along the radial direction)
    nrm = np.cross(p1 - p0, p2 - p0)
    flip = np.einsum("ij,ij->i", nrm, p0 + p1 + p2) < 0
    p1[flip], p2[flip] = p2[flip].copy(), p1[flip].copy()
    m = triangles_from_vertices(p0, p1, p2, potential)
    m.name = f"icosphere-L{level}"
    m.meta = {"radius": radius, "potential": potential, "n_tri": int(m.n)}
    return m


# --------------------------------------------------------------------------- coax
def coax(n_phi: int = 100, n_z: int = 200, n_cap_rings: int = 10, r_in: float = 0.5, r_out: float = 1.0,
         length: float = 4.0, v_in: float = -1000.0, v_out: float = 0.0) -> Mesh:
    """Coaxial electrodes (configuration 2): two faceted cylinders of ``n_phi * n_z`` rectangles
    each, plus annular end caps of ``2 * n_phi * n_cap_rings`` triangles per cap.

    The caps close the gap between the electrodes; they are held at the ideal infinite-coax
    potential V(r) = v_out + (v_in - v_out) * ln(r_out/r) / ln(r_out/r_in) at each triangle's
    centroid radius, so the gap field approaches the analytic coax field far from the caps.
    """
    zs = np.linspace(-length / 2, length / 2, n_z + 1)
    ph = np.linspace(0.0, 2 * np.pi, n_phi + 1)
    meshes = []
    for r, v, outward in ((r_in, v_in, True), (r_out, v_out, False)):
        i, j = np.meshgrid(np.arange(n_phi), np.arange(n_z), indexing="ij")
        i, j = i.ravel(), j.ravel()
        c0 = np.stack([r * np.cos(ph[i]), r * np.sin(ph[i]), zs[j]], axis=1)
        c1 = np.stack([r * np.cos(ph[i + 1]), r * np.sin(ph[i + 1]), zs[j]], axis=1)
        c3 = np.stack([r * np.cos(ph[i]), r * np.sin(ph[i]), zs[j + 1]], axis=1)
        if outward:  # N1 x N2 radially outwards for the inner electrode
            meshes.append(rectangles_from_corners(c0, c1, c3, v))
        else:
            meshes.append(rectangles_from_corners(c0, c3, c1, v))
    rr = np.linspace(r_in, r_out, n_cap_rings + 1)
    for zc in (-length / 2, length / 2):
        i, k = np.meshgrid(np.arange(n_phi), np.arange(n_cap_rings), indexing="ij")
        i, k = i.ravel(), k.ravel()

        def pt(ii, kk):
            return np.stack([rr[kk] * np.cos(ph[ii]), rr[kk] * np.sin(ph[ii]), np.full(ii.shape, zc)], axis=1)

        a, b, c, d = pt(i, k), pt(i + 1, k), pt(i + 1, k + 1), pt(i, k + 1)
        p0 = np.concatenate([a, a])
        p1 = np.concatenate([b, c])
        p2 = np.concatenate([c, d])
        cen_r = np.linalg.norm(((p0 + p1 + p2) / 3.0)[:, :2], axis=1)
        vcap = v_out + (v_in - v_out) * np.log(r_out / cen_r) / np.log(r_out / r_in)
        meshes.append(triangles_from_vertices(p0, p1, p2, vcap))
    m = meshes[0]
    for mm in meshes[1:]:
        m = m.concat(mm)
    m.name = "coax"
    m.meta = {"r_in": r_in, "r_out": r_out, "length": length, "v_in": v_in, "v_out": v_out,
              "n_rect": 2 * n_phi * n_z, "n_tri": 4 * n_phi * n_cap_rings}
    return m


def coax_potential(r, r_in=0.5, r_out=1.0, v_in=-1000.0, v_out=0.0):
    """Ideal infinite-coax potential (analytic sanity bound for configuration 2)."""
    return v_out + (v_in - v_out) * np.log(r_out / r) / np.log(r_out / r_in)


def coax_density(mesh: Mesh, seed: int = 31, spread: float = 0.05, eps0: float = 8.8541878128e-12) -> np.ndarray:
    """A fixed charge density for field evaluations on :func:`coax` meshes without a solve:
    the ideal infinite-coax surface density eps0 (v_out - v_in) / (r ln(r_out / r_in)) (negative
    on the inner electrode, positive on the outer one, a tenth of the outer value on the caps)
    times 1 + spread N(0, 1) from a seeded generator. The direct sum is linear in the density,
    so any fixed density pins the evaluation; this one has the solution's size and signs."""
    meta = mesh.meta
    r_in, r_out = meta.get("r_in", 0.5), meta.get("r_out", 1.0)
    dv = meta.get("v_out", 0.0) - meta.get("v_in", -1000.0)
    c = mesh.centroids()
    r = np.hypot(c[:, 0], c[:, 1])
    s = eps0 * dv / (r * np.log(r_out / r_in))
    inner = (mesh.shape == RECTANGLE) & (np.abs(r - r_in) < 0.5 * (r_out - r_in))
    s = np.where(mesh.shape == RECTANGLE, np.where(inner, -s, s), 0.1 * s)
    rng = np.random.default_rng(seed)
    return s * (1.0 + spread * rng.normal(size=mesh.n))


def sphere_density(mesh: Mesh, radius: float = 1.0, potential: float = 1.0, seed: int | None = None,
                   spread: float = 0.1, eps0: float = 8.8541878128e-12) -> np.ndarray:
    """Surface density eps0 V / R of a conducting sphere at potential V, optionally times
    1 + spread N(0, 1) from a seeded generator (the perturbed density of configuration 4)."""
    s = np.full(mesh.n, eps0 * potential / radius)
    if seed is not None:
        s = s * (1.0 + spread * np.random.default_rng(seed).normal(size=mesh.n))
    return s


# --------------------------------------------------------------------------- stacked rings
def stacked_rings(n_rings: int = 8, n_phi: int = 125, n_z: int = 50, r_min: float = 0.3, r_max: float = 1.0,
                  height: float = 0.2, gap: float = 0.1, jitter: float = 1e-3, seed: int = 5) -> Mesh:
    """Configuration 5: ``n_rings`` coaxial ring electrodes stacked along z, radii spaced
    linearly in [r_min, r_max], each a triangulated cylindrical band of ``2 * n_phi * n_z``
    triangles (8 x 12,500 = 100,000 by default), every mesh vertex displaced by N(0, jitter)
    from a seeded generator. ``value`` holds the electrode index; right-hand sides are built
    with :func:`ring_potentials`."""
    rng = np.random.default_rng(seed)
    radii = np.linspace(r_min, r_max, n_rings)
    meshes = []
    z0 = -0.5 * (n_rings * height + (n_rings - 1) * gap)
    for k, r in enumerate(radii):
        zb = z0 + k * (height + gap)
        ph = np.linspace(0, 2 * np.pi, n_phi, endpoint=False)
        zz = np.linspace(zb, zb + height, n_z + 1)
        P = np.stack(np.broadcast_arrays(r * np.cos(ph)[:, None], r * np.sin(ph)[:, None], zz[None, :]), axis=-1)
        P = P + rng.normal(0.0, jitter, P.shape)
        i, j = np.meshgrid(np.arange(n_phi), np.arange(n_z), indexing="ij")
        i, j = i.ravel(), j.ravel()
        ip = (i + 1) % n_phi
        a, b, c, d = P[i, j], P[ip, j], P[ip, j + 1], P[i, j + 1]
        m = triangles_from_vertices(np.concatenate([a, a]), np.concatenate([b, c]), np.concatenate([c, d]),
                                    float(k))
        meshes.append(m)
    m = meshes[0]
    for mm in meshes[1:]:
        m = m.concat(mm)
    m.name = "stacked-rings"
    m.meta = {"n_rings": n_rings, "radii": radii.tolist(), "jitter": jitter, "seed": seed}
    return m


def ring_potentials(mesh: Mesh, n_rhs: int = 8, seed: int = 7) -> np.ndarray:
    """[n_rhs, n] right-hand sides: per-electrode potentials drawn from U[-1000, 0] V."""
    rng = np.random.default_rng(seed)
    n_rings = int(mesh.value.max()) + 1
    pots = rng.uniform(-1000.0, 0.0, size=(n_rhs, n_rings))
    return pots[:, mesh.value.astype(np.int64)]


# --------------------------------------------------------------------------- points / particles
def shell_points(n: int, r_min: float = 1.2, r_max: float = 3.0, seed: int = 12345) -> np.ndarray:
    """Points uniform in the spherical shell r_min < r < r_max (configurations 1, 3 and 4)."""
    rng = np.random.default_rng(seed)
    u = rng.random(n)
    r = np.cbrt(r_min ** 3 + u * (r_max ** 3 - r_min ** 3))
    z = 2.0 * rng.random(n) - 1.0
    phi = 2.0 * np.pi * rng.random(n)
    s = np.sqrt(1.0 - z * z)
    return np.stack([r * s * np.cos(phi), r * s * np.sin(phi), r * z], axis=1)


def gap_points(n: int, r_in: float = 0.5, r_out: float = 1.0, length: float = 4.0, seed: int = 2024) -> np.ndarray:
    """Points uniform in the annular gap volume of the coax (configuration 2)."""
    rng = np.random.default_rng(seed)
    r = np.sqrt(r_in ** 2 + rng.random(n) * (r_out ** 2 - r_in ** 2))
    phi = 2.0 * np.pi * rng.random(n)
    z = (rng.random(n) - 0.5) * length
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


ELECTRON_MASS = 9.1093837015e-31  # kg, KConst::M_el_kg() (Kommon/Base/Utility/KConst_2021.h:163)
ELEMENTARY_CHARGE = 1.602176634e-19  # C, KConst::Q() (KConst_2021.h:51)
SPEED_OF_LIGHT = 299792458.0  # m/s, KConst::C() (KConst_2021.h:46)


def electrons(n: int, e_min_ev: float = 1000.0, e_max_ev: float = 18600.0, r_min: float = 1.2, r_max: float = 3.0,
              seed: int = 99) -> np.ndarray:
    """[n, 8] exact-trajectory states (t, s, x, y, z, px, py, pz) for configuration 3:
    kinetic energy uniform in [e_min, e_max] eV, isotropic direction, start uniform in the
    shell (state layout: Kassiopeia/Trajectories/Source/KSTrajExactParticle.cxx:102-121)."""
    rng = np.random.default_rng(seed)
    x = shell_points(n, r_min, r_max, seed=seed + 1)
    ekin = (e_min_ev + (e_max_ev - e_min_ev) * rng.random(n)) * ELEMENTARY_CHARGE
    mc2 = ELECTRON_MASS * SPEED_OF_LIGHT ** 2
    pmag = np.sqrt(ekin * ekin + 2.0 * ekin * mc2) / SPEED_OF_LIGHT
    z = 2.0 * rng.random(n) - 1.0
    phi = 2.0 * np.pi * rng.random(n)
    s = np.sqrt(1.0 - z * z)
    d = np.stack([s * np.cos(phi), s * np.sin(phi), z], axis=1)
    st = np.zeros((n, 8))
    st[:, 2:5] = x
    st[:, 5:8] = pmag[:, None] * d
    return st
