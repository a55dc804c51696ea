"""ctypes binding of ``oracle/_ref/libkemref_fm.so``: the reference's fast-multipole (FFTM) code.

Test infrastructure: the checker of the device multipole kernels (see ``oracle/fm_harness.cc``
for what each call drives). The library also carries the reference objects of libkemref.so,
so a problem built here has its own surface container.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libkemref_fm.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle fm)")
        L = C.CDLL(LIB_PATH)
        L.kemref_create.restype = C.c_void_p
        L.kemref_create.argtypes = [C.c_int, _ip, _ip, _dp, _dp]
        L.kemref_destroy.argtypes = [C.c_void_p]
        L.kemref_container_index.argtypes = [C.c_void_p, _ip]
        L.kemref_container_index.restype = C.c_int
        L.kemref_set_sigma.argtypes = [C.c_void_p, _dp]
        L.kemref_fm_moments.argtypes = [C.c_int, _dp, _dp, C.c_int, C.c_int, _dp]
        L.kemref_fm_l2p.argtypes = [C.c_int, _dp, C.c_double, _dp, C.c_int, _dp, _dp]
        L.kemref_fm_response.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp]
        L.kemref_fm_field.argtypes = [C.c_void_p, _ip, _dp, C.c_int, _dp, _dp, _dp]
        L.kemref_fm_matvec.argtypes = [C.c_void_p, _ip, _dp, _dp, _dp]
        L.kemref_get_sigma.argtypes = [C.c_void_p, _dp]
        L.kemref_fm_bvs.argtypes = [C.c_void_p, _ip, _dp, C.c_char_p, C.c_char_p, C.c_double, C.c_int, C.c_int,
                                    C.c_double, C.c_int, C.c_int, _ip, _dp, _dp, _dp]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _c(x):
    return np.ascontiguousarray(x, np.float64)


def moments(verts, origin, degree: int, numeric: bool = False) -> np.ndarray:
    """(degree+1)^2 complex moments (index l(l+1)+m) of the wire / triangle / rectangle with these
    vertices, unit total charge, about origin (ConstructExpansion)."""
    v = _c(verts).reshape(-1, 3)
    o = _c(origin)
    out = np.zeros(2 * (degree + 1) ** 2)
    rc = lib().kemref_fm_moments(v.shape[0], _d(v), _d(o), degree, int(numeric), _d(out))
    if rc:
        raise RuntimeError(f"kemref_fm_moments returned {rc}")
    return out[0::2] + 1j * out[1::2]


def l2p(degree: int, origin, coeff, P, expansion_radius: float = 1.0) -> np.ndarray:
    """(Ex, Ey, Ez, phi) of a local expansion (coefficients for m >= 0, index l(l+1)/2+m) at P."""
    c = np.zeros(2 * len(coeff))
    c[0::2] = np.real(coeff)
    c[1::2] = np.imag(coeff)
    P = _c(P).reshape(-1, 3)
    out = np.zeros((P.shape[0], 4))
    lib().kemref_fm_l2p(degree, _d(_c(origin)), expansion_radius, _d(c), P.shape[0], _d(P), _d(out))
    return out


def response(kind: int, degree: int, source_origin, target_origin) -> np.ndarray:
    """[target, source] complex response matrix of kind 0 M2M, 1 M2L, 2 L2L."""
    S = (degree + 1) ** 2
    out = np.zeros(2 * S * S)
    lib().kemref_fm_response(kind, degree, _d(_c(source_origin)), _d(_c(target_origin)), _d(out))
    return (out[0::2] + 1j * out[1::2]).reshape(S, S)


class FmRefProblem:
    """The reference FFTM field solver on a caller element list (caller order for sigma)."""

    def __init__(self, mesh):
        self.n = mesh.n
        self._shape = np.ascontiguousarray(mesh.shape, np.int32)
        self._bnd = np.ascontiguousarray(mesh.boundary, np.int32)
        self._geom = _c(mesh.geom)
        self._val = _c(mesh.value)
        ip = lambda a: a.ctypes.data_as(_ip)  # noqa: E731
        self.h = lib().kemref_create(self.n, ip(self._shape), ip(self._bnd), _d(self._geom), _d(self._val))
        idx = np.zeros(self.n, np.int32)
        lib().kemref_container_index(self.h, ip(idx))
        self.cidx = idx

    def close(self):
        if self.h:
            lib().kemref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_sigma(self, sigma):
        s = np.empty(self.n)
        s[self.cidx] = np.asarray(sigma, np.float64)
        s = _c(s)
        lib().kemref_set_sigma(self.h, _d(s))

    def matvec(self, x, degree=8, top_level_divisions=2, divisions=2, zeromask=1, maximum_tree_depth=3,
               insertion_ratio=4.0 / 3.0, region_expansion_factor=1.1):
        """A x with the reference's fast-multipole matrix (caller order)."""
        ipar = np.ascontiguousarray([degree, top_level_divisions, divisions, zeromask, maximum_tree_depth],
                                    np.int32)
        dpar = _c([insertion_ratio, region_expansion_factor])
        xc = np.empty(self.n)
        xc[self.cidx] = np.asarray(x, np.float64)
        xc = _c(xc)
        yc = np.zeros(self.n)
        lib().kemref_fm_matvec(self.h, ipar.ctypes.data_as(_ip), _d(dpar), _d(xc), _d(yc))
        return np.ascontiguousarray(yc[self.cidx])

    def field(self, P, degree=8, top_level_divisions=2, divisions=2, zeromask=1, maximum_tree_depth=3,
              insertion_ratio=4.0 / 3.0, region_expansion_factor=1.1):
        """(n x 4 field and potential, world cube (centre xyz, side)) from a freshly built tree."""
        ipar = np.ascontiguousarray([degree, top_level_divisions, divisions, zeromask, maximum_tree_depth],
                                    np.int32)
        dpar = _c([insertion_ratio, region_expansion_factor])
        P = _c(P).reshape(-1, 3)
        out = np.zeros((P.shape[0], 4))
        world = np.zeros(4)
        lib().kemref_fm_field(self.h, ipar.ctypes.data_as(_ip), _d(dpar), P.shape[0], _d(P), _d(out), _d(world))
        return out, world

    def solve(self, solver="gmres", preconditioner="none", tol=1e-6, max_iter=500, restart=0, preconditioner_tol=0.01,
              max_preconditioner_iter=30, preconditioner_degree=1, preconditioner_params=None, **tree):
        """The reference's fast-multipole charge-density solve (KFMElectrostaticFastMultipoleBoundaryValueSolver,
        the solver of krylov_bem_solver): (x in caller order, residual norm over |b|). tree: the
        solver tree's parameters as matvec; preconditioner_params: those of the independent
        preconditioner tree (independent_implicit_krylov)."""
        def params(degree=8, top_level_divisions=2, divisions=2, zeromask=1, maximum_tree_depth=3,
                   insertion_ratio=4.0 / 3.0, region_expansion_factor=1.1):
            return (np.ascontiguousarray([degree, top_level_divisions, divisions, zeromask, maximum_tree_depth],
                                         np.int32), _c([insertion_ratio, region_expansion_factor]))
        ipar, dpar = params(**tree)
        pip, pdp = params(**(preconditioner_params or tree))
        x = np.zeros(self.n)
        r = np.zeros(1)
        rc = lib().kemref_fm_bvs(self.h, ipar.ctypes.data_as(_ip), _d(dpar), solver.encode(), preconditioner.encode(),
                                 tol, max_iter, restart, preconditioner_tol, max_preconditioner_iter,
                                 preconditioner_degree, pip.ctypes.data_as(_ip), _d(pdp), _d(x), _d(r))
        if rc != 0:
            raise RuntimeError(f"kemref_fm_bvs failed ({rc})")
        return np.ascontiguousarray(x[self.cidx]), float(r[0])
