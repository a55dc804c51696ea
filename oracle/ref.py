"""ctypes binding of ``oracle/_ref/libkemref.so`` (the reference's own FP64 CPU path).

Test infrastructure: see ``oracle/ref_harness.cc`` for what each call drives.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libkemref.so")
_lib = None

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle ref)")
        L = C.CDLL(LIB_PATH)
        L.kemref_create.restype = C.c_void_p
        L.kemref_create.argtypes = [C.c_int, _ip, _ip, _dp, _dp]
        L.kemref_destroy.argtypes = [C.c_void_p]
        L.kemref_container_index.argtypes = [C.c_void_p, _ip]
        L.kemref_container_index.restype = C.c_int
        L.kemref_set_sigma.argtypes = [C.c_void_p, _dp]
        L.kemref_get_sigma.argtypes = [C.c_void_p, _dp]
        L.kemref_field.argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_int]
        L.kemref_element_field.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp]
        L.kemref_matrix_rows.argtypes = [C.c_void_p, C.c_int, C.c_int, _dp]
        L.kemref_matvec.argtypes = [C.c_void_p, _dp, _dp]
        L.kemref_rhs.argtypes = [C.c_void_p, _dp]
        L.kemref_gmres.argtypes = [C.c_void_p, C.c_double, C.c_int, _dp, _dp]
        L.kemref_gmres.restype = C.c_int
        L.kemref_robinhood.argtypes = [C.c_void_p, C.c_double, _dp, _dp]
        L.kemref_krylov.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_double,
                                    C.c_int, _dp, _dp]
        L.kemref_krylov.restype = C.c_int
        L.kemref_robinhood.restype = C.c_int
        L.kemref_rk8_track.argtypes = [C.c_void_p, _dp, C.c_double, C.c_int, C.c_double, C.c_double, C.c_double, _dp]
        L.kemref_rk8_track.restype = C.c_int
        L.kemref_constant.argtypes = [C.c_int]
        L.kemref_constant.restype = C.c_double
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def constant(name: str) -> float:
    idx = {"one_over_four_pi_eps0": 0, "eps0": 1, "c": 2, "q": 3, "m_el": 4, "pi": 5}[name]
    return lib().kemref_constant(idx)


class RefProblem:
    """One reference KSurfaceContainer + numeric integrator built from a caller element list.

    All vectors at this interface are in the CALLER's element order; the permutation to the
    container's grouped order (KSurfaceContainer.cc:36-72) is applied here.
    """

    def __init__(self, mesh):
        self.n = mesh.n
        self._shape = np.ascontiguousarray(mesh.shape, np.int32)
        self._bnd = np.ascontiguousarray(mesh.boundary, np.int32)
        self._geom = np.ascontiguousarray(mesh.geom, np.float64)
        self._val = np.ascontiguousarray(mesh.value, np.float64)
        self.h = lib().kemref_create(self.n, _i(self._shape), _i(self._bnd), _d(self._geom), _d(self._val))
        idx = np.zeros(self.n, np.int32)
        lib().kemref_container_index(self.h, _i(idx))
        self.cidx = idx  # caller k -> container i

    def close(self):
        if self.h:
            lib().kemref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # caller order <-> container order
    def _to_c(self, v):
        out = np.empty_like(v)
        out[self.cidx] = v
        return np.ascontiguousarray(out)

    def _from_c(self, v):
        return np.ascontiguousarray(v[self.cidx])

    def set_sigma(self, sigma):
        s = self._to_c(np.asarray(sigma, np.float64))
        lib().kemref_set_sigma(self.h, _d(s))

    def get_sigma(self):
        s = np.zeros(self.n)
        lib().kemref_get_sigma(self.h, _d(s))
        return self._from_c(s)

    def field(self, P, mode=0):
        """[m, 4] = (Ex, Ey, Ez, phi) by KIntegratingFieldSolver (Kahan-summed direct sum)."""
        P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
        out = np.zeros((P.shape[0], 4))
        lib().kemref_field(self.h, P.shape[0], _d(P), _d(out), mode)
        return out

    def element_field(self, k, P):
        """[m, 4] normalised (sigma = 1) field and potential of caller element k."""
        P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
        out = np.zeros((P.shape[0], 4))
        lib().kemref_element_field(self.h, int(self.cidx[k]), P.shape[0], _d(P), _d(out))
        return out

    def matrix(self, rows=None):
        """Boundary-integral matrix A (caller order), optionally only the given caller rows."""
        n = self.n
        inv = np.empty(n, np.int64)
        inv[self.cidx] = np.arange(n)
        rows = np.arange(n) if rows is None else np.asarray(rows)
        out = np.zeros((len(rows), n))
        buf = np.zeros(n)
        for r_i, k in enumerate(rows):
            lib().kemref_matrix_rows(self.h, int(self.cidx[k]), 1, _d(buf))
            out[r_i] = buf[self.cidx]
        return out

    def matvec(self, x):
        xc = self._to_c(np.asarray(x, np.float64))
        y = np.zeros(self.n)
        lib().kemref_matvec(self.h, _d(xc), _d(y))
        return self._from_c(y)

    def rhs(self):
        b = np.zeros(self.n)
        lib().kemref_rhs(self.h, _d(b))
        return self._from_c(b)

    def gmres(self, tol=1e-10, max_iter=0):
        x = np.zeros(self.n)
        r = np.zeros(1)
        it = lib().kemref_gmres(self.h, tol, max_iter, _d(x), _d(r))
        return self._from_c(x), it, float(r[0])

    def krylov(self, solver="gmres", preconditioner="none", tol=1e-8, max_iter=500, restart=0,
               preconditioner_tol=0.01, max_preconditioner_iter=30):
        """The reference's Krylov solver factory on the direct system (KBuildKrylovSolver):
        (x, iterations, residual norm over |b|)."""
        x = np.zeros(self.n)
        r = np.zeros(1)
        pc = {"none": 0, "jacobi": 1, "implicit_krylov": 2}[preconditioner]
        it = lib().kemref_krylov(self.h, int(solver == "bicgstab"), pc, tol, max_iter, restart, preconditioner_tol,
                                 max_preconditioner_iter, _d(x), _d(r))
        return self._from_c(x), it, float(r[0])

    def robinhood(self, tol=1e-8):
        x = np.zeros(self.n)
        r = np.zeros(1)
        it = lib().kemref_robinhood(self.h, tol, _d(x), _d(r))
        return self._from_c(x), it, float(r[0])

    def rk8_track(self, state, dt, nsteps, charge=None, mass=None, stop_radius=0.0, record=False):
        st = np.ascontiguousarray(state, np.float64).copy()
        charge = -constant("q") if charge is None else charge
        mass = constant("m_el") if mass is None else mass
        traj = np.zeros((nsteps, 8)) if record else None
        n = lib().kemref_rk8_track(self.h, _d(st), dt, nsteps, charge, mass, stop_radius,
                                   _d(traj) if record else C.cast(None, _dp))
        return st, n, (traj[:n] if record else None)
