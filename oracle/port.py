"""ctypes binding of oracle/libkemoracle.so, the plain-C restatement (test infrastructure).

The rule tables are taken from tests/golden/rules.npz, i.e. from the reference's own
GaussPoints_* functions, so the restatement carries no third copy of the constants.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libkemoracle.so")
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB_PATH} not built (make -C oracle port)")
        L = C.CDLL(LIB_PATH)
        L.kemo_set_rules.argtypes = [_dp] * 8
        L.kemo_set_constants.argtypes = [C.c_double, C.c_double]
        L.kemo_element.argtypes = [C.c_int, _dp, _dp, _dp]
        L.kemo_field.argtypes = [C.c_size_t, _ip, _dp, _dp, C.c_size_t, _dp, _dp]
        L.kemo_matrix.argtypes = [C.c_size_t, _ip, _ip, _dp, _dp, _dp, _dp]
        L.kemo_gmres.argtypes = [C.c_size_t, _dp, _dp, C.c_double, C.c_int, _dp, _dp]
        L.kemo_gmres.restype = C.c_int
        L.kemo_rk8.argtypes = [C.c_size_t, _ip, _dp, _dp, _dp, C.c_double, C.c_int, C.c_double, C.c_double, _dp]
        from . import golden

        r = golden.load("rules")
        keep = [np.ascontiguousarray(r[k], np.float64) for k in
                ("tri7", "tri12", "tri33", "rect7", "rect12", "rect33", "gl4", "gl16")]
        L.kemo_set_rules(*[k.ctypes.data_as(_dp) for k in keep])
        L.kemo_set_constants(1.0 / (4.0 * np.pi * 8.8541878128e-12), 8.8541878128e-12)
        L._keep = keep
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


class PortProblem:
    """Same interface as oracle.ref.RefProblem, on the C restatement (caller order throughout)."""

    def __init__(self, mesh):
        self.n = mesh.n
        self.shape = np.ascontiguousarray(mesh.shape, np.int32)
        self.boundary = np.ascontiguousarray(mesh.boundary, np.int32)
        self.geom = np.ascontiguousarray(mesh.geom, np.float64)
        self.value = np.ascontiguousarray(mesh.value, np.float64)
        self.sigma = np.zeros(self.n)

    def set_sigma(self, s):
        self.sigma = np.ascontiguousarray(s, np.float64)

    def element_field(self, k, P):
        P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
        out = np.zeros((len(P), 4))
        g = np.ascontiguousarray(self.geom[k])
        for i in range(len(P)):
            lib().kemo_element(int(self.shape[k]), _d(g), _d(np.ascontiguousarray(P[i])), _d(out[i]))
        return out

    def field(self, P):
        P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
        out = np.zeros((len(P), 4))
        lib().kemo_field(self.n, self.shape.ctypes.data_as(_ip), _d(self.geom), _d(self.sigma), len(P), _d(P),
                         _d(out))
        return out

    def matrix(self):
        A = np.zeros((self.n, self.n))
        b = np.zeros(self.n)
        lib().kemo_matrix(self.n, self.shape.ctypes.data_as(_ip), self.boundary.ctypes.data_as(_ip), _d(self.geom),
                          _d(self.value), _d(A), _d(b))
        return A, b

    def gmres(self, tol=1e-10, max_iter=500):
        A, b = self.matrix()
        x = np.zeros(self.n)
        r = np.zeros(1)
        it = lib().kemo_gmres(self.n, _d(A), _d(b), tol, max_iter, _d(x), _d(r))
        return x, it, float(r[0])

    def rk8_track(self, state, dt, nsteps, charge, mass):
        st = np.ascontiguousarray(state, np.float64).copy()
        traj = np.zeros((nsteps, 8))
        lib().kemo_rk8(self.n, self.shape.ctypes.data_as(_ip), _d(self.geom), _d(self.sigma), _d(st), dt, nsteps,
                       charge, mass, _d(traj))
        return st, traj
