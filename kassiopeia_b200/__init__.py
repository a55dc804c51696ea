"""kassiopeia_b200 -- B200-native (sm_100a) backend for KEMField's electrostatic BEM hot path.

The product is ``libkemcu.so`` (C ABI: ``include/kemcu.h``) built from ``csrc/``. This module
is a thin Python mirror of the reference-facing interface, used by the tests and the
benchmark, with the reference's names:

* :class:`CUDAElectrostaticContext` -- one GPU context holding a flattened surface container
  (the KOpenCLSurfaceContainer analogue) and its charge densities;
* :meth:`~CUDAElectrostaticContext.ElectricFieldAndPotential` / ``Potential`` /
  ``ElectricField`` -- batched KIntegratingFieldSolver (direct summation);
* :meth:`~CUDAElectrostaticContext.Multiply` -- KBoundaryIntegralMatrix::Multiply;
* :meth:`~CUDAElectrostaticContext.Solve` -- the GMRES charge-density solve;
* :meth:`~CUDAElectrostaticContext.TrackRK8` -- batched exact-trajectory RK8 steps;
* :meth:`~CUDAElectrostaticContext.FieldVJP` -- adjoint of the direct sum.

Every call goes to the GPU; a missing library or device raises instead of falling back.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from ._native import (FIELD, FIELD_AND_POTENTIAL, FP32, FP64, MIXED, POTENTIAL, SOLVE_ASSEMBLED, SOLVE_ASSEMBLED_FP64,
                      SOLVE_FFTM, SOLVE_FP32, SOLVE_MIXED, SOLVE_PLAIN, KemcuError)

__all__ = ["CUDAElectrostaticContext", "KemcuError", "FP64", "MIXED", "FP32", "SOLVE_PLAIN", "SOLVE_MIXED",
           "SOLVE_ASSEMBLED", "SOLVE_ASSEMBLED_FP64", "SOLVE_FP32", "SOLVE_FFTM", "FIELD_AND_POTENTIAL", "POTENTIAL", "FIELD"]

ONE_OVER_FOUR_PI_EPS0 = 1.0 / (4.0 * np.pi * 8.8541878128e-12)  # KEMConstants (KConst epoch 2021)
EPS0 = 8.8541878128e-12


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


class CUDAElectrostaticContext:
    """One device context; not re-entrant (use one per thread)."""

    def __init__(self, device: int = 0, assembled_budget_bytes: int = 0, autotune: bool = True):
        L = N.lib()
        cfg = N.Config()
        L.kemcu_default_config(C.byref(cfg))
        cfg.device = device
        cfg.one_over_four_pi_eps0 = ONE_OVER_FOUR_PI_EPS0
        cfg.eps0 = EPS0
        cfg.assembled_budget_bytes = assembled_budget_bytes
        cfg.autotune = int(bool(autotune))
        h = C.c_void_p()
        rc = L.kemcu_create(C.byref(h), C.byref(cfg))
        self._h = h
        self._cb = None
        if rc != N.OK:
            msg = L.kemcu_last_error(h).decode() if h else "context creation failed"
            L.kemcu_destroy(h)
            self._h = None
            raise KemcuError(rc, msg)
        self.n = 0

    # -- plumbing
    def _check(self, rc):
        if rc != N.OK:
            raise KemcuError(rc, N.lib().kemcu_last_error(self._h).decode())

    def close(self):
        if getattr(self, "_h", None):
            N.lib().kemcu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def last_kernel_ms(self) -> float:
        return N.lib().kemcu_last_kernel_ms(self._h)

    # -- container
    def SetGeometry(self, mesh):
        self._shape = np.ascontiguousarray(mesh.shape, np.int32)
        self._bnd = np.ascontiguousarray(mesh.boundary, np.int32)
        self._geom = np.ascontiguousarray(mesh.geom, np.float64)
        self._val = np.ascontiguousarray(mesh.value, np.float64)
        self._check(N.lib().kemcu_set_geometry(self._h, mesh.n, _i(self._shape), _i(self._bnd), _d(self._geom),
                                               _d(self._val)))
        self.n = mesh.n

    def SetSigma(self, sigma):
        s = np.ascontiguousarray(sigma, np.float64)
        assert s.shape == (self.n,)
        self._check(N.lib().kemcu_set_sigma(self._h, _d(s)))

    def GetSigma(self):
        s = np.zeros(self.n)
        self._check(N.lib().kemcu_get_sigma(self._h, _d(s)))
        return s

    def RHS(self):
        b = np.zeros(self.n)
        self._check(N.lib().kemcu_rhs(self._h, _d(b)))
        return b

    # -- direct summation
    def ElectricFieldAndPotential(self, P, precision=FP64, what=FIELD_AND_POTENTIAL):
        P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
        out = np.zeros((P.shape[0], 4))
        self._check(N.lib().kemcu_field(self._h, _d(P), P.shape[0], _d(out), precision, what))
        return out

    def Potential(self, P, precision=FP64):
        return self.ElectricFieldAndPotential(P, precision, POTENTIAL)[:, 3]

    def ElectricField(self, P, precision=FP64):
        return self.ElectricFieldAndPotential(P, precision, FIELD)[:, :3]

    def FieldDevice(self, d_points_ptr: int, n: int, d_out_ptr: int, precision=FP64, what=FIELD_AND_POTENTIAL):
        """Device-pointer variant (e.g. torch tensors' data_ptr())."""
        self._check(N.lib().kemcu_field_dev(self._h, C.c_void_p(d_points_ptr), n, C.c_void_p(d_out_ptr), precision,
                                            what))

    # -- autotuner of the direct sum's launch shape
    def TuneField(self, d_points_ptr: int, n: int, d_out_ptr: int, precision=FP64):
        """Time every launch shape of the direct-sum kernel on these device points (the field lands
        in d_out); returns (chosen shape, [K1 milliseconds per shape])."""
        L = N.lib()
        nv = L.kemcu_field_variant_count()
        ms = (C.c_float * nv)()
        v = C.c_int(-1)
        self._check(L.kemcu_tune_field(self._h, C.c_void_p(d_points_ptr), n, C.c_void_p(d_out_ptr), precision,
                                       C.byref(v), ms))
        return v.value, [float(x) for x in ms]

    def FieldVariant(self, n: int, precision=FP64) -> int:
        """The launch shape the autotuner chose for n points (-1: none yet)."""
        v = C.c_int(-1)
        self._check(N.lib().kemcu_field_variant(self._h, n, precision, C.byref(v)))
        return v.value

    @staticmethod
    def FieldVariantInfo(v: int) -> dict:
        mb, rs = C.c_int(), C.c_int()
        if N.lib().kemcu_field_variant_info(v, C.byref(mb), C.byref(rs)) != N.OK:
            raise KemcuError(N.EINVAL, f"no launch shape {v}")
        return {"variant": v, "ctas_per_sm": mb.value, "ring_stages": rs.value}

    # -- matrix
    def MatrixElement(self, i, j):
        a = C.c_double()
        self._check(N.lib().kemcu_matrix_element(self._h, i, j, C.byref(a)))
        return a.value

    def Multiply(self, x, precision=FP64, assembled=False):
        x = np.ascontiguousarray(x, np.float64)
        nr = 1 if x.ndim == 1 else x.shape[0]
        y = np.zeros_like(x)
        self._check(N.lib().kemcu_matvec(self._h, _d(x), _d(y), nr, precision, int(bool(assembled))))
        return y

    # -- solve
    def SetIterationCallback(self, fn):
        """fn(iteration, rel_residual_estimate) -> bool (True stops the solve)."""
        if fn is None:
            self._cb = None
            N.lib().kemcu_set_iteration_callback(self._h, N.ITER_CB(), None)
            return
        self._cb = N.ITER_CB(lambda user, it, r: int(bool(fn(it, r))))
        N.lib().kemcu_set_iteration_callback(self._h, self._cb, None)

    def Solve(self, b=None, tol=1e-10, max_iter=500, mode=SOLVE_PLAIN, raise_on_failure=True):
        """GMRES charge-density solve; returns (x, stats dict). b: None (boundary values),
        [n] or [n_rhs, n]."""
        if b is None:
            x = np.zeros(self.n)
            bp, nr = None, 1
        else:
            bb = np.ascontiguousarray(b, np.float64)
            nr = 1 if bb.ndim == 1 else bb.shape[0]
            x = np.zeros_like(bb)
            bp = _d(bb)
        st = N.SolveStats()
        rc = N.lib().kemcu_gmres(self._h, bp, _d(x), nr, tol, max_iter, mode, C.byref(st))
        stats = {k: getattr(st, k) for k, _ in N.SolveStats._fields_}
        stats["status"] = rc
        if rc != N.OK and raise_on_failure:
            self._check(rc)
        return x, stats

    def KrylovSolve(self, b=None, solver="gmres", mode=SOLVE_PLAIN, tol=1e-8, max_iter=500, restart=0,
                    preconditioner="none", preconditioner_mode=SOLVE_FFTM, preconditioner_tol=0.01,
                    max_preconditioner_iter=30, raise_on_failure=True):
        """Krylov charge-density solve with the reference's solver and preconditioner choices
        (KKrylovSolverFactory, KFMElectrostaticFastMultipoleBoundaryValueSolver): solver "gmres" or
        "bicgstab"; mode: the system's operator (SOLVE_PLAIN, SOLVE_ASSEMBLED_FP64, SOLVE_FFTM);
        restart: iterations between restarts (0 = never); preconditioner "none", "jacobi" or
        "implicit_krylov" (an inner GMRES on preconditioner_mode's operator, SOLVE_FFTM = the tree of
        ConfigureFFTMPreconditioner). Returns (x, stats dict); b as for Solve."""
        solvers = {"gmres": N.KRYLOV_GMRES, "bicgstab": N.KRYLOV_BICGSTAB}
        precons = {"none": N.PRECON_NONE, "jacobi": N.PRECON_JACOBI, "implicit_krylov": N.PRECON_IMPLICIT_KRYLOV}
        if solver not in solvers or preconditioner not in precons:
            raise ValueError(f"solver must be one of {sorted(solvers)} and preconditioner one of {sorted(precons)}")
        prm = N.KrylovParams()
        N.lib().kemcu_krylov_default_params(C.byref(prm))
        prm.solver, prm.mode, prm.tolerance, prm.max_iterations = solvers[solver], mode, tol, max_iter
        prm.iterations_between_restarts, prm.preconditioner = restart, precons[preconditioner]
        prm.preconditioner_mode, prm.preconditioner_tolerance = preconditioner_mode, preconditioner_tol
        prm.max_preconditioner_iterations = max_preconditioner_iter
        if b is None:
            x = np.zeros(self.n)
            bp, nr = None, 1
        else:
            bb = np.ascontiguousarray(b, np.float64)
            nr = 1 if bb.ndim == 1 else bb.shape[0]
            x = np.zeros_like(bb)
            bp = _d(bb)
        st = N.SolveStats()
        rc = N.lib().kemcu_krylov_solve(self._h, bp, _d(x), nr, C.byref(prm), C.byref(st))
        stats = {k: getattr(st, k) for k, _ in N.SolveStats._fields_}
        stats["status"] = rc
        if rc != N.OK and raise_on_failure:
            self._check(rc)
        return x, stats

    def SolveRobinHood(self, b=None, tol=1e-8, x0=None, check_interval=0, max_subiterations=0, assembled=False,
                       raise_on_failure=True):
        """Robin Hood charge-density solve (KRobinHood<double>::Solve); returns (x, stats dict).
        b: None (boundary values) or [n]; x0: initial guess (zeros by default)."""
        x = np.zeros(self.n) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        bp = None if b is None else _d(np.ascontiguousarray(b, np.float64))
        st = N.RhStats()
        rc = N.lib().kemcu_robin_hood(self._h, bp, _d(x), tol, check_interval, max_subiterations, int(bool(assembled)),
                                      C.byref(st))
        stats = {k: getattr(st, k) for k, _ in N.RhStats._fields_}
        stats["status"] = rc
        if rc != N.OK and raise_on_failure:
            self._check(rc)
        return x, stats

    # -- tracking
    def TrackRK8(self, state, dt, max_steps, steps=None, status=None, step_budget=0, charge=None, mass=None,
                 sphere_radius=0.0, max_radius=0.0, precision=FP64, momentum_change=None):
        """Advance the tracks; returns (state, steps, status, stats dict). momentum_change: an [n]
        array that receives, added to its values, each track's sum of |p_after - p_before| per step."""
        from .geometry import ELECTRON_MASS, ELEMENTARY_CHARGE
        st = np.ascontiguousarray(state, np.float64).copy()
        n = st.shape[0]
        steps = np.zeros(n, np.int32) if steps is None else np.ascontiguousarray(steps, np.int32).copy()
        status = np.zeros(n, np.int32) if status is None else np.ascontiguousarray(status, np.int32).copy()
        hit = N.HitModel(sphere_radius, max_radius)
        ts = N.TrackStats()
        q = -ELEMENTARY_CHARGE if charge is None else charge
        m = ELECTRON_MASS if mass is None else mass
        dpp = C.cast(None, C.POINTER(C.c_double))
        if momentum_change is not None:
            assert momentum_change.dtype == np.float64 and momentum_change.shape == (n,)
            assert momentum_change.flags.c_contiguous
            dpp = _d(momentum_change)
        self._check(N.lib().kemcu_track_rk8(self._h, _d(st), _i(steps), _i(status), n, dt, max_steps, step_budget, q, m,
                                            C.byref(hit), precision, C.byref(ts), dpp))
        return st, steps, status, {k: getattr(ts, k) for k, _ in N.TrackStats._fields_}

    # -- fast multipole method (KFMElectrostaticFastMultipoleFieldSolver)
    def ConfigureFFTM(self, **params):
        """Builds the fast-multipole tree for the current geometry. Keyword arguments are the
        fields of kemcu_fftm_params (degree, top_level_divisions, divisions, zeromask,
        maximum_tree_depth, insertion_ratio, region_expansion_factor, world_center,
        world_length, near_analytic); the others keep their defaults."""
        self._check(N.lib().kemcu_fftm_configure(self._h, C.byref(self._fftm_params(params))))

    def ConfigureFFTMPreconditioner(self, **params):
        """Builds the tree whose operator the implicit Krylov preconditioner inverts
        (KrylovSolve with preconditioner_mode=SOLVE_FFTM); keyword arguments as ConfigureFFTM."""
        self._check(N.lib().kemcu_fftm_configure_preconditioner(self._h, C.byref(self._fftm_params(params))))

    @staticmethod
    def _fftm_params(params):
        prm = N.FftmParams()
        N.lib().kemcu_fftm_default_params(C.byref(prm))
        for k, v in params.items():
            if k == "world_center":
                for i in range(3):
                    prm.world_center[i] = float(v[i])
            elif k in ("insertion_ratio", "region_expansion_factor", "world_length"):
                setattr(prm, k, float(v))
            else:
                setattr(prm, k, int(v))
        return prm

    def FFTMField(self, P, what=FIELD_AND_POTENTIAL):
        """n x 4 (Ex, Ey, Ez, phi) by the fast multipole method."""
        P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
        out = np.zeros((P.shape[0], 4))
        self._check(N.lib().kemcu_fftm_field(self._h, _d(P), P.shape[0], _d(out), what))
        return out

    def FFTMMultiply(self, x):
        """A x by the fast multipole operator (x: n, or n_rhs x n)."""
        x = np.ascontiguousarray(x, np.float64)
        nr = 1 if x.ndim == 1 else x.shape[0]
        y = np.zeros_like(x)
        self._check(N.lib().kemcu_fftm_matvec(self._h, _d(x), _d(y), nr))
        return y

    def FFTMFieldDevice(self, d_points_ptr: int, n: int, d_out_ptr: int, what=FIELD_AND_POTENTIAL):
        self._check(N.lib().kemcu_fftm_field_dev(self._h, C.c_void_p(d_points_ptr), n, C.c_void_p(d_out_ptr), what))

    def FFTMInfo(self, depth: int) -> dict:
        world = np.zeros(4)
        counts = np.zeros(depth + 2, np.int32)
        self._check(N.lib().kemcu_fftm_info(self._h, _d(world), _i(counts)))
        return {"world_center": world[:3].copy(), "world_length": float(world[3]), "occupied_cells": int(counts[0]),
                "owned_per_level": counts[1:].tolist()}

    def MultipoleMoments(self, degree: int, origins):
        """n x (degree+1)^2 complex moments of every element (unit total charge) about origins."""
        o = np.ascontiguousarray(origins, np.float64).reshape(-1, 3)
        S = (degree + 1) ** 2
        out = np.zeros(2 * o.shape[0] * S)
        self._check(N.lib().kemcu_fm_moments(self._h, degree, _d(o), _d(out)))
        return (out[0::2] + 1j * out[1::2]).reshape(o.shape[0], S)

    def LocalExpansionField(self, degree: int, origin, coeff, P):
        """(Ex, Ey, Ez, phi) of a local expansion (m >= 0 coefficients, index l(l+1)/2+m) at P."""
        c = np.zeros(2 * len(coeff))
        c[0::2] = np.real(coeff)
        c[1::2] = np.imag(coeff)
        P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
        out = np.zeros((P.shape[0], 4))
        o = np.ascontiguousarray(origin, np.float64)
        self._check(N.lib().kemcu_fm_local_field(self._h, degree, _d(o), _d(c), P.shape[0], _d(P), _d(out)))
        return out

    @staticmethod
    def MultipoleResponse(kind: int, degree: int, source_origin, target_origin):
        """[target, source] complex translation response (0 M2M, 1 M2L, 2 L2L), host arithmetic."""
        S = (degree + 1) ** 2
        out = np.zeros(2 * S * S)
        so = np.ascontiguousarray(source_origin, np.float64)
        to = np.ascontiguousarray(target_origin, np.float64)
        rc = N.lib().kemcu_fm_response(kind, degree, _d(so), _d(to), _d(out))
        if rc:
            raise N.KemcuError(rc, "kemcu_fm_response")
        return (out[0::2] + 1j * out[1::2]).reshape(S, S)

    # -- adjoint
    def FieldVJP(self, P, w, precision=FP64, want_sigma=True, want_vertices=True):
        """Adjoint of the direct sum: (dL/dsigma [N], dL/dvertices [N, 9]) for L = sum_p w_p . out_p."""
        P = np.ascontiguousarray(P, np.float64).reshape(-1, 3)
        w = np.ascontiguousarray(w, np.float64).reshape(-1, 4)
        ds = np.zeros(self.n) if want_sigma else None
        dv = np.zeros((self.n, 9)) if want_vertices else None
        null = C.cast(None, C.POINTER(C.c_double))
        self._check(N.lib().kemcu_field_vjp(self._h, _d(P), P.shape[0], _d(w), _d(ds) if ds is not None else null,
                                            _d(dv) if dv is not None else null, precision))
        return ds, dv
