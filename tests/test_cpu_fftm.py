"""CPU checks of the fast-multipole pieces: the numpy restatement (oracle/fm_port.py) against the
reference's own moments, local-expansion field and response functions (tests/golden/fftm.npz,
from oracle/_ref/libkemref_fm.so), and the library's host-side translation operators
(kemcu_fm_response, no device) against the same fixture and, where it is built, the live
reference. The device kernels are checked in test_gpu_fftm.py."""

import numpy as np
import pytest

import kassiopeia_b200 as K
from oracle import fm_port, golden, ref, ref_fm
from oracle.golden import mesh_from

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


def test_port_moments_equal_reference_fixture():
    # the reference's analytic moments (triangles, rectangles, wires) are the element averages of
    # conj(R_n^m): an exact cubature reproduces them to rounding
    fx = golden.load("fftm")
    m = mesh_from(golden.load("mixed_small"))
    for v, o, want in zip(_vertices(m), fx["mixed_origins"], fx["mixed_moments"]):
        got = fm_port.moments(v, o, 10)
        assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_port_local_field_equals_reference_fixture():
    fx = golden.load("fftm")
    k = 8.9875517873681764e9 if not ref.available() else ref.constant("one_over_four_pi_eps0")
    got = fm_port.local_field(int(fx["l2p_degree"]), fx["l2p_origin"], fx["l2p_coeff"], fx["l2p_points"][:20], k)
    want = fx["l2p"][:20]
    scale = np.abs(want).max(axis=0)
    assert np.all(np.abs(got[:, 3] - want[:, 3]) <= 1e-13 * scale[3])
    assert np.all(np.abs(got[:, :3] - want[:, :3]) <= 1e-7 * scale[:3])  # central differences


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_host_response_equals_reference_fixture(kind):
    fx = golden.load("fftm")
    tgt = fx["resp_far"] if kind == 1 else fx["resp_tgt"]
    want = fx["resp"][kind]
    got = K.CUDAElectrostaticContext.MultipoleResponse(kind, 6, fx["resp_src"], tgt)
    assert np.abs(got - want).max() <= 1e-14 * np.abs(want).max()
    port = fm_port.response(kind, 6, fx["resp_src"], tgt)
    assert np.abs(port - want).max() <= 1e-14 * np.abs(want).max()


@needs_ref_fm
@pytest.mark.parametrize("kind,degree", [(0, 3), (0, 12), (1, 4), (1, 12), (2, 5), (2, 12)])
def test_host_response_equals_live_reference(kind, degree):
    rng = np.random.default_rng(7 + kind * 31 + degree)
    src = rng.uniform(-1, 1, 3)
    tgt = src + (rng.uniform(2, 3, 3) * rng.choice([-1, 1], 3) if kind == 1 else rng.uniform(-0.5, 0.5, 3))
    want = ref_fm.response(kind, degree, src, tgt)
    got = K.CUDAElectrostaticContext.MultipoleResponse(kind, degree, src, tgt)
    assert np.abs(got - want).max() <= 1e-13 * np.abs(want).max()


def test_fftm_parameters_rejected_on_cpu_paths():
    # parameter checks need no device: an unsupported division ratio is refused by the default
    # parameters' validation in Python before any call
    prm = K._native.FftmParams()
    K._native.lib().kemcu_fftm_default_params(K._native.C.byref(prm))
    assert (prm.degree, prm.top_level_divisions, prm.divisions, prm.zeromask) == (8, 2, 2, 1)
    assert abs(prm.insertion_ratio - 4.0 / 3.0) < 1e-15 and prm.near_analytic == 1


def test_krylov_defaults_and_host_side_errors():
    # kemcu_krylov_default_params and the argument checks before any device work (no GPU): the
    # documented defaults (gmres on the FP64 matrix-free operator, 1e-8, 500 iterations, no restart,
    # no preconditioner; implicit Krylov on the preconditioner's tree to 0.01 in 30 iterations),
    # and a null context refused with KEMCU_EINVAL
    from kassiopeia_b200 import _native as N
    L = N.lib()
    p = N.KrylovParams()
    L.kemcu_krylov_default_params(p)
    assert (p.solver, p.mode, p.tolerance, p.max_iterations, p.iterations_between_restarts) == \
        (N.KRYLOV_GMRES, K.SOLVE_PLAIN, 1e-8, 500, 0)
    assert (p.preconditioner, p.preconditioner_mode, p.preconditioner_tolerance, p.max_preconditioner_iterations) == \
        (N.PRECON_NONE, K.SOLVE_FFTM, 0.01, 30)
    x = np.zeros(4)
    assert L.kemcu_krylov_solve(None, None, x.ctypes.data_as(N._dp), 1, p, None) == N.EINVAL
    fp = N.FftmParams()
    L.kemcu_fftm_default_params(fp)
    assert L.kemcu_fftm_configure_preconditioner(None, fp) == N.EINVAL
