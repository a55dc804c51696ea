"""The C++ KEMField adaptors (include/kemfield_cuda.hh, kemfield_cuda_fftm.hh, kassiopeia_cuda.hh,
kemfield_cuda_bindings.hh) on a real device: the reference's own
KSurfaceContainer is solved on the GPU, and the reference CPU field solver, matrix and GMRES
driver are compared with the CUDA adaptors (tests/cxx/adaptor_check.cc, built by
`make -C oracle adaptor` where the reference tree exists)."""

import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "adaptor_check")


@pytest.mark.skipif(not os.path.exists(BIN), reason="adaptor check not built (needs the reference tree)")
def test_kemfield_adaptors_against_reference_classes():
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout


BATCH = os.path.join(ROOT, "oracle", "_ref", "batch_driver_check")


@pytest.mark.skipif(not os.path.exists(BATCH), reason="batch driver check not built (needs the reference tree)")
def test_kassiopeia_batch_driver_against_reference_rk8():
    # include/kassiopeia_cuda.hh: Kassiopeia KSParticles tracked as one batch on the GPU fill
    # KSTrack objects that match the reference's KSMathRK8 driven by the reference field solver
    # (tests/cxx/batch_driver_check.cc, built by `make -C oracle batch`)
    r = subprocess.run([BATCH], capture_output=True, text=True, timeout=900)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout


XML = os.path.join(ROOT, "oracle", "_ref", "bindings_check")


@pytest.mark.skipif(not os.path.exists(XML), reason="bindings check not built (needs the reference tree)")
def test_xml_bindings_configure_the_gpu_solvers():
    # include/kemfield_cuda_bindings.hh: a KEMField-style XML file parsed by the reference's own
    # Kommon tokenizer configures the CUDA solvers (and the use_cuda switch) of boundary fields
    # whose fields then match the reference CPU field solver (tests/cxx/bindings_check.cc)
    r = subprocess.run([XML], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout


FFTM = os.path.join(ROOT, "oracle", "_ref", "fftm_check")


@pytest.mark.skipif(not os.path.exists(FFTM), reason="FFTM check not built (needs the reference tree)")
def test_fast_multipole_drop_ins_against_reference_classes():
    # include/kemfield_cuda_fftm.hh: the reference's KKrylovChargeDensitySolver solving with
    # KCUDAFastMultipoleMatrixGenerator against it solving with its own
    # KFastMultipoleMatrixGenerator, the device FFTM solve, and KCUDAFastMultipoleFieldSolver
    # against KElectricFastMultipoleFieldSolver (tests/cxx/fftm_check.cc)
    r = subprocess.run([FFTM], capture_output=True, text=True, timeout=900)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK" in r.stdout
