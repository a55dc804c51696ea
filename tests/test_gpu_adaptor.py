"""The C++ KEMField adaptors (include/kemfield_cuda.hh) on a real device: the reference's own
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
