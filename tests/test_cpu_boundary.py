"""CPU-only checks of the drop-in boundary: the C-ABI library loads, exports every symbol the
header declares, reports a missing device as an error (no fallback), and its cubature tables
equal the reference's rules node for node."""

import ctypes as C
import subprocess

import numpy as np
import pytest

from kassiopeia_b200 import _native as N
from oracle import golden


def test_library_exports_every_header_symbol():
    L = N.lib()
    syms = N.header_symbols()
    assert len(syms) >= 18
    for s in syms:
        assert hasattr(L, s), f"{s} declared in include/kemcu.h but not exported"
    out = subprocess.run(["nm", "-D", "--defined-only", N.LIB_PATH], capture_output=True, text=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(syms) <= exported


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_is_an_error_not_a_fallback():
    import kassiopeia_b200 as K

    with pytest.raises(K.KemcuError) as e:
        K.CUDAElectrostaticContext(0)
    assert e.value.code == N.ECUDA
    assert "device" in str(e.value)


def _rule(which):
    out = np.zeros((33, 3))
    n = N.lib().kemcu_rule_nodes(which, out.ctypes.data_as(C.POINTER(C.c_double)))
    assert n > 0
    return out[:n]


@pytest.mark.parametrize("which,name", list(enumerate(["tri7", "tri12", "tri33", "rect7", "rect12", "rect33"])))
def test_cubature_tables_match_reference_rules(which, name):
    ref = golden.load("rules")[name]
    mine = _rule(which)
    assert mine.shape == ref.shape
    # same nodes in the same order, same weights (restated tables, bit-level agreement)
    np.testing.assert_allclose(mine[:, :2], ref[:, :2], rtol=0, atol=4e-16)
    np.testing.assert_allclose(mine[:, 2], ref[:, 2], rtol=2e-16, atol=0)
    assert abs(mine[:, 2].sum() - 1.0) < 1e-14


def test_gauss_legendre_rules():
    # the reference tabulates 4-node abscissae to 15 digits and 16-node ones to 17
    # (KElectrostaticQuadratureLineSegmentIntegrator.hh:47-80); ours are computed exactly
    x4 = _rule(6)
    np.testing.assert_allclose(x4[:, 0], [0.339981043584856, 0.861136311594053], atol=1e-15)
    np.testing.assert_allclose(x4[:, 1], [0.652145154862546, 0.347854845137454], atol=1e-15)
    x16 = _rule(7)
    np.testing.assert_allclose(x16[:, 0], [0.09501250983763744, 0.28160355077925891, 0.45801677765722739,
                                           0.61787624440264375, 0.75540440835500303, 0.86563120238783174,
                                           0.94457502307323258, 0.98940093499164993], atol=2e-16)
    assert abs(2 * x16[:, 1].sum() - 2.0) < 1e-14


def test_invalid_rule_index():
    out = np.zeros((33, 3))
    assert N.lib().kemcu_rule_nodes(8, out.ctypes.data_as(C.POINTER(C.c_double))) == N.EINVAL


def test_kemfield_adaptor_builds_against_reference():
    """include/kemfield_cuda.hh compiles against the reference's unchanged KEMField headers and
    links with the reference's objects and libkemcu (the drop-in the integration notes describe)."""
    import os

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if not os.path.isdir(os.path.join(root, "oracle", "_ref", "obj")):
        pytest.skip("the reference's objects were not built here (make -C oracle ref)")
    r = subprocess.run(["make", "-s", "-C", os.path.join(root, "oracle"), "adaptor"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert os.path.exists(os.path.join(root, "oracle", "_ref", "adaptor_check"))


def test_xml_bindings_parse_without_a_device():
    # the XML half of tests/cxx/bindings_check.cc: the reference's Kommon tokenizer reads a
    # configuration with the CUDA elements and the use_cuda switch, and every setting arrives
    import os

    binary = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                          "bindings_check")
    if not os.path.exists(binary):
        pytest.skip("bindings check not built (needs the reference tree)")
    r = subprocess.run([binary, "--parse-only"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "parsed 6 field elements" in r.stdout and "settings from the XML: as written" in r.stdout
    assert "Krylov solver and preconditioner settings from the XML: as written" in r.stdout
