"""Failure detection on the device without a fault: a bounded mbarrier wait that nothing
completes gives up, the host reads KEMCU_ETIMEOUT from the flag word, and the context keeps
working (kemcu_selftest_timeout; the element pipeline of the direct-sum kernels uses the same
wait and flag)."""

import numpy as np
import pytest

import kassiopeia_b200 as K
from kassiopeia_b200 import _native as N
from kassiopeia_b200 import geometry as G

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives():
    with K.CUDAElectrostaticContext(0) as ctx:
        assert N.lib().kemcu_selftest_timeout(ctx._h, 1) == N.OK
        assert N.lib().kemcu_selftest_timeout(ctx._h, 0) == N.ETIMEOUT
        assert b"timed out" in N.lib().kemcu_last_error(ctx._h)
        # the next calls run normally
        assert N.lib().kemcu_selftest_timeout(ctx._h, 1) == N.OK
        m = G.icosphere(2)
        ctx.SetGeometry(m)
        ctx.SetSigma(np.full(m.n, 1e-11))
        out = ctx.ElectricFieldAndPotential(G.shell_points(100))
        assert np.all(np.isfinite(out))
