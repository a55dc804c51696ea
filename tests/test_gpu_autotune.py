"""The autotuner of the direct-sum kernel's launch shape: every shape computes the same
operations in the same order, so exploring them never changes a result bit; the explicit tuner
times every shape and records its choice for the size class."""

import ctypes as C

import numpy as np
import pytest

import kassiopeia_b200 as K
from kassiopeia_b200 import _native as N
from kassiopeia_b200 import geometry as G

pytestmark = pytest.mark.gpu


def test_exploration_keeps_every_bit_and_chooses():
    import torch

    m = G.coax(n_phi=40, n_z=40, n_cap_rings=4)
    with K.CUDAElectrostaticContext(0, autotune=True) as ctx:
        ctx.SetGeometry(m)
        ctx.SetSigma(G.coax_density(m))
        n = 20000
        P = torch.from_numpy(G.gap_points(n, seed=8)).cuda()
        outs = []
        nv = N.lib().kemcu_field_variant_count()
        assert nv >= 2
        assert ctx.FieldVariant(n, K.MIXED) == -1
        for _ in range(nv):  # one shape per call until every shape has run
            o = torch.empty((n, 4), dtype=torch.float64, device="cuda")
            ctx.FieldDevice(P.data_ptr(), n, o.data_ptr(), precision=K.MIXED)
            outs.append(o.cpu().numpy())
        for o in outs[1:]:
            np.testing.assert_array_equal(o, outs[0])
        v = ctx.FieldVariant(n, K.MIXED)
        assert 0 <= v < nv
        info = ctx.FieldVariantInfo(v)
        assert info["ctas_per_sm"] in (4, 5, 6) and info["ring_stages"] in (3, 4)
        # another size class has its own choice; the other precision too
        assert ctx.FieldVariant(2 * n, K.MIXED) == -1 and ctx.FieldVariant(n, K.FP64) == -1
        # the chosen shape gives the same bits again
        o = torch.empty((n, 4), dtype=torch.float64, device="cuda")
        ctx.FieldDevice(P.data_ptr(), n, o.data_ptr(), precision=K.MIXED)
        np.testing.assert_array_equal(o.cpu().numpy(), outs[0])


def test_explicit_tuning_times_every_shape():
    import torch

    m = G.icosphere(4)
    with K.CUDAElectrostaticContext(0, autotune=False) as ctx:
        ctx.SetGeometry(m)
        ctx.SetSigma(G.sphere_density(m))
        n = 30000
        P = torch.from_numpy(G.shell_points(n, seed=9)).cuda()
        ref = torch.empty((n, 4), dtype=torch.float64, device="cuda")
        ctx.FieldDevice(P.data_ptr(), n, ref.data_ptr(), precision=K.FP64)
        assert ctx.FieldVariant(n, K.FP64) == -1  # autotune off: nothing explored
        out = torch.empty_like(ref)
        v, ms = ctx.TuneField(P.data_ptr(), n, out.data_ptr(), precision=K.FP64)
        assert len(ms) == N.lib().kemcu_field_variant_count() and all(t > 0 for t in ms)
        assert v == int(np.argmin(ms)) and ctx.FieldVariant(n, K.FP64) == v
        np.testing.assert_array_equal(out.cpu().numpy(), ref.cpu().numpy())
