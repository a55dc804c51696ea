"""Loader for the committed golden fixtures in tests/golden/ (test infrastructure).

The fixtures were produced by tests/golden/make_golden.py from the reference's own FP64 CPU
code (oracle/_ref/libkemref.so) and travel with the repository, so GPU parity tests and
smoke() need neither the reference tree nor the oracle build on the GPU host.
"""

from __future__ import annotations

import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")


def path(name: str) -> str:
    return os.path.join(GOLDEN_DIR, name + ".npz")


def load(name: str) -> dict:
    with np.load(path(name), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def mesh_from(fx: dict, prefix: str = ""):
    from kassiopeia_b200.geometry import Mesh

    return Mesh(fx[prefix + "shape"].astype(np.int32), fx[prefix + "boundary"].astype(np.int32),
                fx[prefix + "geom"].astype(np.float64), fx[prefix + "value"].astype(np.float64))
