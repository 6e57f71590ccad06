"""Loading helpers for the golden fixtures in tests/golden (written by make_golden.py)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

BND_KEYS = ("zetaClosedOrGradientBCIdx1", "zetaClosedOrGradientBCIdx2", "zetaClampedBCIdx1",
            "ubarClosedBCIdx1", "vbarClosedBCIdx1", "ubarClampedBCIdx1", "vbarClampedBCIdx1",
            "ubarGradientBCIdx1", "ubarGradientBCIdx2", "vbarGradientBCIdx1", "vbarGradientBCIdx2")


def load(name):
    return np.load(os.path.join(GOLDEN, name))


def boundary_dict(d, prefix):
    out = {}
    for k in d.files:
        if k.startswith(prefix):
            out[k[len(prefix):]] = d[k]
    return out
