"""Loaders for the committed golden fixtures (see tests/golden/make_golden.py)."""
import json
import os

import numpy as np

from macis_b200.integrals import fcidump_fill

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def water():
    """Water cc-pVDZ integrals of the reference tests: (norb, T, V, E_core)."""
    z = np.load(os.path.join(GOLDEN, "h2o_ccpvdz_fcidump.npz"))
    T, V, ecore = fcidump_fill(z["idx"], z["val"])
    norb = int(round(len(T) ** 0.5))
    return norb, T, V, ecore


def water_cisd_rowptr():
    return np.load(os.path.join(GOLDEN, "h2o_ccpvdz_cisd_rowptr.npz"))["rowptr"]


def constants():
    with open(os.path.join(GOLDEN, "reference_constants.json")) as f:
        return {k: v[0] for k, v in json.load(f).items()}
