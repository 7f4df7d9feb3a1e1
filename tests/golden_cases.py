"""Loading of the golden fixtures made by tests/golden/make_golden.py from the
reference's own CUDA step, and the relative-error measure the tests use."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cases():
    out = {}
    for f in sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))):
        d = dict(np.load(f))
        d = {k: (v.item() if v.ndim == 0 else v) for k, v in d.items()}
        if "flavour" not in d:  # not a step fixture (e.g. the UPO orbits)
            continue
        out[os.path.basename(f)[:-4]] = d
    return out


def relerr(a, b):
    """max |a - b| / max |b| over the whole array"""
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
