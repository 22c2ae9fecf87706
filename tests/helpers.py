"""Shared helpers of the test suite."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def unpack_mask(packed, shape):
    n = int(np.prod(shape))
    return np.unpackbits(packed)[:n].reshape(tuple(int(s) for s in shape)).astype(np.uint8)


def load_golden(name):
    path = os.path.join(GOLDEN, name)
    z = np.load(path, allow_pickle=False)
    d = {k: z[k] for k in z.files}
    d["mask"] = unpack_mask(d["mask"], d["shape"])
    return d


def spheres(shape, phi, r, seed):
    from lbm_b200 import geometry as G

    return G.overlapping_spheres(shape, phi, r, seed)
