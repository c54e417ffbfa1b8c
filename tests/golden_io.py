"""Readers for the committed golden fixtures (tests/golden)."""
import json
import os

import numpy as np

from rforest_b200.packed import Packed

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def digests():
    with open(os.path.join(GOLDEN, "digests.json")) as f:
        return json.load(f)


def _packed(z, tag):
    return Packed(z[f"{tag}_limbs"].astype(np.uint64), z[f"{tag}_offs"].astype(np.int64),
                  z[f"{tag}_sizes"].astype(np.int32))


def edge_cases():
    """[(m, k, n, A, B, C_expected)] from the reference's own CPU path."""
    z = np.load(os.path.join(GOLDEN, "edge_cases.npz"))
    out = []
    for ci, (m, k, n) in enumerate(z["shapes"]):
        out.append((int(m), int(k), int(n), _packed(z, f"e{ci}_A"), _packed(z, f"e{ci}_B"),
                    _packed(z, f"e{ci}_C")))
    return out


def config1():
    z = np.load(os.path.join(GOLDEN, "config1.npz"))
    return _packed(z, "A"), _packed(z, "B"), _packed(z, "C")
