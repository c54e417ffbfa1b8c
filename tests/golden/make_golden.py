"""Generate the committed golden fixtures from the reference itself.

Run here, where the reference tree exists (it builds oracle/_ref from the
reference's own CPU sources):

    python tests/golden/make_golden.py [small] [config3] [config4] [config5]

Every expected output below is produced by the reference's unmodified CPU
mpz_rmatrix_mult_fft (alexp616/rforest src/lib/hwmpz.c:65-130) through
oracle/_ref, and cross-checked against GMP schoolbook (and, for the small
cases, Python integers) before it is written.  Inputs are not stored for the
seeded workloads: the generator in rforest_b200/workloads.py rebuilds them,
and a digest of the generated inputs pins the generator itself.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from rforest_b200 import packed as PK  # noqa: E402
from rforest_b200 import workloads as W  # noqa: E402

DIGESTS = os.path.join(HERE, "digests.json")


def load_digests():
    if os.path.exists(DIGESTS):
        with open(DIGESTS) as f:
            return json.load(f)
    return {}


def save_digests(d):
    with open(DIGESTS, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
        f.write("\n")


def ref_product(m, k, n, A, B, check_schoolbook=True):
    C = O.matmul_reference(m, k, n, A, B)
    if check_schoolbook:
        S = O.matmul_schoolbook(m, k, n, A, B)
        assert PK.digest(C) == PK.digest(S), "reference and schoolbook disagree"
    return C


def edge_cases():
    """Small hand-built products covering the reference's edge cases."""
    big = (1 << 4096) - 1
    cases = []
    # 1. all-zero operands
    cases.append((3, 3, 3, [0] * 9, [0] * 9))
    # 2. +-1 entries against a dense matrix (identity-like)
    cases.append((2, 3, 3, [1, 0, 0, 0, -1, 0], [big, -big, 7, 1 << 700, -(1 << 64), 0, 5, 6, -7]))
    # 3. all-ones limbs: long carry / borrow chains
    cases.append((2, 2, 2, [big, -big, big, big], [big, big, -big, big]))
    cases.append((1, 2, 1, [(1 << 8192) - 1, 1], [(1 << 8192) - 1, -(1 << 16384) + 1]))
    # 4. mixed sizes in one product: one huge entry, the rest one limb
    cases.append((2, 2, 3, [(3 << 16000) + 12345, -3, 2, 1], [-1, 2, 3, 4, (1 << 63), -(1 << 64)]))
    # 5. the reference's own r x d by d x d shape with r != d
    cases.append((1, 5, 5, [1 << (64 * i + 3) for i in range(5)],
                  [((-1) ** i) * ((1 << (100 * i + 17)) + i) for i in range(25)]))
    # 6. general m x k x n with k != n
    cases.append((3, 5, 2, [((-1) ** i) * (i + 1) << (97 * i) for i in range(15)],
                  [(1 << (211 * i + 1)) - 3 for i in range(10)]))
    # 7. exact cancellation: nonzero operands, zero result
    x, y = (1 << 5000) + 99, (1 << 3000) - 7
    cases.append((1, 2, 1, [x, x], [y, -y]))
    # 8. power-of-two results and single-limb boundaries
    cases.append((2, 2, 2, [1 << 63, 1 << 64, -(1 << 127), 1], [1 << 1, 1 << 0, 1, -(1 << 191)]))
    # 9. 1x1x1 with large operands (lgN well above the small cases)
    cases.append((1, 1, 1, [(1 << 131072) - 12345], [-((1 << 130000) + 999)]))
    # 10. k = 1 outer product
    cases.append((3, 1, 4, [5, -(1 << 300), 0], [1, -1, (1 << 1000) + 1, 3]))
    return cases


def make_small():
    rng_cases = edge_cases()
    arrays = {}
    meta = []
    for ci, (m, k, n, Ai, Bi) in enumerate(rng_cases):
        A, B = PK.from_ints(Ai), PK.from_ints(Bi)
        C = ref_product(m, k, n, A, B)
        assert C.to_ints() == O.matmul_python(m, k, n, Ai, Bi)
        Cc = C.compact()
        for tag, P in (("A", A), ("B", B), ("C", Cc)):
            arrays[f"e{ci}_{tag}_limbs"] = P.limbs
            arrays[f"e{ci}_{tag}_offs"] = P.offs
            arrays[f"e{ci}_{tag}_sizes"] = P.sizes
        meta.append([m, k, n])
    arrays["shapes"] = np.array(meta, dtype=np.int64)
    np.savez_compressed(os.path.join(HERE, "edge_cases.npz"), **arrays)

    # config 1: full vectors
    p = W.config1()
    C = ref_product(p.m, p.k, p.n, p.A, p.B).compact()
    assert C.to_ints() == O.matmul_python(p.m, p.k, p.n, p.A.to_ints(), p.B.to_ints())
    np.savez_compressed(os.path.join(HERE, "config1.npz"),
                        A_limbs=p.A.limbs, A_offs=p.A.offs, A_sizes=p.A.sizes,
                        B_limbs=p.B.limbs, B_offs=p.B.offs, B_sizes=p.B.sizes,
                        C_limbs=C.limbs, C_offs=C.offs, C_sizes=C.sizes)
    d = load_digests()
    d["config1"] = {"A": PK.digest(p.A), "B": PK.digest(p.B), "C": PK.digest(C)}

    # config 2: single product and the 16-matrix chain
    p = W.config2()
    t = time.time()
    C = ref_product(p.m, p.k, p.n, p.A, p.B)
    d["config2"] = {"A": PK.digest(p.A), "B": PK.digest(p.B), "C": PK.digest(C),
                    "ref_seconds": round(time.time() - t, 4)}
    mats = W.config2_chain()
    M = mats[0]
    t = time.time()
    steps = []
    for i in range(1, len(mats)):
        M = ref_product(8, 8, 8, M, mats[i], check_schoolbook=False).compact()
        steps.append(PK.digest(M))
    d["config2_chain"] = {"inputs": [PK.digest(x) for x in mats], "steps": steps,
                          "final": steps[-1], "ref_seconds": round(time.time() - t, 3)}
    save_digests(d)


def make_config3(count=4096):
    d = load_digests()
    shapes, digs = [], []
    t = time.time()
    for i in range(count):
        p = W.random_product(3001, i, 2, 16, 10, 18)
        C = ref_product(p.m, p.k, p.n, p.A, p.B, check_schoolbook=(i < 64))
        shapes.append([p.m, p.k, p.n, p.bits])
        digs.append(PK.digest(C))
    d["config3"] = {"count": count, "shapes": shapes, "C": digs,
                    "ref_seconds": round(time.time() - t, 2)}
    save_digests(d)


def make_config4():
    d = load_digests()
    p = W.config4()
    t = time.time()
    C = ref_product(p.m, p.k, p.n, p.A, p.B, check_schoolbook=False)
    d["config4"] = {"A": PK.digest(p.A), "B": PK.digest(p.B), "C": PK.digest(C),
                    "ref_seconds": round(time.time() - t, 2)}
    save_digests(d)


def make_config5(count=256):
    d = load_digests()
    shapes, digs = [], []
    t = time.time()
    for i in range(count):
        p = W.config5_request(1, i)
        C = ref_product(p.m, p.k, p.n, p.A, p.B, check_schoolbook=False)
        shapes.append([p.m, p.k, p.n, p.bits])
        digs.append(PK.digest(C))
    d["config5"] = {"count": count, "shapes": shapes, "C": digs,
                    "ref_seconds": round(time.time() - t, 2)}
    save_digests(d)


if __name__ == "__main__":
    O.build()
    what = sys.argv[1:] or ["small"]
    if "small" in what:
        make_small()
    if "config3" in what:
        make_config3()
    if "config4" in what:
        make_config4()
    if "config5" in what:
        make_config5()
