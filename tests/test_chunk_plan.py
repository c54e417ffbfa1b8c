"""How a one-shot batch is cut into pipelined chunks (mpzmm_batch_chunks,
the same routine mpzmm_matmul_batch uses), checked on the CPU against a
restatement of the policy: chunks of whole consecutive products, the first
two a quarter and a half of the chunk size, the last one split about 2:1,
automatic size a 32nd of the batch kept within 2^22..2^26 limbs."""
import random

import numpy as np
import pytest

from rforest_b200 import _lib, api, workloads as W


def model(limbs, option):
    n, total = len(limbs), sum(limbs)
    chunk = option if option > 0 else min(max(total // 32, 4 << 20), 64 << 20)
    chunk = max(chunk, 1)
    if n < 2 or total <= chunk:
        return [0, n]
    bounds, acc = [0], 0
    for t, l in enumerate(limbs):
        acc += l
        c = len(bounds) - 1
        target = chunk // 4 if c == 0 else (chunk // 2 if c == 1 else chunk)
        if acc >= target and t + 1 < n:
            bounds.append(t + 1)
            acc = 0
    bounds.append(n)
    if len(bounds) >= 3:
        a, b = bounds[-2], bounds[-1]
        tail = sum(limbs[a:b])
        if tail > chunk // 2 and b - a >= 2:
            acc2, cut = 0, a
            while cut + 1 < b and 3 * (acc2 + limbs[cut]) <= 2 * tail:
                acc2 += limbs[cut]
                cut += 1
            if cut > a:
                bounds.insert(len(bounds) - 1, cut)
    return bounds


@pytest.mark.parametrize("seed", range(6))
def test_matches_policy(product_lib, seed):
    rng = random.Random(seed)
    for _ in range(60):
        n = rng.randrange(0, 300)
        limbs = [rng.choice([0, 1, 7, rng.randrange(1, 5000), rng.randrange(1, 200000)])
                 for _ in range(n)]
        option = rng.choice([0, 1, 1000, 20000, 300000, 1 << 22])
        got = api.batch_chunks(limbs, option)
        assert got == model(limbs, option), (n, option)
        assert got[0] == 0 and got[-1] == n
        assert all(x < y for x, y in zip(got, got[1:])) or n == 0


def test_properties_explicit_size(product_lib):
    rng = random.Random(7)
    limbs = [rng.randrange(100, 3000) for _ in range(2000)]
    chunk = 50000
    b = api.batch_chunks(limbs, chunk)
    sums = [sum(limbs[x:y]) for x, y in zip(b, b[1:])]
    # ramp: a quarter, then a half of the chunk size, each closed by the
    # first product that reaches it
    assert sums[0] >= chunk // 4 and sums[0] - limbs[b[1] - 1] < chunk // 4
    assert sums[1] >= chunk // 2 and sums[1] - limbs[b[2] - 1] < chunk // 2
    for s, end in zip(sums[2:-2], b[3:-2]):
        assert chunk <= s < chunk + limbs[end - 1]
    # a final stretch above half a chunk goes out in two pieces, 2:1
    limbs = [100] * (25 + 50 + 10 * 100 + 90)
    b = api.batch_chunks(limbs, 10000)
    sums = [sum(limbs[x:y]) for x, y in zip(b, b[1:])]
    assert sums == [2500, 5000] + [10000] * 10 + [6000, 3000]


def test_small_batches_run_unchunked(product_lib):
    assert api.batch_chunks([], 0) == [0, 0]
    assert api.batch_chunks([1 << 30], 1000) == [0, 1]           # one product
    assert api.batch_chunks([10] * 100, 1000) == [0, 100]        # total <= chunk
    assert api.batch_chunks([10] * 100, 0) == [0, 100]           # below 2^22 limbs


def test_bad_arguments(product_lib):
    L = _lib.lib()
    n = _lib.C.c_int()
    assert L.mpzmm_batch_chunks(-1, None, 0, None, 0, _lib.C.byref(n)) == _lib.MPZMM_ERR_ARG
    neg = np.array([5, -1], dtype=np.int64)
    assert L.mpzmm_batch_chunks(2, neg.ctypes.data_as(_lib.i64p), 0, None, 0,
                                _lib.C.byref(n)) == _lib.MPZMM_ERR_ARG


def test_default_batch_makes_34_chunks(product_lib):
    """The 4096-product default batch: 34 chunks (the count the pipelined
    end-to-end measurement on B200 reported)."""
    limbs = [int(np.abs(p.A.sizes.astype(np.int64)).sum() + np.abs(p.B.sizes.astype(np.int64)).sum())
             for p in W.config3()]
    b = api.batch_chunks(limbs)
    assert len(b) - 1 == 34
    assert b == model(limbs, 0)
