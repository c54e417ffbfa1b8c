"""Pipelined one-shot batches and straight copies from pinned host memory, on
the GPU.  Every result is compared bit-exactly: with the golden digests of
the 4096-product batch, with the same products computed unchunked, and with
Python integer arithmetic."""
import ctypes as C
import random

import numpy as np
import pytest

from rforest_b200 import _lib, api, packed as PK, workloads as W
from tests import golden_io as G

pytestmark = pytest.mark.gpu


@pytest.fixture
def small_chunks(gpu):
    """Chunks of 20000 input limbs, so a few hundred products make many chunks."""
    api.set_chunk_limbs(20000)
    yield
    api.set_chunk_limbs(0)


def config3_head(count):
    prods = [W.random_product(3001, t, 2, 16, 10, 18) for t in range(count)]
    return prods, [(p.m, p.k, p.n, p.A, p.B) for p in prods]


def want_digest(p):
    A, B = p.A.to_ints(), p.B.to_ints()
    return PK.digest(PK.from_ints(
        [sum(A[i * p.k + l] * B[l * p.n + j] for l in range(p.k))
         for i in range(p.m) for j in range(p.n)]))


def test_chunked_batch_matches_golden(small_chunks):
    d = G.digests()["config3"]["C"]
    count = 96
    _, triples = config3_head(count)
    outs = api.matmul_batch(triples)
    st = api.batch_stats()
    assert st["chunks"] >= 8  # really pipelined, more chunks than slots
    for t, c in enumerate(outs):
        assert PK.digest(c) == d[t], f"product {t}"


def test_batch_timeline(gpu):
    """The per-chunk timeline: host and device times in order, copies in
    stream order, bytes summing to the batch's totals."""
    _, triples = config3_head(48)
    for chunk in (1 << 30, 20000):  # one chunk, then pipelined
        api.set_chunk_limbs(chunk)
        try:
            api.matmul_batch(triples)
        finally:
            api.set_chunk_limbs(0)
        st = api.batch_stats()
        tl = api.batch_timeline()
        assert len(tl) == st["chunks"]
        assert (len(tl) == 1) == (chunk == 1 << 30)
        assert sum(r["h2d_bytes"] for r in tl) == st["h2d_bytes"]
        assert sum(r["d2h_bytes"] for r in tl) == st["d2h_bytes"]
        for c, r in enumerate(tl):
            assert 0 <= r["plan_begin"] <= r["plan_end"] <= r["queue_begin"] <= r["queue_end"]
            assert 0 <= r["h2d_begin"] <= r["h2d_end"] <= r["kernels_end"] <= r["d2h_end"]
            if c:
                assert tl[c - 1]["h2d_end"] <= r["h2d_begin"]
                assert tl[c - 1]["d2h_end"] <= r["d2h_end"]


def test_pinned_batch_matches_golden(gpu):
    d = G.digests()["config3"]["C"]
    count = 64
    _, triples = config3_head(count)
    b = api.Batch(triples, pinned=True)
    try:
        for chunk in (1 << 30, 30000):  # unchunked, then pipelined
            api.set_chunk_limbs(chunk)
            outs = b.run()
            st = api.batch_stats()
            assert st["h2d_direct_bytes"] > 0 and st["d2h_direct_bytes"] > 0
            for t, c in enumerate(outs):
                assert PK.digest(c) == d[t], f"product {t} (chunk limbs {chunk})"
    finally:
        api.set_chunk_limbs(0)
        b.close()


def test_pinned_and_pageable_mixed(small_chunks):
    prods = [W.random_product(41, t, 2, 7, 8, 15) for t in range(30)]
    triples = [(p.m, p.k, p.n, p.A, p.B) for p in prods]
    pinned = api.Batch(triples[::2], pinned=True)
    plain = api.Batch(triples[1::2])
    try:
        # one batch whose products alternate between the two kinds of memory
        hold = [pinned.holders[i // 2] if i % 2 == 0 else plain.holders[i // 2]
                for i in range(len(triples))]
        arr = (_lib.Product * len(hold))(*[h.struct for h in hold])
        _lib.check(_lib.lib().mpzmm_matmul_batch(len(hold), arr, None))
        for p, h in zip(prods, hold):
            assert PK.digest(h.result()) == want_digest(p)
    finally:
        pinned.close()


def exact_cap(p):
    a_bits = max((abs(x).bit_length() for x in p.A.to_ints()), default=0)
    b_bits = max((abs(x).bit_length() for x in p.B.to_ints()), default=0)
    return api.output_limbs(p.k, a_bits, b_bits)


@pytest.mark.parametrize("extra", [0, 1, 3])
def test_pinned_output_strides(gpu, extra):
    """Output capacity equal to the device's bound (extra 0: entries back to
    back, one plain copy for neighbouring products) or larger (a strided copy
    per product)."""
    prods = [W.random_product(43, t, 2, 6, 8, 14) for t in range(12)]
    arena = api.HostArena(1 << 24)
    try:
        holders = []
        for p in prods:
            cap = exact_cap(p) + extra
            h = api._Holder(p.m, p.k, p.n, p.A, p.B,
                            bufs=(arena.take(p.A.limbs.size, np.uint64),
                                  arena.take(p.B.limbs.size, np.uint64),
                                  arena.take(p.m * p.n * cap, np.uint64)))
            h.caps[:] = cap
            h.co[:] = np.arange(p.m * p.n, dtype=np.int64) * cap
            holders.append(h)
        arr = (_lib.Product * len(holders))(*[h.struct for h in holders])
        for chunk in (0, 3000):
            api.set_chunk_limbs(chunk)
            for h in holders:
                h.cl[:] = 0
                h.csz[:] = 0
            _lib.check(_lib.lib().mpzmm_matmul_batch(len(holders), arr, None))
            assert api.batch_stats()["d2h_direct_bytes"] > 0
            for p, h in zip(prods, holders):
                assert PK.digest(h.result()) == want_digest(p)
    finally:
        api.set_chunk_limbs(0)
        arena.close()


def test_registered_user_memory(gpu):
    """Memory the caller pinned itself (mpzmm_host_register) is used in place."""
    prods = [W.random_product(47, t, 2, 8, 8, 14) for t in range(8)]
    pool = np.zeros(1 << 21, dtype=np.uint64)  # 16 MB of the caller's own memory
    _lib.check(_lib.lib().mpzmm_host_register(C.c_void_p(pool.ctypes.data), pool.nbytes))
    try:
        used = 0

        def take(n):
            nonlocal used
            v = pool[used:used + max(n, 1)]
            used += max(n, 1)
            return v

        holders = []
        for p in prods:
            cap = api._Holder.out_cap(p.k, p.A, p.B)
            holders.append(api._Holder(p.m, p.k, p.n, p.A, p.B,
                                       bufs=(take(p.A.limbs.size), take(p.B.limbs.size),
                                             take(p.m * p.n * cap))))
        arr = (_lib.Product * len(holders))(*[h.struct for h in holders])
        _lib.check(_lib.lib().mpzmm_matmul_batch(len(holders), arr, None))
        assert api.batch_stats()["h2d_direct_bytes"] > 0
        for p, h in zip(prods, holders):
            assert PK.digest(h.result()) == want_digest(p)
    finally:
        _lib.check(_lib.lib().mpzmm_host_unregister(C.c_void_p(pool.ctypes.data)))


def test_host_memory_errors(gpu):
    with pytest.raises(_lib.MpzmmError) as e:
        _lib.check(_lib.lib().mpzmm_host_free(C.c_void_p(0x1000)))
    assert e.value.status == _lib.MPZMM_ERR_ARG
    with pytest.raises(_lib.MpzmmError) as e:
        _lib.check(_lib.lib().mpzmm_host_unregister(C.c_void_p(0x1000)))
    assert e.value.status == _lib.MPZMM_ERR_ARG
    arena = api.HostArena(4096)
    with pytest.raises(_lib.MpzmmError):  # owned memory is freed, not unregistered
        _lib.check(_lib.lib().mpzmm_host_unregister(C.c_void_p(arena.ptr)))
    arena.close()


def test_chunked_capacity_error_keeps_other_results(small_chunks):
    """A too-small capacity in one product is reported; every other product
    of the pipelined batch is still written."""
    prods = [W.random_product(53, t, 2, 6, 8, 15) for t in range(40)]
    b = api.Batch([(p.m, p.k, p.n, p.A, p.B) for p in prods])
    bad = 5
    b.holders[bad].caps[:] = 1
    with pytest.raises(_lib.MpzmmError) as e:
        b.run()
    assert e.value.status == _lib.MPZMM_ERR_CAPACITY
    for t, (p, h) in enumerate(zip(prods, b.holders)):
        if t == bad:
            continue
        assert PK.digest(h.result()) == want_digest(p), f"product {t}"


def gapped(arena, P, gaps):
    """Copy of packed vector P in the arena with the given gaps (limbs) of
    garbage before each entry."""
    n = P.nlimbs
    limbs = arena.take(int(n.sum()) + sum(gaps), np.uint64)
    limbs[:] = np.uint64(0xDEADBEEFDEADBEEF)
    offs = np.zeros(len(P), dtype=np.int64)
    pos = 0
    for e in range(len(P)):
        pos += gaps[e]
        offs[e] = pos
        limbs[pos:pos + n[e]] = P.limbs[P.offs[e]:P.offs[e] + n[e]]
        pos += int(n[e])
    return PK.Packed(limbs, offs, P.sizes.copy())


def test_pinned_inputs_with_gaps(gpu):
    """Entries separated by gaps of garbage in pinned memory: short gaps are
    bridged by one copy, long ones split it; results are unaffected."""
    rng = random.Random(61)
    prods = [W.random_product(59, t, 2, 6, 8, 14) for t in range(10)]
    arena = api.HostArena(1 << 25)
    try:
        choices = [0, 1, 5, 31, 255, 256, 257, 1000]
        triples = []
        for p in prods:
            A = gapped(arena, p.A, [rng.choice(choices) for _ in range(len(p.A))])
            B = gapped(arena, p.B, [rng.choice(choices) for _ in range(len(p.B))])
            triples.append((p.m, p.k, p.n, A, B))
        for chunk in (0, 2000):
            api.set_chunk_limbs(chunk)
            holders = [api._Holder(*t) for t in triples]
            for h, t in zip(holders, triples):  # operands stay where they are
                assert h.al.ctypes.data == t[3].limbs.ctypes.data
            arr = (_lib.Product * len(holders))(*[h.struct for h in holders])
            _lib.check(_lib.lib().mpzmm_matmul_batch(len(holders), arr, None))
            assert api.batch_stats()["h2d_direct_bytes"] > 0
            for p, h in zip(prods, holders):
                assert PK.digest(h.result()) == want_digest(p)
    finally:
        api.set_chunk_limbs(0)
        arena.close()


def test_pipeline_edge_cases(small_chunks):
    """Empty batch; zero products, 1 x 1 products and empty-sized entries
    mixed into a pipelined batch (chunks that are partly or wholly zero)."""
    assert api.matmul_batch([]) == []
    rng = random.Random(67)
    prods = []
    for t in range(60):
        kind = t % 5
        m, k, n = rng.randrange(1, 5), rng.randrange(1, 5), rng.randrange(1, 5)
        if kind == 0:    # A is all zero
            A = PK.from_ints([0] * (m * k))
            B = PK.from_ints([rng.getrandbits(3000) for _ in range(k * n)])
        elif kind == 1:  # 1 x 1 x 1
            m = k = n = 1
            A = PK.from_ints([-rng.getrandbits(5000)])
            B = PK.from_ints([rng.getrandbits(5000)])
        else:
            A = PK.from_ints([rng.choice([0, 1, -1]) * rng.getrandbits(rng.choice([1, 64, 4000]))
                              for _ in range(m * k)])
            B = PK.from_ints([rng.choice([0, 1, -1]) * rng.getrandbits(rng.choice([1, 64, 4000]))
                              for _ in range(k * n)])
        prods.append((m, k, n, A, B))
    api.set_chunk_limbs(1000)  # the whole batch is a few thousand limbs
    outs = api.matmul_batch(prods)
    assert api.batch_stats()["chunks"] >= 2
    for (m, k, n, A, B), C in zip(prods, outs):
        a, b = A.to_ints(), B.to_ints()
        want = [sum(a[i * k + l] * b[l * n + j] for l in range(k))
                for i in range(m) for j in range(n)]
        assert C.to_ints() == want
