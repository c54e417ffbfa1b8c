"""Parity of the CUDA path with the oracle and the reference's own outputs.

Every test calls the product through the C ABI of libmpzmm_b200.so and
compares bit-exactly: with Python integers / the GMP schoolbook oracle on
seeded inputs, with the golden outputs the reference's CPU
mpz_rmatrix_mult_fft produced (tests/golden), and, at full sizes, through a
size-independent property (C mod q == (A mod q)(B mod q) mod q for random
61-bit primes q).
"""
import random

import numpy as np
import pytest

from rforest_b200 import api, packed as PK, workloads as W
from tests import golden_io as G

pytestmark = pytest.mark.gpu


def test_config1_golden(gpu):
    A, B, Cexp = G.config1()
    C = api.matmul(4, 4, 4, A, B)
    assert C.to_ints() == Cexp.to_ints()
    assert PK.digest(C) == G.digests()["config1"]["C"]


def test_edge_cases_golden(gpu):
    for (m, k, n, A, B, Cexp) in G.edge_cases():
        C = api.matmul(m, k, n, A, B)
        assert C.to_ints() == Cexp.to_ints(), (m, k, n)


@pytest.mark.parametrize("seed", range(4))
def test_random_small_vs_python(gpu, seed):
    rng = random.Random(100 + seed)
    for _ in range(8):
        m, k, n = rng.randint(1, 7), rng.randint(1, 9), rng.randint(1, 7)
        bits_a = rng.choice([1, 2, 31, 63, 64, 65, 127, 128, 129, 500, 2048, 5000])
        bits_b = rng.choice([1, 64, 65, 300, 4096, 20000])
        Ai = [rng.randrange(-(1 << bits_a), 1 << bits_a) for _ in range(m * k)]
        Bi = [rng.randrange(-(1 << bits_b), 1 << bits_b) for _ in range(k * n)]
        for lst in (Ai, Bi):
            if rng.random() < 0.3:
                lst[rng.randrange(len(lst))] = 0
            if rng.random() < 0.2:
                lst[rng.randrange(len(lst))] = (1 << (64 * rng.randint(1, 4))) - 1
        C = api.matmul(m, k, n, PK.from_ints(Ai), PK.from_ints(Bi))
        want = [sum(Ai[i * k + l] * Bi[l * n + j] for l in range(k))
                for i in range(m) for j in range(n)]
        assert C.to_ints() == want


def test_carry_chains(gpu):
    """Results whose limbs are long runs of 0 / all-ones, both signs."""
    for L in (64, 640, 6400, 64000):
        x = (1 << L) - 1
        cases = [([x, 1], [x, -1]), ([x, x], [1, 1]), ([-(x), 1], [x, 1 << L]),
                 ([1 << L, -1], [1 << L, 1])]
        for Ai, Bi in cases:
            C = api.matmul(1, 2, 1, PK.from_ints(Ai), PK.from_ints(Bi))
            assert C.to_ints() == [Ai[0] * Bi[0] + Ai[1] * Bi[1]]


def test_config2_golden(gpu):
    p = W.config2()
    C = api.matmul(8, 8, 8, p.A, p.B)
    assert PK.digest(C) == G.digests()["config2"]["C"]


def test_config2_chain_golden(gpu):
    d = G.digests()["config2_chain"]
    mats = W.config2_chain()
    M = mats[0]
    for i in range(1, len(mats)):
        M = api.matmul(8, 8, 8, M, mats[i]).compact()
        assert PK.digest(M) == d["steps"][i - 1], f"chain step {i}"


def test_config3_batch_golden(gpu):
    d = G.digests()
    if "config3" not in d:
        pytest.skip("config3 digests not generated")
    count = 256
    prods = [W.random_product(3001, t, 2, 16, 10, 18) for t in range(count)]
    outs = api.matmul_batch([(p.m, p.k, p.n, p.A, p.B) for p in prods])
    for t, C in enumerate(outs):
        assert PK.digest(C) == d["config3"]["C"][t], f"product {t}"


def test_batch_equals_individual(gpu):
    prods = [W.random_product(7, t, 2, 9, 8, 14) for t in range(24)]
    batch = api.matmul_batch([(p.m, p.k, p.n, p.A, p.B) for p in prods])
    for p, C in zip(prods, batch):
        single = api.matmul(p.m, p.k, p.n, p.A, p.B)
        assert PK.digest(single) == PK.digest(C)


def test_plan_reexecute(gpu):
    prods = [W.random_product(11, t, 2, 6, 8, 13) for t in range(10)]
    plan = api.Plan([(p.m, p.k, p.n, p.A, p.B) for p in prods])
    plan.execute()
    first = [PK.digest(c) for c in plan.download()]
    for _ in range(3):
        plan.execute()
    again = [PK.digest(c) for c in plan.download()]
    assert first == again
    for p, dg in zip(prods, first):
        want = [sum(a * b for a, b in zip(p.A.to_ints()[i * p.k:(i + 1) * p.k],
                                          p.B.to_ints()[j::p.n]))
                for i in range(p.m) for j in range(p.n)]
        assert dg == PK.digest(PK.from_ints(want))
    plan.close()


def test_mpz_reference_api(gpu, oracle_mod):
    """The drop-in entry point over real GMP mpz_t arrays (r x d by d x d)."""
    from rforest_b200 import gmp
    gmp.hw_mpz_setup()
    rng = random.Random(5)
    for (r, d, bits) in [(4, 4, 4096), (1, 5, 3000), (3, 2, 100000), (2, 2, 1)]:
        Ai = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(r * d)]
        Bi = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(d * d)]
        A, B = gmp.MpzArray(Ai), gmp.MpzArray(Bi)
        C = gmp.MpzArray(n=r * d)
        C.set(0, 12345)  # pre-existing value must be overwritten
        gmp.mpz_rmatrix_mult_fft(C, A, r, B, d)
        want = [sum(Ai[i * d + l] * Bi[l * d + j] for l in range(d))
                for i in range(r) for j in range(d)]
        assert C.to_ints() == want
        if oracle_mod.reference_available():
            ref = oracle_mod.matmul_reference(r, d, d, PK.from_ints(Ai), PK.from_ints(Bi))
            assert ref.to_ints() == want


def _mod_q(P: PK.Packed, q: int):
    out = []
    for e in range(len(P)):
        out.append(P.entry(e) % q)
    return out


def test_config4_full_size(gpu):
    """64x64 by 64x64 of 2^20-bit entries: golden digest + mod-q property."""
    p = W.config4()
    C = api.matmul(64, 64, 64, p.A, p.B)
    d = G.digests()
    if "config4" in d:
        assert PK.digest(C) == d["config4"]["C"]
    q = (1 << 61) - 1
    Aq, Bq, Cq = _mod_q(p.A, q), _mod_q(p.B, q), _mod_q(C, q)
    for i in range(0, 64, 7):
        for j in range(0, 64, 5):
            s = sum(Aq[i * 64 + l] * Bq[l * 64 + j] for l in range(64)) % q
            assert s == Cq[i * 64 + j]


# ---------------------------------------------------------------------------
# the tensor-core contraction (tcgen05 kind::i8), forced on every eligible
# product, against the same goldens / Python integers
# ---------------------------------------------------------------------------
@pytest.fixture
def tensor_cores(gpu):
    api.set_contract_mode(2)
    yield
    api.set_contract_mode(0)


@pytest.fixture
def cuda_cores(gpu):
    api.set_contract_mode(1)
    yield
    api.set_contract_mode(0)


def test_tc_config1_and_edges(tensor_cores):
    A, B, Cexp = G.config1()
    assert api.matmul(4, 4, 4, A, B).to_ints() == Cexp.to_ints()
    for (m, k, n, A, B, Cexp) in G.edge_cases():
        assert api.matmul(m, k, n, A, B).to_ints() == Cexp.to_ints(), (m, k, n)


@pytest.mark.parametrize("seed", range(3))
def test_tc_random_shapes(tensor_cores, seed):
    rng = random.Random(500 + seed)
    for _ in range(6):
        m, k, n = rng.randint(1, 40), rng.choice([1, 2, 7, 8, 31, 32, 33, 64]), rng.randint(1, 64)
        bits = rng.choice([64, 300, 2000, 9000])
        Ai = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(m * k)]
        Bi = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(k * n)]
        C = api.matmul(m, k, n, PK.from_ints(Ai), PK.from_ints(Bi))
        want = [sum(Ai[i * k + l] * Bi[l * n + j] for l in range(k))
                for i in range(m) for j in range(n)]
        assert C.to_ints() == want, (m, k, n, bits)


def test_tc_packed_slot_edges(tensor_cores):
    """Shapes at the edges of frequency packing (two or four frequencies an
    MMA for m <= 16 and n <= 32, K' slots of k rounded up to 8) and just
    past them, with transforms shorter than a staged block."""
    rng = random.Random(4242)
    for m in (1, 8, 9, 16, 17):
        for k in (1, 8, 9, 24, 33):
            for n in (1, 32, 33):
                bits = rng.choice([40, 700])
                Ai = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(m * k)]
                Bi = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(k * n)]
                C = api.matmul(m, k, n, PK.from_ints(Ai), PK.from_ints(Bi))
                want = [sum(Ai[i * k + l] * Bi[l * n + j] for l in range(k))
                        for i in range(m) for j in range(n)]
                assert C.to_ints() == want, (m, k, n, bits)


def test_tc_row_column_blocks(tensor_cores):
    """Products wider than one 32-row by 32-column block of C: each work
    item covers one block (partial blocks at the edges)."""
    rng = random.Random(777)
    for (m, k, n) in [(33, 3, 1), (1, 64, 65), (64, 64, 64), (100, 20, 70), (200, 9, 33)]:
        bits = rng.choice([50, 600])
        Ai = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(m * k)]
        Bi = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(k * n)]
        C = api.matmul(m, k, n, PK.from_ints(Ai), PK.from_ints(Bi))
        want = [sum(Ai[i * k + l] * Bi[l * n + j] for l in range(k))
                for i in range(m) for j in range(n)]
        assert C.to_ints() == want, (m, k, n, bits)


def test_tc_config2_golden(tensor_cores):
    p = W.config2()
    assert PK.digest(api.matmul(8, 8, 8, p.A, p.B)) == G.digests()["config2"]["C"]


def test_tc_batch_matches_cuda_cores(gpu):
    prods = [W.random_product(9, t, 2, 40, 8, 14) for t in range(12)]
    trip = [(p.m, p.k, p.n, p.A, p.B) for p in prods]
    api.set_contract_mode(1)
    try:
        a = [PK.digest(c) for c in api.matmul_batch(trip)]
        api.set_contract_mode(2)
        b = [PK.digest(c) for c in api.matmul_batch(trip)]
    finally:
        api.set_contract_mode(0)
    assert a == b


def test_tc_config4_full_size(tensor_cores):
    p = W.config4()
    C = api.matmul(64, 64, 64, p.A, p.B)
    d = G.digests()
    assert PK.digest(C) == d["config4"]["C"]


def test_autotune_then_automatic_engine_is_exact(gpu):
    times = api.autotune()
    assert len(times) == 20 and (64, 64) in times
    assert all(c > 0 and t > 0 for c, t in times.values())
    rng = random.Random(77)
    for (m, k, n) in [(5, 40, 7), (32, 64, 3), (2, 9, 2)]:
        Ai = [rng.randrange(-(1 << 3000), 1 << 3000) for _ in range(m * k)]
        Bi = [rng.randrange(-(1 << 2000), 1 << 2000) for _ in range(k * n)]
        C = api.matmul(m, k, n, PK.from_ints(Ai), PK.from_ints(Bi))
        want = [sum(Ai[i * k + l] * Bi[l * n + j] for l in range(k))
                for i in range(m) for j in range(n)]
        assert C.to_ints() == want
