"""The oracle is pinned before it is trusted (CPU only).

* the C restatement, GMP schoolbook and Python integers agree with the
  reference's own CPU output stored in tests/golden (edge cases, config 1,
  config 2 and its chain);
* the seeded generator reproduces the pinned input digests;
* where the reference build (oracle/_ref) is present, all three agree with
  it on fresh seeded cases.
"""
import random

import numpy as np
import pytest

from rforest_b200 import packed as PK
from rforest_b200 import workloads as W
from tests import golden_io as G


def test_edge_cases_restated_and_schoolbook(oracle_mod):
    for (m, k, n, A, B, Cexp) in G.edge_cases():
        want = Cexp.to_ints()
        assert oracle_mod.matmul_restated(m, k, n, A, B).to_ints() == want
        assert oracle_mod.matmul_schoolbook(m, k, n, A, B).to_ints() == want
        assert oracle_mod.matmul_python(m, k, n, A.to_ints(), B.to_ints()) == want


def test_config1_golden(oracle_mod):
    A, B, Cexp = G.config1()
    d = G.digests()["config1"]
    assert PK.digest(A) == d["A"] and PK.digest(B) == d["B"]
    assert PK.digest(Cexp) == d["C"]
    assert PK.digest(oracle_mod.matmul_restated(4, 4, 4, A, B)) == d["C"]
    assert oracle_mod.matmul_python(4, 4, 4, A.to_ints(), B.to_ints()) == Cexp.to_ints()


def test_generator_pinned():
    d = G.digests()
    p = W.config1()
    assert PK.digest(p.A) == d["config1"]["A"]
    p = W.config2()
    assert PK.digest(p.A) == d["config2"]["A"] and PK.digest(p.B) == d["config2"]["B"]
    mats = W.config2_chain()
    assert [PK.digest(x) for x in mats] == d["config2_chain"]["inputs"]


def test_config2_restated_matches_reference_digest(oracle_mod):
    p = W.config2()
    C = oracle_mod.matmul_restated(8, 8, 8, p.A, p.B)
    assert PK.digest(C) == G.digests()["config2"]["C"]


def test_config2_chain_first_steps(oracle_mod):
    d = G.digests()["config2_chain"]
    mats = W.config2_chain()
    M = mats[0]
    for i in range(1, 3):
        M = oracle_mod.matmul_schoolbook(8, 8, 8, M, mats[i]).compact()
        assert PK.digest(M) == d["steps"][i - 1]


def test_config3_sample_schoolbook(oracle_mod):
    d = G.digests()
    if "config3" not in d:
        pytest.skip("config3 digests not generated")
    for t in range(0, 12):
        p = W.random_product(3001, t, 2, 16, 10, 18)
        assert [p.m, p.k, p.n, p.bits] == d["config3"]["shapes"][t]
        if p.bits > 40000:
            continue
        C = oracle_mod.matmul_schoolbook(p.m, p.k, p.n, p.A, p.B)
        assert PK.digest(C) == d["config3"]["C"][t]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_shapes_against_reference(oracle_mod, seed):
    if not oracle_mod.reference_available():
        pytest.skip("reference build oracle/_ref not present")
    rng = random.Random(seed)
    for _ in range(6):
        m, k, n = rng.randint(1, 5), rng.randint(1, 5), rng.randint(1, 5)
        bits = rng.choice([1, 63, 64, 65, 700, 3000, 9000])
        Ai = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(m * k)]
        Bi = [rng.randrange(-(1 << bits), 1 << bits) for _ in range(k * n)]
        if rng.random() < 0.3:
            Ai[0] = 0
        A, B = PK.from_ints(Ai), PK.from_ints(Bi)
        want = oracle_mod.matmul_python(m, k, n, Ai, Bi)
        assert oracle_mod.matmul_reference(m, k, n, A, B).to_ints() == want
        assert oracle_mod.matmul_restated(m, k, n, A, B).to_ints() == want
        assert oracle_mod.matmul_schoolbook(m, k, n, A, B).to_ints() == want


def test_planted_mistake_is_caught(oracle_mod):
    """A single flipped bit in an oracle output must change the digest."""
    p = W.config1()
    C = oracle_mod.matmul_restated(4, 4, 4, p.A, p.B).compact()
    good = PK.digest(C)
    C.limbs[5] ^= np.uint64(1 << 17)
    assert PK.digest(C) != good


def test_reference_params_match_survey(oracle_mod):
    # (r, lgN, points) the reference picks for config 1 / config 2
    assert oracle_mod.reference_params(64, 4) == (119, 7, 71)
    assert oracle_mod.reference_params(1024, 8) == (117, 11, 1122)


def test_reference_mod_pinned(oracle_mod):
    """The reference's own CPU x mod d (mpzfft_mod_mod, Fermat-transform
    reciprocal) against Python integers: the oracle of the GPU reduction."""
    if not oracle_mod.reference_available():
        pytest.skip("reference CPU build not present")
    rng = random.Random(13)
    for dbits in (1, 63, 64, 65, 640, 4096, 30000):
        d = rng.getrandbits(dbits) | (1 << (dbits - 1))
        bits = 2 * dbits + 200
        xs = [0, 1, -1, d, -d, d - 1, 3 * d + 5]
        xs += [rng.choice([1, -1]) * rng.getrandbits(rng.randrange(1, bits)) for _ in range(40)]
        R = oracle_mod.mod_reference(d, PK.from_ints(xs), bits)
        assert R.to_ints() == [x % d for x in xs], dbits
