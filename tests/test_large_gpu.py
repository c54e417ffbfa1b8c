"""Transforms longer than one CTA holds (2^16 .. 2^20 points), on the GPU.

The reference handles any operand size: its CPU transform decomposes long
transforms into twisted sub-transforms (alexp616/rforest
src/lib/fft62.c:490-612 forward, :922-1043 inverse, threshold
src/include/fft62.h:61) and its GPU path runs up to lgN 26
(src/include/cufft62_thresholds.h:3).  Here transforms above 2^15 points run
in four steps (column transforms, twist, block transforms); every result is
compared bit-exactly with GMP schoolbook (mpz_mul / mpz_addmul, the
reference header's mpz_rmatrix_mult_naive) on the same seeded inputs.
"""
import random

import pytest

from rforest_b200 import api, packed as PK

pytestmark = pytest.mark.gpu


def _signed(rng, bits):
    v = rng.getrandbits(bits) | (1 << (bits - 1))
    return -v if rng.random() < 0.5 else v


def _check(m, k, n, Ai, Bi, oracle_mod):
    A, B = PK.from_ints(Ai), PK.from_ints(Bi)
    got = api.matmul(m, k, n, A, B)
    want = oracle_mod.matmul_schoolbook(m, k, n, A, B)
    assert PK.digest(got) == PK.digest(want)
    return A, B


def test_2x2_of_2pow23_bit_signed_entries(gpu, oracle_mod):
    rng = random.Random(23)
    Ai = [_signed(rng, 1 << 23) for _ in range(4)]
    Bi = [_signed(rng, 1 << 23) for _ in range(4)]
    A, B = _check(2, 2, 2, Ai, Bi, oracle_mod)
    P, r, lg = api.choose_params(1 << 23, 1 << 23, 2)
    assert lg > 15  # the four-step path


@pytest.mark.parametrize("bits", [3_300_000, 6_500_000, 13_000_000, 26_000_000, 52_000_000])
def test_each_long_transform_length(gpu, oracle_mod, bits):
    """One product per transform length 2^16 .. 2^20 (1 x 2 by 2 x 1, so the
    contraction sums two products)."""
    P, r, lg = api.choose_params(bits, bits, 2)
    assert 16 <= lg <= 20
    rng = random.Random(bits)
    Ai = [_signed(rng, bits) for _ in range(2)]
    Bi = [_signed(rng, bits - 17) for _ in range(2)]
    _check(1, 2, 1, Ai, Bi, oracle_mod)


def test_unbalanced_operands(gpu, oracle_mod):
    """A 4-Mbit entry times small ones: A's polynomial fills most of the
    transform (no zero upper half), B's a few points."""
    rng = random.Random(7)
    Ai = [_signed(rng, 1 << 22), -1, 0, _signed(rng, 100)]
    Bi = [_signed(rng, 64), _signed(rng, 3), (1 << 64) - 1, _signed(rng, 1 << 21)]
    _check(2, 2, 2, Ai, Bi, oracle_mod)


def test_long_carry_chains(gpu, oracle_mod):
    """All-ones magnitudes: every output word carries (a 2^17-point transform)."""
    big = (1 << (1 << 23)) - 1
    _check(1, 2, 1, [big, -big], [big, big - 2], oracle_mod)
    _check(1, 1, 1, [big], [-big], oracle_mod)


def test_mixed_lengths_in_one_batch(gpu, oracle_mod):
    """Short and long transforms in one batched call."""
    rng = random.Random(11)
    prods, wants = [], []
    for bits in (3000, 1 << 21, 70000, 1 << 22, 500):
        Ai = [_signed(rng, bits) for _ in range(4)]
        Bi = [_signed(rng, bits) for _ in range(4)]
        A, B = PK.from_ints(Ai), PK.from_ints(Bi)
        prods.append((2, 2, 2, A, B))
        wants.append(PK.digest(oracle_mod.matmul_schoolbook(2, 2, 2, A, B)))
    got = [PK.digest(c) for c in api.matmul_batch(prods)]
    assert got == wants


def test_chain_past_4_mbit(gpu, oracle_mod):
    """A device-resident chain of 2x2 matrices of 1-Mbit entries whose running
    product passes 4 Mbit (five factors); each step equals schoolbook."""
    rng = random.Random(5)
    mats = [(2, 2, PK.from_ints([_signed(rng, 1 << 20) for _ in range(4)])) for _ in range(5)]
    M = mats[0][2]
    for _, _, X in mats[1:]:
        M = oracle_mod.matmul_schoolbook(2, 2, 2, M, X).compact()
    assert M.max_bits() > 4 * 1000 * 1000
    C = api.chain(mats)
    assert PK.digest(C) == PK.digest(M)


def test_reference_api_long_operands(gpu, oracle_mod):
    """mpz_rmatrix_gpu_fft_suitable is 1 and mpz_rmatrix_mult_fft is exact for
    operands that need a four-step transform (reference r x d by d x d form)."""
    from rforest_b200 import gmp
    rng = random.Random(3)
    r, d = 1, 2
    Ai = [_signed(rng, 1 << 22) for _ in range(r * d)]
    Bi = [_signed(rng, 1 << 22) for _ in range(d * d)]
    A, B = gmp.MpzArray(Ai), gmp.MpzArray(Bi)
    C = gmp.MpzArray([0] * (r * d))
    try:
        assert gmp.gpu_fft_suitable(A, r, B, d) == 1
        gmp.mpz_rmatrix_mult_fft(C, A, r, B, d)
        want = oracle_mod.matmul_schoolbook(r, d, d, PK.from_ints(Ai), PK.from_ints(Bi))
        assert C.to_ints() == want.to_ints()
    finally:
        for x in (A, B, C):
            x.close()
