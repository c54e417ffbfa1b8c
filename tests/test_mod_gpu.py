"""Modular reduction by a fixed modulus (mpzmm_mod_*) on the GPU, compared
bit-exactly with Python's x % d (the result in [0, d), as the reference's
mpzfft_mod_mod gives it)."""
import random

import pytest

from rforest_b200 import _lib, api, packed as PK

pytestmark = pytest.mark.gpu


def check(d, xs, max_bits):
    m = api.Mod(d, max_bits)
    try:
        R = m.reduce(PK.from_ints(xs))
        assert R.to_ints() == [x % d for x in xs]
    finally:
        m.close()


@pytest.mark.parametrize("dbits", [1, 2, 63, 64, 65, 640, 4096, 65537])
def test_random_moduli(gpu, dbits):
    rng = random.Random(dbits)
    d = rng.getrandbits(dbits) | (1 << (dbits - 1))
    max_bits = 2 * dbits + 130
    xs = [0, 1, -1, d, -d, d - 1, 1 - d, 2 * d, 3 * d - 1, -(3 * d) + 1,
          (1 << max_bits) - 1, -((1 << max_bits) - 1)]
    xs += [rng.choice([1, -1]) * rng.getrandbits(rng.randrange(1, max_bits + 1))
           for _ in range(60)]
    check(d, xs, max_bits)


def test_special_moduli(gpu):
    for d in (1, 2, 1 << 64, 1 << 128, (1 << 128) - 1, (1 << 192) + 1):
        xs = [0, 5, -5, d, d + 1, -(d + 1), (1 << 300) + 12345, -((1 << 299) + 7)]
        check(d, xs, 301)


def test_x_much_longer_than_d(gpu):
    rng = random.Random(5)
    d = rng.getrandbits(200) | (1 << 199)
    xs = [rng.choice([1, -1]) * rng.getrandbits(50000) for _ in range(40)]
    check(d, xs, 50000)


def test_batch_of_many(gpu):
    rng = random.Random(9)
    d = rng.getrandbits(4096) | (1 << 4095)
    xs = [rng.choice([1, -1]) * rng.getrandbits(8192) for _ in range(3000)]
    check(d, xs, 8192)


def test_too_large_and_bad_modulus(gpu):
    m = api.Mod(12345, 64)
    try:
        with pytest.raises(_lib.MpzmmError) as e:
            m.reduce(PK.from_ints([1 << 200]))
        assert e.value.status == _lib.MPZMM_ERR_TOO_LARGE
    finally:
        m.close()
    with pytest.raises(ValueError):
        api.Mod(0, 64)


def test_matches_reference_mod(gpu, oracle_mod):
    """The GPU reduction against the reference's own CPU mpzfft_mod_mod."""
    if not oracle_mod.reference_available():
        pytest.skip("reference CPU build not present")
    rng = random.Random(21)
    for dbits in (64, 1000, 16384):
        d = rng.getrandbits(dbits) | (1 << (dbits - 1))
        bits = 2 * dbits
        X = PK.from_ints([rng.choice([1, -1]) * rng.getrandbits(rng.randrange(1, bits + 1))
                          for _ in range(50)])
        m = api.Mod(d, bits)
        try:
            got = m.reduce(X)
        finally:
            m.close()
        assert PK.digest(got) == PK.digest(oracle_mod.mod_reference(d, X, bits))


def test_mpz_front_end(gpu):
    """mpz_t arrays in and out (rop grown by GMP), rop aliasing op too."""
    from rforest_b200 import gmp
    rng = random.Random(31)
    d = rng.getrandbits(3000) | (1 << 2999)
    xs = [0, 7, -7, d, -(d + 1)] + [rng.choice([1, -1]) * rng.getrandbits(6000) for _ in range(20)]
    m = api.Mod(d, 6000)
    try:
        X = gmp.MpzArray(xs)
        R = gmp.MpzArray(n=len(xs))
        _lib.check(_lib.lib().mpzmm_mod_mpz(m.handle, R.ptr(), X.ptr(), len(xs), None))
        assert R.to_ints() == [x % d for x in xs]
        _lib.check(_lib.lib().mpzmm_mod_mpz(m.handle, X.ptr(), X.ptr(), len(xs), None))
        assert X.to_ints() == [x % d for x in xs]
    finally:
        m.close()
