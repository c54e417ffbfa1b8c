"""The C-ABI library builds, loads and exports every declared symbol, and its
host-only logic (parameter choice, output bounds, error paths) is right.
Runs without a GPU."""
import math
import os
import re

import pytest

from rforest_b200 import _lib, api
from rforest_b200.packed import from_ints

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                      "include", "mpzmm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^MPZMM_API [^;(]*?\b([a-z_0-9]+)\(", src, re.M)))


def test_exports_every_declared_symbol(product_lib):
    names = declared_functions()
    assert "mpz_rmatrix_mult_fft" in names and "hw_mpz_setup" in names
    for name in names:
        assert hasattr(product_lib, name), name


def test_reference_signature_names(product_lib):
    # the drop-in set of the reference's src/include/hwmpz.h
    for name in ("hw_mpz_setup", "hw_mpz_clear", "mpz_rmatrix_mult_fft",
                 "cu_mpz_rmatrix_mult_fft", "mpz_rmatrix_gpu_fft_suitable"):
        assert hasattr(product_lib, name)


def ntt_primes(count=16):
    """The library's primes, found independently: p < 2^30, p = 1 mod 2^20,
    descending."""
    def is_prime(n):
        if n < 2:
            return False
        i = 2
        while i * i <= n:
            if n % i == 0:
                return False
            i += 1
        return True
    out = []
    c = (1 << 10) - 1
    while len(out) < count:
        p = (c << 20) + 1
        if p < (1 << 30) and is_prime(p):
            out.append(p)
        c -= 1
    return out


@pytest.mark.parametrize("a_bits,b_bits,k", [
    (1, 1, 1), (64, 64, 1), (4096, 4096, 4), (65536, 65536, 8), (1 << 20, 1 << 20, 64),
    (1 << 18, 1 << 10, 16), (1 << 21, 1 << 16, 8), (300, 5, 32), (12345, 678, 3),
    (1 << 21, 1 << 21, 2)])
def test_params_exactness_bound(product_lib, a_bits, b_bits, k):
    """Every product coefficient c has 4|c| < p_0...p_{P-1} (the symmetric
    CRT residue is c, with the margin the rounded explicit CRT needs) and the
    product polynomial fits the transform length."""
    P, r, lg = api.choose_params(a_bits, b_bits, k)
    primes = ntt_primes()
    M = math.prod(primes[:P])
    lenA = -(-a_bits // r)
    lenB = -(-b_bits // r)
    bound = k * min(lenA, lenB) * ((1 << r) - 1) ** 2
    assert 4 * bound < M
    assert lenA + lenB - 1 <= (1 << lg)
    assert 2 <= P <= 16 and lg <= 15


def test_params_too_large_rejected(product_lib):
    with pytest.raises(_lib.MpzmmError) as e:
        api.choose_params(1 << 30, 1 << 30, 4)
    assert e.value.status == _lib.MPZMM_ERR_TOO_LARGE


def test_output_limbs_formula(product_lib):
    for k, a, b in [(1, 1, 1), (4, 4096, 4096), (64, 1 << 20, 1 << 20), (3, 100, 7)]:
        want = -(-(a + b + math.ceil(math.log2(k)) + 1) // 64)
        assert api.output_limbs(k, a, b) == want


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES") is None and
                    os.path.exists("/dev/nvidia0"), reason="only meaningful without a GPU")
def test_compute_without_device_fails_loudly(product_lib):
    """No CPU fallback: with no CUDA device the compute entry point returns
    MPZMM_ERR_CUDA instead of producing a result."""
    if product_lib.mpzmm_device_available():
        pytest.skip("a device is present")
    A = from_ints([3, 4])
    B = from_ints([5, 6])
    with pytest.raises(_lib.MpzmmError) as e:
        api.matmul(1, 2, 1, A, B)
    assert e.value.status == _lib.MPZMM_ERR_CUDA


def test_mpz_array_roundtrip():
    """mpz_t arrays built through the GMP runtime keep their values."""
    from rforest_b200 import gmp
    vals = [0, 1, -1, (1 << 64) - 1, -(1 << 200) + 3, 1 << 4096]
    a = gmp.MpzArray(vals)
    assert a.to_ints() == vals
    a.close()
