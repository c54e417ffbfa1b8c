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
    (1 << 21, 1 << 21, 2), (1 << 23, 1 << 23, 2), (1 << 24, 1 << 24, 2),
    (100000000, 100000000, 5), (10000000, 10000000, 5), (1 << 22, 64, 1)])
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
    assert 2 <= P <= 16 and lg <= 20


def test_long_operands_are_suitable(product_lib):
    """Transforms up to 2^20 points (four-step above 2^15): the operand sizes of
    the reference's own benchmark (benchmark/bench_matmul.c: 10^7 and 10^8
    bits, 2x2 and 5x5) all get parameters."""
    for bits, d in [(10000000, 2), (10000000, 5), (100000000, 2), (100000000, 5)]:
        P, r, lg = api.choose_params(bits, bits, d)
        assert 16 <= lg <= 20


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


def test_failure_injection_options_host_only(product_lib):
    """The failure-injection options are host state: set, read back, rejected
    when negative, cleared (no device needed)."""
    L = product_lib
    for opt in (_lib.MPZMM_OPT_TEST_STALL_TC, _lib.MPZMM_OPT_TEST_FAIL_ALLOC):
        assert L.mpzmm_set_option(opt, 3) == _lib.MPZMM_OK
        assert L.mpzmm_get_option(opt) == 3
        assert L.mpzmm_set_option(opt, -1) == _lib.MPZMM_ERR_ARG
        assert L.mpzmm_set_option(opt, 0) == _lib.MPZMM_OK
        assert L.mpzmm_get_option(opt) == 0


def test_bounds_check_option_host_only(product_lib):
    """The debug bounds-check option is host state: 0 or 1, read back."""
    L = product_lib
    assert L.mpzmm_set_option(_lib.MPZMM_OPT_CHECK_BOUNDS, 2) == _lib.MPZMM_ERR_ARG
    assert L.mpzmm_set_option(_lib.MPZMM_OPT_CHECK_BOUNDS, 1) == _lib.MPZMM_OK
    assert L.mpzmm_get_option(_lib.MPZMM_OPT_CHECK_BOUNDS) == 1
    assert L.mpzmm_set_option(_lib.MPZMM_OPT_CHECK_BOUNDS, 0) == _lib.MPZMM_OK
    assert L.mpzmm_get_option(_lib.MPZMM_OPT_CHECK_BOUNDS) == 0


def test_reference_drivers_link_against_the_library():
    """Where the reference tree exists, its own tests/test_matmul.c and
    benchmark/bench_matmul.c compile unmodified with this library's header
    forced in after the reference's (a declaration mismatch would fail the
    compile) and resolve libmpzmm_b200.so at load time."""
    import subprocess
    from oracle import oracle as O
    if not O.reference_tree_present():
        pytest.skip("reference tree not present")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    subprocess.run(["make", "-s", "-C", os.path.join(root, "oracle"),
                    f"REF={O.REFERENCE_DIR}", "dropin"], check=True)
    for exe in ("test_matmul_b200", "bench_matmul_b200"):
        path = os.path.join(root, "oracle", "_ref", exe)
        out = subprocess.run(["ldd", path], capture_output=True, text=True, check=True).stdout
        line = [ln for ln in out.splitlines() if "libmpzmm_b200.so" in ln]
        assert line and "not found" not in line[0], out
