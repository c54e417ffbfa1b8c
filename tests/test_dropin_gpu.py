"""The drop-in, proven in C: the reference's own exact-equality driver runs
against this library.

oracle/Makefile (target ``dropin``) compiles the reference's unmodified
tests/test_matmul.c in place, with the reference's headers and this
library's include/mpzmm_b200.h forced in after them (so the compiler checks
that every declaration the two share agrees), and links it against
libmpzmm_b200.so instead of the reference's src/lib/hwmpz.c.  The driver
fills r x d and d x d matrices with random bits-bit entries (a time-based
seed), multiplies them with mpz_rmatrix_mult_fft -- here, this library's GPU
path -- and compares every entry with GMP schoolbook (the reference header's
mpz_rmatrix_mult_naive), printing PASS and exiting 0 only if all match.

Arguments follow the reference's ctest registrations (CMakeLists.txt:144-145
runs ``test_matmul 50000 2 2``) plus wider and squarer cases.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "test_matmul_b200")

pytestmark = pytest.mark.gpu


def _driver():
    if not os.path.exists(DRIVER):
        pytest.skip("the reference's drivers were not built (reference tree absent where "
                    "this repository was built)")
    return DRIVER


def _run(*args, timeout=600):
    env = dict(os.environ)
    env.setdefault("MPZMM_DEVICE", "0")
    res = subprocess.run([_driver()] + [str(a) for a in args], capture_output=True, text=True,
                         timeout=timeout, env=env)
    return res.returncode, res.stdout + res.stderr


@pytest.mark.parametrize("bits,d,r", [(50000, 2, 2), (65536, 8, 8), (4096, 4, 4),
                                      (262144, 16, 16), (1000, 3, 2), (200000, 5, 1)])
def test_reference_driver_passes(bits, d, r):
    rc, out = _run(bits, d, r)
    assert rc == 0 and "PASS" in out, out[-2000:]
    assert f"all {r * d} entries match" in out
