"""mpz_t matrices from Python, for the reference-compatible entry points.

Allocates real GMP ``mpz_t`` arrays through the GMP runtime (libgmp.so.10),
so ``mpz_rmatrix_mult_fft`` of libmpzmm_b200 is exercised exactly as rforest
would call it: C entries are grown by GMP's own mpz_realloc inside the
library.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence

from . import _lib

_gmp = None


class MpzStruct(C.Structure):
    _fields_ = [("_mp_alloc", C.c_int), ("_mp_size", C.c_int),
                ("_mp_d", C.POINTER(C.c_uint64))]


class _Gmp:
    """The four GMP routines used here, looked up by their exported names
    (attribute access would be name-mangled inside classes)."""

    def __init__(self):
        g = C.CDLL("libgmp.so.10")
        self.init = getattr(g, "__gmpz_init")
        self.init.argtypes = [C.c_void_p]
        self.clear = getattr(g, "__gmpz_clear")
        self.clear.argtypes = [C.c_void_p]
        self.limbs_write = getattr(g, "__gmpz_limbs_write")
        self.limbs_write.argtypes = [C.c_void_p, C.c_long]
        self.limbs_write.restype = C.POINTER(C.c_uint64)
        self.limbs_finish = getattr(g, "__gmpz_limbs_finish")
        self.limbs_finish.argtypes = [C.c_void_p, C.c_long]


def gmp() -> _Gmp:
    global _gmp
    if _gmp is None:
        _gmp = _Gmp()
    return _gmp


class MpzArray:
    """A C array of n initialised mpz_t."""

    def __init__(self, values: Sequence[int] = (), n: int = 0):
        vals = list(values)
        self.n = max(n, len(vals))
        self.arr = (MpzStruct * self.n)()
        g = gmp()
        for i in range(self.n):
            g.init(C.byref(self.arr[i]))
        for i, v in enumerate(vals):
            self.set(i, v)

    def set(self, i: int, v: int) -> None:
        mag = -v if v < 0 else v
        nl = (mag.bit_length() + 63) // 64
        g = gmp()
        if nl == 0:
            g.limbs_finish(C.byref(self.arr[i]), 0)
            return
        d = g.limbs_write(C.byref(self.arr[i]), nl)
        C.memmove(d, mag.to_bytes(8 * nl, "little"), 8 * nl)
        g.limbs_finish(C.byref(self.arr[i]), -nl if v < 0 else nl)

    def get(self, i: int) -> int:
        z = self.arr[i]
        n = abs(z._mp_size)
        if n == 0:
            return 0
        v = int.from_bytes(C.string_at(z._mp_d, 8 * n), "little")
        return -v if z._mp_size < 0 else v

    def to_ints(self) -> List[int]:
        return [self.get(i) for i in range(self.n)]

    def ptr(self):
        return C.cast(self.arr, C.c_void_p)

    def close(self) -> None:
        if self.arr is not None:
            g = gmp()
            for i in range(self.n):
                g.clear(C.byref(self.arr[i]))
            self.arr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hw_mpz_setup() -> None:
    _lib.lib().hw_mpz_setup()


def mpz_rmatrix_mult_fft(C_: MpzArray, A: MpzArray, r: int, B: MpzArray, d: int) -> None:
    """C = A * B through the library's reference-compatible mpz entry point."""
    w = MpzArray(n=1)
    _lib.lib().mpz_rmatrix_mult_fft(C_.ptr(), A.ptr(), r, B.ptr(), d, w.ptr())
    w.close()


def gpu_fft_suitable(A: MpzArray, r: int, B: MpzArray, d: int) -> int:
    """mpz_rmatrix_gpu_fft_suitable: 1 if the library can multiply these."""
    return int(_lib.lib().mpz_rmatrix_gpu_fft_suitable(A.ptr(), r, B.ptr(), d))
