"""ctypes front end to the CPU oracles (TEST INFRASTRUCTURE ONLY).

Only tests, the smoke check and the benchmark's CPU-baseline leg import this
module, and only to check or time the product path.  Three oracles:

* ``restated``  -- oracle/mpzmm_oracle.c, a plain-C restatement of the
  reference pipeline (alexp616/rforest src/lib/hwmpz.c:65-130);
* ``schoolbook`` -- GMP mpz_mul / mpz_addmul (src/include/hwmpz.h:117-124);
* ``reference`` -- the reference's own CPU sources compiled in place
  (oracle/_ref), present wherever it was built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "_build", "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libref_mpzmm.so")

_u64p = C.POINTER(C.c_uint64)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)
_MATMUL_ARGS = [C.c_int, C.c_int, C.c_int, _u64p, _i64p, _i32p, _u64p, _i64p,
                _i32p, _u64p, _i64p, _i64p, _i32p]

_oracle = None
_ref = None

# Where the reference source tree lies (read only while building oracle/_ref;
# nothing reads it at run time).  RFOREST_REFERENCE overrides the default.
REFERENCE_DIR = os.environ.get("RFOREST_REFERENCE", "/root/reference")


def reference_tree_present() -> bool:
    return os.path.isdir(os.path.join(REFERENCE_DIR, "src", "lib"))


def build(with_reference: bool = True) -> None:
    """Compile the oracle (and, where the reference tree exists, oracle/_ref)."""
    targets = ["oracle"]
    if with_reference and reference_tree_present():
        targets.append("ref")
        # the reference's own drivers linked against the product library
        if os.path.exists(os.path.join(HERE, "..", "rforest_b200", "lib", "libmpzmm_b200.so")):
            targets.append("dropin")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_DIR}"] + targets, check=True)


def _load_oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(LIB_ORACLE):
            build(with_reference=False)
        lib = C.CDLL(LIB_ORACLE)
        for name in ("orc_matmul", "orc_matmul_naive"):
            f = getattr(lib, name)
            f.argtypes = _MATMUL_ARGS
            f.restype = C.c_int
        lib.orc_query_params.argtypes = [C.c_size_t, C.c_size_t, C.POINTER(C.c_uint),
                                         C.POINTER(C.c_uint), C.POINTER(C.c_size_t)]
        _oracle = lib
    return _oracle


def reference_available() -> bool:
    return os.path.exists(LIB_REF)


def _load_ref():
    global _ref
    if _ref is None:
        if not os.path.exists(LIB_REF):
            raise RuntimeError("reference CPU build oracle/_ref is not present")
        lib = C.CDLL(LIB_REF)
        lib.ref_matmul.argtypes = _MATMUL_ARGS
        lib.ref_matmul.restype = C.c_int
        lib.ref_setup.argtypes = []
        lib.ref_mod.argtypes = [_u64p, C.c_int32, C.c_int64, C.c_int, _u64p, _i64p, _i32p,
                                _u64p, _i64p, _i64p, _i32p]
        lib.ref_mod.restype = C.c_int
        _ref = lib
    return _ref


def _ptr(a, t):
    return a.ctypes.data_as(t)


def _call(fn, m, k, n, A, B):
    from rforest_b200.packed import Packed, output_layout, product_limb_bound
    cap = product_limb_bound(A, B, k)
    caps = np.full(m * n, cap, dtype=np.int64)
    offs, total = output_layout(caps)
    out = np.zeros(max(total, 1), dtype=np.uint64)
    sizes = np.zeros(m * n, dtype=np.int32)
    al = np.ascontiguousarray(A.limbs, dtype=np.uint64)
    bl = np.ascontiguousarray(B.limbs, dtype=np.uint64)
    if al.size == 0:
        al = np.zeros(1, np.uint64)
    if bl.size == 0:
        bl = np.zeros(1, np.uint64)
    ao = np.ascontiguousarray(A.offs, dtype=np.int64)
    bo = np.ascontiguousarray(B.offs, dtype=np.int64)
    asz = np.ascontiguousarray(A.sizes, dtype=np.int32)
    bsz = np.ascontiguousarray(B.sizes, dtype=np.int32)
    st = fn(m, k, n, _ptr(al, _u64p), _ptr(ao, _i64p), _ptr(asz, _i32p),
            _ptr(bl, _u64p), _ptr(bo, _i64p), _ptr(bsz, _i32p),
            _ptr(out, _u64p), _ptr(offs, _i64p), _ptr(caps, _i64p), _ptr(sizes, _i32p))
    if st != 0:
        raise RuntimeError("oracle output capacity too small")
    return Packed(out, offs, sizes)


def matmul_restated(m, k, n, A, B):
    """C = A*B through the C restatement of the reference pipeline."""
    return _call(_load_oracle().orc_matmul, m, k, n, A, B)


def matmul_schoolbook(m, k, n, A, B):
    """C = A*B with GMP schoolbook multiplication."""
    return _call(_load_oracle().orc_matmul_naive, m, k, n, A, B)


def matmul_reference(m, k, n, A, B):
    """C = A*B with the reference's own CPU mpz_rmatrix_mult_fft."""
    return _call(_load_ref().ref_matmul, m, k, n, A, B)


def mod_reference(d: int, X, bits: int):
    """x mod d in [0, d) for every entry of packed X with the reference's own
    CPU mpzfft_mod_init / mpzfft_mod_mod (|x| and d of at most `bits` bits)."""
    from rforest_b200.packed import Packed, from_ints
    D = from_ints([d])
    n = int(D.sizes[0])
    count = len(X)
    dl = np.ascontiguousarray(D.limbs, dtype=np.uint64)
    xl = np.ascontiguousarray(X.limbs, dtype=np.uint64)
    if xl.size == 0:
        xl = np.zeros(1, np.uint64)
    xo = np.ascontiguousarray(X.offs, dtype=np.int64)
    xs = np.ascontiguousarray(X.sizes, dtype=np.int32)
    out = np.zeros(max(count * n, 1), dtype=np.uint64)
    offs = np.arange(count, dtype=np.int64) * n
    caps = np.full(count, n, dtype=np.int64)
    sizes = np.zeros(count, dtype=np.int32)
    st = _load_ref().ref_mod(_ptr(dl, _u64p), n, int(bits), count, _ptr(xl, _u64p),
                             _ptr(xo, _i64p), _ptr(xs, _i32p), _ptr(out, _u64p),
                             _ptr(offs, _i64p), _ptr(caps, _i64p), _ptr(sizes, _i32p))
    if st != 0:
        raise RuntimeError("oracle output capacity too small")
    return Packed(out, offs, sizes)


def reference_params(maxlimbs: int, terms: int):
    """(r, lgN, points) the reference CPU path picks (src/lib/mpnfft.c:18-78)."""
    lib = _load_oracle()
    r, lg, pts = C.c_uint(), C.c_uint(), C.c_size_t()
    lib.orc_query_params(maxlimbs, terms, C.byref(r), C.byref(lg), C.byref(pts))
    return r.value, lg.value, pts.value


def matmul_python(m, k, n, A_ints, B_ints):
    """Pure-Python exact product (small cases only)."""
    out = []
    for i in range(m):
        for j in range(n):
            out.append(sum(A_ints[i * k + l] * B_ints[l * n + j] for l in range(k)))
    return out
