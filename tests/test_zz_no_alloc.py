"""mpzmm_matmul_noalloc: the entry point for callers that cannot allocate
device memory (their GPU memory belongs to a host framework's pool, or they
cannot pay for cudaMalloc/cudaFree).  It works out of a static scratch array
inside the library; the caller brings device buffers for operands and
results.

Checked through the C ABI against the ordinary entry point (mpzmm_matmul) on
two calls in a row, bit-exact as every parity test here.  Collected last (the
file name sorts last) so that a run stopping at its first failure has already
run every other test; it also passes alone in a fresh process.
"""
import ctypes as C
import random

import numpy as np
import pytest

from rforest_b200 import _lib, api, packed as PK, workloads as W

pytestmark = pytest.mark.gpu


def _noalloc(m, k, n, A: PK.Packed, B: PK.Packed):
    import torch
    L = _lib.lib()
    cap = api.output_limbs(k, 64 * A.max_limbs(), 64 * B.max_limbs())
    dev = torch.device("cuda", 0)
    d_a = torch.from_numpy(np.ascontiguousarray(A.limbs, dtype=np.uint64).view(np.int64)
                           if A.limbs.size else np.zeros(1, np.int64)).to(dev)
    d_b = torch.from_numpy(np.ascontiguousarray(B.limbs, dtype=np.uint64).view(np.int64)
                           if B.limbs.size else np.zeros(1, np.int64)).to(dev)
    d_c = torch.zeros(m * n * cap, dtype=torch.int64, device=dev)
    d_sz = torch.full((m * n,), 777, dtype=torch.int32, device=dev)
    c_offs = np.arange(m * n, dtype=np.int64) * cap
    c_caps = np.full(m * n, cap, dtype=np.int64)
    a_offs = np.ascontiguousarray(A.offs, dtype=np.int64)
    a_sz = np.ascontiguousarray(A.sizes, dtype=np.int32)
    b_offs = np.ascontiguousarray(B.offs, dtype=np.int64)
    b_sz = np.ascontiguousarray(B.sizes, dtype=np.int32)
    stream = torch.cuda.current_stream(dev)
    st = L.mpzmm_matmul_noalloc(
        m, k, n, C.c_void_p(d_a.data_ptr()), a_offs.ctypes.data_as(_lib.i64p),
        a_sz.ctypes.data_as(_lib.i32p), C.c_void_p(d_b.data_ptr()),
        b_offs.ctypes.data_as(_lib.i64p), b_sz.ctypes.data_as(_lib.i32p),
        C.c_void_p(d_c.data_ptr()), c_offs.ctypes.data_as(_lib.i64p),
        c_caps.ctypes.data_as(_lib.i64p), C.c_void_p(d_sz.data_ptr()),
        C.c_void_p(stream.cuda_stream))
    _lib.check(st)
    torch.cuda.synchronize(dev)
    limbs = d_c.cpu().numpy().view(np.uint64)
    return PK.Packed(limbs, c_offs, d_sz.cpu().numpy().astype(np.int32))


def test_noalloc_matches_ordinary_entry_point_twice(product_lib):
    rng = random.Random(2024)
    m2, k2, n2 = 3, 5, 2
    Ai = [rng.randrange(-(1 << 3000), 1 << 3000) for _ in range(m2 * k2)]
    Bi = [rng.randrange(-(1 << 700), 1 << 700) for _ in range(k2 * n2)]
    Ai[4] = 0
    Bi[1] = (1 << 640) - 1
    p1 = W.config1()
    calls = [(p1.m, p1.k, p1.n, p1.A, p1.B),
             (m2, k2, n2, PK.from_ints(Ai), PK.from_ints(Bi))]
    # the no-allocation entry point first, so it also runs from a fresh state
    got = [_noalloc(*c) for c in calls]
    for (m, k, n, A, B), g in zip(calls, got):
        want = api.matmul(m, k, n, A, B)
        assert g.to_ints() == want.to_ints()
        assert PK.digest(g) == PK.digest(want)


def test_noalloc_rejects_oversize(product_lib):
    """Beyond the static scratch: a clear MPZMM_ERR_TOO_LARGE, nothing run."""
    A = PK.from_ints([(1 << 40000) - 1] * 16 * 16)
    B = PK.from_ints([(1 << 40000) - 3] * 16 * 16)
    with pytest.raises(_lib.MpzmmError) as e:
        _noalloc(16, 16, 16, A, B)
    assert e.value.status == _lib.MPZMM_ERR_TOO_LARGE
    assert "scratch" in str(e.value) or "limit" in str(e.value)


def _noalloc_raw(m, k, n, A: PK.Packed, B: PK.Packed, cap_delta=0, capture=False):
    """One call with explicit capacities (the bound plus cap_delta); returns
    (status, result sizes on the device after the call).  capture: the call
    is made on a side stream while it captures a CUDA graph."""
    import torch
    L = _lib.lib()
    cap = api.output_limbs(k, 64 * A.max_limbs(), 64 * B.max_limbs()) + cap_delta
    dev = torch.device("cuda", 0)
    d_a = torch.from_numpy(np.ascontiguousarray(A.limbs, dtype=np.uint64).view(np.int64)).to(dev)
    d_b = torch.from_numpy(np.ascontiguousarray(B.limbs, dtype=np.uint64).view(np.int64)).to(dev)
    d_c = torch.zeros(m * n * max(cap, 1), dtype=torch.int64, device=dev)
    d_sz = torch.full((m * n,), 777, dtype=torch.int32, device=dev)
    c_offs = np.arange(m * n, dtype=np.int64) * max(cap, 1)
    c_caps = np.full(m * n, cap, dtype=np.int64)
    a_offs = np.ascontiguousarray(A.offs, dtype=np.int64)
    a_sz = np.ascontiguousarray(A.sizes, dtype=np.int32)
    b_offs = np.ascontiguousarray(B.offs, dtype=np.int64)
    b_sz = np.ascontiguousarray(B.sizes, dtype=np.int32)
    def call(stream):
        return L.mpzmm_matmul_noalloc(
            m, k, n, C.c_void_p(d_a.data_ptr()), a_offs.ctypes.data_as(_lib.i64p),
            a_sz.ctypes.data_as(_lib.i32p), C.c_void_p(d_b.data_ptr()),
            b_offs.ctypes.data_as(_lib.i64p), b_sz.ctypes.data_as(_lib.i32p),
            C.c_void_p(d_c.data_ptr()), c_offs.ctypes.data_as(_lib.i64p),
            c_caps.ctypes.data_as(_lib.i64p), C.c_void_p(d_sz.data_ptr()),
            C.c_void_p(stream.cuda_stream))

    if capture:
        side = torch.cuda.Stream(dev)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=side, capture_error_mode="relaxed"):
            st = call(side)
        del graph
    else:
        st = call(torch.cuda.current_stream(dev))
    torch.cuda.synchronize(dev)
    return st, d_sz.cpu().numpy().tolist()


def test_noalloc_rejects_long_transform_untouched(product_lib):
    """Few entries but a transform above 2^15 points: refused with
    MPZMM_ERR_TOO_LARGE, and the caller's result sizes are left as they were."""
    A = PK.from_ints([(1 << (1 << 22)) - 5])
    B = PK.from_ints([-((1 << (1 << 22)) - 7)])
    st, sizes = _noalloc_raw(1, 1, 1, A, B)
    assert st == _lib.MPZMM_ERR_TOO_LARGE
    msg = _lib.lib().mpzmm_last_error().decode()
    assert "2^15" in msg or "too large" in msg
    assert sizes == [777]


def test_noalloc_rejects_short_capacity_untouched(product_lib):
    """One limb short of the stated capacity: MPZMM_ERR_CAPACITY, nothing run."""
    A = PK.from_ints([(1 << 1000) + 1, 3, -5, 7])
    B = PK.from_ints([2, (1 << 900) - 1, 11, -(1 << 70)])
    st, sizes = _noalloc_raw(2, 2, 2, A, B, cap_delta=-1)
    assert st == _lib.MPZMM_ERR_CAPACITY
    assert sizes == [777] * 4
    # and with the stated capacity the same call succeeds
    st, sizes = _noalloc_raw(2, 2, 2, A, B)
    assert st == _lib.MPZMM_OK
    assert sizes != [777] * 4


def test_noalloc_refuses_a_capturing_stream(product_lib):
    """Its descriptors come from a host buffer the next call overwrites, so a
    call captured into a CUDA graph would replay stale ones: refused with
    MPZMM_ERR_ARG while the stream captures, nothing touched; the same call
    outside the capture succeeds."""
    A = PK.from_ints([(1 << 300) + 9, -17])
    B = PK.from_ints([5, (1 << 200) - 1])
    st, sizes = _noalloc_raw(1, 2, 1, A, B, capture=True)
    assert st == _lib.MPZMM_ERR_ARG
    assert "captur" in _lib.lib().mpzmm_last_error().decode()
    assert sizes == [777]
    st, sizes = _noalloc_raw(1, 2, 1, A, B)
    assert st == _lib.MPZMM_OK
    assert sizes != [777]
