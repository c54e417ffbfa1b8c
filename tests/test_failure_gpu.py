"""Failure paths on the GPU, made without faulting it.

* A bounded device wait that runs out: the tensor-core contraction waits on
  an mbarrier for its MMAs' commit.  With MPZMM_OPT_TEST_STALL_TC set, one
  launch issues neither the MMAs nor the commit -- a flag that nothing sets
  -- so every CTA's wait gives up after its one-second limit with no tensor
  operation outstanding, frees its TMEM and records a status word that the
  host turns into MPZMM_ERR_TIMEOUT.  The context stays usable: the next
  call is bit-exact.
* A host allocation failure: MPZMM_OPT_TEST_FAIL_ALLOC makes the next
  workspace allocation report out-of-memory (MPZMM_ERR_NOMEM) before any
  CUDA allocation is attempted; the next call succeeds.
* The debug bounds check (MPZMM_OPT_CHECK_BOUNDS): a kernel checks every
  descriptor against the workspace before each execute and writes a status
  word (MPZMM_ERR_BOUNDS, nothing else launched).  No test plants a bad
  descriptor on the GPU; the check is shown to pass every entry point.

The reference has no error reporting to compare with: it asserts or exits
(alexp616/rforest src/lib/hwmpz.c:69,146).
"""
import random

import pytest

from rforest_b200 import _lib, api, packed as PK, workloads as W

pytestmark = pytest.mark.gpu


def _product(seed, m, k, n, bits):
    rng = random.Random(seed)
    Ai = [rng.choice([1, -1]) * rng.getrandbits(bits) for _ in range(m * k)]
    Bi = [rng.choice([1, -1]) * rng.getrandbits(bits) for _ in range(k * n)]
    want = [sum(Ai[i * k + l] * Bi[l * n + j] for l in range(k))
            for i in range(m) for j in range(n)]
    return PK.from_ints(Ai), PK.from_ints(Bi), want


def _opt(option, value=None):
    L = _lib.lib()
    if value is not None:
        _lib.check(L.mpzmm_set_option(option, value))
    return L.mpzmm_get_option(option)


def test_tensor_core_wait_times_out_and_recovers(gpu):
    m, k, n = 4, 8, 4
    A, B, want = _product(5, m, k, n, 3000)
    saved = api.contract_mode()
    api.set_contract_mode(2)  # tensor cores wherever the shape allows
    try:
        assert _opt(_lib.MPZMM_OPT_TEST_STALL_TC, 1) == 1
        with pytest.raises(_lib.MpzmmError) as e:
            api.matmul(m, k, n, A, B)
        assert e.value.status == _lib.MPZMM_ERR_TIMEOUT
        assert "timed out" in str(e.value)
        assert _opt(_lib.MPZMM_OPT_TEST_STALL_TC) == 0  # consumed by that launch
        # same context, same shape: exact again
        assert api.matmul(m, k, n, A, B).to_ints() == want
    finally:
        _opt(_lib.MPZMM_OPT_TEST_STALL_TC, 0)
        api.set_contract_mode(saved)
    # and on CUDA cores
    api.set_contract_mode(1)
    try:
        assert api.matmul(m, k, n, A, B).to_ints() == want
    finally:
        api.set_contract_mode(saved)


def test_allocation_failure_reports_and_recovers(gpu):
    A, B, want = _product(9, 3, 3, 3, 5000)
    try:
        assert _opt(_lib.MPZMM_OPT_TEST_FAIL_ALLOC, 1) == 1
        with pytest.raises(_lib.MpzmmError) as e:
            api.Plan([(3, 3, 3, A, B)])  # a plan's own workspace allocates
        assert e.value.status == _lib.MPZMM_ERR_NOMEM
        assert "injected" in str(e.value)
        assert _opt(_lib.MPZMM_OPT_TEST_FAIL_ALLOC) == 0
        plan = api.Plan([(3, 3, 3, A, B)])
        plan.execute()
        assert plan.download()[0].to_ints() == want
        plan.close()
        # a second failure on a later allocation, then the one-shot path
        _opt(_lib.MPZMM_OPT_TEST_FAIL_ALLOC, 2)
        with pytest.raises(_lib.MpzmmError) as e:
            api.Plan([(3, 3, 3, A, B)])
        assert e.value.status == _lib.MPZMM_ERR_NOMEM
    finally:
        _opt(_lib.MPZMM_OPT_TEST_FAIL_ALLOC, 0)
    assert api.matmul(3, 3, 3, A, B).to_ints() == want


def test_debug_bounds_check_passes_every_entry_point(gpu):
    """With the debug bounds check on, every plan execute first checks all
    descriptors against its workspace on the device (a status word, nothing
    else touched); on correct plans it finds nothing, and the results of a
    product, a pipelined batch, a chain and server batches stay exact."""
    L = _lib.lib()
    assert L.mpzmm_set_option(_lib.MPZMM_OPT_CHECK_BOUNDS, 1) == _lib.MPZMM_OK
    try:
        rng = random.Random(99)
        Ai = [rng.randrange(-(1 << 900), 1 << 900) for _ in range(6)]
        Bi = [rng.randrange(-(1 << 700), 1 << 700) for _ in range(12)]
        C = api.matmul(2, 3, 4, PK.from_ints(Ai), PK.from_ints(Bi))
        assert C.to_ints() == [sum(Ai[i * 3 + l] * Bi[l * 4 + j] for l in range(3))
                               for i in range(2) for j in range(4)]
        prods = [W.random_product(41, t, 2, 9, 8, 14) for t in range(24)]
        trip = [(p.m, p.k, p.n, p.A, p.B) for p in prods]
        want = [PK.digest(api.matmul(*t)) for t in trip]
        saved = api.chunk_limbs()
        api.set_chunk_limbs(1 << 12)  # several chunks: the pipelined path
        try:
            assert [PK.digest(c) for c in api.matmul_batch(trip)] == want
        finally:
            api.set_chunk_limbs(saved)
        mats = [W.random_product(43, t, 3, 3, 10, 10) for t in range(4)]
        X = api.chain([(3, 3, p.A) for p in mats])
        M = mats[0].A.to_ints()
        for p in mats[1:]:
            B = p.A.to_ints()
            M = [sum(M[i * 3 + l] * B[l * 3 + j] for l in range(3))
                 for i in range(3) for j in range(3)]
        assert X.to_ints() == M
        srv = api.Server(slots=2, max_batch=8)
        try:
            tickets = [srv.submit(*t) for t in trip]
            assert [PK.digest(srv.wait(t, 60000)) for t in tickets] == want
        finally:
            srv.close()
    finally:
        L.mpzmm_set_option(_lib.MPZMM_OPT_CHECK_BOUNDS, 0)
