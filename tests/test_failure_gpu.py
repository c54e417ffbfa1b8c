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

The reference has no error reporting to compare with: it asserts or exits
(alexp616/rforest src/lib/hwmpz.c:69,146).
"""
import random

import pytest

from rforest_b200 import _lib, api, packed as PK

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
