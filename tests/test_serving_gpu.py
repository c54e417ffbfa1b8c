"""The continuous-batching server and CUDA-graph plans, on the GPU.

Every result is compared bit-exactly with the same product computed alone
(the ordinary entry point) -- the serving tolerance is exact equality.
"""
import random
import threading
import time

import numpy as np
import pytest

from rforest_b200 import _lib, api, packed as PK, workloads as W

pytestmark = pytest.mark.gpu


def small_requests(count, seed=17):
    return [W.random_product(seed, t, 2, 12, 8, 14) for t in range(count)]


def test_server_results_same_alone_and_in_the_mix(gpu):
    reqs = small_requests(40)
    alone = [PK.digest(api.matmul(p.m, p.k, p.n, p.A, p.B)) for p in reqs]
    srv = api.Server(budget_bytes=0, slots=3, max_batch=4)
    try:
        # alone through the server: one request in flight at a time
        for i in (0, 7, 21):
            t = srv.submit(reqs[i].m, reqs[i].k, reqs[i].n, reqs[i].A, reqs[i].B)
            assert PK.digest(srv.wait(t, 60000)) == alone[i]
        # all at once: batched, several batches in flight
        tickets = [srv.submit(p.m, p.k, p.n, p.A, p.B) for p in reqs]
        got = [PK.digest(srv.wait(t, 60000)) for t in tickets]
        assert got == alone
        st = srv.stats()
        assert st["batches"] >= 10          # max_batch 4 -> at least 10 batches for 40
        assert st["max_in_flight"] >= 2     # batches overlapped on the device
        for t in tickets:
            sub, start, done = srv.times(t)
            assert sub <= start <= done
    finally:
        srv.close()


def test_server_poisson_arrivals(gpu):
    reqs = small_requests(60, seed=23)
    alone = [PK.digest(api.matmul(p.m, p.k, p.n, p.A, p.B)) for p in reqs]
    srv = api.Server(slots=3)
    tickets = [None] * len(reqs)
    rng = random.Random(3)

    def feeder():
        for i, p in enumerate(reqs):
            time.sleep(rng.expovariate(2000.0))
            tickets[i] = srv.submit(p.m, p.k, p.n, p.A, p.B)

    th = threading.Thread(target=feeder)
    th.start()
    th.join()
    try:
        got = [PK.digest(srv.wait(t, 60000)) for t in tickets]
        assert got == alone
    finally:
        srv.close()


def test_server_budget_admission(gpu):
    """A budget that holds one request at a time serialises the batches."""
    reqs = small_requests(6, seed=29)
    alone = [PK.digest(api.matmul(p.m, p.k, p.n, p.A, p.B)) for p in reqs]
    biggest = max(reqs, key=lambda p: p.m * p.k * p.n * p.bits)
    srv = api.Server(budget_bytes=64 << 20, slots=3)
    try:
        tickets = [srv.submit(p.m, p.k, p.n, p.A, p.B) for p in reqs]
        assert [PK.digest(srv.wait(t, 60000)) for t in tickets] == alone
    finally:
        srv.close()
    tiny = api.Server(budget_bytes=4096, slots=2)
    try:
        with pytest.raises(_lib.MpzmmError) as e:
            tiny.submit(biggest.m, biggest.k, biggest.n, biggest.A, biggest.B)
        assert e.value.status == _lib.MPZMM_ERR_TOO_LARGE
    finally:
        tiny.close()


def test_plan_graph_replay_with_new_inputs(gpu):
    prods = [W.random_product(31, t, 2, 8, 8, 13) for t in range(8)]
    plan = api.Plan([(p.m, p.k, p.n, p.A, p.B) for p in prods])
    plan.set_graph(True)
    plan.execute()
    plan.execute()
    first = [PK.digest(c) for c in plan.download()]
    assert first == [PK.digest(api.matmul(p.m, p.k, p.n, p.A, p.B)) for p in prods]
    # new values, same sizes and signs: flip bit 0 of every limb array
    for h, p in zip(plan.holders, prods):
        h.al ^= np.uint64(1)
        h.bl ^= np.uint64(1)
    plan.upload()
    plan.execute()  # graph replay on the new inputs
    second = [PK.digest(c) for c in plan.download()]
    want = []
    for h, p in zip(plan.holders, prods):
        A = PK.Packed(h.al, h.ao, h.asz)
        B = PK.Packed(h.bl, h.bo, h.bsz)
        want.append(PK.digest(api.matmul(p.m, p.k, p.n, A, B)))
    assert second == want
    plan.close()


@pytest.mark.parametrize("mode", [1, 2])
def test_plan_keeps_b_transforms(gpu, mode):
    """A plan that keeps B's transforms (the same B times many A), on CUDA
    cores and on tensor cores: after upload_a the products of new A values
    with the kept B are exact, a B changed in host memory is not read by
    upload_a, and a full upload brings it in."""
    api.set_contract_mode(mode)
    try:
        prods = [W.random_product(37, t, 2, 12, 8, 14) for t in range(10)]
        plan = api.Plan([(p.m, p.k, p.n, p.A, p.B) for p in prods], fixed_b=True)

        def want(bls):
            out = []
            for h, p, bl in zip(plan.holders, prods, bls):
                A = PK.Packed(h.al, h.ao, h.asz)
                B = PK.Packed(bl, h.bo, h.bsz)
                out.append(PK.digest(api.matmul(p.m, p.k, p.n, A, B)))
            return out

        kept = [h.bl.copy() for h in plan.holders]
        plan.execute()
        assert [PK.digest(c) for c in plan.download()] == want(kept)
        for rnd in range(2):  # new A values (same sizes and signs), B's transforms kept
            for h in plan.holders:
                h.al ^= np.uint64(1 << rnd)
            plan.upload_a()
            plan.execute()
            assert [PK.digest(c) for c in plan.download()] == want(kept)
        for h in plan.holders:  # B changes in host memory: upload_a leaves it
            h.bl ^= np.uint64(1)
        plan.upload_a()
        plan.execute()
        assert [PK.digest(c) for c in plan.download()] == want(kept)
        plan.upload()  # a full upload reads the new B, transformed at the next execute
        plan.execute()
        plan.execute()
        assert [PK.digest(c) for c in plan.download()] == want([h.bl for h in plan.holders])
        plan.close()
    finally:
        api.set_contract_mode(0)


def test_server_admission_window(gpu):
    """The admission window changes how requests are batched, never the
    results; a negative window is refused."""
    reqs = small_requests(24, seed=41)
    alone = [PK.digest(api.matmul(p.m, p.k, p.n, p.A, p.B)) for p in reqs]
    for window in (0, 2000):
        srv = api.Server(slots=2, max_batch=8, window_us=window)
        try:
            tickets = [srv.submit(p.m, p.k, p.n, p.A, p.B) for p in reqs]
            assert [PK.digest(srv.wait(t, 60000)) for t in tickets] == alone
            with pytest.raises(_lib.MpzmmError) as e:
                srv.set_admission_window(-1)
            assert e.value.status == _lib.MPZMM_ERR_ARG
        finally:
            srv.close()


def test_server_small_and_large_requests_mixed(gpu):
    """Small requests (at most 16 MB of host data) and large ones (a 64 x 64
    by 64 x 64 product of 2^14-bit entries, about 33 MB) queued together:
    they are batched by class and run on streams of two priorities, and every
    result still equals the product computed alone.  The phase maxima reset
    on reading."""
    small = small_requests(24, seed=23)
    big = [W.random_product(31, t, 64, 64, 14, 14) for t in range(2)]
    order = small[:8] + [big[0]] + small[8:16] + [big[1]] + small[16:]
    alone = [PK.digest(api.matmul(p.m, p.k, p.n, p.A, p.B)) for p in order]
    srv = api.Server(budget_bytes=0, slots=3, max_batch=8)
    try:
        tickets = [srv.submit(p.m, p.k, p.n, p.A, p.B) for p in order]
        got = [PK.digest(srv.wait(t, 120000)) for t in tickets]
        assert got == alone
        mx = srv.phase_max_ms()
        assert set(mx) == {"build", "upload", "launch", "download"}
        assert all(v >= 0 for v in mx.values()) and mx["download"] > 0
        assert all(v == 0 for v in srv.phase_max_ms().values())  # reset by the read
        for t in tickets:
            srv.release(t)
    finally:
        srv.close()
