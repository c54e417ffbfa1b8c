"""Serving-shaped products (config 5) bit-exact on the GPU against the
reference's own outputs.

The first 256 config-5 requests -- m, k, n uniform in 2..32, entry bit
lengths log-uniform in [2^8, 2^20], signed -- were multiplied by the
reference's unmodified CPU mpz_rmatrix_mult_fft (alexp616/rforest
src/lib/hwmpz.c:65-130) when the golden fixtures were made
(tests/golden/make_golden.py, make_config5); digests.json holds the SHA-256
of every result.  These are the widest shapes (k up to 32) and the longest
transforms the server sees, so each result is checked three ways: through the
plain entry point, through the server with every request queued at once, and
through the server with requests arriving while earlier batches run.
"""
import random
import threading
import time

import pytest

from rforest_b200 import api, packed as PK, workloads as W
from tests import golden_io as G

pytestmark = pytest.mark.gpu

COUNT = 256


@pytest.fixture(scope="module")
def config5():
    want = G.digests()["config5"]
    assert want["count"] >= COUNT
    reqs = [W.config5_request(1, t) for t in range(COUNT)]
    for t, p in enumerate(reqs):
        assert [p.m, p.k, p.n, p.bits] == want["shapes"][t]  # the generator is pinned
    return reqs, want["C"][:COUNT]


def test_config5_plain_matches_reference(gpu, config5):
    reqs, want = config5
    bad = [t for t, p in enumerate(reqs)
           if PK.digest(api.matmul(p.m, p.k, p.n, p.A, p.B)) != want[t]]
    assert not bad, f"requests differing from the reference: {bad[:10]}"


def test_config5_server_all_queued(gpu, config5):
    reqs, want = config5
    srv = api.Server(slots=3, max_batch=32)
    try:
        tickets = [srv.submit(p.m, p.k, p.n, p.A, p.B) for p in reqs]
        got = []
        for t in tickets:
            got.append(PK.digest(srv.wait(t, 600000)))
            srv.release(t)
        st = srv.stats()
    finally:
        srv.close()
    bad = [t for t in range(COUNT) if got[t] != want[t]]
    assert not bad, f"served results differing from the reference: {bad[:10]}"
    assert st["products"] >= COUNT
    assert st["batches"] < COUNT  # requests were batched together


def test_config5_server_concurrent_arrivals(gpu, config5):
    """Two producer threads submit interleaved halves of the requests with
    random gaps while batches are on the GPU; every result still equals the
    reference's."""
    reqs, want = config5
    srv = api.Server(slots=3, max_batch=16)
    tickets = [None] * COUNT
    lock = threading.Lock()

    def producer(part, seed):
        rng = random.Random(seed)
        for t in range(part, COUNT, 2):
            time.sleep(rng.expovariate(3000.0))
            p = reqs[t]
            with lock:  # the binding's holder map is not thread-safe
                tickets[t] = srv.submit(p.m, p.k, p.n, p.A, p.B)

    try:
        ths = [threading.Thread(target=producer, args=(i, 40 + i)) for i in range(2)]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        got = [PK.digest(srv.wait(t, 600000)) for t in tickets]
        st = srv.stats()
    finally:
        srv.close()
    bad = [t for t in range(COUNT) if got[t] != want[t]]
    assert not bad, f"served results differing from the reference: {bad[:10]}"
    assert st["max_in_flight"] >= 2
