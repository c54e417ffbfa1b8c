"""The replica (N>1) host logic with gloo ranks on the CPU: per-rank seeds
give independent batches, the timing reduction takes the slowest rank, and
the whole-job rate counts every rank's units."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from rforest_b200 import packed as PK, replicas, workloads as W


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist = replicas.init("gloo", rank, world, timeout_s=60)
    rep = replicas.replicate_of(rank)
    prods = W.config3(rep, count=3)
    digest = PK.digest(prods[0].A)
    elapsed = 10.0 * (rank + 1)  # a made-up per-rank time
    mx = replicas.max_over_ranks(elapsed)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, rep, digest, mx))


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get() for _ in range(world))
    assert [r[1] for r in res] == [1, 2]          # distinct replicates
    assert res[0][2] != res[1][2]                 # hence distinct batches
    assert all(r[3] == 20.0 for r in res)         # max over ranks everywhere
    assert replicas.whole_job_rate(4096, 2, 10, 20.0) == pytest.approx(4096 * 2 * 10 / 0.02)
