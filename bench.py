#!/usr/bin/env python
"""Benchmark of the exact big-integer matrix product on B200.

One step = one pass of the whole pipeline (split + forward NTT, contraction,
inverse NTT, CRT + recompose) over one batch of the workload.  Default
workload: 4096 independent products, m,k,n uniform in {2..16}, signed entries
with bit lengths log-uniform in [2^10, 2^18] (seeded synthetic inputs).

  value      products/s with inputs resident in HBM (device-timed, CUDA events)
  e2e        products/s through the public C ABI (mpzmm_matmul_batch) with
             host buffers: host->device copy of the inputs and device->host
             copy of the results inside the timed region
  roofline   the dominant stage: algorithmic bytes / its event-timed duration
  cpu_baseline  the reference's own CPU mpz_rmatrix_mult_fft (oracle/_ref) on
             a bounded sample of the same workload, on this host's cores

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "bit-exact mpz matmuls/s (4096-product batch, m,k,n in 2..16, 2^10..2^18-bit signed)"
UNIT = "products/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["config3", "config2", "config4", "config1",
                                           "config4_small", "config4_mid"],
                    default="config3")
    ap.add_argument("--count", type=int, default=4096, help="products per batch (config3)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample", type=int, default=256,
                    help="products in the CPU-baseline sample")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--no-verify", action="store_true")
    ap.add_argument("--contract", choices=["auto", "cuda", "tc"], default="auto",
                    help="contraction engine of the headline measurement")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the plain one-product-per-call and forced tensor-core lines")
    ap.add_argument("--plain-sample", type=int, default=256,
                    help="products timed one call each for the plain comparison")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving measurement")
    ap.add_argument("--serve-pool", type=int, default=256,
                    help="distinct serving requests (the first config-5 draws), cycled")
    ap.add_argument("--serve-requests", type=int, default=3000,
                    help="requests per open-loop serving run (at most 8 s of arrivals)")
    ap.add_argument("--serve-long", type=int, default=10000,
                    help="requests of the long serving stream at 0.8 of saturation (0: none)")
    ap.add_argument("--profile-step", action="store_true",
                    help="profiling run: build the plan, execute it --warmup times, then one "
                         "execute between cudaProfilerStart and cudaProfilerStop (for ncu "
                         "--profile-from-start off), and exit without a bench line")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def make_workload(name, replicate, count):
    from rforest_b200 import workloads as W
    if name == "config3":
        return W.config3(replicate, count=count)
    if name == "config2":
        return [W.config2(replicate)]
    if name == "config4":
        return [W.config4(replicate)]
    if name == "config4_small":
        return [W.config4(replicate, bits=1 << 16)]
    if name == "config4_mid":
        return [W.config4(replicate, bits=1 << 18)]
    return [W.config1(replicate)]


def workload_config(name, count):
    if name == "config3":
        return {"workload": "batched exact matmul", "products_per_step": count,
                "dims": "m,k,n uniform in {2..16}", "bits": "log-uniform [2^10, 2^18], signed",
                "seed": "3000 + replicate"}
    if name == "config2":
        return {"workload": "single 8x8x8 exact matmul", "products_per_step": 1,
                "bits": "65536, signed", "seed": 2001}
    if name == "config4":
        return {"workload": "single 64x64x64 exact matmul", "products_per_step": 1,
                "bits": "2^20, unsigned", "seed": 4001}
    if name == "config4_small":
        return {"workload": "single 64x64x64 exact matmul (profiling size)",
                "products_per_step": 1, "bits": "2^16, unsigned", "seed": 4001}
    if name == "config4_mid":
        return {"workload": "single 64x64x64 exact matmul (profiling size, over a wave of CTAs)",
                "products_per_step": 1, "bits": "2^18, unsigned", "seed": 4001}
    return {"workload": "single 4x4x4 exact matmul", "products_per_step": 1,
            "bits": "4096, signed", "seed": 1001}


# Algorithmic bytes of the 3-pass model at the reference's own parameters
# (4 primes, 64-bit residues, N = 2^lgN from its GPU parameter choice,
# src/lib/mpnfft.c:664-708):  R = 8 * 4 * N bytes per polynomial.
_REF_PRIMES = [0x3fffc00000000001, 0x3ffdf00000000001, 0x3ffd900000000001,
               0x3ffd500000000001]


def reference_lgN(maxlimbs: int, terms: int) -> int:
    bits = 64 * (2 * maxlimbs + 1)
    bound = 0.4999
    for p in _REF_PRIMES:
        bound *= float(p)
    bound2 = bound / terms
    r = 62 * 4 // 2
    while True:
        points = (bits - 1) // r + 2
        thing = bound2 / ((points + 1) // 2)
        _, e = math.frexp(thing)
        rr = (e - 1) // 2
        if rr == r:
            return max(0, (points - 1).bit_length())
        r = rr


def pass_bytes(prods, out_limbs_per_product):
    """(pass1, pass2, pass3) algorithmic bytes summed over the batch."""
    b1 = b2 = b3 = 0
    for p, lc in zip(prods, out_limbs_per_product):
        la = int(p.A.nlimbs.sum())
        lb = int(p.B.nlimbs.sum())
        maxl = max(p.A.max_limbs(), p.B.max_limbs())
        N = 1 << reference_lgN(maxl, p.k)
        R = 8 * 4 * N
        nin = p.m * p.k + p.k * p.n
        nout = p.m * p.n
        b1 += 8 * (la + lb) + R * nin
        b2 += R * nin + R * nout
        b3 += R * nout + 8 * lc
    return b1, b2, b3


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"mpzmm_clocks_{os.getpid()}.csv")
        self.dev = device_index

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.dev)], stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    rows.append(parts)
                except ValueError:
                    pass
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for nm, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's own CPU path on this host's cores
# ---------------------------------------------------------------------------
def _cpu_worker(args):
    name, replicate, indices = args
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from rforest_b200 import workloads as W
    if name == "config3":
        prods = [W.random_product(3000 + replicate, t, 2, 16, 10, 18) for t in indices]
    else:
        prods = make_workload(name, replicate, 1)
    t0 = time.perf_counter()
    for p in prods:
        O.matmul_reference(p.m, p.k, p.n, p.A, p.B)
    return time.perf_counter() - t0, len(prods)


def sample_indices(name, replicate, sample, count, square):
    """Batch products the CPU baseline times: the first `sample` of the batch,
    or (square) the first `sample` with k == n -- the shapes the reference's
    r x d by d x d API expresses without zero padding."""
    if name != "config3":
        return [0]
    if not square:
        return list(range(min(sample, count)))
    from rforest_b200 import workloads as W
    shapes = W.config3_shapes(replicate, count)
    return [t for t, (m, k, n, bits) in enumerate(shapes) if k == n][:sample]


def cpu_reference_rate(name, replicate, sample, workers, pool=None, square=True, count=4096):
    """Products/s of the reference CPU path on a sample of the batch
    (sample_indices), `workers` processes (the reference is single-threaded)."""
    from oracle import oracle as O
    kind = "reference" if O.reference_available() else None
    if kind is None:
        raise RuntimeError("oracle/_ref is not built")
    idx = sample_indices(name, replicate, sample, count, square)
    n = len(idx)
    chunks = [idx[i::workers] for i in range(min(workers, n))]
    t0 = time.perf_counter()
    if pool is None or len(chunks) == 1:
        res = [_cpu_worker((name, replicate, c)) for c in chunks]
    else:
        res = pool.map(_cpu_worker, [(name, replicate, c) for c in chunks])
    wall = time.perf_counter() - t0
    done = sum(r[1] for r in res)
    return done / wall, len(chunks), done


def cpu_workers():
    n = os.cpu_count() or 1
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        pass
    return max(1, min(n, 64))


# ---------------------------------------------------------------------------
def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    import multiprocessing as mp
    workers = cpu_workers()
    ctx = mp.get_context("spawn")
    sample = args.cpu_sample
    with ctx.Pool(workers) as pool:
        for _ in range(args.warmup):
            cpu_reference_rate(args.workload, 1, min(sample, workers), workers, pool,
                               count=args.count)
        rates = []
        t0 = time.perf_counter()
        done_total = 0
        for _ in range(args.steps):
            rate, used, done = cpu_reference_rate(args.workload, 1, sample, workers, pool,
                                                  count=args.count)
            rates.append(rate)
            done_total += done
        wall = time.perf_counter() - t0
        # informative: the first products of the batch whatever their shape,
        # zero-padded to d = max(k, n) for the reference's API
        padded, _, padded_done = cpu_reference_rate(args.workload, 1, sample, workers, pool,
                                                    square=False, count=args.count)
    value = done_total / wall
    cfg = workload_config(args.workload, args.count)
    sample_note = (f"the first {done_total // max(1, args.steps)} products of the batch with "
                   f"k == n per step (the reference's r x d by d x d API takes them unpadded), "
                   f"{used} worker processes")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * wall / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": dict(cfg, sample_products_per_step=done_total // max(1, args.steps),
                       cpu_note="sample restricted to k == n products, which the reference's "
                                "r x d by d x d API multiplies without zero padding"),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "reference",
                         "sample": sample_note,
                         "padded": {"value": padded, "unit": UNIT,
                                    "sample": f"first {padded_done} products of the batch, "
                                              f"zero-padded to d = max(k, n)"}},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import multiprocessing as mp
    cpu_pool = None
    workers = cpu_workers()
    if rank == 0 and world == 1 and not args.no_cpu:
        # spawn the CPU pool before the first GPU call
        cpu_pool = mp.get_context("spawn").Pool(workers)

    import torch
    import torch.distributed as dist
    from rforest_b200 import api, packed as PK

    from rforest_b200 import replicas
    torch.cuda.set_device(local_rank)
    if world > 1:
        replicas.init("nccl", rank, world, device=torch.device("cuda", local_rank))
    api.setup(local_rank)
    modes = {"auto": 0, "cuda": 1, "tc": 2}
    api.set_contract_mode(modes[args.contract])
    stream = torch.cuda.Stream()
    tuning = api.autotune(stream)

    replicate = replicas.replicate_of(rank)
    prods = make_workload(args.workload, replicate, args.count)
    units_per_rank = len(prods)
    triples = [(p.m, p.k, p.n, p.A, p.B) for p in prods]

    # ---- device-resident throughput ----
    plan = api.Plan(triples, stream=stream)
    info = plan.info(0)
    if args.profile_step:
        for _ in range(args.warmup):
            plan.execute(stream)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        plan.execute(stream)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"profile_step": args.workload, "products": len(triples),
                          "launches_per_execute": info["launches"],
                          "device_bytes": info["device_bytes"]}), flush=True)
        plan.close()
        return
    for _ in range(args.warmup):
        plan.execute(stream)
    stream.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    plan.set_timing(True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        plan.execute(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    plan.set_timing(False)
    ms = ev0.elapsed_time(ev1)
    stage_ms, stage_launches, timed = plan.stage_times()
    if world > 1:
        ms = replicas.max_over_ranks(ms, device=torch.device("cuda", local_rank))
        dist.barrier()
    value = replicas.whole_job_rate(units_per_rank, world, args.steps, ms)

    # the same plan replayed as one CUDA graph per step
    plan.set_graph(True)
    plan.execute(stream)
    ms_graph = device_time_ms(torch, stream, lambda: plan.execute(stream), args.steps)
    value_graph = units_per_rank * args.steps / (ms_graph / 1000.0)

    outs = plan.download(stream)
    out_limbs = [int(np.abs(c.sizes.astype(np.int64)).sum()) for c in outs]
    verified = None
    if not args.no_verify:
        verified = verify(args.workload, replicate, outs)
    plan.close()
    del plan

    # ---- end to end through the C ABI with host buffers ----
    # The caller's operand and result arrays live in pinned host memory from
    # the library (filled once, outside the timed region); every timed call
    # copies the inputs host->device, runs the kernels and copies the results
    # device->host into those arrays, in chunks pipelined over the copy
    # engines and the SMs.
    def time_batch(batch, steps):
        batch.run(stream=stream)  # warm the workspaces and the output pages
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            batch.run(stream=stream)
        torch.cuda.synchronize()
        ms = (time.perf_counter() - t0) * 1000.0
        if world > 1:
            ms = replicas.max_over_ranks(ms, device=torch.device("cuda", local_rank))
        return ms, api.batch_stats()

    e2e_steps = max(1, args.e2e_steps)
    batch = api.Batch(triples, pinned=True)
    e2e_ms, e2e_stats = time_batch(batch, e2e_steps)
    # the last timed step's chunks: planned, queued, copied in, computed and
    # copied out (ms from the call's start), and MB each way
    e2e_timeline = [[round(r[k], 2) for k in ("plan_end", "queue_end", "h2d_begin", "h2d_end",
                                             "kernels_end", "d2h_end")]
                    + [round(r["h2d_bytes"] / 1e6, 1), round(r["d2h_bytes"] / 1e6, 1)]
                    for r in api.batch_timeline()]
    batch.close()
    del batch
    e2e_value = replicas.whole_job_rate(units_per_rank, world, e2e_steps, e2e_ms)
    h2d = int(e2e_stats["h2d_bytes"])
    d2h = int(e2e_stats["d2h_bytes"])
    e2e_pageable = None
    if not args.no_compare:
        batch = api.Batch(triples)  # ordinary (pageable) numpy arrays: staged copies
        pg_ms, pg_stats = time_batch(batch, e2e_steps)
        del batch
        e2e_pageable = {"value": replicas.whole_job_rate(units_per_rank, world, e2e_steps, pg_ms),
                        "unit": UNIT, "host_ms_per_step": {
                            k: round(v, 2) for k, v in pg_stats.items() if k.endswith("_ms")}}

    serving = None
    if rank == 0 and world == 1 and not args.no_serving and args.workload == "config3":
        serving = serving_benchmark(api, args)

    comparisons = None
    if world == 1 and not args.no_compare and args.workload == "config3":
        comparisons = compare_forms(api, torch, stream, triples, args)
        api.set_contract_mode(modes[args.contract])
        comparisons["mod_reduction"] = mod_benchmark(api)
        comparisons["config4"] = config4_benchmark(api, torch, stream)
        comparisons["fixed_b"] = fixed_b_benchmark(api, triples[:512])

    if rank == 0:
        # roofline of the dominant stage (3-pass model, reference parameters)
        b1, b2, b3 = pass_bytes(prods, out_limbs)
        names = ["split_fwd_ntt", "contract", "inv_ntt", "crt_recompose"]
        dom = int(np.argmax(stage_ms))
        if dom == 0:
            alg, t_ms, kern, stage = b1, stage_ms[0], "k_fwd2 (split + forward NTT launches)", "fwd"
        elif dom == 1:
            alg, t_ms, kern, stage = b2, stage_ms[1], "k_contract", "contract"
        else:
            alg, t_ms, kern, stage = (b3, stage_ms[2] + stage_ms[3], "k_inv2+k_crt_mixed",
                                      "inv_crt")
        # DRAM bytes per step of the stage: the committed ncu summary of the
        # same workload (dram__bytes_read.sum + dram__bytes_write.sum per
        # kernel of one step, profiles/dram_traffic_config3.txt)
        traffic, traffic_src = load_traffic(args.workload, args.count, stage)
        peaks = load_peaks()
        per_launch_s = (t_ms / 1000.0) / max(1, timed)
        achieved = alg / per_launch_s / 1e9
        cpu = None
        if cpu_pool is not None:
            rate, used, done = cpu_reference_rate(args.workload, 1, args.cpu_sample, workers,
                                                  cpu_pool, count=args.count)
            prate, _, pdone = cpu_reference_rate(args.workload, 1, args.cpu_sample, workers,
                                                 cpu_pool, square=False, count=args.count)
            cpu = {"value": rate, "unit": UNIT, "cores": used, "kind": "reference",
                   "sample": f"the first {done} products of the batch with k == n (the "
                             f"reference's r x d by d x d API takes them unpadded), reference "
                             f"CPU mpz_rmatrix_mult_fft, {used} worker processes",
                   "padded": {"value": prate, "unit": UNIT,
                              "sample": f"first {pdone} products of the batch, zero-padded "
                                        f"to d = max(k, n)"}}
            cpu_pool.close()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic",
            "config": dict(workload_config(args.workload, args.count),
                           l2="inputs larger than L2 (residues of the batch >> 126 MB)",
                           params_product0=info, device_bytes=info["device_bytes"],
                           e2e_steps=e2e_steps, parallelism=f"replicas x{world}",
                           contract=args.contract,
                           autotune_contract_ms={f"k{k}_mn{mn}": [round(v[0], 4), round(v[1], 4)]
                                                 for (k, mn), v in tuning.items()}),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "host_memory": "pinned (mpzmm_host_alloc)",
                    "chunks": e2e_stats["chunks"],
                    "direct_bytes_per_step": [e2e_stats["h2d_direct_bytes"],
                                              e2e_stats["d2h_direct_bytes"]],
                    "host_ms_per_step": {k: round(v, 2)
                                         for k, v in e2e_stats.items() if k.endswith("_ms")},
                    "pageable": e2e_pageable,
                    "timeline_fields": ["plan_end", "queue_end", "h2d_begin", "h2d_end",
                                        "kernels_end", "d2h_end", "h2d_MB", "d2h_MB"],
                    "timeline": e2e_timeline},
            "gpu_launches": int(sum(stage_launches) * args.steps),
            "value_cuda_graph": value_graph,
            "stages_ms_per_step": {n: round(t / max(1, timed), 4)
                                   for n, t in zip(names, stage_ms)},
            "roofline": {"bound": "hbm", "kernel": kern, "achieved": achieved,
                         "peak": peaks[0], "unit": "GB/s", "frac": achieved / peaks[0],
                         "peak_source": peaks[1], "traffic": traffic,
                         "traffic_note": traffic_src,
                         "alg_bytes_per_step": alg,
                         "alg_note": "3-pass byte model at the reference's parameters "
                                     "(4 primes, u64 residues)"},
            "cpu_baseline": cpu,
            "clocks": clk,
            "verified": verified,
            "comparisons": comparisons,
            "serving": serving,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def device_time_ms(torch, stream, fn, reps):
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def compare_forms(api, torch, stream, triples, args):
    """Batched forms against the plain one-product-per-call CUDA-core form."""
    out = {}
    # batched, tensor-core contraction forced on every eligible product
    api.set_contract_mode(2)
    plan = api.Plan(triples, stream=stream)
    for _ in range(2):
        plan.execute(stream)
    ms = device_time_ms(torch, stream, lambda: plan.execute(stream), max(2, args.steps // 2))
    out["batched_tensor_cores"] = {"value": len(triples) * max(2, args.steps // 2) / (ms / 1e3),
                                   "unit": UNIT, "timing": "device, inputs resident"}
    plan.close()
    # plain: one product per call, CUDA-core contraction
    api.set_contract_mode(1)
    sample = triples[:args.plain_sample]
    plans = [api.Plan([t], stream=stream) for t in sample]
    for pl in plans:
        pl.execute(stream)
    ms = device_time_ms(torch, stream, lambda: [pl.execute(stream) for pl in plans], 1)
    out["plain_one_per_call_resident"] = {
        "value": len(sample) / (ms / 1e3), "unit": UNIT,
        "timing": f"device, one plan execute per product, first {len(sample)} products"}
    for pl in plans:
        pl.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for t in sample:
        api.matmul(*t, stream=stream)
    dt = time.perf_counter() - t0
    out["plain_one_per_call_e2e"] = {
        "value": len(sample) / dt, "unit": UNIT,
        "timing": f"wall clock, mpzmm_matmul per product with host buffers, first {len(sample)}"}
    api.set_contract_mode(0)
    # config-2 chain (16 signed 8x8 matrices of 65536-bit entries, left to
    # right): device-resident chain against one host round trip per step
    from rforest_b200 import packed as PK, workloads as W
    mats = W.config2_chain()
    api.chain([(8, 8, X) for X in mats])  # warm the workspaces
    t0 = time.perf_counter()
    C = api.chain([(8, 8, X) for X in mats])
    t_dev = time.perf_counter() - t0
    t0 = time.perf_counter()
    M = mats[0]
    for X in mats[1:]:
        M = api.matmul(8, 8, 8, M, X).compact()
    t_host = time.perf_counter() - t0
    out["config2_chain"] = {"device_resident_ms": t_dev * 1e3, "host_round_trips_ms": t_host * 1e3,
                            "same_result": PK.digest(C) == PK.digest(M),
                            "timing": "wall clock, 15 products, inputs and result in host memory"}
    return out


def config4_benchmark(api, torch, stream, reps=3):
    """The large dense contraction (config 4: 64x64 by 64x64, unsigned 2^20-bit
    entries) device-resident, per stage, on CUDA cores and on tensor cores;
    each engine's result checked against the reference's golden digest."""
    from rforest_b200 import packed as PK, workloads as W
    p = W.config4()
    want = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "digests.json")) as f:
            want = json.load(f)["config4"]["C"]
    except (OSError, KeyError, ValueError):
        pass
    saved = api.contract_mode()
    names = ["split_fwd_ntt", "contract", "inv_ntt", "crt_recompose"]
    out = {"workload": "64x64 by 64x64, unsigned 2^20-bit entries", "reps": reps}
    try:
        for label, mode in (("cuda_cores", 1), ("tensor_cores", 2)):
            api.set_contract_mode(mode)
            plan = api.Plan([(p.m, p.k, p.n, p.A, p.B)], stream=stream)
            plan.execute(stream)
            plan.set_timing(True)
            for _ in range(reps):
                plan.execute(stream)
            stage_ms, _, timed = plan.stage_times()
            plan.set_timing(False)
            C = plan.download(stream)[0]
            out[label] = {"ms_per_product": round(sum(stage_ms) / max(1, timed), 3),
                          "stages_ms": {n: round(t / max(1, timed), 3)
                                        for n, t in zip(names, stage_ms)},
                          "verified": None if want is None else PK.digest(C) == want}
            out["params"] = plan.info(0)
            plan.close()
    finally:
        api.set_contract_mode(saved)
    return out


def fixed_b_benchmark(api, triples, reps=5):
    """A plan that keeps B's transforms: one execute after new A values
    (upload_a, B's split and transforms skipped) against one after a full
    upload, per stage, device time (CUDA events on the execute stream), and
    the results checked against the ordinary entry point."""
    from rforest_b200 import packed as PK
    plan = api.Plan(triples, fixed_b=True)
    plan.set_timing(True)
    plan.execute()
    plan.stage_times()  # drop the first execute
    out = {}
    names = ("split_fwd_ntt", "contract", "inv_ntt", "crt_recompose")
    for name, up in (("full_upload", plan.upload), ("upload_a", plan.upload_a)):
        for _ in range(reps):
            up()
            plan.execute()
        ms, _, ex = plan.stage_times()
        ex = max(1, ex)
        out[name] = {"stages_ms": {k: round(v / ex, 3) for k, v in zip(names, ms)},
                     "ms": round(sum(ms) / ex, 3)}
    got = [PK.digest(c) for c in plan.download()]
    want = [PK.digest(api.matmul(m, k, n, A, B)) for (m, k, n, A, B) in triples]
    plan.close()
    out["products"] = len(triples)
    out["verified"] = got == want
    out["timing"] = "device, CUDA events per stage, mean of %d executes" % reps
    return out


def mod_benchmark(api):
    """x mod d beside the product (a remainder-tree step): 2048 signed x of
    2^17 bits by one d of 2^16 bits, through mpzmm_mod_batch (host arrays in,
    host arrays out, wall clock), against the reference's own CPU
    mpzfft_mod_mod (one core) on the first 32 x."""
    from rforest_b200 import packed as PK, workloads as W
    dbits, xbits, count = 1 << 16, 1 << 17, 2048
    d = W.random_matrix(7001, 0, 0, 1, 1, dbits, False).entry(0) | (1 << (dbits - 1))
    X = W.random_matrix(7001, 1, 0, count, 1, xbits, True)
    xs = X.to_ints()
    m = api.Mod(d, xbits)
    try:
        R = m.reduce(X)  # warm the workspaces
        reps = 3
        t0 = time.perf_counter()
        for _ in range(reps):
            R = m.reduce(X)
        gpu = count * reps / (time.perf_counter() - t0)
    finally:
        m.close()
    out = {"workload": f"{count} signed x of 2^17 bits mod one d of 2^16 bits",
           "value": gpu, "unit": "reductions/s", "timing": "wall clock, host arrays in and out",
           "checked": R.slice(0, 16).to_ints() == [x % d for x in xs[:16]]}
    try:
        from oracle import oracle as O
        if O.reference_available():
            sample = PK.from_ints(xs[:32])
            t0 = time.perf_counter()
            ref = O.mod_reference(d, sample, xbits)
            out["cpu_reference"] = {"value": 32 / (time.perf_counter() - t0),
                                    "unit": "reductions/s", "cores": 1,
                                    "kind": "reference mpzfft_mod_mod", "sample": "first 32 x"}
            out["matches_reference"] = PK.digest(ref) == PK.digest(R.slice(0, 32))
    except Exception as e:  # the comparison is informative only
        out["cpu_reference"] = {"unavailable": str(e)[:200]}
    return out


def _pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    i = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[i]


def serving_benchmark(api, args):
    """Open-loop serving of config-5 requests (m,k,n uniform in 2..32, entry
    bit lengths log-uniform in [2^8, 2^20], signed) through the continuous-
    batching server: saturation throughput, then Poisson arrivals at 0.5, 0.8
    and 0.95 of it with p50/p99 latency (submit to result in host memory),
    and one long stream.  The requests are the first `serve_pool` of the
    config-5 stream -- the ones whose results the reference computed for the
    golden digests -- cycled to bound host memory; the first served pass of
    the pool is checked against those digests."""
    import threading
    from rforest_b200 import packed as PK, workloads as W
    pool = [W.config5_request(1, t) for t in range(args.serve_pool)]
    trip = [(p.m, p.k, p.n, p.A, p.B) for p in pool]
    out = {"workload": "config-5 requests: m,k,n uniform in {2..32}, bits log-uniform "
                       "[2^8, 2^20], signed", "pool": len(pool)}
    want = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "digests.json")) as f:
            want = json.load(f)["config5"]["C"]
    except (OSError, KeyError, ValueError):
        pass
    # The arrays of every request (inputs, result arrays) are laid out once,
    # two sets per pool entry, outside the timed regions, so both arms time
    # the library, not the allocation of result arrays: a request reuses its
    # set once the set's previous request has completed.
    sets = [[api.holder(*t) for _ in range(2)] for t in trip]
    # plain GPU path: one call per request over the whole pool, no batching;
    # a first pass grows the library's workspace, as the server's warm-up does
    for h in sets:
        api.matmul_holder(h[0])
    t0 = time.perf_counter()
    for h in sets:
        api.matmul_holder(h[0])
    plain = len(trip) / (time.perf_counter() - t0)
    out["plain_one_call_per_request"] = {"value": plain, "unit": "requests/s",
                                         "note": "mpzmm_matmul per request, same pool, "
                                                 "arrays laid out beforehand"}
    slots, max_batch, window = 6, 32, 200
    srv = api.Server(slots=slots, max_batch=max_batch, window_us=window)
    out["server_config"] = {"slots": slots, "max_batch": max_batch, "window_us": window,
                            "budget": "3/4 of free memory"}
    try:
        # first pass: every pool request once, all queued; results checked
        tickets = [srv.submit_holder(h[1]) for h in sets]
        checked = 0
        bad = 0
        for i, t in enumerate(tickets):
            C = srv.wait(t, 600000)
            if want is not None and i < len(want):
                checked += 1
                bad += PK.digest(C) != want[i]
            srv.release(t)
        out["verified"] = {"checked": checked, "mismatches": bad,
                           "against": "reference digests of config-5 requests 0..255"}
        # warm-up: another pass grows every slot's pinned staging and workspace
        tickets = [srv.submit_holder(h[0]) for h in sets]
        for t in tickets:
            srv.wait(t, 600000)
            srv.release(t)
        # saturation: everything queued at once (both sets of each entry)
        st0 = srv.stats()
        nsat = 2 * len(trip)
        t0 = time.perf_counter()
        tickets = [srv.submit_holder(sets[i % len(trip)][i // len(trip)]) for i in range(nsat)]
        for t in tickets:
            srv.wait(t, 600000)
        sat = nsat / (time.perf_counter() - t0)
        for t in tickets:
            srv.release(t)
        st1 = srv.stats()
        out["saturation"] = {"value": sat, "unit": "requests/s", "requests": nsat,
                             "vs_plain": sat / plain,
                             "products_per_batch": nsat / max(1, st1["batches"] - st0["batches"])}

        def stream(lam, R):
            arr = W.poisson_arrivals(1, R, lam)
            tickets = [None] * R
            finished = [False] * R
            npool = len(trip)

            def feeder():
                base = time.perf_counter()
                for i in range(R):
                    delay = base + float(arr[i]) - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                    # the set's previous request (2 pool passes back) must be done
                    if i >= 2 * npool:
                        while not finished[i - 2 * npool]:
                            time.sleep(0.0001)
                    tickets[i] = srv.submit_holder(sets[i % npool][(i // npool) % 2])

            b0 = srv.stats()["batches"]
            ph0 = srv.phase_ms()
            srv.phase_max_ms()  # reset
            th = threading.Thread(target=feeder)
            th.start()
            lat, subs, dones = [], [], []
            for i in range(R):
                while tickets[i] is None:
                    time.sleep(0.0002)
                srv.wait(tickets[i], 600000)
                s0, _, d0 = srv.times(tickets[i])
                lat.append((d0 - s0) / 1e6)
                subs.append(s0)
                dones.append(d0)
                srv.release(tickets[i])
                finished[i] = True
            th.join()
            span = (max(dones) - min(subs)) / 1e9
            t_first = min(subs)
            worst = sorted(range(R), key=lambda i: -lat[i])[:3]
            return {"offered": lam, "requests": R, "throughput": R / span,
                    "p50_ms": _pct(lat, 50), "p99_ms": _pct(lat, 99), "max_ms": max(lat),
                    "slowest": [{"request": i, "pool_entry": i % npool,
                                 "submitted_s": (subs[i] - t_first) / 1e9,
                                 "latency_ms": lat[i]} for i in worst],
                    "unit": "requests/s",
                    "products_per_batch": R / max(1, srv.stats()["batches"] - b0),
                    "phase_ms": {k: round(v - ph0[k], 1) for k, v in srv.phase_ms().items()},
                    "phase_max_ms": {k: round(v, 2) for k, v in srv.phase_max_ms().items()}}

        runs = []
        for frac in (0.5, 0.8, 0.95):
            lam = frac * sat
            R = int(max(256, min(args.serve_requests, lam * 8.0)))
            runs.append(dict(load=frac, **stream(lam, R)))
        out["runs"] = runs
        if args.serve_long > 0:
            out["long_stream"] = dict(load=0.8, **stream(0.8 * sat, args.serve_long))
        out["server"] = srv.stats()
        out["server_phase_ms"] = srv.phase_ms()
    finally:
        srv.close()
    return out


def load_traffic(name, count, stage):
    """DRAM bytes per step of a stage from the committed ncu summary of this
    workload (a JSON object in profiles/dram_traffic_<workload>.txt with the
    capture's command); (None, why) where there is none."""
    path = os.path.join(ROOT, "profiles", f"dram_traffic_{name}.txt")
    try:
        with open(path) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return None, "no ncu DRAM summary committed for this workload"
    if int(d.get("products_per_step", -1)) != count:
        return None, f"ncu DRAM summary is for {d.get('products_per_step')} products a step"
    v = d.get("bytes_per_step", {}).get(stage)
    if v is None:
        return None, f"ncu DRAM summary has no '{stage}' stage"
    return float(v), f"DRAM bytes per step (ncu, {os.path.basename(path)}: {d.get('captured', '')})"


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6.65 TB/s (of fallback)"


def verify(name, replicate, outs):
    """Digest check against the reference's golden outputs where they exist."""
    from rforest_b200 import packed as PK
    path = os.path.join(ROOT, "tests", "golden", "digests.json")
    try:
        with open(path) as f:
            d = json.load(f)
    except OSError:
        return None
    if replicate != 1:
        return None
    if name == "config3" and "config3" in d:
        want = d["config3"]["C"]
        n = min(len(want), len(outs))
        return all(PK.digest(outs[t]) == want[t] for t in range(n))
    key = {"config1": "config1", "config2": "config2", "config4": "config4"}.get(name)
    if key and key in d:
        return PK.digest(outs[0]) == d[key]["C"]
    return None


if __name__ == "__main__":
    main()
