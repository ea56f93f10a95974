#!/usr/bin/env python
"""Batched fp-NTT product throughput on B200.

Workload (one "step"): 10,000 independent products whose larger operand has
log-uniform limb count in [152, 65536], size ratio (smaller/larger) uniform in
[0.25, 1], 20% squarings, limbs uniform random uint64 with the top limb
nonzero, seeded (numpy PCG64).  The whole batch runs as one replay of the
engine's CUDA graph (one work-queue launch per pipeline step); every step's
operands (~0.7 GB) and workspace (~9 GB) are far larger than the 126 MB L2.

Printed JSON line (rank 0):
  value     output limbs/s, batch replay with operands resident in HBM
  e2e       same metric through nbg_mul_batch (host buffers; H2D + D2H inside)
  unbatched the same products issued one per call (nbg_mul_batch_dev, count 1)
  roofline  dominant kernel's algorithmic FP64 instructions / its measured
            duration, against the FP64 issue rate measured in this run
  cpu_baseline  the CPU oracle (restatement of the reference) on the host cores

--impl reference times the reference's CPU algorithm (the oracle port; Julia
is not available on this machine) on the same workload.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "nativebigint.jl_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

METRIC = "batched fp-NTT mul output limbs/s vs unbatched GPU mul, bit-exact; p50/p99 ms"
WORKLOAD = "10,000 mixed products: larger operand log-uniform [152, 65536] limbs, ratio U[0.25,1], 20% squares"


# ---------------------------------------------------------------------------
# workload (the seeded generator lives in the package: nbgpu/workload.py)

from nbgpu.workload import bits_of, gen_workload  # noqa: E402


# ---------------------------------------------------------------------------
# clocks

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU side (oracle = restatement of the reference; test infrastructure)

def cpu_rate(W, idx: list[int], threads: int) -> tuple[float, float]:
    """Runs the oracle on products idx with `threads` host threads; returns
    (output limbs/s, seconds).  ctypes releases the GIL during the C call."""
    import oracle

    L = oracle.lib()
    limbs = W["limbs"]
    # plans first (the oracle's plan cache is filled single-threaded)
    for k in idx:
        ba = bits_of(limbs, W["off_a"][k], W["m"][k])
        bb = ba if W["sq"][k] else bits_of(limbs, W["off_b"][k], W["n"][k])
        _, N = oracle.ntt_params(ba, bb)
        L.orc_plan_get(N, 0)
        L.orc_plan_get(N, 1)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    base = limbs.ctypes.data
    outs = {k: np.empty(int(W["m"][k] + W["n"][k]), dtype=np.uint64) for k in idx}

    def one(k):
        m, n = int(W["m"][k]), int(W["n"][k])
        pa = ctypes.cast(base + 8 * int(W["off_a"][k]), u64p)
        r = outs[k].ctypes.data_as(u64p)
        if W["sq"][k]:
            L.orc_sqr_fpntt2(r, pa, m)
        else:
            pb = ctypes.cast(base + 8 * int(W["off_b"][k]), u64p)
            L.orc_mul_fpntt2(r, pa, m, pb, n)
        return m + n

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        total = sum(ex.map(one, sorted(idx, key=lambda k: -int(W["m"][k] + W["n"][k]))))
    dt = time.perf_counter() - t0
    return total / dt, dt


def gmp_rate(W, idx: list[int], threads: int) -> tuple[float, float]:
    """GMP 6.3 mpn_mul / mpn_sqr (the arithmetic of Julia's BigInt) on the
    same products, `threads` host threads; returns (output limbs/s, seconds)."""
    import oracle

    limbs = W["limbs"]
    oracle.gmp()

    def one(k):
        m, n = int(W["m"][k]), int(W["n"][k])
        a = limbs[W["off_a"][k]: W["off_a"][k] + m]
        if W["sq"][k]:
            oracle.gmp_sqr(a)
        else:
            oracle.gmp_mul(a, limbs[W["off_b"][k]: W["off_b"][k] + n])
        return m + n

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        total = sum(ex.map(one, sorted(idx, key=lambda k: -int(W["m"][k] + W["n"][k]))))
    dt = time.perf_counter() - t0
    return total / dt, dt


def cpu_sample(W, budget_s: float, threads: int) -> tuple[list[int], str]:
    """A bounded prefix of the workload sized for ~budget_s of CPU work."""
    # single-thread cost model: ~4.5e-7 s per output limb for this size mix (oracle, scalar)
    per = 4.5e-7
    tot, idx = 0.0, []
    for k in range(len(W["m"])):
        c = per * float(W["m"][k] + W["n"][k])
        if idx and tot + c > budget_s * threads:
            break
        idx.append(k)
        tot += c
    return idx, f"first {len(idx)} of the {len(W['m'])} products (same seed), {threads} threads"


# ---------------------------------------------------------------------------

def run_reference(args, rank: int, world: int) -> None:
    if rank != 0:
        return
    W = gen_workload(args.seed, args.products)
    threads = os.cpu_count() or 1
    idx, desc = cpu_sample(W, args.cpu_seconds / max(1, args.steps + args.warmup) * 3, threads)
    for _ in range(args.warmup):
        cpu_rate(W, idx[: max(1, len(idx) // 4)], threads)
    rates, times = [], []
    for _ in range(args.steps):
        r, dt = cpu_rate(W, idx, threads)
        rates.append(r)
        times.append(dt)
    value = float(statistics.median(rates))
    out_limbs = int(sum(int(W["m"][k] + W["n"][k]) for k in idx))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "output limbs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "products": args.products, "seed": args.seed,
                   "sample_products": len(idx), "sample_output_limbs": out_limbs},
        "cpu_baseline": {"value": value, "unit": "output limbs/s", "cores": threads, "kind": "port",
                         "sample": desc + "; CPU restatement of src/fpntt.jl (Julia is not installed)"},
        "e2e": {"value": value, "unit": "output limbs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fp64_peak() -> dict:
    path = os.path.join(ROOT, "nativebigint.jl_b200", "lib", "libnbgpu_peak.so")
    L = ctypes.CDLL(path)
    L.nbgpeak_fp64.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    fma, add = ctypes.c_double(), ctypes.c_double()
    import torch

    rc = L.nbgpeak_fp64(torch.cuda.current_device(), ctypes.byref(fma), ctypes.byref(add))
    if rc:
        raise RuntimeError("fp64 peak probe failed")
    return {"dfma_per_s": fma.value, "dadd_per_s": add.value}


def rank_share(W: dict, rank: int, world: int, scaling: str, params) -> list[int]:
    """Products of workload W that this rank runs.  weak: every rank draws its
    own batch (seed + rank), so it runs all of W.  strong: every rank draws the
    same batch and runs its LPT share by reference-schedule cost
    (nbgpu/shard.py); the shares are disjoint and cover the batch, and no
    exchange is needed to agree on them.  `params` is fp_ntt_params."""
    count = len(W["m"])
    if scaling == "weak" or world == 1:
        return list(range(count))
    from nbgpu import shard

    prods = []
    for k in range(count):
        m, n, sq = int(W["m"][k]), int(W["n"][k]), bool(W["sq"][k])
        ba = bits_of(W["limbs"], int(W["off_a"][k]), m)
        bb = ba if sq else bits_of(W["limbs"], int(W["off_b"][k]), n)
        prods.append((ba, bb, sq))
    return shard.shard(prods, rank, world, params)


def hbm_peak() -> tuple[float, str]:
    """HBM copy bandwidth for the byte roofline: MEASURED_PEAKS.json's hbm_gbs
    when that file is present, else the pool's earlier measured fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        v = d.get("hbm_gbs")
        if isinstance(v, dict):
            v = v.get("value")
        if v:
            return float(v), "measured: MEASURED_PEAKS.json hbm_gbs"
    except (OSError, ValueError, AttributeError):
        pass
    return 6650.0, "fallback: 6.65 TB/s (MEASURED_PEAKS.json absent)"


def traffic_from_profiles(kernel: str, point_primes: float):
    """DRAM bytes of `kernel` for one batch: the committed ncu measurement of
    bytes per transform point per prime (profiles/ncu_traffic.json, taken on
    the 105*2^11-point class) times this batch's points x primes."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        bpp = d.get("kernels", {}).get(kernel)
        return None if bpp is None else float(bpp) * point_primes
    except (OSError, ValueError):
        return None


def run_ours(args, rank: int, world: int) -> None:
    import torch
    import torch.distributed as dist

    import nbgpu

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    nbgpu._check(nbgpu.lib().nbg_init(dev))
    stream = torch.cuda.Stream()
    shape = tuple(int(v) for v in args.shape.split(",")) if args.shape else None
    weak = args.scaling == "weak"
    W = gen_workload(args.seed + (rank if weak else 0), args.products, shape, args.square)
    mine = rank_share(W, rank, world, args.scaling, nbgpu.ntt_params)
    count = len(mine)
    limbs = W["limbs"]
    d_in = torch.from_numpy(limbs).to(f"cuda:{dev}")
    d_out = torch.zeros(W["out_total"], dtype=torch.uint64, device=f"cuda:{dev}")
    ib, ob = d_in.data_ptr(), d_out.data_ptr()
    items = []
    point_primes = 0.0  # sum over products of transform length x 2 primes
    for k in mine:
        m, n, sq = int(W["m"][k]), int(W["n"][k]), bool(W["sq"][k])
        ba = bits_of(limbs, int(W["off_a"][k]), m)
        bb = ba if sq else bits_of(limbs, int(W["off_b"][k]), n)
        point_primes += 2.0 * nbgpu.ntt_params(ba, bb)[1]
        items.append((ob + 8 * int(W["out_off"][k]), ib + 8 * int(W["off_a"][k]),
                      None if sq else ib + 8 * int(W["off_b"][k]), m, n, ba, bb))
    descs = nbgpu.make_descs(items)
    torch.cuda.synchronize()
    bt = nbgpu.Batch(descs)
    out_limbs = int(sum(int(W["m"][k] + W["n"][k]) for k in mine))
    s = stream.cuda_stream

    # warm-up
    for _ in range(args.warmup):
        bt.run(s)
    torch.cuda.synchronize()

    # timed region: K replays of the whole batch
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = nbgpu.launch_count()
    with ClockSampler(dev) as clk:
        with torch.cuda.stream(stream):
            evs[0].record(stream)
            for i in range(args.steps):
                bt.run(s)
                evs[i + 1].record(stream)
        torch.cuda.synchronize()
    launches = nbgpu.launch_count() - l0
    if world > 1:
        dist.barrier()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    total_ms = evs[0].elapsed_time(evs[-1])
    t = torch.tensor([total_ms], dtype=torch.float64, device=f"cuda:{dev}")
    units = torch.tensor([float(out_limbs) * args.steps, float(count)], dtype=torch.float64, device=f"cuda:{dev}")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(units, op=dist.ReduceOp.SUM)
    total_ms_max = float(t.item())
    value = float(units[0].item()) / (total_ms_max / 1e3)
    job_products = int(units[1].item())

    # bit-exactness of this run's results: a seeded sample against GMP
    import oracle

    res = d_out.cpu().numpy()
    chk = np.asarray(mine)[np.random.default_rng(5).choice(count, min(args.check, count), replace=False)]
    bad = 0
    for k in chk:
        m, n = int(W["m"][k]), int(W["n"][k])
        a = limbs[W["off_a"][k]: W["off_a"][k] + m]
        want = oracle.gmp_sqr(a) if W["sq"][k] else oracle.gmp_mul(a, limbs[W["off_b"][k]: W["off_b"][k] + n])
        got = res[W["out_off"][k]: W["out_off"][k] + m + n]
        bad += int(not np.array_equal(got, want))
    if bad:
        raise SystemExit(f"bench: {bad} of {len(chk)} checked products differ from GMP")

    line = None
    if rank == 0:
        # per-launch live timing (CUDA events between launches, same stream)
        stats = bt.stats()
        prof = [bt.profile(s) for _ in range(3)]
        avg = [statistics.mean(p[i] for p in prof) for i in range(len(stats))]
        kern = {}
        for st_, ms in zip(stats, avg):
            d = kern.setdefault(st_["kind"], {"ms": 0.0, "ops": 0.0, "bytes": 0.0, "launches": 0})
            d["ms"] += ms
            d["ops"] += st_["alg_ops"]
            d["bytes"] += st_["alg_bytes"]
            d["launches"] += 1
        dom = max(kern, key=lambda k: kern[k]["ms"])
        D = kern[dom]
        peak = fp64_peak()
        hbm_gbs, hbm_src = hbm_peak()
        achieved = D["ops"] / (D["ms"] / 1e3) / 1e12
        pk = peak["dfma_per_s"] / 1e12
        tot_ops = sum(st_["alg_ops"] for st_ in stats)
        roof = {
            "bound": "fp64", "kernel": dom, "achieved": achieved, "peak": pk, "unit": "T FP64 instr/s",
            "frac": achieved / pk, "traffic": traffic_from_profiles(dom, point_primes),
            "per": "one batch: all launches of the kernel in one step (launches are grouped by shared-memory size)",
            "peak_source": "measured: DFMA issue rate of libnbgpu_peak.so in this run (MEASURED_PEAKS.json has no FP64 figure)",
            "alg_ops": D["ops"], "ms": D["ms"], "launches": D["launches"],
            "traffic_source": "profiles/ncu_traffic.json bytes per point per prime x this batch's points",
            "hbm": {"alg_bytes": D["bytes"],
                    "achieved_gbs": D["bytes"] / (D["ms"] / 1e3) / 1e9, "peak_gbs": hbm_gbs,
                    "peak_source": hbm_src},
            "kernels": {k: {"ms_per_step": v["ms"], "share": v["ms"] / sum(x["ms"] for x in kern.values()),
                            "alg_tops": v["ops"] / (v["ms"] / 1e3) / 1e12 if v["ms"] else 0.0}
                        for k, v in kern.items()},
            "batch_alg_tops": tot_ops / (statistics.median(step_ms) / 1e3) / 1e12,
        }

        # unbatched: the same products one call each (device buffers)
        lat = []
        nb = min(args.unbatched, count)
        unbatched = None
        one = (nbgpu.NbgDesc * 1)()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ul = 0
        for i in range(nb if nb > 0 else 0):
            one[0] = descs[i]
            c0 = time.perf_counter()
            nbgpu.mul_batch_dev(one, s)
            lat.append(1e3 * (time.perf_counter() - c0))
            ul += int(W["m"][mine[i]] + W["n"][mine[i]])
        torch.cuda.synchronize()
        un_s = time.perf_counter() - t0
        if nb > 0:
            unbatched = {"value": ul / un_s, "unit": "output limbs/s", "products": nb,
                         "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                         "products_per_s": nb / un_s}

        # e2e: host buffers through nbg_mul_batch (pinned), copies inside the call
        pin_in = torch.from_numpy(limbs).pin_memory()
        pin_out = torch.zeros(W["out_total"], dtype=torch.uint64).pin_memory()
        hib, hob = pin_in.data_ptr(), pin_out.data_ptr()
        hitems = []
        for k in mine:
            m, n, sq = int(W["m"][k]), int(W["n"][k]), bool(W["sq"][k])
            hitems.append((hob + 8 * int(W["out_off"][k]), hib + 8 * int(W["off_a"][k]),
                           None if sq else hib + 8 * int(W["off_b"][k]), m, n, 0, 0))
        hdescs = nbgpu.make_descs(hitems)
        L = nbgpu.lib()
        for _ in range(1):
            nbgpu._check(L.nbg_mul_batch(ctypes.cast(hdescs, ctypes.c_void_p), count))
        e2e_t = []
        for _ in range(max(2, min(args.steps, 5))):
            t0 = time.perf_counter()
            nbgpu._check(L.nbg_mul_batch(ctypes.cast(hdescs, ctypes.c_void_p), count))
            e2e_t.append(time.perf_counter() - t0)
        e2e_val = out_limbs / statistics.median(e2e_t)
        if not np.array_equal(pin_out.numpy(), res):
            raise SystemExit("bench: e2e results differ from the device-resident batch")
        # the same from pageable host buffers (what a Julia Memory{UInt64} is)
        pg_out = np.zeros(W["out_total"], dtype=np.uint64)
        pib, pob = limbs.ctypes.data, pg_out.ctypes.data
        pitems = []
        for k in mine:
            m, n, sq = int(W["m"][k]), int(W["n"][k]), bool(W["sq"][k])
            pitems.append((pob + 8 * int(W["out_off"][k]), pib + 8 * int(W["off_a"][k]),
                           None if sq else pib + 8 * int(W["off_b"][k]), m, n, 0, 0))
        pdescs = nbgpu.make_descs(pitems)
        nbgpu._check(L.nbg_mul_batch(ctypes.cast(pdescs, ctypes.c_void_p), count))
        pg_t = []
        for _ in range(max(2, min(args.steps, 3))):
            t0 = time.perf_counter()
            nbgpu._check(L.nbg_mul_batch(ctypes.cast(pdescs, ctypes.c_void_p), count))
            pg_t.append(time.perf_counter() - t0)
        if not np.array_equal(pg_out, res):
            raise SystemExit("bench: pageable e2e results differ from the device-resident batch")
        e2e_pageable = {"value": out_limbs / statistics.median(pg_t), "unit": "output limbs/s",
                        "h2d_bytes_per_step": int(8 * len(limbs)), "d2h_bytes_per_step": int(8 * out_limbs),
                        "buffers": "pageable numpy arrays through nbg_mul_batch"}

        # CPU baseline on a bounded sample
        threads = os.cpu_count() or 1
        cpu_base = None
        if args.cpu_seconds > 0:
            idx, desc = cpu_sample(W, args.cpu_seconds, threads)
            cpu_v, _ = cpu_rate(W, idx, threads)
            gmp_v, _ = gmp_rate(W, idx, threads)
            cpu_base = {"value": cpu_v, "unit": "output limbs/s", "cores": threads, "kind": "port",
                        "sample": desc + "; CPU restatement of src/fpntt.jl (Julia is not installed)",
                        "gmp": {"value": gmp_v, "unit": "output limbs/s", "cores": threads,
                                "sample": "the same products through GMP 6.3 mpn_mul / mpn_sqr"}}

        single_2p24 = None
        if args.single_2p24:
            single_2p24 = single_case(24, True, "uniform", max(20, args.steps), peak["dfma_per_s"], stream,
                                      check="residues")
        clocks = clk.summary()
        med = statistics.median(step_ms)
        line = {
            "metric": METRIC, "value": value, "unit": "output limbs/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms_max / args.steps, "higher_is_better": True,
            "scaling": args.scaling, "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "products": job_products, "products_per_rank": count,
                       "seed": args.seed,
                       "output_limbs_per_step": out_limbs, "l2": "inputs larger than L2 (0.7 GB operands, 9 GB workspace)",
                       "parallelism": (f"{world} ranks, each its own seeded batch (seed + rank), no collective"
                                       if args.scaling == "weak" else
                                       f"one batch split by LPT cost over {world} ranks, no collective")},
            "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
            "products_per_s": job_products / (total_ms_max / args.steps / 1e3),
            "vs_unbatched": value / world / unbatched["value"] if unbatched else None,
            "unbatched": unbatched,
            "bitexact": {"checked_vs_gmp": int(len(chk)), "mismatches": bad},
            "e2e": {"value": e2e_val, "unit": "output limbs/s",
                    "h2d_bytes_per_step": int(8 * len(limbs)), "d2h_bytes_per_step": int(8 * out_limbs)},
            "e2e_pageable": e2e_pageable,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "roofline": roof,
            "cpu_baseline": cpu_base,
            "median_step_ms": med,
            "single_2p24_sqr": single_2p24 if args.single_2p24 else None,
        }
        print(json.dumps(line), flush=True)
    bt.close()


SERVE_WORKLOAD = ("Poisson arrivals of products: larger operand log-uniform [152, 2^20] limbs, ratio U[0.25,1], "
                  "uniform random limbs, device-resident operands and results, 60 GB HBM admission budget")


def run_serve(args) -> None:
    """Serving loop at swept Poisson arrival rates, one JSON line per rate.

    A pool of `serve_pool` products (sizes as SERVE_WORKLOAD) stays resident on
    the device.  Each generation of requests is a fresh random permutation of
    the pool, so each generation writes every pool slot once; the results go to
    one of RING copies of the pool's output area, and before a copy is reused
    every request that wrote it is waited for and the whole copy is compared
    with the GMP products on the device (every result is checked).  Requests
    are submitted by libnbgpu_loadgen.so at their Poisson arrival times, one
    generation per call; between generations the benchmark waits for and checks
    the generation that last used the next ring copy (a stall when the server
    is behind).  Latency is the server's submit-to-completion time;
    `submit_lag` is how far submission fell behind the arrival schedule."""
    import torch

    import nbgpu
    import oracle

    RING = args.serve_ring
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    L = nbgpu.lib()
    nbgpu._check(L.nbg_init(dev))
    rng = np.random.Generator(np.random.PCG64(args.seed))
    P = args.serve_pool
    m = np.exp(rng.uniform(math.log(152), math.log(1 << 20), P)).astype(np.int64)
    n = np.maximum(1, np.round(m * rng.uniform(0.25, 1.0, P)).astype(np.int64))
    ops = []
    for k in range(P):
        a = rng.integers(0, 2**64, int(m[k]), dtype=np.uint64)
        b = rng.integers(0, 2**64, int(n[k]), dtype=np.uint64)
        a[-1] = a[-1] or np.uint64(1)
        b[-1] = b[-1] or np.uint64(1)
        ops.append((a, b))
    out_off = np.concatenate([[0], np.cumsum(m + n)[:-1]]).astype(np.int64)
    out_total = int((m + n).sum())
    # GMP products of the pool (threads: ctypes releases the GIL)
    gold_h = np.zeros(out_total, dtype=np.uint64)

    def gmp_one(k):
        gold_h[out_off[k]: out_off[k] + m[k] + n[k]] = oracle.gmp_mul(*ops[k])

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        list(ex.map(gmp_one, sorted(range(P), key=lambda k: -int(m[k] + n[k]))))
    gold = torch.from_numpy(gold_h).cuda()
    d_ops = [(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda()) for a, b in ops]
    ring = [torch.zeros(out_total, dtype=torch.uint64, device="cuda") for _ in range(RING)]
    # per-slot boundaries for the per-product mismatch count
    bounds = torch.from_numpy(np.concatenate([out_off, [out_total]])).cuda()
    descs = []
    for c in range(RING):
        row = (nbgpu.NbgDesc * P)()
        for k in range(P):
            da, db = d_ops[k]
            row[k] = nbgpu.NbgDesc(ring[c].data_ptr() + 8 * int(out_off[k]), da.data_ptr(), db.data_ptr(),
                                   int(m[k]), int(n[k]), oracle.magnitude_bits(ops[k][0]),
                                   oracle.magnitude_bits(ops[k][1]))
        descs.append(row)
    torch.cuda.synchronize()
    # capacity reference: the whole pool as one batch (graph replay), same products
    bt = nbgpu.Batch(descs[0])
    s0 = torch.cuda.current_stream()
    for _ in range(2):
        bt.run(s0.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s0)
    for _ in range(5):
        bt.run(s0.cuda_stream)
    e1.record(s0)
    torch.cuda.synchronize()
    pool_batch_rate = out_total * 5 / (e0.elapsed_time(e1) / 1e3)
    bt.close()

    def check_copy(c: int, slots) -> int:
        """Products among `slots` in ring copy c that differ from GMP."""
        bad = (ring[c] != gold).to(torch.int64).cumsum(0)
        bad = torch.cat([torch.zeros(1, dtype=torch.int64, device="cuda"), bad])
        per = bad[bounds[1:]] - bad[bounds[:-1]]
        idx = torch.as_tensor(np.asarray(slots, dtype=np.int64), device="cuda")
        return int((per[idx] != 0).sum().item())

    lg = ctypes.CDLL(os.path.join(ROOT, "nativebigint.jl_b200", "lib", "libnbgpu_loadgen.so"))
    lg.nbg_loadgen_now.restype = ctypes.c_double
    lg.nbg_loadgen_submit.restype = ctypes.c_int
    lg.nbg_loadgen_submit.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int64, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.POINTER(ctypes.c_int64)]
    rates = [float(x) for x in args.serve_rates.split(",") if x]
    for rate in rates:
        srv = nbgpu.Server(hbm_budget_bytes=int(args.serve_budget_gb * (1 << 30)), max_hold_us=args.serve_hold_us)
        h = srv._h
        arrivals = np.cumsum(rng.exponential(1.0 / rate, int(rate * args.serve_seconds * 1.05) + 16))
        arrivals = arrivals[arrivals < args.serve_seconds][: args.serve_max_requests]
        count = len(arrivals)
        ngen = (count + P - 1) // P
        tickets = np.zeros(count, dtype=np.int64)
        lags = np.zeros(count, dtype=np.float64)
        slots = np.zeros(count, dtype=np.int32)
        mismatches, stalls, stall_s = 0, 0, 0.0
        submitted_limbs = 0
        for c in range(RING):
            ring[c].zero_()
        torch.cuda.synchronize()
        done = ctypes.c_int64()
        t_start = lg.nbg_loadgen_now() + 0.002

        def retire_gen(g: int) -> int:
            """Waits for generation g, checks its ring copy against GMP, clears it."""
            lo, hi = g * P, min((g + 1) * P, count)
            for t in tickets[lo:hi]:
                nbgpu._check(L.nbg_wait(h, int(t), 600_000_000))
                L.nbg_release(h, int(t))
            bad = check_copy(g % RING, slots[lo:hi])
            ring[g % RING].zero_()
            torch.cuda.current_stream().synchronize()
            return bad

        for g in range(ngen):
            lo, hi = g * P, min((g + 1) * P, count)
            if g >= RING:  # ring copy g % RING is reused: its previous generation must be done and checked
                ts = time.perf_counter()
                first = ctypes.c_int32()
                L.nbg_poll(h, int(tickets[(g - RING + 1) * P - 1]), ctypes.byref(first))
                stalls += int(not first.value)
                mismatches += retire_gen(g - RING)
                stall_s += time.perf_counter() - ts
            slots[lo:hi] = rng.permutation(P)[: hi - lo]
            rc = lg.nbg_loadgen_submit(h, ctypes.cast(descs[g % RING], ctypes.c_void_p),
                                       slots[lo:].ctypes.data, arrivals[lo:].ctypes.data, hi - lo, t_start,
                                       tickets[lo:].ctypes.data, lags[lo:].ctypes.data, ctypes.byref(done))
            nbgpu._check(rc)
            submitted_limbs += int((m[slots[lo:hi]] + n[slots[lo:hi]]).sum())
        t_sub = lg.nbg_loadgen_now() - t_start
        for g in range(max(0, ngen - RING), ngen):
            mismatches += retire_gen(g)
        t_all = lg.nbg_loadgen_now() - t_start
        st = srv.stats()
        srv.close()
        line = {
            "metric": "serving: sustained output limbs/s and submit-to-completion latency", "impl": "ours",
            "mode": "serve", "unit": "output limbs/s", "value": st["output_limbs_per_s"],
            "offered_rate": rate, "submitted_rate": count / t_sub if t_sub > 0 else None,
            "requests": count, "window_s": float(arrivals[-1]) if count else 0.0,
            "completed": st["completed"], "failed": st["failed"],
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "submit_lag_p50_ms": float(np.percentile(lags, 50) / 1e3) if count else None,
            "submit_lag_p99_ms": float(np.percentile(lags, 99) / 1e3) if count else None,
            "wall_s": t_all, "output_limbs": submitted_limbs,
            "ring_stalls": stalls, "ring_stall_s": stall_s,
            "batches": st["batches"], "mean_batch_requests": st["mean_batch_requests"],
            "pool_as_one_batch": {"value": pool_batch_rate, "unit": "output limbs/s"},
            "bitexact": {"checked_vs_gmp": count, "mismatches": mismatches},
            "dtype": "f64", "data": "synthetic", "n_gpus": 1,
            "config": {"workload": SERVE_WORKLOAD, "pool_products": P, "pool_output_limbs": out_total,
                       "hbm_budget_gb": args.serve_budget_gb, "seconds": args.serve_seconds, "seed": args.seed,
                       "max_hold_us": args.serve_hold_us, "ring_copies": RING,
                       "submitter": "libnbgpu_loadgen.so (native open-loop submission at the arrival times)"},
        }
        print(json.dumps(line), flush=True)
        if mismatches or st["failed"]:
            raise SystemExit(f"serve: {mismatches} mismatches, {st['failed']} failed at rate {rate}")


POWMOD_WORKLOAD = ("Barrett powermod chains: 256-limb odd and even moduli (alternating), 256-limb bases, "
                   "4096-bit exponents, uniform random limbs")


def run_powmod(args) -> None:
    """Chains of b^e mod m run side by side: each exponent step is one square or
    multiply per chain plus the two Barrett products, batched across chains.
    One bench step = one nbg_powermod_batch_dev call over all chains (device
    buffers); e2e = the same through nbg_powermod_batch with host buffers."""
    import torch

    import nbgpu
    import oracle

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    nbgpu._check(nbgpu.lib().nbg_init(dev))
    rng = np.random.Generator(np.random.PCG64(args.seed))
    n, k, le = args.powmod_chains, 256, max(1, args.powmod_ebits // 64)
    mods, bases, exps = [], [], []
    for i in range(n):
        m = rng.integers(0, 2**64, k, dtype=np.uint64)
        m[-1] |= np.uint64(1)
        m[0] = (m[0] | np.uint64(1)) if i % 2 else (m[0] & ~np.uint64(1))
        e = rng.integers(0, 2**64, le, dtype=np.uint64)
        e[-1] |= np.uint64(1 << 63)
        mods.append(m)
        bases.append(rng.integers(0, 2**64, k, dtype=np.uint64))
        exps.append(e)
    dm = [torch.from_numpy(x).cuda() for x in mods]
    db = [torch.from_numpy(x).cuda() for x in bases]
    de = [torch.from_numpy(x).cuda() for x in exps]
    dr = [torch.zeros(k, dtype=torch.uint64, device="cuda") for _ in range(n)]
    d = (nbgpu.PowmodDesc * n)()
    for i in range(n):
        d[i] = nbgpu.PowmodDesc(dr[i].data_ptr(), db[i].data_ptr(), de[i].data_ptr(), dm[i].data_ptr(), k, le)
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        nbgpu.powermod_batch_dev(d, k)
    torch.cuda.synchronize()
    times = []
    l0 = nbgpu.launch_count()
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            nbgpu.powermod_batch_dev(d, k)
            times.append(time.perf_counter() - t0)
    launches = nbgpu.launch_count() - l0
    res = [r.cpu().numpy() for r in dr]
    # e2e: host buffers
    e2e_t = []
    for _ in range(max(1, min(args.steps, 3))):
        t0 = time.perf_counter()
        host_res = nbgpu.powermod_batch(bases, exps, mods)
        e2e_t.append(time.perf_counter() - t0)
    mism = sum(int(not np.array_equal(a, b)) for a, b in zip(res, host_res))
    # bit-exactness: a seeded sample against integer pow
    chk = np.random.default_rng(5).choice(n, min(args.check, n), replace=False)
    for i in chk:
        want = pow(oracle.to_int(bases[i]), oracle.to_int(exps[i]), oracle.to_int(mods[i]))
        mism += int(oracle.to_int(res[i]) != want)
    if mism:
        raise SystemExit(f"powmod bench: {mism} results differ")
    # CPU baseline: the oracle's restatement of powermod_limbs on a sample of chains
    threads = os.cpu_count() or 1
    cpu = None
    if args.cpu_seconds > 0:
        oracle.powmod_barrett(bases[0], exps[0], mods[0])  # plans cached single-threaded
        oracle.powmod_barrett(bases[1], exps[1], mods[1])
        t0 = time.perf_counter()
        one = oracle.powmod_barrett(bases[2], exps[2], mods[2])
        per = time.perf_counter() - t0
        ns = int(max(threads, min(n, args.cpu_seconds * threads / max(per, 1e-3))))
        with cf.ThreadPoolExecutor(max_workers=threads) as ex:
            t0 = time.perf_counter()
            outs = list(ex.map(lambda i: oracle.powmod_barrett(bases[i % n], exps[i % n], mods[i % n]), range(ns)))
            dt = time.perf_counter() - t0
        if any(not np.array_equal(outs[i], res[i % n]) for i in range(ns)) or not np.array_equal(one, res[2]):
            raise SystemExit("powmod bench: CPU oracle differs from the GPU")
        cpu = {"value": ns / dt, "unit": "chains/s", "cores": threads, "kind": "port",
               "sample": f"{ns} chains of the same workload, {threads} threads; CPU restatement of "
                         "src/algorithms.jl powermod_limbs + src/barrett.jl with fp-NTT products"}
    med = statistics.median(times)
    line = {
        "metric": "Barrett powermod chains/s (256 chains, 16384-bit moduli, 4096-bit exponents), bit-exact",
        "mode": "powmod", "impl": "ours", "value": n / med, "unit": "chains/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * med, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": POWMOD_WORKLOAD, "chains": n, "k": k, "exponent_bits": 64 * le, "seed": args.seed,
                   "timing": "wall clock around each synchronous call (setup, all steps, result copy)"},
        "e2e": {"value": n / statistics.median(e2e_t), "unit": "chains/s",
                "h2d_bytes_per_step": int(8 * n * (2 * k + le)), "d2h_bytes_per_step": int(8 * n * k)},
        "gpu_launches": int(launches / max(1, args.steps)),
        "bitexact": {"checked_vs_pow": int(len(chk)), "gpu_host_vs_device_equal": True, "mismatches": 0},
        "cpu_baseline": cpu, "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)


def single_operands(lg: int, kind: str) -> list[np.ndarray]:
    """Two 2^lg-limb operands: uniform, all-ones or 1%-sparse limbs, top limb nonzero."""
    n = 1 << lg
    rng = np.random.Generator(np.random.PCG64(1000 + lg))
    ops = []
    for _ in range(2):
        if kind == "uniform":
            x = rng.integers(0, 2**64, n, dtype=np.uint64)
        elif kind == "ones":
            x = np.full(n, 2**64 - 1, dtype=np.uint64)
        else:
            x = np.zeros(n, dtype=np.uint64)
            idx = rng.choice(n, n // 100, replace=False)
            x[idx] = rng.integers(1, 2**64, idx.size, dtype=np.uint64)
        x[-1] |= np.uint64(1)
        ops.append(x)
    return ops


RESIDUE_MODULI = (2**61 - 1, 2**64 - 59, 2**127 - 1, 10**18 + 9)


def residues_agree(a: np.ndarray, b: np.ndarray | None, r: np.ndarray) -> bool:
    """r == a*b (a^2 when b is None) modulo four fixed moduli: a size-independent
    check for products too large to recompute in the timed run."""
    A = int.from_bytes(a.tobytes(), "little")
    B = A if b is None else int.from_bytes(b.tobytes(), "little")
    R = int.from_bytes(r.tobytes(), "little")
    return all((A % q) * (B % q) % q == R % q for q in RESIDUE_MODULI)


def single_case(lg: int, sq: bool, kind: str, reps: int, peak: float, s, check: str = "gmp",
                gmp_time: bool = False) -> dict:
    """One balanced 2^lg-limb product or square on the plain one-per-call
    device path (nbg_mul_dev / nbg_sqr_dev: plan lookup, job build, launches)
    and as a captured one-product batch (graph replay).  3 warm-up calls, then
    `reps` timed ones, each by CUDA events on stream `s`; SM clocks sampled
    during the graph replays.  Roofline: the reference schedule's FP64
    instructions / p50 time, against `peak` (the DFMA issue rate measured in
    this run) and against 148 SMs x 64 DFMA per clock x the sampled clock.
    check: "gmp" compares with mpn_mul / mpn_sqr, "residues" with four
    residues (see residues_agree)."""
    import torch

    import nbgpu

    n = 1 << lg
    ops = single_operands(lg, kind)
    da, db = (torch.from_numpy(x).cuda() for x in ops)
    r = torch.empty(2 * n, dtype=torch.uint64, device="cuda")
    ba = 64 * (n - 1) + int(ops[0][-1]).bit_length()
    bb = ba if sq else 64 * (n - 1) + int(ops[1][-1]).bit_length()
    descs = nbgpu.make_descs([(r.data_ptr(), da.data_ptr(), None if sq else db.data_ptr(), n, n, ba, bb)])
    torch.cuda.synchronize()

    def call():
        if sq:
            nbgpu.sqr_dev(r, da, n, s)
        else:
            nbgpu.mul_dev(r, da, n, db, n, s)

    def timed(fn):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        out = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            out.append(e0.elapsed_time(e1))
        return out

    t_call = timed(call)
    bt = nbgpu.Batch(descs)
    dev = torch.cuda.current_device()
    with ClockSampler(dev) as clk:
        t_graph = timed(lambda: bt.run(s.cuda_stream))
    alg = sum(x["alg_ops"] for x in bt.stats())
    per_kernel = {}
    prof = [bt.profile(s) for _ in range(3)]
    for st_, ms in zip(bt.stats(), [statistics.mean(p[i] for p in prof) for i in range(len(prof[0]))]):
        d = per_kernel.setdefault(st_["kind"], {"ms": 0.0, "alg_ops": 0.0, "launches": 0})
        d["ms"] += ms
        d["alg_ops"] += st_["alg_ops"]
        d["launches"] += 1
    for d in per_kernel.values():
        d["frac"] = d["alg_ops"] / (d["ms"] / 1e3) / peak if d["ms"] else 0.0
    bt.close()
    got = r.cpu().numpy()
    if check == "gmp":
        import oracle

        want = oracle.gmp_sqr(ops[0]) if sq else oracle.gmp_mul(ops[0], ops[1])
        ok = bool(np.array_equal(got, want))
    else:
        ok = residues_agree(ops[0], None if sq else ops[1], got)
    if not ok:
        raise SystemExit(f"single: 2^{lg} {kind} {'sqr' if sq else 'mul'} result is wrong ({check})")
    gmp_ms = None
    if gmp_time:
        import oracle

        t0 = time.perf_counter()
        oracle.gmp_sqr(ops[0]) if sq else oracle.gmp_mul(ops[0], ops[1])
        gmp_ms = 1e3 * (time.perf_counter() - t0)
    p50g = float(np.percentile(t_graph, 50))
    clocks = clk.summary()
    nominal = 148 * 64 * clocks["sm_mhz"] * 1e6 if clocks.get("sm_mhz") else None
    del da, db, r
    torch.cuda.empty_cache()
    return {
        "op": "sqr" if sq else "mul", "limbs": n, "pattern": kind,
        "per_call_p50_ms": float(np.percentile(t_call, 50)), "per_call_p99_ms": float(np.percentile(t_call, 99)),
        "graph_p50_ms": p50g, "graph_p99_ms": float(np.percentile(t_graph, 99)),
        "output_limbs_per_s": 2 * n / (p50g / 1e3),
        "roofline": {"bound": "fp64", "alg_ops": alg, "achieved": alg / (p50g / 1e3) / 1e12,
                     "peak": peak / 1e12, "unit": "T FP64 instr/s", "frac": alg / (p50g / 1e3) / peak,
                     "peak_source": "measured: DFMA issue rate of libnbgpu_peak.so in this run",
                     "frac_of_nominal": alg / (p50g / 1e3) / nominal if nominal else None,
                     "nominal_source": "148 SMs x 64 DFMA/clock x median sampled SM clock",
                     "kernels": per_kernel},
        "check": {"kind": check, "ok": ok},
        "clocks": clocks,
        "cpu_baseline": None if gmp_ms is None else {"value": gmp_ms, "unit": "ms", "cores": 1,
                                                      "kind": "gmp", "sample": "one call, GMP 6.3 mpn"},
        "reps": reps,
    }


def run_single(args) -> None:
    """Single large products (balanced mul and sqr at --single-sizes, 2^16,
    2^20, 2^24 limbs by default; uniform, all-ones and 1%-sparse limbs), see
    single_case; GMP mpn_mul/mpn_sqr on one host core beside the uniform
    pattern.  One JSON line per case."""
    import torch

    import nbgpu

    torch.cuda.set_device(0)
    nbgpu._check(nbgpu.lib().nbg_init(0))
    peak = fp64_peak()["dfma_per_s"]
    s = torch.cuda.Stream()
    reps = max(20, args.steps)
    lgs = [int(x) for x in args.single_sizes.split(",")]
    kinds = args.single_patterns.split(",")
    opsel = args.single_ops.split(",")
    for lg in lgs:
        for kind in kinds:
            for sq in (False, True):
                if ("sqr" if sq else "mul") not in opsel:
                    continue
                rec = single_case(lg, sq, kind, reps, peak, s, check=args.single_check,
                                  gmp_time=kind == "uniform" and args.single_check == "gmp")
                line = {"mode": "single", "impl": "ours",
                        "metric": "single large product time, bit-exact", "unit": "ms", "higher_is_better": False,
                        **rec, "dtype": "f64", "data": "synthetic", "n_gpus": 1}
                print(json.dumps(line), flush=True)


def run_route(args) -> None:
    """Per-call time of unbalanced products below the reference's NTT admission
    (smaller operand n < 64: its chunked Karatsuba path) on the GPU (nbg_mul,
    host buffers, copies included) against GMP's mpn_mul on one host core, to
    place the routing threshold.  One JSON line with the grid of timings."""
    import nbgpu
    import oracle

    nbgpu._check(nbgpu.lib().nbg_init(0))
    rng = np.random.Generator(np.random.PCG64(args.seed))
    rows = []
    for n in (8, 29, 48, 63):
        for m in (1000, 10000, 100000, 1000000):
            a = rng.integers(0, 2**64, m, dtype=np.uint64)
            b = rng.integers(0, 2**64, n, dtype=np.uint64)
            a[-1] |= np.uint64(1)
            b[-1] |= np.uint64(1)
            want = oracle.gmp_mul(a, b)
            got = nbgpu.mul(a, b)
            if not np.array_equal(got, want):
                raise SystemExit(f"route bench: {m}x{n} differs from GMP")
            reps = max(3, int(2e6 / (m * n ** 0.585)))
            ts = []
            for _ in range(reps):
                t0 = time.perf_counter()
                nbgpu.mul(a, b)
                ts.append(time.perf_counter() - t0)
            tg = []
            for _ in range(reps):
                t0 = time.perf_counter()
                oracle.gmp_mul(a, b)
                tg.append(time.perf_counter() - t0)
            rows.append({"m": m, "n": n, "gpu_us": 1e6 * statistics.median(ts), "gmp_us": 1e6 * statistics.median(tg),
                         "work": m * n ** 0.585})
    print(json.dumps({"mode": "route", "metric": "per-call us, unbalanced products below NTT admission",
                      "rows": rows, "data": "synthetic", "n_gpus": 1}), flush=True)

    # The per-call crossover above the reference's NTT admission: one
    # host-buffer call (pageable numpy buffers, as a Julia Memory is) against
    # GMP on one core, the oracle port on one core, and an estimate of the
    # reference's own CPU engine (GMP's time x the reference's published
    # mul!/mpn_mul ratio at that size).
    import oracle as O

    xrows = []
    for shape in ("balanced", "quarter", "square"):
        for m in (152, 304, 608, 1216, 2432, 4864, 9728, 19456, 65536, 262144, 1048576):
            n = m if shape != "quarter" else max(64, m // 4)
            a = rng.integers(0, 2**64, m, dtype=np.uint64)
            b = rng.integers(0, 2**64, n, dtype=np.uint64)
            a[-1] |= np.uint64(1)
            b[-1] |= np.uint64(1)
            sq = shape == "square"
            gpu = (lambda: nbgpu.sqr(a)) if sq else (lambda: nbgpu.mul(a, b))
            gmpf = (lambda: O.gmp_sqr(a)) if sq else (lambda: O.gmp_mul(a, b))
            port = (lambda: O.sqr(a)) if sq else (lambda: O.mul(a, b))
            if not np.array_equal(gpu(), gmpf()):
                raise SystemExit(f"route bench: {m}x{n} {shape} differs from GMP")
            reps = max(3, min(200, int(3e7 / (m * max(1.0, math.log2(m)) * 20))))

            def med(fn, r):
                ts = []
                for _ in range(r):
                    t0 = time.perf_counter()
                    fn()
                    ts.append(time.perf_counter() - t0)
                return 1e6 * statistics.median(ts)

            g_us, m_us = med(gpu, reps), med(gmpf, reps)
            p_us = med(port, max(1, min(reps, 5)))
            ref_us = m_us * reference_gmp_ratio(64 * (m + n) // 2)
            xrows.append({"shape": shape, "m": m, "n": n, "gpu_us": g_us, "gmp_us": m_us, "port_us": p_us,
                          "reference_estimate_us": ref_us})
    cross = {}
    for shape in ("balanced", "quarter", "square"):
        rs = [r for r in xrows if r["shape"] == shape]
        cross[shape] = next((r["m"] for i, r in enumerate(rs)
                             if all(x["gpu_us"] < x["reference_estimate_us"] for x in rs[i:])), None)
    print(json.dumps({"mode": "route_crossover",
                      "metric": "per-call us from pageable host buffers: GPU nbg_mul/nbg_sqr vs CPU",
                      "rows": xrows, "crossover_m": cross,
                      "reference_estimate": "GMP mpn time x the reference's published mul!/mpn_mul ratio "
                                            "(README.md:142-148, log-interpolated by operand bits)",
                      "data": "synthetic", "n_gpus": 1}), flush=True)


# The reference's published mul!/__gmpn_mul time ratios for balanced operands
# by operand bits (NativeBigInt.jl README.md:142-148).
REFERENCE_GMP_RATIOS = ((10e3, 0.90), (16e3, 0.68), (33e3, 0.52), (49e3, 0.46), (66e3, 0.38), (98e3, 0.35),
                        (131e3, 0.30), (262e3, 0.29), (524e3, 0.25), (2.1e6, 0.27), (16.8e6, 0.25), (268e6, 0.46))


def reference_gmp_ratio(bits: float) -> float:
    """Log-linear interpolation of REFERENCE_GMP_RATIOS (clamped at the ends)."""
    pts = REFERENCE_GMP_RATIOS
    if bits <= pts[0][0]:
        return pts[0][1]
    for (b0, r0), (b1, r1) in zip(pts, pts[1:]):
        if bits <= b1:
            f = (math.log(bits) - math.log(b0)) / (math.log(b1) - math.log(b0))
            return r0 + f * (r1 - r0)
    return pts[-1][1]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--products", type=int, default=10000)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--check", type=int, default=64, help="products verified against GMP after timing")
    ap.add_argument("--unbatched", type=int, default=10000, help="products issued one per call")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--shape", default="", help="m,n: a batch of one product shape instead of the mixed workload")
    ap.add_argument("--square", action="store_true", help="with --shape: squares of m-limb operands")
    ap.add_argument("--powmod", action="store_true", help="Barrett powermod chains (256-limb moduli)")
    ap.add_argument("--route", action="store_true", help="per-call timings of products below NTT admission")
    ap.add_argument("--single", action="store_true", help="single large products at --single-sizes")
    ap.add_argument("--single-sizes", default="16,20,24", help="log2 limb counts")
    ap.add_argument("--single-patterns", default="uniform,ones,sparse")
    ap.add_argument("--single-ops", default="mul,sqr")
    ap.add_argument("--single-check", default="gmp", choices=["gmp", "residues"])
    ap.add_argument("--powmod-chains", type=int, default=256)
    ap.add_argument("--powmod-ebits", type=int, default=4096, help="exponent bits (a multiple of 64)")
    ap.add_argument("--serve", action="store_true", help="serving loop at swept Poisson arrival rates")
    ap.add_argument("--serve-rates", default="1000,5000,20000,50000,200000")
    ap.add_argument("--serve-seconds", type=float, default=1.0)
    ap.add_argument("--serve-pool", type=int, default=600)
    ap.add_argument("--serve-budget-gb", type=float, default=60.0)
    ap.add_argument("--serve-hold-us", type=int, default=0, help="server max_hold_us (0: library default)")
    ap.add_argument("--serve-max-requests", type=int, default=40000, help="cap on requests per rate")
    ap.add_argument("--serve-ring", type=int, default=8, help="copies of the pool's result area")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="weak: each rank runs its own batch; strong: ranks split one batch by cost")
    ap.add_argument("--single-2p24", type=int, default=1,
                    help="1: the default line also times one 2^24-limb square (its FP64 roofline)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.gpus > 1 and world == 1 and "RANK" not in os.environ:
        # one process per GPU: relaunch this command under torchrun
        import socket

        sk = socket.socket()
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
        sk.close()
        cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
               "--master-addr", "127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
        raise SystemExit(subprocess.call(cmd))
    if world > 1 and args.gpus != world:
        raise SystemExit(f"bench: --gpus {args.gpus} but WORLD_SIZE {world}")
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.single:
            if rank == 0:
                run_single(args)
        elif args.route:
            if rank == 0:
                run_route(args)
        elif args.powmod:
            if rank == 0:
                run_powmod(args)
        elif args.serve:
            if rank == 0:
                run_serve(args)
        elif args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
