"""Multi-GPU batch sharding, exercised with world-size-2 gloo ranks on CPU:
every rank derives the same LPT assignment with no exchange, the shards are
disjoint and cover the batch, and loads are balanced.  The cost model equals
the oracle's counted FP64 instructions."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from conftest import rand_limbs
from nbgpu import shard


def _batch(seed=3, count=400):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        m = int(np.exp(rng.uniform(np.log(152), np.log(65536))))
        n = max(1, int(m * rng.uniform(0.25, 1)))
        sq = bool(rng.random() < 0.2)
        out.append((64 * m, 64 * (m if sq else n), sq))
    return out


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prods = _batch()
        mine = shard.shard(prods, rank, world, O.ntt_params)
        got = [None] * world
        dist.all_gather_object(got, mine)
        if rank == 0:
            q.put(got)
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_cover_batch():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    prods = _batch()
    allidx = sorted(i for part in got for i in part)
    assert allidx == list(range(len(prods)))
    assert not set(got[0]) & set(got[1])
    costs = []
    for ba, bb, sq in prods:
        b, N = O.ntt_params(ba, bb)
        costs.append(shard.product_cost(N, sq, -(-ba // b) + -(-bb // b) - 1))
    loads = [sum(costs[i] for i in part) for part in got]
    assert max(loads) - min(loads) <= max(costs)


def test_cost_model_matches_counted_ops():
    rng = np.random.default_rng(8)
    for m, n, sq in ((4096, 4096, True), (3000, 1200, False), (20000, 15000, False), (65536, 65536, True)):
        a = rand_limbs(rng, m)
        b = None if sq else rand_limbs(rng, n)
        ba = O.magnitude_bits(a)
        bb = ba if sq else O.magnitude_bits(b)
        bch, N = O.ntt_params(ba, bb)
        nconv = -(-ba // bch) + -(-bb // bch) - 1
        assert shard.product_cost(N, sq, nconv) == O.op_count_product(a, b)


def _bench_worker(rank, world, port, q):
    # the benchmark's own rank logic (bench.rank_share) under gloo ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        import nbgpu

        W = bench.gen_workload(1, 600)
        strong = bench.rank_share(W, rank, world, "strong", nbgpu.ntt_params)
        weak = bench.rank_share(W, rank, world, "weak", nbgpu.ntt_params)
        got = [None] * world
        dist.all_gather_object(got, (strong, len(weak)))
        if rank == 0:
            q.put(got)
    finally:
        dist.destroy_process_group()


def test_bench_rank_logic_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = [g[0] for g in got]
    assert sorted(i for part in parts for i in part) == list(range(600))  # strong: disjoint cover of one batch
    assert all(g[1] == 600 for g in got)                                # weak: each rank its whole own batch
    assert min(len(p) for p in parts) > 100
