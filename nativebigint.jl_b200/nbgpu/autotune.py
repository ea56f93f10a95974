"""Autotuner for the pass split of each transform class.

A transform class is (transform length N, square or product).  For each class
present in a workload the tuner enumerates pass splits that fit shared memory
(one pass; a column pass plus the last contiguous pass; two column passes plus
the last pass for large N) and column-tile targets, times each candidate on
the GPU with a batch of that class replayed as a CUDA graph, and keeps the
fastest.  The result is a JSON file keyed by GPU model and library version:

    {"gpu": "NVIDIA B200", "version": "0.4.0", "tuning": {..., "overrides": [...]}}

which the library loads at start-up from <lib dir>/../tuning/<GPU name>.json
(or $NBGPU_TUNING); a file for another GPU or version is ignored.

Run on a GPU:  python -m nbgpu.autotune [--out PATH] [--products 10000]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import time

import numpy as np

from .workload import bits_of, gen_workload
from . import (Batch, NBGError, get_tuning, lib, make_descs, ntt_params, plan_layout, set_tuning, trim_plans,
               _check, version)

SMEM_LIMIT = 220 * 1024
MAX_COLUMN_ROWS = 1024


def _stride(n: int) -> int:
    return ((n + (n >> 4) + 1) + 1) & ~1


def _fits_last(L: int, sqr: bool) -> bool:
    return (2 if sqr else 4) * _stride(L) * 8 <= SMEM_LIMIT


def candidates(N: int, sqr: bool, tile_targets=None) -> list[dict]:
    """Pass splits (last stage of each pass) worth timing for class (N, sqr)."""
    if tile_targets is None:
        # column tiles of at least 16 columns are staged by TMA: G <= 256 rows
        # need a target of 4096 points for that
        tile_targets = (4096,) if N >= 1 << 22 else (2048, 4096, 8192)
    st = plan_layout(N, sqr)["stages"]
    S = len(st)
    out = []
    if _fits_last(N, sqr):
        out.append({"pass_ends": [S - 1]})
    for a in range(1, S):
        if not _fits_last(st[a][1], sqr):
            continue
        g0 = N // st[a - 1][2]
        if g0 <= MAX_COLUMN_ROWS:
            for tt in tile_targets:
                out.append({"pass_ends": [a - 1, S - 1], "tile_target": tt})
        if N >= 1 << 17:
            for b in range(0, a - 1):
                g1 = N // st[b][2]
                g2 = st[b + 1][1] // st[a - 1][2]
                if g1 <= MAX_COLUMN_ROWS and g2 <= MAX_COLUMN_ROWS:
                    for tt in tile_targets:
                        out.append({"pass_ends": [b, a - 1, S - 1], "tile_target": tt})
    return out


def classes_of(shapes) -> dict:
    """Groups (bits_a, bits_b, sqr) products by transform class (N, sqr)."""
    cls: dict = {}
    for ba, bb, sq in shapes:
        _, N = ntt_params(ba, ba if sq else bb)
        cls.setdefault((N, bool(sq)), []).append((ba, bb, sq))
    return cls


def _class_batch(members, target_points: float, torch):
    """Device operands for a batch of one class: the class's products,
    repeated until the batch holds about target_points transform points."""
    ba0, bb0, sq0 = members[0]
    _, N = ntt_params(ba0, ba0 if sq0 else bb0)
    reps = max(1, int(math.ceil(target_points / (N * max(1, len(members))))))
    items, bufs = [], []
    for _ in range(reps):
        for ba, bb, sq in members:
            m = -(-ba // 64)
            n = m if sq else -(-bb // 64)
            a = torch.randint(0, 2**62, (m,), dtype=torch.int64, device="cuda")
            b = None if sq else torch.randint(0, 2**62, (n,), dtype=torch.int64, device="cuda")
            r = torch.empty(m + n, dtype=torch.int64, device="cuda")
            bufs += [a, b, r]
            items.append((r, a, b, m, n, ba, ba if sq else bb))
    return items, bufs


def time_batch(descs, torch, warmup=2, reps=5) -> float:
    bt = Batch(descs)
    try:
        s = torch.cuda.current_stream()
        for _ in range(warmup):
            bt.run(s.cuda_stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            bt.run(s.cuda_stream)
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps
    finally:
        bt.close()


def tune(shapes, base: dict | None = None, target_points: float = 4e7, min_share: float = 0.002,
         log=print) -> dict:
    """Returns a tuning object (the library's JSON) with an override for every
    class holding at least `min_share` of the workload's transform points."""
    import torch

    base = dict(base or json.loads(get_tuning()))
    base["overrides"] = []
    set_tuning(json.dumps(base))
    cls = classes_of(shapes)
    total = sum(N * len(v) for (N, _), v in cls.items())
    chosen = []
    for (N, sq), members in sorted(cls.items(), key=lambda kv: -kv[0][0] * len(kv[1])):
        share = N * len(members) / total
        if share < min_share:
            continue
        items, bufs = _class_batch(members, target_points, torch)
        descs = make_descs(items)
        torch.cuda.synchronize()
        best = None
        default_ms = time_batch(descs, torch)
        for cand in candidates(N, sq):
            ov = dict(cand, N=N, sqr=int(sq))
            trial = dict(base, overrides=chosen + [ov])
            try:
                set_tuning(json.dumps(trial))
                ms = time_batch(descs, torch)
            except NBGError as e:
                log(f"  N={N} sqr={int(sq)} {cand}: rejected ({e})")
                continue
            finally:
                trim_plans()  # candidate plans' tables are not kept
            if best is None or ms < best[0]:
                best = (ms, ov)
        set_tuning(json.dumps(dict(base, overrides=chosen)))
        if best and best[0] < default_ms:
            chosen.append(best[1])
            log(f"N={N:>9} sqr={int(sq)} share={share:.3f}: default {default_ms:.3f} ms -> {best[0]:.3f} ms "
                f"{best[1]['pass_ends']} tt={best[1].get('tile_target')}")
        else:
            log(f"N={N:>9} sqr={int(sq)} share={share:.3f}: default {default_ms:.3f} ms kept")
        del bufs
    out = dict(base, overrides=chosen)
    set_tuning(json.dumps(out))
    return out


def gpu_name(torch) -> str:
    return torch.cuda.get_device_name(torch.cuda.current_device())


def default_path(name: str) -> str:
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    return os.path.join(here, "tuning", name.replace(" ", "_") + ".json")


def main() -> None:
    import torch

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default="")
    ap.add_argument("--products", type=int, default=10000)
    ap.add_argument("--seed", type=int, default=1)
    args = ap.parse_args()

    _check(lib().nbg_init(torch.cuda.current_device()))
    W = gen_workload(args.seed, args.products)
    shapes = []
    for k in range(args.products):
        m, n, sq = int(W["m"][k]), int(W["n"][k]), bool(W["sq"][k])
        ba = bits_of(W["limbs"], int(W["off_a"][k]), m)
        bb = ba if sq else bits_of(W["limbs"], int(W["off_b"][k]), n)
        shapes.append((ba, bb, sq))
    # the single-product sizes of the large-product configuration
    for lg in (16, 20, 24):
        shapes += [(64 << lg, 64 << lg, False), (64 << lg, 64 << lg, True)]
    t0 = time.time()
    tun = tune(shapes)
    name = gpu_name(torch)
    doc = {"gpu": name, "version": version(), "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
           "workload": "bench.py mixed batch (seed %d) + 2^16/2^20/2^24-limb products and squares" % args.seed,
           "seconds": round(time.time() - t0, 1), "tuning": tun}
    out = args.out or default_path(name)
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as f:
        json.dump(doc, f, indent=1)
    print(f"wrote {out}: {len(tun['overrides'])} class overrides")


if __name__ == "__main__":
    main()
