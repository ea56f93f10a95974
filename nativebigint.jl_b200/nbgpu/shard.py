"""Batch sharding across GPUs (one process per GPU, no data-path collective).

Products are independent, so a batch splits by cost: each product's cost is
the FP64 instruction count of the reference schedule for its transform length
(forward transforms per operand, pointwise, reverse, unpack; the per-butterfly
counts of the oracle), and products go longest-first to the least-loaded rank
(LPT).  Every rank computes the same assignment from the same product list,
so no exchange is needed before the launch; results stay with the rank that
computed them.
"""
from __future__ import annotations

import heapq

# FP64 instructions per butterfly, (forward, reverse), by radix
_BFLY = {2: (10, 10), 3: (32, 32), 4: (40, 40), 5: (94, 98), 7: (173, 201)}


def _stages(N: int) -> list[int]:
    k = (N & -N).bit_length() - 1
    m = N >> k
    out = []
    for f in (7, 5, 3, 3):
        if m % f == 0:
            out.append(f)
            m //= f
    out += [4] * (k // 2)
    if k & 1:
        out.append(2)
    return out


def product_cost(N: int, sqr: bool, nconv: int) -> float:
    """Reference-schedule FP64 instructions of one product on length N."""
    st = _stages(N)
    fwd = sum(_BFLY[m][0] * (N // m) for m in st)
    rev = sum(_BFLY[m][1] * (N // m) for m in st)
    nfwd = 1 if sqr else 2
    return 2.0 * (nfwd * fwd + 7 * N + rev) + 28.0 * nconv


def assign(costs: list[float], world: int) -> list[int]:
    """LPT: owner rank of each product (largest first to the least-loaded rank;
    ties broken by rank, so every rank computes the same answer)."""
    owner = [0] * len(costs)
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + costs[i], r))
    return owner


def shard(products: list[tuple[int, int, bool]], rank: int, world: int, params) -> list[int]:
    """Indices of `products` ((bits_a, bits_b, sqr) each) that `rank` runs.
    `params(bits_a, bits_b) -> (b, N)` is the admission rule (fp_ntt_params)."""
    costs = []
    for ba, bb, sq in products:
        b, N = params(ba, ba if sq else bb)
        nconv = -(-ba // b) + -(-(ba if sq else bb) // b) - 1
        costs.append(product_cost(N, sq, nconv))
    own = assign(costs, world)
    return [i for i, r in enumerate(own) if r == rank]
