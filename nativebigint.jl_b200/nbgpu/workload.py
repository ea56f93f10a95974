"""Seeded synthetic product workloads (no public dataset is involved).

`gen_workload` draws the mixed batch of independent products that the
benchmark times and the autotuner tunes for: the larger operand's limb count is
log-uniform in [152, 65536], the size ratio (smaller / larger) uniform in
[0.25, 1], 20% of the products are squares, and limbs are uniform random
uint64 from a numpy PCG64 stream with the top limb forced nonzero.  With
`shape` it draws `count` copies of one m x n shape instead (per-class
profiling).
"""
from __future__ import annotations

import math

import numpy as np


def gen_workload(seed: int, count: int, shape: tuple[int, int] | None = None, square: bool = False,
                 lo: int = 152, hi: int = 65536) -> dict:
    """The mixed batch, or `count` copies of `shape` (all squares with `square`).

    Returns m, n, sq (per product), off_a, off_b (offsets into `limbs`),
    limbs (one flat uint64 array: a_k then, for products, b_k), out_off (each
    product's offset in a flat result array) and out_total."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if shape:
        m = np.full(count, shape[0], dtype=np.int64)
        n = np.full(count, shape[1], dtype=np.int64)
        sq = np.full(count, bool(square))
    else:
        m = np.exp(rng.uniform(math.log(lo), math.log(hi), count)).astype(np.int64)
        ratio = rng.uniform(0.25, 1.0, count)
        n = np.maximum(1, np.round(m * ratio).astype(np.int64))
        sq = rng.random(count) < 0.2
    n = np.where(sq, m, n)
    la = m.copy()
    lb = np.where(sq, 0, n)
    sizes = np.stack([la, lb], axis=1).reshape(-1)
    starts = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    off_a = starts[0::2].copy()
    off_b = starts[1::2].copy()
    pos = int(sizes.sum())
    limbs = rng.integers(0, 2**64, pos, dtype=np.uint64, endpoint=False)
    for top in (off_a + la - 1, (off_b + lb - 1)[~sq]):  # top limbs nonzero
        limbs[top] = np.where(limbs[top] == 0, np.uint64(1), limbs[top])
    out_off = np.concatenate([[0], np.cumsum(m + n)[:-1]]).astype(np.int64)
    return dict(m=m, n=n, sq=sq, off_a=off_a, off_b=off_b, limbs=limbs, out_off=out_off,
                out_total=int((m + n).sum()))


def bits_of(limbs: np.ndarray, off: int, ln: int) -> int:
    """Magnitude bits of the ln-limb operand at limbs[off:] (its top limb nonzero)."""
    return 64 * (ln - 1) + int(limbs[off + ln - 1]).bit_length()
