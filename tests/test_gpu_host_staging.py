"""Host-buffer batches (nbg_mul_batch) whose chunks are large enough to be
staged: operands and results in pageable memory go through pinned staging
buffers copied by host threads, page-locked ones by direct DMA, and a batch
may mix both.  Every product equals GMP's; a second call over the same
buffers rewrites every result."""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import rand_limbs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _pairs(rng, count):
    pairs = []
    for k in range(count):
        m = int(rng.integers(2000, 20000))
        if k % 5 == 0:
            pairs.append((rand_limbs(rng, m), None))
        else:
            pairs.append((rand_limbs(rng, m), rand_limbs(rng, int(rng.integers(500, m + 1)))))
    return pairs


def test_pageable_batch_over_staging_threshold(gpu_lib):
    rng = np.random.default_rng(5150)
    pairs = _pairs(rng, 160)  # about 20 MB of operands and 25 MB of results: staged
    got = gpu_lib.mul_batch(pairs)
    for (a, b), g in zip(pairs, got):
        assert np.array_equal(g, O.gmp_sqr(a) if b is None else O.gmp_mul(a, b))


def test_mixed_pinned_and_pageable_buffers(gpu_lib):
    rng = np.random.default_rng(5151)
    pairs = _pairs(rng, 120)
    keep, items, outs = [], [], []
    for k, (a, b) in enumerate(pairs):
        n = a.size if b is None else b.size
        if k % 2:  # page-locked operands and result
            ta = torch.from_numpy(a).pin_memory()
            tb = None if b is None else torch.from_numpy(b).pin_memory()
            tr = torch.zeros(a.size + n, dtype=torch.uint64).pin_memory()
            keep.append((ta, tb, tr))
            pa, pb, pr = ta.data_ptr(), None if tb is None else tb.data_ptr(), tr.data_ptr()
            outs.append(tr.numpy())
        else:  # pageable
            r = np.zeros(a.size + n, dtype=np.uint64)
            keep.append((a, b, r))
            pa, pb, pr = a.ctypes.data, None if b is None else b.ctypes.data, r.ctypes.data
            outs.append(r)
        items.append((pr, pa, pb, a.size, n, 0, 0))
    descs = gpu_lib.make_descs(items)
    for _ in range(2):
        for r in outs:
            r[:] = 0
        gpu_lib._check(gpu_lib.lib().nbg_mul_batch(ctypes.cast(descs, ctypes.c_void_p), len(items)))
        for (a, b), r in zip(pairs, outs):
            assert np.array_equal(r, O.gmp_sqr(a) if b is None else O.gmp_mul(a, b))
