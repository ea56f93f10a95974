"""nbg_mul_dev_noalloc: the product entry point that allocates no GPU memory.

Some callers cannot call cudaMalloc — code running inside a memory arena that
owns the whole device, under an allocator hook that must not recurse, or a
foreign runtime that only lends its input and output buffers — so this entry
point keeps its whole workspace in a fixed device array inside the library.
Its results must equal the regular entry point's bit for bit (products are
exact integers).  The file sorts last so a run that stops at the first
failure has already run every other test; it also passes alone in a fresh
process (the first call on the device does the array's set-up).
"""
import ctypes

import numpy as np
import pytest

from conftest import adversarial, rand_limbs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _st():
    return torch.cuda.current_stream().cuda_stream


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _regular(nbgpu, a, b):
    n = a.size if b is None else b.size
    r = torch.zeros(a.size + n, dtype=torch.uint64, device="cuda")
    if b is None:
        nbgpu.sqr_dev(r, _dev(a), a.size, _st())
    else:
        nbgpu.mul_dev(r, _dev(a), a.size, _dev(b), b.size, _st())
    torch.cuda.synchronize()
    return r.cpu().numpy()


def _noalloc(nbgpu, a, b):
    n = a.size if b is None else b.size
    r = torch.full((a.size + n,), 7, dtype=torch.uint64, device="cuda")  # stale contents must be overwritten
    da = _dev(a)
    db = None if b is None else _dev(b)
    torch.cuda.synchronize()
    nbgpu.mul_dev_noalloc(r, da, a.size, db, n, _st())
    torch.cuda.synchronize()
    return r.cpu().numpy()


def test_noalloc_matches_regular_entry_point(gpu_lib):
    rng = np.random.default_rng(404)
    cases = [
        (rand_limbs(rng, 3000), rand_limbs(rng, 2500)),   # multi-pass product
        (rand_limbs(rng, 3000), rand_limbs(rng, 2600)),   # same length again: cached tables
        (adversarial(rng, 200), adversarial(rng, 150)),   # one-pass product, new length
        (np.full(4096, 2**64 - 1, dtype=np.uint64), None),  # all-ones square
        (rand_limbs(rng, 65536), rand_limbs(rng, 65536)),  # largest bench size, 105*2^11 points
    ]
    for a, b in cases:
        want = _regular(gpu_lib, a, b)
        # two calls in a row on the shared array
        first = _noalloc(gpu_lib, a, b)
        second = _noalloc(gpu_lib, a, b)
        assert np.array_equal(first, want)
        assert np.array_equal(second, want)


def test_noalloc_rejects_oversized_products(gpu_lib):
    rng = np.random.default_rng(405)
    a, b0 = rand_limbs(rng, 2**17), rand_limbs(rng, 2**17)  # 105*2^12 points: about 21 MB of workspace
    r = torch.zeros(2 * a.size, dtype=torch.uint64, device="cuda")
    da, db = _dev(a), _dev(b0)
    torch.cuda.synchronize()
    rc = gpu_lib.lib().nbg_mul_dev_noalloc(r.data_ptr(), da.data_ptr(), a.size, db.data_ptr(), b0.size, _st())
    assert rc == gpu_lib.NBG_ENOMEM
    assert b"scratch" in gpu_lib.lib().nbg_last_error()
    # the array is still usable afterwards
    b = rand_limbs(rng, 500)
    assert np.array_equal(_noalloc(gpu_lib, b, None), _regular(gpu_lib, b, None))
