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


_FRESH = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, {pkg!r})
import nbgpu

rng = np.random.default_rng(406)
def rl(n):
    a = rng.integers(0, 2**64, n, dtype=np.uint64)
    a[-1] |= np.uint64(1)
    return a
# one-pass product, multi-pass products of two lengths, a square: four transform lengths
shapes = [(rl(700), rl(500)), (rl(3000), rl(2500)), (rl(20000), rl(12000)), (np.full(9000, 2**64 - 1, dtype=np.uint64), None)]
dev = []
for a, b in shapes:
    n = a.size if b is None else b.size
    dev.append((torch.from_numpy(a).cuda(), None if b is None else torch.from_numpy(b).cuda(),
                torch.zeros(a.size + n, dtype=torch.uint64, device="cuda"), a.size, n))
st = torch.cuda.current_stream().cuda_stream
def call(i):
    da, db, r, m, n = dev[i]
    nbgpu.mul_dev_noalloc(r, da, m, db, n, st)
# warm-up: every kernel these shapes use is loaded and has its local memory
for i in range(len(dev)):
    call(i)
torch.cuda.synchronize()
want = [dev[i][2].cpu().numpy().copy() for i in range(len(dev))]
free0, reserved0 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
for order in ([3, 2, 1, 0], [0, 2, 0, 3, 1], [1, 1, 3, 0, 2]):
    for i in order:
        dev[i][2].fill_(7)
        torch.cuda.synchronize()
        call(i)
        torch.cuda.synchronize()
        assert np.array_equal(dev[i][2].cpu().numpy(), want[i]), i
free1, reserved1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()
assert free1 == free0, (free0, free1)
assert reserved1 == reserved0, (reserved0, reserved1)
print("noalloc-fresh-ok", free0 - free1)
"""


def test_noalloc_allocates_nothing_in_a_fresh_process():
    # A process that only ever calls the allocation-free entry point: after one
    # warm-up call per shape, further calls of four transform lengths in
    # changing order leave the device's free memory and torch's reserved
    # memory exactly as they were.
    import os
    import subprocess
    import sys

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from conftest import ROOT

    src = _FRESH.format(pkg=os.path.join(ROOT, "nativebigint.jl_b200"))
    r = subprocess.run([sys.executable, "-c", src], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "noalloc-fresh-ok" in r.stdout
