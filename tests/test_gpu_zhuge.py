"""A square whose transform has more than 2^31 points (600,000,000-limb
operand: N = 35 * 2^26 = 2.35e9), checked by residues modulo three primes
computed on the GPU.  Global offsets of the pass kernels are 64-bit, so every
product whose buffers fit the GPU's memory runs (the reference accepts up to
315 * 2^34 points, src/fpntt.jl:936-951).  The file sorts after the other GPU
tests: the product holds about 90 GB while it runs."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

QS = (2147483629, 2147483587, 1000000007)  # primes below 2^31


def _mod_q(x, q: int, chunk: int = 1 << 24) -> int:
    """x (a uint64 limb tensor on the GPU) mod q, from 32-bit halves times their
    weights 2^(32 j) mod q (every product below 2^63)."""
    v = x.view(torch.int64)
    wl = torch.empty(2 * chunk, dtype=torch.int64, device=v.device)
    wl[0] = 1
    k = 1
    while k < 2 * chunk:
        wl[k: 2 * k] = (wl[:k] * pow(2, 32 * k, q)) % q
        k *= 2
    total = 0
    for start in range(0, v.numel(), chunk):
        c = v[start: start + chunk]
        halves = torch.stack([c & 0xFFFFFFFF, (c >> 32) & 0xFFFFFFFF], dim=1).reshape(-1)
        s = int(((halves * wl[: halves.numel()]) % q).sum().item()) % q
        total = (total + s * pow(2, 64 * start, q)) % q
    return total


def test_residue_helper_on_small_values():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(61)
    a = rng.integers(0, 2**64, 5000, dtype=np.uint64)
    ta = torch.from_numpy(a).cuda()
    for q in QS:
        assert _mod_q(ta, q, chunk=1 << 10) == O.to_int(a) % q


def test_square_beyond_2_31_points(gpu_lib):
    total = torch.cuda.get_device_properties(0).total_memory
    if total < 150 * 2**30:
        pytest.skip("needs about 100 GB of device memory")
    n = 600_000_000
    bch, N = gpu_lib.ntt_params(64 * n, 64 * n)
    assert N > 2**31
    gen = torch.Generator(device="cuda").manual_seed(62)
    # uniform 64-bit limbs: 62 random bits shifted up (wrapping) plus 2 more
    da = torch.randint(0, 2**62, (n,), dtype=torch.int64, device="cuda", generator=gen) * 4
    da += torch.randint(0, 4, (n,), dtype=torch.int64, device="cuda", generator=gen)
    da[-1] = 12345  # top limb nonzero
    da = da.view(torch.uint64)
    r = torch.empty(2 * n, dtype=torch.uint64, device="cuda")
    gpu_lib.sqr_dev(r, da, n, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert gpu_lib.device_faults() == 0
    for q in QS:
        ra = _mod_q(da, q)
        assert _mod_q(r, q) == ra * ra % q, q
    del da, r
    torch.cuda.empty_cache()
    gpu_lib.trim_plans()
