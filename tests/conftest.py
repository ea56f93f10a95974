"""Shared test setup: the `gpu` marker, import paths, seeded operand makers."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "nativebigint.jl_b200"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def rand_limbs(rng: np.random.Generator, n: int, top_nonzero: bool = True) -> np.ndarray:
    a = rng.integers(0, 2**64, n, dtype=np.uint64, endpoint=False)
    if top_nonzero and a[-1] == 0:
        a[-1] = 1
    return a


def adversarial(rng: np.random.Generator, n: int) -> np.ndarray:
    """Magnitude in [2^(64(n-1)), 2^(64n)): uniform, all-ones, or 2^k +- 1
    (the reference's fpntt_randbig, test/test_fpntt.jl:120-131)."""
    style = int(rng.integers(1, 4))
    if style == 1:
        return rand_limbs(rng, n)
    if style == 2:
        return np.full(n, 2**64 - 1, dtype=np.uint64)
    k = int(rng.integers(64 * (n - 1), 64 * n))
    v = (1 << k) + int(rng.integers(-1, 2))
    v = max(v, 1 << (64 * (n - 1))) if n > 1 else max(v, 1)
    return np.frombuffer(v.to_bytes(8 * n, "little"), dtype="<u8").astype(np.uint64)


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library bound to device 0; skips when no GPU is present."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import nbgpu

    nbgpu._check(nbgpu.lib().nbg_init(0))
    return nbgpu
