"""Barrett powermod chains on the GPU (nbg_powermod_batch*): every chain's
result equals b^e mod m (Python's integer pow, GMP-backed like Julia's BigInt
powermod that the reference's tests compare against)."""
import ctypes

import numpy as np
import pytest

import oracle as O
from conftest import rand_limbs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

B = 1 << 64


def _int(a) -> int:
    return O.to_int(np.asarray(a, dtype=np.uint64))


def _check(gpu_lib, bases, exps, mods):
    got = gpu_lib.powermod_batch(bases, exps, mods)
    for r, b, e, m in zip(got, bases, exps, mods):
        assert _int(r) == pow(_int(b), _int(e), _int(m))


@pytest.mark.parametrize("k", [1, 2, 5, 33])
def test_powmod_small_moduli(gpu_lib, k):
    rng = np.random.default_rng(300 + k)
    bases, exps, mods = [], [], []
    for i in range(24):
        m = rand_limbs(rng, k)
        m[0] = (int(m[0]) | 1) if i % 2 else (int(m[0]) & ~1)
        if k == 1:
            m[0] = max(int(m[0]), 2)
        le = int(rng.integers(1, 5))
        e = rand_limbs(rng, le)
        bases.append(rand_limbs(rng, int(rng.integers(1, k + 1))))
        exps.append(e)
        mods.append(m)
    _check(gpu_lib, bases, exps, mods)


def test_powmod_edge_cases(gpu_lib):
    rng = np.random.default_rng(310)
    k = 8
    pow2 = np.zeros(k, dtype=np.uint64)
    pow2[-1] = 1                      # m = β^(k-1): μ has k + 2 limbs
    full = np.full(k, 2**64 - 1, dtype=np.uint64)  # m = β^k − 1
    cases = [
        (rand_limbs(rng, k), np.array([1], dtype=np.uint64), rand_limbs(rng, k)),        # e = 1
        (np.zeros(1, dtype=np.uint64), rand_limbs(rng, 2), rand_limbs(rng, k)),          # b = 0
        (full.copy(), rand_limbs(rng, 3), rand_limbs(rng, k)),                           # b >= m likely
        (rand_limbs(rng, k), rand_limbs(rng, 4), pow2),
        (rand_limbs(rng, 3), np.array([2**63], dtype=np.uint64), full),
        (np.array([2], dtype=np.uint64), np.array([255], dtype=np.uint64), rand_limbs(rng, k)),
    ]
    _check(gpu_lib, *zip(*cases))


def test_powmod_config_chains(gpu_lib):
    """256-limb odd and even moduli, 256-limb bases, 4096-bit exponents."""
    rng = np.random.default_rng(320)
    k, n = 256, 12
    mods = [rand_limbs(rng, k) for _ in range(n)]
    for i, m in enumerate(mods):
        m[0] = (int(m[0]) | 1) if i % 2 else (int(m[0]) & ~1)
    bases = [rand_limbs(rng, k) for _ in range(n)]
    exps = [rand_limbs(rng, 64) for _ in range(n)]
    _check(gpu_lib, bases, exps, mods)
    # the same chains again: nothing carried over between calls
    _check(gpu_lib, bases[:3], exps[:3], mods[:3])


def test_powmod_device_buffers(gpu_lib):
    rng = np.random.default_rng(330)
    k, n = 40, 9
    host = [(rand_limbs(rng, k), rand_limbs(rng, 3), rand_limbs(rng, k)) for _ in range(n)]
    dev = [tuple(torch.from_numpy(x).cuda() for x in t) for t in host]
    outs = [torch.zeros(k, dtype=torch.uint64, device="cuda") for _ in range(n)]
    d = (gpu_lib.PowmodDesc * n)()
    for i, ((b, e, m), r) in enumerate(zip(dev, outs)):
        d[i] = gpu_lib.PowmodDesc(r.data_ptr(), b.data_ptr(), e.data_ptr(), m.data_ptr(), k, 3)
    torch.cuda.synchronize()
    gpu_lib.powermod_batch_dev(d, k)
    for (b, e, m), r in zip(host, outs):
        assert _int(r.cpu().numpy()) == pow(_int(b), _int(e), _int(m))


def test_powmod_rejects_bad_input(gpu_lib):
    k = 4
    m = np.zeros(k, dtype=np.uint64)  # top limb zero
    with pytest.raises(gpu_lib.NBGError):
        gpu_lib.powermod_batch([np.ones(1, dtype=np.uint64)], [np.ones(1, dtype=np.uint64)], [m])
    with pytest.raises(gpu_lib.NBGError):  # base longer than the modulus
        gpu_lib.powermod_batch([np.ones(k + 1, dtype=np.uint64)], [np.ones(1, dtype=np.uint64)],
                               [np.ones(k, dtype=np.uint64)])
    with pytest.raises(gpu_lib.NBGError):  # zero exponent
        gpu_lib.powermod_batch([np.ones(1, dtype=np.uint64)], [np.zeros(1, dtype=np.uint64)],
                               [np.ones(k, dtype=np.uint64)])
