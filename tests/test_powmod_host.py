"""Host side of the Barrett powermod chains (no GPU): the reciprocal μ and the
sliding-window step lists, executed here with Python integers, give b^e mod m
(the reference's powermod_limbs, src/algorithms.jl:17-107, on its Barrett
branch, src/barrett.jl:22-81)."""
import numpy as np
import pytest

import oracle as O
from conftest import rand_limbs
from nbgpu import barrett_mu, powmod_schedule

B = 1 << 64


def _int(a) -> int:
    return O.to_int(np.asarray(a, dtype=np.uint64))


@pytest.mark.parametrize("k", [1, 2, 3, 7, 64, 256])
def test_barrett_mu_matches_integer_division(k):
    rng = np.random.default_rng(100 + k)
    for _ in range(4):
        m = rand_limbs(rng, k)
        if k == 1 and int(m[0]) < 2:
            m[0] = 3
        want = B ** (2 * k) // _int(m)
        assert _int(barrett_mu(m)) == want
    # m = β^(k-1): μ needs k + 2 limbs
    if k > 1:
        m = np.zeros(k, dtype=np.uint64)
        m[-1] = 1
        mu = barrett_mu(m)
        assert _int(mu) == B ** (k + 1) and mu[k + 1] == 1


def _barrett(T: int, m: int, mu: int, k: int) -> int:
    """barrett_reduce! (src/barrett.jl:44-81) on integers."""
    q1 = T // B ** (k - 1)
    q3 = q1 * mu // B ** (k + 1)
    r = (T - q3 * m) % B ** (k + 1)
    n = 0
    while r >= m:
        r -= m
        n += 1
    assert n <= 2
    return r


def _run_schedule(b: int, e_limbs, m: int, k: int) -> int:
    ops, T = powmod_schedule(e_limbs)
    mu = B ** (2 * k) // m
    slots = {T + 2: b, T + 3: 1}
    for d, s1, s2 in ops.tolist():
        if s2 == 255:
            slots[d] = slots[s1]
        else:
            slots[d] = _barrett(slots[s1] * slots[s2], m, mu, k)
    return slots[T + 1]


@pytest.mark.parametrize("k", [1, 3, 16])
def test_schedule_computes_powmod(k):
    rng = np.random.default_rng(7 + k)
    exps = [1, 2, 3, 5, 255, 256, 2**64 - 1, 2**80 + 1, 2**240, 3**150]
    exps += [int.from_bytes(rng.bytes(512), "little") | (1 << 4095) for _ in range(2)]
    for e in exps:
        m = _int(rand_limbs(rng, k)) | 1 if e % 2 else _int(rand_limbs(rng, k)) & ~1
        m = max(m, 3)
        b = _int(rand_limbs(rng, k))
        el = O.from_int(e, max(1, -(-e.bit_length() // 64)))
        assert _run_schedule(b, el, m, k) == pow(b, e, m), e


def test_schedule_window_widths():
    # the reference's widths: <= 8 bits w=1, <= 24 w=2, <= 80 w=3, <= 240 w=4, else 5
    for bits, w in ((8, 1), (9, 2), (24, 2), (25, 3), (80, 3), (81, 4), (240, 4), (241, 5), (4096, 5)):
        _, T = powmod_schedule(O.from_int(1 << (bits - 1), -(-bits // 64)))
        assert T == 1 << (w - 1), bits
    with pytest.raises(Exception):
        powmod_schedule(np.zeros(2, dtype=np.uint64))


@pytest.mark.parametrize("k", [1, 2, 5, 64])
def test_oracle_mu_and_powmod(k):
    """The oracle's restatement (the CPU baseline of the chains) against integers."""
    rng = np.random.default_rng(40 + k)
    for i in range(3):
        m = rand_limbs(rng, k)
        m[0] = (int(m[0]) | 1) if i % 2 else (int(m[0]) & ~1)
        if k == 1:
            m[0] = max(int(m[0]), 2)
        assert _int(O.barrett_mu(m)) == B ** (2 * k) // _int(m)
        b = rand_limbs(rng, k)
        e = rand_limbs(rng, 2 if k > 5 else 5)
        assert _int(O.powmod_barrett(b, e, m)) == pow(_int(b), _int(e), _int(m))
