"""Products the reference keeps off its NTT, routed to the GPU engine and
bit-exact against GMP: low halves (mullo!/sqrlo!, whose full-product branches
keep the low k limbs of mul!/sqr!, src/mul.jl:316-319, :361-364), unbalanced
products below MUL_FPNTT_MIN (the chunked Karatsuba path, src/mul.jl:391-405)
and products below the admission thresholds (src/mul.jl:12-26), alone and in
one batch."""
import numpy as np
import pytest

import oracle as O
from conftest import adversarial, rand_limbs

pytestmark = pytest.mark.gpu


def _low(v: np.ndarray, k: int) -> np.ndarray:
    out = np.zeros(k, dtype=np.uint64)
    out[: min(k, v.size)] = v[:k]
    return out


def test_mullo_sqrlo(gpu_lib):
    rng = np.random.default_rng(501)
    for la, lb, k in ((1, 1, 1), (3, 2, 4), (300, 200, 224), (1000, 1000, 1000), (4000, 3000, 2500),
                      (6000, 700, 9000), (50, 50, 120), (20000, 20000, 448)):
        a, b = adversarial(rng, la), adversarial(rng, lb)
        assert np.array_equal(gpu_lib.mullo(a, b, k), _low(O.gmp_mul(a, b), k)), (la, lb, k)
        assert np.array_equal(gpu_lib.sqrlo(a, k), _low(O.gmp_sqr(a), k)), (la, k)


@pytest.mark.parametrize("n", [1, 2, 29, 48, 63])
def test_unbalanced_below_fpntt_min(gpu_lib, n):
    rng = np.random.default_rng(510 + n)
    for m in (n, 300, 5000, 100000):
        a, b = rand_limbs(rng, m), adversarial(rng, n)
        assert np.array_equal(gpu_lib.mul(a, b), O.gmp_mul(a, b)), (m, n)


def test_below_admission_in_one_batch(gpu_lib):
    # every pair here is below the reference's NTT admission (n < 64 or m + n < 304)
    rng = np.random.default_rng(520)
    pairs = []
    for _ in range(400):
        n = int(rng.integers(1, 64))
        m = int(rng.integers(n, 3000))
        pairs.append((rand_limbs(rng, m), None if rng.random() < 0.15 else adversarial(rng, n)))
    for _ in range(100):
        m = int(rng.integers(1, 152))
        pairs.append((rand_limbs(rng, m), adversarial(rng, int(rng.integers(1, m + 1)))))
    got = gpu_lib.mul_batch(pairs)
    for (a, b), r in zip(pairs, got):
        want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
        assert np.array_equal(r, want)
