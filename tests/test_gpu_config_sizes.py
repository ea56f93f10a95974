"""The single-product configurations on the GPU, bit-exact against GMP:
4096 x 4096 limbs (mul and square, seed 1), balanced products and squares at
2^16, 2^20 and 2^24 limbs in three value patterns (uniform, all-ones, 1%
sparse), and the sizes that land on each odd transform-length multiplier."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

# operand limbs -> transform length N (balanced products), from the admission rules
LANDINGS = ((4096, 3 * 2**12), (6200, 5 * 2**12), (9032, 7 * 2**12), (5512, 9 * 2**11), (110336, 3 * 2**17),
            (94592, 5 * 2**16), (68992, 7 * 2**15), (84096, 9 * 2**15), (1439744, 315 * 2**14),
            (10928128, 315 * 2**17))


def _pattern(rng, n, kind):
    if kind == "uniform":
        a = rng.integers(0, 2**64, n, dtype=np.uint64)
    elif kind == "ones":
        a = np.full(n, 2**64 - 1, dtype=np.uint64)
    else:  # 1% of limbs nonzero at seeded positions
        a = np.zeros(n, dtype=np.uint64)
        idx = rng.choice(n, max(1, n // 100), replace=False)
        a[idx] = rng.integers(1, 2**64, idx.size, dtype=np.uint64)
    if a[-1] == 0:
        a[-1] = 1
    return a


def test_4096_limb_product_and_square(gpu_lib):
    rng = np.random.Generator(np.random.PCG64(1))
    a = _pattern(rng, 4096, "uniform")
    b = _pattern(rng, 4096, "uniform")
    assert np.array_equal(gpu_lib.mul(a, b), O.gmp_mul(a, b))
    assert np.array_equal(gpu_lib.mul(a, b), O.mul(a, b))
    assert np.array_equal(gpu_lib.sqr(a), O.gmp_sqr(a))
    assert np.array_equal(gpu_lib.sqr(a), O.sqr(a))


@pytest.mark.parametrize("lg", [16, 20, 24])
@pytest.mark.parametrize("kind", ["uniform", "ones", "sparse"])
def test_large_balanced(gpu_lib, lg, kind):
    rng = np.random.Generator(np.random.PCG64(1000 + lg))
    n = 1 << lg
    a = _pattern(rng, n, kind)
    b = _pattern(rng, n, kind)
    assert np.array_equal(gpu_lib.mul(a, b), O.gmp_mul(a, b)), (lg, kind, "mul")
    assert np.array_equal(gpu_lib.sqr(a), O.gmp_sqr(a)), (lg, kind, "sqr")


@pytest.mark.parametrize("n,N", LANDINGS)
def test_odd_length_landings(gpu_lib, n, N):
    rng = np.random.Generator(np.random.PCG64(n))
    a = _pattern(rng, n, "uniform")
    b = _pattern(rng, n, "uniform")
    bits = 64 * (n - 1) + int(a[-1]).bit_length()
    bits_b = 64 * (n - 1) + int(b[-1]).bit_length()
    assert gpu_lib.ntt_params(bits, bits_b)[1] == N
    assert np.array_equal(gpu_lib.mul(a, b), O.gmp_mul(a, b)), n
