"""Sums of products for the reference's HGCD callers on the GPU: the 2x2
matrix product (hgcd_matrix_mul!, src/gcd.jl:371-389) and the cofactor update
r = a*x + b*y (cof_mul2!, src/gcd.jl:571-598), against Python integers,
including zero entries and carries that ripple across every 1024-limb tile."""
import numpy as np
import pytest

import oracle as O
from conftest import rand_limbs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev(v: np.ndarray, room: int):
    t = torch.zeros(room, dtype=torch.uint64, device="cuda")
    t[: v.size] = torch.from_numpy(v.astype(np.uint64)).cuda()
    return t


def _int(t) -> int:
    return O.to_int(t.cpu().numpy())


def _entry(rng, n, kind):
    if kind == "zero":
        return np.zeros(n, dtype=np.uint64)
    if kind == "one":
        v = np.zeros(n, dtype=np.uint64)
        v[0] = 1
        return v
    v = rand_limbs(rng, int(rng.integers(1, n + 1)), top_nonzero=True)
    out = np.zeros(n, dtype=np.uint64)
    out[: v.size] = v
    return out


@pytest.mark.parametrize("n,n1", [(1, 1), (7, 3), (300, 250), (3000, 2900), (20000, 9000)])
def test_matrix22_mul(gpu_lib, n, n1):
    rng = np.random.default_rng(600 + n)
    for kinds in (("rand",) * 4, ("one", "zero", "zero", "one"), ("rand", "zero", "rand", "rand")):
        M = [_entry(rng, n, k) for k in kinds]
        M1 = [_entry(rng, n1, k) for k in ("rand", "rand", "zero", "rand")]
        L = n + n1 + 1
        dM = [_dev(x, L) for x in M]
        dM1 = [_dev(x, n1) for x in M1]
        torch.cuda.synchronize()
        gpu_lib.matrix22_mul_dev(dM, n, dM1, n1)
        a = [O.to_int(x) for x in M]
        b = [O.to_int(x) for x in M1]
        want = [a[0] * b[0] + a[1] * b[2], a[0] * b[1] + a[1] * b[3], a[2] * b[0] + a[3] * b[2],
                a[2] * b[1] + a[3] * b[3]]
        assert [_int(t) for t in dM] == want, (n, n1, kinds)


def test_mul2add_long_carries(gpu_lib):
    rng = np.random.default_rng(650)
    # a*x = 2^(64k) - 1 (all ones), b*y = 1: the sum carries through every tile
    for k in (1, 1023, 1024, 5000):
        a = np.full(k, 2**64 - 1, dtype=np.uint64)
        one = np.ones(1, dtype=np.uint64)
        rn = k + 2
        r = torch.zeros(rn, dtype=torch.uint64, device="cuda")
        gpu_lib.mul2add_dev(r, rn, _dev(a, k), k, _dev(one, 1), 1, _dev(one, 1), 1, _dev(one, 1), 1)
        assert _int(r) == 1 << (64 * k)
    for la, lx, lb, ly in ((5, 3, 4, 4), (2000, 1500, 2500, 100), (40000, 30000, 35000, 35000)):
        a, x, b, y = rand_limbs(rng, la), rand_limbs(rng, lx), rand_limbs(rng, lb), rand_limbs(rng, ly)
        rn = max(la + lx, lb + ly) + 1
        r = torch.zeros(rn, dtype=torch.uint64, device="cuda")
        gpu_lib.mul2add_dev(r, rn, _dev(a, la), la, _dev(x, lx), lx, _dev(b, lb), lb, _dev(y, ly), ly)
        assert _int(r) == O.to_int(a) * O.to_int(x) + O.to_int(b) * O.to_int(y)
