"""Radix conversion on the GPU (nbg_radix_combine): the value of base-bb
chunks, the reference's subquadratic radix_combine (src/nbig.jl:410-417) whose
levels run as batched products, equals the integer sum(c_i * bb^i)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _value(c, bb: int) -> int:
    """sum(c[i] * bb**i) by divide and conquer on Python integers."""
    def rec(lo, hi, p):  # chunks [lo, hi), p = bb**((hi - lo) // 2) for even splits
        if hi - lo == 1:
            return int(c[lo])
        mid = (lo + hi) // 2
        return rec(mid, hi, None) * bb ** (mid - lo) + rec(lo, mid, None)
    return rec(0, len(c), None) if len(c) else 0


@pytest.mark.parametrize("bb", [10, 10**19, 2**64 - 1, 3**40])
def test_radix_combine(gpu_lib, bb):
    rng = np.random.default_rng(700 + bb % 997)
    for n in (1, 5, 32, 33, 100, 1000, 5000, 20000):
        c = rng.integers(0, bb, n, dtype=np.uint64) if bb < 2**63 else \
            (rng.integers(0, 2**63, n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, n, dtype=np.uint64)) % np.uint64(bb)
        got = gpu_lib.radix_combine(c, bb)
        assert O.to_int(got) == _value(c, bb), (bb, n)


def test_radix_combine_zeros_and_rejects(gpu_lib):
    c = np.zeros(70, dtype=np.uint64)
    assert gpu_lib.radix_combine(c, 10**19).size == 0
    c[69] = 7
    assert O.to_int(gpu_lib.radix_combine(c, 10**19)) == 7 * 10 ** (19 * 69)
    with pytest.raises(gpu_lib.NBGError):
        gpu_lib.radix_combine(np.array([10], dtype=np.uint64), 10)


@pytest.mark.parametrize("bb", [10**19, 2**64 - 1, 3])
def test_radix_powtab_matches_reference_table(gpu_lib, bb):
    # radix_chunks_dc's table (src/nbig.jl:396-399): bb^(2^(i-1)) while the last entry <= x
    rng = np.random.default_rng(710 + bb % 991)
    for xn in (1, 2, 9, 300, 5000, 70000):
        x = rng.integers(0, 2**64, xn, dtype=np.uint64)
        x[-1] |= np.uint64(1)
        xv = O.to_int(x)
        want = [bb]
        while want[-1] <= xv:
            want.append(want[-1] * want[-1])
        got = gpu_lib.radix_powtab(bb, x)
        assert [O.to_int(g) for g in got] == want, (bb, xn)
        assert all(g.size == 0 or g[-1] != 0 for g in got)  # normalized
    # x below bb: the table is bb alone
    assert [O.to_int(g) for g in gpu_lib.radix_powtab(bb, np.array([1], dtype=np.uint64))] == [bb]
