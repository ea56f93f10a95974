"""Host side of the benchmark (no GPU): the seeded workload generator matches
the stated distributions, and the CPU baseline sample is a bounded prefix."""
import numpy as np

import bench


def test_mixed_workload_shape_and_determinism():
    W1 = bench.gen_workload(1, 2000)
    W2 = bench.gen_workload(1, 2000)
    assert np.array_equal(W1["limbs"], W2["limbs"]) and np.array_equal(W1["m"], W2["m"])
    m, n, sq = W1["m"], W1["n"], W1["sq"]
    assert m.min() >= 152 and m.max() <= 65536
    assert np.all(n <= m) and np.all(n >= 1)
    r = (n / m)[~sq]
    assert r.min() >= 0.24 and r.max() <= 1.0
    assert 0.15 < sq.mean() < 0.25                      # 20% squares
    assert np.all(n[sq] == m[sq])
    # top limbs nonzero, so magnitude bits use every limb
    for k in range(0, 2000, 97):
        a_top = W1["limbs"][W1["off_a"][k] + m[k] - 1]
        assert a_top != 0
        assert bench.bits_of(W1["limbs"], int(W1["off_a"][k]), int(m[k])) > 64 * (int(m[k]) - 1)
    assert W1["out_total"] == int((m + n).sum())


def test_shape_workload_and_cpu_sample():
    W = bench.gen_workload(3, 50, (1000, 600), False)
    assert np.all(W["m"] == 1000) and np.all(W["n"] == 600) and not W["sq"].any()
    Wq = bench.gen_workload(3, 10, (800, 800), True)
    assert Wq["sq"].all()
    W = bench.gen_workload(1, 10000)
    idx, desc = bench.cpu_sample(W, 0.01, 4)
    assert idx == list(range(len(idx))) and 1 <= len(idx) < 10000
    assert "threads" in desc
