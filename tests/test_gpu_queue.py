"""Batches run as one persistent work-queue launch (tuning "queue": k > 0):
`k_queue` claims k jobs at a time in pipeline-step order and waits, per
product, for the previous step's jobs.  Every product equals GMP's and the
same batch run as per-step launches, over one-pass and multi-pass products,
odd and power-of-two lengths, squares, TMA and cp.async column tiles, and
carry runs across tiles; no bounded wait gave up."""
import json

import numpy as np
import pytest

import oracle as O
from conftest import adversarial, rand_limbs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture
def tuning(gpu_lib):
    old = gpu_lib.get_tuning()
    yield gpu_lib
    gpu_lib.set_tuning(old)


def _set(gpu_lib, **kw):
    t = json.loads(gpu_lib.get_tuning())
    t.update(kw)
    gpu_lib.set_tuning(json.dumps(t))


def _run_batch(gpu_lib, pairs, runs=2):
    items, outs, keep = [], [], []
    for a, b in pairs:
        da = torch.from_numpy(a).cuda()
        db = None if b is None else torch.from_numpy(b).cuda()
        n = a.size if b is None else b.size
        r = torch.zeros(a.size + n, dtype=torch.uint64, device="cuda")
        keep.append((da, db))
        outs.append(r)
        items.append((r, da, db, a.size, n, O.magnitude_bits(a), 0 if b is None else O.magnitude_bits(b)))
    descs = gpu_lib.make_descs(items)
    torch.cuda.synchronize()
    bt = gpu_lib.Batch(descs)
    st = torch.cuda.current_stream().cuda_stream
    for _ in range(runs):  # a replay rewrites every result
        bt.run(st)
    torch.cuda.synchronize()
    res = [r.cpu().numpy() for r in outs]
    bt.close()
    return res


def _pairs(rng):
    pairs = []
    for m, n in ((152, 152), (700, 300), (1000, 999), (4096, 4096), (9000, 2500), (30000, 30000),
                 (65536, 65536), (131072, 100000), (250000, 190000), (5000, 5000)):
        pairs.append((rand_limbs(rng, m), rand_limbs(rng, n)))
    for m in (160, 2000, 20000, 100000, 300000):
        pairs.append((rand_limbs(rng, m), None))
    ones = np.full(90000, 2**64 - 1, dtype=np.uint64)
    pairs.append((ones, ones.copy()))
    pairs.append((ones[:3000].copy(), None))
    pairs.append((adversarial(rng, 70000), adversarial(rng, 50000)))
    return pairs


@pytest.mark.parametrize("tma,chunk", [(1, 1), (1, 4), (0, 8)])
def test_queue_batch_matches_gmp_and_step_launches(tuning, tma, chunk):
    rng = np.random.default_rng(4100 + tma + chunk)
    pairs = _pairs(rng)
    _set(tuning, tma=tma, queue=chunk)
    got = _run_batch(tuning, pairs)
    _set(tuning, tma=tma, queue=0)
    ref = _run_batch(tuning, pairs, runs=1)
    for (a, b), g, r in zip(pairs, got, ref):
        want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
        assert np.array_equal(r, want)
        assert np.array_equal(g, want)
    assert tuning.device_faults() == 0


def test_queue_single_big_square(tuning):
    rng = np.random.default_rng(4200)
    a = rand_limbs(rng, 1 << 20)
    _set(tuning, queue=4)
    (got,) = _run_batch(tuning, [(a, None)])
    assert np.array_equal(got, O.gmp_sqr(a))
    assert tuning.device_faults() == 0


def test_queue_mixed_10000_batch_equals_step_launches(tuning):
    # the benchmark's 10,000-product batch: the work queue writes the same
    # limbs as the per-step launches (which the full-size test checks against GMP)
    from nbgpu.workload import bits_of, gen_workload

    W = gen_workload(1, 10000)
    limbs = W["limbs"]
    d_in = torch.from_numpy(limbs).cuda()
    ib = d_in.data_ptr()
    res = []
    for chunk in (0, 4):
        _set(tuning, queue=chunk)
        d_out = torch.zeros(W["out_total"], dtype=torch.uint64, device="cuda")
        ob = d_out.data_ptr()
        items = []
        for k in range(10000):
            m, n, sq = int(W["m"][k]), int(W["n"][k]), bool(W["sq"][k])
            ba = bits_of(limbs, int(W["off_a"][k]), m)
            bb = ba if sq else bits_of(limbs, int(W["off_b"][k]), n)
            items.append((ob + 8 * int(W["out_off"][k]), ib + 8 * int(W["off_a"][k]),
                          None if sq else ib + 8 * int(W["off_b"][k]), m, n, ba, bb))
        bt = tuning.Batch(tuning.make_descs(items))
        st = torch.cuda.current_stream().cuda_stream
        bt.run(st)
        bt.run(st)
        torch.cuda.synchronize()
        res.append(d_out.cpu().numpy())
        bt.close()
    assert np.array_equal(res[0], res[1])
    # spot-check against GMP too
    for k in range(0, 10000, 997):
        m, n = int(W["m"][k]), int(W["n"][k])
        a = limbs[W["off_a"][k]: W["off_a"][k] + m]
        want = O.gmp_sqr(a) if W["sq"][k] else O.gmp_mul(a, limbs[W["off_b"][k]: W["off_b"][k] + n])
        assert np.array_equal(res[1][W["out_off"][k]: W["out_off"][k] + m + n], want)
    assert tuning.device_faults() == 0
