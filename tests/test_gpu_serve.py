"""Continuous-batching server: results of requests served in a mixed stream
are bit-identical to GMP and to the same product computed alone."""
import threading

import numpy as np
import pytest

import oracle as O
from conftest import adversarial, rand_limbs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _mixed(rng, count, lo=100, hi=40000):
    out = []
    for _ in range(count):
        m = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        n = max(1, int(m * rng.uniform(0.25, 1.0)))
        out.append((adversarial(rng, m), None if rng.random() < 0.2 else adversarial(rng, n)))
    return out


def test_server_host_requests_from_threads(gpu_lib):
    rng = np.random.default_rng(71)
    pairs = _mixed(rng, 240)
    srv = gpu_lib.Server(hbm_budget_bytes=2 << 30, max_batch=64)
    results = [None] * len(pairs)
    tickets = [None] * len(pairs)

    def client(k0):
        for k in range(k0, len(pairs), 4):
            a, b = pairs[k]
            r = np.zeros(a.size + (a.size if b is None else b.size), dtype=np.uint64)
            results[k] = r
            tickets[k] = srv.submit(a, b, r)

    th = [threading.Thread(target=client, args=(i,)) for i in range(4)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for t in tickets:
        srv.wait(t, 120.0)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(pairs) and st["failed"] == 0
    assert st["p99_ms"] >= st["p50_ms"] > 0
    for (a, b), r in zip(pairs, results):
        want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
        assert np.array_equal(r, want)
    # the same product alone (plain one-per-call path) is identical
    for k in (0, 17, 101, 239):
        a, b = pairs[k]
        alone = gpu_lib.sqr(a) if b is None else gpu_lib.mul(a, b)
        assert np.array_equal(alone, results[k])


def test_server_device_requests(gpu_lib):
    rng = np.random.default_rng(72)
    pairs = _mixed(rng, 120, lo=152, hi=70000)
    srv = gpu_lib.Server(hbm_budget_bytes=4 << 30)
    outs, keep, tickets = [], [], []
    for a, b in pairs:
        da = torch.from_numpy(a).cuda()
        db = None if b is None else torch.from_numpy(b).cuda()
        n = a.size if b is None else b.size
        r = torch.zeros(a.size + n, dtype=torch.uint64, device="cuda")
        keep.append((da, db))
        outs.append(r)
    torch.cuda.synchronize()
    for (a, b), (da, db), r in zip(pairs, keep, outs):
        n = a.size if b is None else b.size
        tickets.append(srv.submit_dev(r, da, a.size, db, n, O.magnitude_bits(a),
                                      O.magnitude_bits(a) if b is None else O.magnitude_bits(b)))
    for t in tickets:
        srv.wait(t, 120.0)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(pairs)
    for (a, b), r in zip(pairs, outs):
        want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
        assert np.array_equal(r.cpu().numpy(), want)


def test_server_admission_and_bounded_wait(gpu_lib):
    rng = np.random.default_rng(73)
    srv = gpu_lib.Server(hbm_budget_bytes=32 << 20)
    # a product whose workspace exceeds the whole arena fails alone
    big_a, big_b = rand_limbs(rng, 2**18), rand_limbs(rng, 2**18)
    rbig = np.zeros(2**19, dtype=np.uint64)
    tbig = srv.submit(big_a, big_b, rbig)
    small = [(rand_limbs(rng, 500), rand_limbs(rng, 400)) for _ in range(8)]
    rs = [np.zeros(900, dtype=np.uint64) for _ in small]
    ts = [srv.submit(a, b, r) for (a, b), r in zip(small, rs)]
    with pytest.raises(gpu_lib.NBGError) as ei:
        srv.wait(tbig, 60.0)
    assert ei.value.code == gpu_lib.NBG_ENOMEM
    for t in ts:
        srv.wait(t, 60.0)
    for (a, b), r in zip(small, rs):
        assert np.array_equal(r, O.gmp_mul(a, b))
    # a bounded wait that expires returns NBG_ETIMEOUT and leaves the request running
    a = rand_limbs(rng, 2**16)
    r = np.zeros(2**17, dtype=np.uint64)
    t = srv.submit(a, None, r)
    try:
        srv.wait(t, 0.0)
        expired = False
    except gpu_lib.NBGError as e:
        assert e.code == gpu_lib.NBG_ETIMEOUT
        expired = True
    srv.wait(t, 60.0)
    assert np.array_equal(r, O.gmp_sqr(a))
    st = srv.stats()
    srv.close()
    assert st["failed"] == 1 and st["completed"] == 9
    assert expired or st["completed"] == 9
