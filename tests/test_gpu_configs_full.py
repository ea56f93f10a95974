"""The full-size product configurations, every result checked.

* The 10,000-product mixed batch the benchmark times (larger operand
  log-uniform in [152, 65536] limbs, ratio U[0.25, 1], 20% squares, seed 1):
  all 10,000 products run as one device batch and every one is compared with
  GMP's mpn_mul / mpn_sqr (threads: ctypes releases the GIL).
* 256 Barrett powermod chains with 256-limb odd and even moduli, 256-limb
  bases and 4096-bit exponents, every chain compared with GMP's mpz_powm.

The reference's differential tests compare its engine with BigInt over many
shapes (test/test_fpntt.jl:288-331); these do the same at the benchmark's
sizes."""
import concurrent.futures as cf
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def test_mixed_batch_all_10000_products_vs_gmp(gpu_lib):
    from nbgpu.workload import bits_of, gen_workload

    W = gen_workload(1, 10000)
    limbs = W["limbs"]
    d_in = torch.from_numpy(limbs).cuda()
    d_out = torch.zeros(W["out_total"], dtype=torch.uint64, device="cuda")
    ib, ob = d_in.data_ptr(), d_out.data_ptr()
    items = []
    for k in range(10000):
        m, n, sq = int(W["m"][k]), int(W["n"][k]), bool(W["sq"][k])
        ba = bits_of(limbs, int(W["off_a"][k]), m)
        bb = ba if sq else bits_of(limbs, int(W["off_b"][k]), n)
        items.append((ob + 8 * int(W["out_off"][k]), ib + 8 * int(W["off_a"][k]),
                      None if sq else ib + 8 * int(W["off_b"][k]), m, n, ba, bb))
    descs = gpu_lib.make_descs(items)
    torch.cuda.synchronize()
    bt = gpu_lib.Batch(descs)
    st = torch.cuda.current_stream().cuda_stream
    bt.run(st)
    bt.run(st)  # a replay rewrites every result
    torch.cuda.synchronize()
    res = d_out.cpu().numpy()
    bt.close()

    def bad(k):
        m, n = int(W["m"][k]), int(W["n"][k])
        a = limbs[W["off_a"][k]: W["off_a"][k] + m]
        want = O.gmp_sqr(a) if W["sq"][k] else O.gmp_mul(a, limbs[W["off_b"][k]: W["off_b"][k] + n])
        return not np.array_equal(res[W["out_off"][k]: W["out_off"][k] + m + n], want)

    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        wrong = [k for k, b in zip(range(10000), ex.map(bad, range(10000))) if b]
    assert wrong == []


def test_powmod_256_chains_full_size_vs_gmp(gpu_lib):
    # the benchmark's powermod workload: 256-limb moduli (odd and even
    # alternating, top limb nonzero), 256-limb bases, 4096-bit exponents
    rng = np.random.Generator(np.random.PCG64(1))
    n, k, le = 256, 256, 64
    mods, bases, exps = [], [], []
    for i in range(n):
        m = rng.integers(0, 2**64, k, dtype=np.uint64)
        m[-1] |= np.uint64(1)
        m[0] = (m[0] | np.uint64(1)) if i % 2 else (m[0] & ~np.uint64(1))
        e = rng.integers(0, 2**64, le, dtype=np.uint64)
        e[-1] |= np.uint64(1 << 63)
        mods.append(m)
        bases.append(rng.integers(0, 2**64, k, dtype=np.uint64))
        exps.append(e)
    got = gpu_lib.powermod_batch(bases, exps, mods)
    with cf.ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        want = list(ex.map(O.gmp_powm, bases, exps, mods))
    wrong = [i for i in range(n) if not np.array_equal(np.asarray(got[i])[:k], want[i])]
    assert wrong == []
