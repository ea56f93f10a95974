"""GPU parity: every stage output and every product bit-identical to the
oracle (the reference's arithmetic restated) and to GMP.  Calls go through
the C ABI (nbgpu is a thin ctypes binding)."""
import numpy as np
import pytest

import oracle as O
from conftest import adversarial, rand_limbs

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _st():
    return torch.cuda.current_stream().cuda_stream


def dev(a: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t) -> np.ndarray:
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits_equal(x: np.ndarray, y: np.ndarray) -> bool:
    return np.array_equal(np.asarray(x, dtype=np.float64).view(np.uint64), np.asarray(y, dtype=np.float64).view(np.uint64))


def test_kernels_are_the_sm100a_build(gpu_lib):
    # the runtime loaded the kernels' sm_100a machine code (binaryVersion 100),
    # not a JIT of some other architecture's PTX
    import ctypes

    v = ctypes.c_int32(0)
    gpu_lib._check(gpu_lib.lib().nbg_kernel_arch(ctypes.byref(v)))
    assert v.value == 100


@pytest.fixture
def tuned(gpu_lib):
    """Restores the default pass split after a test that changes it."""
    old = gpu_lib.get_tuning()
    yield gpu_lib
    gpu_lib.set_tuning(old)


# ---------------------------------------------------------------------------
# pack (fp_ntt_pack!, src/fpntt.jl:744-768)

def test_pack_bitexact(gpu_lib):
    rng = np.random.default_rng(1)
    for n, b in ((1, 49), (1, 20), (3, 48), (7, 33), (100, 46), (1000, 43), (4097, 37), (50, 64 - 15)):
        a = adversarial(rng, n)
        nbits = O.magnitude_bits(a)
        nch = -(-nbits // b)
        N = max(4, 1 << (nch - 1).bit_length()) + 8
        x = torch.empty(N, dtype=torch.float64, device="cuda")
        gpu_lib.pack_dev(x, N, dev(a), n, b, nch, _st())
        assert bits_equal(host(x), O.pack(a, N, b, nch)), (n, b)


# ---------------------------------------------------------------------------
# transforms (fp_ntt_fwd! / fp_ntt_rev!, src/fpntt.jl:715-733)

SMALL_N = (4, 8, 64, 512, 1024, 12, 20, 48, 96, 160, 240, 1536, 960, 3840, 28, 56, 84, 140, 420, 1680,
           36, 144, 720, 1260, 4032)
MULTI_N = (12288, 20480, 7 * 2**15, 9 * 2**11, 105 * 2**11, 2**16, 315 * 2**10, 63 * 2**12, 45 * 2**11,
           35 * 2**12, 21 * 2**13, 15 * 2**13, 2**17 * 3)


def _check_transform(gpu_lib, N, f, rng):
    P = (O.P1, O.P2)[f]
    pl = O.Plan(N, f)
    # lazy-range inputs: |x| up to ~p, both signs
    x = (rng.integers(0, P, N, dtype=np.uint64).astype(np.float64) - float(rng.integers(0, 2)) * float(P) / 2)
    x = np.floor(x)
    want_f = pl.fwd(x)
    d = dev(x)
    gpu_lib.ntt_fwd_dev(d, N, f, _st())
    got_f = host(d)
    assert bits_equal(got_f, want_f), ("fwd", N, f)
    want_r = pl.rev(want_f)
    gpu_lib.ntt_rev_dev(d, N, f, _st())
    assert bits_equal(host(d), want_r), ("rev", N, f)


@pytest.mark.parametrize("f", [0, 1])
def test_transform_bitexact_small(gpu_lib, f):
    rng = np.random.default_rng(100 + f)
    for N in SMALL_N:
        _check_transform(gpu_lib, N, f, rng)


@pytest.mark.parametrize("f", [0, 1])
def test_transform_bitexact_multipass(gpu_lib, f):
    rng = np.random.default_rng(200 + f)
    for N in MULTI_N:
        assert len(gpu_lib.plan_info(N)["pass_end"]) >= 2
        _check_transform(gpu_lib, N, f, rng)


def test_transform_bitexact_forced_splits(tuned):
    # tiny tiles force many passes, narrow column tiles and every stage as
    # its own pass: the grouping must not change a single bit
    rng = np.random.default_rng(300)
    for tun in ('{"full_max_mul": 4, "full_max_sqr": 4, "last_max": 4, "early_gmax": 2, "tile_target": 8, "cmax": 2}',
                '{"full_max_mul": 16, "full_max_sqr": 16, "last_max": 64, "early_gmax": 16, "tile_target": 64, "cmax": 8}',
                '{"full_max_mul": 256, "full_max_sqr": 256, "last_max": 256, "early_gmax": 64, "tile_target": 512, "cmax": 32}'):
        tuned.set_tuning(tun)
        for N in (48, 240, 420, 1260, 4032, 960, 1680, 12288, 105 * 2**11):
            _check_transform(tuned, N, int(rng.integers(0, 2)), rng)


def test_pointwise_bitexact(gpu_lib):
    rng = np.random.default_rng(4)
    for f, P in ((0, O.P1), (1, O.P2)):
        N = 10007
        xa = np.floor(rng.integers(0, P, N, dtype=np.uint64).astype(np.float64) - float(P) / 2)
        xb = np.floor(rng.integers(0, P, N, dtype=np.uint64).astype(np.float64) - float(P) / 2)
        da, db = dev(xa), dev(xb)
        gpu_lib.pointwise_dev(da, db, N, f, _st())
        assert bits_equal(host(da), O.pointwise(xa, xb, f))


# ---------------------------------------------------------------------------
# unpack (fp_ntt_unpack2!, src/fpntt.jl:869-925)

def _unpack_case(rng, b, cs, N):
    P1, P2 = O.P1, O.P2
    x1 = np.zeros(N)
    x2 = np.zeros(N)
    for i, c in enumerate(cs):
        idx = (N - i) % N
        x1[idx] = float((c * N) % P1) + float(rng.integers(-2, 3)) * float(P1)
        x2[idx] = float((c * N) % P2) + float(rng.integers(-2, 3)) * float(P2)
    return x1, x2


def test_unpack_matches_oracle_and_crt(gpu_lib):
    rng = np.random.default_rng(0x6A3)
    for b in (33, 40, 44, 48, 49):
        for nconv in (1, 7, 64, 200, 5000, 40000):
            N = 1 << max(2, (nconv - 1).bit_length())
            pl = O.Plan(N, 0)
            pl2 = O.Plan(N, 1)
            cs = [int.from_bytes(rng.bytes(13), "little") % (O.P1 * O.P2) for _ in range(nconv)]
            x1, x2 = _unpack_case(rng, b, cs, N)
            rn = -(-(99 + b * (nconv - 1)) // 64) + 1
            want = O.unpack2(rn, x1, x2, nconv, b, pl.ninv, pl.ninvp, pl2.ninv, pl2.ninvp)
            r = torch.zeros(rn, dtype=torch.uint64, device="cuda")
            gpu_lib.unpack_dev(r, rn, dev(x1), dev(x2), N, nconv, b, _st())
            got = host(r)
            assert np.array_equal(got, want), (b, nconv)
            if nconv <= 200:
                assert O.to_int(got) == sum(c << (b * i) for i, c in enumerate(cs))


def test_unpack_long_carry_chains(gpu_lib):
    # coefficients c_i = d_i + e_i 2^b - e_(i-1) whose sum is 2^(64k) - 1:
    # every limb is all-ones after the fold, so carries ripple across tiles
    rng = np.random.default_rng(77)
    b = 41
    nconv = 60000
    N = 1 << (nconv - 1).bit_length()
    total_bits = b * nconv
    k = total_bits // 64 - 2
    T = (1 << (64 * k)) - 1
    d = [(T >> (b * i)) & ((1 << b) - 1) for i in range(nconv)]
    # digits below 64k/b are all-ones (>= 2^40), so any borrow e_(i-1) < 2^40 keeps c_i >= 0
    full = (64 * k) // b
    e = [int(rng.integers(0, 2**40)) if i < full - 1 else 0 for i in range(nconv)]
    cs = [d[i] + (e[i] << b) - (e[i - 1] if i else 0) for i in range(nconv)]
    assert all(0 <= c < O.P1 * O.P2 for c in cs)
    x1, x2 = _unpack_case(rng, b, cs, N)
    rn = k + 2
    r = torch.zeros(rn, dtype=torch.uint64, device="cuda")
    gpu_lib.unpack_dev(r, rn, dev(x1), dev(x2), N, nconv, b, _st())
    got = host(r)
    assert O.to_int(got) == T


# ---------------------------------------------------------------------------
# products (mul_fpntt2! / sqr_fpntt2!, src/fpntt.jl:982-1037)

SHAPES = ((1, 1), (5, 3), (16, 16), (100, 100), (255, 257), (500, 300), (601, 373), (1024, 1024),
          (2500, 2500), (5000, 4900), (152, 152), (160, 160), (4096, 4096), (9000, 64), (65536, 40000))


def test_products_vs_oracle_and_gmp(gpu_lib):
    rng = np.random.default_rng(0x91C4)
    for na, nb in SHAPES:
        for _ in range(2 if na * nb > 10**5 else 4):
            a, b = adversarial(rng, na), adversarial(rng, nb)
            got = gpu_lib.mul(a, b)
            assert np.array_equal(got, O.gmp_mul(a, b)), (na, nb)
            assert np.array_equal(got, O.mul(a, b))


def test_all_ones_max_chunk_width(gpu_lib):
    # b = 49, max-magnitude coefficients (test/test_fpntt.jl:301-307)
    for na in range(1, 9):
        for nb in range(1, na + 1):
            a = np.full(na, 2**64 - 1, dtype=np.uint64)
            b = np.full(nb, 2**64 - 1, dtype=np.uint64)
            assert np.array_equal(gpu_lib.mul(a, b), O.gmp_mul(a, b))
    for n in (1, 6, 160, 4096, 70000):
        a = np.full(n, 2**64 - 1, dtype=np.uint64)
        assert np.array_equal(gpu_lib.sqr(a), O.gmp_sqr(a))


def test_squares_vs_gmp(gpu_lib):
    rng = np.random.default_rng(0x5F2E)
    for n in (1, 7, 100, 160, 1024, 3000, 8192, 20000):
        a = adversarial(rng, n)
        assert np.array_equal(gpu_lib.sqr(a), O.gmp_sqr(a)), n


def test_sparse_operands(gpu_lib):
    rng = np.random.default_rng(5)
    for n in (2**12, 2**16):
        a = np.zeros(n, dtype=np.uint64)
        idx = rng.choice(n, n // 100, replace=False)
        a[idx] = rng.integers(1, 2**63, idx.size, dtype=np.uint64)
        a[-1] = 1
        b = rand_limbs(rng, n)
        assert np.array_equal(gpu_lib.mul(a, b), O.gmp_mul(a, b))
        assert np.array_equal(gpu_lib.sqr(a), O.gmp_sqr(a))


def test_nbig_star(gpu_lib):
    # NBig * (src/nbig.jl:124-140): same buffer -> square, signs, zero
    rng = np.random.default_rng(9)
    for n in (220, 224, 1024, 3000):
        v = O.to_int(adversarial(rng, n))
        x = gpu_lib.NBig(v)
        assert int(x * x) == v * v
        assert int(x * -x) == -(v * v)
    y = gpu_lib.NBig(O.to_int(rand_limbs(rng, 500)))
    z = gpu_lib.NBig(-O.to_int(rand_limbs(rng, 300)))
    assert int(y * z) == int(y) * int(z)
    assert int(gpu_lib.NBig(0) * z) == 0
    assert int(gpu_lib.NBig(-3) * gpu_lib.NBig(5)) == -15


def test_large_radix7_residues(gpu_lib):
    # 144,000 limbs on a 7*2^k length, residues mod 63-bit moduli (test/test_fpntt.jl:308-325)
    rng = np.random.default_rng(0x7777)
    n = 144_000
    a, b = rand_limbs(rng, n), rand_limbs(rng, n)
    r = gpu_lib.mul(a, b)
    assert np.array_equal(r, O.mul(a, b))


def test_square_2_20_limbs(gpu_lib):
    rng = np.random.default_rng(20)
    a = rand_limbs(rng, 2**20)
    assert np.array_equal(gpu_lib.sqr(a), O.sqr(a))


# ---------------------------------------------------------------------------
# batches

def _mixed_pairs(rng, count, lo=1, hi=20000):
    pairs = []
    for _ in range(count):
        m = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        n = max(1, int(m * rng.uniform(0.25, 1.0)))
        if rng.random() < 0.2:
            pairs.append((adversarial(rng, m), None))
        else:
            pairs.append((adversarial(rng, m), adversarial(rng, n)))
    return pairs


def test_batch_host_mixed_sizes(gpu_lib):
    rng = np.random.default_rng(31)
    pairs = _mixed_pairs(rng, 300)
    got = gpu_lib.mul_batch(pairs)
    for (a, b), r in zip(pairs, got):
        want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
        assert np.array_equal(r, want)
    # each result is the same alone and in the mix
    for i in (0, 7, 150, 299):
        a, b = pairs[i]
        alone = gpu_lib.sqr(a) if b is None else gpu_lib.mul(a, b)
        assert np.array_equal(alone, got[i])


def test_batch_dev_and_graph(gpu_lib):
    rng = np.random.default_rng(32)
    pairs = _mixed_pairs(rng, 120, lo=100, hi=30000)
    items, outs, dops = [], [], []
    for a, b in pairs:
        da = dev(a)
        db = None if b is None else dev(b)
        n = a.size if b is None else b.size
        r = torch.zeros(a.size + n, dtype=torch.uint64, device="cuda")
        dops.append((da, db))
        outs.append(r)
        items.append((r, da, db, a.size, n, O.magnitude_bits(a), 0 if b is None else O.magnitude_bits(b)))
    descs = gpu_lib.make_descs(items)
    torch.cuda.synchronize()
    gpu_lib.mul_batch_dev(descs, _st())
    for (a, b), r in zip(pairs, outs):
        want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
        assert np.array_equal(host(r), want)
    bt = gpu_lib.Batch(descs)
    assert bt.launches >= 3
    for r in outs:
        r.zero_()
    for rep in range(2):
        bt.run(_st())
        for (a, b), r in zip(pairs, outs):
            want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
            assert np.array_equal(host(r), want)
    # new operand values with the same magnitude bits: replay computes the new products
    for (a, b), (da, db) in zip(pairs, dops):
        a2 = a.copy()
        a2[:-1] = rng.integers(0, 2**64, a.size - 1, dtype=np.uint64)
        a[:] = a2
        da.copy_(torch.from_numpy(a2))
    bt.run(_st())
    for (a, b), r in zip(pairs, outs):
        want = O.gmp_sqr(a) if b is None else O.gmp_mul(a, b)
        assert np.array_equal(host(r), want)
    bt.close()
