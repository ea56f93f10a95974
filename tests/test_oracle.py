"""Pins the CPU oracle (oracle/fpntt_oracle.c) to the reference.

Ports of the reference's own checks for the fp-NTT path
(NativeBigInt.jl test/test_fpntt.jl) plus differential checks against GMP,
which is the arithmetic Julia's BigInt uses.  The reference's random
operands come from Julia's MersenneTwister and cannot be regenerated here,
so the ports use numpy seeds; the literal known-answer tables are kept as is.
"""
import numpy as np
import pytest

import oracle as O
from conftest import adversarial, rand_limbs

P1, P2 = O.P1, O.P2


def canon(x: float, P: int) -> int:
    return int(x) % P


def test_prime_identities():
    # test/test_fpntt.jl:22-24, :186-189, :208
    L = O.lib()
    assert L.orc_prime(0) == 65205 * 2**34 + 1 == P1
    assert L.orc_prime(1) == 4095 * 2**38 + 1 == 2**50 - 2**38 + 1 == P2
    assert float(P1) == P1 and float(P2) == P2
    assert (P1 - 1) % (315 << 34) == 0 and (P2 - 1) % (315 << 38) == 0
    assert min(L.orc_two_adicity(0), L.orc_two_adicity(1)) == 34


def test_generator_root_orders():
    # test/test_fpntt.jl:61-67: generator-derived roots have exact order
    L = O.lib()
    for f, P in ((0, P1), (1, P2)):
        g = L.orc_generator(f)
        assert 3 <= g <= 63
        for logN in (1, 5, 20, 34):
            N = 2**logN
            w = pow(g, (P - 1) // N, P)
            assert pow(w, N, P) == 1
            assert pow(w, N // 2, P) == P - 1


def test_field_arithmetic_lazy_range():
    # test/test_fpntt.jl:20-60: constant mulmod over |x| <= 4p with
    # minimal-balanced |w| <= p/2, value mulmod |x*y| <= p^2, reduce to 8p
    rng = np.random.default_rng(0xF94)
    L = O.lib()
    FP = float(P1)
    half = (FP - 1) / 2
    edgew = [0.0, 1.0, -1.0, 2.0, 2.0**33, half, -half]
    ws = edgew + [float(rng.choice([-1, 1])) * float(rng.integers(0, (P1 - 1) >> 1)) for _ in range(60)]
    edges = [0.0, 1.0, -1.0, FP - 1, -(FP - 1), FP, -FP, 2 * FP, -2 * FP, 4 * FP - 4, -(4 * FP - 4), 4 * FP, -4 * FP]
    xs = edges + [float(rng.choice([-4, -2, -1, 1, 2, 4])) * float(rng.integers(0, P1)) for _ in range(200)]
    for w in ws:
        for x in xs:
            r = L.orc_fp_mulmod4(x, w, w / FP, 0)
            assert abs(r) < FP
            assert canon(r, P1) == (int(w) * int(x)) % P1
    for x in xs:
        for y in xs:
            if abs(x) <= FP and abs(y) <= FP:
                r = L.orc_fp_mulmod3(x, y, 0)
                assert abs(r) < FP
                assert canon(r, P1) == (int(x) * int(y)) % P1
    for x in xs:
        r = L.orc_fp_reduce(2 * x, 0)
        assert abs(r) < FP
        assert canon(r, P1) == (2 * int(x)) % P1
    for x in ws + [half + 1, -(half + 1), FP - 1, -(FP - 1)]:
        m = L.orc_fp_minbal(x, 0)
        assert abs(m) <= FP / 2
        assert canon(m, P1) == int(x) % P1


def _ntt_len_want(T: int) -> int:
    # brute force of test/test_fpntt.jl:211-221
    ms = (1, 3, 5, 9) if T <= 1 << 14 else (1, 3, 5, 7, 9, 15, 21, 105) if T <= 1 << 20 else \
        (1, 3, 5, 7, 9, 15, 21, 35, 45, 63, 105, 315)
    best = None
    for m in ms:
        for k in range(2, 35):
            c = m << k
            if c >= T and (best is None or c < best):
                best = c
    return best


NTT_LEN_CASES = (1, 4, 5, 100, 1000, 1023, 1025, 13000, 15359, 15360, 20000, 1 << 20,
                 (15 << 14) - 100, 15 << 14, (15 << 14) + 1, (15 << 20) - 1, 15 << 20,
                 (21 << 14) - 1, 21 << 14, (35 << 14) - 1, 35 << 14, (105 << 14) - 1, 105 << 14,
                 (7 << 10) - 1, 7 << 10, (3 << 22) - 1, 3 << 22, (5 << 22) - 1, 5 << 22,
                 (7 << 22) - 1, 7 << 22, 1 << 22, 1 << 25)


def test_ntt_len_known_answers():
    # test/test_fpntt.jl:223-254 (tier table, 2-adic cap, literal answers)
    for T in NTT_LEN_CASES:
        n = O.ntt_len(T)
        assert n == _ntt_len_want(T)
        assert n >= T and ((n & -n).bit_length() - 1) <= 34
        assert (P1 - 1) % n == 0 and (P2 - 1) % n == 0
    assert O.ntt_len(15 << 14) == 15 << 14
    assert O.ntt_len(15 << 13) == 15 << 13
    assert O.ntt_len(7 << 10) == 1 << 13
    assert O.ntt_len(7 << 14) == 7 << 14
    assert O.ntt_len(9 << 10) == 9 << 10
    assert O.ntt_len((1 << 34) + 1) == 35 << 29
    assert O.ntt_len(1 << 34) == 1 << 34
    assert O.ntt_len(33 << 34) == 35 << 34
    assert O.ntt_len(53 << 34) == 63 << 34
    assert O.ntt_len(315 << 34) == 315 << 34
    with pytest.raises(ValueError):
        O.ntt_len((315 << 34) + 1)


def test_ntt_params_documented_landings():
    # chunk widths / lengths at the sizes the engine is measured on
    assert O.ntt_params(64 * 4096, 64 * 4096) == (43, 12288)
    assert O.ntt_params(64 * 2**16, 64 * 2**16)[1] == 105 * 2**11
    assert O.ntt_params(64 * 2**20, 64 * 2**20) == (39, 7 * 2**19)
    assert O.ntt_params(64 * 2**24, 64 * 2**24) == (37, 7 * 2**23)
    assert O.ntt_params(64, 64) == (49, 4)
    b, N = O.ntt_params(64 * 144000, 64 * 144000)  # test_fpntt.jl:314-316: an m = 7 length
    assert N >> ((N & -N).bit_length() - 1) == 7


def test_ntt_params_bound_is_tight():
    # the chosen b is the largest <= 49 with min(nca,ncb)*(2^b-1)^2 <= p1*p2 - 1
    pp = P1 * P2 - 1
    rng = np.random.default_rng(7)
    for _ in range(300):
        ba = int(rng.integers(1, 64 * 2**20))
        bb = int(rng.integers(1, 64 * 2**20))
        b, N = O.ntt_params(ba, bb)
        nca, ncb = -(-ba // b), -(-bb // b)
        assert min(nca, ncb) * (2**b - 1) ** 2 <= pp
        if b < 49:
            b2 = b + 1
            assert min(-(-ba // b2), -(-bb // b2)) * (2**b2 - 1) ** 2 > pp
        assert N == O.ntt_len(nca + ncb - 1)


ROUNDTRIP_N1 = (4, 8, 64, 512, 1024, 12, 20, 48, 96, 160, 240, 1536, 960, 3840, 28, 56, 84, 140, 420, 1680,
                36, 144, 720, 1260, 4032)
ROUNDTRIP_N2 = (4, 8, 64, 512, 12, 20, 48, 240, 1536, 960, 28, 420, 36, 1260)


@pytest.mark.parametrize("f,Ns", [(0, ROUNDTRIP_N1), (1, ROUNDTRIP_N2)])
def test_transform_round_trip(f, Ns):
    # test/test_fpntt.jl:84-99 and :191-202: rev(fwd(x)) = N * x[(N-t) mod N]
    P = (P1, P2)[f]
    rng = np.random.default_rng(0xF18 + f)
    for N in Ns:
        pl = O.Plan(N, f)
        x = rng.integers(0, P, N, dtype=np.uint64).astype(np.float64)
        y = pl.fwd(x)
        assert not np.array_equal(y, x)
        z = pl.rev(y)
        want = [(N * int(x[(N - t) % N])) % P for t in range(N)]
        assert [canon(v, P) for v in z] == want


def test_transform_cyclic_convolution():
    # test/test_fpntt.jl:100-116: fwd, pointwise, rev, 1/N recovers the cyclic convolution
    rng = np.random.default_rng(0xC0)
    L = O.lib()
    for N in (4, 8, 12, 20, 28, 36, 48, 56, 64, 84, 96, 140, 144, 160, 240):
        pl = O.Plan(N, 0)
        a = rng.integers(0, P1, N, dtype=np.uint64)
        b = rng.integers(0, P1, N, dtype=np.uint64)
        c = [0] * N
        ai, bi = [int(v) for v in a], [int(v) for v in b]
        for i in range(N):
            for j in range(N):
                c[(i + j) % N] += ai[i] * bi[j]
        fc = O.pointwise(pl.fwd(a.astype(np.float64)), pl.fwd(b.astype(np.float64)), 0)
        fc = pl.rev(fc)
        got = [canon(L.orc_fp_mulmod4(fc[(N - j) % N], pl.ninv, pl.ninvp, 0), P1) for j in range(N)]
        assert got == [v % P1 for v in c]


def test_tables_minimal_balanced():
    # every stored constant and twiddle is minimal balanced (fpntt.jl:113-121, :170-186)
    for N in (4032, 3840, 1680, 105 * 16, 315 * 4):
        for f, P in ((0, P1), (1, P2)):
            for st in O.Plan(N, f).stages():
                if st["tw"] is not None:
                    assert np.all(np.abs(st["tw"]) <= P / 2)
                if st["m"] in (5, 7):
                    assert all(abs(v) <= P / 2 for v in st["rot"][: st["m"] - 1 if st["m"] == 5 else 8])


def test_garner_unpack_crt():
    # test/test_fpntt.jl:257-286: unreduced either-sign representatives
    rng = np.random.default_rng(0x6A3)
    L = O.lib()
    for b in (33, 40, 44, 48):
        for nconv in (1, 7, 64, 200):
            cs = [int.from_bytes(rng.bytes(13), "little") % (P1 * P2) for _ in range(nconv)]
            N = nconv + int(rng.integers(0, 6))
            x1 = np.zeros(N)
            x2 = np.zeros(N)
            for i, c in enumerate(cs):
                idx = (N - i) % N
                x1[idx] = float((c * N) % P1) + float(rng.integers(-2, 3)) * float(P1)
                x2[idx] = float((c * N) % P2) + float(rng.integers(-2, 3)) * float(P2)
            n1 = L.orc_fp_reduce(float(pow(N, -1, P1)), 0)
            n2 = L.orc_fp_reduce(float(pow(N, -1, P2)), 1)
            rn = -(-(99 + b * (nconv - 1)) // 64) + 1
            r = O.unpack2(rn, x1, x2, nconv, b, n1, n1 / float(P1), n2, n2 / float(P2))
            assert O.to_int(r) == sum(c << (b * i) for i, c in enumerate(cs))


SHAPES = ((1, 1), (5, 3), (16, 16), (100, 100), (255, 257), (500, 300), (601, 373), (1024, 1024),
          (2500, 2500), (5000, 4900))


def test_differential_vs_gmp():
    # test/test_fpntt.jl:288-300 against GMP mpn_mul (= Julia BigInt)
    rng = np.random.default_rng(0x91C4)
    for na, nb in SHAPES:
        for _ in range(2 if na * nb > 10**5 else 6):
            a, b = adversarial(rng, na), adversarial(rng, nb)
            assert np.array_equal(O.mul(a, b), O.gmp_mul(a, b)), (na, nb)


def test_all_ones_max_chunk_width():
    # test/test_fpntt.jl:301-307: b = 49 with max-magnitude coefficients
    for na in range(1, 9):
        for nb in range(1, na + 1):
            a = np.full(na, 2**64 - 1, dtype=np.uint64)
            b = np.full(nb, 2**64 - 1, dtype=np.uint64)
            assert np.array_equal(O.mul(a, b), O.gmp_mul(a, b))
    assert O.ntt_params(64, 64)[0] == 49


def test_squares_vs_gmp():
    # test/test_fpntt.jl:326-330
    rng = np.random.default_rng(0x5F2E)
    for n in (1, 7, 100, 1024, 3000):
        a = adversarial(rng, n)
        assert np.array_equal(O.sqr(a), O.gmp_sqr(a))
    a = np.full(6, 2**64 - 1, dtype=np.uint64)
    assert np.array_equal(O.sqr(a), O.gmp_sqr(a))


def _limbmod(x: np.ndarray, m: int) -> int:
    r = 0
    for v in x[::-1]:
        r = ((r << 64) | int(v)) % m
    return r


def test_large_radix7_residues():
    # test/test_fpntt.jl:308-325: 144,000 limbs on a 7*2^k length, residues mod 63-bit moduli
    rng = np.random.default_rng(0x7777)
    n = 144_000
    a, b = rand_limbs(rng, n), rand_limbs(rng, n)
    r = O.mul(a, b)
    for m in rng.integers(2**62, 2**63 - 1, 4, dtype=np.int64):
        m = int(m)
        assert _limbmod(r, m) == (_limbmod(a, m) * _limbmod(b, m)) % m


def test_op_count_matches_schedule():
    # counting build: per-stage FP64 op counts (ops per butterfly: r4 40, r2 10,
    # r3 32, r5 94 fwd / 98 rev, r7 173 fwd / 201 rev; pointwise 7; unpack 28 per coefficient)
    rng = np.random.default_rng(3)
    a = rand_limbs(rng, 4096)
    N = 12288
    stages = O.Plan(N, 0).stages()
    per = {2: (10, 10), 3: (32, 32), 4: (40, 40), 5: (94, 98), 7: (173, 201)}
    fwd = sum(per[s["m"]][0] * N // s["m"] for s in stages)
    rev = sum(per[s["m"]][1] * N // s["m"] for s in stages)
    b, _ = O.ntt_params(64 * 4096, 64 * 4096)
    nconv = 2 * (-(-O.magnitude_bits(a) // b)) - 1
    want_sqr = 2 * (fwd + 7 * N + rev) + 28 * nconv
    assert O.op_count_product(a, None) == want_sqr
    # a 7*5*3*2^11 length exercises the radix-5/7 counts (mul: two forward transforms)
    a, b = rand_limbs(rng, 2**16), rand_limbs(rng, 2**16)
    bch, N = O.ntt_params(O.magnitude_bits(a), O.magnitude_bits(b))
    assert N == 105 * 2**11
    stages = O.Plan(N, 0).stages()
    assert [s["m"] for s in stages[:3]] == [7, 5, 3]
    fwd = sum(per[s["m"]][0] * N // s["m"] for s in stages)
    rev = sum(per[s["m"]][1] * N // s["m"] for s in stages)
    nconv = -(-O.magnitude_bits(a) // bch) + -(-O.magnitude_bits(b) // bch) - 1
    assert O.op_count_product(a, b) == 2 * (2 * fwd + 7 * N + rev) + 28 * nconv
