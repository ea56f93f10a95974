"""Host-side checks of libnbgpu.so that need no GPU: the library loads,
exports every symbol include/nbgpu.h declares, its admission restatement
agrees with the oracle, and argument errors come back as status codes."""
import ctypes
import os
import re

import numpy as np
import pytest

import nbgpu
import oracle as O
from conftest import ROOT, rand_limbs


def _declared_symbols() -> list[str]:
    src = open(os.path.join(ROOT, "include", "nbgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(nbg_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = nbgpu.lib()
    syms = _declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(nbgpu.EXPORTS)


def test_ntt_len_matches_oracle():
    for T in list(range(1, 5000, 7)) + [15 << 14, (15 << 14) + 1, 7 << 10, 9 << 10, (1 << 34) + 1,
                                       33 << 34, 53 << 34, 315 << 34]:
        assert nbgpu.ntt_len(T) == O.ntt_len(T)
    with pytest.raises(nbgpu.LengthError):
        nbgpu.ntt_len((315 << 34) + 1)


def test_ntt_params_matches_oracle():
    rng = np.random.default_rng(11)
    cases = [(1, 1), (64, 64), (64 * 4096, 64 * 4096), (64 * 2**24, 64 * 2**24), (9728, 64 * 65536)]
    cases += [(int(rng.integers(1, 2**28)), int(rng.integers(1, 2**28))) for _ in range(2000)]
    for ba, bb in cases:
        assert nbgpu.ntt_params(ba, bb) == O.ntt_params(ba, bb)


def test_magnitude_bits():
    rng = np.random.default_rng(12)
    for n in (1, 2, 5, 100):
        a = rand_limbs(rng, n)
        assert nbgpu.magnitude_bits(a) == O.magnitude_bits(a) == O.to_int(a).bit_length()


def test_argument_errors_without_device():
    L = nbgpu.lib()
    r = np.zeros(4, dtype=np.uint64)
    a = np.ones(2, dtype=np.uint64)
    assert L.nbg_mul(r.ctypes.data, a.ctypes.data, 2, None, 2) == nbgpu.NBG_EINVAL
    assert L.nbg_mul(r.ctypes.data, a.ctypes.data, 0, a.ctypes.data, 2) == nbgpu.NBG_EINVAL
    # r aliasing an operand is rejected (src/fpntt.jl:979-981)
    assert L.nbg_mul(a.ctypes.data, a.ctypes.data, 2, a.ctypes.data, 2) == nbgpu.NBG_EINVAL
    assert L.nbg_sqr(None, a.ctypes.data, 2) == nbgpu.NBG_EINVAL
    assert L.nbg_mul(a.ctypes.data, a.ctypes.data, 2, r.ctypes.data, 1) == nbgpu.NBG_EINVAL
    assert b"alias" in L.nbg_last_error()
    N = ctypes.c_int64()
    assert L.nbg_ntt_len(0, ctypes.byref(N)) == nbgpu.NBG_EINVAL
    assert L.nbg_ntt_len((315 << 34) + 1, ctypes.byref(N)) == nbgpu.NBG_ERANGE
    assert L.nbg_last_error()


def test_tuning_round_trip():
    old = nbgpu.get_tuning()
    try:
        nbgpu.set_tuning('{"last_max": 2048, "cmax": 64, "queue": 4}')
        t = nbgpu.get_tuning()
        assert '"last_max": 2048' in t and '"cmax": 64' in t and '"queue": 4' in t
        with pytest.raises(nbgpu.NBGError):
            nbgpu.set_tuning('{"cmax": 3}')
        with pytest.raises(nbgpu.NBGError):
            nbgpu.set_tuning('{"queue": 65}')
    finally:
        nbgpu.set_tuning(old)
    assert nbgpu.get_tuning() == old


def test_dispatch_thresholds():
    # mul! admits the NTT at n >= 64 and m + n >= 304 (src/mul.jl:388); sqr! at n >= 160 (:146)
    assert nbgpu.uses_fpntt_mul(152, 152) and not nbgpu.uses_fpntt_mul(151, 152)
    assert nbgpu.uses_fpntt_mul(1000, 64) and not nbgpu.uses_fpntt_mul(1000, 63)
    assert nbgpu.uses_fpntt_sqr(160) and not nbgpu.uses_fpntt_sqr(159)


# ---------------------------------------------------------------------------
# Index arithmetic of the pass kernels, emulated on the CPU: every tile's loads
# stay inside [0, N), each pass covers every element exactly once, and every
# butterfly a tile runs is the reference's butterfly (same global lanes, same
# twiddle column) for its stage (fp_stage!, src/fpntt.jl:703-713).

def _pad(i):
    return i + (i >> 4)


def _stride(n):
    return ((n + (n >> 4) + 1) + 1) & ~1


def _emulate_plan(N, layout):
    """Emulates the pass kernels' index arithmetic (round_gen, round_r16,
    round_r8, tile loads/stores) with numpy and checks it against the
    reference's enumeration of butterflies."""
    stages, passes, rounds = layout["stages"], layout["passes"], layout["rounds"]
    seen = {s: [] for s in range(len(stages))}
    for (sa, sb, G, C, Qb, ntiles), rds in zip(passes, rounds):
        assert C & (C - 1) == 0 and Qb % C == 0 and 2 * _stride(G * C) * 8 <= 220 * 1024
        La = stages[sa][1]
        assert La % Qb == 0 and La // Qb == G
        per = Qb // C
        t = np.arange(ntiles, dtype=np.int64)
        blk, jc = t // per, t % per
        j0 = jc * C
        tbase = blk * La + j0
        k = np.arange(G, dtype=np.int64)[:, None]
        c = np.arange(C, dtype=np.int64)[None, :]
        idx = tbase[:, None, None] + c[None] + k[None] * Qb
        assert idx.min() >= 0 and idx.max() < N
        assert np.array_equal(np.sort(idx.ravel()), np.arange(N))
        lc = C.bit_length() - 1
        ntile_elems = G * C
        assert _pad(ntile_elems - 1) < _stride(ntile_elems)

        def glob(local):  # tile-local element index -> global index, per tile
            assert local.min() >= 0 and local.max() < ntile_elems
            assert _pad(local).max() < _stride(ntile_elems)
            kk, c2 = local >> lc, local & (C - 1)
            return tbase[:, None] + c2[None, :] + kk[None, :] * Qb

        def check(s, lanes, jcol):
            m, Ls, Qs = stages[s]
            g0 = lanes[0]
            assert np.array_equal(g0 % Ls, jcol) and jcol.max() < Qs
            for tl in range(1, m):
                assert np.array_equal(lanes[tl], g0 + tl * Qs)
            seen[s].append(g0.ravel())

        stage_set = set()
        for kind, s in rds:
            if kind in ("odd", "r4", "r2"):
                m, Ls, Qs = stages[s]
                Lloc, Qloc = Ls // Qb, Qs // Qb
                e = np.arange((G // m) * C, dtype=np.int64)
                cc, row = e & (C - 1), e >> lc
                # multiply-high division of the kernel: (row >> e2) * mg >> 32
                e2 = (Qloc & -Qloc).bit_length() - 1
                odd = Qloc >> e2
                rs = row >> e2
                if odd == 1:
                    bl = rs
                else:
                    mg = (0xFFFFFFFF // odd) + 1
                    bl = (rs * mg) >> 32
                assert np.array_equal(bl, row // Qloc)
                jl = row - bl * Qloc
                lb = ((bl * Lloc + jl) << lc) + cc
                lanes = [glob(lb + tl * (Qloc << lc)) for tl in range(m)]
                jcol = (jl * Qb)[None, :] + j0[:, None] + cc[None, :]
                check(s, lanes, jcol)
                stage_set.add(s)
            elif kind == "r16":
                mA, LA, QA = stages[s]
                mB, LB, QB = stages[s + 1]
                assert mA == 4 and mB == 4 and LB * 4 == LA
                Lloc = LA // Qb
                q16 = Lloc >> 4
                assert q16 >= 1 and q16 & (q16 - 1) == 0
                lq = q16.bit_length() - 1
                e = np.arange((G >> 4) * C, dtype=np.int64)
                cc, r = e & (C - 1), e >> lc
                b, j2 = r >> lq, r & (q16 - 1)
                row0 = b * Lloc + j2
                loc = lambda t1, t2: ((row0 + t1 * 4 * q16 + t2 * q16) << lc) + cc
                for t2 in range(4):
                    lanes = [glob(loc(t1, t2)) for t1 in range(4)]
                    jA = ((j2 + t2 * q16) * Qb)[None, :] + j0[:, None] + cc[None, :]
                    check(s, lanes, jA)
                for t1 in range(4):
                    lanes = [glob(loc(t1, t2)) for t2 in range(4)]
                    jB = (j2 * Qb)[None, :] + j0[:, None] + cc[None, :]
                    check(s + 1, lanes, jB)
                stage_set |= {s, s + 1}
            elif kind == "r8":
                assert C == 1 and Qb == 1
                mA, LA, QA = stages[s]
                assert (mA, LA, QA) == (4, 8, 2) and stages[s + 1][0] == 2
                b = np.arange(G >> 3, dtype=np.int64)
                for j in range(2):
                    lanes = [glob(8 * b + j + 2 * tl) for tl in range(4)]
                    check(s, lanes, np.full((ntiles, b.size), j))
                for i in range(4):
                    lanes = [glob(8 * b + 2 * i + tl) for tl in range(2)]
                    check(s + 1, lanes, np.zeros((ntiles, b.size), dtype=np.int64))
                stage_set |= {s, s + 1}
            else:
                raise AssertionError(kind)
        assert stage_set == set(range(sa, sb + 1))
    for s, (m, Ls, Qs) in enumerate(stages):
        g0 = np.sort(np.concatenate(seen[s]))
        # every butterfly of the stage exactly once: lane-0 indices o + j, o = k*L, j < Q
        want = (np.arange(N // Ls)[:, None] * Ls + np.arange(Qs)[None, :]).ravel()
        assert np.array_equal(g0, np.sort(want)), s
    assert passes[-1][4] == 1 and passes[-1][1] == len(stages) - 1


EMU_N = (4, 8, 12, 48, 240, 420, 1260, 4032, 960, 1680, 12288, 20480, 7 * 2**15, 9 * 2**11, 105 * 2**11,
         2**16, 315 * 2**10, 63 * 2**12, 45 * 2**11, 2**17 * 3)
EMU_TUNINGS = (None,
               '{"full_max_mul": 4, "full_max_sqr": 4, "last_max": 4, "last_max_sqr": 4, "early_gmax": 2, "tile_target": 8, "cmax": 2}',
               '{"full_max_mul": 16, "full_max_sqr": 16, "last_max": 64, "last_max_sqr": 32, "early_gmax": 16, "tile_target": 64, "cmax": 8}',
               '{"full_max_mul": 256, "full_max_sqr": 256, "last_max": 256, "last_max_sqr": 512, "early_gmax": 64, "tile_target": 512, "cmax": 32}',
               '{"full_max_mul": 4096, "full_max_sqr": 8192, "last_max": 4096, "last_max_sqr": 8192, "early_gmax": 1024, "tile_target": 4096, "cmax": 128}')


@pytest.mark.parametrize("tun", EMU_TUNINGS)
def test_pass_index_emulation(tun):
    old = nbgpu.get_tuning()
    try:
        if tun:
            nbgpu.set_tuning(tun)
        for N in EMU_N:
            for sqr in (False, True):
                _emulate_plan(N, nbgpu.plan_layout(N, sqr))
    finally:
        nbgpu.set_tuning(old)


def test_large_plan_layouts():
    for N in (7 * 2**19, 7 * 2**23, 315 * 2**14, 315 * 2**17, 2**26):
        lay = nbgpu.plan_layout(N)
        assert 2 <= len(lay["passes"]) <= 6
        for (sa, sb, G, C, Qb, nt) in lay["passes"]:
            assert 4 * _stride(G * C) * 8 <= 227 * 1024
    _emulate_plan(315 * 2**14, nbgpu.plan_layout(315 * 2**14))


def test_unpack_tile_coefficient_ranges():
    # k_unpack: coefficients overlapping limbs [w0-1, w0+1024) fit its shared
    # memory and index x[(N - i) mod N] inside [0, N)
    TL = 1024
    for bits, b in ((64 * 4096, 43), (64 * 2**16, 41), (64, 49), (64 * 5, 48), (64 * 2**20, 39)):
        nconv = 2 * (-(-bits // b)) - 1
        rn = 2 * (-(-bits // 64))
        N = nbgpu.ntt_len(nconv)
        ncoef_cap = (64 * (TL + 2) + 100) // b + 4
        for tile in range(-(-rn // TL)):
            w0, w1 = tile * TL, min(tile * TL + TL, rn)
            wlo = max(w0 - 1, 0)
            a = 64 * wlo - 99
            ilo = 0 if a <= 0 else -(-a // b)
            ihi = min((64 * (w1 - 1) + 63) // b, nconv - 1)
            assert ihi - ilo + 1 <= ncoef_cap
            assert 0 <= ilo and ihi < N
            for w in (wlo, w1 - 1):
                lo_i = max(0, -(-(64 * w - 99) // b))
                hi_i = (64 * w + 63) // b
                assert lo_i >= ilo and min(hi_i, nconv - 1) <= ihi


def test_autotune_candidates_emulate_cleanly():
    # every split the autotuner may time is a valid plan whose kernels stay in bounds
    import json

    from nbgpu import autotune

    old = nbgpu.get_tuning()
    try:
        for N, sq in ((2048, False), (4096, True), (6144, False), (12288, True), (24576, False),
                      (105 * 2**11, False), (7 * 2**15, True), (315 * 2**10, False)):
            for cand in autotune.candidates(N, sq):
                base = json.loads(old)
                base["overrides"] = [dict(cand, N=N, sqr=int(sq))]
                nbgpu.set_tuning(json.dumps(base))
                lay = nbgpu.plan_layout(N, sq)
                assert [p[1] for p in lay["passes"]] == cand["pass_ends"]
                _emulate_plan(N, lay)
    finally:
        nbgpu.set_tuning(old)


def test_odd_multiplier_landings():
    """Balanced sizes that land on each odd transform-length multiplier (the
    single-product configuration's list), by the oracle and the library."""
    import nbgpu

    for n, N in ((4096, 3 * 2**12), (6200, 5 * 2**12), (9032, 7 * 2**12), (5512, 9 * 2**11),
                 (110336, 3 * 2**17), (94592, 5 * 2**16), (68992, 7 * 2**15), (84096, 9 * 2**15),
                 (1439744, 315 * 2**14), (10928128, 315 * 2**17)):
        assert O.ntt_params(64 * n, 64 * n)[1] == N
        assert nbgpu.ntt_params(64 * n, 64 * n)[1] == N


def test_column_major_tile_order_is_a_permutation():
    """Column passes visit tile t_lin = jc * nblk + blk as tile blk * per + jc
    (job segments, types.h job_at): every tile once, and runs of consecutive
    visits share the column jc (hence the twiddle columns)."""
    rng = np.random.default_rng(3)
    for _ in range(50):
        per = int(rng.integers(2, 300))
        nblk = int(rng.integers(2, 300))
        n = per * nblk
        seen = [(t % nblk) * per + t // nblk for t in range(n)]
        assert sorted(seen) == list(range(n))
        # within a run of nblk consecutive visits the column index is fixed
        for t0 in range(0, n, nblk):
            assert len({seen[t] % per for t in range(t0, t0 + nblk)}) == 1


def test_argument_errors_of_the_caller_entry_points():
    """The powermod, radix, low-half and sum-of-products entry points reject bad
    arguments before they touch a device."""
    L = nbgpu.lib()
    one = np.ones(4, dtype=np.uint64)
    r = np.zeros(4, dtype=np.uint64)
    # powermod: base longer than the modulus, zero-length exponent
    d = (nbgpu.PowmodDesc * 1)()
    d[0] = nbgpu.PowmodDesc(r.ctypes.data, one.ctypes.data, one.ctypes.data, one.ctypes.data, 3, 1)
    assert L.nbg_powermod_batch(ctypes.cast(d, ctypes.c_void_p), 1, 2) == nbgpu.NBG_EINVAL
    d[0] = nbgpu.PowmodDesc(r.ctypes.data, one.ctypes.data, one.ctypes.data, one.ctypes.data, 1, 0)
    assert L.nbg_powermod_batch(ctypes.cast(d, ctypes.c_void_p), 1, 2) == nbgpu.NBG_EINVAL
    assert L.nbg_powermod_batch(None, 1, 2) == nbgpu.NBG_EINVAL
    # radix combine: a chunk not below the base, too small an output
    ln = ctypes.c_int64()
    c = np.array([3, 10], dtype=np.uint64)
    assert L.nbg_radix_combine(r.ctypes.data, 4, c.ctypes.data, 2, 10, ctypes.byref(ln)) == nbgpu.NBG_EINVAL
    assert L.nbg_radix_combine(r.ctypes.data, 1, c.ctypes.data, 2, 100, ctypes.byref(ln)) == nbgpu.NBG_EINVAL
    assert L.nbg_radix_combine(r.ctypes.data, 4, c.ctypes.data, 2, 1, ctypes.byref(ln)) == nbgpu.NBG_EINVAL
    # sums of products: r too short, null matrix entries
    assert L.nbg_mul2add_dev(r.ctypes.data, 3, one.ctypes.data, 2, one.ctypes.data, 2, one.ctypes.data, 1,
                             one.ctypes.data, 1, None) == nbgpu.NBG_EINVAL
    m4 = (ctypes.c_void_p * 4)(None, None, None, None)
    assert L.nbg_matrix22_mul_dev(m4, 1, m4, 1, None) == nbgpu.NBG_EINVAL
    # low halves: null operand, k < 1
    assert L.nbg_mullo(r.ctypes.data, one.ctypes.data, 2, None, 2, 2) == nbgpu.NBG_EINVAL
