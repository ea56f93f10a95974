"""Python handle on the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as a checker or as the timed CPU baseline.
The product library never calls it.

Two independent checkers live here:

* ``liboracle.so`` — a plain-C restatement of the reference engine
  (NativeBigInt.jl ``src/fpntt.jl``), scalar and bit-exact in every
  intermediate double (see ``fpntt_oracle.c``).
* GMP 6.3 (``libgmp.so.10``) ``mpn_mul`` / ``mpn_sqr`` through ctypes — the
  arithmetic Julia's ``BigInt`` uses, so it pins the final products.

Parity is pinned: ``tests/test_oracle.py`` checks the restatement against
the reference's known-answer tables (test/test_fpntt.jl) and against GMP.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")

P1 = 65205 * 2**34 + 1  # src/fpntt.jl:78
P2 = 4095 * 2**38 + 1  # src/fpntt.jl:79

_u64p = ctypes.POINTER(ctypes.c_uint64)
_dblp = ctypes.POINTER(ctypes.c_double)


def build() -> None:
    """Compile the oracle libraries (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _declare(lib: ctypes.CDLL) -> ctypes.CDLL:
    c = ctypes
    sig = {
        "orc_prime": (c.c_uint64, [c.c_int]),
        "orc_generator": (c.c_uint64, [c.c_int]),
        "orc_two_adicity": (c.c_int, [c.c_int]),
        "orc_fp_round": (c.c_double, [c.c_double]),
        "orc_fp_reduce": (c.c_double, [c.c_double, c.c_int]),
        "orc_fp_mulmod3": (c.c_double, [c.c_double, c.c_double, c.c_int]),
        "orc_fp_mulmod4": (c.c_double, [c.c_double, c.c_double, c.c_double, c.c_int]),
        "orc_fp_minbal": (c.c_double, [c.c_double, c.c_int]),
        "orc_plan_build": (c.c_void_p, [c.c_int64, c.c_int]),
        "orc_plan_get": (c.c_void_p, [c.c_int64, c.c_int]),
        "orc_plan_free": (None, [c.c_void_p]),
        "orc_plan_nstages": (c.c_int, [c.c_void_p]),
        "orc_plan_N2": (c.c_int64, [c.c_void_p]),
        "orc_plan_ninv": (c.c_double, [c.c_void_p]),
        "orc_plan_ninvp": (c.c_double, [c.c_void_p]),
        "orc_plan_stage": (c.c_int, [c.c_void_p, c.c_int, c.POINTER(c.c_int64), c.POINTER(c.c_int64),
                                     c.POINTER(c.c_int64), _dblp]),
        "orc_plan_stage_tw": (_dblp, [c.c_void_p, c.c_int]),
        "orc_stage_run": (None, [_dblp, c.c_void_p, c.c_int, c.c_int]),
        "orc_ntt_fwd": (None, [_dblp, c.c_void_p]),
        "orc_ntt_rev": (None, [_dblp, c.c_void_p]),
        "orc_pack": (None, [_dblp, c.c_int64, _u64p, c.c_int64, c.c_int, c.c_int64]),
        "orc_pointwise": (None, [_dblp, _dblp, c.c_int64, c.c_int]),
        "orc_unpack2": (None, [_u64p, c.c_int64, _dblp, _dblp, c.c_int64, c.c_int64, c.c_int,
                               c.c_double, c.c_double, c.c_double, c.c_double]),
        "orc_magnitude_bits": (c.c_int64, [_u64p, c.c_int64]),
        "orc_ntt_len": (c.c_int64, [c.c_int64]),
        "orc_ntt_params": (c.c_int, [c.c_int64, c.c_int64, c.POINTER(c.c_int), c.POINTER(c.c_int64)]),
        "orc_mul_fpntt2": (c.c_int, [_u64p, _u64p, c.c_int64, _u64p, c.c_int64]),
        "orc_sqr_fpntt2": (c.c_int, [_u64p, _u64p, c.c_int64]),
        "orc_barrett_mu": (c.c_int64, [_u64p, c.c_int64, _u64p]),
        "orc_powmod_barrett": (c.c_int, [_u64p, _u64p, c.c_int64, _u64p, c.c_int64, _u64p, c.c_int64]),
        "orc_op_count": (c.c_uint64, []),
        "orc_op_count_reset": (None, []),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_LIBS: dict[str, ctypes.CDLL] = {}


def lib(counting: bool = False) -> ctypes.CDLL:
    name = "liboracle_count.so" if counting else "liboracle.so"
    if name not in _LIBS:
        path = os.path.join(_BUILD, name)
        if not os.path.exists(path):
            build()
        _LIBS[name] = _declare(ctypes.CDLL(path))
    return _LIBS[name]


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


# --------------------------------------------------------------------------
# Thin Pythonic wrappers (arrays are numpy; limbs uint64 little-endian)

def ntt_len(T: int) -> int:
    """ntt_len (src/fpntt.jl:936-951); raises ValueError past 315*2^34."""
    n = lib().orc_ntt_len(T)
    if n < 0:
        raise ValueError(f"fp NTT length {T} exceeds the 315*2^34 the primes support")
    return n


def ntt_params(bits_a: int, bits_b: int) -> tuple[int, int]:
    """fp_ntt_params (src/fpntt.jl:964-977) -> (b, N)."""
    b = ctypes.c_int()
    N = ctypes.c_int64()
    rc = lib().orc_ntt_params(bits_a, bits_b, ctypes.byref(b), ctypes.byref(N))
    if rc:
        raise ValueError("length unsupported")
    return b.value, N.value


def magnitude_bits(a: np.ndarray) -> int:
    return lib().orc_magnitude_bits(_p(a, _u64p), len(a))


class Plan:
    """An oracle plan for (N, prime index f) — build_fp_plan (src/fpntt.jl:236-271)."""

    def __init__(self, N: int, f: int, counting: bool = False):
        self._lib = lib(counting)
        self.ptr = self._lib.orc_plan_build(N, f)
        if not self.ptr:
            raise ValueError(f"no plan for N={N}")
        self.N, self.f = N, f

    def __del__(self):
        if getattr(self, "ptr", None):
            self._lib.orc_plan_free(self.ptr)
            self.ptr = None

    @property
    def ninv(self) -> float:
        return self._lib.orc_plan_ninv(self.ptr)

    @property
    def ninvp(self) -> float:
        return self._lib.orc_plan_ninvp(self.ptr)

    @property
    def N2(self) -> int:
        return self._lib.orc_plan_N2(self.ptr)

    def stages(self) -> list[dict]:
        out = []
        for i in range(self._lib.orc_plan_nstages(self.ptr)):
            span, Q, twlen = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
            rot = (ctypes.c_double * 8)()
            m = self._lib.orc_plan_stage(self.ptr, i, ctypes.byref(span), ctypes.byref(Q), ctypes.byref(twlen), rot)
            tw = None
            if m != 2:
                ptr = self._lib.orc_plan_stage_tw(self.ptr, i)
                tw = np.ctypeslib.as_array(ptr, shape=((m - 1) * twlen.value,)).copy().reshape(m - 1, twlen.value)
            out.append(dict(m=m, span=span.value, Q=Q.value, twlen=twlen.value, rot=list(rot), tw=tw))
        return out

    def fwd(self, x: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(x, dtype=np.float64).copy()
        self._lib.orc_ntt_fwd(_p(y, _dblp), self.ptr)
        return y

    def rev(self, x: np.ndarray) -> np.ndarray:
        y = np.ascontiguousarray(x, dtype=np.float64).copy()
        self._lib.orc_ntt_rev(_p(y, _dblp), self.ptr)
        return y

    def stage(self, x: np.ndarray, i: int, fwd: bool) -> np.ndarray:
        y = np.ascontiguousarray(x, dtype=np.float64).copy()
        self._lib.orc_stage_run(_p(y, _dblp), self.ptr, i, 1 if fwd else 0)
        return y


def pack(limbs: np.ndarray, N: int, b: int, nch: int) -> np.ndarray:
    x = np.empty(N, dtype=np.float64)
    limbs = np.ascontiguousarray(limbs, dtype=np.uint64)
    lib().orc_pack(_p(x, _dblp), N, _p(limbs, _u64p), len(limbs), b, nch)
    return x


def pointwise(xa: np.ndarray, xb: np.ndarray, f: int) -> np.ndarray:
    y = np.ascontiguousarray(xa, dtype=np.float64).copy()
    xb = np.ascontiguousarray(xb, dtype=np.float64)
    lib().orc_pointwise(_p(y, _dblp), _p(xb, _dblp), len(y), f)
    return y


def unpack2(rn: int, x1: np.ndarray, x2: np.ndarray, nconv: int, b: int,
            n1: float, n1p: float, n2: float, n2p: float) -> np.ndarray:
    r = np.zeros(rn, dtype=np.uint64)
    x1 = np.ascontiguousarray(x1, dtype=np.float64)
    x2 = np.ascontiguousarray(x2, dtype=np.float64)
    lib().orc_unpack2(_p(r, _u64p), rn, _p(x1, _dblp), _p(x2, _dblp), len(x1), nconv, b, n1, n1p, n2, n2p)
    return r


def mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """mul_fpntt2! (src/fpntt.jl:982-1014): len(a)+len(b) output limbs."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    r = np.empty(len(a) + len(b), dtype=np.uint64)
    rc = lib().orc_mul_fpntt2(_p(r, _u64p), _p(a, _u64p), len(a), _p(b, _u64p), len(b))
    if rc:
        raise ValueError(f"oracle mul failed rc={rc}")
    return r


def sqr(a: np.ndarray) -> np.ndarray:
    """sqr_fpntt2! (src/fpntt.jl:1016-1037): 2*len(a) output limbs."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    r = np.empty(2 * len(a), dtype=np.uint64)
    rc = lib().orc_sqr_fpntt2(_p(r, _u64p), _p(a, _u64p), len(a))
    if rc:
        raise ValueError(f"oracle sqr failed rc={rc}")
    return r


# --------------------------------------------------------------------------
# GMP (independent checker)

_GMP = None


def gmp() -> ctypes.CDLL:
    global _GMP
    if _GMP is None:
        path = ctypes.util.find_library("gmp") or "libgmp.so.10"
        g = ctypes.CDLL(path)
        g.__gmpn_mul.restype = ctypes.c_uint64
        g.__gmpn_mul.argtypes = [_u64p, _u64p, ctypes.c_long, _u64p, ctypes.c_long]
        g.__gmpn_sqr.restype = None
        g.__gmpn_sqr.argtypes = [_u64p, _u64p, ctypes.c_long]
        _GMP = g
    return _GMP


def gmp_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """mpn_mul (requires len(a) >= len(b) >= 1; swapped here if needed)."""
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    if len(a) < len(b):
        a, b = b, a
    r = np.zeros(len(a) + len(b), dtype=np.uint64)
    gmp().__gmpn_mul(_p(r, _u64p), _p(a, _u64p), len(a), _p(b, _u64p), len(b))
    return r


class _Mpz(ctypes.Structure):
    _fields_ = [("alloc", ctypes.c_int), ("size", ctypes.c_int), ("d", ctypes.c_void_p)]


def _mpz_from(g, z: _Mpz, a: np.ndarray) -> None:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    g.__gmpz_import(ctypes.byref(z), ctypes.c_size_t(a.size), -1, 8, 0, 0, a.ctypes.data_as(ctypes.c_void_p))


def gmp_powm(b: np.ndarray, e: np.ndarray, m: np.ndarray) -> np.ndarray:
    """b^e mod m through GMP's mpz_powm; the result as m.size limbs.  ctypes
    releases the GIL, so independent calls run in parallel threads."""
    g = gmp()
    zs = [_Mpz() for _ in range(4)]
    for z in zs:
        g.__gmpz_init(ctypes.byref(z))
    try:
        _mpz_from(g, zs[0], b)
        _mpz_from(g, zs[1], e)
        _mpz_from(g, zs[2], m)
        g.__gmpz_powm(ctypes.byref(zs[3]), ctypes.byref(zs[0]), ctypes.byref(zs[1]), ctypes.byref(zs[2]))
        out = np.zeros(max(int(np.asarray(m).size), 1) + 1, dtype=np.uint64)
        cnt = ctypes.c_size_t(0)
        g.__gmpz_export(out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(cnt), -1, 8, 0, 0, ctypes.byref(zs[3]))
        return out[: np.asarray(m).size].copy()
    finally:
        for z in zs:
            g.__gmpz_clear(ctypes.byref(z))


def gmp_sqr(a: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    r = np.zeros(2 * len(a), dtype=np.uint64)
    gmp().__gmpn_sqr(_p(r, _u64p), _p(a, _u64p), len(a))
    return r


def barrett_mu(m: np.ndarray) -> np.ndarray:
    """barrett_mu! (src/barrett.jl:22-31): floor(2^(128k) / m), k + 2 limbs."""
    m = np.ascontiguousarray(m, dtype=np.uint64)
    mu = np.zeros(m.size + 2, dtype=np.uint64)
    lib().orc_barrett_mu(_p(m, _u64p), m.size, _p(mu, _u64p))
    return mu


def powmod_barrett(b: np.ndarray, e: np.ndarray, m: np.ndarray) -> np.ndarray:
    """powermod_limbs on its Barrett branch (src/algorithms.jl:17-107):
    b^e mod m, k = len(m) limbs, every product through the fp NTT."""
    b = np.ascontiguousarray(b, dtype=np.uint64)
    e = np.ascontiguousarray(e, dtype=np.uint64)
    m = np.ascontiguousarray(m, dtype=np.uint64)
    r = np.zeros(m.size, dtype=np.uint64)
    rc = lib().orc_powmod_barrett(_p(r, _u64p), _p(b, _u64p), b.size, _p(e, _u64p), e.size, _p(m, _u64p), m.size)
    if rc:
        raise ValueError("powmod_barrett: bad arguments")
    return r


def op_count_product(a: np.ndarray, b: np.ndarray | None) -> int:
    """Algorithmic FP64 op count (DADD/DMUL/DFMA) of one product on the
    reference schedule, measured by the counting build of the oracle."""
    L = lib(counting=True)
    a = np.ascontiguousarray(a, dtype=np.uint64)
    bits_a = L.orc_magnitude_bits(_p(a, _u64p), len(a))
    bits_b = bits_a if b is None else L.orc_magnitude_bits(_p(np.ascontiguousarray(b, dtype=np.uint64), _u64p), len(b))
    bb = ctypes.c_int()
    N = ctypes.c_int64()
    L.orc_ntt_params(bits_a, bits_b, ctypes.byref(bb), ctypes.byref(N))
    L.orc_plan_get(N.value, 0)  # plan construction is not counted
    L.orc_plan_get(N.value, 1)
    L.orc_op_count_reset()
    if b is None:
        r = np.empty(2 * len(a), dtype=np.uint64)
        L.orc_sqr_fpntt2(_p(r, _u64p), _p(a, _u64p), len(a))
    else:
        b = np.ascontiguousarray(b, dtype=np.uint64)
        r = np.empty(len(a) + len(b), dtype=np.uint64)
        L.orc_mul_fpntt2(_p(r, _u64p), _p(a, _u64p), len(a), _p(b, _u64p), len(b))
    return int(L.orc_op_count())


# --------------------------------------------------------------------------
# Small helpers shared by the tests

def to_int(limbs: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(limbs, dtype="<u8").tobytes(), "little")


def from_int(v: int, n: int) -> np.ndarray:
    return np.frombuffer(v.to_bytes(8 * n, "little"), dtype="<u8").astype(np.uint64)
