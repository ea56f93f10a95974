"""Python host binding of libnbgpu.so (ctypes), mirroring the reference's
mpn multiply interface for the fp-NTT path.

Reference interface (NativeBigInt.jl):
  mul!(r, ro, a, ao, m, b, bo, n)   src/mul.jl:383   (NTT branch :388-390)
  sqr!(r, ro, a, ao, n)             src/mul.jl:141   (NTT branch :146)
  mul_fpntt2! / sqr_fpntt2!         src/fpntt.jl:982 / :1016
  NBig *                            src/nbig.jl:124-140

Limb buffers are numpy uint64 arrays, offsets 0-based.  There is no CPU
fallback: importing this module without the built library raises, and every
call goes to the GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("NBGPU_LIB") or os.path.join(os.path.dirname(_HERE), "lib", "libnbgpu.so")

NBG_OK, NBG_EINVAL, NBG_ERANGE, NBG_ENOMEM, NBG_ECUDA, NBG_ETIMEOUT, NBG_EBUSY, NBG_ENODEV = range(8)

# dispatch thresholds of the reference (src/mul.jl:12-26)
MUL_FPNTT_MIN = 64
MUL_FPNTT_THRESHOLD = 152
SQR_FPNTT_THRESHOLD = 160

EXPORTS = [
    "nbg_mul", "nbg_sqr", "nbg_mul_dev", "nbg_sqr_dev", "nbg_mul_batch", "nbg_mul_batch_dev",
    "nbg_batch_create", "nbg_batch_run", "nbg_batch_launches", "nbg_batch_destroy", "nbg_batch_stats",
    "nbg_batch_profile",
    "nbg_ntt_params", "nbg_ntt_len", "nbg_magnitude_bits", "nbg_pack_dev", "nbg_ntt_fwd_dev",
    "nbg_ntt_rev_dev", "nbg_pointwise_dev", "nbg_unpack_dev", "nbg_plan_info", "nbg_plan_layout", "nbg_set_tuning",
    "nbg_get_tuning", "nbg_init", "nbg_last_error", "nbg_default_stream", "nbg_launch_count",
    "nbg_mul_dev_noalloc", "nbg_load_tuning", "nbg_version", "nbg_trim_plans",
    "nbg_server_create", "nbg_submit", "nbg_submit_dev", "nbg_poll", "nbg_wait", "nbg_release",
    "nbg_server_stats", "nbg_server_destroy",
    "nbg_powermod_batch", "nbg_powermod_batch_dev", "nbg_barrett_mu", "nbg_powmod_schedule",
    "nbg_mullo", "nbg_sqrlo", "nbg_matrix22_mul_dev", "nbg_mul2add_dev", "nbg_radix_combine",
    "nbg_kernel_arch", "nbg_radix_powtab", "nbg_device_faults",
]


class NBGError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"nbgpu error {code}: {msg}")
        self.code = code


class LengthError(NBGError, ValueError):
    """Transform length beyond 315*2^34 (the reference's ArgumentError, src/fpntt.jl:948-949)."""


class NbgDesc(ctypes.Structure):
    _fields_ = [("r", ctypes.c_void_p), ("a", ctypes.c_void_p), ("b", ctypes.c_void_p),
                ("m", ctypes.c_int64), ("n", ctypes.c_int64), ("bits_a", ctypes.c_int64),
                ("bits_b", ctypes.c_int64)]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libnbgpu.so not built ({LIB_PATH}); run nativebigint.jl_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        c = ctypes
        vp, i64, i32 = c.c_void_p, c.c_int64, c.c_int32
        sig = {
            "nbg_mul": [vp, vp, i64, vp, i64],
            "nbg_sqr": [vp, vp, i64],
            "nbg_mul_dev": [vp, vp, i64, vp, i64, vp],
            "nbg_sqr_dev": [vp, vp, i64, vp],
            "nbg_mul_dev_noalloc": [vp, vp, i64, vp, i64, vp],
            "nbg_mul_batch": [vp, i64],
            "nbg_mul_batch_dev": [vp, i64, vp],
            "nbg_batch_create": [vp, i64, c.POINTER(vp)],
            "nbg_batch_run": [vp, vp],
            "nbg_batch_launches": [vp],
            "nbg_batch_destroy": [vp],
            "nbg_batch_stats": [vp, c.POINTER(i32), c.POINTER(i64), c.POINTER(c.c_double), c.POINTER(c.c_double), i32],
            "nbg_batch_profile": [vp, vp, c.POINTER(c.c_float), i32],
            "nbg_ntt_params": [i64, i64, c.POINTER(i32), c.POINTER(i64)],
            "nbg_ntt_len": [i64, c.POINTER(i64)],
            "nbg_pack_dev": [vp, i64, vp, i64, i32, i64, vp],
            "nbg_ntt_fwd_dev": [vp, i64, i32, vp],
            "nbg_ntt_rev_dev": [vp, i64, i32, vp],
            "nbg_pointwise_dev": [vp, vp, i64, i32, vp],
            "nbg_unpack_dev": [vp, i64, vp, vp, i64, i64, i32, vp],
            "nbg_plan_info": [i64, c.POINTER(i32), c.POINTER(i32), c.POINTER(i32), c.POINTER(i32), i32],
            "nbg_plan_layout": [i64, i32, c.POINTER(i64), c.POINTER(i32), c.POINTER(i64), c.POINTER(i32),
                                c.POINTER(i32), i32],
            "nbg_set_tuning": [c.c_char_p],
            "nbg_get_tuning": [c.c_char_p, i64],
            "nbg_init": [i32],
            "nbg_server_create": [vp, c.POINTER(vp)],
            "nbg_submit": [vp, vp, c.POINTER(i64)],
            "nbg_submit_dev": [vp, vp, c.POINTER(i64)],
            "nbg_poll": [vp, i64, c.POINTER(i32)],
            "nbg_wait": [vp, i64, i64],
            "nbg_release": [vp, i64],
            "nbg_server_stats": [vp, vp],
            "nbg_server_destroy": [vp],
            "nbg_load_tuning": [c.c_char_p],
            "nbg_powermod_batch": [vp, i64, i64],
            "nbg_mullo": [vp, vp, i64, vp, i64, i64],
            "nbg_matrix22_mul_dev": [vp, i64, vp, i64, vp],
            "nbg_radix_combine": [vp, i64, vp, i64, c.c_uint64, c.POINTER(i64)],
            "nbg_mul2add_dev": [vp, i64, vp, i64, vp, i64, vp, i64, vp, i64, vp],
            "nbg_sqrlo": [vp, vp, i64, i64],
            "nbg_powermod_batch_dev": [vp, i64, i64, vp],
            "nbg_kernel_arch": [c.POINTER(i32)],
            "nbg_device_faults": [c.POINTER(i64)],
            "nbg_radix_powtab": [vp, i64, c.POINTER(i64), i32, c.c_uint64, vp, i64, c.POINTER(i32)],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = c.c_int
        L.nbg_magnitude_bits.argtypes = [vp, i64]
        L.nbg_magnitude_bits.restype = i64
        L.nbg_last_error.argtypes = []
        L.nbg_last_error.restype = c.c_char_p
        L.nbg_default_stream.argtypes = []
        L.nbg_default_stream.restype = vp
        L.nbg_trim_plans.argtypes = []
        L.nbg_trim_plans.restype = c.c_int
        L.nbg_version.argtypes = []
        L.nbg_version.restype = c.c_char_p
        L.nbg_barrett_mu.argtypes = [vp, i64, vp]
        L.nbg_barrett_mu.restype = i64
        L.nbg_powmod_schedule.argtypes = [vp, i64, vp, i64, c.POINTER(i32)]
        L.nbg_powmod_schedule.restype = i64
        L.nbg_launch_count.argtypes = []
        L.nbg_launch_count.restype = i64
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != NBG_OK:
        msg = lib().nbg_last_error().decode(errors="replace")
        if rc == NBG_ERANGE:
            raise LengthError(rc, msg)
        raise NBGError(rc, msg)


def _u64(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a


def _ptr(a: np.ndarray, off: int = 0) -> int:
    return a.ctypes.data + 8 * off


def _dptr(x) -> int:
    """Device pointer of a torch tensor or a raw integer address."""
    if isinstance(x, int):
        return x
    return x.data_ptr()


def _stream(s) -> int | None:
    if s is None:
        return None
    if isinstance(s, int):
        return s
    return getattr(s, "cuda_stream", None) or int(s)


# ---------------------------------------------------------------------------
# mpn-level drop-ins (host buffers)

def mul_(r: np.ndarray, ro: int, a: np.ndarray, ao: int, m: int, b: np.ndarray, bo: int, n: int) -> None:
    """r[ro:ro+m+n] = a[ao:ao+m] * b[bo:bo+n] — the NTT branch of mul!
    (src/mul.jl:383-390) / mul_fpntt2! (src/fpntt.jl:982)."""
    for arr, off, ln in ((r, ro, m + n), (a, ao, m), (b, bo, n)):
        if arr.dtype != np.uint64 or not arr.flags.c_contiguous or off < 0 or off + ln > arr.size:
            raise ValueError("limb buffers must be contiguous uint64 with room for the operands")
    _check(lib().nbg_mul(_ptr(r, ro), _ptr(a, ao), m, _ptr(b, bo), n))


def sqr_(r: np.ndarray, ro: int, a: np.ndarray, ao: int, n: int) -> None:
    """r[ro:ro+2n] = a[ao:ao+n]^2 — sqr! NTT branch (src/mul.jl:141-147) / sqr_fpntt2!."""
    for arr, off, ln in ((r, ro, 2 * n), (a, ao, n)):
        if arr.dtype != np.uint64 or not arr.flags.c_contiguous or off < 0 or off + ln > arr.size:
            raise ValueError("limb buffers must be contiguous uint64 with room for the operands")
    _check(lib().nbg_sqr(_ptr(r, ro), _ptr(a, ao), n))


def mul(a, b) -> np.ndarray:
    a, b = _u64(a), _u64(b)
    r = np.empty(a.size + b.size, dtype=np.uint64)
    mul_(r, 0, a, 0, a.size, b, 0, b.size)
    return r


def sqr(a) -> np.ndarray:
    a = _u64(a)
    r = np.empty(2 * a.size, dtype=np.uint64)
    sqr_(r, 0, a, 0, a.size)
    return r


def mullo(a, b, k: int) -> np.ndarray:
    """Low k limbs of a*b (mullo!'s full-product branch, src/mul.jl:316-319)."""
    a, b = _u64(a), _u64(b)
    r = np.empty(k, dtype=np.uint64)
    _check(lib().nbg_mullo(_ptr(r), _ptr(a), a.size, _ptr(b), b.size, k))
    return r


def sqrlo(a, k: int) -> np.ndarray:
    """Low k limbs of a^2 (sqrlo!'s full-product branch, src/mul.jl:361-364)."""
    a = _u64(a)
    r = np.empty(k, dtype=np.uint64)
    _check(lib().nbg_sqrlo(_ptr(r), _ptr(a), a.size, k))
    return r


def matrix22_mul_dev(m, n: int, m1, n1: int, stream=None) -> None:
    """M <- M*M1 in place (hgcd_matrix_mul!): m, m1 are 4 device buffers each
    (m00, m01, m10, m11); m's entries need n + n1 + 1 limbs of room."""
    pm = (ctypes.c_void_p * 4)(*[_dptr(x) for x in m])
    pm1 = (ctypes.c_void_p * 4)(*[_dptr(x) for x in m1])
    _check(lib().nbg_matrix22_mul_dev(pm, n, pm1, n1, _stream(stream)))


def mul2add_dev(r, rn: int, a, la: int, x, lx: int, b, lb: int, y, ly: int, stream=None) -> None:
    """r = a*x + b*y on device buffers (cof_mul2!)."""
    _check(lib().nbg_mul2add_dev(_dptr(r), rn, _dptr(a), la, _dptr(x), lx, _dptr(b), lb, _dptr(y), ly,
                                 _stream(stream)))


def radix_combine(chunks, bb: int) -> np.ndarray:
    """Binary limbs of sum(chunks[i] * bb**i) (little-endian chunks < bb), e.g.
    bb = 10**19 for 19 decimal digits per chunk (radix_combine)."""
    c = _u64(chunks)
    out = np.zeros(max(1, c.size), dtype=np.uint64)
    n = ctypes.c_int64()
    _check(lib().nbg_radix_combine(_ptr(out), out.size, _ptr(c), c.size, bb, ctypes.byref(n)))
    return out[: n.value]


def radix_powtab(bb: int, x) -> list[np.ndarray]:
    """radix_chunks_dc's power table for x: [bb, bb^2, bb^4, ...] while the
    last entry is <= x (normalized limb arrays; squares on the GPU)."""
    x = _u64(x)
    cap = 4 * x.size + 64
    out = np.zeros(cap, dtype=np.uint64)
    maxe = 70
    offs = (ctypes.c_int64 * (maxe + 1))()
    ne = ctypes.c_int32()
    _check(lib().nbg_radix_powtab(_ptr(out), cap, offs, maxe, int(bb), _ptr(x), x.size, ctypes.byref(ne)))
    return [out[offs[i]: offs[i + 1]].copy() for i in range(ne.value)]


def mul_batch(pairs) -> list[np.ndarray]:
    """Products of a list of (a, b) pairs (b None for a square), one batched
    call; returns the m+n-limb results."""
    ops = []
    descs = (NbgDesc * len(pairs))()
    for k, (a, b) in enumerate(pairs):
        a = _u64(a)
        b = None if b is None else _u64(b)
        r = np.empty(a.size + (a.size if b is None else b.size), dtype=np.uint64)
        ops.append((a, b, r))
        descs[k] = NbgDesc(_ptr(r), _ptr(a), None if b is None else _ptr(b), a.size,
                           a.size if b is None else b.size, 0, 0)
    _check(lib().nbg_mul_batch(ctypes.cast(descs, ctypes.c_void_p), len(pairs)))
    return [r for (_, _, r) in ops]


def uses_fpntt_mul(m: int, n: int) -> bool:
    """mul! sends m x n (m >= n) to the NTT when n >= 64 and m + n >= 304 (src/mul.jl:388)."""
    if m < n:
        m, n = n, m
    return n >= MUL_FPNTT_MIN and m + n >= 2 * MUL_FPNTT_THRESHOLD


def uses_fpntt_sqr(n: int) -> bool:
    """sqr! sends n >= 160 limbs to the NTT (src/mul.jl:146)."""
    return n >= SQR_FPNTT_THRESHOLD


# ---------------------------------------------------------------------------
# device-buffer calls (torch tensors or raw device addresses)

def mul_dev(r, a, m: int, b, n: int, stream=None) -> None:
    _check(lib().nbg_mul_dev(_dptr(r), _dptr(a), m, _dptr(b), n, _stream(stream)))


def sqr_dev(r, a, n: int, stream=None) -> None:
    _check(lib().nbg_sqr_dev(_dptr(r), _dptr(a), n, _stream(stream)))


def mul_dev_noalloc(r, a, m: int, b, n: int, stream=None) -> None:
    """The product of nbg_mul_dev with no device allocation: the workspace is the
    library's fixed 16 MiB device array (b None for a square)."""
    _check(lib().nbg_mul_dev_noalloc(_dptr(r), _dptr(a), m, None if b is None else _dptr(b), n, _stream(stream)))


def make_descs(items) -> ctypes.Array:
    """items: (r, a, b_or_None, m, n, bits_a, bits_b) with device tensors or addresses."""
    descs = (NbgDesc * len(items))()
    for k, (r, a, b, m, n, ba, bb) in enumerate(items):
        descs[k] = NbgDesc(_dptr(r), _dptr(a), None if b is None else _dptr(b), m, n, ba, bb)
    return descs


def mul_batch_dev(descs: ctypes.Array, stream=None) -> None:
    _check(lib().nbg_mul_batch_dev(ctypes.cast(descs, ctypes.c_void_p), len(descs), _stream(stream)))


class Batch:
    """A reusable device batch replayed as one CUDA graph (nbg_batch_*)."""

    def __init__(self, descs: ctypes.Array):
        self._h = ctypes.c_void_p()
        _check(lib().nbg_batch_create(ctypes.cast(descs, ctypes.c_void_p), len(descs), ctypes.byref(self._h)))
        self.launches = lib().nbg_batch_launches(self._h)

    def run(self, stream=None) -> None:
        _check(lib().nbg_batch_run(self._h, _stream(stream)))

    def stats(self) -> list[dict]:
        n = self.launches
        kinds = (ctypes.c_int32 * n)()
        njobs = (ctypes.c_int64 * n)()
        ops = (ctypes.c_double * n)()
        byt = (ctypes.c_double * n)()
        _check(lib().nbg_batch_stats(self._h, kinds, njobs, ops, byt, n))
        names = {0: "k_fwd", 1: "k_pwr", 2: "k_rev", 3: "k_unpack", 4: "k_carry", 5: "k_carry_fix", 6: "k_pwr",
                 7: "k_pwr", 8: "k_col_tma_fwd", 9: "k_col_tma_rev"}
        return [dict(kind=names[kinds[i]], code=kinds[i], jobs=njobs[i], alg_ops=ops[i], alg_bytes=byt[i])
                for i in range(n)]

    def profile(self, stream=None) -> list[float]:
        n = self.launches
        ms = (ctypes.c_float * n)()
        _check(lib().nbg_batch_profile(self._h, _stream(stream), ms, n))
        return list(ms)

    def close(self) -> None:
        if self._h:
            lib().nbg_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# serving (continuous batching)

class ServerOpts(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_int64), ("max_batch", ctypes.c_int64), ("max_queue", ctypes.c_int64),
                ("batch_points", ctypes.c_int64), ("max_hold_us", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("failed", ctypes.c_int64), ("pending", ctypes.c_int64),
                ("in_flight_batches", ctypes.c_int32), ("reserved", ctypes.c_int32), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("output_limbs_per_s", ctypes.c_double), ("batches", ctypes.c_int64),
                ("mean_batch_requests", ctypes.c_double)]


class Server:
    """Continuous-batching product server (nbg_server_*)."""

    def __init__(self, hbm_budget_bytes: int = 1 << 30, max_batch: int = 0, max_queue: int = 0,
                 batch_points: int = 0, max_hold_us: int = 0):
        self._h = ctypes.c_void_p()
        opts = ServerOpts(hbm_budget_bytes, max_batch, max_queue, batch_points, max_hold_us)
        _check(lib().nbg_server_create(ctypes.byref(opts), ctypes.byref(self._h)))
        self._keep: dict = {}

    def submit(self, a: np.ndarray, b, r: np.ndarray) -> int:
        """Host request: r (len(a)+len(b) limbs) receives a*b (b None: a^2)."""
        a = _u64(a)
        d = NbgDesc(_ptr(r), _ptr(a), None if b is None else _ptr(b), a.size, a.size if b is None else b.size, 0, 0)
        t = ctypes.c_int64()
        _check(lib().nbg_submit(self._h, ctypes.byref(d), ctypes.byref(t)))
        self._keep[t.value] = (a, b, r)
        return t.value

    def submit_dev(self, r, a, m: int, b, n: int, bits_a: int, bits_b: int) -> int:
        d = NbgDesc(_dptr(r), _dptr(a), None if b is None else _dptr(b), m, n, bits_a, bits_b)
        t = ctypes.c_int64()
        _check(lib().nbg_submit_dev(self._h, ctypes.byref(d), ctypes.byref(t)))
        return t.value

    def poll(self, ticket: int) -> bool:
        done = ctypes.c_int32()
        _check(lib().nbg_poll(self._h, ticket, ctypes.byref(done)))
        return bool(done.value)

    def wait(self, ticket: int, timeout_s: float = 60.0) -> None:
        _check(lib().nbg_wait(self._h, ticket, int(timeout_s * 1e6)))
        self._keep.pop(ticket, None)

    def release(self, ticket: int) -> None:
        _check(lib().nbg_release(self._h, ticket))

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().nbg_server_stats(self._h, ctypes.byref(st)))
        return {k: getattr(st, k) for k, _ in ServerStats._fields_ if k != "reserved"}

    def close(self) -> None:
        if self._h:
            lib().nbg_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Barrett powermod chains

class PowmodDesc(ctypes.Structure):
    _fields_ = [("r", ctypes.c_void_p), ("b", ctypes.c_void_p), ("e", ctypes.c_void_p), ("m", ctypes.c_void_p),
                ("lb", ctypes.c_int64), ("le", ctypes.c_int64)]


def powermod_batch(bases, exps, mods) -> list[np.ndarray]:
    """r_c = b_c^e_c mod m_c for chains of one modulus size k (limb arrays,
    host memory); every chain's square/multiply and both Barrett products run
    as batched GPU products (nbg_powermod_batch)."""
    mods = [_u64(m) for m in mods]
    bases = [_u64(b) for b in bases]
    exps = [_u64(e) for e in exps]
    k = mods[0].size
    if any(m.size != k for m in mods):
        raise ValueError("all moduli need the same limb count")
    outs = [np.zeros(k, dtype=np.uint64) for _ in mods]
    d = (PowmodDesc * len(mods))()
    for i, (r, b, e, m) in enumerate(zip(outs, bases, exps, mods)):
        d[i] = PowmodDesc(_ptr(r), _ptr(b), _ptr(e), _ptr(m), b.size, e.size)
    _check(lib().nbg_powermod_batch(ctypes.cast(d, ctypes.c_void_p), len(mods), k))
    return outs


def powermod_batch_dev(descs, k: int, stream=None) -> None:
    """Device-buffer form: descs is a PowmodDesc array of device pointers."""
    _check(lib().nbg_powermod_batch_dev(ctypes.cast(descs, ctypes.c_void_p), len(descs), k, _stream(stream)))


def barrett_mu(m) -> np.ndarray:
    """mu = floor(2^(128k) / m) (k + 2 limbs, host computation)."""
    m = _u64(m)
    mu = np.zeros(m.size + 2, dtype=np.uint64)
    n = lib().nbg_barrett_mu(_ptr(m), m.size, _ptr(mu))
    if n < 0:
        _check(int(-n))
    return mu


def powmod_schedule(e) -> tuple[np.ndarray, int]:
    """The chain's step list as an (S, 3) uint8 array (dst, src1, src2) and
    the odd-power table size."""
    e = _u64(e)
    T = ctypes.c_int32()
    n = lib().nbg_powmod_schedule(_ptr(e), e.size, None, 0, ctypes.byref(T))
    if n < 0:
        _check(int(-n))
    ops = np.zeros((n, 3), dtype=np.uint8)
    lib().nbg_powmod_schedule(_ptr(e), e.size, ops.ctypes.data, n, ctypes.byref(T))
    return ops, T.value


# ---------------------------------------------------------------------------
# admission

def ntt_params(bits_a: int, bits_b: int) -> tuple[int, int]:
    b = ctypes.c_int32()
    N = ctypes.c_int64()
    _check(lib().nbg_ntt_params(bits_a, bits_b, ctypes.byref(b), ctypes.byref(N)))
    return b.value, N.value


def ntt_len(T: int) -> int:
    N = ctypes.c_int64()
    _check(lib().nbg_ntt_len(T, ctypes.byref(N)))
    return N.value


def magnitude_bits(a) -> int:
    a = _u64(a)
    return lib().nbg_magnitude_bits(_ptr(a), a.size)


# ---------------------------------------------------------------------------
# transform level (device buffers)

def pack_dev(x, N: int, limbs, n: int, b: int, nch: int, stream=None) -> None:
    _check(lib().nbg_pack_dev(_dptr(x), N, _dptr(limbs), n, b, nch, _stream(stream)))


def ntt_fwd_dev(x, N: int, prime: int, stream=None) -> None:
    _check(lib().nbg_ntt_fwd_dev(_dptr(x), N, prime, _stream(stream)))


def ntt_rev_dev(x, N: int, prime: int, stream=None) -> None:
    _check(lib().nbg_ntt_rev_dev(_dptr(x), N, prime, _stream(stream)))


def pointwise_dev(xa, xb, N: int, prime: int, stream=None) -> None:
    _check(lib().nbg_pointwise_dev(_dptr(xa), _dptr(xb), N, prime, _stream(stream)))


def unpack_dev(r, rn: int, x1, x2, N: int, nconv: int, b: int, stream=None) -> None:
    _check(lib().nbg_unpack_dev(_dptr(r), rn, _dptr(x1), _dptr(x2), N, nconv, b, _stream(stream)))


def plan_info(N: int) -> dict:
    cap = 32
    nst, npass = ctypes.c_int32(), ctypes.c_int32()
    sm = (ctypes.c_int32 * cap)()
    pe = (ctypes.c_int32 * cap)()
    _check(lib().nbg_plan_info(N, ctypes.byref(nst), ctypes.byref(npass), sm, pe, cap))
    return {"stages": list(sm[: nst.value]), "pass_end": list(pe[: npass.value])}


ROUND_KINDS = {0: "odd", 1: "r4", 2: "r16", 3: "r8", 4: "r2"}


def plan_layout(N: int, sqr: bool = False) -> dict:
    """Stages (m, L, Q), passes (sa, sb, G, C, Qb, ntiles) and each pass's
    rounds [(kind, first stage)] for length N; host only."""
    cap = 32
    st = (ctypes.c_int64 * (3 * cap))()
    ps = (ctypes.c_int64 * (7 * cap))()
    rd = (ctypes.c_int32 * (cap * cap))()
    nst, npass = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().nbg_plan_layout(N, 1 if sqr else 0, st, ctypes.byref(nst), ps, ctypes.byref(npass), rd, cap))
    stages = [tuple(st[3 * i: 3 * i + 3]) for i in range(nst.value)]
    passes = [tuple(ps[7 * j: 7 * j + 6]) for j in range(npass.value)]
    rounds = [[(ROUND_KINDS[rd[j * cap + r] >> 8], rd[j * cap + r] & 0xff) for r in range(ps[7 * j + 6])]
              for j in range(npass.value)]
    return {"stages": stages, "passes": passes, "rounds": rounds}


def set_tuning(js: str) -> None:
    _check(lib().nbg_set_tuning(js.encode()))


def get_tuning() -> str:
    buf = ctypes.create_string_buffer(1 << 16)
    _check(lib().nbg_get_tuning(buf, 1 << 16))
    return buf.value.decode()


def load_tuning(path: str) -> None:
    _check(lib().nbg_load_tuning(path.encode()))


def trim_plans() -> None:
    """Frees cached plans' device tables (no Batch may be alive)."""
    _check(lib().nbg_trim_plans())


def device_faults() -> int:
    """Bounded kernel waits that gave up since the last call (0 when healthy); clears the count."""
    n = ctypes.c_int64()
    _check(lib().nbg_device_faults(ctypes.byref(n)))
    return n.value


def version() -> str:
    return lib().nbg_version().decode()


def launch_count() -> int:
    return lib().nbg_launch_count()


def default_stream() -> int:
    return lib().nbg_default_stream()


# ---------------------------------------------------------------------------
# NBig-style value wrapper (src/nbig.jl:124-140): the `*` dispatch of the
# reference, with products on the GPU engine.

def _limbs_of(v: int) -> np.ndarray:
    n = max(1, (v.bit_length() + 63) // 64)
    return np.frombuffer(v.to_bytes(8 * n, "little"), dtype="<u8").astype(np.uint64)


def _int_of(limbs: np.ndarray) -> int:
    return int.from_bytes(np.ascontiguousarray(limbs, dtype="<u8").tobytes(), "little")


class NBig:
    """Sign-magnitude integer whose `*` runs on the GPU engine.

    Like the reference, a product of a value with itself (same limb buffer)
    is a square; otherwise operands are swapped so la >= lb."""

    __slots__ = ("sign", "limbs")

    def __init__(self, v: int = 0):
        self.sign = (v > 0) - (v < 0)
        self.limbs = _limbs_of(abs(v)) if v else np.zeros(0, dtype=np.uint64)

    def __int__(self) -> int:
        return self.sign * _int_of(self.limbs) if self.sign else 0

    def __neg__(self) -> "NBig":
        out = NBig.__new__(NBig)
        out.sign, out.limbs = -self.sign, self.limbs
        return out

    def __mul__(self, other: "NBig") -> "NBig":
        out = NBig.__new__(NBig)
        if self.sign == 0 or other.sign == 0:
            out.sign, out.limbs = 0, np.zeros(0, dtype=np.uint64)
            return out
        if self.limbs is other.limbs:
            r = sqr(self.limbs)
        else:
            a, b = (self.limbs, other.limbs) if self.limbs.size >= other.limbs.size else (other.limbs, self.limbs)
            r = mul(a, b)
        n = r.size
        while n > 0 and r[n - 1] == 0:
            n -= 1
        out.sign, out.limbs = self.sign * other.sign, r[:n].copy()
        return out
