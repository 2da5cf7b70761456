"""ctypes view of the CPU oracle (``oracle/lzx_oracle.c``).

TEST INFRASTRUCTURE ONLY: the correctness oracle for the CUDA path and the
timed CPU baseline.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
legs of ``bench.py`` import this module; the product package ``lzx_b200``
never does.  Every wrapped C function restates a function of the reference
(idrees2516/lzx, Rust) and cites its file:line in ``lzx_oracle.c``.

Parity pin: the Goldilocks and Keccak restatements are checked against the
reference's own known-answer tests (``tests/golden/reference_kats.json``); the
NTT and commitment restatements are checked against the reference's identity
tests and against direct evaluation at psi^(2j+1).  No reference-produced
NTT/commit digests exist to compare with (the reference's KAT manifest is
generated at run time and not committed).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_lock = threading.Lock()
_lib = None
_native = None

GL_P = 0xFFFFFFFF00000001

# CRT set: the four largest 30-bit primes q == 1 (mod 512), with the smallest
# generator of each multiplicative group and the 2-adicity of q - 1.
CRT_PRIMES = (
    (1073738753, 10, 3),
    (1073732609, 10, 3),
    (1073731073, 9, 3),
    (1073726977, 9, 5),
)
# Modulus32 constants of the reference, lattice-ring/src/modulus.rs:46-55
Q_32 = (3221225473, 30, 5)
Q_12289 = (12289, 12, 11)
Q_2013265921 = (2013265921, 27, 31)


class Mod32(C.Structure):
    _fields_ = [("q", C.c_uint32), ("two_adicity", C.c_uint32), ("generator", C.c_uint32),
                ("barrett_recip", C.c_uint64)]


class Ntt32(C.Structure):
    _fields_ = [("modulus", Mod32), ("log_n", C.c_uint32), ("n_inv", C.c_uint32),
                ("pow_psi", C.c_void_p), ("pow_psi_inv", C.c_void_p), ("pow_omega", C.c_void_p),
                ("pow_omega_inv", C.c_void_p), ("level_tw", C.c_void_p),
                ("level_tw_inv", C.c_void_p)]


class Mod50(C.Structure):
    _fields_ = [("q", C.c_uint64), ("recip", C.c_uint64), ("two_adicity", C.c_uint32),
                ("generator", C.c_uint64)]


class Quad50(C.Structure):
    _fields_ = [("modulus", Mod50), ("log_n", C.c_uint32), ("zeta", C.c_uint64), ("level_tw", C.c_void_p),
                ("level_tw_inv", C.c_void_p), ("leaf_gamma", C.c_void_p)]


class NttGl(C.Structure):
    _fields_ = [("log_n", C.c_uint32), ("n_inv", C.c_uint64), ("pow_psi", C.c_void_p),
                ("pow_psi_inv", C.c_void_p), ("level_tw", C.c_void_p), ("level_tw_inv", C.c_void_p)]


def _build(target: str) -> None:
    subprocess.run(["make", "-s", "-C", _HERE, target], check=True)


def _declare(lib):
    P = C.c_void_p
    sz, u32, u64, i32 = C.c_size_t, C.c_uint32, C.c_uint64, C.c_int
    sig = {
        "orc_mod32_new": (Mod32, [u32, u32, u32]),
        "orc_mod32_reduce_u64": (u32, [P, u64]),
        "orc_mod32_reduce_i64": (u32, [P, C.c_int64]),
        "orc_mod32_mul": (u32, [P, u32, u32]),
        "orc_mod32_add": (u32, [P, u32, u32]),
        "orc_mod32_sub": (u32, [P, u32, u32]),
        "orc_mod32_neg": (u32, [P, u32]),
        "orc_mod32_pow": (u32, [P, u32, u64]),
        "orc_mod32_inv": (u32, [P, u32]),
        "orc_mod32_root_of_unity": (u32, [P, u32]),
        "orc_gl_from_u64": (u64, [u64]),
        "orc_gl_from_u128": (u64, [u64, u64]),
        "orc_gl_add": (u64, [u64, u64]),
        "orc_gl_sub": (u64, [u64, u64]),
        "orc_gl_neg": (u64, [u64]),
        "orc_gl_mul": (u64, [u64, u64]),
        "orc_gl_pow": (u64, [u64, u64]),
        "orc_gl_inv": (u64, [u64]),
        "orc_ntt32_new": (i32, [Mod32, u32, P]),
        "orc_ntt32_free": (None, [P]),
        "orc_ntt32_forward": (i32, [P, P, sz]),
        "orc_ntt32_forward_fast": (i32, [P, P, sz]),
        "orc_ntt32_inverse": (i32, [P, P, sz]),
        "orc_ntt32_inverse_fast": (i32, [P, P, sz]),
        "orc_ntt32_forward_partial": (i32, [P, P, sz, u32]),
        "orc_ntt32_complete_partial": (i32, [P, P, sz, u32]),
        "orc_ntt32_forward_batch": (i32, [P, P, sz, i32]),
        "orc_ntt32_inverse_batch": (i32, [P, P, sz, i32]),
        "orc_nttgl_new": (i32, [u32, P]),
        "orc_nttgl_free": (None, [P]),
        "orc_nttgl_forward_fast": (i32, [P, P, sz]),
        "orc_nttgl_inverse_fast": (i32, [P, P, sz]),
        "orc_nttgl_forward_batch": (i32, [P, P, sz, i32]),
        "orc_nttgl_inverse_batch": (i32, [P, P, sz, i32]),
        "orc_ajtai32_commit": (i32, [P, P, sz, sz, P, P]),
        "orc_ajtai32_commit_naive": (i32, [P, P, sz, sz, P, P]),
        "orc_ring32_mul": (i32, [P, P, P, P]),
        "orc_ajtaigl_commit_batch": (i32, [P, P, sz, sz, P, sz, P, i32, i32]),
        "orc_ajtaigl_commit_batch_i8": (i32, [P, P, sz, sz, P, sz, P, i32, i32]),
        "orc_avx512_available": (i32, []),
        "orc_neo_mul": (None, [sz, P, P, P]),
        "orc_neo_commit_naive": (i32, [sz, sz, sz, P, P, sz, P]),
        "orc_neo_commit_pay_per_bit": (i32, [sz, sz, sz, P, P, sz, P, P]),
        "orc_decomp_b": (None, [P, sz, u32, P]),
        "orc_pack_field_elements": (sz, [u32, u32, P, sz, P]),
        "orc_gadget_decompose": (i32, [u64, sz, u64, P]),
        "orc_mod50_new": (Mod50, [u64, u32, u64]),
        "orc_mod50_reduce_u128": (u64, [P, u64, u64]),
        "orc_mod50_mul": (u64, [P, u64, u64]),
        "orc_mod50_add": (u64, [P, u64, u64]),
        "orc_mod50_sub": (u64, [P, u64, u64]),
        "orc_mod50_pow": (u64, [P, u64, u64]),
        "orc_quad50_new": (i32, [Mod50, u32, P]),
        "orc_quad50_free": (None, [P]),
        "orc_quad50_forward": (i32, [P, P, sz]),
        "orc_quad50_inverse": (i32, [P, P, sz]),
        "orc_quad50_slotwise_mul": (i32, [P, P, P, P, sz]),
        "orc_quad50_mul": (i32, [P, P, P, P, sz]),
        "orc_quad50_mul_batch": (i32, [P, P, P, P, sz, i32]),
        "orc_lb_quadratic": (i32, [u32]),
        "orc_lb_psi": (u32, [u32]),
        "orc_lb_tables": (None, [P, P, P, P, P]),
        "orc_lb_ntt": (None, [u32, P, P]),
        "orc_lb_eval_at": (u32, [u32, P, u32]),
        "orc_lb_eval_quad_at": (None, [u32, P, u32, P]),
        "orc_lb_mul_mod_phi": (None, [u32, P, P, P]),
        "orc_lb_mul_quad_slots": (None, [u32, P, P, P]),
        "orc_lb_components": (None, [u32, P, P]),
        "orc_lb_r162_from_coeffs": (None, [u32, P, P]),
        "orc_lb_random_elems": (None, [sz, u64, P]),
        "orc_lb_lift": (None, [P, sz, P]),
        "orc_lb_key_random": (None, [sz, u64, P, sz, P]),
        "orc_lb_commit": (i32, [P, P, sz, sz, P, sz, P, P, P, i32]),
        "orc_keccak_f1600": (None, [P]),
        "orc_sha3_256": (None, [P, sz, P]),
        "orc_shake256": (None, [P, sz, P, sz]),
        "orc_xof": (None, [P, sz, P, sz, P, sz]),
        "orc_hash_domain": (None, [P, sz, P, sz, P]),
        "orc_uniform_from_seed": (None, [P, u32, P, sz, P, sz, u64, P]),
        "orc_ring_random": (None, [P, u32, P, sz, P]),
        "orc_ajtai32_from_seed": (i32, [P, sz, sz, P, P, P]),
        "orc_sample_small_secret": (None, [P, u32, sz, u32, P, sz, P]),
        "orc_synth_u64": (u64, [u64, u64, u64]),
        "orc_synth_mod32": (None, [u64, u64, u32, P, sz, sz]),
        "orc_synth_gl": (None, [u64, u64, P, sz, sz]),
        "orc_synth_i8": (None, [u64, u64, P, sz, sz]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


_prefer_native = False


def prefer_native(flag: bool = True) -> None:
    """Route every oracle call through a copy built with -march=native (for timing)."""
    global _prefer_native
    if flag:
        lib(native=True)
    _prefer_native = flag


def lib(native: bool = False):
    """The oracle shared library (built on first use)."""
    global _lib, _native
    native = native or _prefer_native
    with _lock:
        if native:
            if _native is None:
                path = os.path.join(_BUILD, "liblzx_oracle_native.so")
                if not os.path.exists(path):
                    _build("native")
                _native = _declare(C.CDLL(path))
            return _native
        if _lib is None:
            path = os.path.join(_BUILD, "liblzx_oracle.so")
            if not os.path.exists(path):
                _build("all")
            _lib = _declare(C.CDLL(path))
        return _lib


def ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.c_void_p)


def _bytes_ptr(b: bytes):
    buf = C.create_string_buffer(b, len(b) or 1)
    return buf


# ----------------------------------------------------------------- Modulus32

class Modulus32:
    """Modulus32 (lattice-ring/src/modulus.rs:22-161) over the C restatement."""

    def __init__(self, q: int, two_adicity: int, generator: int):
        self._m = lib().orc_mod32_new(q, two_adicity, generator)
        self.q, self.two_adicity, self.generator = q, two_adicity, generator

    @property
    def barrett_recip(self) -> int:
        return self._m.barrett_recip

    def _p(self):
        return C.byref(self._m)

    def reduce_u64(self, x: int) -> int:
        return lib().orc_mod32_reduce_u64(self._p(), x)

    def reduce_i64(self, x: int) -> int:
        return lib().orc_mod32_reduce_i64(self._p(), x)

    def mul(self, a, b):
        return lib().orc_mod32_mul(self._p(), a, b)

    def add(self, a, b):
        return lib().orc_mod32_add(self._p(), a, b)

    def sub(self, a, b):
        return lib().orc_mod32_sub(self._p(), a, b)

    def neg(self, a):
        return lib().orc_mod32_neg(self._p(), a)

    def pow(self, a, e):
        return lib().orc_mod32_pow(self._p(), a, e)

    def inv(self, a):
        return None if a == 0 else lib().orc_mod32_inv(self._p(), a)

    def root_of_unity(self, k):
        return None if k > self.two_adicity else lib().orc_mod32_root_of_unity(self._p(), k)


# ----------------------------------------------------------------- NTT tables

class NttError(Exception):
    def __init__(self, code):
        super().__init__({1: "LengthMismatch", 2: "AdicityTooSmall"}.get(code, str(code)))
        self.code = code


def _check(rc):
    if rc != 0:
        raise NttError(rc)


class NttTables32:
    """NttTables (lattice-ring/src/ntt.rs:16-317) over a u32 modulus."""

    def __init__(self, modulus: Modulus32, log_n: int):
        self._t = Ntt32()
        _check(lib().orc_ntt32_new(modulus._m, log_n, C.byref(self._t)))
        self.modulus, self.log_n, self.n = modulus, log_n, 1 << log_n

    def __del__(self):
        if getattr(self, "_t", None) is not None and _lib is not None:
            _lib.orc_ntt32_free(C.byref(self._t))
            self._t = None

    def _run(self, fn, a: np.ndarray, *extra):
        a = np.ascontiguousarray(a, dtype=np.uint32).copy()
        _check(getattr(lib(), fn)(C.byref(self._t), ptr(a), a.size, *extra))
        return a

    def forward(self, a):
        return self._run("orc_ntt32_forward", a)

    def forward_fast(self, a):
        return self._run("orc_ntt32_forward_fast", a)

    def inverse(self, a):
        return self._run("orc_ntt32_inverse", a)

    def inverse_fast(self, a):
        return self._run("orc_ntt32_inverse_fast", a)

    def forward_partial(self, a, levels):
        return self._run("orc_ntt32_forward_partial", a, levels)

    def complete_partial(self, a, already):
        return self._run("orc_ntt32_complete_partial", a, already)

    def forward_batch(self, a: np.ndarray, nthreads: int = 0, inplace: bool = False):
        a = a if inplace else np.array(a, dtype=np.uint32, copy=True)
        assert a.dtype == np.uint32 and a.size % self.n == 0
        _check(lib().orc_ntt32_forward_batch(C.byref(self._t), ptr(a), a.size // self.n, nthreads))
        return a

    def inverse_batch(self, a: np.ndarray, nthreads: int = 0, inplace: bool = False):
        a = a if inplace else np.array(a, dtype=np.uint32, copy=True)
        assert a.dtype == np.uint32 and a.size % self.n == 0
        _check(lib().orc_ntt32_inverse_batch(C.byref(self._t), ptr(a), a.size // self.n, nthreads))
        return a

    def ring_mul(self, a, b):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        b = np.ascontiguousarray(b, dtype=np.uint32)
        out = np.empty(self.n, dtype=np.uint32)
        lib().orc_ring32_mul(C.byref(self._t), ptr(a), ptr(b), ptr(out))
        return out


class NttTablesGl:
    """The ntt.rs algorithm instantiated over Goldilocks (field.rs, generator 7)."""

    def __init__(self, log_n: int):
        self._t = NttGl()
        _check(lib().orc_nttgl_new(log_n, C.byref(self._t)))
        self.log_n, self.n = log_n, 1 << log_n

    def __del__(self):
        if getattr(self, "_t", None) is not None and _lib is not None:
            _lib.orc_nttgl_free(C.byref(self._t))
            self._t = None

    def forward_fast(self, a):
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        _check(lib().orc_nttgl_forward_fast(C.byref(self._t), ptr(a), a.size))
        return a

    def inverse_fast(self, a):
        a = np.ascontiguousarray(a, dtype=np.uint64).copy()
        _check(lib().orc_nttgl_inverse_fast(C.byref(self._t), ptr(a), a.size))
        return a

    def forward_batch(self, a, nthreads: int = 0, inplace: bool = False):
        a = a if inplace else np.array(a, dtype=np.uint64, copy=True)
        _check(lib().orc_nttgl_forward_batch(C.byref(self._t), ptr(a), a.size // self.n, nthreads))
        return a

    def inverse_batch(self, a, nthreads: int = 0, inplace: bool = False):
        a = a if inplace else np.array(a, dtype=np.uint64, copy=True)
        _check(lib().orc_nttgl_inverse_batch(C.byref(self._t), ptr(a), a.size // self.n, nthreads))
        return a


# ----------------------------------------------------------------- commits

def ajtai32_commit(tables: NttTables32, matrix_ntt: np.ndarray, k: int, m: int, s: np.ndarray):
    """AjtaiPublicKey::commit (lattice-commitment/src/ajtai.rs:118-153)."""
    matrix_ntt = np.ascontiguousarray(matrix_ntt, dtype=np.uint32)
    s = np.ascontiguousarray(s, dtype=np.uint32)
    out = np.empty(k * tables.n, dtype=np.uint32)
    lib().orc_ajtai32_commit(C.byref(tables._t), ptr(matrix_ntt), k, m, ptr(s), ptr(out))
    return out.reshape(k, tables.n)


def ajtai32_commit_naive(tables: NttTables32, matrix: np.ndarray, k: int, m: int, s: np.ndarray):
    """AjtaiPublicKey::commit_naive_reference (ajtai.rs:158-180)."""
    matrix = np.ascontiguousarray(matrix, dtype=np.uint32)
    s = np.ascontiguousarray(s, dtype=np.uint32)
    out = np.empty(k * tables.n, dtype=np.uint32)
    lib().orc_ajtai32_commit_naive(C.byref(tables._t), ptr(matrix), k, m, ptr(s), ptr(out))
    return out.reshape(k, tables.n)


def ajtaigl_commit_batch(tables: NttTablesGl, matrix_ntt, kappa, m, w, nthreads=0, simd=True,
                         native=False):
    """Cached-NTT commit (ajtai.rs:118-153) over Goldilocks for a batch of witnesses.

    ``w`` is either uint64 residues [B, m, d] or int8 digits [B, m, d]."""
    L = lib(native)
    matrix_ntt = np.ascontiguousarray(matrix_ntt, dtype=np.uint64)
    d = tables.n
    w = np.ascontiguousarray(w)
    batch = w.size // (m * d)
    out = np.empty((batch, kappa, d), dtype=np.uint64)
    fn = L.orc_ajtaigl_commit_batch_i8 if w.dtype == np.int8 else L.orc_ajtaigl_commit_batch
    if w.dtype != np.int8:
        w = w.astype(np.uint64, copy=False)
    fn(C.byref(tables._t), ptr(matrix_ntt), kappa, m, ptr(w), batch, ptr(out), nthreads,
       1 if simd else 0)
    return out


def neo_mul(a, b):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    b = np.ascontiguousarray(b, dtype=np.uint64)
    out = np.empty_like(a)
    lib().orc_neo_mul(a.size, ptr(a), ptr(b), ptr(out))
    return out


def neo_commit_naive(d, kappa, m, matrix, cols):
    matrix = np.ascontiguousarray(matrix, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint64)
    ncols = cols.size // d
    out = np.empty((kappa, d), dtype=np.uint64)
    rc = lib().orc_neo_commit_naive(d, kappa, m, ptr(matrix), ptr(cols), ncols, ptr(out))
    if rc:
        raise ValueError("Shape")
    return out


def neo_commit_pay_per_bit(d, kappa, m, matrix, cols):
    matrix = np.ascontiguousarray(matrix, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint64)
    ncols = cols.size // d
    out = np.empty((kappa, d), dtype=np.uint64)
    adds = C.c_uint64(0)
    rc = lib().orc_neo_commit_pay_per_bit(d, kappa, m, ptr(matrix), ptr(cols), ncols, ptr(out),
                                          C.byref(adds))
    if rc:
        raise ValueError("Shape")
    return out, adds.value


def decomp_b(z, b_bits):
    z = np.ascontiguousarray(z, dtype=np.uint64)
    rows = -(-64 // b_bits)
    out = np.empty((rows, z.size), dtype=np.uint64)
    lib().orc_decomp_b(ptr(z), z.size, b_bits, ptr(out))
    return out


def pack_field_elements(q, log_n, values):
    """pack_field_elements (packing.rs:30-52): [elems][n] residues."""
    values = np.ascontiguousarray(values, dtype=np.uint64)
    n = 1 << log_n
    elems = max(1, -(-3 * values.size // n))
    out = np.empty((elems, n), dtype=np.uint32)
    lib().orc_pack_field_elements(q, log_n, ptr(values), values.size, ptr(out))
    return out


def gadget_decompose(base, num_digits, x):
    out = np.empty(num_digits, dtype=np.int64)
    rc = lib().orc_gadget_decompose(base, num_digits, x, ptr(out))
    if rc:
        raise ValueError("ValueTooLarge")
    return out


# ----------------------------------------------------------------- Modulus50

# Q_50 = 2^50 - 2687, two-adicity 7, generator 3 (lattice-ring/src/modulus50.rs:44-51)
Q_50 = (1125899906839937, 7, 3)


class Modulus50:
    """Modulus50 (modulus50.rs:53-198) through the C restatement."""

    def __init__(self, q: int, two_adicity: int, generator: int):
        self.q, self.two_adicity, self.generator = q, two_adicity, generator
        self.s = lib().orc_mod50_new(q, two_adicity, generator)

    def _p(self):
        return C.byref(self.s)

    def reduce_u128(self, x: int) -> int:
        return lib().orc_mod50_reduce_u128(self._p(), x >> 64, x & (2**64 - 1))

    def mul(self, a, b):
        return lib().orc_mod50_mul(self._p(), a, b)

    def add(self, a, b):
        return lib().orc_mod50_add(self._p(), a, b)

    def sub(self, a, b):
        return lib().orc_mod50_sub(self._p(), a, b)

    def pow(self, a, e):
        return lib().orc_mod50_pow(self._p(), a, e)


class QuadSlotTables50:
    """QuadSlotTables (modulus50.rs:206-411); raises NttError(code) like new()."""

    def __init__(self, modulus: Modulus50, log_n: int):
        self.modulus, self.log_n, self.n = modulus, log_n, 1 << log_n
        self.t = Quad50()
        _check(lib().orc_quad50_new(modulus.s, log_n, C.byref(self.t)))

    def __del__(self):
        if getattr(self, "t", None) is not None and self.t.level_tw and _lib is not None:
            _lib.orc_quad50_free(C.byref(self.t))

    @property
    def zeta(self) -> int:
        return self.t.zeta

    @property
    def leaf_gamma(self) -> np.ndarray:
        return np.ctypeslib.as_array(C.cast(self.t.leaf_gamma, C.POINTER(C.c_uint64)), (self.n // 2,)).copy()

    def _one(self, fn, a):
        a = np.array(a, dtype=np.uint64)
        _check(fn(C.byref(self.t), ptr(a), a.size))
        return a

    def forward(self, a):
        return self._one(lib().orc_quad50_forward, a)

    def inverse(self, a):
        return self._one(lib().orc_quad50_inverse, a)

    def slotwise_mul(self, a, b):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        out = np.empty_like(a)
        _check(lib().orc_quad50_slotwise_mul(C.byref(self.t), ptr(a), ptr(b), ptr(out), a.size))
        return out

    def mul(self, a, b):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        out = np.empty_like(a)
        _check(lib().orc_quad50_mul(C.byref(self.t), ptr(a), ptr(b), ptr(out), a.size))
        return out

    def mul_batch(self, a, b, nthreads: int = 0):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        out = np.empty_like(a)
        lib().orc_quad50_mul_batch(C.byref(self.t), ptr(a), ptr(b), ptr(out), a.size // self.n, nthreads)
        return out


# ----------------------------------------------------------------- labinius (R_648)

LB_PRIMES_SPLIT = (3889, 9721, 17497, 19441)   # lattice-labinius/src/params.rs:27-30
LB_PRIMES_QUAD = (2917, 4861, 12637)           # params.rs:308


class lb:
    """labinius restatement (oracle/labinius.c): transforms, decomposition, key, commit."""

    N, N162 = 648, 162

    @staticmethod
    def quadratic(q):
        return bool(lib().orc_lb_quadratic(q))

    @staticmethod
    def psi(q):
        return lib().orc_lb_psi(q)

    @staticmethod
    def tables():
        se = np.empty(648, np.uint16)
        qse = np.empty(324, np.uint16)
        p3 = np.empty(162, np.uint16)
        s648 = np.empty((4, 162), np.uint16)
        qcs = np.empty((2, 162), np.uint16)
        lib().orc_lb_tables(ptr(se), ptr(qse), ptr(p3), ptr(s648), ptr(qcs))
        return {"slot_exp": se, "quad_slot_exp": qse, "pow3_slot_exp": p3, "slot_648": s648,
                "quad_class_slot": qcs}

    @staticmethod
    def ntt(q, a):
        a = np.ascontiguousarray(a, dtype=np.uint32)
        out = np.empty(648, np.uint32)
        lib().orc_lb_ntt(q, ptr(a), ptr(out))
        return out

    @staticmethod
    def eval_at(q, a, u):
        return lib().orc_lb_eval_at(q, ptr(np.ascontiguousarray(a, dtype=np.uint32)), u)

    @staticmethod
    def eval_quad_at(q, a, u):
        out = np.empty(2, np.uint32)
        lib().orc_lb_eval_quad_at(q, ptr(np.ascontiguousarray(a, dtype=np.uint32)), u, ptr(out))
        return tuple(int(x) for x in out)

    @staticmethod
    def mul_mod_phi(q, a, b):
        out = np.empty(648, np.uint32)
        lib().orc_lb_mul_mod_phi(q, ptr(np.ascontiguousarray(a, dtype=np.uint32)),
                                 ptr(np.ascontiguousarray(b, dtype=np.uint32)), ptr(out))
        return out

    @staticmethod
    def mul_quad_slots(q, a, b):
        out = np.empty(648, np.uint32)
        lib().orc_lb_mul_quad_slots(q, ptr(np.ascontiguousarray(a, dtype=np.uint32)),
                                    ptr(np.ascontiguousarray(b, dtype=np.uint32)), ptr(out))
        return out

    @staticmethod
    def components(q, y):
        out = np.empty((4, 162), np.int16)
        lib().orc_lb_components(q, ptr(np.ascontiguousarray(y, dtype=np.uint32)), ptr(out))
        return out

    @staticmethod
    def r162_from_coeffs(q, c):
        out = np.empty(162, np.int16)
        lib().orc_lb_r162_from_coeffs(q, ptr(np.ascontiguousarray(c, dtype=np.int64)), ptr(out))
        return out

    @staticmethod
    def random_elems(n, seed):
        out = np.empty((n, 3), np.uint64)
        lib().orc_lb_random_elems(n, seed, ptr(out))
        return out

    @staticmethod
    def lift(elems, r):
        out = np.empty(648, np.uint32)
        lib().orc_lb_lift(ptr(np.ascontiguousarray(elems, dtype=np.uint64)), r, ptr(out))
        return out

    @staticmethod
    def key_random(len_f162, seed, primes):
        primes = np.ascontiguousarray(primes, dtype=np.uint32)
        a = np.empty((primes.size, len_f162 // 4, 648), np.int16)
        lib().orc_lb_key_random(len_f162, seed, ptr(primes), primes.size, ptr(a))
        return a

    @staticmethod
    def commit(a, primes, len_f162, witness, r, batches=True, nthreads=0):
        """commit_scalar: (raw [limbs][r][648], matrix [4][r][limbs][162], batches [r*nr][648])."""
        primes = np.ascontiguousarray(primes, dtype=np.uint32)
        a = np.ascontiguousarray(a, dtype=np.int16)
        witness = np.ascontiguousarray(witness, dtype=np.uint64)
        limbs, nr = primes.size, len_f162 // 4
        raw = np.empty((limbs, r, 648), np.uint32)
        mat = np.empty((4, r, limbs, 162), np.int16)
        bat = np.empty((r * nr, 648), np.uint32) if batches else None
        lib().orc_lb_commit(ptr(a), ptr(primes), limbs, len_f162, ptr(witness), r, ptr(raw), ptr(mat),
                            ptr(bat) if batches else None, nthreads)
        return raw, mat, bat


# ----------------------------------------------------------------- hashing

def sha3_256(data: bytes) -> bytes:
    out = C.create_string_buffer(32)
    buf = _bytes_ptr(data)
    lib().orc_sha3_256(buf, len(data), out)
    return out.raw


def shake256(data: bytes, n: int) -> bytes:
    out = C.create_string_buffer(max(n, 1))
    buf = _bytes_ptr(data)
    lib().orc_shake256(buf, len(data), out, n)
    return out.raw[:n]


def xof(domain: bytes, msg: bytes, n: int) -> bytes:
    out = C.create_string_buffer(max(n, 1))
    lib().orc_xof(_bytes_ptr(domain), len(domain), _bytes_ptr(msg), len(msg), out, n)
    return out.raw[:n]


def hash_domain(domain: bytes, msg: bytes) -> bytes:
    out = C.create_string_buffer(32)
    lib().orc_hash_domain(_bytes_ptr(domain), len(domain), _bytes_ptr(msg), len(msg), out)
    return out.raw


def uniform_from_seed(modulus: Modulus32, log_n: int, domain: bytes, seed: bytes, index: int):
    out = np.empty(1 << log_n, dtype=np.uint32)
    lib().orc_uniform_from_seed(modulus._p(), log_n, _bytes_ptr(domain), len(domain),
                                _bytes_ptr(seed), len(seed), index, ptr(out))
    return out


def ring_random(modulus: Modulus32, log_n: int, seed: bytes):
    out = np.empty(1 << log_n, dtype=np.uint32)
    lib().orc_ring_random(modulus._p(), log_n, _bytes_ptr(seed), len(seed), ptr(out))
    return out


def ajtai32_from_seed(tables: NttTables32, k: int, m: int, seed: bytes):
    n = tables.n
    mat = np.empty(k * m * n, dtype=np.uint32)
    mat_ntt = np.empty(k * m * n, dtype=np.uint32)
    lib().orc_ajtai32_from_seed(C.byref(tables._t), k, m, _bytes_ptr(seed), ptr(mat),
                                ptr(mat_ntt))
    return mat, mat_ntt


def sample_small_secret(modulus: Modulus32, log_n: int, m: int, bound: int, seed: bytes):
    out = np.empty(m * (1 << log_n), dtype=np.uint32)
    lib().orc_sample_small_secret(modulus._p(), log_n, m, bound, _bytes_ptr(seed), len(seed),
                                  ptr(out))
    return out


# ----------------------------------------------------------------- synthetic inputs

def synth_u64(seed, stream, index):
    return lib().orc_synth_u64(seed, stream, index)


def synth_mod32(seed, stream, q, count, offset=0):
    out = np.empty(count, dtype=np.uint32)
    lib().orc_synth_mod32(seed, stream, q, ptr(out), count, offset)
    return out


def synth_gl(seed, stream, count, offset=0):
    out = np.empty(count, dtype=np.uint64)
    lib().orc_synth_gl(seed, stream, ptr(out), count, offset)
    return out


def synth_i8(seed, stream, count, offset=0):
    out = np.empty(count, dtype=np.int8)
    lib().orc_synth_i8(seed, stream, ptr(out), count, offset)
    return out


def avx512_available() -> bool:
    return bool(lib().orc_avx512_available())
