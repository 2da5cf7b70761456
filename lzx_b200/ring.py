"""Host-side mirror of the reference ring API over the CUDA NTT.

Same names, argument meaning and error behaviour as idrees2516/lzx's
``lattice-ring`` crate:

* :class:`Modulus32`      -- ``lattice-ring/src/modulus.rs:22-161``
* :class:`NttTables`      -- ``lattice-ring/src/ntt.rs:16-317`` (``new``,
  ``forward``/``forward_fast``, ``inverse``/``inverse_fast``), batched; the
  transform runs on the GPU through ``lc_ntt_*`` of the C ABI.
* :class:`RingConfig`, :class:`RingElement` -- ``lattice-ring/src/ring.rs``.
* :class:`GoldilocksNttTables` -- the same transform over Goldilocks
  (``lattice-core/src/field.rs``), the extension the commitment path uses.

Arrays are numpy (host) or torch CUDA tensors (device).  Host arrays go
through the synchronous host-buffer entry points; CUDA tensors go through the
device entry points on torch's current stream.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import struct
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import LatticeCudaError, check

GOLDILOCKS_P = 0xFFFFFFFF00000001


# --------------------------------------------------------------------------- errors

class NttError(Exception):
    """``NttError`` (lattice-ring/src/ntt.rs:38-42)."""

    LengthMismatch = "LengthMismatch"
    AdicityTooSmall = "AdicityTooSmall"

    def __init__(self, kind: str):
        super().__init__(kind)
        self.kind = kind

    def __eq__(self, other):
        return isinstance(other, NttError) and other.kind == self.kind

    __hash__ = Exception.__hash__


class RingError(Exception):
    """``RingError`` (lattice-ring/src/ring.rs:17-21)."""

    def __init__(self, kind: str, expected=None, got=None):
        super().__init__(kind if expected is None else f"{kind} {{expected: {expected}, got: {got}}}")
        self.kind, self.expected, self.got = kind, expected, got


def _raise_for(status: int, where: str):
    if status == _lib.LC_ERR_LENGTH_MISMATCH:
        raise NttError(NttError.LengthMismatch)
    if status == _lib.LC_ERR_ADICITY_TOO_SMALL:
        raise NttError(NttError.AdicityTooSmall)
    check(status, where)


# --------------------------------------------------------------------------- Modulus32

@dataclass(frozen=True)
class Modulus32:
    """``Modulus32`` (modulus.rs:22-44): a u32 NTT prime with its root metadata."""

    q: int
    two_adicity: int
    generator: int

    def root_of_unity(self, k: int):
        """``root_of_unity`` (modulus.rs:149-156)."""
        if k > self.two_adicity:
            return None
        return pow(self.generator, (self.q - 1) >> k, self.q)

    def root_of_unity_order_2n(self, k: int):
        return self.root_of_unity(k + 1)


Modulus32.Q_32 = Modulus32(3221225473, 30, 5)            # modulus.rs:48
Modulus32.Q_12289 = Modulus32(12289, 12, 11)             # modulus.rs:52
Modulus32.Q_2013265921 = Modulus32(2013265921, 27, 31)   # modulus.rs:55

# The four largest 30-bit primes q == 1 (mod 512) -- a CRT set for d <= 256.
CRT_SET_30BIT = (
    Modulus32(1073738753, 10, 3),
    Modulus32(1073732609, 10, 3),
    Modulus32(1073731073, 9, 3),
    Modulus32(1073726977, 9, 5),
)


# --------------------------------------------------------------------------- plans

def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _current_stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class _Plan:
    """Owns one ``lc_ntt_plan``."""

    elem_dtype = np.uint32

    def __init__(self, handle: C.c_void_p, n: int, num_moduli: int):
        self._h = handle
        self.n = n
        self.num_moduli = num_moduli

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.lc_ntt_plan_destroy(h)
            self._h = None

    def _count(self, size: int) -> int:
        per = self.n * self.num_moduli
        if size % per:
            raise NttError(NttError.LengthMismatch)
        return size // per

    def _run(self, a, inverse: bool, out=None):
        L = _lib.lib()
        if _is_torch_cuda(a):
            count = self._count(a.numel())
            if not a.is_contiguous():
                raise LatticeCudaError(_lib.LC_ERR_INVALID_ARGUMENT, "tensor must be contiguous")
            dst = a if out is None else out
            fn = L.lc_ntt_inverse if inverse else L.lc_ntt_forward
            st = fn(self._h, C.c_void_p(a.data_ptr()), C.c_void_p(dst.data_ptr()), count,
                    _current_stream())
            _raise_for(st, "lc_ntt_inverse" if inverse else "lc_ntt_forward")
            return dst
        arr = np.ascontiguousarray(a, dtype=self.elem_dtype)
        count = self._count(arr.size)
        dst = arr if out is None else out
        fn = L.lc_ntt_inverse_host if inverse else L.lc_ntt_forward_host
        st = fn(self._h, arr.ctypes.data_as(C.c_void_p), dst.ctypes.data_as(C.c_void_p), count)
        _raise_for(st, "lc_ntt_inverse_host" if inverse else "lc_ntt_forward_host")
        return dst


class NttTables(_Plan):
    """``NttTables`` (ntt.rs:16-317) for one modulus or a CRT set sharing ``log_n``.

    ``forward_fast(a)`` / ``inverse_fast(a)`` transform ``a`` in place and
    return it.  ``a`` holds ``count`` polynomials per modulus, laid out
    ``[modulus][count][n]``; a length that is not a multiple of ``n`` raises
    ``NttError.LengthMismatch`` exactly as the reference does.
    """

    elem_dtype = np.uint32

    def __init__(self, modulus, log_n: int):
        mods = list(modulus) if isinstance(modulus, (list, tuple)) else [modulus]
        arr = lambda xs: (C.c_uint32 * len(xs))(*xs)
        h = C.c_void_p()
        st = _lib.lib().lc_ntt_plan_create_u32(
            log_n, arr([m.q for m in mods]), arr([m.two_adicity for m in mods]),
            arr([m.generator for m in mods]), len(mods), C.byref(h))
        _raise_for(st, "lc_ntt_plan_create_u32")
        super().__init__(h, 1 << log_n, len(mods))
        self.moduli = tuple(mods)
        self.modulus = mods[0]
        self.log_n = log_n

    @classmethod
    def new(cls, modulus, log_n: int) -> "NttTables":
        return cls(modulus, log_n)

    def forward_fast(self, a, out=None):
        return self._run(a, False, out)

    def inverse_fast(self, a, out=None):
        return self._run(a, True, out)

    # the reference's generic paths compute the same values (ntt.rs:439-467)
    forward = forward_fast
    inverse = inverse_fast

    def forward_partial(self, a, levels: int):
        """``forward_partial`` (ntt.rs:252-286) in place on the GPU."""
        return self._run_partial(a, levels, _lib.lib().lc_ntt_forward_partial, "lc_ntt_forward_partial")

    def complete_partial(self, a, already: int):
        """``complete_partial`` (ntt.rs:288-316) in place on the GPU."""
        return self._run_partial(a, already, _lib.lib().lc_ntt_complete_partial, "lc_ntt_complete_partial")

    def _run_partial(self, a, lv, fn, name):
        import torch
        on_dev = _is_torch_cuda(a)
        t = a if on_dev else torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()
        count = self._count(t.numel())
        _raise_for(fn(self._h, C.c_void_p(t.data_ptr()), C.c_void_p(t.data_ptr()), count, lv, _current_stream()),
                   name)
        if on_dev:
            return t
        torch.cuda.synchronize()
        out = t.cpu().numpy().view(np.uint32)
        if isinstance(a, np.ndarray) and a.dtype == np.uint32 and a.flags.writeable:
            a[...] = out.reshape(a.shape)
            return a
        return out


class GoldilocksNttTables(_Plan):
    """The ``ntt.rs`` transform over Goldilocks (field.rs), generator 7."""

    elem_dtype = np.uint64

    def __init__(self, log_n: int):
        h = C.c_void_p()
        _raise_for(_lib.lib().lc_ntt_plan_create_goldilocks(log_n, C.byref(h)),
                   "lc_ntt_plan_create_goldilocks")
        super().__init__(h, 1 << log_n, 1)
        self.log_n = log_n

    def forward_fast(self, a, out=None):
        return self._run(a, False, out)

    def inverse_fast(self, a, out=None):
        return self._run(a, True, out)

    forward = forward_fast
    inverse = inverse_fast


# --------------------------------------------------------------------------- ring

def _xof(domain: bytes, message: bytes, out_len: int) -> bytes:
    """``Transcript::xof`` (lattice-core/src/transcript.rs:229-237)."""
    framed = (b"LZXX" + struct.pack("<I", len(domain)) + domain + struct.pack("<I", len(message))
              + message)
    return hashlib.shake_256(framed).digest(out_len)


class RingConfig:
    """``RingConfig`` (ring.rs:11-181): modulus + log_n + shared NTT plan."""

    def __init__(self, modulus: Modulus32, log_n: int):
        self.modulus = modulus
        self.log_n = log_n
        self.tables = NttTables(modulus, log_n)  # NttTables::new -> RingError::Ntt

    @classmethod
    def new(cls, modulus: Modulus32, log_n: int) -> "RingConfig":
        return cls(modulus, log_n)

    def n(self) -> int:
        return 1 << self.log_n

    def __eq__(self, other):
        return (isinstance(other, RingConfig) and self.modulus.q == other.modulus.q
                and self.log_n == other.log_n)

    def zero(self):
        return RingElement(self, np.zeros(self.n(), dtype=np.uint32))

    def one(self):
        c = np.zeros(self.n(), dtype=np.uint32)
        c[0] = 1
        return RingElement(self, c)

    def x_gen(self):
        c = np.zeros(self.n(), dtype=np.uint32)
        c[1] = 1
        return RingElement(self, c)

    def constant(self, c: int):
        v = np.zeros(self.n(), dtype=np.uint32)
        v[0] = c % self.modulus.q
        return RingElement(self, v)

    def random(self, seed: bytes):
        """``RingConfig::random`` (ring.rs:83-98)."""
        b = np.frombuffer(_xof(b"ring-random", seed, self.n() * 4), dtype="<u4")
        return RingElement(self, (b.astype(np.uint64) % self.modulus.q).astype(np.uint32))

    def uniform_from_seed(self, domain: bytes, seed: bytes, index: int):
        """``RingConfig::uniform_from_seed`` (ring.rs:102-180): one element,
        expanded on the GPU by ``lc_uniform_from_seed`` with count 1."""
        import torch
        out = self.uniform_from_seed_batch(domain, seed, index, 1)
        torch.cuda.synchronize()
        return RingElement(self, out[0].cpu().numpy().view(np.uint32).copy())

    def uniform_from_seed_batch(self, domain: bytes, seed: bytes, index0: int, count: int, out=None):
        """``uniform_from_seed`` for indices index0 .. index0+count-1 on the GPU
        (``lc_uniform_from_seed``): a CUDA int32 tensor [count][n] of the residues."""
        import torch
        n = self.n()
        if out is None:
            out = torch.empty((count, n), dtype=torch.int32, device="cuda")
        st = _lib.lib().lc_uniform_from_seed(self.tables.handle, domain, len(domain), seed, len(seed), index0, count,
                                             C.c_void_p(out.data_ptr()), _current_stream())
        _raise_for(st, "lc_uniform_from_seed")
        return out


class RingElement:
    """``RingElement`` (ring.rs:183-447)."""

    def __init__(self, config: RingConfig, coeffs):
        self.config = config
        self._c = np.ascontiguousarray(coeffs, dtype=np.uint32)

    @classmethod
    def from_coeffs(cls, config: RingConfig, coeffs):
        return cls(config, coeffs)

    @classmethod
    def from_signed(cls, config: RingConfig, signed: Sequence[int]):
        q = config.modulus.q
        c = np.zeros(config.n(), dtype=np.uint32)
        vals = np.array([s % q for s in signed], dtype=np.uint64)
        c[: len(vals)] = vals
        return cls(config, c)

    def coeffs(self) -> np.ndarray:
        return self._c

    def is_zero(self) -> bool:
        return not self._c.any()

    def __eq__(self, other):
        return (isinstance(other, RingElement) and self.config == other.config
                and np.array_equal(self._c, other._c))

    def _zip(self, other, f):
        if self.config != other.config:
            raise RingError("LengthMismatch", len(self._c), len(other._c))
        return RingElement(self.config, f(self._c.astype(np.uint64), other._c.astype(np.uint64)))

    def add(self, other):
        q = self.config.modulus.q
        return self._zip(other, lambda a, b: ((a + b) % q).astype(np.uint32))

    def sub(self, other):
        q = self.config.modulus.q
        return self._zip(other, lambda a, b: ((a + q - b) % q).astype(np.uint32))

    def neg(self):
        q = self.config.modulus.q
        return RingElement(self.config, ((q - self._c.astype(np.uint64)) % q).astype(np.uint32))

    def to_ntt(self) -> np.ndarray:
        """``to_ntt`` (ring.rs:344-351): evaluations in the reference's order."""
        return self.config.tables.forward_fast(self._c.copy())

    @classmethod
    def from_ntt(cls, config: RingConfig, evals):
        """``from_ntt`` (ring.rs:354-367)."""
        evals = np.asarray(evals, dtype=np.uint32)
        if evals.size != config.n():
            raise RingError("LengthMismatch", config.n(), evals.size)
        return cls(config, config.tables.inverse_fast(evals.copy()))

    def mul(self, other):
        """Negacyclic product (ring.rs:309-340): two forward NTTs, pointwise, inverse."""
        if self.config != other.config:
            raise RingError("LengthMismatch", len(self._c), len(other._c))
        q = self.config.modulus.q
        both = np.stack([self._c, other._c]).copy()
        self.config.tables.forward_fast(both)
        prod = (both[0].astype(np.uint64) * both[1].astype(np.uint64) % q).astype(np.uint32)
        return RingElement(self.config, self.config.tables.inverse_fast(prod))

    def to_bytes(self) -> bytes:
        return self._c.astype("<u4").tobytes()

    @classmethod
    def from_bytes(cls, config: RingConfig, data: bytes):
        """``from_bytes`` (ring.rs:381-407): rejects wrong length and values >= q."""
        n = config.n()
        if len(data) != n * 4:
            raise RingError("LengthMismatch", n * 4, len(data))
        v = np.frombuffer(data, dtype="<u4").astype(np.uint32)
        bad = v >= config.modulus.q
        if bad.any():
            raise RingError("LengthMismatch", 0, int(v[bad][0]))
        return cls(config, v.copy())

    def infinity_norm(self) -> int:
        q = self.config.modulus.q
        c = self._c.astype(np.int64)
        return int(np.where(c <= q // 2, c, q - c).max(initial=0))
