"""Host-side mirror of lattice-ring's ~2^50 modulus class over the CUDA kernels.

Same names, argument meaning and error behaviour as the reference's
``lattice-ring/src/modulus50.rs``:

* :class:`Modulus50`      -- ``Modulus50`` (:53-198): the prime, its two-adicity
  and generator; ``Q_50 = 2^50 - 2687`` (:44-51).
* :class:`QuadSlotTables` -- ``QuadSlotTables`` (:206-411): ``new``,
  ``forward``, ``inverse``, ``slotwise_mul``, ``mul``, batched over
  ``[count][n]`` arrays and run by ``lc_quad50_*`` of the C ABI.
* :class:`RingConfig50`   -- ``RingConfig50`` (:414-497).

Arrays are numpy uint64 (host) or torch int64 CUDA tensors holding the u64
residues (device).  Device tensors run on torch's current stream; host
arrays are staged through the device (``mul`` uses the host-buffer entry
point).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check

Q_50 = 1125899906839937  # 2^50 - 2687, modulus50.rs:44
Q_50_TWO_ADICITY = 7     # :47
Q_50_GENERATOR = 3       # :50


class Mod50Error(Exception):
    """``Mod50Error`` (modulus50.rs:416-422)."""

    LogNOutOfRange = "LogNOutOfRange"
    AdicityTooSmall = "AdicityTooSmall"
    GeneratorInvalid = "GeneratorInvalid"
    LengthMismatch = "LengthMismatch"

    def __init__(self, kind: str, **fields):
        detail = ", ".join(f"{k}: {v}" for k, v in fields.items())
        super().__init__(f"{kind} {{{detail}}}" if fields else kind)
        self.kind, self.fields = kind, fields


@dataclass(frozen=True)
class Modulus50:
    """``Modulus50`` (modulus50.rs:53-83): a ~2^50 prime with its root metadata."""

    q: int
    two_adicity: int
    generator: int

    @staticmethod
    def new(q: int, two_adicity: int, generator: int) -> "Modulus50":
        return Modulus50(q, two_adicity, generator)

    def root_of_unity(self, k: int):
        """``root_of_unity`` (:191-197)."""
        if k > self.two_adicity:
            return None
        return pow(self.generator, (self.q - 1) >> k, self.q)


Modulus50.Q_50 = Modulus50(Q_50, Q_50_TWO_ADICITY, Q_50_GENERATOR)


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class QuadSlotTables:
    """``QuadSlotTables`` (modulus50.rs:206-411) for n = 2^log_n, log_n in [1, 7]."""

    def __init__(self, modulus: Modulus50, log_n: int):
        L = _lib.lib()
        h = C.c_void_p()
        st = L.lc_quad50_plan_create(modulus.q, modulus.two_adicity, modulus.generator, log_n, C.byref(h))
        if st == _lib.LC_ERR_LOG_N_OUT_OF_RANGE:
            raise Mod50Error(Mod50Error.LogNOutOfRange, got=log_n)
        if st == _lib.LC_ERR_ADICITY_TOO_SMALL:
            raise Mod50Error(Mod50Error.AdicityTooSmall, got=modulus.two_adicity)
        if st == _lib.LC_ERR_GENERATOR_INVALID:
            raise Mod50Error(Mod50Error.GeneratorInvalid)
        check(st, "lc_quad50_plan_create")
        self._h = h
        self.modulus, self.log_n = modulus, log_n
        z = C.c_uint64()
        gam = (C.c_uint64 * (self.n // 2))()
        check(L.lc_quad50_plan_info(h, C.byref(z), gam), "lc_quad50_plan_info")
        self.zeta = z.value
        self.leaf_gamma = np.frombuffer(gam, dtype=np.uint64).copy()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.lc_quad50_plan_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    @property
    def n(self) -> int:
        return 1 << self.log_n

    def slots(self) -> int:
        return self.n // 2

    def _count(self, size: int) -> int:
        if size == 0 or size % self.n:
            raise Mod50Error(Mod50Error.LengthMismatch, expected=self.n, got=size)
        return size // self.n

    def _run(self, fn: str, *ops):
        """Device tensors in place of host arrays: out = fn(ops...) as a new array."""
        import torch
        host = not _is_torch_cuda(ops[0])
        shape = np.shape(ops[0])
        if host:
            ops = tuple(torch.from_numpy(np.ascontiguousarray(o, dtype=np.uint64).view(np.int64)).cuda()
                        for o in ops)
        for o in ops:
            if not _is_torch_cuda(o) or not o.is_contiguous() or o.dtype != torch.int64:
                raise _lib.LatticeCudaError(_lib.LC_ERR_INVALID_ARGUMENT, "contiguous int64 CUDA tensors")
            if o.numel() != ops[0].numel():
                raise Mod50Error(Mod50Error.LengthMismatch, expected=ops[0].numel(), got=o.numel())
        count = self._count(ops[0].numel())
        out = torch.empty_like(ops[0])
        args = [C.c_void_p(o.data_ptr()) for o in ops]
        check(getattr(_lib.lib(), fn)(self._h, *args, C.c_void_p(out.data_ptr()), count, _stream()), fn)
        if host:
            return out.cpu().numpy().view(np.uint64).reshape(shape)
        return out

    def forward(self, a):
        """``forward`` (:313-334): coefficients -> quadratic slots."""
        return self._run("lc_quad50_forward", a)

    def inverse(self, a):
        """``inverse`` (:338-364)."""
        return self._run("lc_quad50_inverse", a)

    def slotwise_mul(self, a, b):
        """``slotwise_mul`` (:368-392) of slot-form operands."""
        return self._run("lc_quad50_slotwise_mul", a, b)

    def mul(self, a, b):
        """``mul`` (:395-411): ring products in Z_q[X]/(X^n + 1)."""
        if _is_torch_cuda(a):
            return self._run("lc_quad50_mul", a, b)
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = np.ascontiguousarray(b, dtype=np.uint64)
        if a.size != b.size:
            raise Mod50Error(Mod50Error.LengthMismatch, expected=a.size, got=b.size)
        count = self._count(a.size)
        out = np.empty_like(a)
        st = _lib.lib().lc_quad50_mul_host(self._h, a.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p),
                                           out.ctypes.data_as(C.c_void_p), count)
        check(st, "lc_quad50_mul_host")
        return out


class RingConfig50:
    """``RingConfig50`` (modulus50.rs:414-497)."""

    def __init__(self, log_n: int, modulus: Modulus50 = Modulus50.Q_50):
        self.modulus, self.log_n = modulus, log_n
        self.tables = QuadSlotTables(modulus, log_n)

    @staticmethod
    def new(log_n: int) -> "RingConfig50":
        return RingConfig50(log_n)

    @staticmethod
    def with_modulus(modulus: Modulus50, log_n: int) -> "RingConfig50":
        return RingConfig50(log_n, modulus)

    def n(self) -> int:
        return 1 << self.log_n

    def slot_constants(self) -> np.ndarray:
        return self.tables.leaf_gamma

    def mul(self, a, b):
        return self.tables.mul(a, b)

    def _pair(self, a, b):
        a = np.asarray(a, dtype=np.uint64)
        b = np.asarray(b, dtype=np.uint64)
        if a.size != self.n() or b.size != self.n():
            raise Mod50Error(Mod50Error.LengthMismatch, expected=self.n(), got=a.size)
        return a.astype(object), b.astype(object)

    def add(self, a, b):
        """Pointwise addition (:456-468), host-side."""
        a, b = self._pair(a, b)
        return np.array([(x + y) % self.modulus.q for x, y in zip(a, b)], dtype=np.uint64)

    def sub(self, a, b):
        """Pointwise subtraction (:471-483), host-side."""
        a, b = self._pair(a, b)
        return np.array([(x - y) % self.modulus.q for x, y in zip(a, b)], dtype=np.uint64)

    def from_signed(self, signed):
        """From balanced coefficients (:486-492): the first n values, zero-padded."""
        out = np.zeros(self.n(), dtype=np.uint64)
        for i, s in enumerate(list(signed)[: self.n()]):
            out[i] = int(s) % self.modulus.q
        return out

    def infinity_norm(self, a) -> int:
        """Infinity norm of the balanced representative (:495-502)."""
        half = self.modulus.q // 2
        return max((int(c) if int(c) <= half else self.modulus.q - int(c) for c in np.asarray(a)), default=0)
