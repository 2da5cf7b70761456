"""Host-side mirror of the labinius commitment (``crates/lattice-labinius``)
over the CUDA kernels of ``lzx_b200/csrc/labinius.cu``.

Same names and argument meaning as the reference:

* :class:`Modulus`          -- ``ring::Modulus`` (ring.rs:21-68): the seven limb primes.
* :class:`CommitmentKey`    -- ``key::CommitmentKey`` (key.rs:45-474): ``random``,
  the accessors and ``commit(witness, r)``.
* :class:`CommitmentMatrix` / :class:`AuxData` -- what a commitment returns (key.rs:24-86).
* :func:`random_witness`    -- ``key::random_witness`` (key.rs:477-480).

Witnesses are F162 streams held as ``[n][3]`` uint64 arrays (numpy on the host,
or a torch int64 CUDA tensor of the same shape on the device).
"""
from __future__ import annotations

import ctypes as C
import enum

import numpy as np

from . import _lib
from ._lib import check

N, N162 = 648, 162


class Modulus(enum.Enum):
    """``Modulus`` (ring.rs:21-68): suffix _FS fully splitting, _Q quadratic slots."""

    Q2917_Q_S = 2917
    Q3889_FS_S = 3889
    Q4861_Q_S = 4861
    Q9721_FS_S = 9721
    Q12637_Q_S = 12637
    Q17497_FS_L = 17497
    Q19441_FS_L = 19441

    def prime(self) -> int:
        return self.value

    def is_quadratic(self) -> bool:
        q = self.value
        return (q - 1) % 972 == 0 and (q - 1) % 1944 != 0

    @staticmethod
    def from_prime(q: int):
        return next((m for m in Modulus if m.value == q), None)


Modulus.ALL = tuple(Modulus)
Modulus.BASE = Modulus.Q3889_FS_S


class CommitmentMatrix:
    """``CommitmentMatrix`` (key.rs:24-43): ``value[row][column][modulus]`` = 162 centered slots."""

    def __init__(self, primes, value: np.ndarray):
        self.primes = list(primes)
        self.value = value
        self.columns = value.shape[1]

    def element(self, row: int, column: int, modulus: int) -> np.ndarray:
        return self.value[row, column, modulus]

    def rows(self) -> int:
        return 4

    def cols(self) -> int:
        return self.columns


class AuxData:
    """``AuxData`` (key.rs:70-86): the base limb's transform of every ring element and the raw rows."""

    def __init__(self, batches, raw, chunks: int):
        self.batches, self.raw, self.chunks = batches, raw, chunks


def random_witness(n: int, seed: int) -> np.ndarray:
    """``random_witness`` / ``random_elems`` (key.rs:477-480, binfield.rs:177-189)."""
    out = np.empty((n, 3), dtype=np.uint64)
    check(_lib.lib().lc_lb_random_elems(n, seed, out.ctypes.data_as(C.c_void_p)), "lc_lb_random_elems")
    return out


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


class CommitmentKey:
    """``CommitmentKey`` (key.rs:45-474) with its rows resident on the GPU."""

    def __init__(self, handle, len_f162: int, limbs):
        self._h = handle
        self._len = len_f162
        self._limbs = list(limbs)

    @staticmethod
    def random(len_f162: int, seed: int, base: Modulus = Modulus.BASE, additional=()) -> "CommitmentKey":
        """``CommitmentKey::random`` (key.rs:94-137), bit-identical rows."""
        limbs = [base] + list(additional)
        primes = (C.c_uint16 * len(limbs))(*[m.prime() for m in limbs])
        h = C.c_void_p()
        check(_lib.lib().lc_lb_key_random(len_f162, seed, primes, len(limbs), C.byref(h)), "lc_lb_key_random")
        return CommitmentKey(h, len_f162, limbs)

    @staticmethod
    def from_rows(len_f162: int, limbs, a: np.ndarray) -> "CommitmentKey":
        """A key from explicit centered rows ``a[limb][i][648]``."""
        limbs = list(limbs)
        a = np.ascontiguousarray(a, dtype=np.int16)
        primes = (C.c_uint16 * len(limbs))(*[m.prime() for m in limbs])
        h = C.c_void_p()
        check(_lib.lib().lc_lb_key_create(len_f162, primes, len(limbs), a.ctypes.data_as(C.c_void_p), C.byref(h)),
              "lc_lb_key_create")
        return CommitmentKey(h, len_f162, limbs)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.lc_lb_key_destroy(h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def len_f162(self) -> int:
        return self._len

    def len_ring(self) -> int:
        return self._len // 4

    def limbs(self) -> int:
        return len(self._limbs)

    def base(self) -> Modulus:
        return self._limbs[0]

    def additional(self):
        return self._limbs[1:]

    def limb(self, k: int) -> Modulus:
        return self._limbs[k]

    def prime(self, k: int) -> int:
        return self._limbs[k].prime()

    def is_quadratic(self, k: int) -> bool:
        return self._limbs[k].is_quadratic()

    def bytes(self) -> int:
        return self.limbs() * self.len_ring() * 2 * N

    @property
    def a(self) -> np.ndarray:
        """The centered transform-domain rows ``[limb][i][648]``."""
        out = np.empty((self.limbs(), self.len_ring(), N), dtype=np.int16)
        check(_lib.lib().lc_lb_key_info(self._h, None, None, None, out.ctypes.data_as(C.c_void_p)), "lc_lb_key_info")
        return out

    def commit(self, witness, r: int, batches: bool = True):
        """``CommitmentKey::commit`` (key.rs:223-231): (CommitmentMatrix, AuxData)."""
        limbs, nr = self.limbs(), self.len_ring()
        L = _lib.lib()
        if _is_torch_cuda(witness):
            import torch
            if tuple(witness.shape) != (r * self._len, 3) or not witness.is_contiguous():
                raise _lib.LatticeCudaError(_lib.LC_ERR_INVALID_ARGUMENT, "witness must be [r * len_f162][3]")
            dev = witness.device
            raw = torch.empty((limbs, r, N), dtype=torch.int32, device=dev)
            mat = torch.empty((4, r, limbs, N162), dtype=torch.int16, device=dev)
            bat = torch.empty((r * nr, N), dtype=torch.int32, device=dev) if batches else None
            st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
            check(L.lc_lb_commit(self._h, C.c_void_p(witness.data_ptr()), r, C.c_void_p(raw.data_ptr()),
                                 C.c_void_p(mat.data_ptr()), C.c_void_p(bat.data_ptr()) if batches else None, st),
                  "lc_lb_commit")
            return (CommitmentMatrix([m.prime() for m in self._limbs], mat),
                    AuxData(bat, raw, r))
        w = np.ascontiguousarray(witness, dtype=np.uint64)
        if w.shape != (r * self._len, 3):
            raise _lib.LatticeCudaError(_lib.LC_ERR_INVALID_ARGUMENT, "witness must be [r * len_f162][3]")
        raw = np.empty((limbs, r, N), dtype=np.uint32)
        mat = np.empty((4, r, limbs, N162), dtype=np.int16)
        bat = np.empty((r * nr, N), dtype=np.uint32) if batches else None
        check(L.lc_lb_commit_host(self._h, w.ctypes.data_as(C.c_void_p), r, raw.ctypes.data_as(C.c_void_p),
                                  mat.ctypes.data_as(C.c_void_p),
                                  bat.ctypes.data_as(C.c_void_p) if batches else None), "lc_lb_commit_host")
        return CommitmentMatrix([m.prime() for m in self._limbs], mat), AuxData(bat, raw, r)
