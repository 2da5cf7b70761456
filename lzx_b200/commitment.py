"""Host-side mirror of the reference commitment API over the CUDA commit.

Same names, argument meaning and error behaviour as idrees2516/lzx's
``lattice-commitment`` crate (``src/ajtai.rs``):

* :class:`AjtaiParams`, :class:`AjtaiError`, :class:`AjtaiPublicKey`
  (``from_seed`` :87-103, ``entry`` :106, ``commit`` :118-153,
  ``commit_naive_reference`` :158-180, ``verify_opening`` :210-230,
  ``pad_to_m`` :245-257), :class:`AjtaiCommitment` (:261-295) and
  :func:`sample_small_secret` (:307-348).
* :class:`GoldilocksAjtaiKey`: the same cached-NTT commitment over Goldilocks
  for batches of witnesses given as residues or int8 digits.

The seed expansion (SHAKE-256, ``lc_uniform_from_seed``), the cached NTT(A)
and every commit run on the GPU (``lc_ajtai_*`` of the C ABI).
"""
from __future__ import annotations

import ctypes as C
import struct
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import LatticeCudaError, check
from .ring import (GOLDILOCKS_P, GoldilocksNttTables, RingConfig, RingElement, RingError, _xof,
                   _is_torch_cuda, _current_stream)


class AjtaiError(Exception):
    """``AjtaiError`` (ajtai.rs:43-49)."""

    def __init__(self, kind: str, **fields):
        super().__init__(kind + (f" {fields}" if fields else ""))
        self.kind = kind
        self.fields = fields


@dataclass
class AjtaiParams:
    """``AjtaiParams`` (ajtai.rs:31-41)."""

    ring: RingConfig
    k: int
    m: int
    norm_bound: int


def _map_status(st: int, where: str):
    if st == _lib.LC_ERR_DIMENSION_MISMATCH:
        raise AjtaiError("DimensionMismatch")
    check(st, where)


class _DeviceKey:
    """Owns one ``lc_ajtai_key``."""

    def __init__(self, plan, k: int, m: int, matrix, flags: int = 0):
        h = C.c_void_p()
        if _is_torch_cuda(matrix):
            matrix = matrix.contiguous()
            ptr, on_dev = C.c_void_p(matrix.data_ptr()), 1
        else:
            matrix = np.ascontiguousarray(matrix)
            ptr, on_dev = matrix.ctypes.data_as(C.c_void_p), 0
        _map_status(_lib.lib().lc_ajtai_key_create_ex(plan.handle, k, m, ptr, on_dev, flags, C.byref(h)),
                    "lc_ajtai_key_create_ex")
        self._h = h
        self.k, self.m, self.n = k, m, plan.n
        self.elem_dtype = plan.elem_dtype

    @property
    def handle(self):
        return self._h

    @property
    def engine(self) -> int:
        return _lib.lib().lc_ajtai_key_get_engine(self._h)

    @engine.setter
    def engine(self, value: int):
        check(_lib.lib().lc_ajtai_key_set_engine(self._h, int(value)), "lc_ajtai_key_set_engine")

    @property
    def fused(self) -> int:
        """One-launch forms (lc_ajtai_key_set_fused): 0 never, 1 where they are
        faster (the default), 2 for every batch shape; truthy unless 0."""
        return _lib.lib().lc_ajtai_key_get_fused(self._h)

    @fused.setter
    def fused(self, value):
        level = value if isinstance(value, int) and not isinstance(value, bool) else (1 if value else 0)
        check(_lib.lib().lc_ajtai_key_set_fused(self._h, level), "lc_ajtai_key_set_fused")

    @property
    def slot_products(self) -> int:
        """LC_PRODUCTS_TENSOR or LC_PRODUCTS_INT64 (lc_ajtai_key_set_slot_products)."""
        return _lib.lib().lc_ajtai_key_get_slot_products(self._h)

    @slot_products.setter
    def slot_products(self, value: int):
        check(_lib.lib().lc_ajtai_key_set_slot_products(self._h, int(value)), "lc_ajtai_key_set_slot_products")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.lc_ajtai_key_destroy(h)
            self._h = None

    def commit_array(self, w, out=None):
        """Batch commit: w [B][m][n] (residues, int8 or uint8 digits) -> [B][k][n]."""
        L = _lib.lib()
        if _is_torch_cuda(w):
            import torch
            batch = w.numel() // (self.m * self.n)
            if batch * self.m * self.n != w.numel():
                raise AjtaiError("DimensionMismatch", expected=self.m * self.n, got=w.numel())
            if out is None:
                dt = torch.int64 if self.elem_dtype == np.uint64 else torch.int32
                out = torch.empty((batch, self.k, self.n), dtype=dt, device=w.device)
            fn = {torch.int8: L.lc_ajtai_commit_i8, torch.uint8: L.lc_ajtai_commit_u8}.get(
                w.dtype, L.lc_ajtai_commit)
            _map_status(fn(self._h, C.c_void_p(w.data_ptr()), batch, C.c_void_p(out.data_ptr()),
                           _current_stream()), "lc_ajtai_commit")
            return out
        w = np.ascontiguousarray(w)
        batch = w.size // (self.m * self.n)
        if batch * self.m * self.n != w.size:
            raise AjtaiError("DimensionMismatch", expected=self.m * self.n, got=w.size)
        res = np.empty((batch, self.k, self.n), dtype=self.elem_dtype) if out is None else out
        if w.dtype in (np.int8, np.uint8):
            fn = L.lc_ajtai_commit_i8_host if w.dtype == np.int8 else L.lc_ajtai_commit_u8_host
            st = fn(self._h, w.ctypes.data_as(C.c_void_p), batch, res.ctypes.data_as(C.c_void_p))
        else:
            w = w.astype(self.elem_dtype, copy=False)
            st = L.lc_ajtai_commit_host(self._h, w.ctypes.data_as(C.c_void_p), batch,
                                        res.ctypes.data_as(C.c_void_p))
        _map_status(st, "lc_ajtai_commit_host")
        return res


class AjtaiCommitment:
    """``AjtaiCommitment`` (ajtai.rs:261-295): k ring elements."""

    def __init__(self, rows: Sequence[RingElement]):
        self.rows = list(rows)

    def __eq__(self, other):
        return isinstance(other, AjtaiCommitment) and len(self.rows) == len(other.rows) and all(
            a == b for a, b in zip(self.rows, other.rows))

    def to_bytes(self) -> bytes:
        return b"".join(r.to_bytes() for r in self.rows)

    @classmethod
    def from_bytes(cls, ring: RingConfig, k: int, data: bytes) -> "AjtaiCommitment":
        expected = k * ring.n() * 4
        if len(data) != expected:
            raise AjtaiError("DimensionMismatch", expected=expected, got=len(data))
        el = ring.n() * 4
        try:
            return cls([RingElement.from_bytes(ring, data[i * el:(i + 1) * el]) for i in range(k)])
        except RingError as e:
            raise AjtaiError("Ring", error=e) from e


class AjtaiPublicKey:
    """``AjtaiPublicKey`` (ajtai.rs:51-258) with its cached NTT(A) on the GPU."""

    def __init__(self, params: AjtaiParams, seed: bytes, matrix: np.ndarray):
        self.params = params
        self.seed = bytes(seed)
        self._matrix = matrix  # [k*m][n] coefficient form
        self._dev = _DeviceKey(params.ring.tables, params.k, params.m, matrix)

    @classmethod
    def from_seed(cls, params: AjtaiParams, seed: bytes) -> "AjtaiPublicKey":
        """Expand A[i][j] = uniform_from_seed(b"ajtai-A", seed, i*m + j) (ajtai.rs:87-103)
        on the GPU (``lc_uniform_from_seed``); NTT(A) is cached from the device copy."""
        if len(seed) != 32:
            raise ValueError("seed must be 32 bytes")
        import torch
        dev = params.ring.uniform_from_seed_batch(b"ajtai-A", seed, 0, params.k * params.m)
        key = cls.__new__(cls)
        key.params, key.seed = params, bytes(seed)
        key._dev = _DeviceKey(params.ring.tables, params.k, params.m, dev)
        torch.cuda.synchronize()
        key._matrix = dev.cpu().numpy().view(np.uint32)
        return key

    @property
    def fused(self) -> bool:
        """Small commitments as one launch (the default); False runs them staged."""
        return self._dev.fused

    @fused.setter
    def fused(self, value: bool):
        self._dev.fused = value

    @property
    def slot_products(self) -> int:
        """Per-slot products of staged commits: LC_PRODUCTS_TENSOR (byte-limb GEMMs
        on the tensor cores, the default) or LC_PRODUCTS_INT64."""
        return self._dev.slot_products

    @slot_products.setter
    def slot_products(self, value: int):
        self._dev.slot_products = value

    def entry(self, i: int, j: int):
        if i < self.params.k and j < self.params.m:
            return RingElement(self.params.ring, self._matrix[i * self.params.m + j].copy())
        return None

    def _as_array(self, s: Sequence[RingElement]) -> np.ndarray:
        if len(s) != self.params.m:
            raise AjtaiError("DimensionMismatch", expected=self.params.m, got=len(s))
        return np.stack([e.coeffs() for e in s]).astype(np.uint32)

    def commit(self, s: Sequence[RingElement]) -> AjtaiCommitment:
        """``commit`` (ajtai.rs:118-153) on the GPU."""
        rows = self._dev.commit_array(self._as_array(s))[0]
        return AjtaiCommitment([RingElement(self.params.ring, r) for r in rows])

    def commit_batch(self, s):
        """Commit B witness vectors at once: s [B][m][n] -> [B][k][n] residues."""
        return self._dev.commit_array(s)

    def commit_naive_reference(self, s: Sequence[RingElement]) -> AjtaiCommitment:
        """``commit_naive_reference`` (ajtai.rs:158-180): per-product ring multiply."""
        arr = self._as_array(s)
        ring = self.params.ring
        rows = []
        for i in range(self.params.k):
            acc = ring.zero()
            for j in range(self.params.m):
                if not arr[j].any():
                    continue
                acc = acc.add(self.entry(i, j).mul(RingElement(ring, arr[j])))
            rows.append(acc)
        return AjtaiCommitment(rows)

    def verify_opening(self, commitment: AjtaiCommitment, s: Sequence[RingElement]) -> None:
        """``verify_opening`` (ajtai.rs:210-230): norm check, recommit, compare."""
        bound = self.params.norm_bound
        for e in s:
            if e.infinity_norm() > bound:
                raise AjtaiError("NormExceeded", norm=e.infinity_norm(), bound=bound)
        if self.commit(s).rows != commitment.rows:
            raise AjtaiError("CommitmentMismatch")

    def pad_to_m(self, elems: Sequence[RingElement]):
        if len(elems) > self.params.m:
            raise AjtaiError("DimensionMismatch", expected=self.params.m, got=len(elems))
        return list(elems) + [self.params.ring.zero() for _ in range(self.params.m - len(elems))]


def sample_small_secret(ring: RingConfig, m: int, bound: int, seed: bytes):
    """``sample_small_secret`` (ajtai.rs:307-348)."""
    n, q = ring.n(), ring.modulus.q
    span = 2 * bound + 1
    limit = (0xFFFFFFFF // span) * span
    out = []
    for i in range(m):
        coeffs = []
        sc = 0
        while len(coeffs) < n:
            inp = seed + struct.pack("<Q", i) + struct.pack("<Q", sc)
            v = np.frombuffer(_xof(b"ajtai-secret", inp, max(n * 16, 64)), dtype="<u4")
            v = v[v < limit][: n - len(coeffs)].astype(np.int64)
            coeffs.extend(((v % span - bound) % q).tolist())
            sc += 1
        out.append(RingElement(ring, np.array(coeffs, dtype=np.uint32)))
    return out


class GoldilocksAjtaiKey:
    """Cached-NTT Ajtai key over Goldilocks R = F_p[X]/(X^d + 1).

    ``matrix``: kappa x m ring elements, coefficient form, [kappa][m][d]
    uint64 residues.  ``commit(w)`` takes w [B][m][d] as uint64 residues or
    int8 digits and returns [B][kappa][d] residues -- the map
    c_i = sum_j A_ij * w_j of ``AjtaiPublicKey::commit`` (ajtai.rs:118-153)
    instantiated over field.rs, equal to the coefficient-domain commit of
    ``NeoAjtaiKey::commit_naive`` (lattice-folding/src/neo.rs:419-441).
    """

    ENGINE_NTT = _lib.LC_ENGINE_NTT
    ENGINE_TENSOR_I8 = _lib.LC_ENGINE_TENSOR_I8

    def __init__(self, log_d: int, kappa: int, m: int, matrix, tensor_cores: bool = False):
        """``tensor_cores=True`` (d = 64 only) also builds the INT8 tensor-core
        tables and makes that engine the default for int8 witnesses."""
        self.tables = GoldilocksNttTables(log_d)
        self.d, self.kappa, self.m = 1 << log_d, kappa, m
        if _is_torch_cuda(matrix):
            size = matrix.numel()
            mat = matrix
        else:
            mat = np.ascontiguousarray(matrix, dtype=np.uint64)
            size = mat.size
        if size != kappa * m * self.d:
            raise AjtaiError("DimensionMismatch", expected=kappa * m * self.d, got=size)
        self._dev = _DeviceKey(self.tables, kappa, m, mat,
                               _lib.LC_KEY_TENSOR_I8 if tensor_cores else 0)

    @property
    def handle(self):
        return self._dev.handle

    @property
    def engine(self) -> int:
        """Engine for int8 witnesses: ENGINE_NTT or ENGINE_TENSOR_I8."""
        return self._dev.engine

    @engine.setter
    def engine(self, value: int):
        self._dev.engine = value

    @property
    def fused(self) -> bool:
        """Small commitments (at most 4 witnesses, 2048 ring elements, 2^20
        multiply-adds) as one launch; False runs every commit staged."""
        return self._dev.fused

    @fused.setter
    def fused(self, value: bool):
        self._dev.fused = value

    PRODUCTS_INT64 = _lib.LC_PRODUCTS_INT64
    PRODUCTS_TENSOR = _lib.LC_PRODUCTS_TENSOR

    @property
    def slot_products(self) -> int:
        """Per-slot products of the NTT engine: PRODUCTS_TENSOR (byte-limb GEMMs on
        the tensor cores, the default) or PRODUCTS_INT64 (CUDA-core integer MAC)."""
        return self._dev.slot_products

    @slot_products.setter
    def slot_products(self, value: int):
        self._dev.slot_products = value

    def commit(self, w, out=None):
        return self._dev.commit_array(w, out)


__all__ = ["AjtaiError", "AjtaiParams", "AjtaiPublicKey", "AjtaiCommitment", "GoldilocksAjtaiKey",
           "sample_small_secret", "GOLDILOCKS_P", "LatticeCudaError"]
