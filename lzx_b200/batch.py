"""Batches of uneven commitment jobs (``lc_batch_*``), key views and u32 keys.

A job is ``AjtaiPublicKey::commit`` (lattice-commitment/src/ajtai.rs:118-153)
of one int8-digit witness under the first ``kappa`` rows and ``n`` columns of
its class's key(s); a class is one Goldilocks key or one u32 key per prime of
a CRT set.  :class:`CommitBatch` runs any mix of ring degrees 64/128/256,
lengths, row counts and moduli in three persistent launches (optionally one
CUDA graph); :func:`key_view` gives the same jobs one by one through the
ordinary commit path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .commitment import _DeviceKey
from .ring import NttTables, _current_stream


class U32AjtaiKey:
    """Cached-NTT key over one u32 modulus (a ``Modulus32``), from its
    coefficient matrix [kappa][m][d] (numpy or CUDA tensor)."""

    def __init__(self, modulus, log_d: int, kappa: int, m: int, matrix):
        self.tables = NttTables(modulus, log_d)
        self.modulus, self.d, self.kappa, self.m = modulus, 1 << log_d, kappa, m
        self._dev = _DeviceKey(self.tables, kappa, m, matrix)

    @property
    def handle(self):
        return self._dev.handle

    def commit(self, w, out=None):
        return self._dev.commit_array(w, out)


class KeyView:
    """``lc_ajtai_key_view``: the first ``kappa`` rows and ``n`` columns of a key."""

    def __init__(self, key, kappa: int, n: int):
        h = C.c_void_p()
        _lib.check(_lib.lib().lc_ajtai_key_view(key.handle, kappa, n, C.byref(h)), "lc_ajtai_key_view")
        self._h, self._parent = h, key
        self.kappa, self.m = kappa, n
        self._dev = key._dev  # element type / degree of the parent

    @property
    def handle(self):
        return self._h

    def commit_i8(self, w, out):
        """Device int8 witness [n][d] -> out (device), same stream semantics as the key."""
        _lib.check(_lib.lib().lc_ajtai_commit_i8(self._h, C.c_void_p(w.data_ptr()), 1, C.c_void_p(out.data_ptr()),
                                                 _current_stream()), "lc_ajtai_commit_i8")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.lc_ajtai_key_destroy(h)
            self._h = None


def key_view(key, kappa: int, n: int) -> KeyView:
    return KeyView(key, kappa, n)


class _Class(C.Structure):
    _fields_ = [("keys", C.c_void_p * 4), ("num_keys", C.c_uint32)]


class _Job(C.Structure):
    _fields_ = [("cls", C.c_uint32), ("kappa", C.c_uint32), ("n", C.c_uint32), ("w", C.c_void_p),
                ("out", C.c_void_p)]


@dataclass
class CommitJob:
    cls: int
    kappa: int
    n: int
    w: object    # CUDA int8 tensor [n][d]
    out: object  # CUDA tensor [num_keys][kappa][d] (int64 for Goldilocks, int32 per prime)


class CommitBatch:
    """``lc_batch_*`` over ``classes`` (lists of keys) and ``jobs``."""

    def __init__(self, classes, jobs, graph: bool = True):
        L = _lib.lib()
        cls_arr = (_Class * max(1, len(classes)))()
        for i, keys in enumerate(classes):
            for k, key in enumerate(keys):
                cls_arr[i].keys[k] = key.handle.value
            cls_arr[i].num_keys = len(keys)
        job_arr = (_Job * max(1, len(jobs)))()
        for i, j in enumerate(jobs):
            job_arr[i] = _Job(j.cls, j.kappa, j.n, j.w.data_ptr(), j.out.data_ptr())
        h = C.c_void_p()
        _lib.check(L.lc_batch_create(cls_arr, len(classes), job_arr, len(jobs), _lib.LC_BATCH_GRAPH if graph else 0,
                                     C.byref(h)), "lc_batch_create")
        self._h = h
        self._keep = (classes, jobs)  # keys and buffers must outlive the batch

    def run(self):
        _lib.check(_lib.lib().lc_batch_run(self._h, _current_stream()), "lc_batch_run")

    def check(self):
        _lib.check(_lib.lib().lc_batch_check(self._h, _current_stream()), "lc_batch_check")

    def set_config(self, chunk: int, ctas_per_sm: int, claim: int):
        _lib.check(_lib.lib().lc_batch_set_config(self._h, chunk, ctas_per_sm, claim), "lc_batch_set_config")

    @property
    def config(self):
        a, b, c = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _lib.check(_lib.lib().lc_batch_get_config(self._h, C.byref(a), C.byref(b), C.byref(c)), "lc_batch_get_config")
        return a.value, b.value, c.value

    PRODUCTS_INT64 = 0   # LC_PRODUCTS_INT64: multiply-accumulates on the CUDA cores
    PRODUCTS_TENSOR = 1  # LC_PRODUCTS_TENSOR: byte-limb GEMMs on the INT8 tensor cores

    @property
    def products(self) -> int:
        """How the per-slot products run (``lc_batch_set_products``); identical results."""
        return _lib.lib().lc_batch_get_products(self._h)

    @products.setter
    def products(self, mode: int):
        _lib.check(_lib.lib().lc_batch_set_products(self._h, mode), "lc_batch_set_products")

    @property
    def info(self):
        a, b, c, d = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32()
        _lib.check(_lib.lib().lc_batch_info(self._h, C.byref(a), C.byref(b), C.byref(c), C.byref(d)),
                   "lc_batch_info")
        return {"items_ntt": a.value, "items_product": b.value, "items_finish": c.value, "lanes": d.value}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.lc_batch_destroy(h)
            self._h = None


__all__ = ["U32AjtaiKey", "KeyView", "key_view", "CommitJob", "CommitBatch"]
