"""The folding step as one graph launch, and the CRT residue split.

:class:`FoldPipeline` wraps ``lc_fold_pipeline_*``: decomp_b(z, 8)
(lattice-folding/src/neo.rs:253-266) -> commitment of the 8 digit rows
(lattice-commitment/src/ajtai.rs:118-153) -> CRT residues of z
(lattice-ring/src/modulus.rs:65) -> forward NTT (ntt.rs:118-146), on device
buffers the pipeline owns, replayed from a CUDA graph after the warm-up run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .ring import _current_stream, _is_torch_cuda


class _DeviceArray:
    """Zero-copy view of a device buffer for ``torch.as_tensor``."""

    def __init__(self, ptr: int, shape, typestr: str):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _view(ptr: int, shape, typestr: str):
    import torch
    return torch.as_tensor(_DeviceArray(ptr, shape, typestr), device="cuda")


def crt_residues(tables, z):
    """z mod every modulus of the u32 plan ``tables``: ``[num_moduli][count]`` u32."""
    import torch
    on_dev = _is_torch_cuda(z)
    zt = z.contiguous() if on_dev else torch.from_numpy(np.ascontiguousarray(z, dtype=np.uint64).view(np.int64)).cuda()
    out = torch.empty((tables.num_moduli, zt.numel()), dtype=torch.int32, device=zt.device)
    _lib.check(_lib.lib().lc_crt_residues(tables.handle, C.c_void_p(zt.data_ptr()), zt.numel(),
                                          C.c_void_p(out.data_ptr()), _current_stream()), "lc_crt_residues")
    if on_dev:
        return out
    torch.cuda.synchronize()
    return out.cpu().numpy().view(np.uint32)


class FoldPipeline:
    """One folding step: ``run()`` reads :attr:`z` and fills :attr:`digits`,
    :attr:`commits` and :attr:`crt_ntt` (torch views of the pipeline's own
    device buffers)."""

    def __init__(self, key, crt_tables, use_graph: bool = True):
        L = _lib.lib()
        h = C.c_void_p()
        _lib.check(L.lc_fold_pipeline_create(key.handle, crt_tables.handle, int(use_graph), C.byref(h)),
                   "lc_fold_pipeline_create")
        self._h, self._key, self._crt = h, key, crt_tables  # keep the key and plan alive
        z, d, c, t = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        _lib.check(L.lc_fold_pipeline_buffers(h, C.byref(z), C.byref(d), C.byref(c), C.byref(t)),
                   "lc_fold_pipeline_buffers")
        m, kappa, nm = key.m, key.kappa, crt_tables.num_moduli
        self.m = m
        self.z = _view(z.value, (m, 64), "<i8")            # uint64 residues, int64 view
        self.digits = _view(d.value, (8, m, 64), "|u1")
        self.commits = _view(c.value, (8, kappa, 64), "<i8")
        self.crt_ntt = _view(t.value, (nm, m, 64), "<i4")  # uint32 residues, int32 view

    def run(self):
        _lib.check(_lib.lib().lc_fold_pipeline_run(self._h, _current_stream()), "lc_fold_pipeline_run")

    def check(self):
        _lib.check(_lib.lib().lc_fold_pipeline_check(self._h, _current_stream()), "lc_fold_pipeline_check")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib._lib is not None:
            _lib._lib.lc_fold_pipeline_destroy(h)
            self._h = None


__all__ = ["FoldPipeline", "crt_residues"]
