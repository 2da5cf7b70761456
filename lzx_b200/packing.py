"""Coefficient packing on the GPU (lattice-ring/src/packing.rs) and the
commit it feeds (lattice-akita/src/pcs.rs:66-76).

:func:`pack_field_elements` mirrors ``pack_field_elements`` (packing.rs:30-52):
three 22-bit limbs per Goldilocks value in consecutive coefficients, zero
padding, at least one ring element.  :func:`akita_commit` is
``AkitaPcs::commit``: pack, ``pad_to_m`` (ajtai.rs:245-257), commit.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .commitment import AjtaiCommitment, AjtaiError
from .ring import RingElement, _current_stream, _is_torch_cuda


def pack_field_elements(ring, values, elems: int | None = None):
    """[elems][n] residues (CUDA int32 tensor); ``elems`` defaults to
    max(1, ceil(3*len/n)) and may be larger (zero ring elements appended)."""
    import torch
    n = ring.n()
    on_dev = _is_torch_cuda(values)
    v = values.contiguous() if on_dev else torch.from_numpy(
        np.ascontiguousarray(values, dtype=np.uint64).view(np.int64)).cuda()
    need = max(1, -(-3 * v.numel() // n))
    elems = need if elems is None else elems
    out = torch.empty((elems, n), dtype=torch.int32, device=v.device)
    st = _lib.lib().lc_pack_field_elements(C.c_void_p(v.data_ptr()), v.numel(), ring.log_n, elems,
                                           C.c_void_p(out.data_ptr()), _current_stream())
    if st == _lib.LC_ERR_DIMENSION_MISMATCH:
        raise AjtaiError("DimensionMismatch", expected=need, got=elems)
    _lib.check(st, "lc_pack_field_elements")
    return out


def akita_commit(pk, evaluations) -> AjtaiCommitment:
    """``AkitaPcs::commit`` (pcs.rs:66-76) of an MLE's evaluations under the
    Ajtai key ``pk`` (an ``AjtaiPublicKey``): pack, pad to m, commit."""
    import torch
    ring = pk.params.ring
    packed = pack_field_elements(ring, evaluations, pk.params.m)  # DimensionMismatch if > m
    rows = pk.commit_batch(packed.view(1, pk.params.m, ring.n()))
    torch.cuda.synchronize()
    rows = rows[0].cpu().numpy().view(np.uint32)
    return AjtaiCommitment([RingElement(ring, r) for r in rows])


__all__ = ["pack_field_elements", "akita_commit"]
