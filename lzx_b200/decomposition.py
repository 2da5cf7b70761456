"""Digit decompositions on the GPU, with the reference's names.

* :func:`decomp_b` -- ``decomp_b`` (lattice-folding/src/neo.rs:253-266):
  unsigned base-2^b digits of Goldilocks residues, ``ceil(64/b)`` rows, row r
  = digit r of every element (``[rows][count]`` uint8, b <= 8).
* :class:`GadgetDecomposition` -- ``GadgetDecomposition``
  (lattice-core/src/decomposition.rs:26-110): balanced digits in base 2^k;
  :meth:`GadgetDecomposition.decompose_batch` runs ``decompose`` (:48-70) on
  every value of a vector at once.

Inputs are numpy arrays (copied through the device) or CUDA tensors (no
copy; the result stays on the device).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .ring import _current_stream, _is_torch_cuda


def decomp_b(z, b_bits: int):
    """Rows of unsigned base-2^b_bits digits of the residues ``z``."""
    if not 1 <= b_bits <= 8:
        raise ValueError("b_bits must be in 1..8 (digits are bytes)")
    rows = -(-64 // b_bits)
    L = _lib.lib()
    if _is_torch_cuda(z):
        import torch
        z = z.contiguous()
        out = torch.empty((rows, z.numel()), dtype=torch.uint8, device=z.device)
        _lib.check(L.lc_decomp_b(C.c_void_p(z.data_ptr()), z.numel(), b_bits, C.c_void_p(out.data_ptr()),
                                 _current_stream()), "lc_decomp_b")
        return out
    import torch
    zt = torch.from_numpy(np.ascontiguousarray(z, dtype=np.uint64).view(np.int64)).cuda()
    out = decomp_b(zt, b_bits)
    torch.cuda.synchronize()
    return out.cpu().numpy()


class GadgetDecomposition:
    """``GadgetDecomposition`` (decomposition.rs:26-110) for power-of-two bases."""

    def __init__(self, base: int, num_digits: int):
        if base < 2 or base & (base - 1) or base > 1 << 15:
            raise ValueError("the GPU decomposition takes power-of-two bases up to 2^15")
        self.base, self.num_digits = base, num_digits
        self.log_base = base.bit_length() - 1

    @classmethod
    def power_of_two(cls, bits: int, log_base: int) -> "GadgetDecomposition":
        """``power_of_two`` (:38-43): ceil((bits+1)/log_base) balanced digits."""
        return cls(1 << log_base, -(-(bits + 1) // log_base))

    def decompose_batch(self, z):
        """Digits ``[num_digits][count]`` (int16) of every value and the number
        of values the reference would reject with ``ValueTooLarge``."""
        import torch
        L = _lib.lib()
        on_dev = _is_torch_cuda(z)
        zt = z.contiguous() if on_dev else torch.from_numpy(
            np.ascontiguousarray(z, dtype=np.uint64).view(np.int64)).cuda()
        out = torch.empty((self.num_digits, zt.numel()), dtype=torch.int16, device=zt.device)
        bad = torch.zeros(1, dtype=torch.int32, device=zt.device)
        _lib.check(L.lc_gadget_decompose(C.c_void_p(zt.data_ptr()), zt.numel(), self.log_base, self.num_digits,
                                         C.c_void_p(out.data_ptr()), C.c_void_p(bad.data_ptr()),
                                         _current_stream()), "lc_gadget_decompose")
        if on_dev:
            return out, bad
        torch.cuda.synchronize()
        return out.cpu().numpy(), int(bad.item())


__all__ = ["decomp_b", "GadgetDecomposition"]
