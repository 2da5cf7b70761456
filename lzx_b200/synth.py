"""Seeded synthetic inputs: a counter-based, prefix-consistent generator.

``x = H(seed, stream, index)`` with a SplitMix64 finaliser, so any slice of a
tensor can be regenerated independently (the property large-batch configs
need).  Uniform residues use rejection on a retry lane (``stream + r << 40``):
``cand < 2^32 - 2^32 mod q`` for u32 primes (the rule of
lattice-ring/src/ring.rs:123) and ``cand < p`` for Goldilocks (the rule of
lattice-core/src/transcript.rs:141-144).  int8 digits are the low byte of H
read as signed.  Vectorised numpy; bit-identical to the C generator used by
the test oracle (pinned by tests/golden).
"""
from __future__ import annotations

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
_G = np.uint64(0x9E3779B97F4A7C15)
_C2 = np.uint64(0xC2B2AE3D27D4EB4F)
_C3 = np.uint64(0x165667B19E3779F9)
P_GL = 0xFFFFFFFF00000001


def _mix64(z: np.ndarray) -> np.ndarray:
    z = z ^ (z >> np.uint64(30))
    z = z * np.uint64(0xBF58476D1CE4E5B9)
    z = z ^ (z >> np.uint64(27))
    z = z * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _base(seed: int, stream: int) -> np.uint64:
    with np.errstate(over="ignore"):
        b = np.array([seed], dtype=np.uint64) * _G + np.array([stream & 0xFFFFFFFFFFFFFFFF],
                                                              dtype=np.uint64) * _C2 + _C3
        return _mix64(b)[0]


def synth_u64(seed: int, stream: int, count: int, offset: int = 0) -> np.ndarray:
    with np.errstate(over="ignore"):
        idx = np.arange(offset, offset + count, dtype=np.uint64)
        return _mix64(_base(seed, stream) + idx * _G)


def _rejection(seed, stream, count, offset, accept, chunk=1 << 22):
    out = np.empty(count, dtype=np.uint64)
    for s in range(0, count, chunk):
        c = min(chunk, count - s)
        vals = synth_u64(seed, stream, c, offset + s)
        ok = accept(vals)
        r = 0
        while not ok.all():
            r += 1
            bad = np.nonzero(~ok)[0]
            with np.errstate(over="ignore"):
                idx = (np.uint64(offset + s) + bad.astype(np.uint64))
                nv = _mix64(_base(seed, (stream + (r << 40)) & 0xFFFFFFFFFFFFFFFF) + idx * _G)
            vals[bad] = nv
            ok[bad] = accept(nv)
        out[s:s + c] = vals
    return out


def synth_mod32(seed: int, stream: int, q: int, count: int, offset: int = 0) -> np.ndarray:
    """Uniform residues mod a u32 prime q."""
    limit = np.uint64((1 << 32) - ((1 << 32) % q))
    mask = np.uint64(0xFFFFFFFF)
    v = _rejection(seed, stream, count, offset, lambda x: (x & mask) < limit)
    return ((v & mask) % np.uint64(q)).astype(np.uint32)


def synth_gl(seed: int, stream: int, count: int, offset: int = 0) -> np.ndarray:
    """Uniform Goldilocks residues."""
    p = np.uint64(P_GL)
    return _rejection(seed, stream, count, offset, lambda x: x < p)


def synth_i8(seed: int, stream: int, count: int, offset: int = 0) -> np.ndarray:
    """int8 digits uniform in [-128, 127]."""
    return (synth_u64(seed, stream, count, offset) & np.uint64(0xFF)).astype(np.uint8).view(np.int8)


def crt_batch(seed: int, moduli, count: int, n: int) -> np.ndarray:
    """[len(moduli)][count][n] residues, modulus i drawn from stream i."""
    out = np.empty((len(moduli), count, n), dtype=np.uint32)
    for i, m in enumerate(moduli):
        q = m.q if hasattr(m, "q") else int(m)
        out[i] = synth_mod32(seed, i, q, count * n).reshape(count, n)
    return out


# ----------------------------------------------------------------- on the device

_KIND = {"u64": 0, "mod32": 1, "gl": 2, "i8": 3}


def fill_device(tensor, kind: str, seed: int, stream: int, q: int = 0, offset: int = 0):
    """Fill a contiguous CUDA tensor with the same stream on the GPU
    (``lc_synth_fill``); int32/int64/int8 tensors hold u32/u64/int8 values."""
    import ctypes as C

    import torch

    from . import _lib
    assert tensor.is_cuda and tensor.is_contiguous()
    st = _lib.lib().lc_synth_fill(_KIND[kind], seed & 0xFFFFFFFFFFFFFFFF, stream & 0xFFFFFFFFFFFFFFFF,
                                  q, C.c_void_p(tensor.data_ptr()), tensor.numel(), offset,
                                  C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(st, "lc_synth_fill")
    return tensor
