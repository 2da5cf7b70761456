"""lzx_b200 -- B200-native (sm_100a) commitment hot path of LZX.

The negacyclic NTT/INTT over Z_q[X]/(X^n+1) (u32 primes, CRT sets of 30-bit
primes, Goldilocks) and the Ajtai commitment c = A.w, as hand-written CUDA
behind the C ABI in ``include/lattice_cuda.h``.  This package holds the
kernels (``csrc/``), their build, the ctypes binding and a host-side mirror of
the reference's ring/commitment API.
"""
from ._lib import LatticeCudaError, lib  # noqa: F401
from .commitment import (AjtaiCommitment, AjtaiError, AjtaiParams, AjtaiPublicKey,  # noqa: F401
                         GoldilocksAjtaiKey, sample_small_secret)
from .decomposition import GadgetDecomposition, decomp_b  # noqa: F401
from .ring import (CRT_SET_30BIT, GoldilocksNttTables, Modulus32, NttError, NttTables,  # noqa: F401
                   RingConfig, RingElement, RingError)

__version__ = "0.1.0"


def device_available() -> bool:
    return bool(lib().lc_device_available())
