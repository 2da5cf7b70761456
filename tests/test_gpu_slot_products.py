"""GPU parity of the NTT engine's per-slot products on the tensor cores.

Goldilocks keys form C_t = A_t^T W_t of every NTT slot either as byte-limb
GEMMs on the INT8 tensor cores (lc_ajtai_key_set_slot_products(...,
LC_PRODUCTS_TENSOR), the default) or with 160-bit integer multiply-adds on the
CUDA cores (LC_PRODUCTS_INT64).  Both must give the oracle's commitment
(AjtaiPublicKey::commit, lattice-commitment/src/ajtai.rs:118-153, over
lattice-core/src/field.rs, and over Modulus32::Q_32 and a 30-bit CRT prime)
bit for bit: every N-tile width (witness rows of 32, 64, 128, 256 bytes and
several tiles of 512), several K-splits of 32768 ring elements, odd
ring-element counts, d = 64/128/256, int8, uint8 and residue witnesses, and a
key view whose row stride differs from its width.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from lzx_b200 import (CRT_SET_30BIT, AjtaiParams, AjtaiPublicKey, GoldilocksAjtaiKey, Modulus32, RingConfig,
                      _lib, synth)
from lzx_b200.batch import key_view

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def make_key(log_d, kappa, m, seed):
    d = 1 << log_d
    A = synth.synth_gl(seed, 0, kappa * m * d)
    return A, GoldilocksAjtaiKey(log_d, kappa, m, A.reshape(kappa, m, d))


def oracle_commit(A, log_d, kappa, m, W):
    t = oracle.NttTablesGl(log_d)
    return oracle.ajtaigl_commit_batch(t, t.forward_batch(A), kappa, m, W)


def both_products(key, W):
    assert key.slot_products == GoldilocksAjtaiKey.PRODUCTS_TENSOR
    tensor = key.commit(W)
    key.slot_products = GoldilocksAjtaiKey.PRODUCTS_INT64
    integer = key.commit(W)
    key.slot_products = GoldilocksAjtaiKey.PRODUCTS_TENSOR
    return tensor, integer


@pytest.mark.parametrize("log_d,kappa,m,batch", [
    (6, 16, 300, 8),        # N tile 64 bytes (64-byte swizzle)
    (6, 5, 1001, 16),       # 128
    (6, 3, 777, 32),        # 256
    (6, 16, 513, 64),       # 512
    (6, 7, 257, 200),       # batch padded to 256: two tiles of 512
    (6, 3, 7, 8),           # fewer ring elements than one 64-row stage
    (6, 2, 1, 64),          # a single ring element
    (7, 8, 300, 16),
    (8, 2, 129, 64),
    (6, 4, 3000, 4),        # N tile 32 bytes: too long for the single launch
])
@pytest.mark.parametrize("digits", ["i8", "u8", "residue"])
def test_tensor_products_match_integer_and_oracle(log_d, kappa, m, batch, digits):
    d = 1 << log_d
    A, key = make_key(log_d, kappa, m, seed=kappa * 7 + m)
    if digits == "residue":
        W = synth.synth_gl(5, batch, batch * m * d).reshape(batch, m, d)
        Wo = W
    else:
        W = synth.synth_i8(5, batch, batch * m * d).reshape(batch, m, d)
        if digits == "u8":
            W = W.view(np.uint8)
        Wo = W if digits == "i8" else W.astype(np.uint64)
    tensor, integer = both_products(key, W)
    assert np.array_equal(tensor, integer)
    idx = sorted({0, batch // 2, batch - 1})
    assert np.array_equal(tensor[idx], oracle_commit(A, log_d, kappa, m, Wo[idx]))


@pytest.mark.parametrize("m,batch", [(40_000, 8), (70_001, 64)])
def test_several_k_splits(m, batch):
    """More than 32768 ring elements: the int32 sums are split and recombined."""
    kappa, log_d = 16, 6
    A = torch.empty(kappa * m * 64, dtype=torch.int64, device="cuda")
    synth.fill_device(A, "gl", 91, m)
    key = GoldilocksAjtaiKey(log_d, kappa, m, A)
    W = torch.empty(batch * m * 64, dtype=torch.int8, device="cuda")
    synth.fill_device(W, "i8", 92, m)
    tensor, integer = both_products(key, W)
    assert torch.equal(tensor, integer)
    # one witness against the oracle
    Ah = A.cpu().numpy().view(np.uint64)
    Wh = W.cpu().numpy().reshape(batch, m, 64)
    got = tensor.cpu().numpy().view(np.uint64)
    assert np.array_equal(got[[batch - 1]], oracle_commit(Ah, log_d, kappa, m, Wh[[batch - 1]]))


def test_key_view_row_stride():
    """A view (first kappa rows, first n ring elements) reads the parent's NTT(A)
    with the parent's row stride."""
    kappa, m, log_d = 8, 600, 6
    A, key = make_key(log_d, kappa, m, seed=5)
    kv, nv, batch = 5, 333, 8
    view = key_view(key, kv, nv)
    W = synth.synth_i8(13, 1, batch * nv * 64).reshape(batch, nv, 64)
    w = torch.from_numpy(W).cuda()
    out = torch.empty((batch, kv, 64), dtype=torch.int64, device="cuda")
    L = _lib.lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.lc_ajtai_key_get_slot_products(view.handle) == _lib.LC_PRODUCTS_TENSOR
    assert L.lc_ajtai_commit_i8(view.handle, C.c_void_p(w.data_ptr()), batch, C.c_void_p(out.data_ptr()), st) == 0
    torch.cuda.synchronize()
    Av = A.reshape(kappa, m, 64)[:kv, :nv].reshape(-1)
    assert np.array_equal(out.cpu().numpy().view(np.uint64), oracle_commit(Av, log_d, kv, nv, W))


@pytest.mark.parametrize("modulus", [Modulus32.Q_32, CRT_SET_30BIT[1]], ids=["q32", "crt30"])
@pytest.mark.parametrize("log_n,k,m,batch", [
    (6, 2, 300, 8),      # u32 rows: 32-byte N tile
    (6, 5, 700, 16),     # 64
    (7, 16, 129, 32),    # 128
    (6, 3, 1000, 64),    # 256
    (8, 2, 257, 128),    # 512
    (6, 7, 300, 200),    # padded to 256: two tiles of 512
])
def test_u32_tensor_products_match_integer_and_oracle(modulus, log_n, k, m, batch):
    """u32 keys: 4 byte limbs, the key's 64-byte rows fill half of M = 128."""
    pk = AjtaiPublicKey.from_seed(AjtaiParams(RingConfig(modulus, log_n), k, m, 1 << 20), bytes([log_n + k]) * 32)
    n, q = 1 << log_n, modulus.q
    W = synth.synth_mod32(7, m + batch, q, batch * m * n).reshape(batch, m, n)
    assert pk.slot_products == GoldilocksAjtaiKey.PRODUCTS_TENSOR
    tensor = pk.commit_batch(W)
    pk.slot_products = GoldilocksAjtaiKey.PRODUCTS_INT64
    integer = pk.commit_batch(W)
    pk.slot_products = GoldilocksAjtaiKey.PRODUCTS_TENSOR
    assert np.array_equal(tensor, integer)
    t = oracle.NttTables32(oracle.Modulus32(modulus.q, modulus.two_adicity, modulus.generator), log_n)
    for b in sorted({0, batch - 1}):
        assert np.array_equal(tensor[b], oracle.ajtai32_commit_naive(t, pk._matrix, k, m, W[b]))


def test_switch_arguments():
    _, key = make_key(6, 2, 8, seed=2)
    L = _lib.lib()
    assert L.lc_ajtai_key_set_slot_products(key.handle, 2) == _lib.LC_ERR_INVALID_ARGUMENT
    assert L.lc_ajtai_key_set_slot_products(None, 0) == _lib.LC_ERR_INVALID_ARGUMENT
    assert L.lc_ajtai_key_get_slot_products(None) == -1
