"""GPU parity of the plain form's products, split sums and inverse NTT in one
launch.

With the per-slot products on the CUDA cores (LC_PRODUCTS_INT64), a commit
after the witness transforms can run as one cooperative kernel: the K-split
products of the shape's form (tiled 128-witness tiles, 4-witness quads, or
one output per thread), a grid barrier, the sum over the splits by every
thread, a second barrier, then the inverse transforms of 32 rows per item
(AjtaiPublicKey::commit, lattice-commitment/src/ajtai.rs:139-150) --
by default for batches of at most 3 witnesses, for every shape with
lc_ajtai_key_set_fused(key, 2).  Its residues must equal the default and the
staged launches (lc_ajtai_key_set_fused(key, 0)) and the oracle bit for bit:
Goldilocks, Q_32 and a 30-bit CRT prime, d = 64/128/256, every form, padded
batches, a key view, repeated calls, and the folding step replayed from a
CUDA graph.
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
INT64 = GoldilocksAjtaiKey.PRODUCTS_INT64


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def one_launch_and_staged(key, commit):
    key.slot_products = INT64
    assert key.fused == 1  # the default: one launch only where it is faster
    default = commit()
    key.fused = 2          # the one-launch products + inverse NTT for every shape
    fused = commit()
    again = commit()  # a second call: the barrier counter and scratch are reused
    key.fused = 0
    staged = commit()
    key.fused = 1
    assert np.array_equal(default, staged)
    return fused, again, staged


# ring elements above 2048 keep small batches off the single-launch commit
@pytest.mark.parametrize("log_d,kappa,m,batch", [
    (6, 16, 3000, 128),   # tiled
    (6, 5, 2100, 130),    # tiled, padded to two 128-witness tiles
    (7, 8, 2500, 64),     # tiled, 64 witnesses padded to 128
    (8, 3, 2049, 128),    # tiled, d = 256
    (6, 16, 3000, 8),     # quads
    (6, 7, 2500, 12),     # quads, phase-2 items of 12 witnesses
    (8, 4, 2100, 40),     # quads, d = 256
    (6, 3, 5000, 1),      # one output per thread
    (7, 9, 3000, 3),
])
def test_goldilocks_one_launch_equals_staged_and_oracle(log_d, kappa, m, batch):
    d = 1 << log_d
    A = synth.synth_gl(m + batch, 0, kappa * m * d)
    key = GoldilocksAjtaiKey(log_d, kappa, m, A.reshape(kappa, m, d))
    W = synth.synth_i8(3, batch, batch * m * d).reshape(batch, m, d)
    fused, again, staged = one_launch_and_staged(key, lambda: key.commit(W))
    assert np.array_equal(fused, staged) and np.array_equal(again, staged)
    t = oracle.NttTablesGl(log_d)
    idx = sorted({0, batch // 2, batch - 1})
    want = oracle.ajtaigl_commit_batch(t, t.forward_batch(A), kappa, m, W[idx])
    assert np.array_equal(fused[idx], want)
    assert _lib.lib().lc_ajtai_key_check(key.handle, None) == 0


@pytest.mark.parametrize("modulus", [Modulus32.Q_32, CRT_SET_30BIT[2]], ids=["q32", "crt30"])
@pytest.mark.parametrize("log_n,k,m,batch", [(6, 2, 2100, 128), (8, 5, 2049, 16), (7, 3, 3000, 2)])
def test_u32_one_launch_equals_staged_and_oracle(modulus, log_n, k, m, batch):
    pk = AjtaiPublicKey.from_seed(AjtaiParams(RingConfig(modulus, log_n), k, m, 1 << 20), bytes([k + 1]) * 32)
    n = 1 << log_n
    W = synth.synth_mod32(11, batch, modulus.q, batch * m * n).reshape(batch, m, n)
    fused, again, staged = one_launch_and_staged(pk, lambda: pk.commit_batch(W))
    assert np.array_equal(fused, staged) and np.array_equal(again, staged)
    t = oracle.NttTables32(oracle.Modulus32(modulus.q, modulus.two_adicity, modulus.generator), log_n)
    for b in sorted({0, batch - 1}):
        assert np.array_equal(fused[b], oracle.ajtai32_commit_naive(t, pk._matrix, k, m, W[b]))


def test_key_view_tiled_products_match_oracle():
    """128 witnesses on a view (rows a_m = 3000 apart, m = 2333 committed):
    the tiled integer products, then the split sums and inverse transforms
    in one launch, equal the oracle's commitment under the view's sub-matrix."""
    kappa, m, log_d = 8, 3000, 6
    A = synth.synth_gl(6, 0, kappa * m * 64).reshape(kappa, m, 64)
    key = GoldilocksAjtaiKey(log_d, kappa, m, A)
    kv, nv, batch = 5, 2333, 128
    view = key_view(key, kv, nv)
    L = _lib.lib()
    assert L.lc_ajtai_key_set_slot_products(view.handle, INT64) == 0
    W = synth.synth_i8(14, 1, batch * nv * 64).reshape(batch, nv, 64)
    w = torch.from_numpy(W).cuda()
    out = torch.empty((batch, kv, 64), dtype=torch.int64, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.lc_ajtai_commit_i8(view.handle, C.c_void_p(w.data_ptr()), batch, C.c_void_p(out.data_ptr()), st) == 0
    assert L.lc_ajtai_key_check(view.handle, st) == 0
    t = oracle.NttTablesGl(log_d)
    sub = np.ascontiguousarray(A[:kv, :nv]).reshape(-1, 64)
    want = oracle.ajtaigl_commit_batch(t, t.forward_batch(sub), kv, nv, W)
    assert np.array_equal(out.cpu().numpy().view(np.uint64).reshape(want.shape), want)


def test_key_view_one_launch():
    """A view's row stride differs from its width; the one-launch form reads it."""
    kappa, m, log_d = 8, 3000, 6
    A = synth.synth_gl(5, 0, kappa * m * 64)
    key = GoldilocksAjtaiKey(log_d, kappa, m, A.reshape(kappa, m, 64))
    kv, nv, batch = 5, 2333, 20
    view = key_view(key, kv, nv)
    L = _lib.lib()
    assert L.lc_ajtai_key_set_slot_products(view.handle, INT64) == 0
    W = synth.synth_i8(13, 1, batch * nv * 64).reshape(batch, nv, 64)
    w = torch.from_numpy(W).cuda()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    outs = []
    for fused in (2, 0):
        assert L.lc_ajtai_key_set_fused(view.handle, fused) == 0
        out = torch.empty((batch, kv, 64), dtype=torch.int64, device="cuda")
        assert L.lc_ajtai_commit_i8(view.handle, C.c_void_p(w.data_ptr()), batch, C.c_void_p(out.data_ptr()),
                                    st) == 0
        outs.append(out.cpu().numpy().view(np.uint64))
    assert np.array_equal(outs[0], outs[1])
    t = oracle.NttTablesGl(log_d)
    Av = A.reshape(kappa, m, 64)[:kv, :nv].reshape(-1)
    assert np.array_equal(outs[0][[0, batch - 1]],
                          oracle.ajtaigl_commit_batch(t, t.forward_batch(Av), kv, nv, W[[0, batch - 1]]))
