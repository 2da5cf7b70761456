"""GPU parity of the INT8 tensor-core Ajtai commit (Goldilocks, d = 64).

The tensor engine computes the coefficient-domain commitment
(lattice-folding/src/neo.rs:138-158, 419-441) as byte-limb integer GEMMs on
tcgen05; every result must equal the oracle's cached-NTT commit
(lattice-commitment/src/ajtai.rs:118-153) and the NTT engine's, bit for bit.
Cases: the smallest key, ragged k / m / batch (k not a multiple of 4, odd m,
partial 128-witness tiles), K-split boundaries (1024 ring elements per CTA),
the extreme int32 partial sums (all key entries p-1 or 1, all digits -128 or
127, a full 1024-element CTA), and the 16 x 2^16 x 128 workload.
"""
import numpy as np
import pytest

import oracle
from lzx_b200 import GoldilocksAjtaiKey, LatticeCudaError, _lib, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = oracle.GL_P


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def oracle_commit(A, kappa, m, W):
    t = oracle.NttTablesGl(6)
    return oracle.ajtaigl_commit_batch(t, t.forward_batch(A), kappa, m, W)


def tc_key(kappa, m, A):
    key = GoldilocksAjtaiKey(6, kappa, m, A.reshape(kappa, m, 64), tensor_cores=True)
    assert key.engine == GoldilocksAjtaiKey.ENGINE_TENSOR_I8
    return key


def both_engines(key, W):
    """Commit with the tensor engine, then the NTT engine, on the same key."""
    key.engine = GoldilocksAjtaiKey.ENGINE_TENSOR_I8
    tc = key.commit(W)
    key.engine = GoldilocksAjtaiKey.ENGINE_NTT
    ntt = key.commit(W)
    key.engine = GoldilocksAjtaiKey.ENGINE_TENSOR_I8
    return tc, ntt


def test_tc_smallest():
    kappa, m, B = 1, 2, 1
    A = synth.synth_gl(1, 0, kappa * m * 64)
    W = synth.synth_i8(1, 1, B * m * 64).reshape(B, m, 64)
    key = tc_key(kappa, m, A)
    assert np.array_equal(key.commit(W), oracle_commit(A, kappa, m, W))


@pytest.mark.parametrize("kappa,m,batch", [(3, 5, 7), (4, 2, 128), (5, 9, 129), (16, 33, 1), (8, 256, 1),
                                           (2, 1, 300), (13, 64, 256)])
def test_tc_ragged_shapes(kappa, m, batch):
    A = synth.synth_gl(kappa, m, kappa * m * 64)
    W = synth.synth_i8(m, batch, batch * m * 64).reshape(batch, m, 64)
    key = tc_key(kappa, m, A)
    tc, ntt = both_engines(key, W)
    assert np.array_equal(tc, ntt)
    idx = sorted({0, batch // 2, batch - 1})
    assert np.array_equal(tc[idx], oracle_commit(A, kappa, m, W[idx]))
    assert _lib.lib().lc_ajtai_key_check(key.handle, None) == 0


@pytest.mark.parametrize("m", [1023, 1024, 1025, 2048, 2049])
def test_tc_split_boundaries(m):
    kappa, batch = 6, 130
    A = synth.synth_gl(2, m, kappa * m * 64)
    W = synth.synth_i8(3, m, batch * m * 64).reshape(batch, m, 64)
    key = tc_key(kappa, m, A)
    tc, ntt = both_engines(key, W)
    assert np.array_equal(tc, ntt)
    assert np.array_equal(tc[[0, 129]], oracle_commit(A, kappa, m, W[[0, 129]]))


@pytest.mark.parametrize("a_val,w_val", [(P - 1, -128), (P - 1, 127), (1, -128), (0xFFFFFFFF, 127)])
@pytest.mark.parametrize("m", [1024, 1025])
def test_tc_extreme_partial_sums(a_val, w_val, m):
    """Largest per-limb int32 sums a CTA can hold: 1024 ring elements of
    identical extreme digits against limbs of 0xFF (p-1 has bytes 4..7 = 0xFF)."""
    kappa, batch = 4, 128
    A = np.full(kappa * m * 64, a_val, dtype=np.uint64)
    W = np.full((batch, m, 64), w_val, dtype=np.int8)
    key = tc_key(kappa, m, A)
    tc, ntt = both_engines(key, W)
    assert np.array_equal(tc, ntt)
    assert np.array_equal(tc[:2], oracle_commit(A, kappa, m, W[:2]))


def test_tc_device_input_and_repeat_calls():
    """Device int8 witnesses (the product path); two calls in a row give the same result."""
    kappa, m, batch = 16, 4096, 128
    A = synth.synth_gl(4, 0, kappa * m * 64)
    key = tc_key(kappa, m, A)
    W = torch.empty(batch * m * 64, dtype=torch.int8, device="cuda")
    synth.fill_device(W, "i8", 9, 4)
    W = W.view(batch, m, 64)
    out1 = key.commit(W)
    out2 = key.commit(W)
    torch.cuda.synchronize()
    assert torch.equal(out1, out2)
    key.engine = GoldilocksAjtaiKey.ENGINE_NTT
    ref = key.commit(W)
    torch.cuda.synchronize()
    assert torch.equal(out1, ref)
    Wh = W.cpu().numpy()
    got = out1.cpu().numpy().view(np.uint64)
    assert np.array_equal(got[[0, 127]], oracle_commit(A, kappa, m, Wh[[0, 127]]))
    assert _lib.lib().lc_ajtai_key_check(key.handle, None) == 0


def test_tc_engine_selection_errors():
    kappa, m = 2, 4
    A = synth.synth_gl(5, 0, kappa * m * 64)
    plain = GoldilocksAjtaiKey(6, kappa, m, A.reshape(kappa, m, 64))
    assert plain.engine == GoldilocksAjtaiKey.ENGINE_NTT
    with pytest.raises(LatticeCudaError):
        plain.engine = GoldilocksAjtaiKey.ENGINE_TENSOR_I8  # no tables: unsupported
    with pytest.raises(LatticeCudaError):
        plain.engine = 7
    A128 = synth.synth_gl(5, 1, kappa * m * 128)
    with pytest.raises(LatticeCudaError):  # tensor tables exist for d = 64 only
        GoldilocksAjtaiKey(7, kappa, m, A128.reshape(kappa, m, 128), tensor_cores=True)
    key = tc_key(kappa, m, A)
    # misaligned device witness pointer: rejected on the host, nothing launched
    buf = torch.zeros(1 + m * 64, dtype=torch.int8, device="cuda")
    out = torch.empty((1, kappa, 64), dtype=torch.int64, device="cuda")
    st = _lib.lib().lc_ajtai_commit_i8(key.handle, buf.data_ptr() + 1, 1, out.data_ptr(), None)
    assert st == _lib.LC_ERR_INVALID_ARGUMENT
    # residue witnesses still go through the NTT engine on a tensor key
    Wr = synth.synth_gl(6, 0, 3 * m * 64).reshape(3, m, 64)
    t = oracle.NttTablesGl(6)
    want = oracle.ajtaigl_commit_batch(t, t.forward_batch(A), kappa, m, Wr)
    assert np.array_equal(key.commit(Wr), want)


def test_tc_config3_full_batch():
    """kappa=16, 2^16 ring elements, 128 int8 witnesses: the tensor engine
    equals the NTT engine on every commitment and the oracle on four."""
    kappa, m, B = 16, 1 << 16, 128
    A = synth.synth_gl(3, 0, kappa * m * 64)
    key = tc_key(kappa, m, A)
    W = torch.empty(B * m * 64, dtype=torch.int8, device="cuda")
    synth.fill_device(W, "i8", 11, 3)
    W = W.view(B, m, 64)
    tc = key.commit(W)
    key.engine = GoldilocksAjtaiKey.ENGINE_NTT
    ntt = key.commit(W)
    torch.cuda.synchronize()
    assert torch.equal(tc, ntt)
    idx = [0, 1, 64, 127]
    Wh = W[idx].cpu().numpy()
    assert np.array_equal(tc[idx].cpu().numpy().view(np.uint64), oracle_commit(A, kappa, m, Wh))
    assert _lib.lib().lc_ajtai_key_check(key.handle, None) == 0


def test_int8_tensor_rate_measurement():
    """lc_tc_i8_rate: the INT8 tensor roofline denominator, measured with
    tcgen05.mma.kind::i8 of the engines' shape; positive, bounded by a few
    times the dense specification (4.5e15 ops/s), errors on bad arguments."""
    import ctypes as C
    L = _lib.lib()
    rate, ms = C.c_double(0.0), C.c_float(0.0)
    for s8 in (1, 0):
        assert L.lc_tc_i8_rate(4096, s8, C.byref(rate), C.byref(ms)) == 0
        assert ms.value > 0
        assert 1e14 < rate.value < 1e16
    assert L.lc_tc_i8_rate(0, 1, C.byref(rate), None) == _lib.LC_ERR_INVALID_ARGUMENT
    assert L.lc_tc_i8_rate(16, 1, None, None) == _lib.LC_ERR_INVALID_ARGUMENT
