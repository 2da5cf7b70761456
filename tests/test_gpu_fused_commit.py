"""GPU parity of the single-launch commitment (lc_ajtai_key_set_fused).

Small commitments -- at most 4 witnesses, 2048 ring elements, 2^20
multiply-adds -- run as one kernel: witness transforms, products against the
cached NTT(A), their sum over the whole witness through 128-bit accumulators
and the row inverse transforms (the whole body of AjtaiPublicKey::commit,
lattice-commitment/src/ajtai.rs:118-153).  Every case is compared bit for bit
with the oracle and with the staged launches on the same key, over Goldilocks,
Modulus32::Q_32 (canonical Montgomery) and a 30-bit CRT prime (lazy Shoup),
d = 64, 128, 256, with residue, int8 and uint8 witnesses.  Repeated and
interleaved calls check that the accumulators and the ticket are left zero.
"""
import numpy as np
import pytest

import oracle
from lzx_b200 import (CRT_SET_30BIT, AjtaiParams, AjtaiPublicKey, GoldilocksAjtaiKey, Modulus32, RingConfig,
                      _lib, synth)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def gl_case(log_d, kappa, m, seed):
    d = 1 << log_d
    A = synth.synth_gl(seed, 0, kappa * m * d)
    return A, GoldilocksAjtaiKey(log_d, kappa, m, A.reshape(kappa, m, d))


def gl_oracle(A, log_d, kappa, m, W):
    t = oracle.NttTablesGl(log_d)
    return oracle.ajtaigl_commit_batch(t, t.forward_batch(A), kappa, m, W)


def both_forms(key, W):
    """Commit with the single launch and with the staged launches."""
    assert key.fused
    fused = key.commit(W)
    key.fused = False
    staged = key.commit(W)
    key.fused = True
    return fused, staged


@pytest.mark.parametrize("log_d,kappa,m,batch", [
    (6, 8, 256, 1),      # the single d = 64, kappa = 8, n = 256 commitment
    (6, 16, 256, 4),
    (6, 1, 1, 1),
    (6, 3, 7, 3),
    (6, 16, 1024, 1),
    (6, 5, 2048, 1),
    (7, 8, 300, 2),
    (8, 4, 129, 3),
    (8, 16, 64, 4),
])
@pytest.mark.parametrize("digits", ["i8", "u8", "residue"])
def test_goldilocks_fused_matches_staged_and_oracle(log_d, kappa, m, batch, digits):
    d = 1 << log_d
    A, key = gl_case(log_d, kappa, m, seed=kappa * 1000 + m)
    if digits == "residue":
        W = synth.synth_gl(3, batch, batch * m * d).reshape(batch, m, d)
        Wo = W
    else:
        W = synth.synth_i8(3, batch, batch * m * d).reshape(batch, m, d)
        if digits == "u8":
            W = W.view(np.uint8)
        Wo = W if digits == "i8" else W.astype(np.uint64)
    fused, staged = both_forms(key, W)
    want = gl_oracle(A, log_d, kappa, m, Wo)
    assert np.array_equal(fused, want)
    assert np.array_equal(staged, want)


def q32_key(modulus, log_n, k, m, seed):
    pk = AjtaiPublicKey.from_seed(AjtaiParams(RingConfig(modulus, log_n), k, m, 1 << 20), bytes([seed]) * 32)
    t = oracle.NttTables32(oracle.Modulus32(modulus.q, modulus.two_adicity, modulus.generator), log_n)
    return pk, t


@pytest.mark.parametrize("modulus", [Modulus32.Q_32, CRT_SET_30BIT[2]], ids=["q32", "crt30"])
@pytest.mark.parametrize("log_n,k,m,batch", [(6, 2, 64, 1), (6, 16, 500, 2), (7, 3, 33, 4), (8, 8, 100, 1),
                                             (8, 1, 2048, 1)])
def test_u32_fused_matches_staged_and_oracle(modulus, log_n, k, m, batch):
    pk, t = q32_key(modulus, log_n, k, m, seed=log_n + k)
    n = 1 << log_n
    q = modulus.q
    W = synth.synth_mod32(5, m, q, batch * m * n).reshape(batch, m, n)
    fused = pk.commit_batch(W)
    pk.fused = False
    staged = pk.commit_batch(W)
    pk.fused = True
    for b in range(batch):
        want = oracle.ajtai32_commit_naive(t, pk._matrix, k, m, W[b])
        assert np.array_equal(fused[b], want)
        assert np.array_equal(staged[b], want)
    # int8 digits on the same key
    D = synth.synth_i8(6, m, batch * m * n).reshape(batch, m, n)
    got = pk._dev.commit_array(D)
    Dq = np.where(D < 0, q + D.astype(np.int64), D.astype(np.int64)).astype(np.uint32)
    for b in range(batch):
        assert np.array_equal(got[b], oracle.ajtai32_commit_naive(t, pk._matrix, k, m, Dq[b]))


def test_repeated_and_interleaved_calls_leave_no_state():
    """The accumulators and the ticket are zero after every call: back-to-back
    device commits, a staged one in between, batch sizes changing."""
    kappa, m, log_d = 8, 256, 6
    A, key = gl_case(log_d, kappa, m, seed=99)
    ws = [synth.synth_i8(11, s, b * m * 64).reshape(b, m, 64) for s, b in ((0, 1), (1, 4), (2, 2), (3, 1))]
    wants = [gl_oracle(A, log_d, kappa, m, w) for w in ws]
    dev = [torch.from_numpy(w).cuda() for w in ws]
    for _ in range(3):
        outs = [key.commit(x) for x in dev]  # queued back to back on one stream
        torch.cuda.synchronize()
        for o, want in zip(outs, wants):
            assert np.array_equal(o.cpu().numpy().view(np.uint64), want)
        key.fused = False
        assert np.array_equal(key.commit(ws[1]), wants[1])
        key.fused = True
    assert _lib.lib().lc_ajtai_key_check(key.handle, None) == 0


def test_shapes_outside_the_single_launch_still_run_staged():
    """More than 4 witnesses or more than 2048 ring elements: the staged path."""
    kappa, log_d = 4, 6
    for m, batch in ((2049, 1), (64, 5)):
        A, key = gl_case(log_d, kappa, m, seed=m + batch)
        W = synth.synth_i8(12, m, batch * m * 64).reshape(batch, m, 64)
        assert np.array_equal(key.commit(W), gl_oracle(A, log_d, kappa, m, W))


def test_fused_switch_arguments():
    _, key = gl_case(6, 2, 8, seed=1)
    L = _lib.lib()
    assert L.lc_ajtai_key_get_fused(key.handle) == 1
    assert L.lc_ajtai_key_set_fused(key.handle, 3) == _lib.LC_ERR_INVALID_ARGUMENT
    assert L.lc_ajtai_key_set_fused(None, 0) == _lib.LC_ERR_INVALID_ARGUMENT
    assert L.lc_ajtai_key_get_fused(None) == -1
    assert L.lc_ajtai_key_set_fused(key.handle, 0) == 0
    assert L.lc_ajtai_key_get_fused(key.handle) == 0


@pytest.mark.parametrize("kind", ["i8", "u8", "residues"])
def test_host_call_reads_and_writes_host_memory(kind):
    """A synchronous host call of a small commitment runs the single-launch
    kernel straight on page-locked host memory (the key's staging buffers for
    pageable arguments, or the caller's pinned buffers), with no copies
    queued; pageable, pinned and misaligned pinned outputs all give the
    device call's residues, on repeated calls."""
    import ctypes as C
    kappa, m, log_d = 8, 256, 6
    A, key = gl_case(log_d, kappa, m, 71)
    L = _lib.lib()
    if kind == "residues":
        W = synth.synth_gl(72, 1, 2 * m * 64).reshape(2, m, 64)
        fn, dev_fn = L.lc_ajtai_commit_host, L.lc_ajtai_commit
        wt = torch.from_numpy(W.view(np.int64))
    else:
        W = synth.synth_i8(72, 1, 2 * m * 64).reshape(2, m, 64)
        if kind == "u8":
            W = W.view(np.uint8)
        fn = L.lc_ajtai_commit_i8_host if kind == "i8" else L.lc_ajtai_commit_u8_host
        dev_fn = L.lc_ajtai_commit_i8 if kind == "i8" else L.lc_ajtai_commit_u8
        wt = torch.from_numpy(W.view(np.int8))
    wd = wt.cuda()
    want = torch.empty((2, kappa, 64), dtype=torch.int64, device="cuda")
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert dev_fn(key.handle, C.c_void_p(wd.data_ptr()), 2, C.c_void_p(want.data_ptr()), st) == 0
    torch.cuda.synchronize()
    want = want.cpu().numpy().view(np.uint64)
    assert np.array_equal(want, gl_oracle(A, log_d, kappa, m, W))
    wp = wt.clone().pin_memory()
    pinned_out = torch.zeros((2, kappa, 64), dtype=torch.int64).pin_memory()
    big = torch.zeros(2 * kappa * 64 + 1, dtype=torch.int64).pin_memory()
    for _ in range(2):
        got = np.zeros((2, kappa, 64), dtype=np.uint64)  # pageable in and out: staged
        assert fn(key.handle, W.ctypes.data_as(C.c_void_p), 2, got.ctypes.data_as(C.c_void_p)) == 0
        assert np.array_equal(got, want)
        # the caller's pinned buffers
        assert fn(key.handle, C.c_void_p(wp.data_ptr()), 2, C.c_void_p(pinned_out.data_ptr())) == 0
        assert np.array_equal(pinned_out.numpy().view(np.uint64), want)
        # a pinned output 8 bytes into its allocation (not 16-byte aligned)
        assert fn(key.handle, C.c_void_p(wp.data_ptr()), 2, C.c_void_p(big.data_ptr() + 8)) == 0
        assert np.array_equal(big[1:].numpy().view(np.uint64).reshape(want.shape), want)
    assert L.lc_ajtai_key_check(key.handle, None) == 0
