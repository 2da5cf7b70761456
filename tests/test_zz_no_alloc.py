"""The commit entry point that allocates no device memory.

lc_ajtai_commit_noalloc serves callers that cannot call cudaMalloc while they
commit: processes whose device memory is already owned by another allocator,
latency-critical verifiers that cannot take cudaMalloc's implicit
synchronisation.  Its scratch is a fixed 16 MiB array inside the library.
These tests call it through the C ABI, twice in a row with different
witnesses, and require exactly the residues that the ordinary
lc_ajtai_commit returns for the same key and input (Goldilocks and Q_32
keys, a key view, a key made for the tensor engine); a request larger than
the fixed scratch must be refused without running.

This file is collected last on purpose, so that a run that stops at the first
failure has already run every other test; it also passes alone in a fresh
process.
"""
import ctypes as C

import numpy as np
import pytest

from lzx_b200 import (AjtaiParams, AjtaiPublicKey, GoldilocksAjtaiKey, Modulus32, RingConfig, _lib,
                      synth)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def _dev(a: np.ndarray):
    return torch.from_numpy(a.view(np.int64 if a.dtype == np.uint64 else np.int32)).cuda()


def _both(handle, s_dev, batch, k, n, dtype):
    """(noalloc result, ordinary result) for one witness batch on the device."""
    L = _lib.lib()
    tdt = torch.int64 if dtype == np.uint64 else torch.int32
    out_na = torch.full((batch, k, n), -1, dtype=tdt, device="cuda")
    out_ref = torch.empty((batch, k, n), dtype=tdt, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    st = L.lc_ajtai_commit_noalloc(handle, C.c_void_p(s_dev.data_ptr()), batch,
                                   C.c_void_p(out_na.data_ptr()), stream)
    assert st == 0, _lib.lib().lc_status_string(st)
    st = L.lc_ajtai_commit(handle, C.c_void_p(s_dev.data_ptr()), batch,
                           C.c_void_p(out_ref.data_ptr()), stream)
    assert st == 0
    assert L.lc_ajtai_key_check(handle, stream) == 0
    return out_na.cpu().numpy().view(dtype), out_ref.cpu().numpy().view(dtype)


@pytest.mark.parametrize("kappa,m,batch", [(8, 256, 1), (16, 64, 128), (4, 96, 37)])
def test_goldilocks_noalloc_matches_commit_twice(kappa, m, batch):
    d = 64
    A = synth.synth_gl(90 + batch, 0, kappa * m * d).reshape(kappa, m, d)
    key = GoldilocksAjtaiKey(6, kappa, m, A)
    for call in range(2):  # two calls in a row share the scratch array
        W = synth.synth_gl(91 + call, batch, batch * m * d).reshape(batch, m, d)
        got, want = _both(key.handle, _dev(W), batch, kappa, d, np.uint64)
        assert np.array_equal(got, want), f"call {call}"


def test_q32_noalloc_matches_commit_twice():
    pk = AjtaiPublicKey.from_seed(AjtaiParams(RingConfig(Modulus32.Q_32, 8), 2, 16, 1 << 20),
                                  bytes([5]) * 32)
    for call in range(2):
        s = synth.synth_mod32(70 + call, 1, Modulus32.Q_32.q, 3 * 16 * 256).reshape(3, 16, 256)
        got, want = _both(pk._dev.handle, _dev(s), 3, 2, 256, np.uint32)
        assert np.array_equal(got, want), f"call {call}"


def test_noalloc_on_a_key_view_and_a_tensor_engine_key():
    """A view (its rows of A are a_m = 300 apart while it commits m = 200) and
    a key created for the tensor engine both give lc_ajtai_commit's residues."""
    from lzx_b200.batch import key_view
    d = 64
    A = synth.synth_gl(21, 0, 16 * 300 * d).reshape(16, 300, d)
    parent = GoldilocksAjtaiKey(6, 16, 300, A, tensor_cores=True)
    view = key_view(parent, 8, 200)
    for handle, k, m in ((parent.handle, 16, 300), (view.handle, 8, 200)):
        for call in range(2):
            W = synth.synth_gl(22 + call, m, 3 * m * d).reshape(3, m, d)
            got, want = _both(handle, _dev(W), 3, k, d, np.uint64)
            assert np.array_equal(got, want), (k, m, call)


def test_noalloc_refuses_requests_beyond_its_scratch():
    kappa, m, d, batch = 2, 1 << 12, 64, 128  # witness NTTs alone need 256 MiB
    A = synth.synth_gl(5, 0, kappa * m * d).reshape(kappa, m, d)
    key = GoldilocksAjtaiKey(6, kappa, m, A)
    s = torch.zeros(batch * m * d, dtype=torch.int64, device="cuda")
    out = torch.full((batch, kappa, d), 7, dtype=torch.int64, device="cuda")
    st = _lib.lib().lc_ajtai_commit_noalloc(key.handle, C.c_void_p(s.data_ptr()), batch,
                                            C.c_void_p(out.data_ptr()), None)
    assert st == _lib.LC_ERR_INVALID_ARGUMENT
    torch.cuda.synchronize()
    assert bool((out == 7).all())
