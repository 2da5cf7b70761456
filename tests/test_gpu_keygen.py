"""GPU parity of the seeded key derivation.

RingConfig::uniform_from_seed (lattice-ring/src/ring.rs:102-180) on the
device against the golden vectors and the oracle -- every modulus family,
every ring degree, domains long enough to need several SHAKE blocks, the
three padding edges of the absorbed message, indices near 2^64 -- and
AjtaiPublicKey::from_seed (lattice-commitment/src/ajtai.rs:87-103) on the
device against the oracle's expansion: same matrix, same commitments.  A
single-element uniform_from_seed runs on the device too.
"""
import numpy as np
import pytest

import oracle
from lzx_b200 import (AjtaiParams, AjtaiPublicKey, CRT_SET_30BIT, GoldilocksNttTables, LatticeCudaError,
                      Modulus32, RingConfig, _lib, sample_small_secret)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def omod(m):
    return oracle.Modulus32(m.q, m.two_adicity, m.generator)


def test_golden_uniform_from_seed(golden):
    for v in golden["uniform_from_seed_q32"]:
        ring = RingConfig(Modulus32.Q_32, v["log_n"])
        got = ring.uniform_from_seed_batch(b"ajtai-A", bytes.fromhex(v["seed_hex"]), v["index"], 1)
        assert got.cpu().numpy().view(np.uint32)[0].tolist() == v["coeffs"]


MODULI = [Modulus32.Q_32, Modulus32.Q_12289, Modulus32.Q_2013265921, CRT_SET_30BIT[0], CRT_SET_30BIT[3]]


@pytest.mark.parametrize("mod", MODULI, ids=lambda m: str(m.q))
@pytest.mark.parametrize("log_n", [1, 4, 6, 8, 10])
def test_uniform_matches_oracle(mod, log_n):
    if log_n + 1 > mod.two_adicity:
        pytest.skip("ring degree needs a larger 2-adicity")
    ring = RingConfig(mod, log_n)
    seed = bytes(range(32))
    got = ring.uniform_from_seed_batch(b"ajtai-A", seed, 1000, 37).cpu().numpy().view(np.uint32)
    for k in (0, 1, 17, 36):
        want = oracle.uniform_from_seed(omod(mod), log_n, b"ajtai-A", seed, 1000 + k)
        assert np.array_equal(got[k], want)


@pytest.mark.parametrize("extra", [0, 1, 2, 109, 110, 111, 245, 246, 247, 300, 489])
def test_uniform_message_lengths_and_blocks(extra):
    """Absorbed message = 27 + |domain| + |seed| bytes: lengths around the
    136-byte rate (padding byte last in a block, alone in a new block) and
    messages of up to 4 blocks."""
    ring = RingConfig(Modulus32.Q_32, 6)
    domain = bytes((7 * i + 3) & 0xFF for i in range(extra))
    seed = b"\x5a" * 27
    idx0 = (1 << 64) - 5  # le64 index bytes near the top, wrapping is not asked for
    got = ring.uniform_from_seed_batch(domain, seed, idx0, 4).cpu().numpy().view(np.uint32)
    for k in range(4):
        want = oracle.uniform_from_seed(omod(Modulus32.Q_32), 6, domain, seed, idx0 + k)
        assert np.array_equal(got[k], want), k


def test_uniform_rejects_oversize_and_goldilocks():
    ring = RingConfig(Modulus32.Q_32, 6)
    with pytest.raises(Exception):
        ring.uniform_from_seed_batch(bytes(500), bytes(32), 0, 1)  # 27 + 532 bytes > 4 blocks
    gl = GoldilocksNttTables(6)
    out = torch.empty((1, 64), dtype=torch.int32, device="cuda")
    st = _lib.lib().lc_uniform_from_seed(gl.handle, b"d", 1, b"s", 1, 0, 1, out.data_ptr(), None)
    assert st == _lib.LC_ERR_UNSUPPORTED


def oracle_key(params, seed):
    """The oracle's AjtaiPublicKey::from_seed (ajtai.rs:87-103) as a key over its matrix."""
    t = oracle.NttTables32(omod(params.ring.modulus), params.ring.log_n)
    mat, _ = oracle.ajtai32_from_seed(t, params.k, params.m, seed)
    return AjtaiPublicKey(params, seed, mat.reshape(params.k * params.m, params.ring.n()))


@pytest.mark.parametrize("log_n,k,m", [(6, 2, 64), (8, 2, 300), (4, 3, 17)])
def test_key_from_seed_matches_oracle_expansion(log_n, k, m):
    params = AjtaiParams(RingConfig(Modulus32.Q_32, log_n), k, m, 1 << 20)
    seed = bytes([0xAB]) * 32
    dev = AjtaiPublicKey.from_seed(params, seed)
    want = oracle_key(params, seed)
    assert np.array_equal(dev._matrix, want._matrix)
    s = sample_small_secret(params.ring, m, 1 << 12, b"kg")
    assert dev.commit(s) == want.commit(s)


def test_single_element_uniform_from_seed_runs_on_device():
    ring = RingConfig(Modulus32.Q_32, 6)
    seed = bytes([0x5A]) * 32
    for idx in (0, 1, 12345):
        got = ring.uniform_from_seed(b"ajtai-A", seed, idx).coeffs()
        assert np.array_equal(got, oracle.uniform_from_seed(omod(Modulus32.Q_32), 6, b"ajtai-A", seed, idx))


def test_c_abi_key_from_seed():
    """lc_ajtai_key_from_seed builds the same key as a key created from the
    oracle-expanded matrix."""
    import ctypes as C
    params = AjtaiParams(RingConfig(Modulus32.Q_32, 6), 2, 40, 1 << 20)
    seed = bytes(range(100, 132))
    host = oracle_key(params, seed)
    h = C.c_void_p()
    L = _lib.lib()
    _lib.check(L.lc_ajtai_key_from_seed(params.ring.tables.handle, 2, 40, seed, C.byref(h)), "from_seed")
    try:
        w = np.stack([e.coeffs() for e in sample_small_secret(params.ring, 40, 255, b"abi")])
        out = np.empty((2, 64), dtype=np.uint32)
        _lib.check(L.lc_ajtai_commit_host(h, w.ctypes.data_as(C.c_void_p), 1, out.ctypes.data_as(C.c_void_p)),
                   "commit")
        assert np.array_equal(out, host._dev.commit_array(w[None])[0])
    finally:
        L.lc_ajtai_key_destroy(h)
