"""GPU parity of pack_field_elements (lattice-ring/src/packing.rs:30-52) and
of the Akita PCS commit it feeds (lattice-akita/src/pcs.rs:66-76): packed
coefficients equal the oracle's for empty, ragged and large inputs and the
limb-boundary values; an AkitaPcs::commit-shaped commitment (Q_32, k = 2,
pad_to_m) equals the oracle's pack + AjtaiPublicKey::commit."""
import numpy as np
import pytest

import oracle
from lzx_b200 import AjtaiError, AjtaiParams, AjtaiPublicKey, Modulus32, RingConfig, _lib, synth
from lzx_b200.packing import akita_commit, pack_field_elements

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = oracle.GL_P
Q32 = Modulus32.Q_32.q


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


EDGES = [0, 1, (1 << 22) - 1, 1 << 22, (1 << 44) - 1, 1 << 44, P - 1, P, 0xFFFFFFFFFFFFFFFF, 0xFFFFFFFF00000000]


@pytest.mark.parametrize("log_n", [2, 6, 8])
@pytest.mark.parametrize("count", [0, 1, 21, 22, 1000])
def test_pack_matches_oracle(log_n, count):
    v = synth.synth_u64(count, log_n, count)
    v[:min(count, len(EDGES))] = EDGES[:min(count, len(EDGES))]
    ring = RingConfig(Modulus32.Q_32, log_n)
    got = pack_field_elements(ring, v).cpu().numpy().view(np.uint32)
    assert np.array_equal(got, oracle.pack_field_elements(Q32, log_n, v))


def test_pack_padding_and_shape_check():
    ring = RingConfig(Modulus32.Q_32, 6)
    v = synth.synth_gl(1, 1, 30)  # 90 limbs -> 2 ring elements
    got = pack_field_elements(ring, v, 5).cpu().numpy().view(np.uint32)
    want = oracle.pack_field_elements(Q32, 6, v)
    assert np.array_equal(got[:2], want) and not got[2:].any()
    with pytest.raises(AjtaiError):
        pack_field_elements(ring, v, 1)


@pytest.mark.parametrize("log_n,m,num_vars", [(6, 16, 8), (8, 8, 9), (6, 64, 10)])
def test_akita_commit_matches_oracle(log_n, m, num_vars):
    params = AjtaiParams(RingConfig(Modulus32.Q_32, log_n), 2, m, 1 << 23)
    seed = bytes([0x42]) * 32
    pk = AjtaiPublicKey.from_seed(params, seed)
    evals = synth.synth_gl(num_vars, 2, 1 << num_vars)
    got = akita_commit(pk, evals)
    packed = oracle.pack_field_elements(Q32, log_n, evals)
    s = np.zeros((m, 1 << log_n), dtype=np.uint32)
    s[:packed.shape[0]] = packed
    t = oracle.NttTables32(oracle.Modulus32(*oracle.Q_32), log_n)
    mat, mat_ntt = oracle.ajtai32_from_seed(t, 2, m, seed)
    want = oracle.ajtai32_commit(t, mat_ntt, 2, m, s)
    assert np.array_equal(np.stack([r.coeffs() for r in got.rows]), want)


def test_akita_commit_too_many_evaluations():
    params = AjtaiParams(RingConfig(Modulus32.Q_32, 6), 2, 4, 1 << 23)
    pk = AjtaiPublicKey.from_seed(params, bytes(32))
    with pytest.raises(AjtaiError):  # 300 values -> 15 ring elements > m = 4 (pad_to_m)
        akita_commit(pk, synth.synth_gl(0, 0, 300))
