"""GPU parity of the digit decompositions and of commits to unsigned digits.

decomp_b (lattice-folding/src/neo.rs:253-266) and GadgetDecomposition::
decompose (lattice-core/src/decomposition.rs:48-70) against the oracle on
seeded values plus the edge values the reference's tests use (0, 1, p-1,
2^32, 2^63, 2^64-1, base/2 boundaries); the recomposition identity
z = sum_r 2^(b r) Z_r at the 2^26-element folding-step size; commits of
unsigned byte digits (NTT and tensor engines) against the oracle, including
the extreme u8 x u8 sums of a full 512-element tensor-core chunk; and the
folding identity sum_r 256^r C(Z_r) = C(z) mod p.
"""
import numpy as np
import pytest

import oracle
from lzx_b200 import GadgetDecomposition, GoldilocksAjtaiKey, _lib, decomp_b, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = oracle.GL_P


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


EDGES = np.array([0, 1, 2, 127, 128, 129, 255, 256, P - 1, P - 2, 1 << 32, (1 << 32) - 1, 1 << 63,
                  (1 << 63) - 1, 0xFFFFFFFF00000000], dtype=np.uint64)


def values(count, seed):
    v = synth.synth_gl(seed, 7, count)
    v[: min(count, EDGES.size)] = EDGES[: min(count, EDGES.size)]
    return v


@pytest.mark.parametrize("b_bits", [1, 2, 3, 4, 5, 7, 8])
@pytest.mark.parametrize("count", [1, 7, 8, 1000, 4099])
def test_decomp_b_matches_oracle(b_bits, count):
    z = values(count, b_bits * 100 + count)
    got = decomp_b(z, b_bits)
    want = oracle.decomp_b(z, b_bits)
    assert got.shape == want.shape
    assert np.array_equal(got.astype(np.uint64), want)


def test_decomp_b_reduces_noncanonical_input():
    """Goldilocks values are canonical in the reference (to_canonical_u64)."""
    z = np.array([P, P + 5, 0xFFFFFFFFFFFFFFFF, P - 1], dtype=np.uint64)
    canon = np.array([0, 5, 0xFFFFFFFFFFFFFFFF - P, P - 1], dtype=np.uint64)
    assert np.array_equal(decomp_b(z, 8).astype(np.uint64), oracle.decomp_b(canon, 8))


@pytest.mark.parametrize("log_b,nd", [(8, 9), (8, 8), (4, 17), (1, 65), (15, 5), (7, 10), (3, 22), (8, 3)])
def test_gadget_matches_oracle(log_b, nd):
    base = 1 << log_b
    z = values(600, log_b * 31 + nd)
    extra = np.array([base // 2, base // 2 + 1, base - 1, 0xFFFFFFFFFFFFFFFF, (base // 2) * (base + 1)],
                     dtype=np.uint64)
    z = np.concatenate([z, extra])
    digits, too_large = GadgetDecomposition(base, nd).decompose_batch(z)
    bad = 0
    for e, x in enumerate(z.tolist()):
        try:
            want = oracle.gadget_decompose(base, nd, x)
        except ValueError:
            bad += 1
            continue
        assert digits[:, e].astype(np.int64).tolist() == want.tolist(), (e, x)
    assert too_large == bad


def test_gadget_power_of_two_covers_u64():
    g = GadgetDecomposition.power_of_two(64, 8)
    assert (g.base, g.num_digits) == (256, 9)  # decomposition.rs:38-43
    z = values(5000, 3)
    digits, too_large = g.decompose_batch(z)
    assert too_large == 0
    assert digits.min() >= -127 and digits.max() <= 128  # the reference keeps +base/2 positive
    acc = [0] * z.size
    for r in reversed(range(g.num_digits)):
        acc = [a * 256 + int(d) for a, d in zip(acc, digits[r].tolist())]
    assert acc == [int(x) for x in z]


def test_decomp_b_recompose_folding_size():
    """2^20 ring elements x 64 coefficients: z = sum_r 256^r Z_r for every value."""
    n = (1 << 20) * 64
    z = torch.empty(n, dtype=torch.int64, device="cuda")
    synth.fill_device(z, "gl", 77, 1)
    rows = decomp_b(z, 8)
    assert rows.shape == (8, n)
    acc = torch.zeros(n, dtype=torch.int64, device="cuda")
    for r in range(8):
        acc |= rows[r].to(torch.int64) << (8 * r)
    assert torch.equal(acc, z)  # canonical residues: exact 64-bit identity


def oracle_commit_res(A, kappa, m, W):
    t = oracle.NttTablesGl(6)
    return oracle.ajtaigl_commit_batch(t, t.forward_batch(A), kappa, m, W.astype(np.uint64))


@pytest.mark.parametrize("kappa,m,batch", [(3, 5, 2), (16, 300, 8), (8, 64, 129)])
def test_commit_u8_both_engines(kappa, m, batch):
    A = synth.synth_gl(kappa + 1, m, kappa * m * 64)
    W = synth.synth_i8(m, batch, batch * m * 64).view(np.uint8).reshape(batch, m, 64)
    key = GoldilocksAjtaiKey(6, kappa, m, A.reshape(kappa, m, 64), tensor_cores=True)
    tc = key.commit(W)
    key.engine = GoldilocksAjtaiKey.ENGINE_NTT
    ntt = key.commit(W)
    assert np.array_equal(tc, ntt)
    idx = sorted({0, batch - 1})
    assert np.array_equal(ntt[idx], oracle_commit_res(A, kappa, m, W[idx]))


@pytest.mark.parametrize("m", [511, 512, 513, 1025])
def test_commit_u8_extreme_chunk_sums(m):
    """All digits 255 against key limbs 0xFF: the largest u8 x u8 int32 sums."""
    kappa, batch = 4, 128
    A = np.full(kappa * m * 64, P - 1, dtype=np.uint64)
    W = np.full((batch, m, 64), 255, dtype=np.uint8)
    key = GoldilocksAjtaiKey(6, kappa, m, A.reshape(kappa, m, 64), tensor_cores=True)
    tc = key.commit(W)
    key.engine = GoldilocksAjtaiKey.ENGINE_NTT
    assert np.array_equal(tc, key.commit(W))
    assert np.array_equal(tc[:1], oracle_commit_res(A, kappa, m, W[:1]))


def test_folding_identity_digit_commitments():
    """sum_r 256^r C(Z_r) == C(z) mod p for z decomposed by decomp_b."""
    kappa, m = 16, 300
    A = synth.synth_gl(9, 0, kappa * m * 64)
    key = GoldilocksAjtaiKey(6, kappa, m, A.reshape(kappa, m, 64), tensor_cores=True)
    z = synth.synth_gl(9, 1, m * 64)
    rows = decomp_b(z, 8).reshape(8, m, 64)
    cz = key.commit(z.reshape(1, m, 64))[0]
    for engine in (GoldilocksAjtaiKey.ENGINE_TENSOR_I8, GoldilocksAjtaiKey.ENGINE_NTT):
        key.engine = engine
        cd = key.commit(rows)
        acc = [0] * cz.size
        for r in reversed(range(8)):
            acc = [(a * 256 + int(c)) % P for a, c in zip(acc, cd[r].reshape(-1).tolist())]
        assert acc == [int(x) for x in cz.reshape(-1)]
