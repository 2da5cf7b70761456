"""GPU parity of the Ajtai commitment against the CPU oracle (bit-exact).

Re-runs the reference's commitment tests (lattice-commitment/src/ajtai.rs:368-570)
on the CUDA path -- KAT-manifest commitments, cached-NTT == naive, linearity,
zero skipping, opening/tamper/norm checks -- and the Goldilocks batch
commitments of the int8-digit workloads: the single d=64, kappa=8, n=256
commitment and the kappa=16, 2^16-element, 128-witness batch, every
commitment compared with the oracle.
"""
import numpy as np
import pytest

import oracle
from lzx_b200 import (AjtaiCommitment, AjtaiError, AjtaiParams, AjtaiPublicKey, GoldilocksAjtaiKey,
                      Modulus32, RingConfig, RingElement, _lib, sample_small_secret, synth)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = oracle.GL_P


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def params(log_n, k, m, bound):
    return AjtaiParams(RingConfig(Modulus32.Q_32, log_n), k, m, bound)


def q32_tables(log_n):
    return oracle.NttTables32(oracle.Modulus32(*oracle.Q_32), log_n)


def test_kat_manifest_commitments(golden):
    """kat_manifest.rs:128-155 commitments (seed 0xAB*32, k=2, m=8)."""
    for v in golden["ajtai_q32_kat_manifest"]:
        pk = AjtaiPublicKey.from_seed(params(v["log_n"], v["k"], v["m"], 1 << 23),
                                      bytes.fromhex(v["seed_hex"]))
        assert pk.entry(0, 0).coeffs().tolist() == v["matrix_row0"]
        s = sample_small_secret(pk.params.ring, v["m"], 1 << 12, b"kat-secret")
        assert [e.coeffs().tolist() for e in s] == v["secret"]
        t = pk.commit(s)
        assert [r.coeffs().tolist() for r in t.rows] == v["rows"]
        assert oracle.hash_domain(b"kat-ajtai", t.to_bytes()).hex() == v["digest"]


@pytest.mark.parametrize("log_n,k,m,bound", [(4, 2, 3, 255), (5, 2, 8, 8), (6, 3, 12, 3), (6, 1, 16, 1),
                                             (8, 2, 16, 32), (7, 2, 64, 1 << 20)])
def test_cached_ntt_matches_naive_and_oracle(log_n, k, m, bound):
    """ajtai.rs:489-506: cached-NTT commit == naive per-product commit."""
    pk = AjtaiPublicKey.from_seed(params(log_n, k, m, bound), bytes([9]) * 32)
    s = sample_small_secret(pk.params.ring, m, bound, b"diff")
    fast = pk.commit(s)
    assert fast == pk.commit_naive_reference(s)
    t = q32_tables(log_n)
    mat, _ = oracle.ajtai32_from_seed(t, k, m, bytes([9]) * 32)
    want = oracle.ajtai32_commit_naive(t, mat, k, m, np.stack([e.coeffs() for e in s]))
    assert np.array_equal(np.stack([r.coeffs() for r in fast.rows]), want)


def test_open_verify_tamper_and_norm():
    """ajtai.rs:368-412."""
    pk = AjtaiPublicKey.from_seed(params(6, 2, 3, 64), bytes([1]) * 32)
    s = sample_small_secret(pk.params.ring, 3, 8, b"secret")
    t = pk.commit(s)
    pk.verify_opening(t, s)
    s2 = sample_small_secret(pk.params.ring, 3, 8, b"other")
    with pytest.raises(AjtaiError) as e:
        pk.verify_opening(t, s2)
    assert e.value.kind == "CommitmentMismatch"
    bad = AjtaiCommitment([RingElement(pk.params.ring, r.coeffs().copy()) for r in t.rows])
    bad.rows[0].coeffs()[0] = (int(bad.rows[0].coeffs()[0]) + 1) % pk.params.ring.modulus.q
    with pytest.raises(AjtaiError):
        pk.verify_opening(bad, s)
    pk8 = AjtaiPublicKey.from_seed(params(6, 2, 3, 8), bytes([3]) * 32)
    big = pk8.params.ring.constant(1000)
    with pytest.raises(AjtaiError) as e:
        pk8.verify_opening(pk8.commit([big, big, big]), [big, big, big])
    assert e.value.kind == "NormExceeded" and e.value.fields == {"norm": 1000, "bound": 8}
    data = t.to_bytes()
    assert AjtaiCommitment.from_bytes(pk.params.ring, 2, data) == t
    with pytest.raises(AjtaiError):
        AjtaiCommitment.from_bytes(pk.params.ring, 2, data[:10])
    with pytest.raises(AjtaiError):
        pk.commit(s[:2])


def test_linearity_and_zero_skip():
    """ajtai.rs:467-487 and :547-570."""
    pk = AjtaiPublicKey.from_seed(params(6, 2, 8, 1 << 20), bytes([6]) * 32)
    ring = pk.params.ring
    s1 = sample_small_secret(ring, 8, 8, b"a")
    s2 = sample_small_secret(ring, 8, 8, b"b")
    t1, t2 = pk.commit(s1), pk.commit(s2)
    tsum = pk.commit([a.add(b) for a, b in zip(s1, s2)])
    assert AjtaiCommitment([a.add(b) for a, b in zip(t1.rows, t2.rows)]) == tsum
    zeros = [ring.zero() for _ in range(8)]
    assert all(r.is_zero() for r in pk.commit(zeros).rows)
    one_hot = [ring.zero() for _ in range(8)]
    c = np.zeros(ring.n(), np.uint32)
    c[0] = 12345
    one_hot[3] = RingElement(ring, c)
    assert pk.commit(one_hot) == pk.commit_naive_reference(one_hot)


def test_batch_commit_equals_single_commits():
    pk = AjtaiPublicKey.from_seed(params(8, 2, 16, 1 << 20), bytes([42]) * 32)
    ring = pk.params.ring
    batch = np.stack([np.stack([e.coeffs() for e in sample_small_secret(ring, 16, 32, bytes([b]))])
                      for b in range(70)])
    got = pk.commit_batch(batch)
    for b in (0, 1, 37, 69):
        single = pk.commit([RingElement(ring, x) for x in batch[b]])
        assert np.array_equal(got[b], np.stack([r.coeffs() for r in single.rows]))


def gl_key(kappa, m, d=64, seed=21):
    A = synth.synth_gl(seed, 0, kappa * m * d)
    return A, GoldilocksAjtaiKey(int(np.log2(d)), kappa, m, A.reshape(kappa, m, d))


def oracle_gl_commit(A, kappa, m, W, d=64):
    t = oracle.NttTablesGl(int(np.log2(d)))
    return oracle.ajtaigl_commit_batch(t, t.forward_batch(A), kappa, m, W)


def test_goldilocks_single_commit_config1():
    """d=64 Goldilocks, kappa=8, n=256 witness elements of int8 digits, one commitment."""
    kappa, m = 8, 256
    A, key = gl_key(kappa, m)
    W = synth.synth_i8(5, 1, m * 64).reshape(1, m, 64)
    got = key.commit(W)
    assert np.array_equal(got, oracle_gl_commit(A, kappa, m, W))
    # the coefficient-domain (Neo) commitment gives the same residues
    Wf = np.where(W < 0, np.uint64(P) - np.abs(W.astype(np.int64)).astype(np.uint64), W.astype(np.uint64))
    assert np.array_equal(got[0], oracle.neo_commit_naive(64, kappa, m, A, Wf.reshape(-1)))
    # residue input path gives the same result
    assert np.array_equal(key.commit(Wf), got)


def test_goldilocks_golden(golden):
    v = golden["ajtai_goldilocks_small"]
    d, kappa, m, B = v["d"], v["kappa"], v["m"], v["batch"]
    A = synth.synth_gl(v["a_seed"], v["a_stream"], kappa * m * d)
    W = synth.synth_i8(v["w_seed"], v["w_stream"], B * m * d).reshape(B, m, d)
    key = GoldilocksAjtaiKey(6, kappa, m, A.reshape(kappa, m, d))
    got = key.commit(W)
    assert [[[str(x) for x in r] for r in o] for o in got.tolist()] == v["out"]


@pytest.mark.parametrize("batch", [1, 3, 64, 100, 128, 256])
def test_goldilocks_batches_small_and_tiled(batch):
    """Small-batch and tiled (128-witness) product paths, padded batches included."""
    kappa, m = 16, 300
    A, key = gl_key(kappa, m, seed=batch)
    W = synth.synth_i8(7, batch, batch * m * 64).reshape(batch, m, 64)
    got = key.commit(W)
    idx = sorted({0, batch // 2, batch - 1})
    assert np.array_equal(got[idx], oracle_gl_commit(A, kappa, m, W[idx]))


@pytest.mark.parametrize("batch,m", [(8, 8192), (16, 4096), (32, 2048), (4, 16384), (1, 65536), (64, 1024),
                                     (130, 512), (128, 513)])
@pytest.mark.parametrize("digits", ["i8", "u8"])
def test_goldilocks_byte_digit_transform_shapes(batch, m, digits):
    """Shapes whose d = 64 witness transform runs as INT8 tensor-core products:
    tiles of 128/BB consecutive ring elements x BB witnesses (BB = 128, 32, 16,
    8, 4, 1), padded batches, an odd ring-element count."""
    kappa = 2
    A, key = gl_key(kappa, m, seed=batch + m)
    if digits == "i8":
        W = synth.synth_i8(9, batch, batch * m * 64).reshape(batch, m, 64)
        Wo = W
    else:
        W = synth.synth_i8(9, batch, batch * m * 64).reshape(batch, m, 64).view(np.uint8)
        Wo = W.astype(np.uint64)
    got = key.commit(W)
    for _ in range(2):  # repeated calls reuse the key's scratch
        assert np.array_equal(key.commit(W), got)
    assert np.array_equal(got, oracle_gl_commit(A, kappa, m, Wo))


@pytest.mark.parametrize("log_d,kappa", [(5, 3), (7, 16), (8, 5), (9, 2)])
def test_goldilocks_other_degrees(log_d, kappa):
    d, m, batch = 1 << log_d, 40, 130
    A, key = gl_key(kappa, m, d=d, seed=log_d)
    W = synth.synth_gl(8, log_d, batch * m * d).reshape(batch, m, d)
    got = key.commit(W)
    idx = [0, 77, 129]
    assert np.array_equal(got[idx], oracle_gl_commit(A, kappa, m, W[idx], d=d))


def test_goldilocks_config3_full_batch():
    """kappa=16, 2^16 witness elements, 128 int8 witnesses (the bench workload):
    every commitment of the batch checked against the oracle."""
    kappa, m, B, d = 16, 1 << 16, 128, 64
    A, key = gl_key(kappa, m, seed=3)
    W = synth.synth_i8(11, 3, B * m * d).reshape(B, m, d)
    dev = torch.from_numpy(W).cuda()
    got = key.commit(dev)
    torch.cuda.synchronize()
    got = got.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, oracle_gl_commit(A, kappa, m, W))
    assert _lib.lib().lc_ajtai_key_check(key.handle, None) == 0
