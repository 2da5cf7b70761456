"""GPU parity of the folding-step pipeline and the CRT residue split.

Every output of a folding step (decomp_b digit rows, the 8 digit
commitments, the CRT-set forward NTT of z) equals the oracle on the same
seeded z, on the eager run, on graph replays, after z changes in place, and
after the key's scratch was reallocated by another commit (the graph is
captured again).  At the 2^20-element folding-step size: the folding identity
sum_r 256^r C(Z_r) = C(z), the CRT NTT round trip, oracle rows of the NTT.
"""
import numpy as np
import pytest

import oracle
from lzx_b200 import CRT_SET_30BIT, GoldilocksAjtaiKey, NttTables, _lib, synth
from lzx_b200.pipeline import FoldPipeline, crt_residues

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = oracle.GL_P


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def crt_oracle_tables():
    return [oracle.NttTables32(oracle.Modulus32(*q), 6) for q in oracle.CRT_PRIMES]


def test_crt_residues_match_modulo():
    tables = NttTables(CRT_SET_30BIT, 6)
    z = synth.synth_u64(3, 3, 10001)
    z[:6] = [0, 1, 0xFFFFFFFFFFFFFFFF, 1073738753, 1073738752, P - 1]
    got = crt_residues(tables, z)
    for i, (q, _, _) in enumerate(oracle.CRT_PRIMES):
        assert np.array_equal(got[i], (z % np.uint64(q)).astype(np.uint32))


def expected_step(A, kappa, m, z):
    digits = oracle.decomp_b(z, 8).astype(np.uint8)
    t = oracle.NttTablesGl(6)
    commits = oracle.ajtaigl_commit_batch(t, t.forward_batch(A), kappa, m,
                                          digits.reshape(8, m, 64).astype(np.uint64))
    crt = np.stack([tb.forward_batch((z % np.uint64(q)).astype(np.uint32))
                    for tb, (q, _, _) in zip(crt_oracle_tables(), oracle.CRT_PRIMES)])
    return digits.reshape(8, m, 64), commits, crt.reshape(4, m, 64)


def check_outputs(pipe, want):
    torch.cuda.synchronize()
    digits, commits, crt = want
    assert np.array_equal(pipe.digits.cpu().numpy(), digits)
    assert np.array_equal(pipe.commits.cpu().numpy().view(np.uint64), commits)
    assert np.array_equal(pipe.crt_ntt.cpu().numpy().view(np.uint32), crt)


@pytest.mark.parametrize("use_graph,products", [(False, GoldilocksAjtaiKey.PRODUCTS_TENSOR),
                                                (True, GoldilocksAjtaiKey.PRODUCTS_TENSOR),
                                                (True, GoldilocksAjtaiKey.PRODUCTS_INT64)])
def test_fold_pipeline_small(use_graph, products):
    """The integer-product form runs its products, split sums and inverse
    transforms as one cooperative launch, captured in the graph too."""
    kappa, m = 16, 300
    A = synth.synth_gl(31, 0, kappa * m * 64)
    key = GoldilocksAjtaiKey(6, kappa, m, A.reshape(kappa, m, 64))
    key.slot_products = products
    crt = NttTables(CRT_SET_30BIT, 6)
    pipe = FoldPipeline(key, crt, use_graph=use_graph)
    z = synth.synth_gl(31, 1, m * 64)
    pipe.z.copy_(torch.from_numpy(z.view(np.int64)).reshape(m, 64))
    want = expected_step(A, kappa, m, z)
    for _ in range(3):  # eager warm-up, capture + launch, replay
        pipe.run()
        check_outputs(pipe, want)
    # new witness in place: the replay reads the buffer again
    z2 = synth.synth_gl(31, 2, m * 64)
    pipe.z.copy_(torch.from_numpy(z2.view(np.int64)).reshape(m, 64))
    pipe.run()
    check_outputs(pipe, expected_step(A, kappa, m, z2))
    # another commit on the key reallocates its scratch: the next run recaptures
    W = synth.synth_i8(1, 1, 200 * m * 64).reshape(200, m, 64)
    key.commit(W)
    pipe.run()
    check_outputs(pipe, expected_step(A, kappa, m, z2))
    pipe.check()


def test_fold_pipeline_crt_branch_montgomery_moduli():
    """The CRT branch (residues of z formed in shared memory and transformed
    in the same launch) over a plan of primes above 2^30, which run the
    signed-Montgomery arithmetic: every row equals the oracle's NTT of
    z mod q, with a ragged last tile (m = 333)."""
    from lzx_b200 import Modulus32
    kappa, m = 2, 333
    A = synth.synth_gl(32, 0, kappa * m * 64)
    key = GoldilocksAjtaiKey(6, kappa, m, A.reshape(kappa, m, 64))
    mods = [Modulus32.Q_32, Modulus32.Q_2013265921]
    crt = NttTables(mods, 6)
    pipe = FoldPipeline(key, crt, use_graph=False)
    z = synth.synth_u64(32, 1, m * 64)
    pipe.z.copy_(torch.from_numpy(z.view(np.int64)).reshape(m, 64))
    pipe.run()
    pipe.check()
    torch.cuda.synchronize()
    got = pipe.crt_ntt.cpu().numpy().view(np.uint32).reshape(len(mods), m, 64)
    for i, md in enumerate(mods):
        tb = oracle.NttTables32(oracle.Modulus32(md.q, md.two_adicity, md.generator), 6)
        want = tb.forward_batch((z % np.uint64(md.q)).astype(np.uint32).reshape(m, 64))
        assert np.array_equal(got[i], want), md.q


def test_fold_pipeline_folding_size():
    """2^20 ring elements, kappa = 16 (the folding-step workload)."""
    kappa, m = 16, 1 << 20
    A = torch.empty(kappa * m * 64, dtype=torch.int64, device="cuda")
    synth.fill_device(A, "gl", 55, 0)
    key = GoldilocksAjtaiKey(6, kappa, m, A)
    crt = NttTables(CRT_SET_30BIT, 6)
    pipe = FoldPipeline(key, crt, use_graph=True)
    synth.fill_device(pipe.z, "gl", 55, 1)
    for _ in range(3):
        pipe.run()
    pipe.check()
    torch.cuda.synchronize()
    z = pipe.z.clone()
    # digit rows recompose to z
    acc = torch.zeros_like(z)
    for r in range(8):
        acc |= pipe.digits[r].to(torch.int64) << (8 * r)
    assert torch.equal(acc, z)
    # folding identity against the residue commitment of z itself
    cz = key.commit(z.view(1, m, 64)).cpu().numpy().view(np.uint64)[0].reshape(-1)
    cd = pipe.commits.cpu().numpy().view(np.uint64).reshape(8, -1)
    acc = [0] * cz.size
    for r in reversed(range(8)):
        acc = [(a * 256 + int(c)) % P for a, c in zip(acc, cd[r].tolist())]
    assert acc == [int(x) for x in cz]
    # CRT NTT: inverse gives z mod q_i back; oracle rows of the forward
    fwd = pipe.crt_ntt.clone()
    back = fwd.clone()
    crt.inverse_fast(back.view(-1))
    torch.cuda.synchronize()
    zc = z.cpu().numpy().view(np.uint64).reshape(-1)
    for i, (q, _, _) in enumerate(oracle.CRT_PRIMES):
        assert np.array_equal(back[i].cpu().numpy().view(np.uint32).reshape(-1),
                              (zc % np.uint64(q)).astype(np.uint32))
    rows = [0, 12345, m - 1]
    for i, tb in enumerate(crt_oracle_tables()):
        q = oracle.CRT_PRIMES[i][0]
        src = (zc.reshape(m, 64)[rows] % np.uint64(q)).astype(np.uint32)
        assert np.array_equal(fwd[i][rows].cpu().numpy().view(np.uint32), tb.forward_batch(src))
