"""Oracle parity at the full sizes of the uneven batch and the folding step.

* Uneven batch (512 jobs, d in {64,128,256}, n log-uniform in [2^10, 2^18],
  kappa in {8,16}, Goldilocks or the 4-prime 30-bit CRT set, int8 witnesses):
  the graph-captured batch equals the jobs committed one by one through key
  views, and sampled jobs -- the longest job of every key class plus random
  ones -- equal the oracle's AjtaiPublicKey::commit
  (lattice-commitment/src/ajtai.rs:118-153) on their first and last key rows
  over the job's whole length n, so every K range and staircase offset of the
  long jobs is checked.
* Folding step (2^20 ring elements, kappa = 16): every one of the 8 digit
  commitments (lattice-folding/src/neo.rs:253-266 digits, committed as by
  ajtai.rs:118-153) equals the oracle in all 16 x 64 residues.

A commitment row depends only on its key row, so the oracle regenerates a
few key rows at a time from the same counter-based stream the device keys
were filled from (at most 2 GiB of key on the host instead of 8 GiB).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    from lzx_b200 import _lib
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def _u(x):
    a = x.cpu().numpy()
    return a.view(np.uint64) if a.dtype == np.int64 else a.view(np.uint32)


def _oracle_row_gl(seed, log_d, m, row, n, w):
    """Oracle commitment row `row` of a Goldilocks key filled from stream (seed, 0)."""
    d = 1 << log_d
    t = oracle.NttTablesGl(log_d)
    a = oracle.synth_gl(seed, 0, n * d, offset=row * m * d)
    a_ntt = t.forward_batch(a.reshape(n, d), nthreads=0)
    return oracle.ajtaigl_commit_batch(t, a_ntt, 1, n, w.reshape(-1, n, d), nthreads=0)[:, 0]


def _oracle_row_u32(seed, prime_index, log_d, m, row, n, w_i8):
    """Oracle commitment row `row` of the u32 key of CRT prime `prime_index`."""
    q, adic, g = oracle.CRT_PRIMES[prime_index]
    d = 1 << log_d
    t = oracle.NttTables32(oracle.Modulus32(q, adic, g), log_d)
    a = oracle.synth_mod32(seed, prime_index, q, n * d, offset=row * m * d)
    a_ntt = t.forward_batch(a.reshape(n, d), nthreads=0)
    s = np.where(w_i8 < 0, q - np.abs(w_i8.astype(np.int64)), w_i8).astype(np.uint32)
    return oracle.ajtai32_commit(t, a_ntt, 1, n, s)[0]


def test_uneven_batch_full_size_against_oracle():
    import bench
    from lzx_b200.batch import CommitBatch, key_view
    wl = bench.uneven_workload(0, 512, 18)
    specs, classes, jobs, m = wl["specs"], wl["classes"], wl["jobs"], wl["m"]
    batch = CommitBatch(classes, jobs, graph=True)
    for _ in range(2):  # capture + launch, replay
        batch.run()
    batch.check()
    torch.cuda.synchronize()
    # every job against the same job committed one call at a time
    for j in jobs:
        ref = torch.empty_like(j.out)
        for k, key in enumerate(classes[j.cls]):
            key_view(key, j.kappa, j.n).commit_i8(j.w, ref[k])
        assert torch.equal(j.out, ref), (j.cls, j.kappa, j.n)
    # sampled jobs against the oracle: the longest job of each class, plus random ones
    rng = np.random.default_rng(5)
    sample = set()
    for c in range(len(specs)):
        idx = [i for i, j in enumerate(jobs) if j.cls == c]
        if idx:
            sample.add(max(idx, key=lambda i: jobs[i].n))
    sample |= set(int(i) for i in rng.choice(len(jobs), 6, replace=False))
    assert max(jobs[i].n for i in sample) > 1 << 17
    for i in sorted(sample):
        j = jobs[i]
        log_d, gl = specs[j.cls]
        seed = wl["key_seeds"][j.cls]
        w = j.w.cpu().numpy()
        got = _u(j.out)
        for row in (0, j.kappa - 1):
            if gl:
                want = _oracle_row_gl(seed, log_d, m, row, j.n, w)[0]
                assert np.array_equal(got[0, row], want), (i, row)
            else:
                for p in range(4):
                    want = _oracle_row_u32(seed, p, log_d, m, row, j.n, w)
                    assert np.array_equal(got[p, row], want), (i, p, row)
    del batch, jobs, classes, wl
    torch.cuda.empty_cache()


def test_fold_step_full_size_commitments_against_oracle():
    from lzx_b200 import CRT_SET_30BIT, GoldilocksAjtaiKey, NttTables, synth
    from lzx_b200.pipeline import FoldPipeline
    kappa, m, seed = 16, 1 << 20, 77
    A = torch.empty(kappa * m * 64, dtype=torch.int64, device="cuda")
    synth.fill_device(A, "gl", seed, 0)
    key = GoldilocksAjtaiKey(6, kappa, m, A)
    del A
    crt = NttTables(CRT_SET_30BIT, 6)
    pipe = FoldPipeline(key, crt, use_graph=True)
    synth.fill_device(pipe.z, "gl", seed, 1)
    for _ in range(2):
        pipe.run()
    pipe.check()
    torch.cuda.synchronize()
    digits = pipe.digits.cpu().numpy()              # [8][m][64] unsigned bytes
    got = _u(pipe.commits)                            # [8][kappa][64]
    z = oracle.synth_gl(seed, 1, m * 64)
    assert np.array_equal(_u(pipe.z).reshape(-1), z)
    assert np.array_equal(digits.reshape(8, -1), oracle.decomp_b(z, 8).astype(np.uint8))
    t = oracle.NttTablesGl(6)
    wide = digits.astype(np.uint64)                   # the 8 digit rows as residue witnesses
    rows = 4                                          # key rows per oracle call (2 GiB of NTT(A))
    for r0 in range(0, kappa, rows):
        a = oracle.synth_gl(seed, 0, rows * m * 64, offset=r0 * m * 64)
        a_ntt = t.forward_batch(a.reshape(rows * m, 64), nthreads=0)
        want = oracle.ajtaigl_commit_batch(t, a_ntt, rows, m, wide, nthreads=0)   # [8][rows][64]
        assert np.array_equal(got[:, r0:r0 + rows], want), r0
    del pipe, key
    torch.cuda.empty_cache()
