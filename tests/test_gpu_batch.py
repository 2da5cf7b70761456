"""GPU parity of the uneven-job commit batch and of key views.

Every job of a mixed batch (ring degrees 64/128/256; Goldilocks, the 4-prime
30-bit CRT set and Q_32; kappa 8 or 16; lengths from 1 to the key's m) must
equal the same job committed one by one through a key view
(lc_ajtai_key_view + lc_ajtai_commit_i8), and sampled jobs the oracle's
AjtaiPublicKey::commit (lattice-commitment/src/ajtai.rs:118-153) on the key's
first kappa rows and n columns -- with the products on the tensor cores (the
default) and on the CUDA cores.  Also: jobs longer than one exact int32
chunk of the tensor products, lanes split at 128 jobs, every tuning
configuration, graph replay after the witnesses change in place, and the
argument checks.
"""
import numpy as np
import pytest

import oracle
from lzx_b200 import CRT_SET_30BIT, GoldilocksAjtaiKey, LatticeCudaError, Modulus32, _lib, synth
from lzx_b200.batch import CommitBatch, CommitJob, U32AjtaiKey, key_view

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
P = oracle.GL_P


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def gl_class(log_d, m, seed):
    d = 1 << log_d
    A = synth.synth_gl(seed, 0, 16 * m * d)
    return {"keys": [GoldilocksAjtaiKey(log_d, 16, m, A.reshape(16, m, d))], "A": [A.reshape(16, m, d)],
            "d": d, "m": m, "moduli": [None]}


def u32_class(moduli, log_d, m, seed):
    d = 1 << log_d
    keys, mats = [], []
    for i, mod in enumerate(moduli):
        A = synth.synth_mod32(seed, i, mod.q, 16 * m * d).reshape(16, m, d)
        keys.append(U32AjtaiKey(mod, log_d, 16, m, A))
        mats.append(A)
    return {"keys": keys, "A": mats, "d": d, "m": m, "moduli": list(moduli)}


def make_jobs(classes, count, seed, n_cap=None):
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(count):
        c = int(rng.integers(len(classes)))
        cl = classes[c]
        m = cl["m"] if n_cap is None else min(cl["m"], n_cap)
        n = int(rng.integers(1, m + 1))
        kappa = int(rng.choice([8, 16]))
        w = torch.empty(n * cl["d"], dtype=torch.int8, device="cuda")
        synth.fill_device(w, "i8", seed, k)
        dt = torch.int64 if cl["moduli"][0] is None else torch.int32
        out = torch.full((len(cl["keys"]), kappa, cl["d"]), -1, dtype=dt, device="cuda")
        jobs.append(CommitJob(c, kappa, n, w.view(n, cl["d"]), out))
    return jobs


def one_by_one(classes, job):
    cl = classes[job.cls]
    res = torch.empty_like(job.out)
    for k, key in enumerate(cl["keys"]):
        v = key_view(key, job.kappa, job.n)
        v.commit_i8(job.w, res[k])
    return res


def oracle_job(cl, job):
    W = job.w.cpu().numpy()
    outs = []
    for A, mod in zip(cl["A"], cl["moduli"]):
        sub = np.ascontiguousarray(A[:job.kappa, :job.n])
        if mod is None:
            t = oracle.NttTablesGl(int(np.log2(cl["d"])))
            outs.append(oracle.ajtaigl_commit_batch(t, t.forward_batch(sub), job.kappa, job.n,
                                                    W.reshape(1, job.n, cl["d"]))[0])
        else:
            t = oracle.NttTables32(oracle.Modulus32(mod.q, mod.two_adicity, mod.generator), int(np.log2(cl["d"])))
            s = np.where(W < 0, mod.q - np.abs(W.astype(np.int64)), W).astype(np.uint32)
            outs.append(oracle.ajtai32_commit(t, t.forward_batch(sub.reshape(-1, cl["d"])), job.kappa, job.n, s))
    return np.stack(outs)


def as_u(x):
    a = x.cpu().numpy()
    return a.view(np.uint64) if a.dtype == np.int64 else a.view(np.uint32)


@pytest.fixture(scope="module")
def mixed_classes():
    return [gl_class(6, 300, 1), gl_class(7, 200, 2), gl_class(8, 90, 3),
            u32_class(CRT_SET_30BIT, 6, 300, 4), u32_class(CRT_SET_30BIT, 8, 90, 5),
            u32_class([Modulus32.Q_32], 6, 150, 6), u32_class(CRT_SET_30BIT[1:3], 7, 140, 7),
            u32_class([Modulus32.Q_12289], 7, 60, 8)]


def test_key_view_matches_submatrix_key(mixed_classes):
    cl = mixed_classes[0]
    A = cl["A"][0]
    sub = GoldilocksAjtaiKey(6, 8, 77, np.ascontiguousarray(A[:8, :77]))
    W = synth.synth_i8(3, 3, 77 * 64).reshape(1, 77, 64)
    w = torch.from_numpy(W[0]).cuda()
    out = torch.empty((8, 64), dtype=torch.int64, device="cuda")
    key_view(cl["keys"][0], 8, 77).commit_i8(w, out)
    torch.cuda.synchronize()
    assert np.array_equal(as_u(out), sub.commit(W)[0])
    with pytest.raises(LatticeCudaError):
        key_view(cl["keys"][0], 17, 10)
    with pytest.raises(LatticeCudaError):
        key_view(cl["keys"][0], 8, 301)


@pytest.mark.parametrize("graph,products", [(False, CommitBatch.PRODUCTS_TENSOR), (True, CommitBatch.PRODUCTS_TENSOR),
                                            (True, CommitBatch.PRODUCTS_INT64)])
def test_batch_mixed_jobs(mixed_classes, graph, products):
    jobs = make_jobs(mixed_classes, 60, 7)
    batch = CommitBatch([c["keys"] for c in mixed_classes], jobs, graph=graph)
    assert batch.products == CommitBatch.PRODUCTS_TENSOR  # the default
    batch.products = products
    assert batch.products == products
    for _ in range(3):  # eager, capture + launch, replay
        batch.run()
        batch.check()
        for j in jobs:
            assert torch.equal(j.out, one_by_one(mixed_classes, j)), (j.cls, j.kappa, j.n)
    for j in jobs[:12]:
        assert np.array_equal(as_u(j.out), oracle_job(mixed_classes[j.cls], j)), (j.cls, j.kappa, j.n)


@pytest.mark.parametrize("chunk,ctas,claim", [(1024, 1, 1), (2048, 3, 4), (16384, 4, 16), (4096, 2, 7)])
def test_batch_configs_agree(mixed_classes, chunk, ctas, claim):
    jobs = make_jobs(mixed_classes, 30, 11)
    batch = CommitBatch([c["keys"] for c in mixed_classes], jobs, graph=True)
    batch.set_config(chunk, ctas, claim)
    assert batch.config == (chunk, ctas, claim)
    batch.run()
    batch.run()
    batch.check()
    for j in jobs:
        assert torch.equal(j.out, one_by_one(mixed_classes, j))


def test_batch_lane_split_and_replay(mixed_classes):
    """300 jobs of one key: three lanes; new witness data under a replayed graph."""
    cls = [mixed_classes[0]]
    jobs = make_jobs(cls, 300, 13, n_cap=40)
    batch = CommitBatch([cls[0]["keys"]], jobs, graph=True)
    assert batch.info["lanes"] == 3
    batch.run()
    batch.run()
    for j in jobs[::7]:
        assert torch.equal(j.out, one_by_one(cls, j))
    for k, j in enumerate(jobs):
        synth.fill_device(j.w.view(-1), "i8", 99, k)
    batch.run()
    batch.check()
    for j in jobs[::5]:
        assert torch.equal(j.out, one_by_one(cls, j))


def test_batch_tensor_products_over_several_chunks():
    """Jobs longer than one exact int32 chunk (32768 ring elements) and blocks
    whose jobs end at different ring elements: tensor products = CUDA-core
    products = one-by-one commits = the oracle, after switching modes back
    and forth under a captured graph."""
    m = 70000
    classes = [gl_class(6, m, 41), u32_class(CRT_SET_30BIT[:1], 6, m, 42)]
    lens = [70000, 69999, 40000, 32769, 32768, 100, 1]
    jobs = []
    for c in range(2):
        for k, n in enumerate(lens + [int(x) for x in np.random.default_rng(c).integers(1, m, 30)]):
            w = torch.empty(n * 64, dtype=torch.int8, device="cuda")
            synth.fill_device(w, "i8", 43 + c, k)
            dt = torch.int64 if c == 0 else torch.int32
            out = torch.full((1, 16 if k % 2 else 8, 64), -1, dtype=dt, device="cuda")
            jobs.append(CommitJob(c, out.shape[1], n, w.view(n, 64), out))
    batch = CommitBatch([c["keys"] for c in classes], jobs, graph=True)
    outs = {}
    for mode in (CommitBatch.PRODUCTS_TENSOR, CommitBatch.PRODUCTS_INT64, CommitBatch.PRODUCTS_TENSOR):
        batch.products = mode
        for _ in range(2):
            batch.run()
        batch.check()
        outs.setdefault(mode, []).append([j.out.clone() for j in jobs])
    for a, b in zip(outs[CommitBatch.PRODUCTS_TENSOR][0], outs[CommitBatch.PRODUCTS_INT64][0]):
        assert torch.equal(a, b)
    for a, b in zip(outs[CommitBatch.PRODUCTS_TENSOR][0], outs[CommitBatch.PRODUCTS_TENSOR][1]):
        assert torch.equal(a, b)
    for j in jobs:
        assert torch.equal(j.out, one_by_one(classes, j)), (j.cls, j.kappa, j.n)
    for j in (jobs[0], jobs[3], jobs[len(lens)], jobs[len(lens) + 2]):
        assert np.array_equal(as_u(j.out), oracle_job(classes[j.cls], j)), (j.cls, j.kappa, j.n)


def test_batch_argument_checks(mixed_classes):
    cl = mixed_classes[0]
    keys = [cl["keys"]]
    w = torch.zeros(301 * 64 + 1, dtype=torch.int8, device="cuda")
    out = torch.empty((1, 8, 64), dtype=torch.int64, device="cuda")
    with pytest.raises(LatticeCudaError):  # n > m
        CommitBatch(keys, [CommitJob(0, 8, 301, w, out)])
    with pytest.raises(LatticeCudaError):  # kappa > k
        CommitBatch(keys, [CommitJob(0, 17, 10, w, out)])
    with pytest.raises(LatticeCudaError):  # misaligned witness
        CommitBatch(keys, [CommitJob(0, 8, 10, w[1:], out)])
    with pytest.raises(LatticeCudaError):  # class index
        CommitBatch(keys, [CommitJob(1, 8, 10, w, out)])
    empty = CommitBatch(keys, [])
    empty.run()
    empty.check()
    with pytest.raises(LatticeCudaError):  # no such product mode
        empty.products = 7
