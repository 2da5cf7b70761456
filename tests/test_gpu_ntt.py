"""GPU parity of the batched NTT/INTT against the CPU oracle (bit-exact).

Re-runs the reference's NTT tests (lattice-ring/src/ntt.rs:364-479,
ring.rs:485-568) on the CUDA path, checks the golden vectors, every modulus
family and ring degree the kernels build, the edge values, and the full-size
CRT batch (2^16 polynomials x 4 primes x d=256) through size-independent
properties plus a sampled oracle comparison.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from lzx_b200 import (CRT_SET_30BIT, GoldilocksNttTables, Modulus32, NttError, NttTables, RingConfig,
                      RingElement, _lib)
from lzx_b200 import synth, tune

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def ora_tables(m: Modulus32, log_n):
    return oracle.NttTables32(oracle.Modulus32(m.q, m.two_adicity, m.generator), log_n)


def to_dev(a: np.ndarray):
    if a.dtype == np.uint32:
        return torch.from_numpy(a.view(np.int32)).cuda()
    return torch.from_numpy(a.view(np.int64)).cuda()


def from_dev(t, dtype):
    return t.cpu().numpy().view(dtype)


MODULI = [Modulus32.Q_32, Modulus32.Q_12289, Modulus32.Q_2013265921, CRT_SET_30BIT[0],
          CRT_SET_30BIT[3]]


@pytest.mark.parametrize("m", MODULI, ids=lambda m: str(m.q))
@pytest.mark.parametrize("log_n", list(range(1, 12)))
def test_u32_forward_inverse_match_oracle(m, log_n):
    if log_n + 1 > m.two_adicity:
        with pytest.raises(NttError):
            NttTables(m, log_n)
        return
    n, count = 1 << log_n, 37
    a = synth.synth_mod32(100 + log_n, 1, m.q, count * n).reshape(count, n)
    t = NttTables(m, log_n)
    ot = ora_tables(m, log_n)
    want = ot.forward_batch(a)
    dev = to_dev(a.copy())
    t.forward_fast(dev)
    torch.cuda.synchronize()
    got = from_dev(dev, np.uint32)
    assert np.array_equal(got, want)
    t.inverse_fast(dev)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(dev, np.uint32), a)
    # inverse of arbitrary (non-image) input equals the oracle's inverse_fast
    b = synth.synth_mod32(200 + log_n, 2, m.q, count * n).reshape(count, n)
    assert np.array_equal(t.inverse_fast(b.copy()), ot.inverse_batch(b))


@pytest.mark.parametrize("log_n", list(range(1, 11)))
def test_goldilocks_forward_inverse_match_oracle(log_n):
    n, count = 1 << log_n, 33
    a = synth.synth_gl(300 + log_n, 1, count * n).reshape(count, n)
    t = GoldilocksNttTables(log_n)
    ot = oracle.NttTablesGl(log_n)
    want = ot.forward_batch(a)
    got = t.forward_fast(a.copy())
    assert np.array_equal(got, want)
    assert np.array_equal(t.inverse_fast(got.copy()), a)
    b = synth.synth_gl(400 + log_n, 2, count * n).reshape(count, n)
    assert np.array_equal(t.inverse_fast(b.copy()), ot.inverse_batch(b))


def test_golden_vectors(golden):
    for v in golden["ntt_q32_kat_manifest"] + golden["ntt_q32_extra"]:
        t = NttTables(Modulus32.Q_32, v["log_n"])
        a = np.array(v["input"], dtype=np.uint32)
        assert t.forward_fast(a.copy()).tolist() == v["forward"]
    for v in golden["ntt_crt"]:
        t = NttTables(Modulus32(v["q"], v["two_adicity"], v["generator"]), v["log_n"])
        a = np.array(v["input"], dtype=np.uint32)
        assert t.forward_fast(a.copy()).tolist() == v["forward"]
    for v in golden["ntt_goldilocks"]:
        t = GoldilocksNttTables(v["log_n"])
        a = np.array([int(x) for x in v["input"]], dtype=np.uint64)
        assert [str(x) for x in t.forward_fast(a.copy()).tolist()] == v["forward"]


def test_crt_set_layout_matches_per_prime_plans():
    """A 4-prime plan on [prime][count][n] equals four single-prime transforms."""
    count, n = 513, 256
    a = synth.crt_batch(5, CRT_SET_30BIT, count, n)
    t = NttTables(CRT_SET_30BIT, 8)
    got = t.forward_fast(a.copy())
    for i, m in enumerate(CRT_SET_30BIT):
        assert np.array_equal(got[i], ora_tables(m, 8).forward_batch(a[i]))
    assert np.array_equal(t.inverse_fast(got.copy()), a)


@pytest.mark.parametrize("m", [Modulus32.Q_32, CRT_SET_30BIT[1]], ids=lambda m: str(m.q))
def test_edge_values(m):
    """Zeros, q-1 everywhere (lazy-reduction extremes), impulses, count 0 and 1."""
    log_n, n = 8, 256
    t = NttTables(m, log_n)
    ot = ora_tables(m, log_n)
    cases = np.stack([np.zeros(n, np.uint32), np.full(n, m.q - 1, np.uint32),
                      np.eye(n, dtype=np.uint32)[0], np.eye(n, dtype=np.uint32)[n - 1],
                      np.full(n, 1, np.uint32)])
    assert np.array_equal(t.forward_fast(cases.copy()), ot.forward_batch(cases))
    assert np.array_equal(t.inverse_fast(cases.copy()), ot.inverse_batch(cases))
    one = cases[1:2].copy()
    assert np.array_equal(t.forward_fast(one), ot.forward_batch(cases[1:2]))
    empty = np.zeros((0, n), np.uint32)
    assert t.forward_fast(empty).shape == (0, n)


def test_length_mismatch_and_alignment():
    t = NttTables(Modulus32.Q_32, 8)
    with pytest.raises(NttError) as e:
        t.forward_fast(np.zeros(128, np.uint32))  # ntt.rs:469-479
    assert e.value.kind == "LengthMismatch"
    buf = torch.zeros(256 * 4 + 1, dtype=torch.int32, device="cuda")
    L = _lib.lib()
    st = L.lc_ntt_forward(t.handle, C.c_void_p(buf.data_ptr() + 4), C.c_void_p(buf.data_ptr() + 4),
                          4, None)
    assert st == _lib.LC_ERR_INVALID_ARGUMENT


def test_out_of_place_device_and_host_agree():
    count, n = 1000, 256
    a = synth.crt_batch(9, CRT_SET_30BIT, count, n)
    t = NttTables(CRT_SET_30BIT, 8)
    src = to_dev(a.copy())
    dst = torch.empty_like(src)
    t.forward_fast(src, out=dst)
    torch.cuda.synchronize()
    host = t.forward_fast(a.copy())
    assert np.array_equal(from_dev(dst, np.uint32).reshape(host.shape), host)
    assert np.array_equal(from_dev(src, np.uint32).reshape(a.shape), a)  # input untouched
    assert _lib.lib().lc_ntt_plan_check(t.handle, None) == 0


def test_host_entry_points_over_many_chunks():
    """The host-buffer transforms stream each modulus's polynomials in chunks
    of about 16 MiB; a batch of two full chunks plus a ragged one per modulus
    gives the device transform's residues and comes back by the inverse."""
    count, n = 2 * 16384 + 123, 256
    a = synth.crt_batch(31, CRT_SET_30BIT, count, n)
    t = NttTables(CRT_SET_30BIT, 8)
    dev = to_dev(a.copy())
    t.forward_fast(dev)
    torch.cuda.synchronize()
    host = t.forward_fast(a.copy())
    assert np.array_equal(from_dev(dev, np.uint32).reshape(host.shape), host)
    back = t.inverse_fast(host)
    assert np.array_equal(back, a)
    assert _lib.lib().lc_ntt_plan_check(t.handle, None) == 0


@pytest.mark.parametrize("kind", ["crt", "q32", "goldilocks"])
def test_host_entry_points_on_pinned_buffers(kind):
    """Pinned host buffers through the host-buffer entry points (chunks copied
    straight from and to them): the residues equal the device transform's,
    out of place and in place, and for a buffer starting 4 bytes into a
    pinned allocation, with the inverse bringing the input back each time."""
    L = _lib.lib()
    if kind == "goldilocks":
        count, n, log_n = 3001, 64, 6
        t = GoldilocksNttTables(log_n)
        a = synth.synth_gl(41, 0, count * n).reshape(count, n)
        tdt, ndt = torch.int64, np.uint64
    else:
        mods = CRT_SET_30BIT if kind == "crt" else [Modulus32.Q_32]
        count, n, log_n = (20003, 256, 8) if kind == "crt" else (777, 128, 7)
        t = NttTables(mods, log_n)
        a = synth.crt_batch(43, mods, count, n) if kind == "crt" else \
            synth.synth_mod32(43, 0, Modulus32.Q_32.q, count * n).reshape(count, n)
        tdt, ndt = torch.int32, np.uint32
    want = to_dev(a.copy())
    t.forward_fast(want)
    torch.cuda.synchronize()
    want = from_dev(want, ndt).reshape(a.shape)
    flat = a.reshape(-1)
    size, eb = flat.size, flat.itemsize
    src = torch.from_numpy(flat.view(np.int64 if eb == 8 else np.int32).copy()).pin_memory()
    dst = torch.empty_like(src).pin_memory()
    for inp, outp in ((src, dst), (dst, dst)):
        if inp is dst:
            dst.copy_(src)
        st = L.lc_ntt_forward_host(t.handle, C.c_void_p(inp.data_ptr()), C.c_void_p(outp.data_ptr()), count)
        assert st == 0, _lib.lib().lc_status_string(st)
        assert np.array_equal(outp.numpy().view(ndt).reshape(a.shape), want)
        st = L.lc_ntt_inverse_host(t.handle, C.c_void_p(outp.data_ptr()), C.c_void_p(outp.data_ptr()), count)
        assert st == 0
        assert np.array_equal(outp.numpy().view(ndt).reshape(a.shape), a)
    big = torch.zeros(size + 16 // eb, dtype=tdt).pin_memory()
    big[1:1 + size] = src
    p = C.c_void_p(big.data_ptr() + eb)
    assert L.lc_ntt_forward_host(t.handle, p, p, count) == 0
    assert np.array_equal(big[1:1 + size].numpy().view(ndt).reshape(a.shape), want)
    assert L.lc_ntt_plan_check(t.handle, None) == 0


def test_full_size_crt_round_trip_and_samples():
    """2^16 polynomials x d=256 x 4 primes: the bench workload."""
    count, n = 1 << 16, 256
    a = synth.crt_batch(2024, CRT_SET_30BIT, count, n)
    t = NttTables(CRT_SET_30BIT, 8)
    dev = to_dev(a.copy())
    t.forward_fast(dev)
    torch.cuda.synchronize()
    fwd = from_dev(dev, np.uint32).reshape(a.shape)
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(count, 1024, replace=False))
    idx = np.unique(np.concatenate([idx, [0, count - 1]]))
    for i, m in enumerate(CRT_SET_30BIT):
        assert np.array_equal(fwd[i, idx], ora_tables(m, 8).forward_batch(a[i, idx]))
    # linearity: NTT(a + b) == NTT(a) + NTT(b) on the whole batch
    b = synth.crt_batch(77, CRT_SET_30BIT, count, n)
    qs = np.array([m.q for m in CRT_SET_30BIT], dtype=np.uint64)[:, None, None]
    s = ((a.astype(np.uint64) + b) % qs).astype(np.uint32)
    fb = t.forward_fast(b.copy())
    fs = t.forward_fast(s.copy())
    assert np.array_equal(fs, ((fwd.astype(np.uint64) + fb) % qs).astype(np.uint32))
    t.inverse_fast(dev)
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(dev, np.uint32).reshape(a.shape), a)
    assert _lib.lib().lc_ntt_plan_check(t.handle, None) == 0


def test_ring_element_api():
    """ring.rs:485-568 on the GPU-backed ring."""
    c = RingConfig(Modulus32.Q_32, 6)
    a = c.random(b"m-a")
    assert a.mul(c.one()) == a
    assert a.mul(c.zero()).is_zero()
    x_nm1 = RingElement.from_coeffs(c, np.eye(c.n(), dtype=np.uint32)[c.n() - 1])
    assert c.x_gen().mul(x_nm1) == c.constant(c.modulus.q - 1)
    b = c.random(b"m-b")
    om = oracle.Modulus32(*oracle.Q_32)
    assert np.array_equal(a.mul(b).coeffs(), ora_tables(Modulus32.Q_32, 6).ring_mul(a.coeffs(), b.coeffs()))
    assert np.array_equal(c.random(b"m-a").coeffs(), oracle.ring_random(om, 6, b"m-a"))
    ev = a.to_ntt()
    assert RingElement.from_ntt(c, ev) == a
    u = c.uniform_from_seed(b"ajtai-A", bytes([42]) * 32, 7)
    assert np.array_equal(u.coeffs(), oracle.uniform_from_seed(om, 6, b"ajtai-A", bytes([42]) * 32, 7))


@pytest.mark.parametrize("variant", range(tune.NUM_VARIANTS))
def test_every_kernel_variant_is_bit_exact(variant):
    """The tuner may pick any instantiated kernel shape; all must agree with the oracle."""
    count = 1003  # not a multiple of any tile size
    a = synth.crt_batch(31, CRT_SET_30BIT, count, 256)
    t = NttTables(CRT_SET_30BIT, 8)
    assert _lib.lib().lc_ntt_plan_set_variant(t.handle, variant) == 0
    got = t.forward_fast(a.copy())
    for i, m in enumerate(CRT_SET_30BIT):
        assert np.array_equal(got[i], ora_tables(m, 8).forward_batch(a[i]))
    assert np.array_equal(t.inverse_fast(got.copy()), a)
    g = synth.synth_gl(32, 0, 777 * 64).reshape(777, 64)
    tg = GoldilocksNttTables(6)
    assert _lib.lib().lc_ntt_plan_set_variant(tg.handle, variant) == 0
    fg = tg.forward_fast(g.copy())
    assert np.array_equal(fg, oracle.NttTablesGl(6).forward_batch(g))
    assert np.array_equal(tg.inverse_fast(fg.copy()), g)
    assert _lib.lib().lc_ntt_plan_set_variant(t.handle, tune.NUM_VARIANTS) == _lib.LC_ERR_INVALID_ARGUMENT
    assert _lib.lib().lc_ntt_plan_set_variant(t.handle, -1) == _lib.LC_ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("variant", range(tune.NUM_VARIANTS))
def test_every_kernel_variant_on_many_tiles_per_cta(variant):
    """2^17 + 3 polynomials per prime: about ten tiles per CTA, so each
    variant's load/store ring wraps several times.  Inputs come from the device
    generator; full round trip on the device plus oracle rows from the host
    generator at three places of the batch."""
    count, n = (1 << 17) + 3, 256
    t = NttTables(CRT_SET_30BIT, 8)
    L = _lib.lib()
    assert L.lc_ntt_plan_set_variant(t.handle, variant) == 0
    x = torch.empty(len(CRT_SET_30BIT) * count * n, dtype=torch.int32, device="cuda")
    for i, m in enumerate(CRT_SET_30BIT):
        synth.fill_device(x[i * count * n:(i + 1) * count * n], "mod32", 77, i, q=m.q)
    y, z = torch.empty_like(x), torch.empty_like(x)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.lc_ntt_forward(t.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), count, st) == 0
    assert L.lc_ntt_inverse(t.handle, C.c_void_p(y.data_ptr()), C.c_void_p(z.data_ptr()), count, st) == 0
    assert L.lc_ntt_plan_check(t.handle, st) == 0
    assert torch.equal(z, x)
    got = from_dev(y, np.uint32).reshape(len(CRT_SET_30BIT), count, n)
    for i, m in enumerate(CRT_SET_30BIT):
        for r0, r1 in ((0, 24), (70_000, 70_016), (count - 24, count)):
            a = synth.synth_mod32(77, i, m.q, (r1 - r0) * n, offset=r0 * n).reshape(-1, n)
            assert np.array_equal(got[i][r0:r1], ora_tables(m, 8).forward_batch(a))
    cg = 300_007
    g = torch.empty(cg * 64, dtype=torch.int64, device="cuda")
    synth.fill_device(g, "gl", 78, 0)
    tg = GoldilocksNttTables(6)
    assert L.lc_ntt_plan_set_variant(tg.handle, variant) == 0
    fg, bg = torch.empty_like(g), torch.empty_like(g)
    assert L.lc_ntt_forward(tg.handle, C.c_void_p(g.data_ptr()), C.c_void_p(fg.data_ptr()), cg, st) == 0
    assert L.lc_ntt_inverse(tg.handle, C.c_void_p(fg.data_ptr()), C.c_void_p(bg.data_ptr()), cg, st) == 0
    assert L.lc_ntt_plan_check(tg.handle, st) == 0
    assert torch.equal(bg, g)
    fh = from_dev(fg, np.uint64).reshape(cg, 64)
    for r0, r1 in ((0, 32), (cg - 32, cg)):
        a = synth.synth_gl(78, 0, (r1 - r0) * 64, offset=r0 * 64).reshape(-1, 64)
        assert np.array_equal(fh[r0:r1], oracle.NttTablesGl(6).forward_batch(a))


def test_device_synth_matches_host_generator():
    """lc_synth_fill reproduces the seeded host stream bit for bit."""
    n = 100_003
    for kind, q, dt, host in (("u64", 0, torch.int64, lambda: synth.synth_u64(7, 3, n, 11)),
                              ("mod32", Modulus32.Q_32.q, torch.int32,
                               lambda: synth.synth_mod32(7, 3, Modulus32.Q_32.q, n, 11)),
                              ("mod32", CRT_SET_30BIT[0].q, torch.int32,
                               lambda: synth.synth_mod32(7, 3, CRT_SET_30BIT[0].q, n, 11)),
                              ("gl", 0, torch.int64, lambda: synth.synth_gl(7, 3, n, 11)),
                              ("i8", 0, torch.int8, lambda: synth.synth_i8(7, 3, n, 11))):
        t = torch.empty(n, dtype=dt, device="cuda")
        synth.fill_device(t, kind, 7, 3, q, offset=11)
        got = t.cpu().numpy()
        want = host()
        assert np.array_equal(got.view(want.dtype), want), kind
