"""GPU parity of the Modulus50 quadratic-slot ring (lattice-ring/src/
modulus50.rs) against the oracle: forward, inverse, slotwise Karatsuba and
the fused ring product for every log_n in [1, 7], Q_50 and two other
two-adicity-7 primes, one / ragged / large batches, in-place calls, the
host-buffer entry point, and the reference's errors."""
import numpy as np
import pytest

import oracle
from lzx_b200 import _lib
from lzx_b200.ring50 import Mod50Error, Modulus50, QuadSlotTables, RingConfig50

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MODULI = [oracle.Q_50, (1125899905792897, 7, 5), (1125891316907393, 7, 3)]


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def residues(q, count, n, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, q, size=(count, n), dtype=np.uint64)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def host(t):
    return t.cpu().numpy().view(np.uint64)


def per_poly(fn, *arrs):
    return np.stack([fn(*(a[i] for a in arrs)) for i in range(arrs[0].shape[0])])


@pytest.mark.parametrize("mod", MODULI, ids=lambda m: str(m[0]))
@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 5, 6, 7])
def test_transforms_and_products_match_oracle(mod, log_n):
    q, n = mod[0], 1 << log_n
    ot = oracle.QuadSlotTables50(oracle.Modulus50(*mod), log_n)
    t = QuadSlotTables(Modulus50(*mod), log_n)
    assert t.zeta == ot.zeta and np.array_equal(t.leaf_gamma, ot.leaf_gamma)
    for count in (1, 37):
        a = residues(q, count, n, 10 * log_n + count)
        b = residues(q, count, n, 10 * log_n + count + 1)
        a[0, 0], b[0, -1] = q - 1, q - 1  # top residue
        fa = host(t.forward(dev(a)))
        assert np.array_equal(fa, per_poly(ot.forward, a))
        assert np.array_equal(host(t.inverse(dev(a))), per_poly(ot.inverse, a))
        assert np.array_equal(host(t.inverse(dev(fa))), a)
        fb = per_poly(ot.forward, b)
        assert np.array_equal(host(t.slotwise_mul(dev(fa), dev(fb))), per_poly(ot.slotwise_mul, fa, fb))
        want = per_poly(ot.mul, a, b)
        assert np.array_equal(host(t.mul(dev(a), dev(b))), want)
        assert np.array_equal(t.mul(a, b), want)  # host-buffer entry point


def test_large_batch_and_in_place():
    log_n, count = 7, 1 << 15
    mod = oracle.Q_50
    ot = oracle.QuadSlotTables50(oracle.Modulus50(*mod), log_n)
    t = QuadSlotTables(Modulus50(*mod), log_n)
    a = residues(mod[0], count, 128, 1)
    b = residues(mod[0], count, 128, 2)
    want = ot.mul_batch(a, b)
    da, db = dev(a), dev(b)
    L = _lib.lib()
    import ctypes as C
    st = torch.cuda.current_stream().cuda_stream
    # in place: out aliases a
    assert L.lc_quad50_mul(t.handle, C.c_void_p(da.data_ptr()), C.c_void_p(db.data_ptr()),
                           C.c_void_p(da.data_ptr()), count, C.c_void_p(st)) == 0
    assert np.array_equal(host(da), want)
    assert np.array_equal(t.mul(a, b), want)  # host path, several staging chunks
    dx = dev(a)
    assert L.lc_quad50_forward(t.handle, C.c_void_p(dx.data_ptr()), C.c_void_p(dx.data_ptr()), count,
                               C.c_void_p(st)) == 0
    assert L.lc_quad50_inverse(t.handle, C.c_void_p(dx.data_ptr()), C.c_void_p(dx.data_ptr()), count,
                               C.c_void_p(st)) == 0
    assert np.array_equal(host(dx), a)
    assert L.lc_quad50_mul(t.handle, None, None, None, 0, C.c_void_p(st)) == 0  # empty batch


def test_ring_config50_api():
    ring = RingConfig50.new(4)
    q = ring.modulus.q
    v = ring.from_signed([-3, -2, -1, 0, 1, 2, 3, 4, 5, 5, 5, 5, 5, 5, 5, 5])  # modulus50.rs:765-771
    assert ring.infinity_norm(v) == 5 and v[0] == q - 3
    a, b = residues(q, 1, 16, 3)[0], residues(q, 1, 16, 4)[0]
    ot = oracle.QuadSlotTables50(oracle.Modulus50(*oracle.Q_50), 4)
    assert np.array_equal(ring.mul(a, b), ot.mul(a, b))
    assert np.array_equal(ring.sub(ring.add(a, b), b), a)
    assert len(ring.slot_constants()) == 8


def test_errors():
    with pytest.raises(Mod50Error) as e:
        RingConfig50.new(0)
    assert e.value.kind == Mod50Error.LogNOutOfRange
    with pytest.raises(Mod50Error) as e:
        RingConfig50.new(8)
    assert e.value.kind == Mod50Error.LogNOutOfRange
    with pytest.raises(Mod50Error) as e:
        RingConfig50.with_modulus(Modulus50.new(oracle.Q_50[0], 5, 3), 3)
    assert e.value.kind == Mod50Error.AdicityTooSmall
    with pytest.raises(Mod50Error) as e:
        RingConfig50.with_modulus(Modulus50.new(oracle.Q_50[0], 7, 4), 3)
    assert e.value.kind == Mod50Error.GeneratorInvalid
    ring = RingConfig50.new(3)
    with pytest.raises(Mod50Error) as e:
        ring.mul(np.array([1, 2, 3], dtype=np.uint64), np.array([1, 2, 3], dtype=np.uint64))
    assert e.value.kind == Mod50Error.LengthMismatch
