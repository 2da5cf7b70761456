"""GPU parity of the incomplete NTT (NttTables::forward_partial /
complete_partial, lattice-ring/src/ntt.rs:252-316) against the oracle:
every level count 0..log n, several moduli (a CRT set plan included),
batches of polynomials; completing a partial transform equals the full
forward transform; the reference's argument errors."""
import numpy as np
import pytest

import oracle
from lzx_b200 import CRT_SET_30BIT, GoldilocksNttTables, Modulus32, NttError, NttTables, _lib, synth

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


def otab(m, log_n):
    return oracle.NttTables32(oracle.Modulus32(m.q, m.two_adicity, m.generator), log_n)


@pytest.mark.parametrize("mod", [Modulus32.Q_32, Modulus32.Q_12289, Modulus32.Q_2013265921, CRT_SET_30BIT[1]],
                         ids=lambda m: str(m.q))
@pytest.mark.parametrize("log_n", [1, 3, 6, 8])
def test_partial_levels_match_oracle(mod, log_n):
    n, count = 1 << log_n, 5
    t = NttTables(mod, log_n)
    ot = otab(mod, log_n)
    a = synth.synth_mod32(log_n, 3, mod.q, count * n).reshape(count, n)
    full = t.forward_fast(a.copy())
    for levels in range(log_n + 1):
        part = t.forward_partial(a.copy(), levels)
        for p in range(count):
            assert np.array_equal(part[p], ot.forward_partial(a[p], levels)), (levels, p)
        done = t.complete_partial(part.copy(), levels)
        for p in range(count):
            assert np.array_equal(done[p], ot.complete_partial(part[p], levels)), (levels, p)
        assert np.array_equal(done, full), levels


def test_partial_crt_set_and_degree_11():
    log_n, count = 8, 33
    t = NttTables(CRT_SET_30BIT, log_n)
    a = synth.crt_batch(7, CRT_SET_30BIT, count, 1 << log_n)
    full = t.forward_fast(a.copy())
    for levels in (0, 3, 8):
        part = t.forward_partial(a.copy(), levels)
        for i, m in enumerate(CRT_SET_30BIT):
            ot = otab(m, log_n)
            for p in (0, 32):
                assert np.array_equal(part[i, p], ot.forward_partial(a[i, p], levels))
        assert np.array_equal(t.complete_partial(part, levels), full)
    t11 = NttTables(Modulus32.Q_32, 11)
    a11 = synth.synth_mod32(11, 1, Modulus32.Q_32.q, 3 << 11).reshape(3, 1 << 11)
    part = t11.forward_partial(a11.copy(), 7)
    assert np.array_equal(part[2], otab(Modulus32.Q_32, 11).forward_partial(a11[2], 7))
    assert np.array_equal(t11.complete_partial(part, 7), t11.forward_fast(a11.copy()))


def test_partial_errors():
    t = NttTables(Modulus32.Q_32, 6)
    a = np.zeros((2, 64), dtype=np.uint32)
    with pytest.raises(NttError):  # ntt.rs:258-260
        t.forward_partial(a, 7)
    with pytest.raises(NttError):  # ntt.rs:292-294
        t.complete_partial(a, 7)
    with pytest.raises(NttError):  # length not a multiple of n
        t.forward_partial(np.zeros(65, dtype=np.uint32), 2)
    gl = GoldilocksNttTables(6)
    x = torch.zeros(64, dtype=torch.int64, device="cuda")
    assert _lib.lib().lc_ntt_forward_partial(gl.handle, x.data_ptr(), x.data_ptr(), 1, 2, None) == \
        _lib.LC_ERR_UNSUPPORTED
