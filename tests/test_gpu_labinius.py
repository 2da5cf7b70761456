"""GPU parity of the labinius commitment (crates/lattice-labinius, key.rs:
94-137 and :382-474) against the oracle: CommitmentKey::random rows, the
general transform of every limb prime on both trees, and commitments (raw
rows, the 4 x r matrix of R_162 elements and the base limb's kept
transform) for split, quadratic and mixed limb lists, several chunk counts and
lengths, through the device and the host-buffer entry points; plus the
reference's argument checks."""
import ctypes as C

import numpy as np
import pytest

import oracle
from oracle import lb
from lzx_b200 import _lib
from lzx_b200.labinius import CommitmentKey, Modulus, random_witness

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    if not torch.cuda.is_available() or not _lib.lib().lc_device_available():
        pytest.fail("GPU tests need an sm_100 device and the CUDA library")


LIMB_LISTS = [
    [Modulus.Q3889_FS_S, Modulus.Q2917_Q_S],
    [Modulus.Q9721_FS_S],
    [Modulus.Q2917_Q_S, Modulus.Q4861_Q_S, Modulus.Q12637_Q_S],
    [Modulus.Q17497_FS_L, Modulus.Q19441_FS_L, Modulus.Q3889_FS_S],
]


@pytest.mark.parametrize("limbs", LIMB_LISTS, ids=lambda l: "-".join(str(m.prime()) for m in l))
def test_key_random_matches_oracle(limbs):
    key = CommitmentKey.random(64, 0xC0FFEE, limbs[0], limbs[1:])
    assert np.array_equal(key.a, lb.key_random(64, 0xC0FFEE, [m.prime() for m in limbs]))
    assert key.len_ring() == 16 and key.limbs() == len(limbs) and key.bytes() == len(limbs) * 16 * 2 * 648


@pytest.mark.parametrize("q", [m.prime() for m in Modulus])
def test_transform_matches_oracle(q):
    key = CommitmentKey.random(4, 1, Modulus.from_prime(q))
    rng = np.random.default_rng(q)
    count = 37
    a = rng.integers(0, 2**20, (count, 648), dtype=np.uint32)  # reduced mod q first, as ntt_of
    a[0] = q - 1
    din = torch.from_numpy(a.view(np.int32)).cuda()
    dout = torch.empty_like(din)
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(_lib.lib().lc_lb_ntt(key.handle, 0, C.c_void_p(din.data_ptr()), C.c_void_p(dout.data_ptr()),
                                    count, st), "lc_lb_ntt")
    got = dout.cpu().numpy().view(np.uint32)
    for i in range(count):
        assert np.array_equal(got[i], lb.ntt(q, a[i] % q)), i


@pytest.mark.parametrize("limbs", LIMB_LISTS, ids=lambda l: "-".join(str(m.prime()) for m in l))
@pytest.mark.parametrize("len_f162,r", [(4, 2), (64, 4), (132, 8), (1024, 2)])
def test_commit_matches_oracle(limbs, len_f162, r):
    primes = [m.prime() for m in limbs]
    key = CommitmentKey.random(len_f162, 7 + len_f162, limbs[0], limbs[1:])
    w = random_witness(r * len_f162, 99 + r)
    raw, mat, bat = lb.commit(key.a, primes, len_f162, w, r)
    cm, aux = key.commit(w, r)
    assert np.array_equal(aux.raw, raw)
    assert np.array_equal(cm.value, mat)
    assert np.array_equal(aux.batches, bat)
    assert cm.cols() == r and cm.rows() == 4 and cm.primes == primes
    dw = torch.from_numpy(w.view(np.int64)).cuda()
    dcm, daux = key.commit(dw, r, batches=False)
    assert daux.batches is None
    assert np.array_equal(daux.raw.cpu().numpy().view(np.uint32), raw)
    assert np.array_equal(dcm.value.cpu().numpy(), mat)


def test_commit_suite_shape_sizexs():
    """suite sizexs (scheme.rs:91-99): 2^14 F162 in 16 columns, moduli 3889 + 2917."""
    limbs = [Modulus.Q3889_FS_S, Modulus.Q2917_Q_S]
    len_f162, r = (1 << 14) // 16, 16
    key = CommitmentKey.random(len_f162, 2024, limbs[0], limbs[1:])
    w = random_witness(r * len_f162, 42)
    raw, mat, bat = lb.commit(key.a, [3889, 2917], len_f162, w, r)
    cm, aux = key.commit(w, r)
    assert np.array_equal(aux.raw, raw) and np.array_equal(cm.value, mat) and np.array_equal(aux.batches, bat)


def test_commit_linearity_and_zero():
    key = CommitmentKey.random(64, 5, Modulus.Q3889_FS_S, [Modulus.Q2917_Q_S])
    zero = np.zeros((2 * 64, 3), np.uint64)
    cm, aux = key.commit(zero, 2)
    assert not aux.raw.any() and not cm.value.any() and not aux.batches.any()


def test_argument_errors():
    L = _lib.lib()
    h = C.c_void_p()
    primes = (C.c_uint16 * 2)(3889, 3889)
    assert L.lc_lb_key_random(64, 1, primes, 2, C.byref(h)) == _lib.LC_ERR_INVALID_ARGUMENT  # limb twice
    primes = (C.c_uint16 * 1)(7681)
    assert L.lc_lb_key_random(64, 1, primes, 1, C.byref(h)) == _lib.LC_ERR_INVALID_ARGUMENT  # not a limb prime
    primes = (C.c_uint16 * 1)(3889)
    assert L.lc_lb_key_random(6, 1, primes, 1, C.byref(h)) == _lib.LC_ERR_INVALID_ARGUMENT  # not a multiple of 4
    key = CommitmentKey.random(8, 1)
    w = random_witness(3 * 8, 1)
    with pytest.raises(_lib.LatticeCudaError):
        key.commit(w, 3)  # r must be a power of two >= 2
    with pytest.raises(_lib.LatticeCudaError):
        key.commit(w[:8], 1)
