"""The Modulus50 quadratic-slot oracle (oracle/, restating
lattice-ring/src/modulus50.rs) pinned by the reference's own tests of that
file (modulus50.rs:499-772): the paper prime's structure, Barrett against
division on random and boundary values, the round trip for every log_n,
products against the schoolbook negacyclic convolution, the ring axioms, the
slot-constant structure and the error cases.  Also the C ABI's plan-creation
errors, which return before any device work."""
import ctypes as C

import numpy as np
import pytest

import oracle
from lzx_b200 import _lib

Q = oracle.Q_50[0]
M64 = (1 << 64) - 1
# two more two-adicity-7 primes in (2^49, 2^50) with their smallest non-residue generators
OTHER_MODULI = [(1125899905792897, 7, 5), (1125891316907393, 7, 3)]


def xorshift_stream(seed):
    """The generator of the reference's tests (modulus50.rs:523-533)."""
    state = seed

    def nxt():
        nonlocal state
        state ^= state >> 12
        state ^= (state << 25) & M64
        state ^= state >> 27
        return (state * 0x2545F4914F6CDD1D) & M64
    return nxt


def random_vec(q, n, seed):
    nxt = xorshift_stream(seed)
    return np.array([(nxt() >> 20) % q for _ in range(n)], dtype=np.uint64)


def schoolbook_negacyclic(q, a, b):
    """modulus50.rs:504-521"""
    n = len(a)
    acc = [0] * n
    for i in range(n):
        for j in range(n):
            prod = int(a[i]) * int(b[j])
            k = i + j
            if k < n:
                acc[k] += prod
            else:
                acc[k - n] -= prod
    return np.array([c % q for c in acc], dtype=np.uint64)


def is_prime(n):
    for p in [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37]:
        if n % p == 0:
            return n == p
    d, r = n - 1, 0
    while d % 2 == 0:
        d, r = d // 2, r + 1
    for a in [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37]:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(r - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def tables(log_n, mod=oracle.Q_50):
    return oracle.QuadSlotTables50(oracle.Modulus50(*mod), log_n)


def test_modulus_is_the_paper_prime():  # modulus50.rs:536-555
    m = oracle.Modulus50(*oracle.Q_50)
    assert Q == 2**50 - 2687 and Q % 256 == 129 and ((Q - 1) >> 7) & 1 == 1
    zeta = m.pow(m.generator, (Q - 1) >> 7)
    assert m.pow(zeta, 128) == 1 and m.pow(zeta, 64) == Q - 1
    assert is_prime(Q)
    for q, adic, g in OTHER_MODULI:
        assert is_prime(q) and q % 256 == 129 and pow(g, (q - 1) // 2, q) == q - 1


@pytest.mark.parametrize("mod", [oracle.Q_50] + OTHER_MODULI, ids=lambda m: str(m[0]))
def test_barrett_matches_division(mod):  # modulus50.rs:597-633
    m = oracle.Modulus50(*mod)
    q = mod[0]
    nxt = xorshift_stream(0x123456789ABCDEF0)
    for _ in range(50_000 if mod == oracle.Q_50 else 5_000):
        a, b = nxt() % q, nxt() % q
        assert m.mul(a, b) == a * b % q
    for x in [0, 1, q - 1, q, q + 1, (1 << 50) - 1, 1 << 50, (1 << 62) - 1, 1 << 62, (1 << 99) - 1,
              (q - 1) * (q - 1)]:
        assert m.reduce_u128(x) == x % q, x


def test_roundtrip_all_log_n():  # modulus50.rs:635-645
    for log_n in range(1, 8):
        t = tables(log_n)
        a = random_vec(Q, 1 << log_n, 0xABCD + log_n)
        assert np.array_equal(t.inverse(t.forward(a)), a), log_n


def test_mul_matches_schoolbook_all_log_n():  # modulus50.rs:647-659
    for log_n in [1, 2, 3, 5, 7]:
        t = tables(log_n)
        for trial in range(4):
            a = random_vec(Q, 1 << log_n, 0x1111 + trial * 7 + log_n)
            b = random_vec(Q, 1 << log_n, 0x2222 + trial * 13 + log_n)
            assert np.array_equal(t.mul(a, b), schoolbook_negacyclic(Q, a, b)), (log_n, trial)


@pytest.mark.parametrize("mod", OTHER_MODULI, ids=lambda m: str(m[0]))
def test_other_moduli_mul_matches_schoolbook(mod):
    for log_n in (1, 4, 7):
        t = tables(log_n, mod)
        a = random_vec(mod[0], 1 << log_n, 5 + log_n)
        b = random_vec(mod[0], 1 << log_n, 9 + log_n)
        assert np.array_equal(t.mul(a, b), schoolbook_negacyclic(mod[0], a, b))
        assert np.array_equal(t.inverse(t.forward(a)), a)


def test_mul_ring_axioms():  # modulus50.rs:661-712
    t = tables(7)
    n = 128
    a, b, c = (random_vec(Q, n, s) for s in (1, 2, 3))
    mul = t.mul
    assert np.array_equal(mul(a, b), mul(b, a))
    assert np.array_equal(mul(mul(a, b), c), mul(a, mul(b, c)))
    add = lambda x, y: np.array([(int(u) + int(v)) % Q for u, v in zip(x, y)], dtype=np.uint64)  # noqa: E731
    assert np.array_equal(mul(add(a, b), c), add(mul(a, c), mul(b, c)))
    one = np.zeros(n, dtype=np.uint64)
    one[0] = 1
    assert np.array_equal(mul(a, one), a)
    assert not mul(a, np.zeros(n, dtype=np.uint64)).any()
    x = np.zeros(n, dtype=np.uint64)
    x[1] = 1
    xn1 = np.zeros(n, dtype=np.uint64)
    xn1[n - 1] = 1
    prod = mul(x, xn1)
    assert prod[0] == Q - 1 and not prod[1:].any()


def test_slot_constants_have_the_paper_structure():  # modulus50.rs:714-741
    m = oracle.Modulus50(*oracle.Q_50)
    g7 = tables(7).leaf_gamma
    assert len(g7) == 64 and all(m.pow(int(g), 64) == Q - 1 for g in g7)
    assert len(set(g7.tolist())) == 64
    g6 = tables(6).leaf_gamma
    assert len(g6) == 32 and all(m.pow(int(g), 32) == Q - 1 for g in g6)


def test_errors_rejected():  # modulus50.rs:743-763
    with pytest.raises(oracle.NttError) as e:
        tables(0)
    assert e.value.code == 13
    with pytest.raises(oracle.NttError) as e:
        tables(8)
    assert e.value.code == 13
    with pytest.raises(oracle.NttError) as e:
        tables(3, (Q, 5, 3))
    assert e.value.code == 2
    with pytest.raises(oracle.NttError) as e:
        tables(3, (Q, 7, 4))  # 4 is a square: zeta^64 = 1
    assert e.value.code == 14
    t = tables(3)
    with pytest.raises(oracle.NttError) as e:
        t.mul(np.array([1, 2, 3], dtype=np.uint64), np.array([1, 2, 3], dtype=np.uint64))
    assert e.value.code == 1


def test_abi_plan_errors_without_device():
    """lc_quad50_plan_create validates in the reference's order before any device call."""
    L = _lib.lib()
    h = C.c_void_p()
    assert L.lc_quad50_plan_create(Q, 7, 3, 0, C.byref(h)) == _lib.LC_ERR_LOG_N_OUT_OF_RANGE
    assert L.lc_quad50_plan_create(Q, 7, 3, 8, C.byref(h)) == _lib.LC_ERR_LOG_N_OUT_OF_RANGE
    assert L.lc_quad50_plan_create(Q, 5, 3, 3, C.byref(h)) == _lib.LC_ERR_ADICITY_TOO_SMALL
    assert L.lc_quad50_plan_create(Q, 7, 4, 3, C.byref(h)) == _lib.LC_ERR_GENERATOR_INVALID
    assert L.lc_quad50_plan_create((1 << 50) + 1, 7, 3, 3, C.byref(h)) == _lib.LC_ERR_INVALID_ARGUMENT
    assert L.lc_quad50_plan_create(Q + 1, 7, 3, 3, C.byref(h)) == _lib.LC_ERR_INVALID_ARGUMENT
    assert h.value is None
    assert L.lc_quad50_plan_create(Q, 7, 3, 3, None) == _lib.LC_ERR_INVALID_ARGUMENT
