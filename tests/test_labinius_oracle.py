"""The labinius oracle (oracle/labinius.c, restating crates/lattice-labinius)
pinned by the defining identities the reference states and checks:
the split transform is evaluation at psi^SLOT_EXP[j] (scalar.rs:36-37, eval_at
:88-97), the quadratic transform is reduction mod X^2 - psi'^u (scalar.rs:164,
eval_quad_at :215-226), transform products equal the schoolbook product mod
Phi_1944 (scalar.rs:10-34), the 4 x 162 decomposition equals the R_162
evaluations of the X^4-decimated coefficients (ring.rs:190-192,
from_coeffs :131-149), the slot-order invariants asserted at compile time in
params.rs:298-312 and ring.rs:101-109, the lift semantics (binfield.rs:126-154)
and the scalar commitment loop (key.rs:382-474) against a direct numpy
restatement.  Also the C ABI's host-only F162 generator."""
import numpy as np
import pytest

import oracle
from oracle import lb

SPLIT, QUAD = oracle.LB_PRIMES_SPLIT, oracle.LB_PRIMES_QUAD
T = lb.tables()


@pytest.mark.parametrize("q", SPLIT)
def test_split_transform_is_evaluation_and_multiplies(q):
    rng = np.random.default_rng(q)
    a = rng.integers(0, q, 648, dtype=np.uint32)
    b = rng.integers(0, q, 648, dtype=np.uint32)
    t = lb.ntt(q, a)
    for j in range(0, 648, 5):
        assert t[j] == lb.eval_at(q, a, int(T["slot_exp"][j]))
    prod = (t.astype(np.uint64) * lb.ntt(q, b) % q).astype(np.uint32)
    assert np.array_equal(prod, lb.ntt(q, lb.mul_mod_phi(q, a, b)))


@pytest.mark.parametrize("q", QUAD)
def test_quadratic_transform_is_leaf_reduction_and_multiplies(q):
    rng = np.random.default_rng(q)
    a = rng.integers(0, q, 648, dtype=np.uint32)
    b = rng.integers(0, q, 648, dtype=np.uint32)
    t = lb.ntt(q, a)
    for j in range(0, 324, 3):
        assert (int(t[2 * j]), int(t[2 * j + 1])) == lb.eval_quad_at(q, a, int(T["quad_slot_exp"][j]))
    assert np.array_equal(lb.mul_quad_slots(q, t, lb.ntt(q, b)), lb.ntt(q, lb.mul_mod_phi(q, a, b)))


def test_schoolbook_uses_the_cyclotomic_relation():
    q = 3889
    x = np.zeros(648, np.uint32)
    x[1] = 1
    x647 = np.zeros(648, np.uint32)
    x647[647] = 1
    prod = lb.mul_mod_phi(q, x, x647)  # X^648 = X^324 - 1
    want = np.zeros(648, np.uint32)
    want[0], want[324] = q - 1, 1
    assert np.array_equal(prod, want)


@pytest.mark.parametrize("q", SPLIT + QUAD)
def test_components_are_r162_evaluations(q):
    rng = np.random.default_rng(q + 1)
    c = rng.integers(0, q, 648, dtype=np.uint32)
    comps = lb.components(q, lb.ntt(q, c))
    if q in SPLIT:
        for k in range(4):
            assert np.array_equal(comps[k], lb.r162_from_coeffs(q, c[k::4].astype(np.int64)))
    else:
        theta = pow(lb.psi(q), 2, q)  # c^2 = theta^v for both leaves of class v
        for k in range(4):
            ck = [int(x) for x in c[k::4]]
            for s in range(0, 162, 7):
                x = pow(theta, int(T["pow3_slot_exp"][s]), q)
                val = sum(cc * pow(x, i, q) for i, cc in enumerate(ck)) % q
                assert comps[k][s] == (val - q if val > (q - 1) // 2 else val)


def test_slot_order_invariants():
    qse = T["quad_slot_exp"].astype(int)
    assert all(u % 2 == 1 and u % 3 != 0 for u in qse) and len(set(qse.tolist())) == 324
    se = T["slot_exp"].astype(int)
    assert sorted(se.tolist()) == sorted(u for u in range(1944) if u % 2 and u % 3)
    p3 = T["pow3_slot_exp"].astype(int)
    assert len(set(p3.tolist())) == 162
    for t in range(4):
        for s in range(162):
            assert se[T["slot_648"][t][s]] == p3[s] + 486 * t
    for s in range(162):
        assert qse[T["quad_class_slot"][0][s]] == p3[s] and qse[T["quad_class_slot"][1][s]] == p3[s] + 486
    for q in SPLIT + QUAD:
        assert lb.quadratic(q) == (q in QUAD)


def test_lift_interleaves_bits():
    elems = lb.random_elems(8, 5)
    for r in range(2):
        c = lb.lift(elems, r)
        for m in range(162):
            for k in range(4):
                e = elems[4 * r + k]
                assert c[4 * m + k] == (int(e[m >> 6]) >> (m & 63)) & 1
    assert all(int(e[2]) < (1 << 34) for e in elems)


def test_random_elems_matches_the_abi_generator():
    from lzx_b200 import labinius
    assert np.array_equal(labinius.random_witness(100, 0xABC), lb.random_elems(100, 0xABC))


def test_commit_loop_matches_direct_restatement():
    primes = [3889, 2917]
    len_f162, r = 16, 2
    a = lb.key_random(len_f162, 11, primes)
    half = [(q - 1) // 2 for q in primes]
    assert all(np.abs(a[k]).max() <= half[k] for k in range(2))
    w = lb.random_elems(r * len_f162, 3)
    raw, mat, bat = lb.commit(a, primes, len_f162, w, r)
    nr = len_f162 // 4
    for k, q in enumerate(primes):
        for c in range(r):
            y = np.zeros(648, dtype=object)
            for i in range(nr):
                t = lb.ntt(q, lb.lift(w[c * len_f162:], i))
                if k == 0:
                    assert np.array_equal(bat[c * nr + i], t)
                acoef = (a[k, i].astype(np.int64) % q).astype(np.uint32)
                if lb.quadratic(q):
                    y += lb.mul_quad_slots(q, acoef, t).astype(object)
                else:
                    y += acoef.astype(object) * t.astype(object)
            yc = np.array([int(v) % q for v in y], dtype=np.uint32)
            assert np.array_equal(raw[k, c], yc)
            comps = lb.components(q, yc)
            for row in range(4):
                assert np.array_equal(mat[row, c, k], comps[row])
