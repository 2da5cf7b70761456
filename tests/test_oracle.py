"""The CPU oracle against the reference's own KATs, golden vectors and identity tests.

Each test names the reference test (idrees2516/lzx, file:line) that it re-runs
against the C restatement in ``oracle/``.
"""
import numpy as np
import pytest

import oracle
from oracle import GL_P

Q32 = oracle.Modulus32(*oracle.Q_32)
MODS = [oracle.Modulus32(*oracle.Q_32), oracle.Modulus32(*oracle.Q_12289),
        oracle.Modulus32(*oracle.Q_2013265921)] + [oracle.Modulus32(*c) for c in oracle.CRT_PRIMES]


def xorshift(state):
    """xorshift64* as in lattice-ring/src/modulus.rs:186-192."""
    M = (1 << 64) - 1
    while True:
        state ^= state >> 12
        state ^= (state << 25) & M
        state ^= state >> 27
        yield (state * 0x2545F4914F6CDD1D) & M


# ------------------------------------------------------------- reference KATs

def test_goldilocks_reference_kats(ref_kats):
    """field.rs:267-313 python_cross_validated_kats."""
    L = oracle.lib()
    for a, b, e in ref_kats["goldilocks"]["sub"]:
        assert L.orc_gl_sub(a, b) == e
    for a, b, e in ref_kats["goldilocks"]["add"]:
        assert L.orc_gl_add(a, b) == e
    for a, b, e in ref_kats["goldilocks"]["mul"]:
        assert L.orc_gl_mul(a, b) == e
    assert len(ref_kats["goldilocks"]["sub"]) == 6 and len(ref_kats["goldilocks"]["mul"]) == 4


def test_keccak_reference_kats(ref_kats):
    """keccak.rs:415-448 FIPS-202 digests."""
    for c in ref_kats["keccak"]["cases"]:
        msg = bytes.fromhex(c["msg_hex"])
        if c["fn"] == "sha3_256":
            assert oracle.sha3_256(msg).hex() == c["digest_hex"]
        else:
            assert oracle.shake256(msg, c["out_len"]).hex() == c["digest_hex"]
    # keccak.rs:444-446 prefix consistency
    assert oracle.shake256(b"hello", 64)[:32] == oracle.shake256(b"hello", 32)


def test_keccak_matches_hashlib():
    import hashlib
    for n in (0, 1, 135, 136, 137, 271, 272, 1000):
        msg = bytes((i * 7 + 3) & 0xFF for i in range(n))
        assert oracle.sha3_256(msg) == hashlib.sha3_256(msg).digest()
        assert oracle.shake256(msg, 300) == hashlib.shake_256(msg).digest(300)


def test_modulus_constants_match_reference(ref_kats):
    m = ref_kats["modulus32"]
    assert (m["Q_32"]["q"], m["Q_32"]["two_adicity"], m["Q_32"]["generator"]) == oracle.Q_32
    assert (m["Q_12289"]["q"], m["Q_12289"]["two_adicity"], m["Q_12289"]["generator"]) == oracle.Q_12289


# ------------------------------------------------------------- Modulus32 tests

def test_barrett_matches_division_random():
    """modulus.rs:180-223 (200k xorshift u64s + boundary shapes per prime)."""
    for m in MODS[:3] + MODS[3:4]:
        q = m.q
        gen = xorshift(0x243F6A8885A308D3)
        cases = [next(gen) for _ in range(200_000)]
        for k in range(1, 64):
            cases += [(1 << k) - 1, 1 << k, (1 << k) + 1]
        M = (1 << 64) - 1
        for k in range(1, 1000):
            cases += [(k * q) & M, (k * q - 1) & M, (k * q + 1) & M]
        cases += [M, M - 1, (q - 1) * (q - 1)]
        for x in cases:
            assert m.reduce_u64(x) == x % q


def test_barrett_all_products_and_corners():
    """modulus.rs:225-251."""
    q = Q32.q
    gen = xorshift(0x9E3779B97F4A7C15)
    for _ in range(100_000):
        a, b = next(gen) % q, next(gen) % q
        assert Q32.mul(a, b) == a * b % q
    for a in (0, 1, 2, q - 2, q - 1):
        for b in (0, 1, 2, q - 2, q - 1):
            assert Q32.mul(a, b) == a * b % q
    x = q - 1
    assert Q32.add(x, 2) == 1 and Q32.sub(1, 2) == q - 1 and Q32.neg(x) == 1


def test_inverse_and_negative_values():
    """modulus.rs:253-265."""
    for a in (1, 2, 12345, Q32.q - 1):
        assert Q32.mul(a, Q32.inv(a)) == 1
    assert Q32.inv(0) is None
    assert Q32.reduce_i64(-1) == Q32.q - 1
    assert Q32.reduce_i64(-Q32.q) == 0
    assert Q32.reduce_i64(-(Q32.q - 5)) == 5


def test_root_orders_and_reciprocal():
    """modulus.rs:267-290, extended to the CRT primes and their generators."""
    for m in MODS:
        for k in range(1, min(m.two_adicity, 12) + 1):
            w = m.root_of_unity(k)
            assert m.pow(w, 1 << k) == 1 and m.pow(w, 1 << (k - 1)) != 1
        assert m.root_of_unity(m.two_adicity + 1) is None
        assert m.barrett_recip == ((1 << 64) - 1) // m.q
        assert m.q * m.barrett_recip < 1 << 64 < m.q * (m.barrett_recip + 1) + 1


def test_crt_primes_are_the_four_largest():
    """Config: the four largest 30-bit primes q == 1 (mod 512), exact adicity."""
    def is_prime(n):
        if n < 2:
            return False
        for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
            if n % p == 0:
                return n == p
        d, s = n - 1, 0
        while d % 2 == 0:
            d //= 2
            s += 1
        for a in (2, 3, 5, 7, 11, 13, 17):
            x = pow(a, d, n)
            if x in (1, n - 1):
                continue
            for _ in range(s - 1):
                x = x * x % n
                if x == n - 1:
                    break
            else:
                return False
        return True
    found = []
    q = (1 << 30) - 1
    q -= (q - 1) % 512
    while len(found) < 4:
        if is_prime(q):
            found.append(q)
        q -= 512
    assert tuple(found) == tuple(c[0] for c in oracle.CRT_PRIMES)
    for q, adic, g in oracle.CRT_PRIMES:
        assert ((q - 1) >> adic) & 1 == 1 and (q - 1) % (1 << adic) == 0
        # g generates the full 2-Sylow part: g^((q-1)/2) == -1
        assert pow(g, (q - 1) // 2, q) == q - 1


# ------------------------------------------------------------- NTT

def test_ntt_golden_q32_kat_manifest(golden):
    """kat_manifest.rs:62-102 vectors (digests re-derived through the oracle's SHA3)."""
    for v in golden["ntt_q32_kat_manifest"]:
        t = oracle.NttTables32(Q32, v["log_n"])
        a = np.array(v["input"], dtype=np.uint32)
        f = t.forward_fast(a)
        assert f.tolist() == v["forward"]
        assert oracle.hash_domain(b"kat-ntt-fwd", f.astype("<u4").tobytes()).hex() == v["digest_forward"]
        r = t.inverse_fast(f)
        assert oracle.hash_domain(b"kat-ntt-inv", r.astype("<u4").tobytes()).hex() == v["digest_roundtrip"]
    for v in golden["ntt_q32_extra"]:
        t = oracle.NttTables32(Q32, v["log_n"])
        assert t.forward_fast(np.array(v["input"], dtype=np.uint32)).tolist() == v["forward"]


def test_ntt_golden_crt_and_goldilocks(golden):
    for v in golden["ntt_crt"]:
        t = oracle.NttTables32(oracle.Modulus32(v["q"], v["two_adicity"], v["generator"]), v["log_n"])
        a = np.array(v["input"], dtype=np.uint32)
        assert t.forward_batch(a).tolist() == v["forward"]
        assert (t.inverse_batch(t.forward_batch(a)) == a).all()
    for v in golden["ntt_goldilocks"]:
        t = oracle.NttTablesGl(v["log_n"])
        a = np.array([int(x) for x in v["input"]], dtype=np.uint64)
        f = t.forward_batch(a)
        assert [str(x) for x in f.tolist()] == v["forward"]
        assert (t.inverse_batch(f) == a).all()


@pytest.mark.parametrize("log_n", [1, 2, 3, 4, 5, 6, 8])
def test_ntt_fast_matches_generic_and_roundtrip(log_n):
    """ntt.rs:364-380 and ntt.rs:439-467."""
    t = oracle.NttTables32(Q32, log_n)
    a = oracle.ring_random(Q32, log_n, b"fast-a")
    g = t.forward(a)
    f = t.forward_fast(a)
    assert (g == f).all()
    assert (t.inverse_fast(f) == a).all()
    assert (t.inverse(g) == t.inverse_fast(g)).all()


def test_ntt_natural_order_direct_evaluation():
    """forward output j is a(psi^(2j+1)) -- the order the reference code produces."""
    for m, log_n in ((Q32, 5), (oracle.Modulus32(*oracle.CRT_PRIMES[2]), 4)):
        q = m.q
        n = 1 << log_n
        psi = m.root_of_unity(log_n + 1)
        a = oracle.ring_random(m, log_n, b"eval").astype(object) % q
        f = oracle.NttTables32(m, log_n).forward_fast(oracle.ring_random(m, log_n, b"eval"))
        for j in range(n):
            x = pow(psi, 2 * j + 1, q)
            assert int(f[j]) == sum(int(c) * pow(x, i, q) for i, c in enumerate(a)) % q
    n = 16
    t = oracle.NttTablesGl(4)
    a = oracle.synth_gl(1, 2, n)
    f = t.forward_fast(a)
    psi = pow(7, (GL_P - 1) >> 5, GL_P)
    for j in range(n):
        x = pow(psi, 2 * j + 1, GL_P)
        assert int(f[j]) == sum(int(c) * pow(x, i, GL_P) for i, c in enumerate(a)) % GL_P


def test_ntt_mul_matches_schoolbook():
    """ntt.rs:382-415 and neo.rs:138-158 (Goldilocks schoolbook)."""
    log_n = 5
    t = oracle.NttTables32(Q32, log_n)
    a = oracle.ring_random(Q32, log_n, b"sb-a")
    b = oracle.ring_random(Q32, log_n, b"sb-b")
    n, q = 1 << log_n, Q32.q
    school = [0] * n
    for i in range(n):
        for j in range(n):
            v = int(a[i]) * int(b[j]) % q
            if i + j < n:
                school[i + j] = (school[i + j] + v) % q
            else:
                school[i + j - n] = (school[i + j - n] - v) % q
    assert t.ring_mul(a, b).tolist() == school
    tg = oracle.NttTablesGl(6)
    x, y = oracle.synth_gl(3, 1, 64), oracle.synth_gl(3, 2, 64)
    prod = tg.inverse_fast(np.array([oracle.lib().orc_gl_mul(int(u), int(v)) for u, v in
                                     zip(tg.forward_fast(x), tg.forward_fast(y))], dtype=np.uint64))
    assert (prod == oracle.neo_mul(x, y)).all()


def test_partial_then_complete_equals_full():
    """ntt.rs:417-437."""
    t = oracle.NttTables32(Q32, 5)
    a = oracle.ring_random(Q32, 5, b"pc-a")
    full = t.forward(a)
    for levels in range(6):
        p = t.forward_partial(a, levels)
        assert (t.complete_partial(p, levels) == full).all()


def test_rejects_bad_geometry():
    """ntt.rs:469-479."""
    m = oracle.Modulus32(*oracle.Q_12289)
    oracle.NttTables32(m, 11)
    with pytest.raises(oracle.NttError) as e:
        oracle.NttTables32(m, 12)
    assert str(e.value) == "AdicityTooSmall"
    t = oracle.NttTables32(m, 8)
    with pytest.raises(oracle.NttError) as e:
        t.forward(np.zeros(128, dtype=np.uint32))
    assert str(e.value) == "LengthMismatch"


# ------------------------------------------------------------- seeded keys and commits

def test_uniform_from_seed_golden(golden):
    """ring.rs:102-180 vs the counter-loop shapes of uniform_check.rs:95-137."""
    for v in golden["uniform_from_seed_q32"]:
        got = oracle.uniform_from_seed(Q32, v["log_n"], b"ajtai-A", bytes.fromhex(v["seed_hex"]),
                                       v["index"])
        assert got.tolist() == v["coeffs"]


def test_ajtai_kat_manifest_commitments(golden):
    """kat_manifest.rs:128-155: from_seed + sample_small_secret + commit."""
    for v in golden["ajtai_q32_kat_manifest"]:
        t = oracle.NttTables32(Q32, v["log_n"])
        mat, mat_ntt = oracle.ajtai32_from_seed(t, v["k"], v["m"], bytes.fromhex(v["seed_hex"]))
        assert mat[: t.n].tolist() == v["matrix_row0"]
        s = oracle.sample_small_secret(Q32, v["log_n"], v["m"], 1 << 12, b"kat-secret")
        assert s.reshape(v["m"], -1).tolist() == v["secret"]
        rows = oracle.ajtai32_commit(t, mat_ntt, v["k"], v["m"], s)
        assert rows.tolist() == v["rows"]
        assert oracle.hash_domain(b"kat-ajtai", rows.astype("<u4").tobytes()).hex() == v["digest"]


@pytest.mark.parametrize("log_n,k,m,bound", [(4, 2, 3, 255), (5, 2, 8, 8), (6, 3, 12, 3), (6, 1, 16, 1)])
def test_cached_ntt_matches_naive(log_n, k, m, bound):
    """ajtai.rs:489-506 cached-NTT commit == naive per-product commit."""
    t = oracle.NttTables32(Q32, log_n)
    mat, mat_ntt = oracle.ajtai32_from_seed(t, k, m, bytes([9]) * 32)
    s = oracle.sample_small_secret(Q32, log_n, m, bound, b"diff")
    assert (oracle.ajtai32_commit(t, mat_ntt, k, m, s) ==
            oracle.ajtai32_commit_naive(t, mat, k, m, s)).all()


def test_linearity_and_zero_skip():
    """ajtai.rs:467-487 linearity; ajtai.rs:547-570 zero witnesses commit to zero."""
    t = oracle.NttTables32(Q32, 4)
    k, m, q = 2, 3, Q32.q
    _, mat_ntt = oracle.ajtai32_from_seed(t, k, m, bytes([6]) * 32)
    s1 = oracle.sample_small_secret(Q32, 4, m, 8, b"a")
    s2 = oracle.sample_small_secret(Q32, 4, m, 8, b"b")
    ssum = ((s1.astype(np.uint64) + s2) % q).astype(np.uint32)
    t1 = oracle.ajtai32_commit(t, mat_ntt, k, m, s1).astype(np.uint64)
    t2 = oracle.ajtai32_commit(t, mat_ntt, k, m, s2).astype(np.uint64)
    assert (((t1 + t2) % q) == oracle.ajtai32_commit(t, mat_ntt, k, m, ssum)).all()
    z = np.zeros(m * 16, dtype=np.uint32)
    assert not oracle.ajtai32_commit(t, mat_ntt, k, m, z).any()


def test_goldilocks_commit_golden(golden):
    """Cached-NTT commit over Goldilocks == the coefficient-domain (neo.rs) values."""
    v = golden["ajtai_goldilocks_small"]
    d, kappa, m, B = v["d"], v["kappa"], v["m"], v["batch"]
    A = oracle.synth_gl(v["a_seed"], v["a_stream"], kappa * m * d)
    W = oracle.synth_i8(v["w_seed"], v["w_stream"], B * m * d)
    t = oracle.NttTablesGl(6)
    A_ntt = t.forward_batch(A)
    for simd in (False, True):
        out = oracle.ajtaigl_commit_batch(t, A_ntt, kappa, m, W.reshape(B, m, d), simd=simd)
        assert [[[str(x) for x in r] for r in o] for o in out.tolist()] == v["out"]
    Wf = np.where(W < 0, np.uint64(GL_P) - np.abs(W.astype(np.int64)).astype(np.uint64),
                  W.astype(np.uint64))
    for b in range(B):
        naive = oracle.neo_commit_naive(d, kappa, m, A, Wf[b * m * d:(b + 1) * m * d])
        ppb, _ = oracle.neo_commit_pay_per_bit(d, kappa, m, A, Wf[b * m * d:(b + 1) * m * d])
        assert [[str(x) for x in r] for r in naive.tolist()] == v["out"][b]
        assert (ppb == naive).all()


def test_neo_pay_per_bit_cost_profile():
    """neo.rs:986-1041: binary witnesses pay a fraction of wide ones; values agree."""
    d, kappa, m = 8, 2, 64
    A = oracle.synth_gl(4, 4, kappa * m * d)
    bits = np.array([(i % 3 == 0) for i in range(m)], dtype=np.uint64)
    cols_bits = oracle.decomp_b(bits, 1)[:d].T.copy()
    wide = np.array([(i * 0x9E3779B97F4A7C15) % (1 << 64) for i in range(m)], dtype=np.uint64)
    cols_wide = oracle.decomp_b(wide, 8).T.copy()
    cb, adds_bits = oracle.neo_commit_pay_per_bit(d, kappa, m, A, cols_bits)
    cw, adds_wide = oracle.neo_commit_pay_per_bit(d, kappa, m, A, cols_wide)
    assert adds_wide > 4 * adds_bits
    assert (cb == oracle.neo_commit_naive(d, kappa, m, A, cols_bits)).all()
    assert (cw == oracle.neo_commit_naive(d, kappa, m, A, cols_wide)).all()


def test_decomposition(golden):
    """decomp_b (neo.rs:253-266, test neo.rs:969-979) and the balanced gadget (decomposition.rs:48-70)."""
    v = golden["decomp_b8"]
    z = np.array([int(x) for x in v["z"]], dtype=np.uint64)
    rows = oracle.decomp_b(z, 8)
    assert [[str(x) for x in r] for r in rows.tolist()] == v["rows"]
    for x in (0, 1, 127, 128, 129, 255, 256, (1 << 64) - 1, GL_P - 1, 0xDEADBEEFCAFEF00D):
        digits = oracle.gadget_decompose(256, 9, x)
        assert all(-128 <= int(dd) <= 128 for dd in digits)
        assert sum(int(dd) * 256 ** i for i, dd in enumerate(digits)) == x
    with pytest.raises(ValueError):
        oracle.gadget_decompose(256, 2, 1 << 20)


def test_synthetic_generator_golden(golden):
    s = golden["synth"]
    for seed, stream, idx, val in s["u64"]:
        assert oracle.synth_u64(seed, stream, idx) == int(val)
    assert oracle.synth_mod32(3, 9, oracle.CRT_PRIMES[0][0], 64).tolist() == s["mod32_q0_seed3_stream9"]
    assert [str(x) for x in oracle.synth_gl(3, 9, 64).tolist()] == s["gl_seed3_stream9"]
    assert oracle.synth_i8(3, 9, 64).tolist() == s["i8_seed3_stream9"]


def test_pack_field_elements_restatement():
    """packing.rs:30-52 restated in Python big integers against the oracle."""
    p = oracle.GL_P
    q = oracle.Q_32[0]
    vals = [0, 1, (1 << 22) - 1, 1 << 22, (1 << 44) + 5, p - 1, p + 3, (1 << 64) - 1] + list(range(7, 70, 9))
    for log_n in (1, 2, 6):
        n = 1 << log_n
        limbs = []
        for v in vals:
            raw = v % p
            limbs += [raw & ((1 << 22) - 1), (raw >> 22) & ((1 << 22) - 1), raw >> 44]
        elems = max(1, -(-len(limbs) // n))
        want = (limbs + [0] * (elems * n - len(limbs)))
        got = oracle.pack_field_elements(q, log_n, np.array(vals, dtype=np.uint64))
        assert got.reshape(-1).tolist() == [x % q for x in want]
    assert oracle.pack_field_elements(q, 6, np.zeros(0, dtype=np.uint64)).shape == (1, 64)
