"""Generate ``golden_vectors.json``: golden inputs/outputs for the hot path.

A second, independent restatement of the reference algorithms in plain Python
(big integers and ``%`` instead of Barrett/Montgomery; ``hashlib`` SHAKE256 and
SHA3-256 instead of the oracle's Keccak) so that the C oracle and the CUDA
path are both checked against vectors neither of them produced.  The sizes are
small: every vector finishes in well under a second of pure Python.

Restated reference functions (idrees2516/lzx):
  NttTables::new / forward_fast / inverse_fast   lattice-ring/src/ntt.rs:46-216
  RingConfig::uniform_from_seed                  lattice-ring/src/ring.rs:102-180
  AjtaiPublicKey::from_seed / commit             lattice-commitment/src/ajtai.rs:87-153
  sample_small_secret                            lattice-commitment/src/ajtai.rs:307-348
  Transcript::xof / hash_domain                  lattice-core/src/transcript.rs:218-237
  NeoRing::mul / NeoAjtaiKey::commit_naive       lattice-folding/src/neo.rs:138-158, 419-441
  decomp_b                                       lattice-folding/src/neo.rs:253-266
  KAT manifest NTT + commitment vectors          lattice-bench/src/bin/kat_manifest.rs:62-155

Usage: python tests/golden/make_golden.py   (writes golden_vectors.json here)
"""
from __future__ import annotations

import hashlib
import json
import os
import struct

HERE = os.path.dirname(os.path.abspath(__file__))
P = 0xFFFFFFFF00000001
M64 = (1 << 64) - 1

Q_32 = (3221225473, 30, 5)
CRT = [(1073738753, 10, 3), (1073732609, 10, 3), (1073731073, 9, 3), (1073726977, 9, 5)]


# ------------------------------------------------------------------ hashing

def _frame(tag: bytes, domain: bytes, msg: bytes) -> bytes:
    return tag + struct.pack("<I", len(domain)) + domain + struct.pack("<I", len(msg)) + msg


def xof(domain: bytes, msg: bytes, n: int) -> bytes:
    return hashlib.shake_256(_frame(b"LZXX", domain, msg)).digest(n)


def hash_domain(domain: bytes, msg: bytes) -> bytes:
    return hashlib.sha3_256(_frame(b"LZXD", domain, msg)).digest()


# ------------------------------------------------------------------ NTT

def _bitrev(a):
    n = len(a)
    bits = n.bit_length() - 1
    out = list(a)
    for i in range(n):
        j = int(format(i, f"0{bits}b")[::-1], 2) if bits else 0
        if i < j:
            out[i], out[j] = out[j], out[i]
    return out


class Ntt:
    """ntt.rs NttTables over modulus q with psi = g^((q-1)/2^(log_n+1))."""

    def __init__(self, q: int, g: int, log_n: int):
        n = 1 << log_n
        self.q, self.n, self.log_n = q, n, log_n
        psi = pow(g, (q - 1) >> (log_n + 1), q)
        psi_inv = pow(psi, q - 2, q)
        omega = psi * psi % q
        omega_inv = pow(omega, q - 2, q)
        self.n_inv = pow(n, q - 2, q)
        self.pow_psi = [pow(psi, i, q) for i in range(n)]
        self.pow_psi_inv = [pow(psi_inv, i, q) for i in range(n)]
        half = max(n // 2, 1)
        pw = [pow(omega, i, q) for i in range(half)]
        pwi = [pow(omega_inv, i, q) for i in range(half)]
        self.lv = []
        self.lvi = []
        for level in range(log_n):
            ln = 1 << (level + 1)
            stride = n // ln
            self.lv.append([pw[t * stride] for t in range(ln // 2)])
            self.lvi.append([pwi[t * stride] for t in range(ln // 2)])

    def forward(self, a):
        q, n = self.q, self.n
        a = _bitrev([x * self.pow_psi[i] % q for i, x in enumerate(a)])
        for tw in self.lv:
            sl = len(tw)
            for start in range(0, n, 2 * sl):
                for t in range(sl):
                    u = a[start + t]
                    v = a[start + t + sl] * tw[t] % q
                    a[start + t] = (u + v) % q
                    a[start + t + sl] = (u - v) % q
        return a

    def inverse(self, a):
        q, n = self.q, self.n
        a = list(a)
        for tw in reversed(self.lvi):
            sl = len(tw)
            for start in range(0, n, 2 * sl):
                for t in range(sl):
                    u = a[start + t]
                    v = a[start + t + sl]
                    a[start + t] = (u + v) % q
                    a[start + t + sl] = (u - v) * tw[t] % q
        a = _bitrev(a)
        return [x * self.pow_psi_inv[i] % q * self.n_inv % q for i, x in enumerate(a)]


def negacyclic_schoolbook(a, b, q):
    n = len(a)
    out = [0] * n
    for i in range(n):
        if a[i] == 0:
            continue
        for j in range(n):
            k = i + j
            if k < n:
                out[k] = (out[k] + a[i] * b[j]) % q
            else:
                out[k - n] = (out[k - n] - a[i] * b[j]) % q
    return out


# ------------------------------------------------------------------ seeded ring elements

def uniform_from_seed(q: int, n: int, domain: bytes, seed: bytes, index: int):
    salt = domain + seed + struct.pack("<Q", index)
    limit = (1 << 32) - ((1 << 32) % q)
    slack = max(n, 16)
    stream = xof(b"uniform", salt, 8 + 4 * (n + slack))
    coeffs = []
    w = 8
    while len(coeffs) < n and w + 4 <= len(stream):
        c = struct.unpack_from("<I", stream, w)[0]
        w += 4
        if c < limit:
            coeffs.append(c % q)
    counter = (len(stream) - 8) // 4
    while len(coeffs) < n:  # ring.rs:155-175 fallback
        b = xof(b"uniform", salt, 8 + counter * 4 + 4)
        c = struct.unpack_from("<I", b, len(b) - 4)[0]
        if c < limit:
            coeffs.append(c % q)
        counter += 1
    return coeffs


def sample_small_secret(q: int, n: int, m: int, bound: int, seed: bytes):
    span = 2 * bound + 1
    limit = (0xFFFFFFFF // span) * span
    out = []
    for i in range(m):
        coeffs = []
        sc = 0
        while len(coeffs) < n:
            inp = seed + struct.pack("<Q", i) + struct.pack("<Q", sc)
            b = xof(b"ajtai-secret", inp, max(n * 16, 64))
            for c in range(0, len(b) - 3, 4):
                if len(coeffs) == n:
                    break
                v = struct.unpack_from("<I", b, c)[0]
                if v < limit:
                    coeffs.append((v % span - bound) % q)
            sc += 1
        out.append(coeffs)
    return out


def ajtai_commit(ntt: Ntt, matrix_ntt, k, m, s):
    q, n = ntt.q, ntt.n
    s_ntt = [None if not any(sj) else ntt.forward(sj) for sj in s]
    rows = []
    for i in range(k):
        acc = [0] * n
        for j in range(m):
            if s_ntt[j] is None:
                continue
            a = matrix_ntt[i * m + j]
            acc = [(x + y * z) % q for x, y, z in zip(acc, a, s_ntt[j])]
        rows.append(ntt.inverse(acc))
    return rows


# ------------------------------------------------------------------ synthetic generator

def mix64(z):
    z ^= z >> 30
    z = z * 0xBF58476D1CE4E5B9 & M64
    z ^= z >> 27
    z = z * 0x94D049BB133111EB & M64
    z ^= z >> 31
    return z


def synth_u64(seed, stream, index):
    base = mix64((seed * 0x9E3779B97F4A7C15 + stream * 0xC2B2AE3D27D4EB4F + 0x165667B19E3779F9)
                 & M64)
    return mix64((base + index * 0x9E3779B97F4A7C15) & M64)


def synth_mod32(seed, stream, q, count, offset=0):
    limit = (1 << 32) - ((1 << 32) % q)
    out = []
    for i in range(offset, offset + count):
        r = 0
        while True:
            c = synth_u64(seed, (stream + (r << 40)) & M64, i) & 0xFFFFFFFF
            if c < limit:
                out.append(c % q)
                break
            r += 1
    return out


def synth_gl(seed, stream, count, offset=0):
    out = []
    for i in range(offset, offset + count):
        r = 0
        while True:
            c = synth_u64(seed, (stream + (r << 40)) & M64, i)
            if c < P:
                out.append(c)
                break
            r += 1
    return out


def synth_i8(seed, stream, count, offset=0):
    return [((synth_u64(seed, stream, i) & 0xFF) ^ 0x80) - 0x80 for i in range(offset, offset + count)]


# ------------------------------------------------------------------ vectors

def le32(vals):
    return b"".join(struct.pack("<I", v) for v in vals)


def main():
    g = {"generator": "tests/golden/make_golden.py (pure Python + hashlib)"}

    # KAT-manifest NTT vectors, kat_manifest.rs:62-102
    kat = []
    q, _, gen = Q_32
    for log_n in (4, 6, 8):
        n = 1 << log_n
        b = xof(b"kat-ntt", bytes([log_n]), n * 4)
        coeffs = [struct.unpack_from("<I", b, 4 * i)[0] % q for i in range(n)]
        t = Ntt(q, gen, log_n)
        fwd = t.forward(coeffs)
        inv = t.inverse(fwd)
        assert inv == coeffs
        kat.append({"log_n": log_n, "input": coeffs, "forward": fwd,
                    "digest_forward": hash_domain(b"kat-ntt-fwd", le32(fwd)).hex(),
                    "digest_roundtrip": hash_domain(b"kat-ntt-inv", le32(inv)).hex()})
    g["ntt_q32_kat_manifest"] = kat

    # Q_32 at further sizes (ntt.rs tests use log_n in {1,2,3,5,8})
    extra = []
    for log_n in (1, 2, 3, 5, 10):
        n = 1 << log_n
        t = Ntt(q, gen, log_n)
        a = synth_mod32(11, 100 + log_n, q, n)
        extra.append({"log_n": log_n, "input": a, "forward": t.forward(a)})
    g["ntt_q32_extra"] = extra

    # CRT primes, d = 256 (two polynomials each)
    crt = []
    for pi, (qq, adic, gg) in enumerate(CRT):
        t = Ntt(qq, gg, 8)
        a = synth_mod32(7, pi, qq, 512)
        fwd = t.forward(a[:256]) + t.forward(a[256:])
        crt.append({"q": qq, "two_adicity": adic, "generator": gg, "log_n": 8, "seed": 7,
                    "stream": pi, "input": a, "forward": fwd})
    # also d = 64 and 128 under the first prime
    for log_n in (6, 7, 9):
        qq, adic, gg = CRT[0]
        t = Ntt(qq, gg, log_n)
        a = synth_mod32(8, log_n, qq, 1 << log_n)
        crt.append({"q": qq, "two_adicity": adic, "generator": gg, "log_n": log_n, "seed": 8,
                    "stream": log_n, "input": a, "forward": t.forward(a)})
    g["ntt_crt"] = crt

    # Goldilocks, generator 7 (field.rs:195-200)
    gl = []
    for log_n in (6, 7, 8):
        t = Ntt(P, 7, log_n)
        a = synth_gl(5, log_n, 2 << log_n)
        n = 1 << log_n
        fwd = t.forward(a[:n]) + t.forward(a[n:])
        gl.append({"log_n": log_n, "seed": 5, "stream": log_n, "input": [str(x) for x in a],
                   "forward": [str(x) for x in fwd]})
    g["ntt_goldilocks"] = gl

    # KAT-manifest Ajtai commitments, kat_manifest.rs:128-155
    com = []
    for log_n, m in ((4, 8), (6, 8)):
        n = 1 << log_n
        t = Ntt(q, gen, log_n)
        seed = bytes([0xAB]) * 32
        mat = [uniform_from_seed(q, n, b"ajtai-A", seed, i) for i in range(2 * m)]
        mat_ntt = [t.forward(x) for x in mat]
        s = sample_small_secret(q, n, m, 1 << 12, b"kat-secret")
        rows = ajtai_commit(t, mat_ntt, 2, m, s)
        com.append({"log_n": log_n, "k": 2, "m": m, "seed_hex": seed.hex(),
                    "matrix_row0": mat[0], "secret": s, "rows": rows,
                    "digest": hash_domain(b"kat-ajtai", b"".join(le32(r) for r in rows)).hex()})
    g["ajtai_q32_kat_manifest"] = com

    # uniform_from_seed windows (ring.rs:102-180; uniform_check.rs:120-137 shapes)
    uni = []
    for log_n, idx, tag in ((3, 0, 0), (5, 7, 42), (6, 4096, 255), (6, 1 << 20, 1)):
        uni.append({"log_n": log_n, "index": idx, "seed_hex": (bytes([tag]) * 32).hex(),
                    "coeffs": uniform_from_seed(q, 1 << log_n, b"ajtai-A", bytes([tag]) * 32, idx)})
    g["uniform_from_seed_q32"] = uni

    # Goldilocks commit, d = 64: cached-NTT form == coefficient-domain (neo.rs) form
    d, kappa, m, B = 64, 2, 4, 2
    t = Ntt(P, 7, 6)
    A = [synth_gl(21, 0, d, offset=e * d) for e in range(kappa * m)]
    W = synth_i8(21, 1, B * m * d)
    outs = []
    for b in range(B):
        cols = [[(x % P) for x in W[(b * m + j) * d:(b * m + j + 1) * d]] for j in range(m)]
        rows = ajtai_commit(t, [t.forward(a) for a in A], kappa, m, cols)
        for i in range(kappa):
            acc = [0] * d
            for j in range(m):
                prod = negacyclic_schoolbook(A[i * m + j], cols[j], P)
                acc = [(x + y) % P for x, y in zip(acc, prod)]
            assert acc == rows[i], "cached-NTT commit != coefficient-domain commit"
        outs.append([[str(x) for x in r] for r in rows])
    g["ajtai_goldilocks_small"] = {"d": d, "kappa": kappa, "m": m, "batch": B, "a_seed": 21,
                                   "a_stream": 0, "w_seed": 21, "w_stream": 1, "out": outs}

    # decomp_b (neo.rs:253-266) on the neo.rs:969-979 values
    zs = [0xDEADBEEF, 12345, 0, 1 << 63, P - 1]
    g["decomp_b8"] = {"z": [str(z) for z in zs],
                      "rows": [[str((z >> (8 * r)) & 0xFF) for z in zs] for r in range(8)]}

    # the synthetic generator itself (pins C, Python and CUDA copies to one stream)
    g["synth"] = {
        "u64": [[s, st, i, str(synth_u64(s, st, i))] for s, st, i in
                ((0, 0, 0), (1, 2, 3), (7, 1 << 40, 12345), (2**64 - 1, 5, 2**33))],
        "mod32_q0_seed3_stream9": synth_mod32(3, 9, CRT[0][0], 64),
        "gl_seed3_stream9": [str(x) for x in synth_gl(3, 9, 64)],
        "i8_seed3_stream9": synth_i8(3, 9, 64),
    }

    with open(os.path.join(HERE, "golden_vectors.json"), "w") as f:
        json.dump(g, f, separators=(",", ":"))
        f.write("\n")
    print("wrote", os.path.join(HERE, "golden_vectors.json"))


if __name__ == "__main__":
    main()
