"""CPU models of the limb folds and residue steps of the tensor-core and CRT kernels.

The tensor-core witness transforms (lzx_b200/csrc/tc_commit.cu ``tn_fold``,
lzx_b200/csrc/batch.cu ``tw_fold_gl``) turn eight signed limb sums D_l into
one 64-bit value congruent to sum_l 2^(8l) D_l mod p (p = 2^64 - 2^32 + 1),
not necessarily canonical: S = A + hi(B) (2^32 - 1) with A, B the sums of
limbs 0-3 and 4-7, R = (S + 2^32 lo(B)) mod 2^64 and the result
R + k (2^32 - 1), k = carry - [S < 0].  This restates those steps in 64-bit
wrapping arithmetic and checks, on random and extreme limb sets, that the
result is congruent mod p and inside [0, 2^64) for |D_l| < 2^23 (the largest
limb sums the d = 256 batch transforms form).  The GPU suites check the
kernels themselves against the oracle.
"""
import numpy as np

P = (1 << 64) - (1 << 32) + 1
EPS = (1 << 32) - 1
M64 = (1 << 64) - 1


def fold(d):
    """The device steps on Python ints, wrapping like the 64-bit registers."""
    a = d[0] + 256 * d[1] + 65536 * d[2] + 16777216 * d[3]
    b = d[4] + 256 * d[5] + 65536 * d[6] + 16777216 * d[7]
    s = a + (b >> 32) * EPS  # int64, |s| < 2^49
    lo = (b & 0xFFFFFFFF) << 32
    r = ((s & M64) + lo) & M64
    k = int(r < lo) - int(s < 0)
    out = (r + k * EPS) & M64
    assert out == r + k * EPS, "the correction never wraps"
    return out


def test_fold_is_congruent_and_in_range():
    rng = np.random.default_rng(7)
    lim = (1 << 23) - 1
    cases = [[0] * 8, [lim] * 8, [-lim] * 8, [lim, -lim] * 4, [-lim, lim] * 4,
             [0, 0, 0, 0, -lim, -lim, -lim, -lim], [lim, lim, lim, lim, -lim, 0, 0, 0]]
    cases += rng.integers(-lim, lim + 1, size=(20000, 8)).tolist()
    cases += (rng.choice([-lim, -1, 0, 1, lim], size=(5000, 8))).tolist()
    for d in cases:
        d = [int(x) for x in d]
        got = fold(d)
        want = sum(x << (8 * l) for l, x in enumerate(d)) % P
        assert 0 <= got <= M64
        assert got % P == want, d


def test_crt_residue_step_needs_one_correction():
    """The CRT residues of z (lzx_b200/csrc/pipeline.cu ``crt_residues_kernel``
    and ``crt_ntt_kernel``): t = x - floor(x mu / 2^64) q with
    mu = floor((2^64 - 1) / q) stays below 2q for every 64-bit x (the
    quotient estimate is short by at most one, since
    x/q - x mu/2^64 = x (1 + (2^64 - 1) mod q) / (q 2^64) < 1), so one
    conditional subtraction gives x mod q; checked on random values, on
    multiples of q and their neighbours up to 2^64 - 1."""
    rng = np.random.default_rng(11)
    for q in (1073738753, 1073732609, 1073731073, 1073726977, 3 * (1 << 30) + 1, 2013265921, 12289):
        mu = M64 // q
        xs = [int(x) for x in rng.integers(0, 1 << 63, size=2000, dtype=np.int64)] + [M64, P - 1, 0, 1]
        top = M64 // q
        xs += [k * q + d for k in range(top - 500, top + 1) for d in (0, 1, q - 1) if k * q + d <= M64]
        for x in xs:
            t = x - ((x * mu) >> 64) * q
            assert 0 <= t < 2 * q
            assert (t - q if t >= q else t) == x % q


def test_crt_lane_fold_matches_modulo():
    """The uneven batch's tensor-core fold for 30-bit lanes
    (lzx_b200/csrc/batch.cu ``tw_fold``, admitted by ``tw_fold_exact``):
    v = sum_l 2^(8l) D_l plus the offset q 2^19, two folds by 2^30 == c
    (q = 2^30 - c) in the 64- and 32-bit widths the kernel uses, and one
    min(y, y - q), equal v mod q for the CRT primes at d = 128 and 256 on
    random and extreme limb sums (|D_l| <= d 128 255)."""
    rng = np.random.default_rng(13)
    mask30, m32 = (1 << 30) - 1, (1 << 32) - 1
    for q in (1073738753, 1073732609, 1073731073, 1073726977):
        c, off = (1 << 30) - q, q << 19
        for d in (128, 256):
            lim = d * 128 * 255
            vmax = d * 128 * 255 * 16843009
            assert off > vmax and c <= (1 << 20)  # what tw_fold_exact requires
            cases = [[lim] * 4, [-lim] * 4, [0] * 4, [lim, -lim, lim, -lim], [-lim, 0, 0, lim]]
            cases += rng.integers(-lim, lim + 1, size=(3000, 4)).tolist()
            for x in cases:
                v = off + x[0] + 256 * x[1] + 65536 * x[2] + 16777216 * x[3]
                assert 0 < v < (1 << 63)
                u = v
                w = (u >> 30) * c + (u & mask30)
                assert (u >> 30) < (1 << 32) and w < (1 << 64)
                y = ((w >> 30) * c + (w & mask30))
                assert y <= m32 and y < 2 * q  # the 32-bit sum does not wrap
                got = min(y, (y - q) & m32)
                assert got == (x[0] + 256 * x[1] + 65536 * x[2] + 16777216 * x[3]) % q
