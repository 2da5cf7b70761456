"""CPU model of the witness-transform limb fold.

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
