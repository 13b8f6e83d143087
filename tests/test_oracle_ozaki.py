"""The oracle's split-precision restatement, checked on the CPU.

* Non-finite rule: a row / column holding an Inf or a NaN is sliced as a
  zero row, and orc_nonfinite_fixup gives every C entry in it the value BLAS
  gives (numpy's A @ B through OpenBLAS): NaN, +Inf or -Inf.
* Accuracy of the recombination: with 7 slices on exponent-spread inputs the
  restated product is within k u |A||B| of the double-double truth, also when
  a row is subnormal or its exponent sits at the other end of the range from
  the column's (the power of two 2^(E_i + F_j) is applied once, at the end).
"""
import numpy as np
import pytest

from oracle import oracle as orc

U = 2.0 ** -53


def _split(A, B, s=7):
    m, k = A.shape
    n = B.shape[1]
    qa, ea = orc.ozaki_slices_rows(np.asfortranarray(A), 0, m, k, s)
    qb, eb = orc.ozaki_slices_cols(np.asfortranarray(B), 0, k, n, s)
    return orc.ozaki_gemm(qa, ea, qb, eb, m, n, k, s)


def _classes(C):
    return np.where(np.isnan(C), 3, np.where(np.isposinf(C), 1, np.where(np.isneginf(C), 2, 0)))


@pytest.mark.parametrize("seed", range(6))
def test_nonfinite_rule_matches_blas(seed):
    rng = np.random.default_rng(seed)
    m, n, k = (int(x) for x in rng.integers(5, 60, 3))
    A = orc.gen_signed_exp(seed + 1, m, k)
    B = orc.gen_signed_exp(seed + 2, k, n)
    for X in (A, B):
        for val in (np.nan, np.inf, -np.inf, np.inf):
            X[rng.integers(X.shape[0]), rng.integers(X.shape[1])] = val
        X[rng.integers(X.shape[0]), :] = 0.0
    qa, ea = orc.ozaki_slices_rows(np.asfortranarray(A), 0, m, k, 7)
    bad_rows = ~np.all(np.isfinite(A), axis=1)
    assert np.all(ea[bad_rows] == 0) and np.all(qa[:, bad_rows, :] == 0)
    C = orc.nonfinite_fixup(A, B, 0, 0, m, n, k, np.asfortranarray(_split(A, B)))
    with np.errstate(invalid="ignore", over="ignore"):
        ref = A @ B
    assert np.array_equal(_classes(C), _classes(ref))
    fin = np.all(np.isfinite(A), axis=1)[:, None] & np.all(np.isfinite(B), axis=0)[None, :]
    Af = np.where(np.isfinite(A), A, 0.0)
    Bf = np.where(np.isfinite(B), B, 0.0)
    assert np.array_equal(C[fin], _split(Af, Bf)[fin])


def test_recombination_extreme_exponents():
    m, n, k = 40, 30, 200
    A = orc.gen_signed_exp(3, m, k)
    B = orc.gen_signed_exp(4, k, n)
    A[0, :] *= 2.0 ** -1060
    A[1, :] *= 2.0 ** -1000
    B[:, 0] *= 2.0 ** 1000
    B[:, 1] *= 2.0 ** -950
    C = _split(A, B)
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    err = np.abs((C - hi) - lo)
    assert np.all(err <= k * U * ab + (4 * k + 64) * 2.0 ** -1074)
    for i, j in ((0, 0), (1, 0)):
        assert abs(C[i, j] - hi[i, j]) <= k * U * ab[i, j]


@pytest.mark.parametrize("nmod,seed", [(8, 0), (12, 1), (15, 2), (16, 3), (18, 4)])
def test_crt_modular_route_equals_exact_integers(nmod, seed):
    """The modular restatement (residues of a', b' in [-128, 127], INT32 dot
    products reduced mod p_t, Garner reconstruction) gives exactly the
    integer product the scheme's result is rounded from."""
    rng = np.random.default_rng(seed)
    m, n = (int(x) for x in rng.integers(3, 12, 2))
    k = int(rng.integers(1, 400))
    A = orc.gen_signed_exp(seed + 7, m, k)
    B = orc.gen_signed_exp(seed + 8, k, n)
    P = orc.crt_bits(nmod, k)
    assert P >= 2
    exact = orc.crt_exact_ints(A, B, 0, 0, m, n, k, P)
    modular = orc.crt_modular_ints(A, B, 0, 0, m, n, k, P, nmod)
    assert modular is not None and (exact == modular).all()
    assert max(abs(int(x)) for x in exact.ravel()) <= k * 2 ** (2 * P)


def test_crt_bits_rule():
    """P is the largest width <= 53 with k 2^(2P+1) < prod p_t."""
    import math
    for nmod in (8, 12, 15, 16, 18):
        lm = sum(math.log2(orc.crt_modulus(t)) for t in range(nmod))
        for k in (1, 100, 2667, 8000, 32768, 131072):
            P = orc.crt_bits(nmod, k)
            assert P <= 53
            assert math.log2(k) + 2 * P + 1 < lm
            if P < 53:
                assert math.log2(k) + 2 * (P + 1) + 1 >= lm - 1e-9
    assert [orc.crt_modulus(t) for t in range(4)] == [256, 255, 253, 251]
    assert orc.crt_bits(15, 8000) == 51 and orc.crt_bits(16, 32768) == 53
