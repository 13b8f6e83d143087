"""Non-finite and subnormal inputs.

The reference's local GEMM is BLAS / cuBLAS DGEMM (src/cannon.c:410-418,
src/cuda_proxy.cu:211-230), which carries NaN and Inf through by IEEE rules.
Both GEMM modes must do the same: every C entry's class (NaN, +Inf, -Inf or
finite) equals numpy's A @ B (BLAS) on the same operands.  In split precision
a row of op(A) or a column of op(B) holding an Inf or a NaN is sliced as a
zero row and its C entries get their IEEE value afterwards, so the finite
entries stay bit-exact against the oracle's slab-by-slab restatement.
Subnormal rows and rows whose exponents sit at opposite ends of the range are
checked against the double-double truth, with the underflow allowance of
gradual underflow (a few units of 2^-1074 per accumulation step).
"""
import numpy as np
import pytest
import torch

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu
U = 2.0 ** -53
ETA = 2.0 ** -1074


def _classes(C):
    return np.where(np.isnan(C), 3, np.where(np.isposinf(C), 1, np.where(np.isneginf(C), 2, 0)))


def _plant(X, seed, nnan=2, npinf=2, nninf=2, zero_lines=True):
    """Plant NaN, +Inf and -Inf at seeded positions of X (and some zeros, so
    that Inf * 0 products occur)."""
    rng = np.random.default_rng(seed)
    X = X.copy()
    r, c = X.shape
    for val, cnt in ((np.nan, nnan), (np.inf, npinf), (-np.inf, nninf)):
        for _ in range(cnt):
            X[rng.integers(r), rng.integers(c)] = val
    if zero_lines:
        X[rng.integers(r), :] = 0.0
        X[:, rng.integers(c)] = 0.0
    return X


def _ref_classes(A, B, ta, tb):
    with np.errstate(invalid="ignore", over="ignore"):
        return _classes((A.T if ta else A) @ (B.T if tb else B))


def _oracle_split(A, B, m, n, k, ta, tb, kp, s):
    """Slab by slab (the oracle's slicing of each slab's k range, zero rows for
    non-finite ones), slab sum in slab order, then the IEEE values of the
    entries in non-finite rows and columns over all of k."""
    opA = np.asfortranarray(A.T if ta else A)
    opB = np.asfortranarray(B.T if tb else B)
    out = None
    for sl in range(kp):
        k0, kz = orc.block_spos_size(k, kp, sl)
        a = np.asfortranarray(opA[:, k0:k0 + kz])
        b = np.asfortranarray(opB[k0:k0 + kz, :])
        qa, ea = orc.ozaki_slices_rows(a, 0, m, kz, s)
        qb, eb = orc.ozaki_slices_cols(b, 0, kz, n, s)
        c = orc.ozaki_gemm(qa, ea, qb, eb, m, n, kz, s)
        out = c if out is None else out + c
    return orc.nonfinite_fixup(opA, opB, 0, 0, m, n, k, np.asfortranarray(out))


def _engine(A, B, m, n, k, ta, tb, p, grid, mode, slices=7):
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid)
    assert e.ok
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, slices) == 0
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    kp = e.s.kp
    got = from_dev(dC, m, n)
    e.free()
    return got, kp


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid", [
    (300, 200, 700, 0, 0, 1, None),
    (400, 300, 900, 1, 0, 6, None),
    (333, 444, 555, 1, 1, 12, (2, 2, 3)),       # kp = 3, chained slab sums
    (257, 129, 1000, 0, 1, 24, (4, 2, 3)),
    (64, 80, 5000, 0, 0, 8, None),              # k-dominant grid
])
@pytest.mark.parametrize("mode", [cb.GEMM_OZAKI, cb.GEMM_PLAIN])
def test_nonfinite_classes_and_finite_entries(cuda, m, n, k, ta, tb, p, grid, mode):
    A = _plant(orc.gen_signed_exp(91, *((k, m) if ta else (m, k))), 1)
    B = _plant(orc.gen_signed_exp(92, *((n, k) if tb else (k, n))), 2)
    got, kp = _engine(A, B, m, n, k, ta, tb, p, grid, mode)
    ref = _ref_classes(A, B, ta, tb)
    assert np.array_equal(_classes(got), ref)
    assert np.any(ref == 3) and np.any(ref == 1) and np.any(ref == 2) and np.any(ref == 0)
    fin = ref == 0
    if mode == cb.GEMM_OZAKI:
        want = _oracle_split(A, B, m, n, k, ta, tb, kp, 7)
        assert np.array_equal(_classes(want), ref)
        assert np.array_equal(got[fin], want[fin])
    else:
        Af = np.where(np.isfinite(A), A, 0.0)
        Bf = np.where(np.isfinite(B), B, 0.0)
        hi, lo, ab = orc.dd_gemm(Af, Bf, ta, tb, m, n, k)
        err = np.abs((got - hi) - lo)[fin] / np.maximum(ab[fin], 1e-300)
        assert np.max(err) <= k * U


def test_nonfinite_infinities_only(cuda):
    """Only infinities: +Inf * +x and -Inf * -x give +Inf, mixed signs in one
    dot product NaN, Inf * 0 NaN; no NaN in the inputs."""
    m, n, k = 200, 130, 300
    A = orc.gen_signed_exp(5, m, k)
    B = orc.gen_signed_exp(6, k, n)
    A[3, 10] = np.inf
    A[7, 11] = -np.inf
    A[7, 12] = np.inf                    # row 7: both signs -> NaN where B rows 11, 12 agree in sign
    B[20, 4] = -np.inf
    B[50, :] = 0.0
    A[9, 50] = np.inf                    # Inf * 0 on every column -> row 9 NaN
    for mode in (cb.GEMM_OZAKI, cb.GEMM_PLAIN):
        got, kp = _engine(A, B, m, n, k, 0, 0, 4, None, mode)
        ref = _ref_classes(A, B, 0, 0)
        assert not np.any(np.isnan(A)) and not np.any(np.isnan(B))
        assert np.array_equal(_classes(got), ref), mode
        if mode == cb.GEMM_OZAKI:
            want = _oracle_split(A, B, m, n, k, 0, 0, kp, 7)
            fin = ref == 0
            assert np.array_equal(got[fin], want[fin])


def test_nonfinite_btb(cuda):
    n, k = 130, 4000
    Bm = orc.gen_btb(8, k, n)
    Bm[17, 5] = np.nan
    Bm[300, 40] = np.inf
    Bm[301, 41] = -np.inf
    dB, ldb = to_dev(Bm)
    for mode in (cb.GEMM_OZAKI, cb.GEMM_PLAIN):
        e = cb.Ca3dmmEngine(n, n, k, p=8, btb=True, proc_grid=(1, 1, 8))
        assert e.ok
        if mode == cb.GEMM_OZAKI:
            assert e.set_gemm_mode(cb.GEMM_OZAKI, 7) == 0
        dC = dev_zeros(n * n)
        assert e.exec(None, 0, dB, ldb, dC, n) == 0
        kp = e.s.kp
        e.free()
        got = from_dev(dC, n, n)
        ref = _ref_classes(Bm, Bm, 1, 0)
        assert np.array_equal(_classes(got), ref), mode
        if mode == cb.GEMM_OZAKI:
            want = _oracle_split(Bm, Bm, n, n, k, 1, 0, kp, 7)
            fin = ref == 0
            assert np.array_equal(got[fin], want[fin])


def test_nonfinite_grouped(cuda):
    rng = np.random.default_rng(3)
    probs = []
    for i in range(12):
        m, n, k = (int(x) for x in rng.integers(20, 400, 3))
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        A = orc.gen_signed_exp(300 + i, *((k, m) if ta else (m, k)))
        B = orc.gen_signed_exp(400 + i, *((n, k) if tb else (k, n)))
        if i % 3 == 0:
            A = _plant(A, 10 + i, 1, 1, 1, zero_lines=False)
        if i % 4 == 1:
            B = _plant(B, 20 + i, 1, 1, 1)
        probs.append((m, n, k, ta, tb, A, B))
    for mode, slices in ((cb.GEMM_OZAKI, 7), (cb.GEMM_PLAIN, 0)):
        g = cb.GroupedGemm([p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                           [p[3] for p in probs], [p[4] for p in probs], mode=mode, slices=slices)
        assert g.ok
        dA, dB, dC, lda, ldb, ldc = [], [], [], [], [], []
        for m, n, k, ta, tb, A, B in probs:
            a, la = to_dev(A)
            b, lb = to_dev(B)
            dA.append(a); lda.append(la); dB.append(b); ldb.append(lb)
            dC.append(dev_zeros(m * n)); ldc.append(m)
        assert g.exec(dA, lda, dB, ldb, dC, ldc) == 0
        for i, (m, n, k, ta, tb, A, B) in enumerate(probs):
            got = from_dev(dC[i], m, n)
            ref = _ref_classes(A, B, ta, tb)
            assert np.array_equal(_classes(got), ref), (mode, i)
            if mode == cb.GEMM_OZAKI:
                want = _oracle_split(A, B, m, n, k, ta, tb, 1, 7)
                fin = ref == 0
                assert np.array_equal(got[fin], want[fin]), i


@pytest.mark.parametrize("mode", [cb.GEMM_OZAKI, cb.GEMM_PLAIN])
def test_nonfinite_exec_host(cuda, mode):
    """Host buffers, copies pipelined in row bands: the same bits as the
    device exec, non-finite entries included."""
    m, n, k = 4100, 300, 900
    A = _plant(orc.gen_signed_exp(11, m, k), 4)
    B = _plant(orc.gen_signed_exp(12, k, n), 5)
    e = cb.Ca3dmmEngine(m, n, k, 0, 0, p=24, proc_grid=(4, 2, 3))
    assert e.ok
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, 7) == 0
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    want = from_dev(dC, m, n)
    assert np.array_equal(_classes(want), _ref_classes(A, B, 0, 0))
    hA = torch.from_numpy(A.ravel(order="F").copy()).pin_memory()
    hB = torch.from_numpy(B.ravel(order="F").copy()).pin_memory()
    hC = torch.zeros(m * n, dtype=torch.float64).pin_memory()
    assert e.exec_host(hA, lda, hB, ldb, hC, m) == 0
    got = hC.numpy().reshape((m, n), order="F")
    assert np.array_equal(got, want, equal_nan=True)


@pytest.mark.parametrize("mode", [cb.GEMM_OZAKI, cb.GEMM_PLAIN])
def test_subnormal_and_extreme_exponent_rows(cuda, mode):
    """Row 0 of A is subnormal (2^-1060 scale), row 1 tiny (2^-1000); column 0
    of B is huge (2^+1000), column 1 tiny (2^-950).  Row 0 or 1 times column 0
    is a normal-range product although one factor's exponent is extreme; row 0
    against the ordinary columns gives subnormal results, rows 0 and 1 against
    column 1 underflow to zero.  Checked against the double-double truth with
    k u |A||B| plus the gradual-underflow allowance, relative accuracy where
    the result is normal, and bit for bit against the oracle (split mode)."""
    m, n, k = 140, 90, 600
    A = orc.gen_signed_exp(31, m, k)
    B = orc.gen_signed_exp(32, k, n)
    A[0, :] *= 2.0 ** -1060
    A[1, :] *= 2.0 ** -1000
    B[:, 0] *= 2.0 ** 1000
    B[:, 1] *= 2.0 ** -950
    got, kp = _engine(A, B, m, n, k, 0, 0, 4, None, mode)
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    err = np.abs((got - hi) - lo)
    bound = k * U * ab + (4 * k + 64) * ETA
    assert np.all(err <= bound), np.max(err / bound)
    for i, j in ((0, 0), (1, 0), (5, 0), (5, 1)):
        assert abs(got[i, j]) > 2.0 ** -1022
        assert abs(got[i, j] - hi[i, j]) <= k * U * ab[i, j], (i, j)
    assert 0 < np.max(np.abs(got[0, 2:])) < 2.0 ** -1022       # subnormal results
    if mode == cb.GEMM_OZAKI:
        want = _oracle_split(A, B, m, n, k, 0, 0, kp, 7)
        assert np.array_equal(got, want)
