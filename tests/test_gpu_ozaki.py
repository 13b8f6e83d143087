"""Split-precision (Ozaki INT8 on tcgen05) path against the oracle.

Bit-exact: with the slices computed by the oracle's restatement of the
slicing rule, the same exact k chunks and the same FP64 recombination order,
every C entry of the device result equals the oracle's, slab by slab.
Accuracy: the error against the double-double truth shrinks by ~2^-8 per
slice; at 7 slices (55 bits) it is no worse than the plain FP64 DMMA error
on the exponent-spread inputs."""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu


def _run(A, B, m, n, k, ta, tb, p, grid, mode, slices):
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid)
    assert e.ok
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, slices) == 0
    rc = e.exec(dA, lda, dB, ldb, dC, m)
    assert rc == 0, rc
    s = e.s
    out = from_dev(dC, m, n), (s.mp, s.np, s.kp)
    e.free()
    return out


def _oracle_ozaki(A, B, m, n, k, ta, tb, kp, s):
    """Slab-by-slab oracle: slices over each slab's k range, recombination,
    then the slab sum in slab order (src/ca3dmm.c:1287-1343)."""
    opA = A.T if ta else A
    opB = B.T if tb else B
    out = None
    for sl in range(kp):
        k0, kz = orc.block_spos_size(k, kp, sl)
        a = np.asfortranarray(opA[:, k0:k0 + kz])
        b = np.asfortranarray(opB[k0:k0 + kz, :])
        qa, ea = orc.ozaki_slices_rows(a, 0, m, kz, s)
        qb, eb = orc.ozaki_slices_cols(b, 0, kz, n, s)
        c = orc.ozaki_gemm(qa, ea, qb, eb, m, n, kz, s)
        out = c if out is None else out + c
    return out


@pytest.mark.parametrize("m,n,k,s", [(128, 64, 64, 2), (1, 1, 1, 3), (130, 70, 100, 5),
                                     (300, 200, 777, 7), (257, 129, 1000, 8), (64, 500, 333, 4)])
def test_ozaki_bitexact_single_group(cuda, m, n, k, s):
    A = orc.gen_signed_exp(61, m, k)
    B = orc.gen_signed_exp(62, k, n)
    got, _ = _run(A, B, m, n, k, 0, 0, 1, None, cb.GEMM_OZAKI, s)
    want = _oracle_ozaki(A, B, m, n, k, 0, 0, 1, s)
    assert np.array_equal(got, want), np.max(np.abs(got - want))


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid,s", [
    (400, 300, 900, 0, 0, 6, None, 7),
    (400, 300, 900, 1, 0, 6, None, 6),
    (400, 300, 900, 0, 1, 6, None, 8),
    (333, 444, 555, 1, 1, 12, (2, 2, 3), 7),
    (64, 80, 5000, 0, 0, 8, None, 8),
])
def test_ozaki_bitexact_virtual_grid(cuda, m, n, k, ta, tb, p, grid, s):
    A = orc.gen_signed_exp(71, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(72, *((n, k) if tb else (k, n)))
    got, (mp, np_, kp) = _run(A, B, m, n, k, ta, tb, p, grid, cb.GEMM_OZAKI, s)
    want = _oracle_ozaki(A, B, m, n, k, ta, tb, kp, s)
    assert np.array_equal(got, want), np.max(np.abs(got - want))


def test_ozaki_error_shrinks_with_slices_and_matches_plain(cuda):
    m = n = k = 768
    A = orc.gen_signed_exp(81, m, k)
    B = orc.gen_signed_exp(82, k, n)
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    errs = {}
    for s in (3, 4, 5, 6, 7, 8):
        got, _ = _run(A, B, m, n, k, 0, 0, 4, None, cb.GEMM_OZAKI, s)
        errs[s] = orc.errors(got.ravel(order="F"), hi.ravel(order="F"), lo.ravel(order="F"),
                             ab.ravel(order="F"))["normwise"]
    plain, _ = _run(A, B, m, n, k, 0, 0, 4, None, cb.GEMM_PLAIN, 0)
    e_plain = orc.errors(plain.ravel(order="F"), hi.ravel(order="F"), lo.ravel(order="F"),
                         ab.ravel(order="F"))["normwise"]
    for s in (3, 4, 5, 6, 7):
        assert errs[s + 1] < errs[s] or errs[s + 1] <= e_plain, errs
    assert errs[7] <= e_plain, (errs, e_plain)
    assert errs[8] <= e_plain, (errs, e_plain)


def test_ozaki_chained_slabs_bitexact(cuda):
    """A C large enough that each output tile runs its kp slabs in one CTA and
    adds them into C in slab order (no slab buffers): still bit-exact."""
    m, n, k = 3200, 3000, 400
    A = orc.gen_signed_exp(111, m, k)
    B = orc.gen_signed_exp(112, k, n)
    got, (mp, np_, kp) = _run(A, B, m, n, k, 0, 0, 6, (2, 1, 3), cb.GEMM_OZAKI, 7)
    assert kp == 3
    assert np.array_equal(got, _oracle_ozaki(A, B, m, n, k, 0, 0, kp, 7))


@pytest.mark.parametrize("s", [5, 8])
def test_ozaki_k_chunks_bitexact(cuda, s):
    """k longer than one exact INT32 chunk: chunked recombination matches."""
    kc = orc.ozaki_kchunk(s)
    m, n, k = 130, 70, 2 * kc + 77
    A = orc.gen_signed_exp(101, m, k)
    B = orc.gen_signed_exp(102, k, n)
    got, _ = _run(A, B, m, n, k, 0, 0, 1, None, cb.GEMM_OZAKI, s)
    assert np.array_equal(got, _oracle_ozaki(A, B, m, n, k, 0, 0, 1, s))


@pytest.mark.parametrize("n,k,p,grid,s", [
    (96, 4000, 8, (1, 1, 8), 8),
    (100, 3000, 8, (1, 1, 8), 7),     # 128-row A tiles over 64-row B tiles: padded half
    (50, 2000, 4, (1, 1, 4), 6),      # fewer rows than one B tile
    (200, 1500, 8, None, 7),          # the reference's default B^T B grid (fold)
    (130, 1000, 16, (2, 2, 4), 5),
    (64, 70000, 4, (1, 1, 4), 7),     # columns of B more than 512 KB apart
])
def test_ozaki_btb(cuda, n, k, p, grid, s):
    """B^T B: the op(A) = B^T blocks reuse the slices of the B blocks."""
    Bm = orc.gen_btb(5, k, n)
    dB, ldb = to_dev(Bm)
    dC = dev_zeros(n * n)
    e = cb.Ca3dmmEngine(n, n, k, p=p, btb=True, proc_grid=grid)
    assert e.ok and e.set_gemm_mode(cb.GEMM_OZAKI, s) == 0
    assert e.exec(None, 0, dB, ldb, dC, n) == 0
    got = from_dev(dC, n, n)
    want = _oracle_ozaki(Bm, Bm, n, n, k, 1, 0, e.s.kp, s)
    assert np.array_equal(got, want)


def test_ozaki_zero_rows_and_columns(cuda):
    m, n, k = 200, 150, 300
    A = orc.gen_signed_exp(91, m, k)
    B = orc.gen_signed_exp(92, k, n)
    A[17, :] = 0.0
    B[:, 33] = 0.0
    got, _ = _run(A, B, m, n, k, 0, 0, 1, None, cb.GEMM_OZAKI, 6)
    assert np.all(got[17, :] == 0.0) and np.all(got[:, 33] == 0.0)
    assert np.array_equal(got, _oracle_ozaki(A, B, m, n, k, 0, 0, 1, 6))
