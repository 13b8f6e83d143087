"""Seeded random sweep of the engine over small shapes: virtual grids (given or
the reference's own choice), transposes, padded and odd leading dimensions,
the three GEMM modes and B^T B with and without the symmetric option.  Split
precision must equal the oracle's slab-by-slab restatement bit for bit; plain
FP64 must stay within k u |op(A)||op(B)| of the double-double truth."""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu
U = 2.0 ** -53


def _oracle_split(A, B, ta, tb, m, n, k, kp, s):
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


def _cases(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m, n, k = (int(x) for x in np.exp(rng.uniform(np.log(3), np.log(700), 3)).round())
        p = int(rng.choice([1, 2, 3, 4, 6, 8, 12, 16]))
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        pad_a, pad_b = int(rng.integers(0, 3)), int(rng.integers(0, 3))
        mode = int(rng.integers(0, 2))
        s = int(rng.integers(5, 9))
        out.append((i, m, n, k, p, ta, tb, pad_a, pad_b, mode, s))
    return out


@pytest.mark.parametrize("i,m,n,k,p,ta,tb,pad_a,pad_b,mode,s", _cases(2024, 40))
def test_engine_random(cuda, i, m, n, k, p, ta, tb, pad_a, pad_b, mode, s):
    A = orc.gen_signed_exp(300 + i, *((k, m) if ta else (m, k)), emin=-6, emax=6)
    B = orc.gen_signed_exp(600 + i, *((n, k) if tb else (k, n)), emin=-6, emax=6)
    dA, lda = to_dev(A, pad_ld=A.shape[0] + pad_a)
    dB, ldb = to_dev(B, pad_ld=B.shape[0] + pad_b)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p)
    assert e.ok
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, s) == 0
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    got = from_dev(dC, m, n)
    if mode == cb.GEMM_OZAKI:
        assert np.array_equal(got, _oracle_split(A, B, ta, tb, m, n, k, e.s.kp, s))
    else:
        hi, lo, ab = orc.dd_gemm(A, B, ta, tb, m, n, k)
        err = orc.errors(got.ravel(order="F"), hi.ravel(order="F"), lo.ravel(order="F"),
                         ab.ravel(order="F"))
        assert err["vs_absprod"] <= max(k, 1) * U, err


def _btb_cases(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(3), np.log(400))).round())
        k = int(np.exp(rng.uniform(np.log(50), np.log(20000))).round())
        p = int(rng.choice([1, 2, 4, 8, 16]))
        out.append((i, n, k, p, int(rng.integers(0, 2)), int(rng.integers(0, 2)),
                    int(rng.integers(5, 9))))
    return out


@pytest.mark.parametrize("i,n,k,p,sym,mode,s", _btb_cases(77, 16))
def test_btb_random(cuda, monkeypatch, i, n, k, p, sym, mode, s):
    monkeypatch.setenv("CA3DMM_BTB_SYMMETRIC", str(sym))
    Bm = orc.gen_btb(900 + i, k, n)
    dB, ldb = to_dev(Bm)
    dC = dev_zeros(n * n)
    e = cb.Ca3dmmEngine(n, n, k, p=p, btb=True)
    assert e.ok
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, s) == 0
    assert e.exec(None, 0, dB, ldb, dC, n) == 0
    got = from_dev(dC, n, n)
    if sym:
        assert np.array_equal(got, got.T)
    if mode == cb.GEMM_OZAKI:
        assert np.array_equal(got, _oracle_split(Bm, Bm, 1, 0, n, n, k, e.s.kp, s))
    else:
        hi, lo, ab = orc.dd_gemm(Bm, Bm, 1, 0, n, n, k)
        err = orc.errors(got.ravel(order="F"), hi.ravel(order="F"), lo.ravel(order="F"),
                         ab.ravel(order="F"))
        assert err["vs_absprod"] <= k * U, err


def _crt_cases(seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        m, n, k = (int(x) for x in np.exp(rng.uniform(np.log(3), np.log(1500), 3)).round())
        p = int(rng.choice([1, 2, 3, 4, 6, 8, 12, 16]))
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        pad_a, pad_b = int(rng.integers(0, 3)), int(rng.integers(0, 3))
        nmod = int(rng.choice([0, 8, 11, 14, 15, 16, 18]))
        tile = int(rng.choice([128, 256]))
        band = int(rng.choice([1, 2, 8, 32]))
        overlap = int(rng.integers(0, 2))
        out.append((i, m, n, k, p, ta, tb, pad_a, pad_b, nmod, tile, band, overlap))
    return out


@pytest.mark.parametrize("i,m,n,k,p,ta,tb,pad_a,pad_b,nmod,tile,band,overlap",
                         _crt_cases(4242, 32))
def test_engine_random_modular(cuda, monkeypatch, i, m, n, k, p, ta, tb, pad_a, pad_b, nmod,
                               tile, band, overlap):
    """The modular mode over random shapes, grids, padded leading dimensions,
    modulus counts, tile widths, work-order bands and with or without the
    reconstruction beside the GEMM: bit-exact against the oracle's 128-bit
    integer product (one k slab: k < 131072, whatever the grid)."""
    monkeypatch.setenv("CA3DMM_CRT_OVERLAP", str(overlap))
    A = orc.gen_signed_exp(1300 + i, *((k, m) if ta else (m, k)), emin=-6, emax=6)
    B = orc.gen_signed_exp(1600 + i, *((n, k) if tb else (k, n)), emin=-6, emax=6)
    dA, lda = to_dev(A, pad_ld=A.shape[0] + pad_a)
    dB, ldb = to_dev(B, pad_ld=B.shape[0] + pad_b)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p)
    assert e.ok
    assert e.set_tune((cb.GEMM_CRT, nmod, 1, band, tile)) == 0
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    got = from_dev(dC, m, n)
    nm = e.s.crt_moduli
    assert nmod == 0 or nm == nmod
    P = orc.crt_bits(nm, k)
    want = orc.crt_gemm(np.asfortranarray(A.T if ta else A), np.asfortranarray(B.T if tb else B),
                        0, 0, m, n, k, P)
    assert np.array_equal(got, want), np.max(np.abs(got - want))
    e.free()
