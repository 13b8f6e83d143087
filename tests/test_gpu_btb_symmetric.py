"""B^T B with CA3DMM_BTB_SYMMETRIC=1: only the upper block triangle of C is
computed (one group per 128-row block row and slab) and the strictly lower
triangle is mirrored from it.  Split precision: the same bits as computing the
whole C (the slice products of (i, j) and (j, i) are the same integers and the
scalings differ by exact powers of two).  Plain FP64: within k u |B^T||B| of the
double-double truth and exactly symmetric."""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu
U = 2.0 ** -53

CASES = [(130, 1000, 4, (1, 1, 4)), (300, 2000, 8, (1, 1, 8)), (96, 4000, 8, None),
         (513, 700, 2, (1, 1, 2)), (40, 900, 1, None)]


def _run(Bm, n, k, p, grid, mode, sym, monkeypatch, dst=None):
    monkeypatch.setenv("CA3DMM_BTB_SYMMETRIC", "1" if sym else "0")
    dB, ldb = to_dev(Bm)
    kw = {} if dst is None else {"dst_C": dst}
    e = cb.Ca3dmmEngine(n, n, k, p=p, btb=True, proc_grid=grid, **kw)
    assert e.ok and e.s.btb_symmetric == (1 if sym else 0)
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, 7) == 0
    rows = n if dst is None else dst[1]
    cols = n if dst is None else dst[3]
    dC = dev_zeros(rows * cols)
    assert e.exec(None, 0, dB, ldb, dC, rows) == 0
    out = from_dev(dC, rows, cols)
    e.free()
    return out


@pytest.mark.parametrize("n,k,p,grid", CASES)
def test_symmetric_split_equals_full(cuda, monkeypatch, n, k, p, grid):
    Bm = orc.gen_btb(21, k, n)
    full = _run(Bm, n, k, p, grid, cb.GEMM_OZAKI, False, monkeypatch)
    sym = _run(Bm, n, k, p, grid, cb.GEMM_OZAKI, True, monkeypatch)
    assert np.array_equal(sym, full)
    assert np.array_equal(sym, sym.T)


@pytest.mark.parametrize("n,k,p,grid", CASES)
def test_symmetric_plain_within_tolerance(cuda, monkeypatch, n, k, p, grid):
    Bm = orc.gen_btb(22, k, n)
    got = _run(Bm, n, k, p, grid, cb.GEMM_PLAIN, True, monkeypatch)
    assert np.array_equal(got, got.T)
    hi, lo, ab = orc.dd_gemm(Bm, Bm, 1, 0, n, n, k)
    err = orc.errors(got.ravel(order="F"), hi.ravel(order="F"), lo.ravel(order="F"),
                     ab.ravel(order="F"))
    assert err["vs_absprod"] <= k * U, err


def test_symmetric_dst_block(cuda, monkeypatch):
    """A dst_C block that is not the whole C: mirrored in the engine's C_out, then copied."""
    n, k = 260, 1500
    Bm = orc.gen_btb(23, k, n)
    full = _run(Bm, n, k, 4, (1, 1, 4), cb.GEMM_OZAKI, False, monkeypatch)
    part = _run(Bm, n, k, 4, (1, 1, 4), cb.GEMM_OZAKI, True, monkeypatch, dst=(30, 200, 10, 150))
    assert np.array_equal(part, full[30:230, 10:160])
