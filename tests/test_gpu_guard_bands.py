"""Guard bands of the engine's work buffer (CA3DMM_CANARY=1).

The work buffer holds the plan, the packed operands, slab buffers, C and the
split-precision regions back to back; 256-byte bands filled with 0xA5 sit
between them and are checked on the device after every exec.  Every GEMM
mode and layout below must leave them intact (no kernel writes outside its
region), and a byte written into a band -- what a kernel overrunning its
region would do -- must be reported as CA3DMM_ECANARY."""
import ctypes as C

import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu


def _engine(m, n, k, ta, tb, p, grid, mode, arg, btb=False):
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid, btb=btb)
    assert e.ok
    if mode != cb.GEMM_PLAIN:
        assert e.set_gemm_mode(mode, arg) == 0
    return e


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid,mode,arg", [
    (600, 500, 700, 0, 0, 4, None, cb.GEMM_PLAIN, 0),
    (301, 257, 900, 1, 1, 12, (2, 2, 3), cb.GEMM_PLAIN, 0),        # packed, k sub-slabs, slab sum
    (600, 500, 700, 1, 0, 6, None, cb.GEMM_OZAKI, 7),
    (2100, 1700, 900, 0, 0, 24, (4, 2, 3), cb.GEMM_OZAKI, 7),      # slabs chained in the GEMM
    (600, 500, 700, 0, 1, 4, None, cb.GEMM_CRT, 15),
    (1100, 1300, 1200, 1, 0, 24, (4, 2, 3), cb.GEMM_CRT, 0),
])
def test_bands_intact_in_every_mode(cuda, monkeypatch, m, n, k, ta, tb, p, grid, mode, arg):
    monkeypatch.setenv("CA3DMM_CANARY", "1")
    A = orc.gen_signed_exp(3, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(4, *((n, k) if tb else (k, n)))
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = _engine(m, n, k, ta, tb, p, grid, mode, arg)
    for _ in range(2):
        assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    offs = (C.c_longlong * 8)()
    assert cb.lib().ca3dmm_engine_guard_bands(e.e, offs, 8) == 7
    assert all(offs[i] % 256 == 0 and offs[i + 1] > offs[i] for i in range(6))
    e.free()


@pytest.mark.parametrize("mode,arg", [(cb.GEMM_OZAKI, 7), (cb.GEMM_CRT, 16), (cb.GEMM_PLAIN, 0)])
def test_bands_btb(cuda, monkeypatch, mode, arg):
    monkeypatch.setenv("CA3DMM_CANARY", "1")
    n, k = 300, 20000
    Bm = orc.gen_btb(9, k, n)
    dB, ldb = to_dev(Bm)
    dC = dev_zeros(n * n)
    e = _engine(n, n, k, 0, 0, 8, (1, 1, 8), mode, arg, btb=True)
    assert e.exec(None, 0, dB, ldb, dC, n) == 0
    e.free()


def test_overwritten_band_is_reported(cuda, monkeypatch):
    monkeypatch.setenv("CA3DMM_CANARY", "1")
    m, n, k = 400, 300, 500
    A = orc.gen_signed_exp(5, m, k)
    B = orc.gen_signed_exp(6, k, n)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = _engine(m, n, k, 0, 0, 4, None, cb.GEMM_CRT, 15)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    want = from_dev(dC, m, n)
    offs = (C.c_longlong * 8)()
    nb = cb.lib().ca3dmm_engine_guard_bands(e.e, offs, 8)
    wb = e.s.workbuf_d
    for band in (0, 3, nb - 1):
        # one byte inside the band, as a kernel writing past its region would
        cb.lib().dev_type_memset(C.c_void_p(wb + offs[band] + 17), 0, 1, cb.DEV_TYPE_CUDA)
        assert e.exec(dA, lda, dB, ldb, dC, m) == cb.ECANARY
        # a new plan upload refills the bands; the result is unchanged
        assert e.set_gemm_mode(cb.GEMM_CRT, 15) == 0
        assert e.exec(dA, lda, dB, ldb, dC, m) == 0
        assert np.array_equal(from_dev(dC, m, n), want)
    e.free()


def test_bands_unchecked_without_the_variable(cuda, monkeypatch):
    monkeypatch.delenv("CA3DMM_CANARY", raising=False)
    m, n, k = 200, 200, 200
    A = orc.gen_signed_exp(7, m, k)
    B = orc.gen_signed_exp(8, k, n)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = _engine(m, n, k, 0, 0, 1, None, cb.GEMM_PLAIN, 0)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    offs = (C.c_longlong * 8)()
    cb.lib().ca3dmm_engine_guard_bands(e.e, offs, 8)
    cb.lib().dev_type_memset(C.c_void_p(e.s.workbuf_d + offs[0]), 0, 1, cb.DEV_TYPE_CUDA)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0       # the check is opt-in
    e.free()
