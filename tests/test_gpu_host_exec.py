"""ca3dmm_engine_exec_host: host buffers in and out, the copies pipelined
with the computation in bands of output rows.  The result must equal the
device-pointer exec bit for bit (same kernels, same reduction order), in both
GEMM modes, with pinned and pageable host memory."""
import numpy as np
import pytest
import torch

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu


def _pinned(x):
    t = torch.from_numpy(np.asfortranarray(x).ravel(order="F").copy()).pin_memory()
    return t, x.shape[0]


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid", [
    (4100, 300, 900, 0, 0, 24, (4, 2, 3)),      # 2 task_m blocks x 3 bands, kp = 3
    (3000, 257, 700, 1, 0, 6, None),
    (2600, 300, 500, 0, 1, 4, (2, 1, 2)),
    (1500, 1500, 64, 1, 1, 1, None),
    (2600, 300, 901, 1, 0, 8, (2, 2, 2)),       # odd ldA on the device, even in staging; odd slab start
    (4100, 2600, 300, 0, 0, 24, (4, 2, 3)),    # split mode chains the 3 slabs per tile
])
@pytest.mark.parametrize("mode,slices", [(cb.GEMM_PLAIN, 0), (cb.GEMM_OZAKI, 7)])
def test_exec_host_equals_device_exec(cuda, m, n, k, ta, tb, p, grid, mode, slices):
    A = orc.gen_signed_exp(11, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(12, *((n, k) if tb else (k, n)))
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid)
    assert e.ok
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, slices) == 0
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    want = from_dev(dC, m, n)
    hA, _ = _pinned(A)
    hB, _ = _pinned(B)
    hC = torch.zeros(m * n, dtype=torch.float64).pin_memory()
    for _ in range(2):                       # second call reuses staging and bands
        hC.zero_()
        assert e.exec_host(hA, lda, hB, ldb, hC, m) == 0
        got = hC.numpy().reshape((m, n), order="F")
        assert np.array_equal(got, want), np.max(np.abs(got - want))


def test_exec_host_pageable_and_padded_leading_dims(cuda):
    m, n, k = 2300, 200, 400
    A = orc.gen_signed_exp(21, m + 3, k)      # ldA = m + 3
    B = orc.gen_signed_exp(22, k + 1, n)      # ldB = k + 1
    e = cb.Ca3dmmEngine(m, n, k, 0, 0, p=8)
    assert e.ok and e.set_gemm_mode(cb.GEMM_OZAKI, 6) == 0
    hA = np.asfortranarray(A)
    hB = np.asfortranarray(B)
    hC = np.zeros((m + 5, n), order="F")      # ldC = m + 5
    assert e.exec_host(hA, m + 3, hB, k + 1, hC, m + 5) == 0
    dA, _ = to_dev(A)
    dB, _ = to_dev(B)
    dC = dev_zeros(m * n)
    assert e.exec(dA, m + 3, dB, k + 1, dC, m) == 0
    assert np.array_equal(hC[:m], from_dev(dC, m, n))
    assert np.all(hC[m:] == 0.0)


@pytest.mark.parametrize("n,k,grid,mode,sym", [
    (96, 5000, (1, 1, 8), cb.GEMM_OZAKI, 0),      # slab pipeline, split precision
    (96, 5000, (1, 1, 8), cb.GEMM_PLAIN, 0),      # slab pipeline, plain (k sub-slabs too)
    (300, 20000, (1, 1, 4), cb.GEMM_OZAKI, 1),    # symmetric option through the pipeline
    (300, 20000, (1, 1, 4), cb.GEMM_PLAIN, 1),
    (130, 3000, (1, 1, 1), cb.GEMM_OZAKI, 0),     # kp = 1: serial path
])
def test_exec_host_btb(cuda, monkeypatch, n, k, grid, mode, sym):
    """B^T B from host buffers: B arrives slab by slab while earlier slabs are
    sliced and multiplied; the result equals the device exec bit for bit."""
    monkeypatch.setenv("CA3DMM_BTB_SYMMETRIC", str(sym))
    Bm = orc.gen_btb(7, k, n)
    e = cb.Ca3dmmEngine(n, n, k, p=grid[2], btb=True, proc_grid=grid)
    assert e.ok
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(cb.GEMM_OZAKI, 7) == 0
    hB, ldb = _pinned(Bm)
    hC = torch.zeros(n * n, dtype=torch.float64).pin_memory()
    dB, _ = to_dev(Bm)
    dC = dev_zeros(n * n)
    assert e.exec(None, 0, dB, ldb, dC, n) == 0
    want = from_dev(dC, n, n)
    for _ in range(2):                       # the second call reuses the staging and descriptors
        hC.zero_()
        assert e.exec_host(None, 0, hB, ldb, hC, n) == 0
        assert np.array_equal(hC.numpy().reshape((n, n), order="F"), want)
