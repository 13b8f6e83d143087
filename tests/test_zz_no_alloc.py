"""The allocation-free k-slab GEMM entry point (ca3dmm_dgemm_kslab_noalloc).

It exists for callers that may not allocate device memory themselves -- code
inside a process whose device memory is owned by another allocator (a serving
framework's pool, a memory-capped MPS client), or code that must not meet an
allocation failure half-way through a job -- and keeps its partial slabs in a
fixed device array of the library instead.  This file is collected last on
purpose.  It checks, through the C ABI, that two calls in a row agree with
the double-double truth within k u |A||B| (the tolerance the other GPU tests
use) and with the existing engine entry point (ca3dmm_engine_exec on a
1 x 1 x kp grid), and that oversized problems and slab starts the TMA cannot
reach are refused.
"""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu
U = 2.0 ** -53


def _engine_result(A, B, m, n, k, kp):
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, 0, 0, p=kp, proc_grid=(1, 1, kp))
    assert e.ok and (e.s.mp, e.s.np, e.s.kp) == (1, 1, kp)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    out = from_dev(dC, m, n)
    e.free()
    return out


@pytest.mark.parametrize("m,n,k,kp", [(300, 200, 1000, 4), (257, 129, 640, 1), (96, 500, 2000, 8)])
def test_noalloc_matches_engine_two_calls(cuda, m, n, k, kp):
    L = cb.lib()
    A = orc.gen_signed_exp(41, m, k)
    B = orc.gen_signed_exp(42, k, n)
    want = _engine_result(A, B, m, n, k, kp)
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    assert np.max(np.abs((want - hi) - lo) / ab) <= k * U
    dA, lda = to_dev(A, pad_ld=m + (m % 2))
    dB, ldb = to_dev(B, pad_ld=k + (k % 2))
    for call in range(2):
        dC = dev_zeros(m * n)
        rc = L.ca3dmm_dgemm_kslab_noalloc(m, n, k, kp, dA.data_ptr(), lda, dB.data_ptr(), ldb,
                                          dC.data_ptr(), m, None)
        assert rc == 0, (call, rc)
        got = from_dev(dC, m, n)
        # against the double-double truth hi + lo, and against the engine
        assert np.max(np.abs((got - hi) - lo) / ab) <= k * U, call
        assert np.max(np.abs(got - want) / ab) <= 2 * k * U, call


def test_noalloc_rejects_oversized_and_misaligned(cuda):
    L = cb.lib()
    cap = L.ca3dmm_dgemm_kslab_noalloc_scratch_bytes()
    assert cap == 32 << 20
    m = n = 2048                      # 2 slabs of 2048 x 2048 doubles = 64 MiB > 32 MiB
    dA = dev_zeros(m * 64)
    dB = dev_zeros(64 * n)
    dC = dev_zeros(m * n)
    assert L.ca3dmm_dgemm_kslab_noalloc(m, n, 64, 2, dA.data_ptr(), m, dB.data_ptr(), 64,
                                        dC.data_ptr(), m, None) == 1
    # odd leading dimension of B violates the TMA rule: refused, nothing runs
    assert L.ca3dmm_dgemm_kslab_noalloc(64, 64, 63, 1, dA.data_ptr(), 64, dB.data_ptr(), 63,
                                        dC.data_ptr(), 64, None) == 1


def test_noalloc_rejects_odd_slab_start(cuda):
    """k = 6 on kp = 2 slabs puts slab 1 at k0 = 3: the TMA base B + 3 is not
    16-byte aligned, so the call is refused before anything runs."""
    L = cb.lib()
    dA = dev_zeros(64 * 8)            # room for k = 8 (the second call)
    dB = dev_zeros(8 * 64)
    dC = dev_zeros(64 * 64)
    assert L.ca3dmm_dgemm_kslab_noalloc(64, 64, 6, 2, dA.data_ptr(), 64, dB.data_ptr(), 6,
                                        dC.data_ptr(), 64, None) == 1
    # k = 8 on the same two slabs (k0 = 4) runs
    assert L.ca3dmm_dgemm_kslab_noalloc(64, 64, 8, 2, dA.data_ptr(), 64, dB.data_ptr(), 8,
                                        dC.data_ptr(), 64, None) == 0
