"""The bounded device wait of every kernel: a barrier nothing completes makes
the wait return an error status after its limit (no hang, no fault), and the
context stays usable for a normal exec afterwards."""
import time

import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu


def test_wait_runs_out_and_context_survives(cuda):
    t0 = time.time()
    assert cb.device_wait_check(0.2, 0) == cb.ETIMEOUT
    assert 0.15 < time.time() - t0 < 10.0
    assert cb.device_wait_check(0.2, 1) == cb.OK
    m, n, k = 300, 200, 100
    A = orc.gen_uniform(5, m, k)
    B = orc.gen_uniform(6, k, n)
    e = cb.Ca3dmmEngine(m, n, k, p=2)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    assert np.allclose(from_dev(dC, m, n), A @ B, rtol=1e-12, atol=1e-12)
