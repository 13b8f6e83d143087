"""Results of the GPU engine against the reference's own CPU path on the same
inputs (the reference compiled unmodified under the thread-backed MPI subset,
DEV_TYPE_HOST): the 2048^3 example on 4 virtual ranks and a transposed,
uneven shape, in both GEMM modes, under the reference's validation rule
(componentwise relative difference <= 1e-12, examples/example_AB.c:262-304)."""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(orc.ref_lib() is None, reason="reference CPU path not built")]


@pytest.mark.parametrize("m,n,k,ta,tb,p", [(2048, 2048, 2048, 0, 0, 4), (1500, 700, 900, 1, 0, 6)])
@pytest.mark.parametrize("mode,slices", [(cb.GEMM_PLAIN, 0), (cb.GEMM_OZAKI, 7)])
def test_engine_matches_reference_cpu_path(cuda, m, n, k, ta, tb, p, mode, slices):
    A = orc.gen_uniform(1, *((k, m) if ta else (m, k)))      # uniform in [-1, 1)
    B = orc.gen_uniform(2, *((n, k) if tb else (k, n)))
    Cref, _, geom, gout = orc.ref_ca3dmm(p, m, n, k, ta, tb, A, B)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p)
    assert e.ok
    assert (e.s.mp, e.s.np, e.s.kp, e.s.rp) == gout
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, slices) == 0
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    got = from_dev(dC, m, n)
    rel = np.abs(got - Cref) / np.maximum(np.abs(Cref), 1e-300)
    # entries near zero from cancellation: relative to the row/column scale
    scale = np.abs(np.asarray(A.T if ta else A)) @ np.abs(np.asarray(B.T if tb else B))
    bad = (rel > 1e-12) & (np.abs(got - Cref) > 1e-15 * scale)
    assert not bad.any(), (int(bad.sum()), float(rel.max()))
