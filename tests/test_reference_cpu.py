"""Parity with the reference's own CPU path (compiled unmodified under vmpi).

* the product's per-virtual-rank geometry equals every rank's engine fields
  of the real reference engine (src/ca3dmm.c:146-356, :468-642);
* the reference computes the same C (sanity of the reference build);
* the vmpi harness reports a dead rank by timeout instead of hanging.
"""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc

pytestmark = pytest.mark.skipif(orc.ref_lib() is None, reason="reference CPU path not built")

CASES = [  # m, n, k, p, ta, tb, grid
    (200, 150, 300, 6, 0, 0, None),
    (150, 200, 300, 6, 1, 0, None),
    (301, 77, 129, 8, 0, 1, None),
    (96, 96, 2000, 8, 1, 1, None),
    (240, 240, 240, 12, 0, 0, (2, 2, 3)),
    (64, 300, 90, 10, 0, 0, None),     # idle ranks
]


@pytest.mark.parametrize("m,n,k,p,ta,tb,grid", CASES)
def test_engine_geometry_equals_reference(m, n, k, p, ta, tb, grid):
    A = orc.gen_uniform(1, *((k, m) if ta else (m, k)))
    B = orc.gen_uniform(2, *((n, k) if tb else (k, n)))
    Cref, _, geom, gout = orc.ref_ca3dmm(p, m, n, k, ta, tb, A, B, grid=grid)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid, caller_workbuf=True)
    assert e.ok
    assert (e.s.mp, e.s.np, e.s.kp, e.s.rp) == gout
    for r in range(p):
        assert e.vrank_info(r) == list(geom[r]), r
    want = (A.T if ta else A) @ (B.T if tb else B)
    assert np.max(np.abs(Cref - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


def test_btb_geometry_equals_reference():
    n, k, p = 64, 3000, 8
    Bm = orc.gen_btb(3, k, n)
    Cref, _, geom, gout = orc.ref_ca3dmm(p, n, n, k, 0, 0, None, Bm, btb=True)
    e = cb.Ca3dmmEngine(n, n, k, p=p, btb=True, caller_workbuf=True)
    assert (e.s.mp, e.s.np, e.s.kp, e.s.rp) == gout
    for r in range(p):
        assert e.vrank_info(r) == list(geom[r]), r
    assert np.max(np.abs(Cref - Bm.T @ Bm)) <= 1e-12 * np.max(np.abs(Bm.T @ Bm))


def test_dead_rank_is_reported_not_hung():
    import time
    t0 = time.time()
    assert orc.ref_fault_run(4, 2, 64, 1.0) != 0
    assert time.time() - t0 < 30
