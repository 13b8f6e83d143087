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


def _grid_rects(R, Cc, pr, pc):
    rs = [R * i // pr for i in range(pr + 1)]
    cs = [Cc * j // pc for j in range(pc + 1)]
    return [(rs[i], cs[j], rs[i + 1] - rs[i], cs[j + 1] - cs[j]) for i in range(pr) for j in range(pc)]


@pytest.mark.parametrize("R,Cc,src,req", [
    (37, 53, (2, 3), (3, 2)),
    (64, 40, (1, 6), (6, 1)),        # 1D column blocks -> 1D row blocks
    (50, 50, (4, 1), (2, 2)),
])
def test_reference_mat_redist_between_layouts(R, Cc, src, req):
    """The reference's own mat_redist (src/mat_redist.c, vmpi rank threads) moves
    every required block out of the source layout: the pin for the GPU's
    folded layout redistribution."""
    if orc.ref_lib() is None:
        pytest.skip("reference CPU path not built")
    G = orc.gen_uniform(77, R, Cc)
    sr = _grid_rects(R, Cc, *src)
    rr = _grid_rects(R, Cc, *req)
    out = orc.ref_redist(sr, rr, G)
    for o, r in zip(out, rr):
        assert np.array_equal(o, G[r[0]:r[0] + r[2], r[1]:r[1] + r[3]])


def test_reference_gpu_build_loads_and_serialises_cublas():
    """The reference's GPU path build (context figures) loads without a GPU and
    routes every wrapper that touches the reference's static cuBLAS handle
    through the serialising shim (the originals renamed vgpu_raw_*)."""
    import os
    path = os.path.join(os.path.dirname(orc.HERE), "oracle", "_ref", "libref_ca3dmm_cuda.so")
    if not os.path.exists(path):
        pytest.skip("reference GPU path not built")
    L = orc.ref_cuda_lib()
    assert L is not None and hasattr(L, "ref_ca3dmm_cuda")
    for f in ("cuda_cublas_dgemm", "cuda_cublas_dgeam", "cuda_cublas_dcopy"):
        assert hasattr(L, f) and hasattr(L, "vgpu_raw_" + f), f
