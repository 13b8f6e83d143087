"""Engine init (host only, no GPU): grid choice, per-virtual-rank geometry and
work-buffer sizing against the oracle's restatement of src/ca3dmm.c:146-356."""
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc

CASES = [  # m, n, k, p, trans_A, trans_B, proc_grid
    (8000, 8000, 8000, 24, 0, 0, None),
    (8000, 8000, 8000, 24, 1, 0, None),
    (2048, 2048, 2048, 4, 0, 0, None),
    (1000, 3000, 700, 12, 0, 1, None),
    (3000, 1000, 700, 12, 1, 1, None),
    (517, 1031, 2049, 16, 0, 0, (2, 4, 2)),
    (64, 64, 100000, 8, 0, 0, None),
    (5, 7, 3, 6, 0, 0, None),
    (4096, 128, 128, 32, 0, 0, None),
]


@pytest.mark.parametrize("m,n,k,p,ta,tb,grid", CASES)
def test_vrank_geometry_matches_oracle(m, n, k, p, ta, tb, grid):
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid, caller_workbuf=True)
    assert e.ok
    s = e.s
    if grid is None:
        assert (s.mp, s.np, s.kp, s.rp) == cb.calc_3d_decomposition_cannon(p, m, n, k)
    else:
        assert (s.mp, s.np, s.kp) == tuple(grid)
    for r in range(p):
        want = orc.rank_geometry(m, n, k, s.mp, s.np, s.kp, r, 0)
        assert e.vrank_info(r) == want, r
    g0 = orc.rank_geometry(m, n, k, s.mp, s.np, s.kp, 0, 0)
    assert (s.A_2dmm_srow, s.A_2dmm_scol, s.A_2dmm_nrow, s.A_2dmm_ncol) == tuple(g0[10:14])
    assert (s.B_2dmm_srow, s.B_2dmm_scol, s.B_2dmm_nrow, s.B_2dmm_ncol) == tuple(g0[14:18])
    assert (s.C_2dmm_srow, s.C_2dmm_scol, s.C_2dmm_nrow, s.C_2dmm_ncol) == tuple(g0[18:22])
    assert (s.B_rd_srow, s.B_rd_scol, s.B_rd_nrow, s.B_rd_ncol) == tuple(g0[30:34])
    assert (s.C_out_nrow, s.C_out_ncol) == (m, n)
    assert e.workbuf_bytes >= 8 * (m * k + k * n + m * n)
    # every C entry is owned by exactly one active rank's C_out block
    cover = {}
    for r in range(p):
        g = orc.rank_geometry(m, n, k, s.mp, s.np, s.kp, r, 0)
        if g[0]:
            cover[(g[22], g[23])] = cover.get((g[22], g[23]), 0) + g[24] * g[25]
    assert sum(cover.values()) == m * n
    e.free()


def test_8000cube_24_ranks_matches_readme():
    e = cb.Ca3dmmEngine(8000, 8000, 8000, 0, 0, p=24, caller_workbuf=True)
    s = e.s
    # README.md:66-67: task_m_num = 2, Cannon 2 x 2, per-rank blocks
    assert (s.mp, s.np, s.kp) == (4, 2, 3)
    assert (s.task_m_num, s.task_n_num, s.task_k_num) == (2, 1, 3)
    assert (s.A_2dmm_nrow, s.A_2dmm_ncol) == (2000, 1334)
    assert (s.B_rd_nrow, s.B_rd_ncol) == (1334, 2000)
    assert (s.B_2dmm_nrow, s.B_2dmm_ncol) == (1334, 4000)
    assert (s.C_2dmm_nrow, s.C_2dmm_ncol) == (2000, 4000)
    assert s.n_group == 3          # one grouped GEMM per k-slab (task_m blocks merged on one GPU)


def test_btb_grid_default_fold_and_forced():
    e = cb.Ca3dmmEngine(512, 512, 1 << 20, p=32, btb=True, caller_workbuf=True)
    assert (e.s.mp, e.s.np, e.s.kp) == (2, 2, 8)          # CA3DMM_REDUCE_KP default 1
    e2 = cb.Ca3dmmEngine(512, 512, 1 << 20, p=32, btb=True, proc_grid=(1, 1, 32),
                         caller_workbuf=True)
    assert (e2.s.mp, e2.s.np, e2.s.kp) == (1, 1, 32)
    for r in range(32):
        assert e2.vrank_info(r) == orc.rank_geometry(512, 512, 1 << 20, 1, 1, 32, r, 1)


def test_invalid_arguments_give_null_engine(capfd):
    assert not cb.Ca3dmmEngine(64, 64, 64, p=4, dev_type=cb.DEV_TYPE_HOST, caller_workbuf=True).ok
    assert not cb.Ca3dmmEngine(64, 64, 64, p=4, dev_type=7, caller_workbuf=True).ok
    assert not cb.Ca3dmmEngine(0, 64, 64, p=4, caller_workbuf=True).ok
    # a grid needing more ranks than p is rejected, one breaking max%min is regenerated
    # grids needing more ranks than p, or breaking max % min == 0, are
    # replaced by the planner's choice (src/ca3dmm.c:55-70)
    for grid, p in (((4, 4, 4), 4), ((2, 3, 1), 6)):
        e = cb.Ca3dmmEngine(64, 64, 64, p=p, proc_grid=grid, caller_workbuf=True)
        assert e.ok
        assert (e.s.mp, e.s.np, e.s.kp) == cb.calc_3d_decomposition_cannon(p, 64, 64, 64)[:3]
    err = capfd.readouterr().err
    assert "Invalid device type" in err and "Invalid process grid" in err


def test_cannon_engine_geometry():
    c = cb.CannonEngine(1000, 900, 800, p=4)
    # host-only: cannon init allocates its work buffer itself only with a GPU;
    # here it must at least size it and report rank 0's blocks.
    if c.ok:
        s = c.s
        assert s.np_dim == 2
        assert (s.A_nrow, s.A_ncol, s.B_nrow, s.B_ncol) == (500, 400, 400, 450)
