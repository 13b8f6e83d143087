"""The C multi-GPU engine's host logic (include/ca3dmm_dist.h) on CPU: ranks
are threads of this process over the library's thread transport, and
ca3dmm_dist_engine_init makes no CUDA call, so every rank's grid, cuboid and
exchange plan is checked without a GPU:
  * the grid and each rank's C_2dmm block are those of the folded engine for
    p = the rank count (the reference's partition);
  * what rank r sends to rank d in each exchange is what d receives from r;
  * every rank receives exactly its op(A) and op(B) panels, and kp slab
    partials of every entry of its dst_C block;
  * ranks whose arguments disagree all fail."""
import threading

import pytest

import ca3dmm_b200 as cb


def _cols(total, p, r):
    return cb.calc_block_spos_size(total, p, r)


def _run_ranks(p, make):
    tr = cb.ThreadTransports(p)
    assert tr.rc == 0
    out = [None] * p

    def body(r):
        out[r] = make(r, tr[r])

    th = [threading.Thread(target=body, args=(r,)) for r in range(p)]
    for t in th:
        t.start()
    for t in th:
        t.join(60)
    assert not any(t.is_alive() for t in th)
    tr.free()
    return out


def _column_layout(m, n, k, ta, tb, p, r, btb=False):
    """The reference example's 1D column blocks (examples/example_AB.c:85-98)."""
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (k, n) if btb else ((n, k) if tb else (k, n))
    a0, az = _cols(ac, p, r)
    b0, bz = _cols(bc, p, r)
    c0, cz = _cols(n, p, r)
    return (0, ar, a0, az), (0, br, b0, bz), (0, n if btb else m, c0, cz)


def _panel_areas(info, ta, tb, btb, k):
    mp, np_, kp = info[0], info[1], info[2]
    if not info[4]:
        return 0
    slab = info[5]
    k0, kz = cb.calc_block_spos_size(k, kp, slab)
    cr, cn = info[7], info[9]
    a = cr * kz
    b = kz * cn
    if btb and info[6] == info[8] and cr == cn:
        return a           # identical panels are sent once
    return a + b


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid,btb", [
    (300, 200, 500, 0, 0, 4, None, False),
    (257, 129, 1000, 1, 0, 6, None, False),
    (64, 500, 333, 0, 1, 3, None, False),
    (1100, 1300, 1200, 1, 1, 24, (4, 2, 3), False),
    (200, 200, 4000, 0, 0, 8, (2, 2, 2), False),
    (512, 512, 40000, 1, 0, 8, None, True),
    (96, 96, 700, 1, 0, 5, None, True),
])
def test_plans_are_consistent(m, n, k, ta, tb, p, grid, btb):
    geo = cb.Ca3dmmEngine(m, n, k, 0 if btb else ta, tb, p=p, proc_grid=grid, btb=btb,
                          caller_workbuf=True)
    want_grid = (geo.s.mp, geo.s.np, geo.s.kp, geo.s.rp)
    want_c = [geo.vrank_info(r) for r in range(p)]
    geo.free()

    def make(r, t):
        sa, sb, dc = _column_layout(m, n, k, ta, tb, p, r, btb)
        e = cb.DistEngine(m, n, k, ta, tb, None if btb else sa, sb, dc, t, proc_grid=grid,
                          btb=btb)
        res = (e.rc, e.info(), e.counts()) if e.ok else (e.rc, None, None)
        e.free()
        return res

    res = _run_ranks(p, make)
    assert all(rc == 0 for rc, _, _ in res), [rc for rc, _, _ in res]
    for r, (_, info, _) in enumerate(res):
        assert tuple(info[:4]) == want_grid
        g = want_c[r]
        assert info[4] == g[0]
        if g[0]:
            assert info[5] == g[9] and info[6:10] == [g[18], g[20], g[19], g[21]]
    kp = want_grid[2]
    for r in range(p):
        send_ab, recv_ab, send_c, recv_c = res[r][2]
        for d in range(p):
            assert send_ab[d] == res[d][2][1][r]
            assert send_c[d] == res[d][2][3][r]
        assert sum(recv_ab) == _panel_areas(res[r][1], ta, tb, btb, k)
        _, _, dc = _column_layout(m, n, k, ta, tb, p, r, btb)
        assert sum(recv_c) == kp * dc[1] * dc[3]


def test_inconsistent_calls_fail_on_every_rank():
    p = 3

    def make(r, t):
        sa, sb, dc = _column_layout(120, 90, 70, 0, 0, p, r)
        e = cb.DistEngine(120, 90, 70 + (r == 2), 0, 0, sa, sb, dc, t)
        rc = e.rc
        e.free()
        return rc

    assert all(rc != 0 for rc in _run_ranks(p, make))


def test_uncovered_panel_fails():
    """Source blocks that leave part of an operand on no rank."""
    p = 2

    def make(r, t):
        sa, sb, dc = _column_layout(100, 80, 60, 0, 0, p, r)
        if r == 1:
            sa = (0, 100, sa[2], sa[3] - 1)
        e = cb.DistEngine(100, 80, 60, 0, 0, sa, sb, dc, t)
        rc = e.rc
        e.free()
        return rc

    assert all(rc != 0 for rc in _run_ranks(p, make))


def test_a_rank_that_never_arrives_fails_the_others(monkeypatch):
    """Failure on the host: rank 2 of 3 never joins the init's allgather.  The
    thread transport's barrier has a time limit (CA3DMM_DIST_TIMEOUT), so ranks
    0 and 1 fail instead of hanging, and a later collective fails at once."""
    import time
    monkeypatch.setenv("CA3DMM_DIST_TIMEOUT", "1")
    p = 3
    tr = cb.ThreadTransports(p)
    assert tr.rc == 0
    out = [None] * p

    def body(r):
        sa, sb, dc = _column_layout(120, 90, 70, 0, 0, p, r)
        t0 = time.time()
        e = cb.DistEngine(120, 90, 70, 0, 0, sa, sb, dc, tr[r])
        out[r] = (e.rc, time.time() - t0)
        e.free()

    th = [threading.Thread(target=body, args=(r,)) for r in (0, 1)]
    for t in th:
        t.start()
    for t in th:
        t.join(30)
    assert not any(t.is_alive() for t in th)
    for r in (0, 1):
        rc, dt = out[r]
        assert rc != 0 and dt < 10, out[r]
    # the exchange area stays broken: rank 2 arriving late fails at once
    body(2)
    assert out[2][0] != 0 and out[2][1] < 1.0
    tr.free()
