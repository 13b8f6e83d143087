"""The multi-GPU exec on CPU gloo ranks, two ways:
  * the model of tests/_dist_model.py runs the whole exchange -- the
    reference's grid and cuboids for p = the group's size, the pieces each rank
    sends and receives in the operand and C all-to-alls, the unpacking into
    panels and slab layers and the slab-ordered sum -- with numpy copies and
    the oracle's GEMMs for the device side (test only), so that the assembled C
    must equal the single-process oracle bit for bit in split precision (slab
    by slab, slab order) and within k u |A||B| in plain FP64;
  * the product's C engine (ca3dmm_dist_engine_init over the torch.distributed
    transport of ca3dmm_b200/dist.py; init makes no CUDA call) plans the same
    exchanges: its per-peer element counts must equal the model's, case by
    case.
Several rank counts, grids, transposes, source/destination layouts and B^T B."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
U = 2.0 ** -53


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inter_shift(a, b):
    """Intersection of two stacked rectangles (srow, nrow, scol, ncol, tag, off)."""
    r0, r1 = max(a[0], b[0]), min(a[0] + a[1], b[0] + b[1])
    c0, c1 = max(a[2] + a[5], b[2] + b[5]), min(a[2] + a[5] + a[3], b[2] + b[5] + b[3])
    if r1 <= r0 or c1 <= c0:
        return None
    return r0, r1 - r0, c0, c1 - c0


class NumpyOps:
    """CPU stand-in for the device side of the distributed engine (test only)."""

    def __init__(self):
        import torch
        self.torch = torch
        self.device = torch.device("cpu")

    def empty(self, count):
        return self.torch.full((max(int(count), 1),), np.nan, dtype=self.torch.float64)

    def zeros(self, count):
        return self.torch.zeros(max(int(count), 1), dtype=self.torch.float64)

    @staticmethod
    def _view(t, off, ld, nrow, ncol):
        base = t.numpy()[off:]
        return np.lib.stride_tricks.as_strided(base, shape=(nrow, ncol), strides=(8, 8 * ld))

    def copier(self, src_rects, dst_rects):
        if not src_rects or not dst_rects:
            return None
        return (list(src_rects), list(dst_rects))

    def copy(self, L, srcs, dsts):
        if L is None:
            return
        sr, dr = L
        for s, (st, so, sl) in zip(sr, srcs):
            for d, (dt, do, dl) in zip(dr, dsts):
                x = _inter_shift(s, d)
                if x is None:
                    continue
                sv = self._view(st, so, sl, s[1], s[3])
                dv = self._view(dt, do, dl, d[1], d[3])
                dv[x[0] - d[0]:x[0] - d[0] + x[1], x[2] - d[2] - d[5]:x[2] - d[2] - d[5] + x[3]] = \
                    sv[x[0] - s[0]:x[0] - s[0] + x[1], x[2] - s[2] - s[5]:x[2] - s[2] - s[5] + x[3]]

    def gemm_engine(self, m, n, k, ta, tb, mode, slices):
        return (m, n, k, ta, tb, mode, slices)

    def gemm(self, e, A, lda, B, ldb, C, ldc):
        from oracle import oracle as orc
        m, n, k, ta, tb, mode, s = e
        a = self._view(A, 0, lda, *((k, m) if ta else (m, k)))
        b = self._view(B, 0, ldb, *((n, k) if tb else (k, n)))
        a = np.asfortranarray(a.T if ta else a)
        b = np.asfortranarray(b.T if tb else b)
        if mode == 1:
            qa, ea = orc.ozaki_slices_rows(a, 0, m, k, s)
            qb, eb = orc.ozaki_slices_cols(b, 0, k, n, s)
            c = orc.ozaki_gemm(qa, ea, qb, eb, m, n, k, s)
        else:
            c = a @ b
        self._view(C, 0, ldc, m, n)[:, :] = c

    def ordered_sum(self, layers, kp, nr, nc, out, ldo):
        z = nr * nc
        acc = self._view(layers, 0, nr, nr, nc).copy()
        for j in range(1, kp):
            acc = acc + self._view(layers, j * z, nr, nr, nc)
        self._view(out, 0, ldo, nr, nc)[:, :] = acc

    def sync(self):
        pass


def _split(length, parts, i):
    base, rem = divmod(length, parts)
    return i * base + min(i, rem), base + (1 if i < rem else 0)


def _random_layout(seed, nrow, ncol, world, rank):
    """Irregular blocks: random row and column cuts into pr x pc blocks dealt to
    a random permutation of the ranks (ranks beyond pr x pc own nothing)."""
    rng = np.random.default_rng(seed)
    pr = int(rng.integers(1, world + 1))
    pc = int(rng.integers(1, world // pr + 1))
    rc = np.sort(rng.choice(np.arange(1, max(nrow, 2)), size=min(pr - 1, max(nrow - 1, 0)),
                            replace=False)) if pr > 1 else np.array([], dtype=int)
    cc = np.sort(rng.choice(np.arange(1, max(ncol, 2)), size=min(pc - 1, max(ncol - 1, 0)),
                            replace=False)) if pc > 1 else np.array([], dtype=int)
    rs = [0] + [int(x) for x in rc] + [nrow]
    cs = [0] + [int(x) for x in cc] + [ncol]
    blocks = [(rs[i], rs[i + 1] - rs[i], cs[j], cs[j + 1] - cs[j])
              for i in range(len(rs) - 1) for j in range(len(cs) - 1)]
    order = rng.permutation(world)
    slot = int(np.where(order == rank)[0][0])
    return blocks[slot] if slot < len(blocks) else (0, 0, 0, 0)


def _layout(kind, nrow, ncol, world, rank):
    """This rank's (srow, nrow, scol, ncol) of an nrow x ncol matrix."""
    if isinstance(kind, int):                  # a seed: irregular blocks
        return _random_layout(kind, nrow, ncol, world, rank)
    if kind == "cols":                         # examples/example_AB.c:85-98
        s, z = _split(ncol, world, rank)
        return (0, nrow, s, z)
    if kind == "rows":
        s, z = _split(nrow, world, rank)
        return (s, z, 0, ncol)
    pr = 2 if world % 2 == 0 else 1            # 2D blocks
    pc = world // pr
    rs, rz = _split(nrow, pr, rank // pc)
    cs, cz = _split(ncol, pc, rank % pc)
    return (rs, rz, cs, cz)


def _case_data(case):
    from oracle import oracle as orc
    m, n, k, ta, tb, grid, lay, mode, s, btb, seed = case
    if btb:
        return None, orc.gen_btb(seed, k, n)
    A = orc.gen_signed_exp(seed, *((k, m) if ta else (m, k)), emin=-6, emax=6)
    B = orc.gen_signed_exp(seed + 1, *((n, k) if tb else (k, n)), emin=-6, emax=6)
    return A, B


def _worker(rank, world, port, cases, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import ca3dmm_b200 as cb
    from ca3dmm_b200.dist import TorchTransport
    from tests._dist_model import DistModel
    tt = TorchTransport()
    out = []
    for case in cases:
        m, n, k, ta, tb, grid, lay, mode, s, btb, seed = case
        A, B = _case_data(case)
        cm = n if btb else m
        sa = _layout(lay, *A.shape, world, rank) if A is not None else (0, 0, 0, 0)
        sb = _layout(lay, *B.shape, world, rank)
        dc = _layout(lay, cm, n, world, rank)

        def block(X, r):
            blk = np.asfortranarray(X[r[0]:r[0] + r[1], r[2]:r[2] + r[3]])
            return torch.from_numpy(blk.ravel(order="F").copy() if blk.size else np.zeros(1)), \
                max(r[1], 1)

        e = DistModel(m, n, k, ta, tb, sa, sb, dc, proc_grid=grid, btb=btb, gemm_mode=mode,
                      slices=s, ops=NumpyOps())
        # the C engine's plan of the same call (no exec: that needs a GPU)
        ce = cb.DistEngine(m, n, k, ta, tb, None if btb else sa, sb, dc, tt.t, proc_grid=grid,
                           btb=btb, gemm_mode=mode, slices=s if mode else 0)
        plan_c = ce.counts() if ce.ok else ce.rc
        ce.free()
        plan_model = [list(e.send_counts), list(e.recv_counts), list(e.c_send_counts),
                      list(e.c_recv_counts)]
        tA, lda = block(A, sa) if A is not None else (torch.zeros(1, dtype=torch.float64), 1)
        tB, ldb = block(B, sb)
        ldc = max(dc[1], 1) + 1                 # a padded leading dimension
        tC = torch.full((ldc * max(dc[3], 1),), -1.0, dtype=torch.float64)
        e.exec(tA, lda, tB, ldb, tC, ldc)
        Cloc = tC.numpy().reshape(max(dc[3], 1), ldc).T[:dc[1], :dc[3]].copy()
        out.append((dc, Cloc, (e.mp, e.np_, e.kp, e.rp), plan_c, plan_model))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


def _oracle_split(A, B, ta, tb, m, n, k, kp, s):
    from oracle import oracle as orc
    opA = A.T if ta else A
    opB = B.T if tb else B
    acc = None
    for sl in range(kp):
        k0, kz = orc.block_spos_size(k, kp, sl)
        a = np.asfortranarray(opA[:, k0:k0 + kz])
        b = np.asfortranarray(opB[k0:k0 + kz, :])
        qa, ea = orc.ozaki_slices_rows(a, 0, m, kz, s)
        qb, eb = orc.ozaki_slices_cols(b, 0, kz, n, s)
        c = orc.ozaki_gemm(qa, ea, qb, eb, m, n, kz, s)
        acc = c if acc is None else acc + c
    return acc


def _run(world, cases):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, cases, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = {}
    import queue
    import time
    t0 = time.time()
    while len(res) < world:
        try:
            r, o = q.get(timeout=2)
            res[r] = o
        except queue.Empty:
            assert not any(p.exitcode not in (None, 0) for p in procs), "a rank failed"
            assert time.time() - t0 < 300, "ranks timed out"
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for i, case in enumerate(cases):
        m, n, k, ta, tb, grid, lay, mode, s, btb, seed = case
        A, B = _case_data(case)
        cm = n if btb else m
        C = np.full((cm, n), np.nan)
        for r in range(world):
            dc, Cloc, g, plan_c, plan_model = res[r][i]
            C[dc[0]:dc[0] + dc[1], dc[2]:dc[2] + dc[3]] = Cloc
            assert plan_c == plan_model, (case, r, plan_c, plan_model)
        kp = res[0][i][2][2]
        if grid is not None:
            assert res[0][i][2][:3] == tuple(grid)
        if btb:
            A, ta, tb = B, 1, 0
        if mode == 1:
            assert np.array_equal(C, _oracle_split(A, B, ta, tb, cm, n, k, kp, s)), case
        else:
            opA, opB = (A.T if ta else A), (B.T if tb else B)
            assert np.all(np.abs(C - opA @ opB) <= 2 * k * U * (np.abs(opA) @ np.abs(opB))), case


CASES = {
    1: [(70, 50, 90, 1, 0, None, "cols", 1, 7, False, 81),      # one rank: in place
        (40, 40, 300, 0, 0, None, "cols", 1, 7, True, 82)],
    2: [(90, 70, 130, 0, 0, None, "cols", 1, 7, False, 1),
        (64, 96, 200, 1, 1, (1, 1, 2), "blocks", 1, 6, False, 2),
        (50, 40, 300, 0, 0, None, "rows", 0, 0, False, 3),
        (3, 40, 60, 0, 0, None, "cols", 0, 0, False, 4),
        (30, 30, 500, 0, 0, None, "cols", 1, 7, True, 5)],
    3: [(120, 60, 90, 0, 1, None, "cols", 1, 7, False, 11),
        (45, 80, 160, 1, 0, (1, 1, 3), "rows", 1, 5, False, 12),
        (33, 33, 700, 0, 0, None, "blocks", 1, 7, True, 13)],
    4: [(128, 64, 96, 0, 0, (2, 1, 2), "blocks", 1, 7, False, 21),
        (100, 100, 100, 1, 1, None, "cols", 1, 8, False, 22),
        (64, 64, 256, 0, 0, (2, 2, 1), "cols", 0, 0, False, 23),
        (40, 40, 900, 0, 0, (1, 1, 4), "cols", 1, 7, True, 24),
        (80, 60, 150, 0, 0, (1, 1, 3), "cols", 1, 7, False, 25),       # one idle rank
        (64, 64, 300, 0, 0, (2, 2, 1), "blocks", 1, 7, True, 26)],
    5: [(97, 61, 143, 1, 0, None, "cols", 1, 7, False, 41),
        (50, 50, 50, 0, 1, (2, 2, 1), "rows", 0, 0, False, 42)],       # one idle rank
    6: [(150, 75, 120, 0, 0, (3, 1, 2), "cols", 1, 7, False, 31),
        (60, 90, 80, 1, 0, None, "blocks", 1, 7, False, 32),
        (70, 70, 400, 0, 0, None, "rows", 0, 0, True, 33),
        (96, 96, 96, 0, 0, (2, 2, 1), "cols", 1, 7, False, 34)],       # two idle ranks
}


@pytest.mark.parametrize("world", sorted(CASES))
def test_dist_engine_on_gloo_ranks(world):
    _run(world, CASES[world])


def _random_cases(world, seed, count):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        btb = bool(rng.integers(0, 4) == 0)
        m, n, k = (int(x) for x in rng.integers(5, 160, 3))
        if btb:
            m = n
            k = int(rng.integers(50, 900))
        out.append((m, n, k, 0 if btb else int(rng.integers(0, 2)),
                    0 if btb else int(rng.integers(0, 2)), None, 1000 * seed + i,
                    int(rng.integers(0, 2)), int(rng.integers(5, 9)), btb, 500 + 7 * i + seed))
    return out


@pytest.mark.parametrize("world,seed", [(3, 1), (5, 2), (7, 3)])
def test_dist_engine_irregular_layouts(world, seed):
    """Random shapes, grids chosen by the planner and irregular source and
    destination blocks (random cuts dealt to a random permutation of ranks,
    some ranks owning nothing)."""
    _run(world, _random_cases(world, seed, 6))


def _bad_worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import ca3dmm_b200 as cb
    from ca3dmm_b200.dist import TorchTransport
    from tests._dist_model import DistModel
    tt = TorchTransport()
    m, n, k = 40, 30, 50
    cols = lambda nr, nc: _layout("cols", nr, nc, world, rank)
    args = {
        # rank 1 passes another m
        "sizes": (m + rank, n, k, cols(m, k), cols(k, n), cols(m, n)),
        # rank 1 owns no part of A: rank panels are not covered
        "cover": (m, n, k, cols(m, k) if rank == 0 else (0, 0, 0, 0), cols(k, n), cols(m, n)),
        # a source rectangle beyond the matrix
        "bounds": (m, n, k, cols(m, k), (0, k + 1, 0, n), cols(m, n)),
    }
    out = {}
    for name, (mm, nn, kk, sa, sb, dc) in args.items():
        try:
            DistModel(mm, nn, kk, 0, 0, sa, sb, dc, ops=NumpyOps())
            out[name] = None
        except ValueError as exc:
            out[name] = str(exc)
        # the C engine refuses the same call on every rank
        ce = cb.DistEngine(mm, nn, kk, 0, 0, sa, sb, dc, tt.t)
        out[name + "_c"] = ce.rc
        ce.free()
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


def test_dist_engine_rejects_inconsistent_calls_on_every_rank():
    """Inconsistent arguments, uncovered panels and out-of-range blocks raise
    ValueError on every rank before any exchange (no rank is left waiting) in
    the model, and make ca3dmm_dist_engine_init return CA3DMM_EINVAL on every
    rank."""
    import queue
    import time
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bad_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res, t0 = {}, time.time()
    while len(res) < 2:
        try:
            r, o = q.get(timeout=2)
            res[r] = o
        except queue.Empty:
            assert not any(p.exitcode not in (None, 0) for p in procs), "a rank failed"
            assert time.time() - t0 < 120, "ranks timed out"
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        assert "disagree" in res[r]["sizes"]
        assert "do not cover" in res[r]["cover"]
        assert "outside" in res[r]["bounds"]
        assert res[r]["sizes_c"] == res[r]["cover_c"] == res[r]["bounds_c"] == 1
