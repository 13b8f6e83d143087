"""A model of the multi-GPU CA3DMM exec in Python, for the CPU tests (test
infrastructure: the product is the C engine of include/ca3dmm_dist.h, which
ca3dmm_b200/dist.py drives over torch.distributed).

It plans the same two all-to-alls as ca3dmm_b200/csrc/dist.c -- each rank's
op(A) / op(B) panels of its cuboid (the grid and cuboids of
ca3dmm_engine_init / _init_BTB, src/ca3dmm.c:23-722, for p = the group's size),
the pieces of every rank's A and B blocks that fall into every peer's panels,
the pieces of every C_2dmm block that fall into every peer's dst_C block, and
the slab-ordered sum of the kp partials (src/ca3dmm.c:977-1171, 1287-1372) --
written independently in Python, so that gloo ranks on CPU can run the whole
exchange with numpy stand-ins for the device side (tests/test_dist_host.py)
and the C engine's plan can be checked against it piece count by piece count.

Rectangles are (srow, nrow, scol, ncol) of a column-major matrix, the
reference's argument order.
"""
import time

import ca3dmm_b200 as cb

_A, _B = 0, 1


def _inter(a, b):
    r0, r1 = max(a[0], b[0]), min(a[0] + a[1], b[0] + b[1])
    c0, c1 = max(a[2], b[2]), min(a[2] + a[3], b[2] + b[3])
    if r1 <= r0 or c1 <= c0:
        return None
    return (r0, r1 - r0, c0, c1 - c0)


def _area(r):
    return r[1] * r[3] if r is not None else 0


def _rm(r):
    """A column-major rectangle of layer/matrix `r[4]` as the row-major rectangle
    of the transposed matrix that mat_redist_layouts works on, stacked by the
    offset r[5] so that different matrices (or slab layers) never meet."""
    return (r[2] + r[5], r[0], r[3], r[1])


class DistModel:
    """One rank of the model over a torch.distributed group.

    ``DistCa3dmmEngine(m, n, k, trans_A, trans_B, src_A, src_B, dst_C)`` mirrors
    ``ca3dmm_engine_init`` called by every rank with its own blocks:
    ``src_A`` / ``src_B`` / ``dst_C`` are this rank's rectangles (srow, nrow,
    scol, ncol) of A, B (as stored, before op) and C.  ``btb=True`` mirrors
    ``ca3dmm_engine_init_BTB`` (C = B^T B, ``src_A`` ignored).  ``proc_grid``
    forces mp x np x kp as in the reference.  ``exec(A, ldA, B, ldB, C, ldC)``
    takes this rank's blocks as flat float64 device tensors (column-major)."""

    def __init__(self, m, n, k, trans_A, trans_B, src_A, src_B, dst_C, proc_grid=None,
                 group=None, btb=False, gemm_mode=cb.GEMM_PLAIN, slices=7, ops=None):
        import torch
        import torch.distributed as dist
        self.dist, self.torch = dist, torch
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.btb = bool(btb)
        self.m, self.n, self.k = (n if btb else m), n, k
        self.ta, self.tb = (1 if btb else int(trans_A)), (0 if btb else int(trans_B))
        self.direct = dist.get_backend(group) == "nccl"
        if ops is None:
            raise ValueError("the model needs its device-side stand-in (ops)")
        self.ops = ops
        self.comm_device = ops.device if self.direct else torch.device("cpu")
        # every rank's rectangles
        # every rank's rectangles and call arguments: each rank checks all of
        # them, so an inconsistent call raises on every rank before any exchange
        g3 = list(proc_grid) if proc_grid is not None else [-1, -1, -1]
        mine = list(src_A if not btb else (0, 0, 0, 0)) + list(src_B) + list(dst_C) + \
            [m, n, k, self.ta, self.tb, int(self.btb), int(gemm_mode), int(slices)] + g3
        allr = self._allgather_ints(mine)
        if any(r[12:] != allr[0][12:] for r in allr):
            raise ValueError("ranks disagree on m, n, k, transposes, mode or grid")
        self.srcA = [tuple(r[0:4]) for r in allr]
        self.srcB = [tuple(r[4:8]) for r in allr]
        self.dstC = [tuple(r[8:12]) for r in allr]
        a_shape = (k, m) if self.ta else (m, k)
        b_shape = (k, n) if btb else ((n, k) if self.tb else (k, n))
        c_shape = (self.m, n)
        for rects, shape, what in ((self.srcA if not btb else [], a_shape, "src_A"),
                                   (self.srcB, b_shape, "src_B"), (self.dstC, c_shape, "dst_C")):
            for r in rects:
                if min(r) < 0 or r[0] + r[1] > shape[0] or r[2] + r[3] > shape[1]:
                    raise ValueError("%s rectangle %s outside the %d x %d matrix" %
                                     ((what, r) + shape))
        # the reference's grid and every rank's cuboid (no device call)
        geo = cb.Ca3dmmEngine(m, n, k, self.ta if not btb else 0, self.tb, p=self.world,
                              proc_grid=proc_grid, btb=btb, caller_workbuf=True)
        if not geo.ok:
            raise ValueError("CA3DMM grid planning failed")
        s = geo.s
        self.mp, self.np_, self.kp, self.rp = s.mp, s.np, s.kp, s.rp
        info = [geo.vrank_info(r) for r in range(self.world)]
        geo.free()
        self.active = [bool(g[0]) for g in info]
        self.slab = [g[9] if g[0] else -1 for g in info]
        # C_2dmm block (srow, nrow, scol, ncol) and k range of every rank
        self.cblk = [(g[18], g[20], g[19], g[21]) if g[0] else None for g in info]
        self.krange = [cb.calc_block_spos_size(k, self.kp, g[9]) if g[0] else (0, 0)
                       for g in info]
        self._check_cover()
        self.panels = [self._panels(r) for r in range(self.world)]
        # every panel must be covered by the ranks' source blocks
        for r in range(self.world):
            for mat, rect in self.panels[r]:
                got = sum(_area(_inter(self._src(mat, q), rect)) for q in range(self.world))
                if got < _area(rect):
                    raise ValueError("the source blocks do not cover rank %d's %s panel %s" %
                                     (r, "A" if mat == _A else "B", rect))
        self._plan_operands()
        self._plan_c()
        self.gemm_mode, self.slices = gemm_mode, slices
        self.local = None
        r = self.rank
        if self.active[r]:
            cm, cn, kz = self.cblk[r][1], self.cblk[r][3], self.krange[r][1]
            if cm > 0 and cn > 0 and kz > 0:
                self.local = self.ops.gemm_engine(cm, cn, kz, self._panel_trans(0),
                                                  self._panel_trans(1), gemm_mode, slices)
        self.stats = {"n_exec": 0, "exchange_ab_ms": 0.0, "gemm_ms": 0.0, "exchange_c_ms": 0.0,
                      "exec_ms": 0.0}

    # ------------------------------------------------------------------ planning
    def _allgather_ints(self, vals):
        t = self.torch.tensor(vals, dtype=self.torch.int64, device=self.comm_device)
        out = self.torch.empty(self.world * len(vals), dtype=self.torch.int64,
                               device=self.comm_device)
        self.dist.all_gather_into_tensor(out, t, group=self.group)
        o = out.cpu().tolist()
        w = len(vals)
        return [o[i * w:(i + 1) * w] for i in range(self.world)]

    def _check_cover(self):
        """The active ranks of each slab must tile C exactly (src/ca3dmm.c:212-261)."""
        area = [0] * self.kp
        for r in range(self.world):
            if self.active[r]:
                area[self.slab[r]] += _area(self.cblk[r])
        if any(a != self.m * self.n for a in area):
            raise ValueError("cuboids do not tile C: %s" % area)

    def _panels(self, r):
        """(matrix, rectangle) of rank r's op(A) and op(B) panels, in the stored
        matrix's coordinates."""
        if not self.active[r]:
            return [(_A, (0, 0, 0, 0)), (_B, (0, 0, 0, 0))]
        cm0, cmz, cn0, cnz = self.cblk[r]
        k0, kz = self.krange[r]
        if self.btb:             # op(A) = B^T: rows k, columns = C rows
            return [(_B, (k0, kz, cm0, cmz)), (_B, (k0, kz, cn0, cnz))]
        a = (k0, kz, cm0, cmz) if self.ta else (cm0, cmz, k0, kz)
        b = (cn0, cnz, k0, kz) if self.tb else (k0, kz, cn0, cnz)
        return [(_A, a), (_B, b)]

    def _panel_trans(self, i):
        return self.ta if i == 0 else self.tb

    def _moff(self, mat):
        """Stacking offset of a matrix in the transposed coordinates (columns of A first)."""
        if mat == _A or self.btb:
            return 0
        return self.k if not self.ta else self.m          # columns of the stored A

    def _src(self, mat, r):
        return self.srcB[r] if (mat == _B or self.btb) else self.srcA[r]

    def _plan_operands(self):
        """Pieces of A and B each rank sends to each peer (identical panels of one
        rank are sent once)."""
        W, me = self.world, self.rank

        def uniq(r):
            out = []
            for mat, rect in self.panels[r]:
                if (mat, rect) not in out:
                    out.append((mat, rect))
            return out

        self.uniq = [uniq(r) for r in range(W)]
        self.send_pieces, self.send_counts = [], []
        for d in range(W):
            cnt = 0
            for mat, rect in self.uniq[d]:
                x = _inter(self._src(mat, me), rect)
                if x is not None:
                    self.send_pieces.append((mat, x, sum(self.send_counts) + cnt))
                    cnt += _area(x)
            self.send_counts.append(cnt)
        self.recv_pieces, self.recv_counts = [], []
        for q in range(W):
            cnt = 0
            for mat, rect in self.uniq[me]:
                x = _inter(self._src(mat, q), rect)
                if x is not None:
                    self.recv_pieces.append((mat, x, sum(self.recv_counts) + cnt))
                    cnt += _area(x)
            self.recv_counts.append(cnt)
        # the device copies: my blocks -> send pieces; received pieces -> my panels
        mats = [_B] if self.btb else [_A, _B]
        self.my_blocks = [(mat, self._src(mat, me)) for mat in mats if _area(self._src(mat, me)) > 0]
        ext = lambda mat, r: r + (mat, self._moff(mat))
        self.pack_ab = self.ops.copier([ext(mat, r) for mat, r in self.my_blocks],
                                       [ext(mat, r) for mat, r, _ in self.send_pieces])
        self.panel_size = [_area(rect) for _, rect in self.uniq[me]]
        self.unpack_ab = self.ops.copier([ext(mat, r) for mat, r, _ in self.recv_pieces],
                                         [ext(mat, r) for mat, r in self.uniq[me]])

    def _plan_c(self):
        W, me = self.world, self.rank
        N = self.n
        self.c_send, self.c_send_counts = [], []
        mine = self.cblk[me]
        for d in range(W):
            x = _inter(mine, self.dstC[d]) if mine is not None else None
            self.c_send_counts.append(_area(x))
            if x is not None:
                self.c_send.append((x, sum(self.c_send_counts[:-1])))
        self.c_recv, self.c_recv_counts = [], []
        for q in range(W):
            x = _inter(self.cblk[q], self.dstC[me]) if self.cblk[q] is not None else None
            self.c_recv_counts.append(_area(x))
            if x is not None:
                self.c_recv.append((x, self.slab[q], sum(self.c_recv_counts[:-1])))
        ext = lambda r, layer: r + (layer, layer * N)
        self.pack_c = self.ops.copier([ext(mine, 0)] if mine is not None and _area(mine) else [],
                                      [ext(x, 0) for x, _ in self.c_send])
        d = self.dstC[me]
        layers = self.kp if self.kp > 1 else 1
        self.unpack_c = self.ops.copier([ext(x, sl if self.kp > 1 else 0) for x, sl, _ in self.c_recv],
                                        [ext(d, j) for j in range(layers)] if _area(d) else [])

    # ------------------------------------------------------------------ exec
    def _a2a(self, send, send_counts, recv_counts):
        t = send if self.direct else send.cpu()
        out = self.torch.empty(max(sum(recv_counts), 1), dtype=self.torch.float64,
                               device=t.device)
        ins, outs = t[:sum(send_counts)], out[:sum(recv_counts)]
        self.dist.all_to_all_single(outs, ins, list(recv_counts), list(send_counts),
                                    group=self.group)
        if not self.direct:
            dev = self.ops.empty(out.numel())
            dev.copy_(out)
            out = dev
        return out

    def _whole_on_one_rank(self):
        """One rank holding all of A, B and C with a 1x1x1 grid: its panels are
        its blocks, so the local GEMM reads and writes them in place."""
        if self.world != 1 or self.local is None or self.kp != 1:
            return False
        full = lambda r, shape: r == (0, shape[0], 0, shape[1])
        a_shape = (self.k, self.m) if self.ta else (self.m, self.k)
        b_shape = (self.k, self.n) if self.btb else ((self.n, self.k) if self.tb else
                                                      (self.k, self.n))
        return ((self.btb or full(self.srcA[0], a_shape)) and full(self.srcB[0], b_shape) and
                full(self.dstC[0], (self.m, self.n)))

    def exec(self, A, ldA, B, ldB, C, ldC):
        """This rank's part of C = op(A) op(B) (or B^T B): every rank calls it."""
        ops, me = self.ops, self.rank
        t0 = time.perf_counter()
        if self._whole_on_one_rank():
            if self.btb:
                A, ldA = B, ldB
            ops.gemm(self.local, A, ldA, B, ldB, C, ldC)
            ops.sync()
            dt = 1e3 * (time.perf_counter() - t0)
            self.stats["n_exec"] += 1
            self.stats["gemm_ms"] += dt
            self.stats["exec_ms"] += dt
            return 0
        blocks = {_A: (A, ldA), _B: (B, ldB)}
        send = ops.empty(sum(self.send_counts))
        ops.copy(self.pack_ab, [(blocks[mat][0], 0, blocks[mat][1]) for mat, _ in self.my_blocks],
                 [(send, off, x[1]) for _, x, off in self.send_pieces])
        recv = self._a2a(send, self.send_counts, self.recv_counts)
        panels = [ops.empty(z) for z in self.panel_size]
        ops.copy(self.unpack_ab, [(recv, off, x[1]) for _, x, off in self.recv_pieces],
                 [(p, 0, rect[1]) for p, (_, rect) in zip(panels, self.uniq[me])])
        ops.sync()
        t1 = time.perf_counter()
        cblk = self.cblk[me]
        cbuf = None
        if cblk is not None:
            cbuf = ops.zeros(_area(cblk))
            if self.local is not None:
                pa = self.uniq[me].index(self.panels[me][0])
                pb = self.uniq[me].index(self.panels[me][1])
                ops.gemm(self.local, panels[pa], self.panels[me][0][1][1], panels[pb],
                         self.panels[me][1][1][1], cbuf, cblk[1])
        ops.sync()
        t2 = time.perf_counter()
        csend = ops.empty(sum(self.c_send_counts))
        if cbuf is not None:
            ops.copy(self.pack_c, [(cbuf, 0, cblk[1])], [(csend, off, x[1]) for x, off in self.c_send])
        crecv = self._a2a(csend, self.c_send_counts, self.c_recv_counts)
        d = self.dstC[me]
        if _area(d):
            if self.kp > 1:
                z = _area(d)
                layers = ops.empty(self.kp * z)
                ops.copy(self.unpack_c, [(crecv, off, x[1]) for x, _, off in self.c_recv],
                         [(layers, j * z, d[1]) for j in range(self.kp)])
                ops.ordered_sum(layers, self.kp, d[1], d[3], C, ldC)
            else:
                ops.copy(self.unpack_c, [(crecv, off, x[1]) for x, _, off in self.c_recv],
                         [(C, 0, ldC)])
        ops.sync()
        t3 = time.perf_counter()
        st = self.stats
        st["n_exec"] += 1
        st["exchange_ab_ms"] += 1e3 * (t1 - t0)
        st["gemm_ms"] += 1e3 * (t2 - t1)
        st["exchange_c_ms"] += 1e3 * (t3 - t2)
        st["exec_ms"] += 1e3 * (t3 - t0)
        return 0

    def reset_stat(self):
        for key in self.stats:
            self.stats[key] = 0 if key == "n_exec" else 0.0

    def free(self):
        local = getattr(self, "local", None)
        if local is not None and hasattr(local, "free"):
            local.free()
        self.local = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
