"""The multi-GPU engine from Python (ca3dmm_b200.dist: the C engine of
include/ca3dmm_dist.h over a torch.distributed transport) with its device
side: batched rectangle copies, the single-GPU engine for each rank's cuboid
and the slab-ordered sum kernel.  Only one GPU is visible, so the ranks are
processes sharing it over gloo, which stages the exchanged pieces through host
memory (the reference's DEV_TYPE_CUDA); no kernel waits on another rank.  One
rank over NCCL runs the device-direct exchange (DEV_TYPE_CUDA_MPI_DIRECT).
INT8-slice split precision must equal the single-GPU engine on the same grid
bit for bit; plain FP64 and the modular mode stay within 2 k u |A||B| of the
exact product."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.test_dist_host import ROOT, U, _case_data, _free_port, _layout

pytestmark = pytest.mark.gpu


def _worker(rank, world, port, backend, cases, q):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import ca3dmm_b200 as cb
    from ca3dmm_b200.dist import DistCa3dmmEngine
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
            h = blk.ravel(order="F").copy() if blk.size else np.zeros(1)
            return torch.from_numpy(h).cuda(), max(r[1], 1)

        e = DistCa3dmmEngine(m, n, k, ta, tb, sa, sb, dc, proc_grid=grid, btb=btb,
                             gemm_mode=mode, slices=s)
        tA, lda = block(A, sa) if A is not None else (torch.zeros(1, dtype=torch.float64,
                                                                   device="cuda"), 1)
        tB, ldb = block(B, sb)
        ldc = max(dc[1], 1) + 2
        tC = torch.full((ldc * max(dc[3], 1),), -1.0, dtype=torch.float64, device="cuda")
        for _ in range(2):                      # a second exec reuses every plan
            e.exec(tA, lda, tB, ldb, tC, ldc)
        Cloc = tC.cpu().numpy().reshape(max(dc[3], 1), ldc).T[:dc[1], :dc[3]].copy()
        grid_used = (e.mp, e.np_, e.kp)
        e.free()
        want = None
        if rank == 0:
            # the single-GPU engine on the same virtual grid, whole matrices
            g = cb.Ca3dmmEngine(m, n, k, ta, tb, p=world, proc_grid=grid_used, btb=btb)
            assert g.ok and g.set_gemm_mode(mode, s) == 0
            dA = None if btb else torch.from_numpy(A.ravel(order="F").copy()).cuda()
            dB = torch.from_numpy(B.ravel(order="F").copy()).cuda()
            dC = torch.zeros(cm * n, dtype=torch.float64, device="cuda")
            assert g.exec(dA, 0 if btb else A.shape[0], dB, B.shape[0], dC, cm) == 0
            want = dC.cpu().numpy().reshape(n, cm).T.copy()
            g.free()
        out.append((dc, Cloc, want))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, out))


def _run(world, backend, cases):
    import queue
    import time
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, backend, cases, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res, t0 = {}, time.time()
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
            dc, Cloc, _ = res[r][i]
            C[dc[0]:dc[0] + dc[1], dc[2]:dc[2] + dc[3]] = Cloc
        want = res[0][i][2]
        if mode == 1:
            assert np.array_equal(C, want), case
        else:
            if btb:
                A, ta, tb = B, 1, 0
            opA, opB = (A.T if ta else A), (B.T if tb else B)
            assert np.all(np.abs(C - opA @ opB) <= 2 * k * U * (np.abs(opA) @ np.abs(opB))), case


def test_dist_engine_three_ranks_host_staged(cuda):
    _run(3, "gloo", [(300, 200, 700, 0, 0, None, "cols", 1, 7, False, 51),
                     (256, 384, 512, 1, 1, (1, 1, 3), "rows", 1, 6, False, 52),
                     (180, 180, 2000, 0, 0, None, "cols", 1, 7, True, 53),
                     (200, 300, 400, 0, 1, (3, 1, 1), "blocks", 0, 0, False, 54),
                     (300, 200, 700, 1, 0, None, "rows", 2, 0, False, 55)])


def test_dist_engine_four_ranks_host_staged(cuda):
    _run(4, "gloo", [(512, 512, 512, 0, 0, (2, 2, 1), "blocks", 1, 7, False, 61),
                     (400, 300, 900, 1, 0, (2, 1, 2), "cols", 1, 7, False, 62),
                     (333, 222, 444, 0, 0, (1, 1, 3), "cols", 1, 7, False, 63),   # one idle rank
                     (128, 128, 4000, 0, 0, (1, 1, 4), "cols", 0, 0, True, 64)])


def test_dist_engine_one_rank_nccl_direct(cuda):
    _run(1, "nccl", [(700, 500, 300, 0, 0, None, "cols", 1, 7, False, 71),
                     (300, 300, 300, 1, 1, None, "cols", 0, 0, False, 72)])
