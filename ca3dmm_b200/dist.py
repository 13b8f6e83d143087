"""CA3DMM across GPUs from Python: one process per GPU over torch.distributed.

The engine is the C one of include/ca3dmm_dist.h (ca3dmm_dist_engine_*,
csrc/dist.c): every rank computes the reference's grid and every rank's
cuboid for p = the group's size (ca3dmm_engine_init / _init_BTB,
src/ca3dmm.c:23-722), and an exec is two all-to-alls around the local GEMM --
the pieces of every rank's A and B blocks that fall into each peer's op(A) /
op(B) panels, the local GEMM of the panels on this GPU, the pieces of every
C_2dmm block that fall into each peer's dst_C block, summed over the kp slabs
in slab order (src/ca3dmm.c:977-1171, 1287-1372).  This module gives it a
transport whose two collectives are torch.distributed calls on the caller's
process group: with NCCL the engine exchanges device buffers (the reference's
DEV_TYPE_CUDA_MPI_DIRECT), with any other backend (gloo) pinned host buffers
(its DEV_TYPE_CUDA), src/dev_type.h:9-14.

Rectangles are (srow, nrow, scol, ncol) of a column-major matrix, the
reference's argument order.
"""
import ctypes as C
import sys

import numpy as np

import ca3dmm_b200 as cb

_ALLGATHER = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_longlong), C.c_int,
                         C.POINTER(C.c_longlong))
_ALLTOALLV = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_longlong),
                         C.POINTER(C.c_longlong), C.c_void_p, C.POINTER(C.c_longlong),
                         C.POINTER(C.c_longlong), C.c_void_p)


class _DeviceDoubles:
    """n doubles of device memory at ptr, for torch.as_tensor (no copy)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 2,
                                         "strides": None}


class TorchTransport:
    """ca3dmm_transport_t over a torch.distributed group.  ``t`` is the
    structure to pass to the engine; this object must outlive it (it holds the
    callbacks)."""

    def __init__(self, group=None, device=None):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.direct = dist.get_backend(group) == "nccl"
        self.device = device
        self.comm_device = device if self.direct else torch.device("cpu")
        self._ag = _ALLGATHER(self._allgather)
        self._a2a = _ALLTOALLV(self._alltoallv)
        self.t = cb.Transport(self.rank, self.size, 1 if self.direct else 0, None,
                              C.cast(self._ag, C.c_void_p), C.cast(self._a2a, C.c_void_p))

    def _allgather(self, ctx, mine, n, out):
        try:
            torch = self.torch
            t = torch.tensor([mine[i] for i in range(n)], dtype=torch.int64, device=self.comm_device)
            parts = [torch.empty_like(t) for _ in range(self.size)]
            self.dist.all_gather(parts, t, group=self.group)
            for r, part in enumerate(parts):
                for i, v in enumerate(part.cpu().tolist()):
                    out[r * n + i] = v
            return 0
        except Exception as ex:            # the engine reports the failure
            print("ca3dmm dist transport: allgather failed: %r" % (ex,), file=sys.stderr)
            return 1

    def _view(self, ptr, count):
        torch = self.torch
        if self.direct:
            return torch.as_tensor(_DeviceDoubles(ptr, max(count, 1)), device=self.device)[:count]
        arr = np.ctypeslib.as_array((C.c_double * max(count, 1)).from_address(ptr))
        return torch.from_numpy(arr)[:count]

    def _alltoallv(self, ctx, send, scounts, sdispls, recv, rcounts, rdispls, stream):
        try:
            W = self.size
            sc = [int(scounts[i]) for i in range(W)]
            rc = [int(rcounts[i]) for i in range(W)]
            # the engine lays each peer's piece out contiguously in rank order
            if any(int(sdispls[i]) != sum(sc[:i]) or int(rdispls[i]) != sum(rc[:i])
                   for i in range(W)):
                raise ValueError("displacements are not the prefix sums of the counts")
            if self.direct:
                # the engine's packing ran on its own stream: finish it first
                self.torch.cuda.synchronize(self.device)
            st, rt = self._view(send, sum(sc)), self._view(recv, sum(rc))
            self.dist.all_to_all_single(rt, st, rc, sc, group=self.group)
            if self.direct:
                self.torch.cuda.synchronize(self.device)
            return 0
        except Exception as ex:
            print("ca3dmm dist transport: all-to-all failed: %r" % (ex,), file=sys.stderr)
            return 1


class DistCa3dmmEngine:
    """One rank of CA3DMM over a torch.distributed group, one GPU per rank.

    ``DistCa3dmmEngine(m, n, k, trans_A, trans_B, src_A, src_B, dst_C)`` mirrors
    ``ca3dmm_engine_init`` called by every rank with its own blocks:
    ``src_A`` / ``src_B`` / ``dst_C`` are this rank's rectangles of A, B (as
    stored, before op) and C.  ``btb=True`` mirrors ``ca3dmm_engine_init_BTB``
    (C = B^T B, ``src_A`` ignored).  ``proc_grid`` forces mp x np x kp as in the
    reference.  ``gemm_mode`` / ``slices``: the local GEMM (plain FP64, INT8
    slices with `slices` slices, or the modular mode with `slices` moduli, 0 =
    the engine's choice).  ``exec(A, ldA, B, ldB, C, ldC)`` takes this rank's
    blocks as flat float64 device tensors (column-major).  Ranks whose
    arguments disagree all raise."""

    def __init__(self, m, n, k, trans_A, trans_B, src_A, src_B, dst_C, proc_grid=None,
                 group=None, btb=False, gemm_mode=cb.GEMM_PLAIN, slices=7, device=None):
        import torch
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.transport = TorchTransport(group, device)
        self.rank, self.world = self.transport.rank, self.transport.size
        sl = int(slices) if gemm_mode in (cb.GEMM_OZAKI, cb.GEMM_CRT) else 0
        self.e = cb.DistEngine(m, n, k, 0 if btb else trans_A, 0 if btb else trans_B,
                               None if btb else src_A, src_B, dst_C, self.transport.t,
                               proc_grid=proc_grid, btb=btb, gemm_mode=gemm_mode, slices=sl)
        if not self.e.ok:
            raise ValueError("ca3dmm_dist_engine_init failed: %s" % cb.ERRORS.get(self.e.rc,
                                                                                   self.e.rc))
        info = self.e.info()
        self.mp, self.np_, self.kp, self.rp = info[:4]
        self.active, self.slab = bool(info[4]), info[5]
        self.cblk = tuple(info[6:10])
        self._base = (0, [0.0] * 4)

    @property
    def stats(self):
        """Per-phase wall time (ms) accumulated over the execs since reset_stat."""
        n, t = self.e.stats()
        n0, t0 = self._base
        d = [a - b for a, b in zip(t, t0)]
        return {"n_exec": n - n0, "exchange_ab_ms": d[0], "gemm_ms": d[1], "exchange_c_ms": d[2],
                "exec_ms": d[3]}

    def reset_stat(self):
        self._base = self.e.stats()

    def counts(self):
        """Elements this rank sends to / receives from each peer: operand send,
        operand receive, C send, C receive."""
        return self.e.counts()

    def exec(self, A, ldA, B, ldB, C_, ldC):
        """This rank's part of C = op(A) op(B) (or B^T B): every rank calls it."""
        rc = self.e.exec(A, ldA, B, ldB, C_, ldC)
        if rc:
            raise RuntimeError("ca3dmm_dist_engine_exec failed: %s" % cb.ERRORS.get(rc, rc))
        return 0

    def free(self):
        e = getattr(self, "e", None)
        if e is not None:
            e.free()
        self.e = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
