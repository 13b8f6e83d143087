"""ca3dmm_b200 -- CA3DMM's FP64 GEMM path, B200-native.

The product is the C-ABI shared library ``libca3dmm_b200.so`` (headers in
``include/``): the reference's ``ca3dmm_engine_*`` / ``cannon_engine_*`` /
partition API on one GPU.  This module is the Python host mirror of that
interface -- the same entry points, argument meaning and error behaviour
(an engine that fails to initialise is ``None``; exec errors are reported by
``last_error``) -- over ctypes.  Device memory is passed as raw pointers
(``torch.Tensor.data_ptr()`` or any CUDA allocation).

There is no CPU fallback: when the library is missing, ``lib()`` raises.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libca3dmm_b200.so")
# MLP trained on B200 timings of the 18 standard candidates (costmodel.CANDS)
# over 2000 shapes log-uniform in [128, 16384]^3
DEFAULT_COST_MODEL = os.path.join(HERE, "data", "costmodel_b200.txt")

DEV_TYPE_HOST, DEV_TYPE_CUDA, DEV_TYPE_CUDA_MPI_DIRECT = 0, 1, 2
GEMM_PLAIN, GEMM_OZAKI, GEMM_CRT, GEMM_AUTO = 0, 1, 2, 3
# return codes of the C ABI (ca3dmm_kernels.h)
OK, EINVAL, ECUDA, ETIMEOUT, ENOMEM, ENODEV, ECANARY = 0, 1, 2, 3, 4, 5, 6
ERRORS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "device wait timed out",
          4: "out of memory", 5: "no device", 6: "work buffer guard band overwritten"}

_lib = None


class Ca3dmmEngineS(C.Structure):
    """Mirror of ``struct ca3dmm_engine`` (include/ca3dmm.h)."""
    _fields_ = [(n, C.c_int) for n in (
        "m", "n", "k", "mp", "np", "kp", "rp", "my_rank", "n_proc", "is_active",
        "rank_m", "rank_n", "rank_k", "trans_A", "trans_B", "task_m_num", "task_m_id",
        "task_n_num", "task_n_id", "task_k_num", "task_k_id", "is_BTB", "use_ag", "use_rsb",
        "A_rd_srow", "A_rd_scol", "B_rd_srow", "B_rd_scol", "A_2dmm_srow", "A_2dmm_scol",
        "B_2dmm_srow", "B_2dmm_scol", "C_2dmm_srow", "C_2dmm_scol", "C_out_srow", "C_out_scol",
        "A_rd_nrow", "A_rd_ncol", "B_rd_nrow", "B_rd_ncol", "A_2dmm_nrow", "A_2dmm_ncol",
        "B_2dmm_nrow", "B_2dmm_ncol", "C_2dmm_nrow", "C_2dmm_ncol", "C_out_nrow", "C_out_ncol",
        "alloc_workbuf")] + [
        ("AB_agv_recvcnts", C.POINTER(C.c_int)), ("AB_agv_displs", C.POINTER(C.c_int)),
        ("C_rs_recvcnts", C.POINTER(C.c_int))] + [(n, C.c_void_p) for n in (
            "A_rd_recv_h", "A_trans_h", "A_2dmm_h", "B_rd_recv_h", "B_trans_h", "B_2dmm_h",
            "C_2dmm_h", "C_out_h", "A_rd_recv_d", "A_trans_d", "A_2dmm_d", "B_rd_recv_d",
            "B_trans_d", "B_2dmm_d", "C_2dmm_d", "C_out_d", "workbuf_h", "workbuf_d")] + [
        (n, C.c_size_t) for n in ("rdA_workbuf_bytes", "rdB_workbuf_bytes", "rdC_workbuf_bytes",
                                  "cannon_workbuf_bytes", "self_workbuf_bytes")] + [
        (n, C.c_void_p) for n in ("comm_AB_agv", "comm_C_rs", "comm_2dmm", "redist_A",
                                  "redist_B", "redist_C", "cannon_engine")] + [
        ("dev_type", C.c_int), ("print_timing", C.c_int)] + [
        (n, C.c_double) for n in ("init_ms", "redist_ms", "agvAB_ms", "cannon_ms", "reduce_ms",
                                  "hd_trans_ms", "exec_ms")] + [
        ("n_exec", C.c_int), ("n_group", C.c_int), ("gemm_mode", C.c_int),
        ("ozaki_slices", C.c_int), ("last_error", C.c_int), ("stream", C.c_void_p),
        ("sync_exec", C.c_int), ("workbuf_bytes", C.c_size_t), ("impl", C.c_void_p),
        ("raster", C.c_int), ("btb_symmetric", C.c_int), ("crt_moduli", C.c_int),
        ("crt_bits", C.c_int), ("gemm_auto", C.c_int), ("tune_ms", C.c_double)]


class TuneCfg(C.Structure):
    """Mirror of ca3dmm_tune_cfg_t (include/ca3dmm_tune.h)."""
    _fields_ = [("gemm_mode", C.c_int), ("slices", C.c_int), ("kp", C.c_int), ("raster", C.c_int),
                ("tile_n", C.c_int)]

    def tuple(self):
        return (self.gemm_mode, self.slices, self.kp, self.raster, self.tile_n)


def _cfg(c):
    """(mode, slices, kp, raster[, tile_n]) -> TuneCfg"""
    c = tuple(c)
    return TuneCfg(*(c + (0,) * (5 - len(c))))


NFEAT = 14


class Transport(C.Structure):
    """Mirror of ca3dmm_transport_t (include/ca3dmm_dist.h)."""
    _fields_ = [("rank", C.c_int), ("size", C.c_int), ("device_buffers", C.c_int),
                ("ctx", C.c_void_p), ("allgather_ll", C.c_void_p), ("alltoallv_d", C.c_void_p)]


class CannonEngineS(C.Structure):
    """Mirror of ``struct cannon_engine`` (include/cannon.h), leading fields."""
    _fields_ = [(n, C.c_int) for n in (
        "m", "n", "k", "my_rank", "rank_row", "rank_col", "np_dim", "A_srow", "A_scol", "B_srow",
        "B_scol", "C_srow", "C_scol", "A_nrow", "A_ncol", "B_nrow", "B_ncol", "C_nrow", "C_ncol",
        "gemm_cycle", "max_A_blk_size", "max_B_blk_size", "max_C_blk_size", "alloc_workbuf")] + [
        (n, C.POINTER(C.c_int)) for n in ("m_displs", "n_displs", "k_displs")] + [
        (n, C.c_void_p) for n in ("A_recv_h", "A_stack_h", "B_recv_h", "B_stack_h", "A_recv_d",
                                  "A_stack_d", "B_recv_d", "B_stack_d", "workbuf_h", "workbuf_d",
                                  "A_gemm_h", "B_gemm_h")] + [
        ("dev_type", C.c_int), ("comm", C.c_void_p)] + [
        (n, C.c_double) for n in ("init_ms", "shift0_ms", "lshift_ms", "gemm_ms", "exec_ms",
                                  "hd_trans_ms")] + [
        ("n_exec", C.c_int), ("workbuf_bytes", C.c_size_t), ("impl", C.c_void_p),
        ("last_error", C.c_int)]


def lib():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libca3dmm_b200.so is not built: run `python -m ca3dmm_b200.build`")
    L = C.CDLL(LIB_PATH)
    i, p, d, sz = C.c_int, C.c_void_p, C.c_double, C.c_size_t
    pi = C.POINTER(C.c_int)
    EP = C.POINTER(Ca3dmmEngineS)
    sig = {
        "ca3dmm_vcomm_create": (i, [i, C.POINTER(p)]),
        "ca3dmm_vcomm_free": (None, [C.POINTER(p)]),
        "ca3dmm_vcomm_size": (i, [p]),
        "calc_3d_decomposition_cannon": (None, [i, i, i, i, pi, pi, pi, pi]),
        "calc_3d_decomposition_nk": (None, [i, i, i, pi, pi, pi]),
        "calc_block_spos_size": (None, [i, i, i, pi, pi]),
        "ca3dmm_engine_init": (None, [i] * 17 + [pi, p, i, C.POINTER(EP), C.POINTER(sz)]),
        "ca3dmm_engine_init_BTB": (None, [i] * 10 + [pi, p, i, C.POINTER(EP), C.POINTER(sz)]),
        "ca3dmm_engine_attach_workbuf": (None, [EP, p, p]),
        "ca3dmm_engine_free": (None, [C.POINTER(EP)]),
        "ca3dmm_engine_exec": (None, [EP, p, i, p, i, p, i]),
        "ca3dmm_engine_reset_stat": (None, [EP]),
        "ca3dmm_engine_print_stat": (None, [EP]),
        "ca3dmm_engine_last_error": (i, [EP]),
        "ca3dmm_engine_set_stream": (None, [EP, p, i]),
        "ca3dmm_engine_set_gemm_mode": (i, [EP, i, i]),
        "ca3dmm_engine_workbuf_bytes": (sz, [EP]),
        "ca3dmm_engine_vrank_info": (i, [EP, i, pi]),
        "ca3dmm_engine_guard_bands": (i, [EP, C.POINTER(C.c_longlong), i]),
        "cannon_engine_init": (None, [i, i, i, p, i, C.POINTER(C.POINTER(CannonEngineS)),
                                      C.POINTER(sz)]),
        "cannon_engine_attach_workbuf": (None, [C.POINTER(CannonEngineS), p, p]),
        "cannon_engine_free": (None, [C.POINTER(C.POINTER(CannonEngineS))]),
        "cannon_engine_exec": (None, [C.POINTER(CannonEngineS), d, d, p, p, p]),
        "cannon_engine_reset_stat": (None, [C.POINTER(CannonEngineS)]),
        "cannon_engine_print_stat": (None, [C.POINTER(CannonEngineS)]),
        "dev_type_malloc": (p, [sz, i]),
        "dev_type_free": (None, [p, i]),
        "dev_type_memcpy": (None, [p, p, sz, i, i]),
        "dev_type_memset": (None, [p, i, sz, i]),
        "dev_type_copy_mat_blk": (None, [sz, i, i, p, i, p, i, i]),
        "ca3dmm_dgemm_kslab_noalloc": (i, [i, i, i, i, p, i, p, i, p, i, p]),
        "ca3dmm_dgemm_kslab_noalloc_scratch_bytes": (sz, []),
        "ca3dmm_grouped_init": (i, [i, pi, pi, pi, pi, pi, i, i, C.POINTER(p), C.POINTER(sz)]),
        "ca3dmm_grouped_attach_workbuf": (i, [p, p]),
        "ca3dmm_grouped_set_stream": (None, [p, p, i]),
        "ca3dmm_grouped_exec": (i, [p, C.POINTER(p), pi, C.POINTER(p), pi, C.POINTER(p), pi]),
        "ca3dmm_grouped_last_ms": (d, [p]),
        "ca3dmm_grouped_free": (None, [C.POINTER(p)]),
        "ca3dmm_engine_set_raster": (i, [EP, i]),
        "ca3dmm_tune_features": (i, [i, i, i, i, i, C.POINTER(TuneCfg), C.c_float,
                                     C.POINTER(C.c_float)]),
        "ca3dmm_tune_measure": (i, [i, i, i, i, i, p, i, p, i, p, i, C.POINTER(TuneCfg), i,
                                    C.POINTER(C.c_float)]),
        "ca3dmm_autotune": (i, [i, i, i, i, i, p, i, p, i, p, i, C.POINTER(TuneCfg), i, C.c_float,
                                p, i, i, pi, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "ca3dmm_engine_set_tune": (i, [EP, C.POINTER(TuneCfg)]),
        "ca3dmm_transport_threads_create": (i, [i, C.POINTER(Transport)]),
        "ca3dmm_transport_threads_free": (None, [C.POINTER(Transport)]),
        "ca3dmm_nccl_unique_id": (i, [C.POINTER(C.c_ubyte)]),
        "ca3dmm_transport_nccl_create": (i, [i, i, C.POINTER(C.c_ubyte), C.POINTER(Transport)]),
        "ca3dmm_transport_nccl_free": (None, [C.POINTER(Transport)]),
        "ca3dmm_dist_engine_init": (i, [i] * 18 + [pi, C.POINTER(Transport), i, i, C.POINTER(p)]),
        "ca3dmm_dist_engine_exec": (i, [p, p, i, p, i, p, i]),
        "ca3dmm_dist_engine_info": (i, [p, pi]),
        "ca3dmm_dist_engine_counts": (i, [p] + [C.POINTER(C.c_longlong)] * 4),
        "ca3dmm_dist_engine_stats": (i, [p, C.POINTER(C.c_double)]),
        "ca3dmm_dist_engine_free": (None, [C.POINTER(p)]),
        "ca3dmm_engine_get_tune": (i, [EP, C.POINTER(TuneCfg)]),
        "ca3dmm_engine_autotune": (i, [EP, p, i, p, i, p, i, i, C.POINTER(TuneCfg)]),
        "ca3dmm_engine_tune_report": (i, [EP, C.POINTER(TuneCfg), C.POINTER(C.c_float),
                                          C.POINTER(C.c_float), i]),
        "ca3dmm_mlp_create": (i, [i, i, i, C.c_ulonglong, C.POINTER(p)]),
        "ca3dmm_mlp_free": (None, [C.POINTER(p)]),
        "ca3dmm_mlp_nparams": (i, [p]),
        "ca3dmm_mlp_inputs": (i, [p]),
        "ca3dmm_mlp_get_params": (i, [p, C.POINTER(C.c_float)]),
        "ca3dmm_mlp_set_params": (i, [p, C.POINTER(C.c_float)]),
        "ca3dmm_mlp_set_normalisation": (i, [p, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "ca3dmm_mlp_fwd_bwd": (i, [p, C.POINTER(C.c_float), C.POINTER(C.c_float), i,
                                   C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "ca3dmm_mlp_train": (i, [p, C.POINTER(C.c_float), C.POINTER(C.c_float), i, i, i,
                                 C.c_float, C.c_ulonglong, C.POINTER(C.c_float)]),
        "ca3dmm_mlp_predict": (i, [p, C.POINTER(C.c_float), i, C.POINTER(C.c_float)]),
        "ca3dmm_mlp_save": (i, [p, C.c_char_p]),
        "ca3dmm_mlp_load": (i, [C.c_char_p, C.POINTER(p)]),
        "ca3dmm_kernel_launches": (C.c_ulonglong, []),
        "ca3dmm_engine_exec_host": (i, [EP, p, i, p, i, p, i]),
        "ca3dmm_device_wait_check": (i, [d, i]),
        "mat_redist_layouts_init": (i, [i, pi, i, pi, C.POINTER(p)]),
        "mat_redist_layouts_pieces": (i, [p]),
        "mat_redist_layouts_exec": (i, [p, C.POINTER(p), pi, C.POINTER(p), pi, p]),
        "mat_redist_layouts_free": (None, [C.POINTER(p)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class VComm:
    """Virtual communicator of p ranks (the reference's MPI_Comm)."""

    def __init__(self, p):
        self.h = C.c_void_p()
        if lib().ca3dmm_vcomm_create(int(p), C.byref(self.h)) != 0:
            raise ValueError("invalid number of virtual ranks: %r" % (p,))
        self.p = int(p)

    def __del__(self):
        try:
            if self.h:
                lib().ca3dmm_vcomm_free(C.byref(self.h))
        except Exception:
            pass


def device_wait_check(timeout_s, arrive):
    """ca3dmm_device_wait_check: 0, or ETIMEOUT when the bounded wait ran out."""
    return int(lib().ca3dmm_device_wait_check(float(timeout_s), int(arrive)))


def kernel_launches():
    """Kernels the library has launched since it was loaded (host count)."""
    return int(lib().ca3dmm_kernel_launches())


def calc_3d_decomposition_cannon(p, m, n, k):
    """src/partition.h:16-19 -> (mp, np, kp, rp)."""
    o = [C.c_int() for _ in range(4)]
    lib().calc_3d_decomposition_cannon(p, m, n, k, *[C.byref(x) for x in o])
    return tuple(x.value for x in o)


def calc_3d_decomposition_nk(p, n, k):
    """src/partition.h:27-30 -> (np, kp, rp)."""
    o = [C.c_int() for _ in range(3)]
    lib().calc_3d_decomposition_nk(p, n, k, *[C.byref(x) for x in o])
    return tuple(x.value for x in o)


def calc_block_spos_size(length, nblk, iblk):
    s, z = C.c_int(), C.c_int()
    lib().calc_block_spos_size(length, nblk, iblk, C.byref(s), C.byref(z))
    return s.value, z.value


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return x.data_ptr()
    return x.ctypes.data          # numpy array (host memory)


class Ca3dmmEngine:
    """Python mirror of ca3dmm_engine_{init,init_BTB,attach_workbuf,exec,free}.

    ``Ca3dmmEngine(m, n, k, trans_A, trans_B, p=..., proc_grid=None)`` folds
    the reference's SPMD call onto one GPU: the source blocks are the whole
    matrices and the output (``dst_C`` whole C unless a block is given) is
    written by ``exec``.  ``gemm_mode`` selects plain FP64 DMMA or the
    split-precision path.  ``workbuf`` may be a caller-owned device pointer
    (then the engine does not allocate; size via ``workbuf_bytes``).
    """

    def __init__(self, m, n, k, trans_A=0, trans_B=0, p=1, proc_grid=None, dst_C=True,
                 btb=False, dev_type=DEV_TYPE_CUDA, caller_workbuf=False):
        L = lib()
        self.comm = VComm(p)
        self.m, self.n, self.k = m, n, k
        self.btb = btb
        self.e = C.POINTER(Ca3dmmEngineS)()
        grid = (C.c_int * 3)(*proc_grid) if proc_grid is not None else None
        wb = C.c_size_t(0)
        wbp = C.byref(wb) if caller_workbuf else None
        if dst_C is True:
            dst = (0, m if not btb else n, 0, n)
        elif dst_C is None or dst_C is False:
            dst = (-1, -1, -1, -1)
        else:
            dst = tuple(dst_C)
        if btb:
            L.ca3dmm_engine_init_BTB(n, k, 0, k, 0, n, dst[0], dst[1], dst[2], dst[3],
                                     grid, self.comm.h, dev_type, C.byref(self.e), wbp)
        else:
            a_r, a_c = (k, m) if trans_A else (m, k)
            b_r, b_c = (n, k) if trans_B else (k, n)
            L.ca3dmm_engine_init(m, n, k, int(trans_A), int(trans_B), 0, a_r, 0, a_c, 0, b_r, 0,
                                 b_c, dst[0], dst[1], dst[2], dst[3], grid, self.comm.h,
                                 dev_type, C.byref(self.e), wbp)
        self.workbuf_bytes = wb.value if caller_workbuf else None

    @property
    def ok(self):
        return bool(self.e)

    @property
    def s(self):
        return self.e.contents

    def attach_workbuf(self, workbuf_d, workbuf_h=None):
        lib().ca3dmm_engine_attach_workbuf(self.e, _ptr(workbuf_h), _ptr(workbuf_d))

    def set_gemm_mode(self, mode, slices=7):
        return lib().ca3dmm_engine_set_gemm_mode(self.e, int(mode), int(slices))

    def set_stream(self, stream, sync=1):
        lib().ca3dmm_engine_set_stream(self.e, C.c_void_p(stream), int(sync))

    def set_raster(self, raster):
        """Tile rows per raster band of the GEMM tile order (L2 reuse)."""
        return lib().ca3dmm_engine_set_raster(self.e, int(raster))

    def set_tune(self, cfg):
        """ca3dmm_engine_set_tune: (mode, slices, kp, raster[, tile_n])."""
        c = _cfg(cfg)
        return lib().ca3dmm_engine_set_tune(self.e, C.byref(c))

    def get_tune(self):
        c = TuneCfg()
        lib().ca3dmm_engine_get_tune(self.e, C.byref(c))
        return c.tuple()

    def autotune(self, A, ldA, B, ldB, Cout, ldC, how=1):
        """ca3dmm_engine_autotune (how: 0 off, 1 model, 2 exhaustive); returns
        (rc, chosen configuration)."""
        c = TuneCfg()
        rc = lib().ca3dmm_engine_autotune(self.e, _ptr(A), int(ldA), _ptr(B), int(ldB),
                                          _ptr(Cout), int(ldC), int(how), C.byref(c))
        return rc, c.tuple()

    def tune_report(self):
        """[(configuration, ms, guard error)] of the last tuning (ms -1 not
        timed, -2 rejected by the accuracy guard)."""
        n = 32
        cf = (TuneCfg * n)()
        ms = (C.c_float * n)()
        er = (C.c_float * n)()
        got = lib().ca3dmm_engine_tune_report(self.e, cf, ms, er, n)
        return [(cf[i].tuple(), ms[i], er[i]) for i in range(max(0, min(got, n)))]

    def required_workbuf_bytes(self):
        return lib().ca3dmm_engine_workbuf_bytes(self.e)

    def exec(self, A, ldA, B, ldB, Cout=None, ldC=0):
        lib().ca3dmm_engine_exec(self.e, _ptr(A), int(ldA), _ptr(B), int(ldB), _ptr(Cout),
                                 int(ldC))
        return lib().ca3dmm_engine_last_error(self.e)

    def exec_host(self, A, ldA, B, ldB, Cout, ldC):
        """ca3dmm_engine_exec_host: host (preferably page-locked) buffers in and
        out, copies overlapped with the computation."""
        return lib().ca3dmm_engine_exec_host(self.e, _ptr(A), int(ldA), _ptr(B), int(ldB),
                                             _ptr(Cout), int(ldC))

    def vrank_info(self, r):
        out = (C.c_int * 34)()
        rc = lib().ca3dmm_engine_vrank_info(self.e, int(r), out)
        if rc:
            raise ValueError("bad virtual rank %d" % r)
        return list(out)

    def reset_stat(self):
        lib().ca3dmm_engine_reset_stat(self.e)

    def print_stat(self):
        lib().ca3dmm_engine_print_stat(self.e)

    def free(self):
        if self.e:
            lib().ca3dmm_engine_free(C.byref(self.e))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class ThreadTransports:
    """ca3dmm_transport_threads_create: `size` transports for ranks that are
    threads of this process (host-staged exchange)."""

    def __init__(self, size):
        self.arr = (Transport * size)()
        self.rc = lib().ca3dmm_transport_threads_create(int(size), self.arr)

    def __getitem__(self, r):
        return self.arr[r]

    def free(self):
        if self.rc == 0 and self.arr[0].ctx:
            lib().ca3dmm_transport_threads_free(self.arr)


class DistEngine:
    """Python mirror of ca3dmm_dist_engine_{init,exec,info,counts,stats,free}:
    one rank of the multi-GPU engine over a ca3dmm_transport_t.  Rectangles
    are (srow, nrow, scol, ncol)."""

    def __init__(self, m, n, k, ta, tb, src_A, src_B, dst_C, transport, proc_grid=None,
                 btb=False, gemm_mode=GEMM_PLAIN, slices=0):
        self.h = C.c_void_p()
        self.size = transport.size
        grid = (C.c_int * 3)(*proc_grid) if proc_grid is not None else None
        a = list(src_A) if src_A is not None else [0, 0, 0, 0]
        self.rc = lib().ca3dmm_dist_engine_init(int(m), int(n), int(k), int(ta), int(tb),
                                                int(bool(btb)), *[int(x) for x in a],
                                                *[int(x) for x in src_B],
                                                *[int(x) for x in dst_C], grid,
                                                C.byref(transport), int(gemm_mode), int(slices),
                                                C.byref(self.h))

    @property
    def ok(self):
        return self.rc == 0 and bool(self.h)

    def exec(self, A, ldA, B, ldB, Cout, ldC):
        return lib().ca3dmm_dist_engine_exec(self.h, _ptr(A), int(ldA), _ptr(B), int(ldB),
                                             _ptr(Cout), int(ldC))

    def info(self):
        out = (C.c_int * 10)()
        lib().ca3dmm_dist_engine_info(self.h, out)
        return list(out)

    def counts(self):
        arrs = [(C.c_longlong * self.size)() for _ in range(4)]
        lib().ca3dmm_dist_engine_counts(self.h, *arrs)
        return [list(a) for a in arrs]

    def stats(self):
        out = (C.c_double * 4)()
        n = lib().ca3dmm_dist_engine_stats(self.h, out)
        return n, list(out)

    def free(self):
        if self.h:
            lib().ca3dmm_dist_engine_free(C.byref(self.h))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class CannonEngine:
    """Python mirror of cannon_engine_{init,exec,free} (np_dim^2 virtual ranks)."""

    def __init__(self, m, n, k, p=1, dev_type=DEV_TYPE_CUDA):
        self.comm = VComm(p)
        self.e = C.POINTER(CannonEngineS)()
        lib().cannon_engine_init(m, n, k, self.comm.h, dev_type, C.byref(self.e), None)

    @property
    def ok(self):
        return bool(self.e)

    @property
    def s(self):
        return self.e.contents

    def exec(self, alpha, beta, A, B, Cm):
        lib().cannon_engine_exec(self.e, float(alpha), float(beta), _ptr(A), _ptr(B), _ptr(Cm))
        return self.e.contents.last_error

    def free(self):
        if self.e:
            lib().cannon_engine_free(C.byref(self.e))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class GroupedGemm:
    """Python mirror of ca3dmm_grouped_{init,exec,free}: a batch of independent
    C_i = op(A_i) op(B_i) run as one persistent grouped launch."""

    def __init__(self, ms, ns, ks, trans_a=None, trans_b=None, mode=GEMM_PLAIN, slices=7):
        L = lib()
        npb = len(ms)
        arr = lambda v: (C.c_int * npb)(*[int(x) for x in v])
        self.n = npb
        self.ms, self.ns, self.ks = list(ms), list(ns), list(ks)
        self.ta = list(trans_a) if trans_a is not None else [0] * npb
        self.tb = list(trans_b) if trans_b is not None else [0] * npb
        self.h = C.c_void_p()
        self.rc = L.ca3dmm_grouped_init(npb, arr(ms), arr(ns), arr(ks), arr(self.ta), arr(self.tb),
                                        int(mode), int(slices), C.byref(self.h), None)

    @property
    def ok(self):
        return self.rc == 0 and bool(self.h)

    def set_stream(self, stream, sync=1):
        lib().ca3dmm_grouped_set_stream(self.h, C.c_void_p(stream), int(sync))

    def exec(self, A, ldA, B, ldB, Cs, ldC):
        npb = self.n
        P = C.c_void_p * npb
        I = C.c_int * npb
        return lib().ca3dmm_grouped_exec(self.h, P(*[_ptr(x) for x in A]), I(*ldA),
                                         P(*[_ptr(x) for x in B]), I(*ldB),
                                         P(*[_ptr(x) for x in Cs]), I(*ldC))

    def last_ms(self):
        return lib().ca3dmm_grouped_last_ms(self.h)

    def free(self):
        if self.h:
            lib().ca3dmm_grouped_free(C.byref(self.h))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class RedistLayouts:
    """Python mirror of mat_redist_layouts_{init,exec,free}: redistribution of
    a row-major matrix between two layouts of rectangles {srow, scol, nrow,
    ncol} (the reference's mat_redist with every rank's call folded into one)."""

    def __init__(self, src_rects, req_rects):
        L = lib()
        sr = [int(x) for r in src_rects for x in r]
        rr = [int(x) for r in req_rects for x in r]
        self.nsrc, self.nreq = len(src_rects), len(req_rects)
        self.h = C.c_void_p()
        self.rc = L.mat_redist_layouts_init(self.nsrc, (C.c_int * len(sr))(*sr), self.nreq,
                                            (C.c_int * len(rr))(*rr), C.byref(self.h))

    @property
    def ok(self):
        return self.rc == 0 and bool(self.h)

    def pieces(self):
        return lib().mat_redist_layouts_pieces(self.h)

    def exec(self, src_blks, src_lds, dst_blks, dst_lds, stream=None):
        P1, P2 = C.c_void_p * self.nsrc, C.c_void_p * self.nreq
        return lib().mat_redist_layouts_exec(
            self.h, P1(*[_ptr(x) for x in src_blks]), (C.c_int * self.nsrc)(*src_lds),
            P2(*[_ptr(x) for x in dst_blks]), (C.c_int * self.nreq)(*dst_lds),
            C.c_void_p(stream) if stream is not None else None)

    def free(self):
        if self.h:
            lib().mat_redist_layouts_free(C.byref(self.h))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _fp(a):
    import numpy as np
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(C.POINTER(C.c_float))


def tune_features(m, n, k, ta, tb, cfg, spread):
    import numpy as np
    out = np.zeros(NFEAT, dtype=np.float32)
    c = _cfg(cfg)
    rc = lib().ca3dmm_tune_features(m, n, k, ta, tb, C.byref(c), float(spread),
                                    out.ctypes.data_as(C.POINTER(C.c_float)))
    if rc:
        raise ValueError("bad features request")
    return out


class CostModel:
    """Python mirror of ca3dmm_mlp_*: the FP32 MLP cost model trained and run by
    the library's CUDA kernels."""

    def __init__(self, nin=NFEAT, h1=64, h2=64, seed=1, path=None):
        self.h = C.c_void_p()
        if path is not None:
            rc = lib().ca3dmm_mlp_load(path.encode(), C.byref(self.h))
        else:
            rc = lib().ca3dmm_mlp_create(nin, h1, h2, seed, C.byref(self.h))
        if rc:
            raise RuntimeError("cost model creation failed: %d" % rc)

    @classmethod
    def default(cls):
        """The shipped model (DEFAULT_COST_MODEL)."""
        return cls(path=DEFAULT_COST_MODEL)

    @property
    def nparams(self):
        return lib().ca3dmm_mlp_nparams(self.h)

    def params(self):
        import numpy as np
        out = np.zeros(self.nparams, dtype=np.float32)
        lib().ca3dmm_mlp_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def set_params(self, p):
        a, ptr = _fp(p)
        return lib().ca3dmm_mlp_set_params(self.h, ptr)

    def fwd_bwd(self, X, y):
        import numpy as np
        X, xp = _fp(X)
        y, yp = _fp(y)
        loss = C.c_float()
        g = np.zeros(self.nparams, dtype=np.float32)
        rc = lib().ca3dmm_mlp_fwd_bwd(self.h, xp, yp, len(y), C.byref(loss),
                                      g.ctypes.data_as(C.POINTER(C.c_float)))
        if rc:
            raise RuntimeError("fwd_bwd failed: %d" % rc)
        return loss.value, g

    def train(self, X, y, epochs=200, batch=256, lr=3e-3, seed=7):
        X, xp = _fp(X)
        y, yp = _fp(y)
        loss = C.c_float()
        rc = lib().ca3dmm_mlp_train(self.h, xp, yp, len(y), epochs, batch, lr, seed, C.byref(loss))
        if rc:
            raise RuntimeError("training failed: %d" % rc)
        return loss.value

    def predict(self, X):
        import numpy as np
        X, xp = _fp(X)
        out = np.zeros(X.shape[0], dtype=np.float32)
        rc = lib().ca3dmm_mlp_predict(self.h, xp, X.shape[0], out.ctypes.data_as(C.POINTER(C.c_float)))
        if rc:
            raise RuntimeError("predict failed: %d" % rc)
        return out

    def save(self, path):
        return lib().ca3dmm_mlp_save(self.h, path.encode())

    def free(self):
        if self.h:
            lib().ca3dmm_mlp_free(C.byref(self.h))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def autotune(m, n, k, ta, tb, A, ldA, B, ldB, Cm, ldC, cands, spread=0.0, model=None, topk=2,
             reps=2, with_err=False):
    """Run ca3dmm_autotune; returns (best index, ms per candidate: -1 not
    timed, -2 rejected by the accuracy guard[, guard errors])."""
    import numpy as np
    arr = (TuneCfg * len(cands))(*[_cfg(c) for c in cands])
    best = C.c_int()
    ms = np.zeros(len(cands), dtype=np.float32)
    er = np.zeros(len(cands), dtype=np.float32)
    rc = lib().ca3dmm_autotune(m, n, k, ta, tb, _ptr(A), ldA, _ptr(B), ldB, _ptr(Cm), ldC, arr,
                               len(cands), float(spread), model.h if model is not None else None,
                               int(topk), int(reps), C.byref(best),
                               ms.ctypes.data_as(C.POINTER(C.c_float)),
                               er.ctypes.data_as(C.POINTER(C.c_float)))
    if rc:
        raise RuntimeError("autotune failed: %d" % rc)
    return (best.value, ms, er) if with_err else (best.value, ms)


def measure(m, n, k, ta, tb, A, ldA, B, ldB, Cm, ldC, cfg, reps=2):
    t = C.c_float()
    c = _cfg(cfg)
    rc = lib().ca3dmm_tune_measure(m, n, k, ta, tb, _ptr(A), ldA, _ptr(B), ldB, _ptr(Cm), ldC,
                                   C.byref(c), int(reps), C.byref(t))
    return (t.value if rc == 0 else None)
