"""The C multi-GPU engine (include/ca3dmm_dist.h) on one B200: ranks are
threads of this process over the thread transport (host-staged exchange, the
reference's DEV_TYPE_CUDA), each with its own engine and device buffers; no
kernel waits on another rank.  Each rank holds the reference example's 1D
column blocks (or an irregular layout); the assembled C must be
  * bit-identical to the single-GPU engine on the same grid in INT8-slice
    mode (slab by slab, slab order),
  * bit-identical to the oracle's slab-by-slab modular product in the modular
    mode (each rank's local GEMM covers its slab),
  * within k u |A||B| of the double-double truth in plain FP64.
The C driver example_ab_dist (the reference's example_AB.c under mpirun -np p)
runs with 0 errors, and the NCCL transport carries a one-rank exchange."""
import os
import re
import subprocess
import threading

import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
U = 2.0 ** -53


def _blocks(m, n, k, ta, tb, p, r, irregular=False):
    ar, ac = (k, m) if ta else (m, k)
    br, bc = (n, k) if tb else (k, n)
    if irregular == "root":
        # rank 0 holds all of A and B, C in 1D column blocks
        c0, cz = cb.calc_block_spos_size(n, p, r)
        whole = lambda rows, cols: (0, rows, 0, cols) if r == 0 else (0, 0, 0, 0)
        return whole(ar, ac), whole(br, bc), (0, m, c0, cz)
    if not irregular:
        a0, az = cb.calc_block_spos_size(ac, p, r)
        b0, bz = cb.calc_block_spos_size(bc, p, r)
        c0, cz = cb.calc_block_spos_size(n, p, r)
        return (0, ar, a0, az), (0, br, b0, bz), (0, m, c0, cz)
    # row blocks of A, column blocks of B, row blocks of C
    a0, az = cb.calc_block_spos_size(ar, p, r)
    b0, bz = cb.calc_block_spos_size(bc, p, r)
    c0, cz = cb.calc_block_spos_size(m, p, r)
    return (a0, az, 0, ac), (0, br, b0, bz), (c0, cz, 0, n)


def _dist_run(A, B, m, n, k, ta, tb, p, grid, mode, slices, irregular=False, reps=2):
    tr = cb.ThreadTransports(p)
    assert tr.rc == 0
    C = np.full((m, n), np.nan, order="F")
    errs = [None] * p
    infos = [None] * p

    def body(r):
        sa, sb, dc = _blocks(m, n, k, ta, tb, p, r, irregular)
        blk = lambda X, rc: np.asfortranarray(X[rc[0]:rc[0] + rc[1], rc[2]:rc[2] + rc[3]])
        dA, lda = to_dev(blk(A, sa)) if sa[1] * sa[3] else (dev_zeros(1), 1)
        dB, ldb = to_dev(blk(B, sb)) if sb[1] * sb[3] else (dev_zeros(1), 1)
        dC = dev_zeros(dc[1] * dc[3])
        e = cb.DistEngine(m, n, k, ta, tb, sa, sb, dc, tr[r], proc_grid=grid, gemm_mode=mode,
                          slices=slices)
        if not e.ok:
            errs[r] = "init %d" % e.rc
            return
        infos[r] = e.info()
        for _ in range(reps):
            rc = e.exec(dA, max(lda, 1), dB, max(ldb, 1), dC, max(dc[1], 1))
            if rc:
                errs[r] = "exec %d" % rc
                e.free()
                return
        if dc[1] * dc[3]:
            C[dc[0]:dc[0] + dc[1], dc[2]:dc[2] + dc[3]] = from_dev(dC, dc[1], dc[3])
        e.free()

    th = [threading.Thread(target=body, args=(r,)) for r in range(p)]
    for t in th:
        t.start()
    for t in th:
        t.join(300)
    assert not any(t.is_alive() for t in th)
    tr.free()
    assert all(x is None for x in errs), errs
    return C, infos[0]


def _single(A, B, m, n, k, ta, tb, p, grid, mode, slices):
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid)
    assert e.set_gemm_mode(mode, slices) == 0
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    out = from_dev(dC, m, n)
    e.free()
    return out


def _crt_slabs(A, B, m, n, k, ta, tb, kp, nmod):
    opA = np.asfortranarray(A.T if ta else A)
    opB = np.asfortranarray(B.T if tb else B)
    out = None
    for s in range(kp):
        k0, kz = orc.block_spos_size(k, kp, s)
        nm = nmod
        if nm == 0:
            nm = next(x for x in range(8, 19) if orc.crt_bits(x, kz) >= 51)
        c = orc.crt_gemm(np.asfortranarray(opA[:, k0:k0 + kz]),
                         np.asfortranarray(opB[k0:k0 + kz, :]), 0, 0, m, n, kz, orc.crt_bits(nm, kz))
        out = c if out is None else out + c
    return out


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid,irregular", [
    (300, 200, 500, 0, 0, 4, None, False),
    (257, 129, 1000, 1, 0, 6, None, True),
    (400, 360, 2000, 0, 1, 8, (2, 2, 2), False),
    (1100, 1300, 1200, 1, 1, 12, (2, 2, 3), True),
])
@pytest.mark.parametrize("mode", [cb.GEMM_PLAIN, cb.GEMM_OZAKI, cb.GEMM_CRT])
def test_threads_match(cuda, m, n, k, ta, tb, p, grid, irregular, mode):
    A = orc.gen_signed_exp(71, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(72, *((n, k) if tb else (k, n)))
    slices = 7 if mode == cb.GEMM_OZAKI else 0
    got, info = _dist_run(A, B, m, n, k, ta, tb, p, grid, mode, slices, irregular)
    assert not np.isnan(got).any()
    if mode == cb.GEMM_OZAKI:
        want = _single(A, B, m, n, k, ta, tb, p, grid, mode, slices)
        assert np.array_equal(got, want)
    elif mode == cb.GEMM_CRT:
        want = _crt_slabs(A, B, m, n, k, ta, tb, info[2], 0)
        assert np.array_equal(got, want), np.max(np.abs(got - want))
    else:
        hi, lo, ab = orc.dd_gemm(A, B, ta, tb, m, n, k)
        assert np.all(np.abs(got - hi) <= k * U * ab + 1e-300)


@pytest.mark.parametrize("mode", [cb.GEMM_PLAIN, cb.GEMM_OZAKI])
def test_threads_operands_on_one_rank(cuda, mode):
    """Rank 0 holds all of A and B and C is split in 1D column blocks on the
    grid 1 x 1 x 8: every rank's C block (all of C for its slab) goes to all
    eight ranks while the other ranks send no operand piece, so the C
    exchange has more pieces than the operand exchange."""
    m, n, k, p, grid = 96, 96, 4096, 8, (1, 1, 8)
    A = orc.gen_signed_exp(91, m, k)
    B = orc.gen_signed_exp(92, k, n)
    slices = 7 if mode == cb.GEMM_OZAKI else 0
    got, info = _dist_run(A, B, m, n, k, 0, 0, p, grid, mode, slices, "root")
    assert tuple(info[:3]) == grid
    if mode == cb.GEMM_OZAKI:
        assert np.array_equal(got, _single(A, B, m, n, k, 0, 0, p, grid, mode, slices))
    else:
        hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
        assert np.all(np.abs(got - hi) <= k * U * ab + 1e-300)


def test_nccl_one_rank_exchange(cuda):
    """One NCCL rank whose dst_C is a sub-block: the operand and C exchanges run
    through NCCL (self send / receive on device buffers)."""
    m, n, k = 300, 250, 400
    A = orc.gen_uniform(81, m, k)
    B = orc.gen_uniform(82, k, n)
    import ctypes as C
    uid = (C.c_ubyte * 128)()
    assert cb.lib().ca3dmm_nccl_unique_id(uid) == 0
    t = cb.Transport()
    assert cb.lib().ca3dmm_transport_nccl_create(1, 0, uid, C.byref(t)) == 0
    assert t.device_buffers == 1
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dc = (20, 200, 30, 150)
    dC = dev_zeros(dc[1] * dc[3])
    e = cb.DistEngine(m, n, k, 0, 0, (0, m, 0, k), (0, k, 0, n), dc, t, gemm_mode=cb.GEMM_OZAKI,
                      slices=7)
    assert e.ok
    assert e.exec(dA, lda, dB, ldb, dC, dc[1]) == 0
    got = from_dev(dC, dc[1], dc[3])
    e.free()
    cb.lib().ca3dmm_transport_nccl_free(C.byref(t))
    full = _single(A, B, m, n, k, 0, 0, 1, None, cb.GEMM_OZAKI, 7)
    assert np.array_equal(got, full[20:220, 30:180])


@pytest.mark.parametrize("mode", ["0", "1", "2"])
def test_example_ab_dist(cuda, mode):
    exe = os.path.join(ROOT, "ca3dmm_b200", "examples", "example_ab_dist")
    r = subprocess.run([exe, "2048", "2048", "2048", "0", "0", "1", "2", "1"], capture_output=True,
                       text=True, timeout=600,
                       env=dict(os.environ, CA3DMM_DIST_RANKS="4", CA3DMM_GEMM_MODE=mode))
    out = r.stdout + r.stderr
    assert r.returncode == 0, out
    assert re.search(r"Process grid mp \* np \* kp  : 2 \* 1 \* 2", out), out
    assert "CA3DMM output : 0 error(s)" in out
    assert re.search(r"total execution  : [0-9]+ [0-9]+ \n", out), out
