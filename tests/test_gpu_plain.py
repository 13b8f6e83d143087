"""Plain FP64 DMMA path on the GPU against the double-double oracle."""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

U = 2.0 ** -53
pytestmark = pytest.mark.gpu


def _dd_check(Cg, A, B, ta, tb, m, n, k, full=True):
    if full:
        hi, lo, ab = orc.dd_gemm(A, B, ta, tb, m, n, k)
        err = orc.errors(Cg.ravel(order="F"), hi.ravel(order="F"), lo.ravel(order="F"),
                         ab.ravel(order="F"))
    else:
        ii, jj = orc.sample_indices(m, n)
        hi, lo, ab = orc.dd_entries(A, B, ta, tb, k, ii, jj)
        err = orc.errors(Cg[ii, jj], hi, lo, ab)
    # |C - T| <= gamma_k |A||B| with gamma_k ~ k u (blocked sums do better)
    assert err["vs_absprod"] <= max(k, 1) * U, err
    return err


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 3), (63, 65, 129), (128, 128, 16),
                                   (129, 257, 100), (300, 200, 1000), (1000, 999, 1001),
                                   (256, 384, 4099)])
def test_cannon_engine_gemm(cuda, m, n, k):
    A = orc.gen_uniform(1, m, k)
    B = orc.gen_uniform(2, k, n)
    dA, _ = to_dev(A)
    dB, _ = to_dev(B)
    dC = dev_zeros(m * n)
    ce = cb.CannonEngine(m, n, k, p=1)
    assert ce.ok
    assert ce.exec(1.0, 0.0, dA, dB, dC) == 0
    _dd_check(from_dev(dC, m, n), A, B, 0, 0, m, n, k)


def test_cannon_alpha_beta_and_unaligned(cuda):
    m, n, k = 131, 77, 259           # odd m, k: operands are packed before TMA
    A = orc.gen_uniform(3, m, k)
    B = orc.gen_uniform(4, k, n)
    C0 = orc.gen_uniform(5, m, n)
    dA, _ = to_dev(A)
    dB, _ = to_dev(B)
    dC, _ = to_dev(C0)
    ce = cb.CannonEngine(m, n, k, p=4)
    assert ce.ok and ce.s.np_dim == 2
    assert ce.exec(-0.5, 2.0, dA, dB, dC) == 0
    got = from_dev(dC, m, n)
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    want = -0.5 * (hi + lo) + 2.0 * C0
    assert np.max(np.abs(got - want) / (0.5 * ab + 2 * np.abs(C0))) <= k * U


ENGINE_CASES = [  # m, n, k, p, ta, tb, grid
    (256, 256, 256, 1, 0, 0, None),
    (600, 500, 700, 6, 0, 0, None),
    (600, 500, 700, 6, 1, 0, None),
    (600, 500, 700, 6, 0, 1, None),
    (600, 500, 700, 6, 1, 1, None),
    (517, 1031, 2049, 16, 0, 0, (2, 4, 2)),
    (1031, 517, 333, 12, 1, 0, None),
    (64, 80, 20000, 8, 0, 0, None),
    (5, 7, 3, 6, 0, 0, None),
    (2048, 2048, 2048, 4, 0, 0, None),
]


@pytest.mark.parametrize("m,n,k,p,ta,tb,grid", ENGINE_CASES)
def test_engine_vs_dd(cuda, m, n, k, p, ta, tb, grid):
    A = orc.gen_uniform(11, *((k, m) if ta else (m, k)))
    B = orc.gen_uniform(12, *((n, k) if tb else (k, n)))
    dA, lda = to_dev(A, pad_ld=A.shape[0] + 3)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid)
    assert e.ok
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    _dd_check(from_dev(dC, m, n), A, B, ta, tb, m, n, k, full=m * n * k <= 2e9)
    # repeated exec reuses the plan and gives the same bits
    got1 = from_dev(dC, m, n)
    dC.zero_()
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    assert np.array_equal(got1, from_dev(dC, m, n))


@pytest.mark.parametrize("m,n,k,p,ta,tb", [(2048, 2048, 2048, 4, 0, 0), (700, 900, 1100, 24, 1, 0),
                                           (333, 444, 555, 7, 0, 1)])
def test_example_ab_validation_rule(cuda, m, n, k, p, ta, tb):
    """examples/example_AB.c:222-313: deterministic fill, 0 entries over 1e-12."""
    A = orc.gen_example_fill(*((k, m) if ta else (m, k)), 0.19, 0.24)
    B = orc.gen_example_fill(*((n, k) if tb else (k, n)), 0.11, 0.12)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p)
    assert e.ok and e.exec(dA, lda, dB, ldb, dC, m) == 0
    Cg = from_dev(dC, m, n)
    ii, jj = orc.sample_indices(m, n, nrand=20000)
    hi, lo, ab = orc.dd_entries(A, B, ta, tb, k, ii, jj)
    err = orc.errors(Cg[ii, jj], hi, lo, ab, tol=1e-12)
    assert err["n_over_tol"] == 0, err
    # the reference checks against cblas_dgemm; numpy's BLAS stands in here
    ref = (A.T if ta else A) @ (B.T if tb else B)
    assert np.max(np.abs(Cg - ref) / np.abs(ref)) <= 1e-12


def test_btb_engine(cuda):
    n, k, p = 96, 5000, 8
    Bm = orc.gen_btb(3, k, n)
    dB, ldb = to_dev(Bm)
    dC = dev_zeros(n * n)
    for grid in (None, (1, 1, 8), (2, 2, 2)):
        e = cb.Ca3dmmEngine(n, n, k, p=p, btb=True, proc_grid=grid)
        assert e.ok
        assert e.exec(None, 0, dB, ldb, dC, n) == 0
        _dd_check(from_dev(dC, n, n), Bm, Bm, 1, 0, n, n, k)


def test_dst_block_and_c_out(cuda):
    m, n, k = 300, 260, 410
    A = orc.gen_uniform(21, m, k)
    B = orc.gen_uniform(22, k, n)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    ref = A @ B
    # a sub-block of C as the destination (row range 50..249, column range 10..139)
    e = cb.Ca3dmmEngine(m, n, k, p=6, dst_C=(50, 200, 10, 130))
    dC = dev_zeros(210 * 130)
    assert e.ok and e.exec(dA, lda, dB, ldb, dC, 210) == 0
    got = from_dev(dC, 200, 130, ld=210)
    assert np.max(np.abs(got - ref[50:250, 10:140])) <= 1e-12 * np.max(np.abs(ref))
    # no destination: the whole C stays in the engine's C_out buffer (ld = m)
    e2 = cb.Ca3dmmEngine(m, n, k, p=6, dst_C=None)
    assert e2.ok and e2.exec(dA, lda, dB, ldb, None, 0) == 0
    import torch
    s = e2.s
    assert (s.C_out_srow, s.C_out_scol, s.C_out_nrow, s.C_out_ncol) == (0, 0, m, n)
    out = torch.empty(m * n, dtype=torch.float64, device="cuda")
    cb.lib().dev_type_memcpy(out.data_ptr(), s.C_out_d, m * n * 8, cb.DEV_TYPE_CUDA,
                             cb.DEV_TYPE_CUDA)
    assert np.max(np.abs(from_dev(out, m, n) - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_caller_workbuf_and_bad_ld(cuda):
    import torch
    m, n, k = 200, 150, 300
    A = orc.gen_uniform(31, m, k)
    B = orc.gen_uniform(32, k, n)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    e = cb.Ca3dmmEngine(m, n, k, p=4, caller_workbuf=True)
    assert e.ok and e.workbuf_bytes > 0
    wb = torch.empty(e.workbuf_bytes // 8 + 1, dtype=torch.float64, device="cuda")
    e.attach_workbuf(wb)
    dC = dev_zeros(m * n)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    assert np.max(np.abs(from_dev(dC, m, n) - A @ B)) <= 1e-12 * np.max(np.abs(A @ B))
    assert e.exec(dA, m - 1, dB, ldb, dC, m) == 1     # ldA < m is rejected, nothing runs


@pytest.mark.parametrize("k", [1600, 1601])
def test_transposed_a_in_place_matches_packed(cuda, k):
    """op(A) = A^T read K-major (even ldA: slabs with an aligned start in place,
    k = 1601's second slab, starting at the odd k index 801, copied into the
    K-major layout) gives the same bits as the transposing pack into the
    M-major layout (odd ldA): the DMMA sequence per output element is the same."""
    m, n = 700, 600
    A = orc.gen_uniform(41, k, m)
    B = orc.gen_uniform(42, k, n)
    dB, ldb = to_dev(B)
    outs = []
    even_ld = k + 2 - k % 2
    for ld in (even_ld, even_ld + 1):        # K-major (in place / copied), M-major (packed)
        dA, lda = to_dev(A, pad_ld=ld)
        dC = dev_zeros(m * n)
        e = cb.Ca3dmmEngine(m, n, k, 1, 0, p=8, proc_grid=(2, 2, 2))
        assert e.ok and e.exec(dA, lda, dB, ldb, dC, m) == 0
        outs.append(from_dev(dC, m, n))
    assert np.array_equal(outs[0], outs[1])
    _dd_check(outs[0], A, B, 1, 0, m, n, k)


@pytest.mark.parametrize("n,k,grid", [(200, 40000, (1, 1, 4)), (130, 9000, (1, 1, 2))])
def test_btb_k_split_sub_slabs(cuda, n, k, grid):
    """Few output tiles and long slabs: each slab's k range runs as several
    sub-slabs with their own C buffers, summed by the slab reduction."""
    Bm = orc.gen_btb(7, k, n)
    dB, ldb = to_dev(Bm)
    dC = dev_zeros(n * n)
    e = cb.Ca3dmmEngine(n, n, k, p=grid[2], btb=True, proc_grid=grid)
    assert e.ok and e.exec(None, 0, dB, ldb, dC, n) == 0
    _dd_check(from_dev(dC, n, n), Bm, Bm, 1, 0, n, n, k)


@pytest.mark.parametrize("ta,pad", [(0, 0), (0, 1), (1, 0)])
def test_plain_slabs_merged_when_tiles_suffice(cuda, ta, pad):
    """kp = 2 over a C of 25 x 25 = 625 tiles (>= 4 per SM): with every operand
    block read in place (even ld, M-major or K-major A) the two slabs run as one
    GEMM over all of k writing C directly; with an odd ldA (packed blocks) they
    run per slab and are summed.  Both stay within k u |A||B| (sampled), and
    the host-buffer exec gives the device exec's bits."""
    import torch
    m, n, k = 3200, 3100, 1500
    A = orc.gen_signed_exp(51, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(52, k, n)
    dA, lda = to_dev(A, pad_ld=A.shape[0] + pad)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = cb.Ca3dmmEngine(m, n, k, ta, 0, p=2, proc_grid=(1, 1, 2))
    assert e.ok and e.s.kp == 2
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    Cg = from_dev(dC, m, n)
    _dd_check(Cg, A, B, ta, 0, m, n, k, full=False)
    hA = np.zeros((lda, A.shape[1]), order="F")
    hA[:A.shape[0], :] = A
    hC = torch.zeros(m * n, dtype=torch.float64).pin_memory()
    hAt = torch.from_numpy(hA.ravel(order="F").copy()).pin_memory()
    hBt = torch.from_numpy(np.asfortranarray(B).ravel(order="F").copy()).pin_memory()
    assert e.exec_host(hAt, lda, hBt, ldb, hC, m) == 0
    if pad == 0:
        assert np.array_equal(hC.numpy().reshape(n, m).T, Cg)


def test_plain_slab_merge_can_be_switched_off(cuda, monkeypatch):
    """CA3DMM_PLAIN_MERGE_SLABS=0 keeps the kp-slab decomposition (per-slab
    GEMMs summed in slab order, the reference's rounding order) where the
    merged GEMM would run; both within k u |A||B|, and the two orders differ."""
    m, n, k = 3200, 3100, 1500
    A = orc.gen_signed_exp(61, m, k)
    B = orc.gen_signed_exp(62, k, n)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    outs = []
    for merge in ("1", "0"):
        monkeypatch.setenv("CA3DMM_PLAIN_MERGE_SLABS", merge)
        e = cb.Ca3dmmEngine(m, n, k, 0, 0, p=3, proc_grid=(1, 1, 3))
        dC = dev_zeros(m * n)
        assert e.ok and e.exec(dA, lda, dB, ldb, dC, m) == 0
        outs.append(from_dev(dC, m, n))
        _dd_check(outs[-1], A, B, 0, 0, m, n, k, full=False)
        e.free()
    assert not np.array_equal(outs[0], outs[1])


@pytest.mark.gpu
@pytest.mark.parametrize("nrow,ncol,lds,ldd", [(37, 300, 310, 305), (1, 1, 1, 1), (2000, 17, 20, 40)])
def test_dev_type_copy_mat_blk(cuda, nrow, ncol, lds, ldd):
    """dev_type_copy_mat_blk (src/dev_type.c:133-156): row-major nrow x ncol
    block copy, stream-ordered on the default stream; bit-exact."""
    import torch
    rng = np.random.default_rng(nrow + ncol)
    src = torch.from_numpy(rng.standard_normal(nrow * lds)).cuda()
    dst = torch.full((nrow * ldd,), -7.0, dtype=torch.float64, device="cuda")
    cb.lib().dev_type_copy_mat_blk(8, nrow, ncol, src.data_ptr(), lds, dst.data_ptr(), ldd,
                                   cb.DEV_TYPE_CUDA)
    torch.cuda.synchronize()
    s = src.cpu().numpy().reshape(nrow, lds)
    d = dst.cpu().numpy().reshape(nrow, ldd)
    assert np.array_equal(d[:, :ncol], s[:, :ncol])
    assert np.all(d[:, ncol:] == -7.0)


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid,pad", [
    (300, 200, 1000, 0, 0, 1, None, 0),
    (129, 65, 77, 1, 0, 1, None, 0),            # K-major A read in place
    (1000, 999, 1001, 0, 1, 6, None, 1),         # packed blocks (odd ldA)
    (700, 333, 2500, 1, 1, 4, (1, 1, 4), 0),    # kp slabs (k split)
    (3200, 3100, 1500, 0, 0, 2, (1, 1, 2), 0),  # slabs merged into one GEMM over k
    (2049, 63, 640, 0, 0, 24, (4, 2, 3), 0),    # several task blocks, a thin C
])
def test_plain_64_column_tiles_match_128(cuda, monkeypatch, m, n, k, ta, tb, p, grid, pad):
    """The DMMA GEMM with 128 x 64 output tiles (CA3DMM_PLAIN_TILE_N=64, or
    set_tune tile_n = 64) gives the 128 x 128 tiles' bits: every C entry is
    summed by one thread over the same k order either way.  The host-buffer
    exec (row bands over the 64-column tile numbering) gives the same bits."""
    import torch
    A = orc.gen_signed_exp(71, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(72, *((n, k) if tb else (k, n)))
    dA, lda = to_dev(A, pad_ld=A.shape[0] + pad)
    dB, ldb = to_dev(B)
    outs = []
    for tn in ("128", "64"):
        monkeypatch.setenv("CA3DMM_PLAIN_TILE_N", tn)
        e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid)
        assert e.ok
        dC = dev_zeros(m * n)
        assert e.exec(dA, lda, dB, ldb, dC, m) == 0
        outs.append(from_dev(dC, m, n))
        e.free()
    assert np.array_equal(outs[0], outs[1])
    _dd_check(outs[1], A, B, ta, tb, m, n, k, full=False)
    # set_tune switches the width on a live engine; exec_host over row bands
    monkeypatch.delenv("CA3DMM_PLAIN_TILE_N")
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid)
    assert e.set_tune((cb.GEMM_PLAIN, 0, e.s.kp, 8, 64)) == 0
    assert e.get_tune()[4] == 64
    hA = np.zeros((lda, A.shape[1]), order="F")
    hA[:A.shape[0], :] = A
    hAt = torch.from_numpy(hA.ravel(order="F").copy()).pin_memory()
    hBt = torch.from_numpy(np.asfortranarray(B).ravel(order="F").copy()).pin_memory()
    hC = torch.zeros(m * n, dtype=torch.float64).pin_memory()
    assert e.exec_host(hAt, lda, hBt, ldb, hC, m) == 0
    assert np.array_equal(hC.numpy().reshape(n, m).T, outs[0])
    e.free()


def test_plain_64_column_tiles_refused_for_symmetric_btb(cuda, monkeypatch):
    """The symmetric B^T B plan tiles C by 128-row block rows: a 64-column tile
    is refused there (set_tune returns CA3DMM_EINVAL; the variable is ignored)."""
    monkeypatch.setenv("CA3DMM_BTB_SYMMETRIC", "1")
    e = cb.Ca3dmmEngine(256, 256, 1000, btb=True, p=1)
    assert e.ok
    assert e.set_tune((cb.GEMM_PLAIN, 0, 1, 8, 64)) == cb.EINVAL
    assert e.set_tune((cb.GEMM_PLAIN, 0, 1, 8, 0)) == 0
    e.free()


@pytest.mark.parametrize("n,k,grid", [(300, 2000, (1, 1, 4)), (257, 5000, None)])
def test_plain_64_column_tiles_btb(cuda, monkeypatch, n, k, grid):
    """B^T B with 128 x 64 tiles (the plan of kp slabs, the host-buffer exec
    pipelined over them) gives the 128 x 128 tiles' bits."""
    import torch
    Bm = orc.gen_signed_exp(81, k, n)
    dB, ldb = to_dev(Bm)
    outs = []
    for tn in ("128", "64"):
        monkeypatch.setenv("CA3DMM_PLAIN_TILE_N", tn)
        e = cb.Ca3dmmEngine(n, n, k, btb=True, p=grid[2] if grid else 4, proc_grid=grid)
        assert e.ok
        dC = dev_zeros(n * n)
        assert e.exec(None, 0, dB, ldb, dC, n) == 0
        outs.append(from_dev(dC, n, n))
        if tn == "64":
            hB = torch.from_numpy(np.asfortranarray(Bm).ravel(order="F").copy()).pin_memory()
            hC = torch.zeros(n * n, dtype=torch.float64).pin_memory()
            assert e.exec_host(None, 0, hB, ldb, hC, n) == 0
            assert np.array_equal(hC.numpy().reshape(n, n).T, outs[0])
        e.free()
    assert np.array_equal(outs[0], outs[1])
