"""Modular split precision (CA3DMM_GEMM_CRT) against the oracle.

Bit-exact: the device forms the exact integer product of the P-bit row /
column integers from one INT8 tensor-core GEMM per modulus and the Chinese
remainder theorem, and rounds it once; the oracle forms the same integers
directly in 128-bit arithmetic (oracle/oracle.c section 8), so every C entry
must be equal.  Accuracy: at 15 moduli (P = 51 at k = 8000) the error
against the double-double truth is well below the plain FP64 error.
"""
import numpy as np
import pytest
import torch

import ca3dmm_b200 as cb
from oracle import oracle as orc
from tests._util import dev_zeros, from_dev, to_dev

pytestmark = pytest.mark.gpu
MAX_K = 131072


def _engine(m, n, k, ta, tb, p, grid, nmod, btb=False):
    e = cb.Ca3dmmEngine(m, n, k, ta, tb, p=p, proc_grid=grid, btb=btb)
    assert e.ok
    assert e.set_gemm_mode(cb.GEMM_CRT, nmod) == 0
    return e


def _run(A, B, m, n, k, ta, tb, p=1, grid=None, nmod=15):
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = _engine(m, n, k, ta, tb, p, grid, nmod)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    got = from_dev(dC, m, n)
    info = (e.s.crt_moduli, e.s.crt_bits)
    e.free()
    return got, info


def _oracle(A, B, m, n, k, ta, tb, nmod, btb=False, kp=1):
    """Slab sums in slab order: B^T B keeps the reference's kp slabs, other
    problems split k only above the exact INT32 range."""
    opA = np.asfortranarray(A.T if ta else A)
    opB = np.asfortranarray(B.T if tb else B)
    ns = kp if btb else max(1, -(-k // MAX_K))
    out = None
    for s in range(ns):
        k0, kz = orc.block_spos_size(k, ns, s)
        P = orc.crt_bits(nmod, kz)
        c = orc.crt_gemm(np.asfortranarray(opA[:, k0:k0 + kz]), np.asfortranarray(opB[k0:k0 + kz, :]),
                         0, 0, m, n, kz, P)
        out = c if out is None else out + c
    return orc.nonfinite_fixup(opA, opB, 0, 0, m, n, k, np.asfortranarray(out))


@pytest.mark.parametrize("m,n,k,ta,tb,p,grid,nmod", [
    (128, 256, 128, 0, 0, 1, None, 15),
    (1, 1, 1, 0, 0, 1, None, 8),
    (130, 70, 100, 0, 0, 1, None, 12),
    (300, 200, 777, 1, 0, 6, None, 15),
    (257, 129, 1000, 0, 1, 4, None, 16),
    (64, 500, 333, 1, 1, 1, None, 18),
    (1100, 1300, 1200, 0, 0, 24, (4, 2, 3), 15),   # several bands and tile columns
    (700, 300, 4000, 1, 0, 8, None, 0),            # automatic modulus count
])
def test_crt_bitexact(cuda, m, n, k, ta, tb, p, grid, nmod):
    A = orc.gen_signed_exp(51, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(52, *((n, k) if tb else (k, n)))
    got, (nm, P) = _run(A, B, m, n, k, ta, tb, p, grid, nmod)
    if nmod:
        assert nm == nmod
    assert P == orc.crt_bits(nm, k)
    want = _oracle(A, B, m, n, k, ta, tb, nm)
    assert np.array_equal(got, want), np.max(np.abs(got - want))


@pytest.mark.parametrize("tile_n", [256, 128])
def test_crt_edge_tiles_bitexact(cuda, monkeypatch, tile_n):
    """The last tile column holding 1 .. TN - 1 columns of C (the GEMM multiplies
    only those, rounded up to 16) and k ending anywhere in the last 128-byte k
    block (the k steps past k are not issued): bit-exact against the oracle."""
    monkeypatch.setenv("CA3DMM_CRT_TILE_N", str(tile_n))
    cases = [(130, 257, 1), (129, 256 + 15, 33), (128, 256 + 16, 64), (200, 256 + 17, 95),
             (64, 511, 96), (100, 255, 127), (70, 1, 129), (33, 384 + 112, 200),
             (260, 128 + 113, 32), (5, 16, 31)]
    for i, (m, n, k) in enumerate(cases):
        A = orc.gen_signed_exp(60 + i, m, k)
        B = orc.gen_signed_exp(80 + i, k, n)
        got, (nm, P) = _run(A, B, m, n, k, 0, 0, 1, None, 15)
        want = _oracle(A, B, m, n, k, 0, 0, nm)
        assert np.array_equal(got, want), (tile_n, m, n, k, np.max(np.abs(got - want)))


def test_crt_automatic_count_and_refusals(cuda):
    e = cb.Ca3dmmEngine(8000, 64, 8000, p=1)
    assert e.ok
    assert e.set_gemm_mode(cb.GEMM_CRT, 0) == 0
    assert e.s.crt_moduli == 15                      # fewest moduli with 51-bit integers at k = 8000
    assert e.set_gemm_mode(cb.GEMM_CRT, 7) == cb.EINVAL
    assert e.set_gemm_mode(cb.GEMM_CRT, 19) == cb.EINVAL
    assert e.s.crt_moduli == 15                      # a refused call changes nothing
    e.free()


def test_crt_error_below_plain(cuda):
    """Exponent-spread entries (e in [-8, 8]): the modular result at 15 moduli
    is at least twice as accurate as plain FP64, normwise and against
    |A||B|, on the full double-double truth."""
    m = n = k = 1024
    A = orc.gen_signed_exp(81, m, k)
    B = orc.gen_signed_exp(82, k, n)
    hi, lo, ab = orc.dd_gemm(A, B, 0, 0, m, n, k)
    errs = {}
    for mode, arg in ((cb.GEMM_PLAIN, 0), (cb.GEMM_CRT, 15)):
        dA, _ = to_dev(A)
        dB, _ = to_dev(B)
        dC = dev_zeros(m * n)
        e = cb.Ca3dmmEngine(m, n, k, 0, 0, p=4)
        assert e.ok and e.set_gemm_mode(mode, arg) == 0
        assert e.exec(dA, m, dB, k, dC, m) == 0
        e.free()
        C = from_dev(dC, m, n)
        errs[mode] = orc.errors(C.ravel(order="F"), hi.ravel(order="F"), lo.ravel(order="F"),
                                ab.ravel(order="F"))
    assert errs[cb.GEMM_CRT]["normwise"] * 2 <= errs[cb.GEMM_PLAIN]["normwise"], errs
    assert errs[cb.GEMM_CRT]["vs_absprod"] * 2 <= errs[cb.GEMM_PLAIN]["vs_absprod"], errs


def test_crt_btb_slabs(cuda):
    n, k, kp = 300, 20000, 8
    Bm = orc.gen_btb(9, k, n)
    dB, ldb = to_dev(Bm)
    e = cb.Ca3dmmEngine(n, n, k, p=kp, btb=True, proc_grid=(1, 1, kp))
    assert e.ok and e.set_gemm_mode(cb.GEMM_CRT, 16) == 0
    dC = dev_zeros(n * n)
    assert e.exec(None, 0, dB, ldb, dC, n) == 0
    got = from_dev(dC, n, n)
    e.free()
    want = _oracle(Bm, Bm, n, n, k, 1, 0, 16, btb=True, kp=kp)
    assert np.array_equal(got, want)
    assert np.array_equal(got, got.T)


def test_crt_deep_k_two_slabs(cuda):
    """k above the exact INT32 range of one GEMM: two k slabs, each with its
    own exponents and integer width, summed in slab order."""
    m, n, k = 70, 130, MAX_K + 9000
    A = orc.gen_signed_exp(13, m, k, emin=-2, emax=2)
    B = orc.gen_signed_exp(14, k, n, emin=-2, emax=2)
    got, (nm, P) = _run(A, B, m, n, k, 0, 0, 1, None, 16)
    assert P == orc.crt_bits(16, -(-k // 2))
    want = _oracle(A, B, m, n, k, 0, 0, 16)
    assert np.array_equal(got, want)


def _classes(C):
    return np.where(np.isnan(C), 3, np.where(np.isposinf(C), 1, np.where(np.isneginf(C), 2, 0)))


def test_crt_nonfinite(cuda):
    m, n, k = 333, 444, 555
    A = orc.gen_signed_exp(91, m, k)
    B = orc.gen_signed_exp(92, k, n)
    A[3, 10] = np.nan
    A[50, 11] = np.inf
    A[51, 12] = -np.inf
    B[20, 4] = np.inf
    B[:, 7] = 0.0
    A[9, :] = 0.0
    B[30, 100] = -np.inf
    got, (nm, _) = _run(A, B, m, n, k, 0, 0, 6, None, 15)
    with np.errstate(invalid="ignore", over="ignore"):
        ref = _classes(A @ B)
    assert np.array_equal(_classes(got), ref)
    want = _oracle(A, B, m, n, k, 0, 0, nm)
    fin = ref == 0
    assert np.array_equal(got[fin], want[fin])


@pytest.mark.parametrize("m,n,k,ta,p,grid", [(4100, 300, 900, 0, 24, (4, 2, 3)),
                                             (3000, 257, 700, 1, 6, None)])
def test_crt_exec_host_equals_device(cuda, m, n, k, ta, p, grid):
    A = orc.gen_signed_exp(11, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(12, k, n)
    A[17, 5] = np.nan
    e = _engine(m, n, k, ta, 0, p, grid, 15)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    want = from_dev(dC, m, n)
    hA = torch.from_numpy(A.ravel(order="F").copy()).pin_memory()
    hB = torch.from_numpy(B.ravel(order="F").copy()).pin_memory()
    hC = torch.zeros(m * n, dtype=torch.float64).pin_memory()
    for _ in range(2):
        hC.zero_()
        assert e.exec_host(hA, lda, hB, ldb, hC, m) == 0
        assert np.array_equal(hC.numpy().reshape((m, n), order="F"), want, equal_nan=True)


def test_crt_exec_host_btb(cuda):
    n, k, kp = 96, 5000, 8
    Bm = orc.gen_btb(7, k, n)
    e = cb.Ca3dmmEngine(n, n, k, p=kp, btb=True, proc_grid=(1, 1, kp))
    assert e.ok and e.set_gemm_mode(cb.GEMM_CRT, 16) == 0
    dB, ldb = to_dev(Bm)
    dC = dev_zeros(n * n)
    assert e.exec(None, 0, dB, ldb, dC, n) == 0
    want = from_dev(dC, n, n)
    hB = torch.from_numpy(Bm.ravel(order="F").copy()).pin_memory()
    hC = torch.zeros(n * n, dtype=torch.float64).pin_memory()
    for _ in range(2):
        hC.zero_()
        assert e.exec_host(None, 0, hB, ldb, hC, n) == 0
        assert np.array_equal(hC.numpy().reshape((n, n), order="F"), want)


def test_crt_grouped_batch_and_graph(cuda):
    """The modular mode on a batch of independent uneven GEMMs: bit-exact per
    problem against the oracle, then captured in a CUDA graph and replayed."""
    rng = np.random.default_rng(12)
    probs = []
    for i in range(30):
        m, n, k = (int(x) for x in np.exp(rng.uniform(np.log(16), np.log(900), 3)).round())
        ta, tb = int(rng.integers(0, 2)), int(rng.integers(0, 2))
        A = orc.gen_signed_exp(500 + i, *((k, m) if ta else (m, k)), emin=-4, emax=4)
        B = orc.gen_signed_exp(600 + i, *((n, k) if tb else (k, n)), emin=-4, emax=4)
        probs.append((m, n, k, ta, tb, A, B))
    g = cb.GroupedGemm([p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs],
                       [p[3] for p in probs], [p[4] for p in probs], mode=cb.GEMM_CRT, slices=0)
    assert g.ok
    dA, dB, dC, lda, ldb, ldc = [], [], [], [], [], []
    for m, n, k, ta, tb, A, B in probs:
        a, la = to_dev(A, pad_ld=A.shape[0] + 1)
        b, lb = to_dev(B)
        dA.append(a); lda.append(la); dB.append(b); ldb.append(lb)
        dC.append(dev_zeros(m * n)); ldc.append(m)
    assert g.exec(dA, lda, dB, ldb, dC, ldc) == 0
    kmax = max(p[2] for p in probs)
    nm = next(x for x in range(8, 19) if orc.crt_bits(x, kmax) >= 51)
    ref = []
    for i, (m, n, k, ta, tb, A, B) in enumerate(probs):
        got = from_dev(dC[i], m, n)
        want = _oracle(A, B, m, n, k, ta, tb, nm)
        assert np.array_equal(got, want), i
        ref.append(got)
    s = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    g.set_stream(s.cuda_stream, 0)
    with torch.cuda.graph(graph, stream=s):
        assert g.exec(dA, lda, dB, ldb, dC, ldc) == 0
    for _ in range(2):
        for c in dC:
            c.zero_()
        graph.replay()
        torch.cuda.synchronize()
        for i, p in enumerate(probs):
            assert np.array_equal(from_dev(dC[i], p[0], p[1]), ref[i]), i
    del graph


@pytest.mark.parametrize("band,m,n,k,ta", [(2, 1100, 700, 900, 0), (1, 1100, 500, 600, 1),
                                           (1, 2600, 300, 400, 0)])
def test_crt_bands_reconstructed_beside_the_gemm(cuda, monkeypatch, band, m, n, k, ta):
    """The device exec runs the GEMM band by band and reconstructs band b on a
    second stream beside the GEMM of band b + 1 (more than 16 bands: several
    per launch).  The result is the oracle's, bit for bit, and the same with
    the overlap switched off; graph capture of the two-stream exec replays it."""
    monkeypatch.setenv("CA3DMM_CRT_BAND", str(band))
    monkeypatch.setenv("CA3DMM_CRT_OVERLAP", "1")
    A = orc.gen_signed_exp(91, *((k, m) if ta else (m, k)))
    B = orc.gen_signed_exp(92, k, n)
    want = _oracle(A, B, m, n, k, ta, 0, 15)
    got, _ = _run(A, B, m, n, k, ta, 0, 1, None, 15)
    assert np.array_equal(got, want), np.max(np.abs(got - want))
    monkeypatch.setenv("CA3DMM_CRT_OVERLAP", "0")
    got0, _ = _run(A, B, m, n, k, ta, 0, 1, None, 15)
    assert np.array_equal(got0, want)
    monkeypatch.setenv("CA3DMM_CRT_OVERLAP", "1")
    # captured into a CUDA graph (the auxiliary stream forks and joins inside it)
    dA, lda = to_dev(A)
    dB, ldb = to_dev(B)
    dC = dev_zeros(m * n)
    e = _engine(m, n, k, ta, 0, 1, None, 15)
    s = torch.cuda.Stream()
    e.set_stream(s.cuda_stream, 1)
    assert e.exec(dA, lda, dB, ldb, dC, m) == 0          # plan upload outside the capture
    e.set_stream(s.cuda_stream, 0)
    g = torch.cuda.CUDAGraph()
    dC.zero_()
    torch.cuda.synchronize()
    with torch.cuda.graph(g, stream=s):
        assert e.exec(dA, lda, dB, ldb, dC, m) == 0
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(from_dev(dC, m, n), want)
    e.free()
