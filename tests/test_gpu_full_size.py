"""The benchmark configurations at their full sizes, checked through properties
that do not need the whole product on the CPU.

* split precision: sampled rows x sampled columns of C equal, bit for bit, the
  oracle's slicing and recombination (INT8 slices) or its 128-bit integer
  product (modular scheme) of those rows of op(A) and columns of op(B), slab
  by slab in slab order (each row's exponent depends on that row alone, so a
  row subset is scaled exactly as inside the full block);
* plain FP64: the same sampled entries within k u |A||B| of the double-double
  truth;
* B^T B: the split-precision C is exactly symmetric.

Operands are generated on the device (seeded torch generators with each
configuration's value distribution); only the sampled rows and columns come
back to the host."""
import numpy as np
import pytest

import ca3dmm_b200 as cb
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
U = 2.0 ** -53


def _signed_exp(n_elem, seed):
    """sign * (1 + u) * 2^e, e uniform in [-8, 8] (the 8000^3 workload)."""
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    u = torch.rand(n_elem, generator=g, device="cuda", dtype=torch.float64)
    e = torch.randint(-8, 9, (n_elem,), generator=g, device="cuda", dtype=torch.int32)
    s = torch.randint(0, 2, (n_elem,), generator=g, device="cuda", dtype=torch.int32) * 2 - 1
    return torch.ldexp(s.double() * (1.0 + u), e)


def _uniform(n_elem, seed, lo=-1.0, hi=1.0):
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    return torch.rand(n_elem, generator=g, device="cuda", dtype=torch.float64) * (hi - lo) + lo


def _rows(flat, nrow, ncol, sel, trans):
    """Rows `sel` of op(X) for a column-major nrow x ncol X (op = transpose if trans)."""
    cm = flat[: nrow * ncol].view(ncol, nrow)          # cm[c, r] = X(r, c)
    out = cm[sel, :] if trans else cm[:, sel].T
    return np.ascontiguousarray(out.cpu().numpy())


def _cols(flat, nrow, ncol, sel, trans):
    """Columns `sel` of op(X) as a k x len(sel) array."""
    cm = flat[: nrow * ncol].view(ncol, nrow)
    out = cm[:, sel] if trans else cm[sel, :].T
    return np.asfortranarray(out.cpu().numpy())


def _sample(n, count, seed):
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(n, size=min(count, n), replace=False))
    idx[0], idx[-1] = 0, n - 1                         # first and last row / column too
    return np.unique(idx)


def _oracle_split(ra, cb_, k, kp, s):
    """Slab-by-slab split-precision oracle for rows ra (r x k) and columns cb_ (k x c)."""
    out = None
    for sl in range(kp):
        k0, kz = orc.block_spos_size(k, kp, sl)
        a = np.asfortranarray(ra[:, k0:k0 + kz])
        b = np.asfortranarray(cb_[k0:k0 + kz, :])
        qa, ea = orc.ozaki_slices_rows(a, 0, a.shape[0], kz, s)
        qb, eb = orc.ozaki_slices_cols(b, 0, kz, b.shape[1], s)
        c = orc.ozaki_gemm(qa, ea, qb, eb, a.shape[0], b.shape[1], kz, s)
        out = c if out is None else out + c
    return out


def _oracle_crt(ra, cb_, k, nslab, nmod):
    """Modular oracle for rows ra and columns cb_, slab by slab (nslab k slabs)."""
    out = None
    for sl in range(nslab):
        k0, kz = orc.block_spos_size(k, nslab, sl)
        a = np.asfortranarray(ra[:, k0:k0 + kz])
        b = np.asfortranarray(cb_[k0:k0 + kz, :])
        c = orc.crt_gemm(a, b, 0, 0, a.shape[0], b.shape[1], kz, orc.crt_bits(nmod, kz))
        out = c if out is None else out + c
    return out


def _dd_ok(got, ra, cb_, k):
    hi, lo, ab = orc.dd_gemm(np.asfortranarray(ra), cb_, 0, 0, ra.shape[0], cb_.shape[1], k)
    err = orc.errors(np.asfortranarray(got).ravel(order="F"), hi.ravel(order="F"),
                     lo.ravel(order="F"), ab.ravel(order="F"))
    assert err["vs_absprod"] <= k * U, err


def _engine_run(m, n, k, ta, A, B, p, grid, mode, slices=7, btb=False):
    import torch
    e = cb.Ca3dmmEngine(m, n, k, ta, 0, p=p, proc_grid=grid, btb=btb)
    assert e.ok
    if mode == cb.GEMM_OZAKI:
        assert e.set_gemm_mode(mode, slices) == 0
    if mode == cb.GEMM_CRT:
        assert e.set_gemm_mode(mode, 0) == 0            # the engine's modulus count
    C = torch.empty(m * n, dtype=torch.float64, device="cuda")
    lda = 0 if btb else (k if ta else m)
    assert e.exec(None if btb else A, lda, B, k, C, m) == 0
    kp = e.s.kp
    if mode == cb.GEMM_CRT:
        kp = (kp, e.s.crt_moduli)
    e.free()
    return C, kp


def _check_square(n, ta, p, grid, gen, seed, nsel, mode):
    A = gen(n * n, seed)
    B = gen(n * n, seed + 1)
    C, kp = _engine_run(n, n, n, ta, A, B, p, grid, mode)
    ri = _sample(n, nsel, seed + 2)
    cj = _sample(n, nsel, seed + 3)
    ra = _rows(A, n, n, ri, ta)                         # op(A) rows, len(ri) x n
    cbm = _cols(B, n, n, cj, 0)                         # op(B) columns, n x len(cj)
    got = C.view(n, n).T[ri][:, cj].cpu().numpy()       # C(ri, cj)
    if mode == cb.GEMM_OZAKI:
        assert np.array_equal(got, _oracle_split(ra, cbm, n, kp, 7))
    elif mode == cb.GEMM_CRT:
        # one k slab below 131072, whatever the grid's kp
        assert np.array_equal(got, _oracle_crt(ra, cbm, n, 1, kp[1]))
    else:
        _dd_ok(got, ra, cbm, n)


@pytest.mark.parametrize("mode", [cb.GEMM_CRT, cb.GEMM_OZAKI, cb.GEMM_PLAIN])
@pytest.mark.parametrize("ta", [0, 1])
def test_8000cube_grid_4x2x3(cuda, mode, ta):
    """The headline configuration: 8000^3 on 24 virtual ranks, grid 4 x 2 x 3."""
    _check_square(8000, ta, 24, (4, 2, 3), _signed_exp, 101 + ta, 40, mode)


@pytest.mark.parametrize("mode", [cb.GEMM_CRT, cb.GEMM_OZAKI, cb.GEMM_PLAIN])
def test_2048cube_4_ranks(cuda, mode):
    """2048^3 on 4 virtual ranks with the reference's own grid choice (2 x 1 x 2)."""
    _check_square(2048, 0, 4, None, _uniform, 201, 64, mode)


@pytest.mark.parametrize("mode", [cb.GEMM_CRT, cb.GEMM_OZAKI, cb.GEMM_PLAIN])
def test_btb_1048576x512_grid_1x1x32(cuda, mode):
    """B^T B with B of 1,048,576 x 512 (columns N(0,1) 10^u, u in [-3, 3]) on grid 1x1x32."""
    import torch
    K, N = 1048576, 512
    g = torch.Generator(device="cuda")
    g.manual_seed(303)
    B = torch.randn(N, K, generator=g, device="cuda", dtype=torch.float64)
    u = torch.rand(N, generator=g, device="cuda", dtype=torch.float64) * 6.0 - 3.0
    B.mul_(torch.pow(10.0, u)[:, None])
    B = B.reshape(-1)                                   # column-major K x N
    C, kp = _engine_run(N, N, K, 0, None, B, 32, (1, 1, 32), mode, btb=True)
    nmod = 0
    if mode == cb.GEMM_CRT:
        kp, nmod = kp
    assert kp == 32
    sel = _sample(N, 16, 7)
    cols = _cols(B, K, N, sel, 0)                       # K x len(sel) columns of B
    Cm = C.view(N, N).T
    got = Cm[sel][:, sel].cpu().numpy()
    if mode == cb.GEMM_OZAKI:
        assert np.array_equal(got, _oracle_split(np.ascontiguousarray(cols.T), cols, K, kp, 7))
        assert torch.equal(Cm, Cm.T)
    elif mode == cb.GEMM_CRT:
        # the modular B^T B keeps the reference's kp slabs
        assert np.array_equal(got, _oracle_crt(np.ascontiguousarray(cols.T), cols, K, kp, nmod))
    else:
        _dd_ok(got, np.ascontiguousarray(cols.T), cols, K)


@pytest.mark.parametrize("mode", [cb.GEMM_CRT, cb.GEMM_OZAKI, cb.GEMM_PLAIN])
def test_256_uneven_gemms(cuda, mode):
    """256 independent GEMMs, m, n, k log-uniform in [64, 4096], random transposes."""
    import torch
    rng = np.random.default_rng(2024)
    dims = np.exp(rng.uniform(np.log(64), np.log(4096), size=(256, 3))).round().astype(int)
    tas = rng.integers(0, 2, 256)
    tbs = rng.integers(0, 2, 256)
    A, B, C, lda, ldb, ldc = [], [], [], [], [], []
    for i, (m, n, k) in enumerate(dims):
        A.append(_uniform(int(m * k), 5000 + i) * 2.0 ** int(i % 9 - 4))
        B.append(_uniform(int(k * n), 9000 + i))
        C.append(torch.empty(int(m * n), dtype=torch.float64, device="cuda"))
        lda.append(int(k if tas[i] else m))
        ldb.append(int(n if tbs[i] else k))
        ldc.append(int(m))
    g = cb.GroupedGemm([int(d[0]) for d in dims], [int(d[1]) for d in dims],
                       [int(d[2]) for d in dims], [int(t) for t in tas], [int(t) for t in tbs],
                       mode=mode, slices=7 if mode == cb.GEMM_OZAKI else 0)
    assert g.ok
    assert g.exec(A, lda, B, ldb, C, ldc) == 0
    for i, (m, n, k) in enumerate(dims):
        m, n, k = int(m), int(n), int(k)
        ri = _sample(m, 6, 100 + i)
        cj = _sample(n, 6, 300 + i)
        ar, ac = (k, m) if tas[i] else (m, k)
        br, bc = (n, k) if tbs[i] else (k, n)
        ra = _rows(A[i], ar, ac, ri, int(tas[i]))
        cbm = _cols(B[i], br, bc, cj, int(tbs[i]))
        got = C[i].view(n, m).T[ri][:, cj].cpu().numpy()
        if mode == cb.GEMM_OZAKI:
            assert np.array_equal(got, _oracle_split(ra, cbm, k, 1, 7)), i
        elif mode == cb.GEMM_CRT:
            # one modulus count for the batch (the deepest product's), P per product
            kmax = int(dims[:, 2].max())
            nm = next(x for x in range(8, 19) if orc.crt_bits(x, kmax) >= 51)
            assert np.array_equal(got, _oracle_crt(ra, cbm, k, 1, nm)), i
        else:
            _dd_ok(got, ra, cbm, k)
