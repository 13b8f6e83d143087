"""Python front of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Used by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
checker; the product never imports it.

  * seeded counter-based input generators (splitmix64 of (seed, i, j)) with
    the value distributions of each workload;
  * double-double truth for GEMM entries (oracle.c, Dot2), full or sampled;
  * error metrics against that truth;
  * the CA3DMM virtual-rank algorithm on the CPU with BLAS local GEMMs
    (numpy), restating src/ca3dmm.c:926-1372 -- the timed CPU baseline.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            from . import build_oracle  # noqa: F401
            build_oracle.build()
        L = C.CDLL(path)
        dp, lp, ip, i8p = (C.POINTER(C.c_double), C.POINTER(C.c_long), C.POINTER(C.c_int),
                           C.POINTER(C.c_int8))
        L.orc_dd_entries.argtypes = [dp, C.c_long, C.c_int, dp, C.c_long, C.c_int, C.c_int,
                                     C.c_int, lp, lp, dp, dp, dp]
        L.orc_dd_gemm.argtypes = [dp, C.c_long, C.c_int, dp, C.c_long, C.c_int, C.c_int, C.c_int,
                                  C.c_int, dp, dp, dp]
        L.orc_errors.argtypes = [C.c_int, dp, dp, dp, dp, C.c_double, dp]
        L.orc_rank_geometry.argtypes = [C.c_int] * 8 + [ip]
        L.orc_block_spos_size.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip]
        u8p = C.POINTER(C.c_int8)
        L.orc_ozaki_slice_rows.argtypes = [dp, C.c_long, C.c_int, C.c_int, C.c_int, C.c_int, u8p,
                                           ip]
        L.orc_ozaki_slice_cols.argtypes = [dp, C.c_long, C.c_int, C.c_int, C.c_int, C.c_int, u8p,
                                           ip]
        L.orc_ozaki_gemm.argtypes = [u8p, ip, u8p, ip, C.c_int, C.c_int, C.c_int, C.c_int, dp]
        L.orc_nonfinite_fixup.argtypes = [dp, C.c_long, C.c_int, dp, C.c_long, C.c_int, C.c_int,
                                          C.c_int, C.c_int, dp]
        llp = C.POINTER(C.c_longlong)
        L.orc_crt_modulus.argtypes = [C.c_int]
        L.orc_crt_bits.argtypes = [C.c_int, C.c_long]
        L.orc_crt_gemm.argtypes = [dp, C.c_long, C.c_int, dp, C.c_long, C.c_int, C.c_int,
                                   C.c_int, C.c_int, C.c_int, dp]
        L.orc_crt_modular.argtypes = [dp, C.c_long, C.c_int, dp, C.c_long, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, C.c_int, llp]
        L.orc_crt_exact.argtypes = [dp, C.c_long, C.c_int, dp, C.c_long, C.c_int, C.c_int,
                                    C.c_int, C.c_int, C.c_int, llp]
        L.orc_ozaki_kchunk.argtypes = [C.c_int]
        L.orc_ozaki_kchunk.restype = C.c_int
        fp = C.POINTER(C.c_float)
        L.orc_mlp_fwd_bwd.argtypes = [C.c_int] * 4 + [fp] * 9 + [fp] * 6
        L.orc_mlp_fwd_bwd.restype = C.c_float
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


# ---------------------------------------------------------------- generators
_M1, _M2, _G = np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB), np.uint64(
    0x9E3779B97F4A7C15)


def _mix(z):
    with np.errstate(over="ignore"):
        z = z + _G
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


def hash_grid(seed, nrow, ncol, salt=0):
    """uint64 hash of (seed, i, j) for an nrow x ncol column-major grid."""
    i = np.arange(nrow, dtype=np.uint64)[:, None]
    j = np.arange(ncol, dtype=np.uint64)[None, :]
    key = (np.uint64(seed) << np.uint64(42)) ^ (i << np.uint64(21)) ^ j ^ np.uint64(salt)
    return _mix(key)


def uniform01(h):
    return (h >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def gen_uniform(seed, nrow, ncol):
    """Entries uniform in [-1, 1) (the 2048^3 example workload)."""
    return np.asfortranarray(2.0 * uniform01(hash_grid(seed, nrow, ncol)) - 1.0)


def gen_signed_exp(seed, nrow, ncol, emin=-8, emax=8, unit=False):
    """sign * (1 + u) * 2^e with integer e uniform in [emin, emax] (the 8000^3 workload);
    unit=True gives u' * 2^e with u' uniform in [-1, 1) (the uneven batched GEMMs)."""
    u = uniform01(hash_grid(seed, nrow, ncol))
    h2 = hash_grid(seed, nrow, ncol, salt=0xD6E8FEB86659FD93)
    e = ((h2 >> np.uint64(32)) % np.uint64(emax - emin + 1)).astype(np.int64) + emin
    if unit:
        return np.asfortranarray(np.ldexp(2.0 * u - 1.0, e))
    s = np.where((h2 & np.uint64(1)) == 1, -1.0, 1.0)
    return np.asfortranarray(s * np.ldexp(1.0 + u, e))


def gen_btb(seed, nrow, ncol):
    """Column j ~ N(0, 1) * 10^{u_j}, u_j uniform in [-3, 3] (the tall-skinny B^T B workload)."""
    u1 = uniform01(hash_grid(seed, nrow, ncol))
    u2 = uniform01(hash_grid(seed, nrow, ncol, salt=0x5851F42D4C957F2D))
    z = np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)
    uj = uniform01(hash_grid(seed + 7, 1, ncol))[0] * 6.0 - 3.0
    return np.asfortranarray(z * (10.0 ** uj)[None, :])


def gen_example_fill(nrow, ncol, ci, cj):
    """examples/example_AB.c:107-128: X(i,j) = ci*i + cj*j in stored coordinates."""
    i = np.arange(nrow, dtype=np.float64)[:, None]
    j = np.arange(ncol, dtype=np.float64)[None, :]
    return np.asfortranarray(ci * i + cj * j)


# ---------------------------------------------------------------- truth
def dd_gemm(A, B, tA, tB, m, n, k):
    """Full double-double C = op(A) op(B): returns (hi, lo, |A||B|) m x n."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    hi = np.zeros((m, n), order="F")
    lo = np.zeros((m, n), order="F")
    ab = np.zeros((m, n), order="F")
    lib().orc_dd_gemm(_d(A), A.shape[0], int(tA), _d(B), B.shape[0], int(tB), m, n, k, _d(hi),
                      _d(lo), _d(ab))
    return hi, lo, ab


def dd_entries(A, B, tA, tB, k, ii, jj):
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    ii = np.ascontiguousarray(ii, dtype=np.int64)
    jj = np.ascontiguousarray(jj, dtype=np.int64)
    ne = len(ii)
    hi, lo, ab = np.zeros(ne), np.zeros(ne), np.zeros(ne)
    lp = C.POINTER(C.c_long)
    lib().orc_dd_entries(_d(A), A.shape[0], int(tA), _d(B), B.shape[0], int(tB), k, ne,
                         ii.ctypes.data_as(lp), jj.ctypes.data_as(lp), _d(hi), _d(lo), _d(ab))
    return hi, lo, ab


def sample_indices(m, n, seed=11, nrand=4096, nlines=2):
    """4096 random entries plus nlines full rows and columns (seeded)."""
    rng = np.random.default_rng(seed)
    ii = [rng.integers(0, m, nrand)]
    jj = [rng.integers(0, n, nrand)]
    for r in rng.integers(0, m, nlines):
        ii.append(np.full(n, r)); jj.append(np.arange(n))
    for c in rng.integers(0, n, nlines):
        ii.append(np.arange(m)); jj.append(np.full(m, c))
    return np.concatenate(ii).astype(np.int64), np.concatenate(jj).astype(np.int64)


def errors(Cvals, hi, lo, ab, tol=1e-12):
    """(max componentwise, max |dC|/(|A||B|), normwise, count over tol)."""
    Cvals = np.ascontiguousarray(Cvals, dtype=np.float64).ravel()
    hi = np.ascontiguousarray(hi).ravel()
    lo = np.ascontiguousarray(lo).ravel()
    ab = np.ascontiguousarray(ab).ravel()
    res = np.zeros(4)
    lib().orc_errors(len(Cvals), _d(Cvals), _d(hi), _d(lo), _d(ab), tol, _d(res))
    return {"componentwise": res[0], "vs_absprod": res[1], "normwise": res[2],
            "n_over_tol": int(res[3])}


def rank_geometry(m, n, k, mp, np_, kp, rank, is_btb=0):
    out = (C.c_int * 34)()
    lib().orc_rank_geometry(m, n, k, mp, np_, kp, rank, int(is_btb), out)
    return list(out)


def ozaki_slices_rows(A, tA, m, k, s):
    """Slices of the rows of op(A): (int8 [s, m, k], exponents [m])."""
    A = np.asfortranarray(A, dtype=np.float64)
    q = np.zeros((s, m, k), dtype=np.int8)
    e = np.zeros(m, dtype=np.int32)
    lib().orc_ozaki_slice_rows(_d(A), A.shape[0], int(tA), m, k, s,
                               q.ctypes.data_as(C.POINTER(C.c_int8)),
                               e.ctypes.data_as(C.POINTER(C.c_int)))
    return q, e


def ozaki_slices_cols(B, tB, k, n, s):
    B = np.asfortranarray(B, dtype=np.float64)
    q = np.zeros((s, n, k), dtype=np.int8)
    e = np.zeros(n, dtype=np.int32)
    lib().orc_ozaki_slice_cols(_d(B), B.shape[0], int(tB), k, n, s,
                               q.ctypes.data_as(C.POINTER(C.c_int8)),
                               e.ctypes.data_as(C.POINTER(C.c_int)))
    return q, e


def ozaki_kchunk(s):
    return lib().orc_ozaki_kchunk(int(s))


def ozaki_gemm(qa, ea, qb, eb, m, n, k, s):
    Cm = np.zeros((m, n), order="F")
    u8 = C.POINTER(C.c_int8)
    ip = C.POINTER(C.c_int)
    lib().orc_ozaki_gemm(np.ascontiguousarray(qa).ctypes.data_as(u8),
                         np.ascontiguousarray(ea, dtype=np.int32).ctypes.data_as(ip),
                         np.ascontiguousarray(qb).ctypes.data_as(u8),
                         np.ascontiguousarray(eb, dtype=np.int32).ctypes.data_as(ip),
                         m, n, k, s, _d(Cm))
    return Cm


def nonfinite_fixup(A, B, tA, tB, m, n, k, Cm):
    """IEEE value of the C entries in rows of op(A) / columns of op(B) that
    hold an Inf or a NaN (orc_nonfinite_fixup); Cm (m x n, Fortran order) is
    updated in place and returned."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    assert Cm.flags["F_CONTIGUOUS"] and Cm.dtype == np.float64
    lib().orc_nonfinite_fixup(_d(A), A.shape[0], int(tA), _d(B), B.shape[0], int(tB), m, n, k,
                              _d(Cm))
    return Cm


def crt_modulus(t):
    """Modulus t of the modular scheme's list (pairwise coprime, <= 256)."""
    return lib().orc_crt_modulus(int(t))


def crt_bits(nmod, k):
    """Integer width P of the modular scheme with nmod moduli and depth k."""
    return lib().orc_crt_bits(int(nmod), int(k))


def crt_gemm(A, B, tA, tB, m, n, k, P):
    """The modular scheme's result C (m x n, Fortran order) from the exact
    integer product of the P-bit row / column integers."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    Cm = np.zeros((m, n), order="F")
    lib().orc_crt_gemm(_d(A), A.shape[0], int(tA), _d(B), B.shape[0], int(tB), m, n, k, int(P),
                       _d(Cm))
    return Cm


def _i128(buf, m, n):
    lo = buf[0::2].astype(np.uint64).astype(object)
    hi = buf[1::2].astype(object)
    return np.array([int(h) * (1 << 64) + int(l) for l, h in zip(lo, hi)],
                    dtype=object).reshape((m, n), order="F")


def crt_exact_ints(A, B, tA, tB, m, n, k, P):
    """C' = sum_l a'_il b'_lj as Python integers (m x n object array)."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    buf = np.zeros(2 * m * n, dtype=np.int64)
    lib().orc_crt_exact(_d(A), A.shape[0], int(tA), _d(B), B.shape[0], int(tB), m, n, k, int(P),
                        buf.ctypes.data_as(C.POINTER(C.c_longlong)))
    return _i128(buf, m, n)


def crt_modular_ints(A, B, tA, tB, m, n, k, P, nmod):
    """The same integers through residues modulo nmod moduli and a Garner
    reconstruction (None when the modulus product is too small for P, k)."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    buf = np.zeros(2 * m * n, dtype=np.int64)
    rc = lib().orc_crt_modular(_d(A), A.shape[0], int(tA), _d(B), B.shape[0], int(tB), m, n, k,
                               int(P), int(nmod), buf.ctypes.data_as(C.POINTER(C.c_longlong)))
    return None if rc else _i128(buf, m, n)


# ---------------------------------------------------------------- CPU CA3DMM
def block_spos_size(length, nblk, iblk):
    """src/utils.c:26-48"""
    rem, bs0 = length % nblk, length // nblk
    if iblk < rem:
        return (bs0 + 1) * iblk, bs0 + 1
    return bs0 * iblk + rem, bs0


def cpu_ca3dmm(A, B, tA, tB, m, n, k, mp, np_, kp):
    """The reference's virtual-rank algorithm on the CPU (src/ca3dmm.c:926-1372):
    every active rank multiplies its A_2dmm x B_2dmm Cannon blocks with BLAS
    (numpy), the kp partial C planes are summed in rank order.  Returns C."""
    opA = A.T if tA else A
    opB = B.T if tB else B
    slabs = []
    tmn = mp // np_ if mp > np_ else 1
    tnn = np_ // mp if np_ > mp else 1
    for tk in range(kp):
        k0, kz = block_spos_size(k, kp, tk)
        Cs = np.zeros((m, n), order="F")
        for tm in range(tmn):
            m0, mz = block_spos_size(m, tmn, tm)
            for tn in range(tnn):
                n0, nz = block_spos_size(n, tnn, tn)
                side = min(mp, np_)
                for r in range(side):
                    rm0, rmz = block_spos_size(mz, side, r)
                    for c in range(side):
                        cn0, cnz = block_spos_size(nz, side, c)
                        a = opA[m0 + rm0:m0 + rm0 + rmz, k0:k0 + kz]
                        b = opB[k0:k0 + kz, n0 + cn0:n0 + cn0 + cnz]
                        Cs[m0 + rm0:m0 + rm0 + rmz, n0 + cn0:n0 + cn0 + cnz] = a @ b
        slabs.append(Cs)
    out = slabs[0]
    for s in slabs[1:]:
        out = out + s
    return out


# ---------------------------------------------------------------- MLP reference
def mlp_split(params, nin, h1, h2):
    p = np.asarray(params, dtype=np.float32)
    o = 0
    out = []
    for size in (h1 * nin, h1, h2 * h1, h2, h2, 1):
        out.append(p[o:o + size].copy())
        o += size
    return out


def mlp_fwd_bwd(params, X, y, nin, h1, h2):
    """CPU FP32 reference of the cost-model MLP (oracle.c section 7):
    returns (loss, yhat, flat gradients in the parameter layout)."""
    W1, b1, W2, b2, W3, b3 = mlp_split(params, nin, h1, h2)
    X = np.ascontiguousarray(X, dtype=np.float32)
    y = np.ascontiguousarray(y, dtype=np.float32)
    B = X.shape[0]
    g = [np.zeros_like(a) for a in (W1, b1, W2, b2, W3, b3)]
    yhat = np.zeros(B, dtype=np.float32)
    fp = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
    loss = lib().orc_mlp_fwd_bwd(B, nin, h1, h2, fp(X), fp(y), fp(W1), fp(b1), fp(W2), fp(b2),
                                 fp(W3), fp(b3), fp(yhat), fp(g[0]), fp(g[1]), fp(g[2]), fp(g[3]),
                                 fp(g[4]), fp(g[5]))
    return float(loss), yhat, np.concatenate(g)


# ---------------------------------------------------------------- reference CPU path
_ref = None


def ref_lib():
    """The reference's own CPU path compiled under vmpi (oracle/_ref), or None."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libref_ca3dmm.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.ref_ca3dmm.argtypes = [C.c_int] * 7 + [ip, dp, dp, dp, C.c_int, dp, ip, ip, C.c_double]
        L.ref_fault_run.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double]
        L.ref_redist.argtypes = [C.c_int, ip, ip, dp, C.c_int, dp, C.POINTER(C.c_longlong),
                                 C.c_double]
        _ref = L
    return _ref


def ref_ca3dmm(p, m, n, k, ta, tb, A, B, grid=None, ntest=1, btb=False, timeout=300.0):
    """Run the unmodified reference (DEV_TYPE_HOST, OpenBLAS) on p vmpi rank threads
    the way examples/example_AB.c does.  Returns (C, times [ntest x 2] of rank 0:
    total exec ms and matmul-only ms, per-rank geometry [p x 34], (mp, np, kp, rp))."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference CPU path not built (oracle/_ref)")
    A = np.asfortranarray(A if A is not None else np.zeros((1, 1)), dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    cm = n if btb else m
    Cm = np.zeros((cm, n), order="F")
    times = np.zeros((max(ntest, 1), 2))
    geom = np.zeros((p, 34), dtype=np.int32)
    gout = np.zeros(4, dtype=np.int32)
    g = (C.c_int * 3)(*grid) if grid is not None else None
    ip = C.POINTER(C.c_int)
    rc = L.ref_ca3dmm(p, m, n, k, int(ta), int(tb), int(btb), g, _d(A), _d(B), _d(Cm), ntest,
                      _d(times), geom.ctypes.data_as(ip), gout.ctypes.data_as(ip), float(timeout))
    if rc:
        raise RuntimeError("reference run failed")
    return Cm, times, geom, tuple(int(x) for x in gout)


def ref_redist(src_rects, req_rects, G, timeout=60.0):
    """The reference's own mat_redist on p = len(src_rects) vmpi rank threads
    (rank r: source rectangle src_rects[r], required rectangle req_rects[r],
    row-major {srow, scol, nrow, ncol} of the row-major matrix G).  Returns the
    p required blocks as row-major arrays."""
    L = ref_lib()
    if L is None:
        raise RuntimeError("reference CPU path not built (oracle/_ref)")
    p = len(src_rects)
    assert len(req_rects) == p
    G = np.ascontiguousarray(G, dtype=np.float64)
    sizes = [int(r[2]) * int(r[3]) for r in req_rects]
    offs = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    out = np.zeros(max(sum(sizes), 1))
    ip = C.POINTER(C.c_int)
    sr = np.ascontiguousarray(np.array(src_rects, dtype=np.int32).ravel())
    rr = np.ascontiguousarray(np.array(req_rects, dtype=np.int32).ravel())
    rc = L.ref_redist(p, sr.ctypes.data_as(ip), rr.ctypes.data_as(ip), _d(G), G.shape[1], _d(out),
                      offs.ctypes.data_as(C.POINTER(C.c_longlong)), float(timeout))
    if rc:
        raise RuntimeError("reference redistribution failed")
    return [out[o:o + z].reshape(int(r[2]), int(r[3])) for o, z, r in zip(offs, sizes, req_rects)]


def ref_fault_run(p, dead_rank, m=64, timeout=1.0):
    """One rank returns at once; the others must stop by timeout (nonzero)."""
    return ref_lib().ref_fault_run(p, dead_rank, m, float(timeout))


# ---------------------------------------------------------------- reference GPU path
_ref_cuda = None


def ref_cuda_lib():
    """The reference's own GPU path (USE_CUDA, cuda_proxy.cu rebuilt for sm_100a)
    under vmpi (oracle/_ref/libref_ca3dmm_cuda.so), or None."""
    global _ref_cuda
    if _ref_cuda is None:
        path = os.path.join(HERE, "_ref", "libref_ca3dmm_cuda.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.ref_ca3dmm_cuda.argtypes = [C.c_int] * 7 + [ip, dp, dp, dp, C.c_int, dp, ip, C.c_double]
        _ref_cuda = L
    return _ref_cuda


def ref_ca3dmm_cuda(p, m, n, k, ta, tb, A, B, grid=None, ntest=1, btb=False, timeout=300.0):
    """Run the unmodified reference with DEV_TYPE_CUDA (cuBLAS DGEMM, host-staged
    MPI steps) on p vmpi rank threads sharing one GPU, the way
    examples/example_AB.c does.  Returns (C, times [ntest x 2] of rank 0: total
    exec ms and matmul-only ms, (mp, np, kp, rp))."""
    L = ref_cuda_lib()
    if L is None:
        raise RuntimeError("reference GPU path not built (oracle/_ref)")
    A = np.asfortranarray(A if A is not None else np.zeros((1, 1)), dtype=np.float64)
    B = np.asfortranarray(B, dtype=np.float64)
    Cm = np.zeros((n if btb else m, n), order="F")
    times = np.zeros((max(ntest, 1), 2))
    gout = np.zeros(4, dtype=np.int32)
    g = (C.c_int * 3)(*grid) if grid is not None else None
    rc = L.ref_ca3dmm_cuda(p, m, n, k, int(ta), int(tb), int(btb), g, _d(A), _d(B), _d(Cm), ntest,
                           _d(times), gout.ctypes.data_as(C.POINTER(C.c_int)), float(timeout))
    if rc:
        raise RuntimeError("reference GPU run failed")
    return Cm, times, tuple(int(x) for x in gout)
