/*
 * CPU oracle for the CA3DMM FP64 GEMM path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker.
 *
 * Contents
 *   1. Balanced 1D split          -- restates src/utils.c:26-48 (calc_block_spos_size)
 *   2. Per-virtual-rank geometry  -- restates src/ca3dmm.c:146-185 (task groups),
 *                                    src/ca3dmm.c:212-261 (block ranges, C_out split),
 *                                    src/ca3dmm.c:298-356 (A/B replication split),
 *                                    src/cannon.c:68-77 (Cannon block layout)
 *   3. Double-double GEMM entries -- Ogita/Rump/Oishi Dot2 (TwoProduct by fma,
 *                                    TwoSum); the truth for every error figure
 *   4. Error metrics              -- componentwise |dC|/|C| (examples/example_AB.c:296-304),
 *                                    |dC|/(|A||B|), normwise
 *   5. Closed-form answers        -- the example_AB / example_BTB deterministic fills
 *                                    (examples/example_AB.c:107-128, example_BTB.c:70-80)
 *   6. Ozaki slicing restatement  -- the split-precision path's exponent scaling and
 *                                    balanced base-256 INT8 slicing, bit-exact
 *   7. MLP cost-model reference   -- FP32 forward / backward / Adam for gradient checks
 */
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------- */
/* 1. Balanced split (src/utils.c:26-48)                                   */
/* ---------------------------------------------------------------------- */
void orc_block_spos_size(int len, int nblk, int iblk, int *spos, int *size)
{
    if (iblk < 0 || iblk > nblk) { *spos = -1; *size = 0; return; }
    int rem = len % nblk, bs0 = len / nblk;
    if (iblk < rem) { *spos = (bs0 + 1) * iblk; *size = bs0 + 1; }
    else            { *spos = bs0 * iblk + rem;  *size = bs0; }
}

/* ---------------------------------------------------------------------- */
/* 2. Per-virtual-rank geometry of the general (A*B) engine                */
/*    out[] layout (32 ints):                                              */
/*     0 is_active 1 rank_m 2 rank_n 3 rank_k 4 task_m_num 5 task_m_id      */
/*     6 task_n_num 7 task_n_id 8 task_k_num 9 task_k_id                    */
/*    10..13 A_2dmm srow,scol,nrow,ncol  14..17 B_2dmm  18..21 C_2dmm       */
/*    22..25 C_out srow,scol,nrow,ncol   26..29 A_rd srow,scol,nrow,ncol    */
/*    30..33 B_rd srow,scol,nrow,ncol (out must hold 34 ints)               */
/*    (src/ca3dmm.c:146-185, 212-261, 298-346; src/cannon.c:68-77)          */
/* ---------------------------------------------------------------------- */
void orc_rank_geometry(int m, int n, int k, int mp, int np, int kp, int rank,
                       int is_btb, int *out)
{
    memset(out, 0, sizeof(int) * 34);
    int active = rank < mp * np * kp;
    out[0] = active;
    if (!active) return;
    int rank_k = rank / (mp * np), rank_mn = rank % (mp * np);
    int rank_n = rank_mn / mp, rank_m = rank_mn % mp;
    int tmn = 1, tmi = 0, tnn = 1, tni = 0, nproc2d = mp * np;
    if (!is_btb) {
        if (mp > np) { tmn = mp / np; tmi = rank_mn / (np * np); nproc2d = np * np; }
        if (np > mp) { tnn = np / mp; tni = rank_mn / (mp * mp); nproc2d = mp * mp; }
    }
    out[1] = rank_m; out[2] = rank_n; out[3] = rank_k;
    out[4] = tmn; out[5] = tmi; out[6] = tnn; out[7] = tni; out[8] = kp; out[9] = rank_k;
    int tms, tmz, tns, tnz, tks, tkz;
    orc_block_spos_size(m, tmn, tmi, &tms, &tmz);
    orc_block_spos_size(n, tnn, tni, &tns, &tnz);
    orc_block_spos_size(k, kp, rank_k, &tks, &tkz);
    /* Cannon rank inside the 2D group: the group communicator is split with
     * key = global rank, so the in-group rank is the position of this rank
     * among the group's members, which are consecutive in rank_mn order. */
    int in_group = rank_mn % nproc2d;
    int npd = (int) sqrt((double) nproc2d);
    /* MPI_Cart_create with reorder: the engine keeps row-major coords of the
     * in-group rank (coords[0] = rank / npd). */
    int rr = in_group / npd, rc = in_group % npd;
    int As, An, Aks, Akn, Bks, Bkn, Bs, Bn, Cs, Cn, Ccs, Ccn;
    orc_block_spos_size(tmz, npd, rr, &As, &An);
    orc_block_spos_size(tkz, npd, rc, &Aks, &Akn);
    orc_block_spos_size(tkz, npd, rr, &Bks, &Bkn);
    orc_block_spos_size(tnz, npd, rc, &Bs, &Bn);
    orc_block_spos_size(tmz, npd, rr, &Cs, &Cn);
    orc_block_spos_size(tnz, npd, rc, &Ccs, &Ccn);
    out[10] = tms + As;  out[11] = tks + Aks; out[12] = An;  out[13] = Akn;
    out[14] = tks + Bks; out[15] = tns + Bs;  out[16] = Bkn; out[17] = Bn;
    out[18] = tms + Cs;  out[19] = tns + Ccs; out[20] = Cn;  out[21] = Ccn;
    int cos_, con;
    orc_block_spos_size(Ccn, kp, rank_k, &cos_, &con);
    out[22] = out[18]; out[23] = out[19] + cos_; out[24] = Cn; out[25] = con;
    /* redistribution request (before any transpose swap) */
    out[26] = out[10]; out[27] = out[11]; out[28] = out[12]; out[29] = out[13];
    out[30] = out[14]; out[31] = out[15]; out[32] = out[16]; out[33] = out[17];
    if (!is_btb && tnn > 1) {
        int s, z; orc_block_spos_size(out[13], tnn, tni, &s, &z);
        out[27] = out[11] + s; out[29] = z;
    }
    if (!is_btb && tmn > 1) {
        int s, z; orc_block_spos_size(out[17], tmn, tmi, &s, &z);
        out[31] = out[15] + s; out[33] = z;
    }
}

/* ---------------------------------------------------------------------- */
/* 3. Double-double dot products (Ogita, Rump, Oishi 2005, "Accurate sum   */
/*    and dot product", Algorithm Dot2)                                    */
/* ---------------------------------------------------------------------- */
static inline void two_sum(double a, double b, double *s, double *e)
{
    double x = a + b, z = x - a;
    *s = x; *e = (a - (x - z)) + (b - z);
}

/* A: op(A) element (i,l) = transA ? A[l + i*lda] : A[i + l*lda] */
static inline double opA(const double *A, long lda, int tA, long i, long l)
{ return tA ? A[l + i * lda] : A[i + l * lda]; }
static inline double opB(const double *B, long ldb, int tB, long l, long j)
{ return tB ? B[j + l * ldb] : B[l + j * ldb]; }

/* One C(i,j) entry of op(A)*op(B) as a double-double hi+lo, plus sum |a||b| */
static void dd_entry(const double *A, long lda, int tA, const double *B, long ldb,
                     int tB, int k, long i, long j, double *hi, double *lo,
                     double *absdot)
{
    double s = 0.0, c = 0.0, ab = 0.0;
    for (long l = 0; l < k; l++) {
        double a = opA(A, lda, tA, i, l), b = opB(B, ldb, tB, l, j);
        double p = a * b, pe = fma(a, b, -p), q;
        two_sum(s, p, &s, &q);
        c += q + pe;
        ab += fabs(p);
    }
    two_sum(s, c, hi, lo);
    *absdot = ab;
}

/* Double-double reference for a list of (i,j) entries (OpenMP over entries). */
void orc_dd_entries(const double *A, long lda, int tA, const double *B, long ldb,
                    int tB, int k, int nent, const long *ii, const long *jj,
                    double *hi, double *lo, double *absdot)
{
    #pragma omp parallel for schedule(dynamic, 16)
    for (int e = 0; e < nent; e++)
        dd_entry(A, lda, tA, B, ldb, tB, k, ii[e], jj[e], hi + e, lo + e, absdot + e);
}

/* Full double-double GEMM (small sizes): C_hi/C_lo/absdot are m x n col-major. */
void orc_dd_gemm(const double *A, long lda, int tA, const double *B, long ldb, int tB,
                 int m, int n, int k, double *hi, double *lo, double *absdot)
{
    #pragma omp parallel for collapse(2) schedule(static)
    for (long j = 0; j < n; j++)
        for (long i = 0; i < m; i++)
            dd_entry(A, lda, tA, B, ldb, tB, k, i, j, hi + i + j * m, lo + i + j * m,
                     absdot + i + j * m);
}

/* ---------------------------------------------------------------------- */
/* 4. Error metrics against a double-double truth                          */
/*    res[0] = max |C - T| / |T|    (componentwise, entries with T != 0)    */
/*    res[1] = max |C - T| / (|A||B|)_ij                                    */
/*    res[2] = ||C - T||_F / ||T||_F                                        */
/*    res[3] = count of entries with |C - T|/|T| > tol (example_AB rule)     */
/* ---------------------------------------------------------------------- */
void orc_errors(int nent, const double *C, const double *hi, const double *lo,
                const double *absdot, double tol, double *res)
{
    double cw = 0, ab = 0, num = 0, den = 0, bad = 0;
    for (int e = 0; e < nent; e++) {
        double t = hi[e], d = (C[e] - hi[e]) - lo[e];
        double ad = fabs(d);
        if (t != 0.0) { double r = ad / fabs(t); if (r > cw) cw = r; if (r > tol) bad += 1; }
        else if (ad != 0.0) { cw = INFINITY; bad += 1; }
        if (absdot[e] > 0) { double r = ad / absdot[e]; if (r > ab) ab = r; }
        num += d * d; den += t * t;
    }
    res[0] = cw; res[1] = ab; res[2] = den > 0 ? sqrt(num / den) : sqrt(num); res[3] = bad;
}

/* ---------------------------------------------------------------------- */
/* 5. Closed forms for the example drivers' fills                          */
/*    example_AB: A(i,l) = 0.19 i + 0.24 l,  B(l,j) = 0.11 l + 0.12 j       */
/*    (stored-matrix coordinates, examples/example_AB.c:115,126).            */
/*    C(i,j) = sum_l opA(i,l) opB(l,j) is a quadratic in l, summed exactly  */
/*    with the stored (rounded) coefficients evaluated as the driver does   */
/*    is NOT closed form, so the known answer uses the exact real values    */
/*    0.19 etc. in double-double: it pins the example's validation rule.    */
/* ---------------------------------------------------------------------- */
void orc_fill_example_ab(double *X, int nrow, int ncol, double ci, double cj)
{
    for (long j = 0; j < ncol; j++)
        for (long i = 0; i < nrow; i++)
            X[i + j * (long) nrow] = ci * (double) i + cj * (double) j;
}

/* ---------------------------------------------------------------------- */
/* 6. Ozaki INT8 slicing (bit-exact restatement of the product's rule)     */
/*    Per row i of op(A) over l in [0,k): E_i = max over the row of the      */
/*    effective exponent of a: e + 1 if the frexp mantissa of |a| exceeds    */
/*    127/128, else e (so max|a| <= 2^E_i * 127/128); E_i = 0 for a zero row. */
/*    N = rint(a 2^(8s-1-E)) is written in balanced base-256 digits          */
/*    q_t in [-128, 127]:  N = sum_t q_t 256^(s-1-t), least significant digit */
/*    first: q = ((N + 128) mod 256) - 128, N = (N - q) / 256.  Hence          */
/*    a = sum_t q_t 2^(E-7-8t) + r with |r| <= 2^(E-8s).                      */
/*    out_q[t * m * k + i * k + l] (K-major int8), out_e[i] = E_i.            */
/* ---------------------------------------------------------------------- */
static int eff_exponent(double v)
{
    if (v == 0.0) return INT_MIN;
    int e;
    double m = frexp(fabs(v), &e);
    return m > 0.9921875 ? e + 1 : e;
}

static void slice_one(double a, int E, int s, int8_t *q, long stride)
{
    long long N = llrint(ldexp(a, 8 * s - 1 - E));
    for (int t = s - 1; t >= 0; t--) {
        long long d = ((N + 128) & 255) - 128;
        q[t * stride] = (int8_t) d;
        N = (N - d) / 256;
    }
}

static int row_exponent(double mxe)
{
    return mxe == INT_MIN ? 0 : (int) mxe;
}

/*    A row (or column) holding an Inf or a NaN is sliced as a zero row       */
/*    (E = 0, all digits 0); orc_nonfinite_fixup then gives its C entries     */
/*    their IEEE value.                                                       */
void orc_ozaki_slice_rows(const double *A, long lda, int tA, int m, int k, int s,
                          int8_t *out_q, int *out_e)
{
    for (long i = 0; i < m; i++) {
        int mx = INT_MIN, fin = 1;
        for (long l = 0; l < k; l++) {
            double v = opA(A, lda, tA, i, l);
            if (!isfinite(v)) { fin = 0; continue; }
            int e = eff_exponent(v);
            if (e > mx) mx = e;
        }
        int E = fin ? row_exponent(mx) : 0;
        out_e[i] = E;
        for (long l = 0; l < k; l++)
            slice_one(fin ? opA(A, lda, tA, i, l) : 0.0, E, s, out_q + i * k + l, (long) m * k);
    }
}

/* Same for the columns of op(B): column j over l. out_q[t*n*k + j*k + l]. */
void orc_ozaki_slice_cols(const double *B, long ldb, int tB, int k, int n, int s,
                          int8_t *out_q, int *out_e)
{
    for (long j = 0; j < n; j++) {
        int mx = INT_MIN, fin = 1;
        for (long l = 0; l < k; l++) {
            double v = opB(B, ldb, tB, l, j);
            if (!isfinite(v)) { fin = 0; continue; }
            int e = eff_exponent(v);
            if (e > mx) mx = e;
        }
        int E = fin ? row_exponent(mx) : 0;
        out_e[j] = E;
        for (long l = 0; l < k; l++)
            slice_one(fin ? opB(B, ldb, tB, l, j) : 0.0, E, s, out_q + j * k + l, (long) n * k);
    }
}

/* k range of one exactly-accumulated chunk: every diagonal sum
 * sum_{t+u=d} sum_l q_t q_u must stay below 2^31 with |q q| <= 2^14, i.e.
 * s * kc * 16384 < 2^31; kc is rounded down to the GEMM's 32-byte k step. */
int orc_ozaki_kchunk(int s)
{
    long kc = (2147483647L / 16384L) / s;
    return (int) (kc / 32 * 32);
}

/* Ozaki product from slices, for small sizes: per k chunk (orc_ozaki_kchunk),
 * diagonals d = t + u <= s - 1 as exact integer sums, recombined into one
 * running FP64 sum per entry: for each chunk in order, d = s-1 down to 0,
 * acc += 2^(-14 - 8d) * D_d (the product's order); then C = 2^(E_i + F_j) acc
 * with one rounding (ldexp).  C is m x n column-major. */
void orc_ozaki_gemm(const int8_t *qa, const int *ea, const int8_t *qb, const int *eb,
                    int m, int n, int k, int s, double *C)
{
    const int kc = orc_ozaki_kchunk(s);
    #pragma omp parallel for collapse(2) schedule(static)
    for (long j = 0; j < n; j++)
        for (long i = 0; i < m; i++) {
            double acc = 0.0;
            for (long c0 = 0; c0 < k || (k == 0 && c0 == 0); c0 += kc) {
                long c1 = c0 + kc < k ? c0 + kc : k;
                for (int d = s - 1; d >= 0; d--) {
                    long long sum = 0;
                    for (int t = 0; t <= d; t++) {
                        int u = d - t;
                        const int8_t *a = qa + (long) t * m * k + i * k;
                        const int8_t *b = qb + (long) u * n * k + j * k;
                        for (long l = c0; l < c1; l++)
                            sum += (long long) a[l] * b[l];
                    }
                    acc += ldexp((double) sum, -14 - 8 * d);
                }
                if (k == 0) break;
            }
            C[i + j * m] = ldexp(acc, ea[i] + eb[j]);
        }
}

/* IEEE value of the C entries whose row of op(A) or column of op(B) holds an
 * Inf or a NaN (every other entry is left as it is).  Each such entry is
 * non-finite whatever the summation order: NaN when a product is NaN (a NaN
 * factor, or Inf times 0) or products of both infinite signs occur, else the
 * infinity of the products' sign.  C is m x n column-major. */
void orc_nonfinite_fixup(const double *A, long lda, int tA, const double *B, long ldb, int tB,
                         int m, int n, int k, double *C)
{
    char *rbad = (char *) calloc((size_t) (m > 0 ? m : 1), 1);
    char *cbad = (char *) calloc((size_t) (n > 0 ? n : 1), 1);
    for (long i = 0; i < m; i++)
        for (long l = 0; l < k; l++) if (!isfinite(opA(A, lda, tA, i, l))) rbad[i] = 1;
    for (long j = 0; j < n; j++)
        for (long l = 0; l < k; l++) if (!isfinite(opB(B, ldb, tB, l, j))) cbad[j] = 1;
    for (long j = 0; j < n; j++)
        for (long i = 0; i < m; i++) {
            if (!rbad[i] && !cbad[j]) continue;
            int nan_ = 0, pinf = 0, ninf = 0;
            for (long l = 0; l < k; l++) {
                double a = opA(A, lda, tA, i, l), b = opB(B, ldb, tB, l, j);
                if (isnan(a) || isnan(b)) nan_ = 1;
                else if (isinf(a) || isinf(b)) {
                    if (a == 0.0 || b == 0.0) nan_ = 1;
                    else if (signbit(a) != signbit(b)) ninf = 1;
                    else pinf = 1;
                }
            }
            if (nan_ || (pinf && ninf)) C[i + j * m] = NAN;
            else if (pinf) C[i + j * m] = INFINITY;
            else if (ninf) C[i + j * m] = -INFINITY;
        }
    free(rbad);
    free(cbad);
}

/* ---------------------------------------------------------------------- */
/* 7. MLP cost model reference (FP32): in -> H1 (relu) -> H2 (relu) -> 1   */
/*    W1 [H1][in], b1[H1], W2 [H2][H1], b2[H2], W3[H2], b3[1].              */
/*    loss = mean over batch of 0.5 (y_hat - y)^2.                          */
/*    Gradients are accumulated (summed) over the batch then divided by B.  */
/* ---------------------------------------------------------------------- */
float orc_mlp_fwd_bwd(int B, int nin, int h1, int h2, const float *X, const float *y,
                      const float *W1, const float *b1, const float *W2, const float *b2,
                      const float *W3, const float *b3, float *yhat,
                      float *gW1, float *gb1, float *gW2, float *gb2, float *gW3, float *gb3)
{
    float *a1 = (float *) malloc(sizeof(float) * h1), *a2 = (float *) malloc(sizeof(float) * h2);
    float *d1 = (float *) malloc(sizeof(float) * h1), *d2 = (float *) malloc(sizeof(float) * h2);
    if (gW1) {
        memset(gW1, 0, sizeof(float) * h1 * nin); memset(gb1, 0, sizeof(float) * h1);
        memset(gW2, 0, sizeof(float) * h2 * h1);  memset(gb2, 0, sizeof(float) * h2);
        memset(gW3, 0, sizeof(float) * h2);       gb3[0] = 0.f;
    }
    double loss = 0.0;
    for (int b = 0; b < B; b++) {
        const float *x = X + (long) b * nin;
        for (int o = 0; o < h1; o++) {
            float s = b1[o];
            for (int i = 0; i < nin; i++) s += W1[o * nin + i] * x[i];
            a1[o] = s > 0.f ? s : 0.f;
        }
        for (int o = 0; o < h2; o++) {
            float s = b2[o];
            for (int i = 0; i < h1; i++) s += W2[o * h1 + i] * a1[i];
            a2[o] = s > 0.f ? s : 0.f;
        }
        float out = b3[0];
        for (int i = 0; i < h2; i++) out += W3[i] * a2[i];
        if (yhat) yhat[b] = out;
        if (!y) continue;
        float g = out - y[b];
        loss += 0.5 * (double) g * g;
        if (!gW1) continue;
        gb3[0] += g;
        for (int i = 0; i < h2; i++) { gW3[i] += g * a2[i]; d2[i] = a2[i] > 0.f ? g * W3[i] : 0.f; }
        for (int o = 0; o < h2; o++) {
            gb2[o] += d2[o];
            for (int i = 0; i < h1; i++) gW2[o * h1 + i] += d2[o] * a1[i];
        }
        for (int i = 0; i < h1; i++) {
            float s = 0.f;
            for (int o = 0; o < h2; o++) s += W2[o * h1 + i] * d2[o];
            d1[i] = a1[i] > 0.f ? s : 0.f;
        }
        for (int o = 0; o < h1; o++) {
            gb1[o] += d1[o];
            for (int i = 0; i < nin; i++) gW1[o * nin + i] += d1[o] * x[i];
        }
    }
    if (gW1 && B > 0) {
        float inv = 1.f / (float) B;
        for (int i = 0; i < h1 * nin; i++) gW1[i] *= inv;
        for (int i = 0; i < h1; i++) gb1[i] *= inv;
        for (int i = 0; i < h2 * h1; i++) gW2[i] *= inv;
        for (int i = 0; i < h2; i++) { gb2[i] *= inv; gW3[i] *= inv; }
        gb3[0] *= inv;
    }
    free(a1); free(a2); free(d1); free(d2);
    return B > 0 ? (float) (loss / B) : 0.f;
}

/* ---------------------------------------------------------------------- */
/* 8. Modular (CRT) split precision                                        */
/*    Row i of op(A): E_i = frexp exponent of max_l |a_il| (max < 2^E_i,    */
/*    0 for a zero row), a'_il = rint(a_il 2^(P - E_i)), |a'| <= 2^P; column */
/*    j of op(B) likewise (F_j, b').  C'_ij = sum_l a'_il b'_lj exactly     */
/*    (|C'| <= k 2^(2P)); the device obtains it from the residues of the    */
/*    products modulo N pairwise coprime moduli <= 256 (one INT8 GEMM each) */
/*    by the Chinese remainder theorem, which is exact while               */
/*    k 2^(2P+1) < M = prod p_t.  C_ij = (C' rounded to double, round to   */
/*    nearest even) 2^(E_i + F_j - 2P).  Rows / columns holding an Inf or a */
/*    NaN are zero rows here too (orc_nonfinite_fixup gives their entries). */
/* ---------------------------------------------------------------------- */
static const int crt_mod_list[18] = {256, 255, 253, 251, 247, 241, 239, 233, 229,
                                     227, 223, 217, 211, 199, 197, 193, 191, 181};

int orc_crt_modulus(int t) { return (t >= 0 && t < 18) ? crt_mod_list[t] : 0; }

/* Largest P <= 53 with k 2^(2P+1) < M_N (M_N the product of the first N moduli). */
int orc_crt_bits(int nmod, long k)
{
    double lm = 0.0;
    for (int t = 0; t < nmod && t < 18; t++) lm += log2((double) crt_mod_list[t]);
    double lk = log2((double) (k > 1 ? k : 1));
    int P = (int) floor((lm - 1.0 - lk - 1e-9) / 2.0);
    return P > 53 ? 53 : P;
}

/* a' of one row / column: exponent from the largest magnitude, then rint of
 * the scaled values (ldexp is exact; rint rounds half to even). */
static int crt_row_ints(const double *v, long n, long stride, int P, long long *out)
{
    double mx = 0.0;
    int fin = 1;
    for (long l = 0; l < n; l++) {
        double x = v[l * stride];
        if (!isfinite(x)) fin = 0;
        else if (fabs(x) > mx) mx = fabs(x);
    }
    int E = 0;
    if (fin && mx > 0.0) frexp(mx, &E);
    for (long l = 0; l < n; l++)
        out[l] = fin ? (long long) rint(ldexp(v[l * stride], P - E)) : 0;
    return E;
}

/* double of a signed integer below 2^127 in magnitude, rounded to nearest even,
 * times 2^e: a 64-bit window with the leading bit at bit 63 and the bits below
 * it ORed into bit 0, converted once, then scaled by a power of two (one more
 * rounding only if the result leaves the normal range).  Same steps as the
 * device. */
static double crt_to_double(__int128 c, int e)
{
    int neg = c < 0;
    unsigned __int128 mag = neg ? (unsigned __int128) (-c) : (unsigned __int128) c;
    uint64_t hi = (uint64_t) (mag >> 64), lo = (uint64_t) mag;
    double d;
    if (hi == 0) {
        d = (double) lo;     /* rounds to nearest even */
    } else {
        int lz = __builtin_clzll(hi);
        int sh = 64 - lz;                       /* bits below the window */
        unsigned __int128 top = mag >> sh;      /* < 2^64, leading bit at 63 */
        uint64_t w = (uint64_t) top;
        if ((mag & ((((unsigned __int128) 1) << sh) - 1)) != 0) w |= 1ull;
        /* w has bit 63 set: round to 53 bits, nearest even (round bit 10,
         * sticky bits 0-9) */
        uint64_t m53 = w >> 11, rb = (w >> 10) & 1, st = (w & 0x3ffull) != 0;
        if (rb && (st || (m53 & 1))) m53 += 1;
        d = ldexp((double) m53, 11);
        e += sh;
    }
    double r;
    if (e >= -1022 && e <= 1023) r = d * ldexp(1.0, e);
    else r = ldexp(d, e);
    return neg ? -r : r;
}

/* The CRT scheme's result (m x n, column-major C), from the exact integer product. */
void orc_crt_gemm(const double *A, long lda, int tA, const double *B, long ldb, int tB, int m,
                  int n, int k, int P, double *C)
{
    long long *ai = (long long *) malloc(sizeof(long long) * (size_t) m * (k > 0 ? k : 1));
    long long *bj = (long long *) malloc(sizeof(long long) * (size_t) n * (k > 0 ? k : 1));
    int *ea = (int *) malloc(sizeof(int) * (size_t) (m > 0 ? m : 1));
    int *fb = (int *) malloc(sizeof(int) * (size_t) (n > 0 ? n : 1));
    for (long i = 0; i < m; i++)
        ea[i] = crt_row_ints(tA ? A + i * lda : A + i, k, tA ? 1 : lda, P, ai + i * k);
    for (long j = 0; j < n; j++)
        fb[j] = crt_row_ints(tB ? B + j : B + j * ldb, k, tB ? ldb : 1, P, bj + j * k);
    #pragma omp parallel for collapse(2) schedule(static)
    for (long j = 0; j < n; j++)
        for (long i = 0; i < m; i++) {
            __int128 s = 0;
            const long long *a = ai + i * k, *b = bj + j * k;
            for (long l = 0; l < k; l++) s += (__int128) a[l] * b[l];
            C[i + j * m] = crt_to_double(s, ea[i] + fb[j] - 2 * P);
        }
    free(ai); free(bj); free(ea); free(fb);
}

/* The modular route for the same integers, for small sizes: residues of a'
 * and b' modulo each p_t in [-128, 127] (r = a' mod p in [0, p), minus p when
 * r >= 128), the INT32 dot products of the residues reduced mod p_t, and a
 * Garner (mixed radix) reconstruction in 128-bit integers, symmetric around
 * 0.  Writes C'_ij (as two 64-bit halves, low first) so that a test can
 * compare it with the direct integer product.  Returns 0, or 1 when the
 * bound k 2^(2P+1) < M is not met. */
static int crt_inv_mod(int a, int p)
{
    a %= p;
    if (a < 0) a += p;
    for (int x = 1; x < p; x++) if ((a * x) % p == 1) return x;
    return 0;
}

int orc_crt_modular(const double *A, long lda, int tA, const double *B, long ldb, int tB, int m,
                    int n, int k, int P, int nmod, long long *out_lo_hi)
{
    if (nmod < 2 || nmod > 18 || orc_crt_bits(nmod, k) < P) return 1;
    long long *ai = (long long *) malloc(sizeof(long long) * (size_t) m * (k > 0 ? k : 1));
    long long *bj = (long long *) malloc(sizeof(long long) * (size_t) n * (k > 0 ? k : 1));
    for (long i = 0; i < m; i++)
        crt_row_ints(tA ? A + i * lda : A + i, k, tA ? 1 : lda, P, ai + i * k);
    for (long j = 0; j < n; j++)
        crt_row_ints(tB ? B + j : B + j * ldb, k, tB ? ldb : 1, P, bj + j * k);
    int u[18];
    for (long j = 0; j < n; j++)
        for (long i = 0; i < m; i++) {
            for (int t = 0; t < nmod; t++) {
                const long long p = crt_mod_list[t];
                long long acc = 0;
                for (long l = 0; l < k; l++) {
                    long long ra = ((ai[i * k + l] % p) + p) % p, rb = ((bj[j * k + l] % p) + p) % p;
                    if (ra >= 128) ra -= p;
                    if (rb >= 128) rb -= p;
                    acc += ra * rb;
                }
                u[t] = (int) (((acc % p) + p) % p);
            }
            /* Garner: x = v_0 + p_0 (v_1 + p_1 (v_2 + ...)) */
            long long v[18];
            for (int t = 0; t < nmod; t++) {
                const int p = crt_mod_list[t];
                long long x = 0, w = 1;
                for (int s2 = 0; s2 < t; s2++) {
                    x = (x + v[s2] % p * w) % p;
                    w = w * crt_mod_list[s2] % p;
                }
                long long d = ((u[t] - x) % p + p) % p;
                v[t] = d * crt_inv_mod((int) w, p) % p;
            }
            unsigned __int128 x = 0, w = 1, M = 1;
            for (int t = 0; t < nmod; t++) { x += (unsigned __int128) v[t] * w; w *= crt_mod_list[t]; }
            M = w;
            __int128 c = x >= M / 2 ? (__int128) x - (__int128) M : (__int128) x;
            out_lo_hi[2 * (i + j * m)] = (long long) (uint64_t) c;
            out_lo_hi[2 * (i + j * m) + 1] = (long long) (c >> 64);
        }
    free(ai); free(bj);
    return 0;
}

/* The exact integer product C'_ij (two 64-bit halves, low first). */
void orc_crt_exact(const double *A, long lda, int tA, const double *B, long ldb, int tB, int m,
                   int n, int k, int P, long long *out_lo_hi)
{
    long long *ai = (long long *) malloc(sizeof(long long) * (size_t) m * (k > 0 ? k : 1));
    long long *bj = (long long *) malloc(sizeof(long long) * (size_t) n * (k > 0 ? k : 1));
    for (long i = 0; i < m; i++)
        crt_row_ints(tA ? A + i * lda : A + i, k, tA ? 1 : lda, P, ai + i * k);
    for (long j = 0; j < n; j++)
        crt_row_ints(tB ? B + j : B + j * ldb, k, tB ? ldb : 1, P, bj + j * k);
    for (long j = 0; j < n; j++)
        for (long i = 0; i < m; i++) {
            __int128 s = 0;
            for (long l = 0; l < k; l++) s += (__int128) ai[i * k + l] * bj[j * k + l];
            out_lo_hi[2 * (i + j * m)] = (long long) (uint64_t) s;
            out_lo_hi[2 * (i + j * m) + 1] = (long long) (s >> 64);
        }
    free(ai); free(bj);
}
