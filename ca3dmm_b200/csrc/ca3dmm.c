/* CA3DMM engine on one B200: the reference's mp x np x kp virtual process
 * grid folded into one host call (src/ca3dmm.c:23-1410).
 *
 * Init reproduces the reference's grid choice and per-rank block arithmetic
 * (src/ca3dmm.c:47-356 general, :468-642 B^T*B) and turns the active grid
 * into work groups: one group per (task_k, task_m, task_n) Cannon task, whose
 * np_dim^2 ranks' cuboid GEMMs tile one group GEMM
 *     C_g = op(A)[task m rows, slab k] * op(B)[slab k, task n cols].
 * Exec runs, on one stream:
 *   1. pack op(A) blocks (task_m x task_k) and op(B) blocks (task_k x task_n)
 *      into the work buffer, transposing on the way when trans_A / trans_B
 *      (src/ca3dmm.c:970-1060: redistribution + cublasDgeam; replication by
 *      allgather, :1062-1167, becomes groups reading the same packed block);
 *   2. one grouped GEMM launch over all groups (src/cannon.c:319-684), plain
 *      FP64 DMMA or split precision;
 *   3. the kp-slab FP64 reduction in slab order (src/ca3dmm.c:1287-1343), or a
 *      direct write when kp == 1;
 *   4. a block copy into dst_C when a dst_C block other than the whole C was
 *      requested (src/ca3dmm.c:1348-1364).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <strings.h>
#include <cuda_runtime_api.h>
#include <nvtx3/nvToolsExt.h>
#include "ca3dmm_util.h"
#include "ca3dmm_kernels.h"
#include "ca3dmm_ozaki.h"
#include "ca3dmm_crt.h"
#include "ca3dmm.h"
#include "ca3dmm_tune_internal.h"

#define ALIGN_BYTES 256
#define CANARY_BYTES 256
#define CANARY_BYTE 0xA5

typedef struct {
    int tk, tm, tn;        /* task ids */
    int m0, n0, k0;        /* first row of op(A) / column of op(B) / k index */
    int mz, nz, kz;        /* group GEMM size */
    int a_blk, b_blk;      /* packed block indices */
} group_t;

typedef struct {
    int rows, cols, r0, c0;   /* block of op(X): rows x cols starting at (r0, c0) */
    long long ld;             /* leading dimension of the packed copy (M-major op(A), K-major op(B)) */
    long long kld;            /* op(A) blocks: leading dimension of a K-major packed copy */
    size_t off;               /* byte offset of the packed copy in the work buffer */
    const double *direct;     /* plain mode: the caller's block used in place (NULL: packed) */
    long long direct_ld;
} blk_t;

#define CRT_MAX_BANDS 16

typedef struct {
    int ngroup, nA, nB;
    int tmn, tnn;             /* row / column blocks of the internal grouping (1: merged) */
    int ksplit;               /* plain mode: each slab's k range runs as ksplit sub-slabs */
    int sym;                  /* B^T B upper block triangle only: one group per 128-row block
                                 row and slab, the lower triangle mirrored after the sum */
    group_t *groups;
    blk_t *A, *B;
    /* work buffer layout (byte offsets) */
    size_t off_status, off_packA, off_packB, off_copy, off_tmapA, off_tmapB, off_gemm, off_ozplan;
    size_t off_A, off_B, off_slab, off_cout, off_oz, total;
    size_t gemm_plan_bytes, oz_plan_bytes, oz_bytes;
    long long slab_ld;        /* leading dimension of each C slab */
    size_t slab_stride;       /* elements between slabs */
    /* pinned host staging for plan uploads */
    void *stage;
    size_t stage_bytes;
    int *status_h;
    /* cached exec arguments the device plan was built for */
    int plan_valid, c_ldA, c_ldB, c_ldC;
    const void *c_A, *c_B;
    void *c_dst;
    int gemm_tiles;
    int pack_tiles_A, pack_tiles_B, pack_tiles_C;
    int packA_tma, packB_tma;     /* transposing packs staged by TMA (tensor maps in the plan) */
    int a_kmajor;                 /* plain mode: transposed A blocks read in place, K-major */
    int plain_merged;             /* plain mode: the kp slabs run as one GEMM over all of k */
    int merge_allowed;            /* CA3DMM_PLAIN_MERGE_SLABS (default 1) */
    /* dst_C block */
    int has_dst, dst_srow, dst_nrow, dst_scol, dst_ncol;
    cudaEvent_t ev[5];
    int events_ok;
    ca3dmm_oz_plan_t oz;
    ca3dmm_dgemm_desc_t *gd;      /* per-group GEMM descriptors (plan build scratch) */
    ca3dmm_oz_blk_t *ob;
    ca3dmm_oz_src_t *os;
    ca3dmm_oz_group_t *og;
    ca3dmm_oz_unit_t *ou;
    int oz_fused;                 /* split mode adds its kp slabs into C itself */
    /* modular split precision (CA3DMM_GEMM_CRT): crt_nsl k slabs of at most
     * CA3DMM_CRT_MAX_K (B^T B: the kp slabs), each one group over all of C,
     * summed by the slab reduction when there are several */
    int crt_nsl;
    ca3dmm_crt_plan_t crt;
    ca3dmm_oz_blk_t *cb;          /* crt_nsl op(A) blocks, then crt_nsl op(B) blocks */
    ca3dmm_oz_src_t *cs;
    ca3dmm_crt_group_t *cg;
    size_t off_crtplan, crt_plan_bytes, off_crt, crt_bytes;
    int crt_band;                 /* tile rows per band of the device exec's CRT work list
                                     (env CA3DMM_CRT_BAND, default 32 -- measured best at
                                     8000^3; 0: all tile rows in one band) */
    int crt_band_env;             /* crt_band as the environment set it */
    int crt_overlap;              /* device exec: reconstruct band b beside the GEMM of band b + 1
                                     (env CA3DMM_CRT_OVERLAP, default 1) */
    int crt_overlap_blocks;       /* reconstruction blocks per SM beside the GEMM (1 or 2) */
    cudaStream_t st_aux;          /* the reconstruction stream of the overlapped exec */
    cudaEvent_t ev_band[CRT_MAX_BANDS], ev_join;
    int aux_ok;
    int crt_tile_n;               /* CRT GEMM tile columns, 128 or 256 (env CA3DMM_CRT_TILE_N) */
    int plain_tile_n;             /* plain DMMA GEMM tile columns, 128 or 64 (env
                                     CA3DMM_PLAIN_TILE_N; 128 for the symmetric B^T B plan,
                                     whose tiles follow 128-row block rows) */
    int plain_tile_n_env;
    int upload_for_host;          /* the plan being uploaded serves exec_host's row bands */
    /* guard bands: 256-byte canaries between the work buffer's regions, filled
     * with CANARY_BYTE at each plan upload and, with CA3DMM_CANARY=1, checked
     * on the device after every exec */
    int ncanary, check_canary;
    long long canary[CA3DMM_MAX_CANARIES];
    struct host_exec *hx;         /* state of ca3dmm_engine_exec_host (lazily created) */
    ca3dmm_tune_report_t report;  /* the candidates of the last tuning */
} plan_t;

/* ca3dmm_engine_exec_host: device staging of A, B and C and the row-band
 * pipeline.  Band c covers output rows [r0, r1) inside one task_m block; its
 * op(A) rows are copied in, packed or sliced, multiplied (one tile range per
 * (slab, task_n) group: the GEMM kernels number tiles in raster bands of
 * `raster` 128-row tile rows, so a band of raster * 128 rows is contiguous),
 * reduced over the slabs and copied out while the next band's rows arrive. */
#define HX_MAX_BANDS 64
struct host_exec {
    double *dA, *dB, *dC;
    long long lda, ldb, ldc;
    cudaStream_t s_in, s_out;
    cudaEvent_t ev_b, ev_a[HX_MAX_BANDS], ev_c[HX_MAX_BANDS];
    int nband, r0[HX_MAX_BANDS], r1[HX_MAX_BANDS];
    ca3dmm_tile_ranges_t rng[HX_MAX_BANDS];
    void *desc_h, *desc_d;        /* per-band A descriptors (pack or slicing) */
    size_t desc_stride;
    int ndesc, ntile[HX_MAX_BANDS][3];  /* per band: Ozaki exponent items + KC + RC slicing tiles, or pack tiles */
    int built_mode, built_slices, built_raster;
    int slab_built;               /* B^T B: per-slab slicing descriptors uploaded (split mode) */
    int ok;                       /* streams and events created */
};


/* Geometry of one virtual rank (same 34-int layout as the oracle):
 * src/ca3dmm.c:146-185 (task ids), :212-261 (block ranges, C_out),
 * :298-346 (replication split of the redistribution request),
 * src/cannon.c:68-77 (Cannon block of the rank's in-group coordinates). */
static void vrank_geometry(int m, int n, int k, int mp, int np, int kp, int rank, int is_btb,
                           int *out)
{
    memset(out, 0, sizeof(int) * 34);
    if (rank >= mp * np * kp) return;
    out[0] = 1;
    const int plane = mp * np;
    const int rank_k = rank / plane, rank_mn = rank % plane;
    int tmn = 1, tmi = 0, tnn = 1, tni = 0, group = plane;
    if (!is_btb && mp > np) { tmn = mp / np; tmi = rank_mn / (np * np); group = np * np; }
    if (!is_btb && np > mp) { tnn = np / mp; tni = rank_mn / (mp * mp); group = mp * mp; }
    out[1] = rank_mn % mp; out[2] = rank_mn / mp; out[3] = rank_k;
    out[4] = tmn; out[5] = tmi; out[6] = tnn; out[7] = tni; out[8] = kp; out[9] = rank_k;
    int ms, mz, ns, nz, ks, kz;
    calc_block_spos_size(m, tmn, tmi, &ms, &mz);
    calc_block_spos_size(n, tnn, tni, &ns, &nz);
    calc_block_spos_size(k, kp, rank_k, &ks, &kz);
    const int side = (int) sqrt((double) group);
    const int in_group = rank_mn % group, row = in_group / side, col = in_group % side;
    int a_r, a_rz, a_c, a_cz, b_r, b_rz, b_c, b_cz, c_r, c_rz, c_c, c_cz;
    calc_block_spos_size(mz, side, row, &a_r, &a_rz);
    calc_block_spos_size(kz, side, col, &a_c, &a_cz);
    calc_block_spos_size(kz, side, row, &b_r, &b_rz);
    calc_block_spos_size(nz, side, col, &b_c, &b_cz);
    calc_block_spos_size(mz, side, row, &c_r, &c_rz);
    calc_block_spos_size(nz, side, col, &c_c, &c_cz);
    out[10] = ms + a_r; out[11] = ks + a_c; out[12] = a_rz; out[13] = a_cz;
    out[14] = ks + b_r; out[15] = ns + b_c; out[16] = b_rz; out[17] = b_cz;
    out[18] = ms + c_r; out[19] = ns + c_c; out[20] = c_rz; out[21] = c_cz;
    int o_c, o_cz;
    calc_block_spos_size(c_cz, kp, rank_k, &o_c, &o_cz);
    out[22] = out[18]; out[23] = out[19] + o_c; out[24] = c_rz; out[25] = o_cz;
    memcpy(out + 26, out + 10, 4 * sizeof(int));
    memcpy(out + 30, out + 14, 4 * sizeof(int));
    if (!is_btb && tnn > 1) {
        int s, z;
        calc_block_spos_size(out[13], tnn, tni, &s, &z);
        out[27] = out[11] + s; out[29] = z;
    }
    if (!is_btb && tmn > 1) {
        int s, z;
        calc_block_spos_size(out[17], tmn, tmi, &s, &z);
        out[31] = out[15] + s; out[33] = z;
    }
}

static size_t align_up(size_t x) { return (x + ALIGN_BYTES - 1) / ALIGN_BYTES * ALIGN_BYTES; }

/* Byte layout of the device work buffer for the current gemm mode. */
#define GUARD_BAND(off)                                                                      \
    do {                                                                                     \
        if (pl->ncanary < CA3DMM_MAX_CANARIES) pl->canary[pl->ncanary++] = (long long) (off); \
        (off) += CANARY_BYTES;                                                               \
    } while (0)

static void plan_layout(ca3dmm_engine_p e, plan_t *pl)
{
    size_t off = 0;
    pl->ncanary = 0;
    pl->off_status = off; off = align_up(off + 64);
    pl->off_packA = off; off = align_up(off + sizeof(ca3dmm_pack_desc_t) * pl->nA);
    pl->off_packB = off; off = align_up(off + sizeof(ca3dmm_pack_desc_t) * pl->nB);
    pl->off_copy = off; off = align_up(off + sizeof(ca3dmm_pack_desc_t));
    pl->off_tmapA = off; off = align_up(off + 128 * (size_t) pl->nA);
    pl->off_tmapB = off; off = align_up(off + 128 * (size_t) pl->nB);
    pl->gemm_plan_bytes = ca3dmm_dgemm_plan_bytes(pl->ngroup * pl->ksplit);
    pl->off_gemm = off; off = align_up(off + pl->gemm_plan_bytes);
    pl->oz_plan_bytes = ca3dmm_oz_plan_bytes(pl->ngroup);
    pl->off_ozplan = off; off = align_up(off + pl->oz_plan_bytes);
    pl->crt_plan_bytes = ca3dmm_crt_plan_bytes(2 * pl->crt_nsl, pl->crt_nsl);
    pl->off_crtplan = off; off = align_up(off + pl->crt_plan_bytes);
    GUARD_BAND(off);
    size_t packs = 0;
    pl->off_A = off;
    for (int i = 0; i < pl->nA; i++) {
        pl->A[i].off = off + packs;
        /* room for either packed layout: M-major (ld x cols) or K-major (kld x rows) */
        const size_t mm = (size_t) pl->A[i].ld * (size_t) pl->A[i].cols;
        const size_t km = (size_t) pl->A[i].kld * (size_t) pl->A[i].rows;
        packs += align_up(sizeof(double) * (mm > km ? mm : km));
    }
    off += packs;
    GUARD_BAND(off);
    packs = 0;
    pl->off_B = off;
    for (int i = 0; i < pl->nB; i++) {
        pl->B[i].off = off + packs;
        packs += align_up(sizeof(double) * (size_t) pl->B[i].ld * (size_t) pl->B[i].cols);
    }
    off += packs;
    GUARD_BAND(off);
    pl->slab_ld = ca3dmm_round_up(e->m, 2);
    pl->slab_stride = (size_t) pl->slab_ld * (size_t) e->n;
    pl->off_slab = off;
    int nslab = e->kp * pl->ksplit;          /* plain mode's sub-slabs; split mode uses kp of them */
    if (pl->crt_nsl > nslab) nslab = pl->crt_nsl;
    if (nslab > 1) off = align_up(off + sizeof(double) * pl->slab_stride * (size_t) nslab);
    GUARD_BAND(off);
    pl->off_cout = off;
    off = align_up(off + sizeof(double) * (size_t) e->m * (size_t) e->n);
    GUARD_BAND(off);
    pl->off_oz = off;
    pl->oz_bytes = 0;
    if (e->gemm_mode == CA3DMM_GEMM_OZAKI) {
        int *dims = (int *) malloc(sizeof(int) * 2 * (size_t) (pl->nA + pl->nB));
        if (dims) {
            int *am = dims, *ak = dims + pl->nA, *bk = dims + 2 * pl->nA, *bn = bk + pl->nB;
            for (int i = 0; i < pl->nA; i++) { am[i] = pl->A[i].rows; ak[i] = pl->A[i].cols; }
            for (int i = 0; i < pl->nB; i++) { bk[i] = pl->B[i].rows; bn[i] = pl->B[i].cols; }
            pl->oz_bytes = ca3dmm_oz_work_bytes(pl->nA, am, ak, pl->nB, bk, bn, e->ozaki_slices);
            free(dims);
        }
        off = align_up(off + pl->oz_bytes);
    }
    GUARD_BAND(off);
    pl->off_crt = off;
    pl->crt_bytes = 0;
    if (e->gemm_mode == CA3DMM_GEMM_CRT) {
        const int ns = pl->crt_nsl;
        int *d = (int *) malloc(sizeof(int) * 6 * (size_t) ns);
        if (d) {
            int *am = d, *ak = d + ns, *bk = d + 2 * ns, *bn = d + 3 * ns, *gm = d + 4 * ns,
                *gn = d + 5 * ns;
            for (int i = 0; i < ns; i++) {
                /* an aliased op(A) block (B^T B) has no residues of its own */
                am[i] = pl->cb[i].alias >= 0 ? 0 : pl->cb[i].rows;
                ak[i] = pl->cb[i].cols;
                bk[i] = pl->cb[ns + i].rows; bn[i] = pl->cb[ns + i].cols;
                gm[i] = pl->cg[i].m; gn[i] = pl->cg[i].n;
            }
            pl->crt_bytes = ca3dmm_crt_work_bytes(ns, am, ak, ns, bk, bn, ns, gm, gn,
                                                  e->crt_moduli > 0 ? e->crt_moduli : 1);
            free(d);
        }
        off = align_up(off + pl->crt_bytes);
    }
    GUARD_BAND(off);
    pl->total = off;
}

/* Plain-mode k split of every slab against the tail wave: the DMMA launch
 * runs one 128 x 128 tile per SM at a time, so T tiles take ceil(T / SMs)
 * rounds; with each slab's k range cut into s sub-slabs (their own C slab
 * buffers, summed in order by the slab reduction) the rounds are s times
 * shorter and ceil(s T / SMs) / s can come closer to T / SMs.  Only for few
 * rounds, sub-slabs of at least 512 k, and slab buffers of at most 1 GiB.
 * (The reference runs one DGEMM per Cannon step, src/cannon.c:410-418.) */
#define CA3DMM_KSPLIT_MAX 8
#define CA3DMM_SMS_B200 148
static int choose_ksplit(const ca3dmm_engine_p e, int sym)
{
    const long long tb = (e->m + 127) / 128;
    const long long tiles = (sym ? tb * (tb + 1) / 2 : tb * ((e->n + 127) / 128)) * e->kp;
    const int kz = e->k / e->kp;
    const double slab_bytes = 8.0 * (double) ca3dmm_round_up(e->m, 2) * (double) e->n;
    if (tiles <= 0 || tiles >= 4LL * CA3DMM_SMS_B200) return 1;
    int best = 1;
    double best_cost = (double) ((tiles + CA3DMM_SMS_B200 - 1) / CA3DMM_SMS_B200);
    for (int s = 2; s <= CA3DMM_KSPLIT_MAX; s++) {
        if (kz / s < 512 || slab_bytes * e->kp * s > 1073741824.0) break;
        const double cost =
            (double) ((tiles * s + CA3DMM_SMS_B200 - 1) / CA3DMM_SMS_B200) / (double) s;
        if (cost < 0.99 * best_cost) { best = s; best_cost = cost; }
    }
    return best;
}

/* Modular split precision: k slabs of at most CA3DMM_CRT_MAX_K (the exact
 * INT32 range of the residue products); B^T B keeps the reference's kp slabs. */
static int crt_slabs(const ca3dmm_engine_p e)
{
    if (e->is_BTB) return e->kp > 0 ? e->kp : 1;
    const int ns = (e->k + CA3DMM_CRT_MAX_K - 1) / CA3DMM_CRT_MAX_K;
    return ns > 0 ? ns : 1;
}

/* Moduli for the modular mode: `want` (8..18), or 0 for the fewest whose
 * product admits 51-bit operand integers for the deepest slab.  Returns 0 when
 * no count works (a slab deeper than CA3DMM_CRT_MAX_K). */
static int crt_resolve(const ca3dmm_engine_p e, int want)
{
    const int ns = crt_slabs(e);
    const int kmax = (e->k + ns - 1) / ns;
    if (kmax > CA3DMM_CRT_MAX_K) return 0;
    if (want != 0) {
        if (want < 8 || want > CA3DMM_CRT_MAX_MODULI) return 0;
        return ca3dmm_crt_bits(want, kmax) >= 2 ? want : 0;
    }
    for (int nm = 8; nm <= CA3DMM_CRT_MAX_MODULI; nm++)
        if (ca3dmm_crt_bits(nm, kmax) >= 51) return nm;
    return CA3DMM_CRT_MAX_MODULI;
}

static int plan_build(ca3dmm_engine_p e)
{
    plan_t *pl = (plan_t *) calloc(1, sizeof(plan_t));
    if (!pl) return CA3DMM_ENOMEM;
    e->impl = pl;
    /* One GEMM per k-slab over the whole C: the reference's task_m / task_n
     * replication groups (src/ca3dmm.c:155-169) compute disjoint blocks of the
     * same slab product, and every C entry is the same k-ordered dot product
     * whichever block holds it, so on one GPU the blocks merge; fewer, larger
     * GEMMs leave fewer partial edge tiles. */
    const int tmn = 1, tnn = 1;
    pl->tmn = tmn;
    pl->tnn = tnn;
    const int kp = e->kp;
    /* symmetric B^T B: per slab one group for each 128-row block row bi, over
     * rows [128 bi, 128 bi + 128) and columns [128 bi, n) -- the upper block
     * triangle (C = B^T B is symmetric; the reference computes all of it) */
    pl->sym = e->is_BTB && e->btb_symmetric;
    const int nbr = pl->sym ? (e->m + 127) / 128 : 1;
    pl->nA = tmn * kp;
    pl->nB = tnn * kp;
    pl->ngroup = kp * (pl->sym ? nbr : tmn * tnn);
    pl->groups = (group_t *) calloc((size_t) pl->ngroup, sizeof(group_t));
    pl->A = (blk_t *) calloc((size_t) pl->nA, sizeof(blk_t));
    pl->B = (blk_t *) calloc((size_t) pl->nB, sizeof(blk_t));
    pl->ksplit = choose_ksplit(e, pl->sym);
    int merge;
    GET_ENV_INT_VAR(merge, "CA3DMM_PLAIN_MERGE_SLABS", "plain_merge_slabs", 1, 0, 1);
    pl->merge_allowed = merge;
    GET_ENV_INT_VAR(pl->crt_band, "CA3DMM_CRT_BAND", "crt_band", 32, 0, 1 << 20);
    pl->crt_band_env = pl->crt_band;
    GET_ENV_INT_VAR(pl->crt_tile_n, "CA3DMM_CRT_TILE_N", "crt_tile_n", 256, 128, 256);
    GET_ENV_INT_VAR(pl->plain_tile_n, "CA3DMM_PLAIN_TILE_N", "plain_tile_n", 128, 64, 128);
    if (pl->plain_tile_n != 64 || pl->sym) pl->plain_tile_n = 128;
    pl->plain_tile_n_env = pl->plain_tile_n;
    GET_ENV_INT_VAR(pl->crt_overlap, "CA3DMM_CRT_OVERLAP", "crt_overlap", 1, 0, 1);
    GET_ENV_INT_VAR(pl->crt_overlap_blocks, "CA3DMM_CRT_OVERLAP_BLOCKS", "crt_overlap_blocks", 2, 1, 2);
    if (pl->crt_tile_n != 128) pl->crt_tile_n = 256;
    GET_ENV_INT_VAR(pl->check_canary, "CA3DMM_CANARY", "check_canary", 0, 0, 1);
    pl->gd = (ca3dmm_dgemm_desc_t *) calloc((size_t) pl->ngroup * (size_t) pl->ksplit,
                                            sizeof(ca3dmm_dgemm_desc_t));
    pl->ob = (ca3dmm_oz_blk_t *) calloc((size_t) (pl->nA + pl->nB), sizeof(ca3dmm_oz_blk_t));
    pl->os = (ca3dmm_oz_src_t *) calloc((size_t) (pl->nA + pl->nB), sizeof(ca3dmm_oz_src_t));
    pl->og = (ca3dmm_oz_group_t *) calloc((size_t) pl->ngroup, sizeof(ca3dmm_oz_group_t));
    pl->ou = (ca3dmm_oz_unit_t *) calloc((size_t) pl->ngroup, sizeof(ca3dmm_oz_unit_t));
    if (!pl->groups || !pl->A || !pl->B || !pl->gd || !pl->ob || !pl->os || !pl->og || !pl->ou)
        return CA3DMM_ENOMEM;
    for (int tk = 0; tk < kp; tk++) {
        int ks, kz;
        calc_block_spos_size(e->k, kp, tk, &ks, &kz);
        for (int tm = 0; tm < tmn; tm++) {
            int ms, mz;
            calc_block_spos_size(e->m, tmn, tm, &ms, &mz);
            blk_t *a = &pl->A[tk * tmn + tm];
            a->rows = mz; a->cols = kz; a->r0 = ms; a->c0 = ks;
            a->ld = ca3dmm_round_up(mz > 0 ? mz : 1, 2);
            a->kld = ca3dmm_round_up(kz > 0 ? kz : 1, 2);
        }
        for (int tn = 0; tn < tnn; tn++) {
            int ns, nz;
            calc_block_spos_size(e->n, tnn, tn, &ns, &nz);
            blk_t *b = &pl->B[tk * tnn + tn];
            b->rows = kz; b->cols = nz; b->r0 = ks; b->c0 = ns;
            b->ld = ca3dmm_round_up(kz > 0 ? kz : 1, 2);
        }
        for (int bi = 0; pl->sym && bi < nbr; bi++) {
            group_t *g = &pl->groups[tk * nbr + bi];
            g->tk = tk; g->tm = 0; g->tn = 0;
            g->a_blk = tk; g->b_blk = tk;
            g->m0 = 128 * bi; g->mz = e->m - g->m0 < 128 ? e->m - g->m0 : 128;
            g->n0 = 128 * bi; g->nz = e->n - g->n0;
            g->k0 = ks; g->kz = kz;
        }
        for (int tm = 0; !pl->sym && tm < tmn; tm++)
            for (int tn = 0; tn < tnn; tn++) {
                group_t *g = &pl->groups[(tk * tmn + tm) * tnn + tn];
                g->tk = tk; g->tm = tm; g->tn = tn;
                g->a_blk = tk * tmn + tm;
                g->b_blk = tk * tnn + tn;
                g->m0 = pl->A[g->a_blk].r0; g->mz = pl->A[g->a_blk].rows;
                g->n0 = pl->B[g->b_blk].c0; g->nz = pl->B[g->b_blk].cols;
                g->k0 = ks; g->kz = kz;
            }
    }
    /* modular split precision: one group over all of C per k slab */
    const int ns = crt_slabs(e);
    pl->crt_nsl = ns;
    pl->cb = (ca3dmm_oz_blk_t *) calloc(2 * (size_t) ns, sizeof(ca3dmm_oz_blk_t));
    pl->cs = (ca3dmm_oz_src_t *) calloc(2 * (size_t) ns, sizeof(ca3dmm_oz_src_t));
    pl->cg = (ca3dmm_crt_group_t *) calloc((size_t) ns, sizeof(ca3dmm_crt_group_t));
    if (!pl->cb || !pl->cs || !pl->cg) return CA3DMM_ENOMEM;
    for (int s2 = 0; s2 < ns; s2++) {
        int ks, kz;
        calc_block_spos_size(e->k, ns, s2, &ks, &kz);
        ca3dmm_oz_blk_t *a = &pl->cb[s2], *b = &pl->cb[ns + s2];
        a->r0 = 0; a->c0 = ks; a->rows = e->m; a->cols = kz;
        a->alias = e->is_BTB ? s2 : -1;      /* op(A) = B^T: the B block's residues */
        b->r0 = ks; b->c0 = 0; b->rows = kz; b->cols = e->n; b->alias = -1;
        ca3dmm_crt_group_t *g = &pl->cg[s2];
        g->a_blk = s2; g->b_blk = s2;
        g->m = e->m; g->n = e->n; g->k = kz;
    }
    plan_layout(e, pl);
    pl->stage_bytes = pl->off_crtplan + pl->crt_plan_bytes;
    return CA3DMM_OK;
}

/* CUDA-side resources of the plan, created when a work buffer is attached so
 * that init itself makes no CUDA call (it only sizes the work buffer). */
static int plan_cuda_init(plan_t *pl)
{
    if (pl->stage) return CA3DMM_OK;
    if (cudaMallocHost(&pl->stage, pl->stage_bytes) != cudaSuccess) {
        pl->stage = NULL;
        return CA3DMM_ECUDA;
    }
    if (cudaMallocHost((void **) &pl->status_h, 64) != cudaSuccess) {
        pl->status_h = NULL;
        return CA3DMM_ECUDA;
    }
    memset(pl->status_h, 0, 64);
    pl->events_ok = 1;
    for (int i = 0; i < 5; i++)
        if (cudaEventCreate(&pl->ev[i]) != cudaSuccess) pl->events_ok = 0;
    return CA3DMM_OK;
}

static void plan_free(plan_t *pl)
{
    if (!pl) return;
    free(pl->groups);
    free(pl->A);
    free(pl->B);
    free(pl->gd);
    free(pl->ob);
    free(pl->os);
    free(pl->og);
    free(pl->ou);
    free(pl->cb);
    free(pl->cs);
    free(pl->cg);
    if (pl->hx) {
        struct host_exec *x = pl->hx;
        cudaFree(x->dA);
        cudaFree(x->dB);
        cudaFree(x->dC);
        cudaFree(x->desc_d);
        if (x->desc_h) cudaFreeHost(x->desc_h);
        if (x->ok) {
            cudaStreamDestroy(x->s_in);
            cudaStreamDestroy(x->s_out);
            cudaEventDestroy(x->ev_b);
            for (int i = 0; i < HX_MAX_BANDS; i++) {
                cudaEventDestroy(x->ev_a[i]);
                cudaEventDestroy(x->ev_c[i]);
            }
        }
        free(x);
    }
    if (pl->stage) cudaFreeHost(pl->stage);
    if (pl->status_h) cudaFreeHost(pl->status_h);
    if (pl->events_ok)
        for (int i = 0; i < 5; i++) cudaEventDestroy(pl->ev[i]);
    if (pl->aux_ok) {
        cudaStreamDestroy(pl->st_aux);
        for (int i = 0; i < CRT_MAX_BANDS; i++) cudaEventDestroy(pl->ev_band[i]);
        cudaEventDestroy(pl->ev_join);
    }
    free(pl);
}

/* Reference-style grid selection for the general engine (src/ca3dmm.c:47-136). */
static int choose_grid(int p, int m, int n, int k, const int *proc_grid, int *mp, int *np, int *kp,
                       int *rp)
{
    int gen = 1;
    if (proc_grid != NULL) {
        *mp = proc_grid[0]; *np = proc_grid[1]; *kp = proc_grid[2];
        *rp = p - (*mp) * (*np) * (*kp);
        int hi = *mp > *np ? *mp : *np, lo = *mp < *np ? *mp : *np;
        if (lo < 1 || (hi % lo) || (*rp < 0))
            WARNING_PRINTF("Invalid process grid specified: mp, np, kp = %d, %d, %d\n", *mp, *np,
                           *kp);
        else
            gen = 0;
    }
    if (gen) {
        calc_3d_decomposition_cannon(p, m, n, k, mp, np, kp, rp);
        int reduce_kp;
        GET_ENV_INT_VAR(reduce_kp, "CA3DMM_REDUCE_KP", "reduce_kp", 0, 0, 1);
        if (reduce_kp) {
            /* fold a factor 3 (else 2) of kp into the smaller of mp / np when
             * the divisibility rule still holds (src/ca3dmm.c:75-124) */
            int f = (*kp >= 3 && *kp % 3 == 0) ? 3 : ((*kp >= 2 && *kp % 2 == 0) ? 2 : 0);
            if (f) {
                int *grow = (*mp <= *np) ? mp : np, *other = (*mp <= *np) ? np : mp;
                int g = *grow * f;
                int hi = g > *other ? g : *other, lo = g < *other ? g : *other;
                if (hi % lo == 0) {
                    *kp /= f;
                    *grow = g;
                }
            }
        }
    }
    if (*mp < 1 || *np < 1 || *kp < 1 || (*mp) * (*np) * (*kp) > p) {
        ERROR_PRINTF("Invalid process grid generated: p = %d, mp, np, kp = %d, %d, %d\n", p, *mp,
                     *np, *kp);
        return CA3DMM_EINVAL;
    }
    return CA3DMM_OK;
}

static void fill_rank0_fields(ca3dmm_engine_p e)
{
    int g[34];
    vrank_geometry(e->m, e->n, e->k, e->mp, e->np, e->kp, 0, e->is_BTB, g);
    e->is_active = g[0];
    e->rank_m = g[1]; e->rank_n = g[2]; e->rank_k = g[3];
    e->task_m_num = g[4]; e->task_m_id = g[5];
    e->task_n_num = g[6]; e->task_n_id = g[7];
    e->task_k_num = g[8]; e->task_k_id = g[9];
    e->A_2dmm_srow = g[10]; e->A_2dmm_scol = g[11]; e->A_2dmm_nrow = g[12]; e->A_2dmm_ncol = g[13];
    e->B_2dmm_srow = g[14]; e->B_2dmm_scol = g[15]; e->B_2dmm_nrow = g[16]; e->B_2dmm_ncol = g[17];
    e->C_2dmm_srow = g[18]; e->C_2dmm_scol = g[19]; e->C_2dmm_nrow = g[20]; e->C_2dmm_ncol = g[21];
    e->A_rd_srow = g[26]; e->A_rd_scol = g[27]; e->A_rd_nrow = g[28]; e->A_rd_ncol = g[29];
    e->B_rd_srow = g[30]; e->B_rd_scol = g[31]; e->B_rd_nrow = g[32]; e->B_rd_ncol = g[33];
    /* rank 0's reduce-scatter and allgather count arrays (src/ca3dmm.c:246-261, :298-336) */
    int tk = e->task_k_num > 0 ? e->task_k_num : 1;
    e->C_rs_recvcnts = (int *) calloc((size_t) tk, sizeof(int));
    int s, z, z0 = -1;
    e->use_rsb = 1;
    for (int i = 0; i < e->task_k_num; i++) {
        calc_block_spos_size(e->C_2dmm_ncol, e->task_k_num, i, &s, &z);
        if (z0 == -1) z0 = z;
        if (z != z0) e->use_rsb = 0;
        e->C_rs_recvcnts[i] = z * e->C_2dmm_nrow;
    }
    int tmn = e->task_m_num * e->task_n_num;
    if (tmn < 1) tmn = 1;
    e->AB_agv_recvcnts = (int *) calloc((size_t) tmn, sizeof(int));
    e->AB_agv_displs = (int *) calloc((size_t) tmn + 1, sizeof(int));
    if (e->task_n_num > 1 || e->task_m_num > 1) {
        int nt = e->task_n_num > 1 ? e->task_n_num : e->task_m_num;
        int ncol = e->task_n_num > 1 ? e->A_2dmm_ncol : e->B_2dmm_ncol;
        int nrow = e->task_n_num > 1 ? e->A_2dmm_nrow : e->B_2dmm_nrow;
        z0 = -1;
        e->use_ag = 1;
        for (int i = 0; i < nt; i++) {
            calc_block_spos_size(ncol, nt, i, &s, &z);
            if (z0 == -1) z0 = z;
            if (z != z0) e->use_ag = 0;
            e->AB_agv_recvcnts[i] = z * nrow;
            e->AB_agv_displs[i + 1] = e->AB_agv_displs[i] + e->AB_agv_recvcnts[i];
        }
    }
    e->C_out_srow = 0; e->C_out_scol = 0; e->C_out_nrow = e->m; e->C_out_ncol = e->n;
}

/* Shared tail of both init functions: plan, sizes, optional allocation. */
/* ---------------------------------------------------------------------------
 * Tuning support: the candidate configurations of this engine and the work
 * buffer each needs. */

int ca3dmm_engine_crt_resolve(ca3dmm_engine_p e, int want) { return crt_resolve(e, want); }

size_t ca3dmm_engine_layout_bytes(ca3dmm_engine_p e, int mode, int count)
{
    plan_t *pl = (plan_t *) e->impl;
    const int om = e->gemm_mode, os = e->ozaki_slices, oc = e->crt_moduli;
    const size_t kept = pl->total;
    e->gemm_mode = mode;
    if (mode == CA3DMM_GEMM_OZAKI) e->ozaki_slices = count;
    if (mode == CA3DMM_GEMM_CRT) e->crt_moduli = crt_resolve(e, count);
    size_t need = 0;
    if (mode != CA3DMM_GEMM_CRT || e->crt_moduli > 0) {
        plan_layout(e, pl);
        need = pl->total;
    }
    e->gemm_mode = om;
    e->ozaki_slices = os;
    e->crt_moduli = oc;
    plan_layout(e, pl);
    if (pl->total < kept) pl->total = kept;
    return need;
}

/* Plain FP64 at raster 8 and 16; 7 and 8 INT8 slices; the modular mode at the
 * fewest moduli for 51-bit integers with 256- and 128-column tiles and bands
 * of 32 and 8 tile rows, and two moduli more (for operands whose exponent
 * spread the accuracy guard rejects at the fewest).  Candidate 0 is the plain
 * GEMM, the guard's reference. */
int ca3dmm_engine_candidates(ca3dmm_engine_p e, ca3dmm_tune_cfg_t *c, int max)
{
    ca3dmm_tune_cfg_t l[CA3DMM_TUNE_MAX_CANDS];
    int n = 0;
#define CA3DMM_CAND(md, sl, r, tn)                                                           \
    do {                                                                                     \
        l[n].gemm_mode = (md); l[n].slices = (sl); l[n].kp = e->kp;                          \
        l[n].raster = (r); l[n].tile_n = (tn); n++;                                          \
    } while (0)
    const plan_t *pl = (const plan_t *) e->impl;
    CA3DMM_CAND(CA3DMM_GEMM_PLAIN, 0, 8, 0);
    CA3DMM_CAND(CA3DMM_GEMM_PLAIN, 0, 16, 0);
    if (!pl->sym) CA3DMM_CAND(CA3DMM_GEMM_PLAIN, 0, 8, 64);
    CA3DMM_CAND(CA3DMM_GEMM_OZAKI, 7, 8, 0);
    CA3DMM_CAND(CA3DMM_GEMM_OZAKI, 7, 16, 0);
    CA3DMM_CAND(CA3DMM_GEMM_OZAKI, 8, 8, 0);
    const int nm = crt_resolve(e, 0);
    if (nm > 0) {
        CA3DMM_CAND(CA3DMM_GEMM_CRT, nm, 32, 256);
        CA3DMM_CAND(CA3DMM_GEMM_CRT, nm, 8, 256);
        CA3DMM_CAND(CA3DMM_GEMM_CRT, nm, 32, 128);
        CA3DMM_CAND(CA3DMM_GEMM_CRT, nm, 8, 128);
        const int nm2 = nm + 2 <= CA3DMM_CRT_MAX_MODULI ? nm + 2 : CA3DMM_CRT_MAX_MODULI;
        if (nm2 != nm && crt_resolve(e, nm2) == nm2) CA3DMM_CAND(CA3DMM_GEMM_CRT, nm2, 32, 256);
    }
#undef CA3DMM_CAND
    for (int i = 0; i < n && i < max && c; i++) c[i] = l[i];
    return n;
}

static size_t auto_bytes(ca3dmm_engine_p e)
{
    ca3dmm_tune_cfg_t c[CA3DMM_TUNE_MAX_CANDS];
    const int n = ca3dmm_engine_candidates(e, c, CA3DMM_TUNE_MAX_CANDS);
    size_t mx = 0;
    for (int i = 0; i < n; i++) {
        const size_t b = ca3dmm_engine_layout_bytes(e, c[i].gemm_mode, c[i].slices);
        if (b > mx) mx = b;
    }
    return mx;
}

static void finish_init(ca3dmm_engine_p e, int dst_srow, int dst_nrow, int dst_scol, int dst_ncol,
                        ca3dmm_engine_p *engine_, size_t *workbuf_bytes, double t0)
{
    fill_rank0_fields(e);
    /* rank 0's Cannon geometry, for callers that read engine->cannon_engine */
    e->cannon_engine = (cannon_engine_p) calloc(1, sizeof(cannon_engine_s));
    if (e->cannon_engine) {
        cannon_engine_p ce = e->cannon_engine;
        int side = (int) sqrt((double) (e->is_BTB ? e->mp * e->np
                                                  : (e->mp > e->np ? e->np * e->np : e->mp * e->mp)));
        if (side < 1) side = 1;
        int ms, mz, ns, nz, ks, kz;
        calc_block_spos_size(e->m, e->task_m_num, 0, &ms, &mz);
        calc_block_spos_size(e->n, e->task_n_num, 0, &ns, &nz);
        calc_block_spos_size(e->k, e->kp, 0, &ks, &kz);
        ce->m = mz; ce->n = nz; ce->k = kz; ce->np_dim = side; ce->dev_type = e->dev_type;
        ce->A_srow = e->A_2dmm_srow - ms; ce->A_scol = e->A_2dmm_scol - ks;
        ce->A_nrow = e->A_2dmm_nrow; ce->A_ncol = e->A_2dmm_ncol;
        ce->B_srow = e->B_2dmm_srow - ks; ce->B_scol = e->B_2dmm_scol - ns;
        ce->B_nrow = e->B_2dmm_nrow; ce->B_ncol = e->B_2dmm_ncol;
        ce->C_srow = e->C_2dmm_srow - ms; ce->C_scol = e->C_2dmm_scol - ns;
        ce->C_nrow = e->C_2dmm_nrow; ce->C_ncol = e->C_2dmm_ncol;
        ce->max_A_blk_size = (mz / side + 1) * (kz / side + 1);
        ce->max_B_blk_size = (kz / side + 1) * (nz / side + 1);
        ce->max_C_blk_size = (mz / side + 1) * (nz / side + 1);
        ce->gemm_cycle = 1;
    }
    int gm;
    const char *gms = getenv("CA3DMM_GEMM_MODE");
    if (gms && strcasecmp(gms, "auto") == 0) {
        INFO_PRINTF("Overriding parameter gemm_mode: 0 (default) --> auto (runtime)\n");
        gm = CA3DMM_GEMM_AUTO;
    } else {
        GET_ENV_INT_VAR(gm, "CA3DMM_GEMM_MODE", "gemm_mode", 0, 0, 3);
    }
    e->gemm_auto = gm == CA3DMM_GEMM_AUTO ? 1 : 0;
    if (gm == CA3DMM_GEMM_AUTO) gm = CA3DMM_GEMM_PLAIN;   /* until the tuner chooses */
    e->gemm_mode = gm;
    int cm;
    GET_ENV_INT_VAR(cm, "CA3DMM_CRT_MODULI", "crt_moduli", 0, 0, CA3DMM_CRT_MAX_MODULI);
    e->crt_moduli = crt_resolve(e, cm);
    if (e->gemm_mode == CA3DMM_GEMM_CRT && e->crt_moduli == 0) {
        WARNING_PRINTF("CA3DMM_GEMM_MODE=2: no modulus count fits this k; using plain FP64\n");
        e->gemm_mode = CA3DMM_GEMM_PLAIN;
    }
    int sl;
    GET_ENV_INT_VAR(sl, "CA3DMM_OZAKI_SLICES", "ozaki_slices", 7, 2, 8);
    e->ozaki_slices = sl;
    e->sync_exec = 1;
    e->raster = 8;
    if (e->is_BTB) {
        int sym;
        GET_ENV_INT_VAR(sym, "CA3DMM_BTB_SYMMETRIC", "btb_symmetric", 0, 0, 1);
        e->btb_symmetric = sym;
    }
    int rc = plan_build(e);
    if (rc) {
        ERROR_PRINTF("Failed to build the device plan (error %d)\n", rc);
        ca3dmm_engine_free(&e);
        return;
    }
    plan_t *pl = (plan_t *) e->impl;
    if (!((dst_srow == -1) || (dst_nrow == -1) || (dst_scol == -1) || (dst_ncol == -1))) {
        if (dst_srow < 0 || dst_scol < 0 || dst_nrow < 0 || dst_ncol < 0 ||
            dst_srow + dst_nrow > e->m || dst_scol + dst_ncol > e->n) {
            ERROR_PRINTF("Invalid dst_C block: (%d, %d) + %d x %d for a %d x %d C\n", dst_srow,
                         dst_scol, dst_nrow, dst_ncol, e->m, e->n);
            ca3dmm_engine_free(&e);
            return;
        }
        pl->has_dst = 1;
        pl->dst_srow = dst_srow; pl->dst_nrow = dst_nrow;
        pl->dst_scol = dst_scol; pl->dst_ncol = dst_ncol;
    }
    e->n_group = pl->ngroup;
    if (e->gemm_auto) {
        /* a work buffer that holds every candidate of the tuner */
        const size_t need = auto_bytes(e);
        if (pl->total < need) pl->total = need;
    }
    e->workbuf_bytes = pl->total;
    e->self_workbuf_bytes = pl->total;
    GET_ENV_INT_VAR(e->print_timing, "CA3DMM_PRINT_TIMING", "engine->print_timing", 0, 0, 1);
    if (workbuf_bytes != NULL) {
        e->alloc_workbuf = 0;
        *workbuf_bytes = pl->total;
    } else {
        e->alloc_workbuf = 1;
        void *wh = NULL, *wd = NULL;
        MALLOC_ATTACH_WORKBUF(ca3dmm_engine_attach_workbuf, ca3dmm_engine_free, e, e->dev_type,
                              pl->total, wh, wd);
        if (e == NULL) return;
    }
    e->init_ms = 1000.0 * (ca3dmm_wtime_sec() - t0);
    *engine_ = e;
}

void ca3dmm_engine_init(const int m, const int n, const int k, const int trans_A,
                        const int trans_B, const int src_A_srow, const int src_A_nrow,
                        const int src_A_scol, const int src_A_ncol, const int src_B_srow,
                        const int src_B_nrow, const int src_B_scol, const int src_B_ncol,
                        const int dst_C_srow, const int dst_C_nrow, const int dst_C_scol,
                        const int dst_C_ncol, const int *proc_grid, MPI_Comm comm,
                        dev_type_t dev_type, ca3dmm_engine_p *engine_, size_t *workbuf_bytes)
{
    if (engine_ == NULL) return;
    *engine_ = NULL;
    if (is_dev_type_valid(dev_type) == 0) {
        ERROR_PRINTF("Invalid device type %d\n", dev_type);
        return;
    }
    int p = ca3dmm_vcomm_size(comm);
    if (p < 1) {
        ERROR_PRINTF("Invalid communicator\n");
        return;
    }
    if (m < 1 || n < 1 || k < 1) {
        ERROR_PRINTF("Invalid matrix size m, n, k = %d, %d, %d\n", m, n, k);
        return;
    }
    const int a_nrow = trans_A ? k : m, a_ncol = trans_A ? m : k;
    const int b_nrow = trans_B ? n : k, b_ncol = trans_B ? k : n;
    if (src_A_srow != 0 || src_A_scol != 0 || src_A_nrow != a_nrow || src_A_ncol != a_ncol ||
        src_B_srow != 0 || src_B_scol != 0 || src_B_nrow != b_nrow || src_B_ncol != b_ncol) {
        ERROR_PRINTF("Folded call: src_A / src_B must describe the whole %d x %d A and %d x %d B\n",
                     a_nrow, a_ncol, b_nrow, b_ncol);
        return;
    }
    double t0 = ca3dmm_wtime_sec();
    ca3dmm_engine_p e = (ca3dmm_engine_p) calloc(1, sizeof(ca3dmm_engine_s));
    if (!e) return;
    e->m = m; e->n = n; e->k = k;
    e->n_proc = p;
    e->my_rank = 0;
    e->trans_A = trans_A ? 1 : 0;
    e->trans_B = trans_B ? 1 : 0;
    e->dev_type = dev_type;
    int mp, np, kp, rp;
    if (choose_grid(p, m, n, k, proc_grid, &mp, &np, &kp, &rp)) {
        ca3dmm_engine_free(&e);
        return;
    }
    e->mp = mp; e->np = np; e->kp = kp; e->rp = rp;
    e->is_BTB = 0;
    finish_init(e, dst_C_srow, dst_C_nrow, dst_C_scol, dst_C_ncol, engine_, workbuf_bytes, t0);
}

void ca3dmm_engine_init_BTB(const int n, const int k, const int src_B_srow, const int src_B_nrow,
                            const int src_B_scol, const int src_B_ncol, const int dst_C_srow,
                            const int dst_C_nrow, const int dst_C_scol, const int dst_C_ncol,
                            const int *proc_grid, MPI_Comm comm, dev_type_t dev_type,
                            ca3dmm_engine_p *engine_, size_t *workbuf_bytes)
{
    if (engine_ == NULL) return;
    *engine_ = NULL;
    if (is_dev_type_valid(dev_type) == 0) {
        ERROR_PRINTF("Invalid device type %d\n", dev_type);
        return;
    }
    int p = ca3dmm_vcomm_size(comm);
    if (p < 1 || n < 1 || k < 1) {
        ERROR_PRINTF("Invalid communicator or size n, k = %d, %d\n", n, k);
        return;
    }
    if (src_B_srow != 0 || src_B_scol != 0 || src_B_nrow != k || src_B_ncol != n) {
        ERROR_PRINTF("Folded call: src_B must describe the whole %d x %d B\n", k, n);
        return;
    }
    double t0 = ca3dmm_wtime_sec();
    ca3dmm_engine_p e = (ca3dmm_engine_p) calloc(1, sizeof(ca3dmm_engine_s));
    if (!e) return;
    e->m = n; e->n = n; e->k = k;
    e->n_proc = p;
    e->dev_type = dev_type;
    int mp, np, kp, rp, gen = 1;
    if (proc_grid != NULL) {
        mp = proc_grid[0]; np = proc_grid[1]; kp = proc_grid[2];
        rp = p - mp * np * kp;
        if ((mp != np) || (rp < 0))
            WARNING_PRINTF("Invalid process grid specified: mp, np, kp = %d, %d, %d\n", mp, np, kp);
        else
            gen = 0;
    }
    if (gen) {
        /* src/ca3dmm.c:492-502: n x n x k planner, then (default on) fold a
         * factor 4 of kp into a 2 x 2 larger mn-plane */
        calc_3d_decomposition_nk(p, n, k, &np, &kp, &rp);
        int reduce_kp;
        GET_ENV_INT_VAR(reduce_kp, "CA3DMM_REDUCE_KP", "reduce_kp", 1, 0, 1);
        if (reduce_kp && kp >= 4 && kp % 4 == 0) {
            kp /= 4;
            np *= 2;
        }
    }
    mp = np;
    if (mp < 1 || np < 1 || kp < 1 || mp * np * kp > p) {
        ERROR_PRINTF("3D decomposition function error: p = %d, mp, np, kp = %d, %d, %d\n", p, mp,
                     np, kp);
        free(e);
        return;
    }
    e->mp = mp; e->np = np; e->kp = kp; e->rp = rp;
    e->is_BTB = 1;
    e->trans_A = 1;   /* op(A) = B^T, read from B */
    e->trans_B = 0;
    finish_init(e, dst_C_srow, dst_C_nrow, dst_C_scol, dst_C_ncol, engine_, workbuf_bytes, t0);
}

void ca3dmm_engine_attach_workbuf(ca3dmm_engine_p e, void *workbuf_h, void *workbuf_d)
{
    if (e == NULL) return;
    plan_t *pl = (plan_t *) e->impl;
    e->workbuf_h = workbuf_h;
    e->workbuf_d = workbuf_d;
    if (workbuf_d == NULL) {
        ERROR_PRINTF("A device work buffer is required\n");
        e->last_error = CA3DMM_EINVAL;
        return;
    }
    if (plan_cuda_init(pl) != CA3DMM_OK) {
        ERROR_PRINTF("Failed to create the engine's CUDA resources\n");
        e->last_error = CA3DMM_ECUDA;
        return;
    }
    char *w = (char *) workbuf_d;
    e->A_rd_recv_d = w + pl->off_A;
    e->A_trans_d = e->A_rd_recv_d;
    e->A_2dmm_d = e->A_rd_recv_d;
    e->B_rd_recv_d = w + pl->off_B;
    e->B_trans_d = e->B_rd_recv_d;
    e->B_2dmm_d = e->B_rd_recv_d;
    e->C_2dmm_d = e->kp > 1 ? (void *) (w + pl->off_slab) : NULL;
    e->C_out_d = w + pl->off_cout;
    pl->plan_valid = 0;
}

void ca3dmm_engine_free(ca3dmm_engine_p *engine_)
{
    if (engine_ == NULL || *engine_ == NULL) return;
    ca3dmm_engine_p e = *engine_;
    free(e->AB_agv_recvcnts);
    free(e->AB_agv_displs);
    free(e->C_rs_recvcnts);
    if (e->alloc_workbuf && e->workbuf_d) dev_type_free(e->workbuf_d, DEV_TYPE_CUDA);
    free(e->cannon_engine);
    plan_free((plan_t *) e->impl);
    free(e);
    *engine_ = NULL;
}

/* Pack descriptor of op(A) rows [r, rend) of block b from a source with
 * leading dimension lds: an M-major (transposing when trans_A) copy, or, when
 * the launch reads A K-major, a plain copy of the transposed source's columns
 * into the K-major layout. */
static void a_pack_desc(const ca3dmm_engine_p e, const plan_t *pl, const blk_t *b, int r, int rend,
                        long long lds, ca3dmm_pack_desc_t *d)
{
    memset(d, 0, sizeof(*d));
    d->lds = lds;
    if (pl->a_kmajor) {
        d->rows = b->cols; d->cols = rend - r; d->trans = 0;
        d->src_off = (long long) b->c0 + (long long) (b->r0 + r) * lds;
        d->dst_off = (long long) (b->off / sizeof(double)) + (long long) r * b->kld;
        d->ldd = b->kld;
    } else {
        d->rows = rend - r; d->cols = b->cols; d->trans = e->trans_A;
        d->src_off = e->trans_A ? (long long) b->c0 + (long long) (b->r0 + r) * lds
                                : (long long) (b->r0 + r) + (long long) b->c0 * lds;
        d->dst_off = (long long) (b->off / sizeof(double)) + r;
        d->ldd = b->ld;
    }
}

/* Build the per-call device plan into pinned staging and upload it. */
static int plan_upload(ca3dmm_engine_p e, const void *A, int ldA, const void *B, int ldB,
                       void *dst, int ldC, cudaStream_t st)
{
    plan_t *pl = (plan_t *) e->impl;
    char *w = (char *) e->workbuf_d, *h = (char *) pl->stage;
    /* An operand block whose address and leading dimension suit the GEMM's
     * tensor maps (16-byte aligned start, even ld) is read in place: op(B)
     * untransposed (K-major), op(A) untransposed (M-major) or transposed
     * (K-major, when every A block qualifies: one A layout per launch).  The
     * others are packed (and transposed) into the work buffer. */
    ca3dmm_pack_desc_t *pa = (ca3dmm_pack_desc_t *) (h + pl->off_packA);
    /* A transposed op(A) with an even ldA is read K-major: blocks with an
     * aligned start in place, the others (an odd first k index) copied, not
     * transposed, into the K-major layout. */
    pl->a_kmajor = e->trans_A && (ldA & 1) == 0;
    for (int i = 0; i < pl->nA; i++) {
        blk_t *b = &pl->A[i];
        ca3dmm_pack_desc_t *d = &pa[i];
        a_pack_desc(e, pl, b, 0, b->rows, ldA, d);
        b->direct = NULL;
        if ((!e->trans_A || pl->a_kmajor) && (ldA & 1) == 0 &&
            (((uintptr_t) A + sizeof(double) * (uintptr_t) d->src_off) & 15) == 0) {
            b->direct = (const double *) A + d->src_off;
            b->direct_ld = ldA;
            d->rows = 0;
        }
    }
    pl->packA_tma = 0;
    if (e->trans_A && !pl->a_kmajor &&
        ca3dmm_pack_tma_prepare(pa, pl->nA, (const double *) A, h + pl->off_tmapA,
                                &pl->pack_tiles_A) == CA3DMM_OK)
        pl->packA_tma = 1;
    else
        pl->pack_tiles_A = ca3dmm_pack_tiles(pa, pl->nA);
    ca3dmm_pack_desc_t *pb = (ca3dmm_pack_desc_t *) (h + pl->off_packB);
    for (int i = 0; i < pl->nB; i++) {
        blk_t *b = &pl->B[i];
        ca3dmm_pack_desc_t *d = &pb[i];
        memset(d, 0, sizeof(*d));
        d->rows = b->rows; d->cols = b->cols; d->trans = e->trans_B; d->lds = ldB;
        d->src_off = e->trans_B ? (long long) b->c0 + (long long) b->r0 * ldB
                                : (long long) b->r0 + (long long) b->c0 * ldB;
        d->dst_off = (long long) ((b->off) / sizeof(double));
        d->ldd = b->ld;
        b->direct = NULL;
        if (!e->trans_B && (ldB & 1) == 0 &&
            (((uintptr_t) B + sizeof(double) * (uintptr_t) d->src_off) & 15) == 0) {
            b->direct = (const double *) B + d->src_off;
            b->direct_ld = ldB;
            d->rows = 0;
        }
    }
    /* Plain FP64 with slab 0's operand blocks read in place (a 16-byte aligned
     * start and an even ld, so the same tensor maps reach every k): the kp
     * slabs of the one (merged) group are consecutive k ranges of the same A
     * and B, so when one slab alone has enough tiles for every SM they run as
     * one GEMM over all of k that writes C directly -- no packs of the other
     * slabs' blocks, no slab buffers, no slab sum.  The plain path's contract
     * is k u |A||B| accuracy, not the slab sum's rounding order (split
     * precision keeps the slabs: its exponents are per slab). */
    pl->plain_merged = 0;
    if (pl->merge_allowed && e->gemm_mode == CA3DMM_GEMM_PLAIN && !pl->sym && !e->is_BTB &&
        pl->ksplit == 1 &&
        e->kp > 1 && pl->tmn == 1 && pl->tnn == 1 && pl->A[0].direct && pl->B[0].direct &&
        (long long) ((e->m + 127) / 128) * ((e->n + 127) / 128) >= 4LL * CA3DMM_SMS_B200) {
        pl->plain_merged = 1;
        for (int i = 1; i < pl->nA; i++) pa[i].rows = 0;
        for (int i = 1; i < pl->nB; i++) pb[i].rows = 0;
        pl->packA_tma = 0;
        pl->pack_tiles_A = ca3dmm_pack_tiles(pa, pl->nA);
    }
    pl->packB_tma = 0;
    if (e->trans_B && !pl->plain_merged && ca3dmm_pack_tma_prepare(pb, pl->nB, (const double *) B, h + pl->off_tmapB,
                                              &pl->pack_tiles_B) == CA3DMM_OK)
        pl->packB_tma = 1;
    else
        pl->pack_tiles_B = ca3dmm_pack_tiles(pb, pl->nB);
    /* output target of the GEMM (kp == 1) or of the reduction (kp > 1) */
    int whole = pl->has_dst && pl->dst_srow == 0 && pl->dst_scol == 0 && pl->dst_nrow == e->m &&
                pl->dst_ncol == e->n;
    double *out = whole ? (double *) dst : (double *) (w + pl->off_cout);
    long long ldo = whole ? ldC : e->m;
    ca3dmm_pack_desc_t *pc = (ca3dmm_pack_desc_t *) (h + pl->off_copy);
    memset(pc, 0, sizeof(*pc));
    if (pl->has_dst && !whole) {
        pc->rows = pl->dst_nrow; pc->cols = pl->dst_ncol; pc->lds = e->m; pc->ldd = ldC;
        pc->src_off = (long long) pl->dst_srow + (long long) pl->dst_scol * e->m;
    }
    pl->pack_tiles_C = ca3dmm_pack_tiles(pc, 1);
    ca3dmm_dgemm_desc_t *gd = pl->gd;
    const int ks = pl->ksplit, nslab = e->kp * ks;

    for (int i = 0; i < pl->ngroup; i++) {
        group_t *g = &pl->groups[i];
        const blk_t *ba = &pl->A[g->a_blk], *bb = &pl->B[g->b_blk];
        const double *a = ba->direct ? ba->direct : (const double *) (w + ba->off);
        const long long lda = ba->direct ? ba->direct_ld : (pl->a_kmajor ? ba->kld : ba->ld);
        const double *b = bb->direct ? bb->direct : (const double *) (w + bb->off);
        const long long ldb = bb->direct ? bb->direct_ld : bb->ld;
        /* the group's first row inside its A block and first column inside its B block */
        const long long dr = g->m0 - ba->r0, dc = g->n0 - bb->c0;
        a += pl->a_kmajor ? dr * lda : dr;
        b += dc * ldb;
        for (int sub = 0; sub < ks; sub++) {
            /* sub-slab k range: a multiple of 16 (whole k-tiles, 16-byte aligned starts) */
            const int k0 = (int) ((long long) g->kz * sub / ks) / 16 * 16;
            const int k1 = sub + 1 < ks ? (int) ((long long) g->kz * (sub + 1) / ks) / 16 * 16 : g->kz;
            ca3dmm_dgemm_desc_t *q = &gd[i * ks + sub];
            q->A = a + (pl->a_kmajor ? (long long) k0 : (long long) k0 * lda);
            q->lda = lda;
            q->B = b + k0;
            q->ldb = ldb;
            if (pl->plain_merged) {
                /* slab 0's group carries all of k (its blocks start at k = 0); the
                 * other slabs' groups are empty */
                const int first = g->tk == 0;
                q->C = out + g->m0 + (size_t) g->n0 * ldo;
                q->ldc = ldo;
                q->m = first ? g->mz : 0; q->n = first ? g->nz : 0; q->k = first ? e->k : 0;
                q->alpha = 1.0; q->beta = 0.0;
                q->raster = e->raster;
                q->a_kmajor = pl->a_kmajor;
                continue;
            }
            if (nslab > 1) {
                q->C = (double *) (w + pl->off_slab) + (size_t) (g->tk * ks + sub) * pl->slab_stride +
                       g->m0 + (size_t) g->n0 * pl->slab_ld;
                q->ldc = pl->slab_ld;
            } else {
                q->C = out + g->m0 + (size_t) g->n0 * ldo;
                q->ldc = ldo;
            }
            q->m = g->mz; q->n = g->nz; q->k = k1 - k0;
            q->alpha = 1.0; q->beta = 0.0;
            q->raster = e->raster;
            q->a_kmajor = pl->a_kmajor;
        }
    }
    int rc = ca3dmm_dgemm_plan_encode_tn(gd, pl->ngroup * ks, h + pl->off_gemm, &pl->gemm_tiles,
                                         pl->plain_tile_n);
    if (rc) return rc;
    if (e->gemm_mode == CA3DMM_GEMM_OZAKI) {
        ca3dmm_oz_blk_t *ob = pl->ob;
        ca3dmm_oz_src_t *os = pl->os;
        ca3dmm_oz_group_t *og = pl->og;
        for (int i = 0; i < pl->nA + pl->nB; i++) {
            os[i].base = NULL;
            os[i].ld = i < pl->nA ? ldA : ldB;
            os[i].trans = i < pl->nA ? e->trans_A : e->trans_B;
            os[i].pad = 0;
        }
        for (int i = 0; i < pl->nA; i++) {
            ob[i].r0 = pl->A[i].r0; ob[i].c0 = pl->A[i].c0;
            ob[i].rows = pl->A[i].rows; ob[i].cols = pl->A[i].cols;
            ob[i].alias = -1;
            /* B^T B: the op(A) block Bt(r0.., c0..) holds the elements of the B
             * block B(c0.., r0..); slice it once */
            for (int j = 0; e->is_BTB && j < pl->nB && ob[i].alias < 0; j++)
                if (pl->B[j].r0 == pl->A[i].c0 && pl->B[j].rows == pl->A[i].cols &&
                    pl->B[j].c0 == pl->A[i].r0 && pl->B[j].cols == pl->A[i].rows)
                    ob[i].alias = j;
        }
        for (int i = 0; i < pl->nB; i++) {
            ob[pl->nA + i].r0 = pl->B[i].r0; ob[pl->nA + i].c0 = pl->B[i].c0;
            ob[pl->nA + i].rows = pl->B[i].rows; ob[pl->nA + i].cols = pl->B[i].cols;
            ob[pl->nA + i].alias = -1;
        }
        /* The kp slabs of one (task_m, task_n) block form one work unit that
         * adds its slabs into the output in slab order (no slab buffers, no
         * reduction launch) -- when the chained units still give every SM
         * several output tiles; otherwise (e.g. B^T B with a small C) each
         * slab is its own unit and the slab reduction runs after the GEMM. */
        const int tmn = pl->tmn, tnn = pl->tnn;
        long long unit_tiles = 0;
        for (int u = 0; u < tmn * tnn; u++) {
            const group_t *g = &pl->groups[u];
            unit_tiles += (long long) ((g->mz + 127) / 128) * ((g->nz + 63) / 64);
        }
        pl->oz_fused = e->kp > 1 && !pl->sym && unit_tiles >= 8LL * ca3dmm_device_sm_count();
        for (int i = 0; i < pl->ngroup; i++) {
            const group_t *g = &pl->groups[i];
            og[i].a_blk = g->a_blk; og[i].b_blk = g->b_blk;
            og[i].row0 = g->m0 - pl->A[g->a_blk].r0;
            og[i].col0 = g->n0 - pl->B[g->b_blk].c0;
            if (pl->oz_fused || e->kp == 1) {
                og[i].C = out + g->m0 + (size_t) g->n0 * ldo;
                og[i].ldc = ldo;
            } else {
                og[i].C = (double *) (w + pl->off_slab) + (size_t) g->tk * pl->slab_stride + g->m0 +
                          (size_t) g->n0 * pl->slab_ld;
                og[i].ldc = pl->slab_ld;
            }
            og[i].m = g->mz; og[i].n = g->nz; og[i].k = g->kz;
            og[i].raster = e->raster;
        }
        ca3dmm_oz_unit_t *un = pl->ou;
        for (int u = 0; u < tmn * tnn; u++) {
            un[u].group = u;             /* (tk = 0, tm, tn) = tm * tnn + tn */
            un[u].nsub = e->kp;
            un[u].sub_stride = tmn * tnn;
        }
        rc = ca3dmm_oz_plan_encode(&pl->oz, e->ozaki_slices, pl->nA, ob, os, pl->nB,
                                   ob + pl->nA, os + pl->nA, pl->ngroup, og,
                                   pl->oz_fused ? tmn * tnn : 0, pl->oz_fused ? un : NULL,
                                   w + pl->off_oz, pl->oz_bytes, h + pl->off_ozplan,
                                   w + pl->off_ozplan);
        if (rc) return rc;
    }
    if (e->gemm_mode == CA3DMM_GEMM_CRT) {
        const int ns = pl->crt_nsl;
        for (int i = 0; i < 2 * ns; i++) {
            pl->cs[i].base = NULL;
            pl->cs[i].ld = i < ns ? ldA : ldB;
            pl->cs[i].trans = i < ns ? e->trans_A : e->trans_B;
            pl->cs[i].pad = 0;
        }
        for (int s2 = 0; s2 < ns; s2++) {
            ca3dmm_crt_group_t *g = &pl->cg[s2];
            if (ns > 1) {
                g->C = (double *) (w + pl->off_slab) + (size_t) s2 * pl->slab_stride;
                g->ldc = pl->slab_ld;
            } else {
                g->C = out;
                g->ldc = ldo;
            }
            /* host-buffer exec: bands of the pipeline's rows; device exec: wide
             * bands, so that one modulus' residues of op(A) stay in L2 while
             * the tile columns stream through */
            g->band = pl->upload_for_host ? e->raster
                                          : (pl->crt_band > 0 ? pl->crt_band : (e->m + 127) / 128);
            g->tile_n = pl->crt_tile_n;
        }
        rc = ca3dmm_crt_plan_encode(&pl->crt, e->crt_moduli, ns, pl->cb, pl->cs, ns, pl->cb + ns,
                                    pl->cs + ns, ns, pl->cg, w + pl->off_crt, pl->crt_bytes,
                                    h + pl->off_crtplan, w + pl->off_crtplan);
        if (rc) return rc;
        e->crt_bits = pl->crt.p_min;
    }
    memset(h + pl->off_status, 0, 64);
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(w, h, pl->stage_bytes, cudaMemcpyHostToDevice, st));
    for (int i = 0; i < pl->ncanary; i++)
        CA3DMM_CUDA_TRY(cudaMemsetAsync(w + pl->canary[i], CANARY_BYTE, CANARY_BYTES, st));
    pl->c_A = A; pl->c_B = B; pl->c_ldA = ldA; pl->c_ldB = ldB;
    pl->c_dst = dst; pl->c_ldC = ldC;
    pl->plan_valid = 1;
    return CA3DMM_OK;
}

/* Pack the op(A) (which = 0) or op(B) (which = 1) blocks that are not read in
 * place: TMA-staged transposes when the plan prepared them, else the plain
 * pack kernel. */
static int launch_pack_side(ca3dmm_engine_p e, int which, const void *src, cudaStream_t st)
{
    plan_t *pl = (plan_t *) e->impl;
    char *w = (char *) e->workbuf_d;
    const size_t off_desc = which ? pl->off_packB : pl->off_packA;
    const int nd = which ? pl->nB : pl->nA, tiles = which ? pl->pack_tiles_B : pl->pack_tiles_A;
    if (which ? pl->packB_tma : pl->packA_tma)
        return ca3dmm_pack_tma_launch(w + (which ? pl->off_tmapB : pl->off_tmapA),
                                      (const ca3dmm_pack_desc_t *) (w + off_desc), nd, tiles,
                                      (double *) w, (int *) (w + pl->off_status), 5.0, st);
    return ca3dmm_pack_launch((const double *) src, (double *) w,
                              (const ca3dmm_pack_desc_t *) (w + off_desc), nd, tiles, st);
}

/* The device status word after a call: 0, a bounded wait that ran out, or
 * an overwritten guard band (status[1] holds its index). */
static int device_status_error(const plan_t *pl)
{
    const int code = pl->status_h[0];
    if (code == 0) return CA3DMM_OK;
    if (code == 6) {
        const int b = pl->status_h[1];
        ERROR_PRINTF("Work buffer guard band %d (bytes %lld .. %lld) was overwritten\n", b,
                     b >= 0 && b < pl->ncanary ? pl->canary[b] : -1LL,
                     b >= 0 && b < pl->ncanary ? pl->canary[b] + CANARY_BYTES - 1 : -1LL);
        return CA3DMM_ECANARY;
    }
    ERROR_PRINTF("Device status %d: a bounded wait ran out\n", code);
    return CA3DMM_ETIMEOUT;
}

/* With CA3DMM_CANARY=1: compare every guard band with its fill pattern. */
static int launch_guard_check(const ca3dmm_engine_p e, const plan_t *pl, int *status_d,
                              cudaStream_t st)
{
    if (!pl->check_canary || pl->ncanary == 0) return CA3DMM_OK;
    ca3dmm_guard_bands_t g;
    memset(&g, 0, sizeof(g));
    g.n = pl->ncanary;
    g.bytes = CANARY_BYTES;
    g.pattern = CANARY_BYTE;
    for (int i = 0; i < pl->ncanary; i++) g.off[i] = pl->canary[i];
    return ca3dmm_guard_check_launch(e->workbuf_d, &g, status_d, st);
}

/* Modular mode, device exec of one group: the bands of its work list (crt_band
 * tile rows each) run as one GEMM launch per band on `st`, and the
 * reconstruction of band b runs on the auxiliary stream as soon as band b's
 * residue planes are complete -- beside the GEMM of band b + 1 (two blocks per
 * SM fit next to the GEMM's CTA: 2 x 256 x 48 registers and 2 x 4 KB of shared
 * memory, with the same shared-memory carveout).  Returns the number of bands
 * so run (0: not overlapped). */
static int crt_overlapped_gemm(ca3dmm_engine_p e, plan_t *pl, int *status_d, cudaStream_t st,
                               int *rc_out)
{
    *rc_out = CA3DMM_OK;
    if (!pl->crt_overlap || pl->crt_nsl != 1 || pl->upload_for_host || e->m <= 0) return 0;
    const int tiles_m = (e->m + 127) / 128;
    const int band = pl->crt_band > 0 ? pl->crt_band : tiles_m;
    int per = band, nb = (tiles_m + band - 1) / band;
    while (nb > CRT_MAX_BANDS) {              /* several work-list bands per launch */
        per += band;
        nb = (tiles_m + per - 1) / per;
    }
    if (nb < 2) return 0;
    if (!pl->aux_ok) {
        if (cudaStreamCreateWithFlags(&pl->st_aux, cudaStreamNonBlocking) != cudaSuccess) return 0;
        for (int i = 0; i < CRT_MAX_BANDS; i++)
            cudaEventCreateWithFlags(&pl->ev_band[i], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&pl->ev_join, cudaEventDisableTiming);
        pl->aux_ok = 1;
    }
    const char *hp = (const char *) pl->stage + pl->off_crtplan;
    const int sms = ca3dmm_device_sm_count();
    int rc = CA3DMM_OK;
    for (int b = 0; b < nb && !rc; b++) {
        const int lo = b * per, hi = lo + per < tiles_m ? lo + per : tiles_m;
        int begin = 0, count = 0;
        rc = ca3dmm_crt_group_items(hp, 0, lo, hi, &begin, &count);
        if (rc) break;
        ca3dmm_tile_ranges_t rg;
        memset(&rg, 0, sizeof(rg));
        rg.n = 1;
        rg.begin[0] = begin;
        rg.len[0] = count;
        rc = ca3dmm_crt_run_gemm(&pl->crt, &rg, status_d, 5.0, st);
        if (rc) break;
        if (cudaEventRecord(pl->ev_band[b], st) != cudaSuccess ||
            cudaStreamWaitEvent(pl->st_aux, pl->ev_band[b], 0) != cudaSuccess) {
            rc = CA3DMM_ECUDA;
            break;
        }
        /* one or two blocks per SM beside the next band's GEMM; the last band alone */
        const int r1 = hi * 128 < e->m ? hi * 128 : e->m;
        rc = ca3dmm_crt_run_reconstruct_capped(&pl->crt, 0, 1, lo * 128, r1,
                                               b + 1 < nb ? pl->crt_overlap_blocks * sms : 0,
                                               pl->st_aux);
    }
    if (rc) {
        /* nothing of this exec may still run on the auxiliary stream after it returns */
        cudaEventRecord(pl->ev_join, pl->st_aux);
        cudaStreamWaitEvent(st, pl->ev_join, 0);
    }
    *rc_out = rc;
    return nb;
}

static int exec_device(ca3dmm_engine_p e, const void *src_A, int ldA, const void *src_B, int ldB,
                       void *dst_C, int ldC, cudaStream_t st)
{
    plan_t *pl = (plan_t *) e->impl;
    char *w = (char *) e->workbuf_d;
    if (e->is_BTB) { src_A = src_B; ldA = ldB; }
    const int a_rows = e->trans_A ? e->k : e->m, b_rows = e->trans_B ? e->n : e->k;
    if (!src_A || !src_B || ldA < a_rows || ldB < b_rows) {
        ERROR_PRINTF("Invalid operands: ldA = %d (>= %d), ldB = %d (>= %d)\n", ldA, a_rows, ldB,
                     b_rows);
        return CA3DMM_EINVAL;
    }
    if (pl->has_dst && (dst_C == NULL || ldC < pl->dst_nrow)) {
        ERROR_PRINTF("Invalid dst_C / ldC = %d (>= %d)\n", ldC, pl->dst_nrow);
        return CA3DMM_EINVAL;
    }
    int rc;
    if (!pl->plan_valid || pl->c_A != src_A || pl->c_B != src_B || pl->c_ldA != ldA ||
        pl->c_ldB != ldB || pl->c_dst != dst_C || pl->c_ldC != ldC) {
        rc = plan_upload(e, src_A, ldA, src_B, ldB, dst_C, ldC, st);
        if (rc) return rc;
    } else if (cudaMemsetAsync(w + pl->off_status, 0, 64, st) != cudaSuccess) {
        return CA3DMM_ECUDA;
    }
    int timing = e->sync_exec && pl->events_ok;
    if (timing) cudaEventRecord(pl->ev[0], st);
    const int crt = e->gemm_mode == CA3DMM_GEMM_CRT;
    /* NVTX ranges mark the phases of the reference's timers on the host
     * timeline (visible to nsys and to ncu --nvtx); each closes before an
     * error return */
    nvtxRangePushA("ca3dmm: redistribute (pack / slice operands)");
    if (crt) {
        rc = ca3dmm_crt_run_pack(&pl->crt, src_A, src_B, st);
    } else if (e->gemm_mode == CA3DMM_GEMM_OZAKI) {
        rc = ca3dmm_oz_run_pack(&pl->oz, src_A, src_B, st);
    } else {
        rc = launch_pack_side(e, 0, src_A, st);
        if (!rc) rc = launch_pack_side(e, 1, src_B, st);
    }
    nvtxRangePop();
    if (rc) return rc;
    if (timing) cudaEventRecord(pl->ev[1], st);
    int *status_d = (int *) (w + pl->off_status);
    nvtxRangePushA("ca3dmm: GEMM (2D Cannon)");
    int crt_bands = 0;
    if (crt) {
        crt_bands = crt_overlapped_gemm(e, pl, status_d, st, &rc);
        if (!crt_bands && !rc) rc = ca3dmm_crt_run_gemm(&pl->crt, NULL, status_d, 5.0, st);
    } else if (e->gemm_mode == CA3DMM_GEMM_OZAKI) {
        rc = ca3dmm_oz_run_gemm(&pl->oz, status_d, 5.0, st);
        if (!rc) rc = ca3dmm_oz_run_nonfinite(&pl->oz, NULL, src_A, src_B, st);
    } else
        rc = ca3dmm_dgemm_launch_tn(w + pl->off_gemm, pl->ngroup * pl->ksplit, pl->gemm_tiles,
                                    pl->a_kmajor, status_d, 5.0, st, pl->plain_tile_n);
    nvtxRangePop();
    if (rc) return rc;
    if (timing) cudaEventRecord(pl->ev[2], st);
    nvtxRangePushA("ca3dmm: reduce (slab sum, reconstruction)");
    if (crt) {
        /* the modular mode's reconstruction of C (with the slab sum below, the
         * "reduce" phase of the timers); overlapped: what is left of it after
         * the last GEMM band */
        if (crt_bands) {
            if (cudaEventRecord(pl->ev_join, pl->st_aux) != cudaSuccess ||
                cudaStreamWaitEvent(st, pl->ev_join, 0) != cudaSuccess)
                rc = CA3DMM_ECUDA;
        } else {
            rc = ca3dmm_crt_run_reconstruct(&pl->crt, 0, pl->crt_nsl, 0, INT32_MAX, st);
        }
        if (!rc) rc = ca3dmm_crt_run_nonfinite(&pl->crt, 0, pl->crt_nsl, 0, INT32_MAX, src_A, src_B,
                                               st);
    }
    int whole = pl->has_dst && pl->dst_srow == 0 && pl->dst_scol == 0 && pl->dst_nrow == e->m &&
                pl->dst_ncol == e->n;
    double *out = whole ? (double *) dst_C : (double *) (w + pl->off_cout);
    long long ldo = whole ? ldC : e->m;
    const int nred = crt ? pl->crt_nsl
                         : e->gemm_mode == CA3DMM_GEMM_OZAKI ? (pl->oz_fused ? 1 : e->kp)
                                                              : (pl->plain_merged ? 1 : e->kp * pl->ksplit);
    if (!rc && nred > 1)
        rc = ca3dmm_reduce_slabs_launch((const double *) (w + pl->off_slab),
                                        (long long) pl->slab_stride, pl->slab_ld, nred, e->m,
                                        e->n, out, ldo, st);
    if (!rc && pl->sym && !crt)      /* the modular mode computes all of C */
        rc = ca3dmm_mirror_upper_launch(out, ldo, e->m, st);
    nvtxRangePop();
    if (rc) return rc;
    if (timing) cudaEventRecord(pl->ev[3], st);
    if (pl->has_dst && !whole) {
        nvtxRangePushA("ca3dmm: C to dst_C");
        rc = ca3dmm_pack_launch((const double *) (w + pl->off_cout), (double *) dst_C,
                                (const ca3dmm_pack_desc_t *) (w + pl->off_copy), 1,
                                pl->pack_tiles_C, st);
        nvtxRangePop();
        if (rc) return rc;
    }
    if (timing) cudaEventRecord(pl->ev[4], st);
    rc = launch_guard_check(e, pl, status_d, st);
    if (rc) return rc;
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(pl->status_h, status_d, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                                    st));
    if (e->sync_exec) {
        CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
        rc = device_status_error(pl);
        if (rc) return rc;
        if (timing) {
            float t_pack = 0, t_gemm = 0, t_red = 0, t_copy = 0;
            cudaEventElapsedTime(&t_pack, pl->ev[0], pl->ev[1]);
            cudaEventElapsedTime(&t_gemm, pl->ev[1], pl->ev[2]);
            cudaEventElapsedTime(&t_red, pl->ev[2], pl->ev[3]);
            cudaEventElapsedTime(&t_copy, pl->ev[3], pl->ev[4]);
            e->redist_ms += t_pack + t_copy;
            e->cannon_ms += t_gemm;
            e->reduce_ms += t_red;
            if (e->cannon_engine) {
                e->cannon_engine->gemm_ms += t_gemm;
                e->cannon_engine->exec_ms += t_gemm;
                e->cannon_engine->n_exec++;
            }
            if (e->print_timing) {
                INFO_PRINTF("Redistribute A & B time = %.2f ms\n", t_pack);
                INFO_PRINTF("2D Cannon time          = %.2f ms\n", t_gemm);
                INFO_PRINTF("Reduce-scatter C time   = %.2f ms\n", t_red);
                INFO_PRINTF("Redistribute C time     = %.2f ms\n", t_copy);
            }
        }
    }
    return CA3DMM_OK;
}

void ca3dmm_engine_exec(ca3dmm_engine_p e, const void *src_A, const int ldA, const void *src_B,
                        const int ldB, void *dst_C, const int ldC)
{
    if (e == NULL) {
        ERROR_PRINTF("ca3dmm_engine not initialized\n");
        return;
    }
    if (e->workbuf_d == NULL || ((plan_t *) e->impl)->stage == NULL) {
        ERROR_PRINTF("ca3dmm_engine has no device work buffer attached\n");
        e->last_error = CA3DMM_EINVAL;
        return;
    }
    if (e->gemm_auto == 1) {
        /* CA3DMM_GEMM_AUTO: tune on this exec's operands first */
        int rc = ca3dmm_engine_autotune_env(e, src_A, ldA, src_B, ldB, dst_C, ldC);
        if (rc) {
            e->last_error = rc;
            ERROR_PRINTF("ca3dmm_engine_exec: tuning failed (error %d)\n", rc);
            return;
        }
    }
    double t0 = ca3dmm_wtime_sec();
    nvtxRangePushA("ca3dmm_engine_exec");
    int rc = exec_device(e, src_A, ldA, src_B, ldB, dst_C, ldC, (cudaStream_t) e->stream);
    nvtxRangePop();
    e->last_error = rc;
    if (rc) {
        ERROR_PRINTF("ca3dmm_engine_exec failed (error %d)\n", rc);
        return;
    }
    if (e->sync_exec) {
        double ms = 1000.0 * (ca3dmm_wtime_sec() - t0);
        e->exec_ms += ms;
        e->n_exec++;
        if (e->print_timing) INFO_PRINTF("CA3DMM exec time        = %.2f ms\n\n", ms);
    }
}

/* ---------------------------------------------------------------------------
 * ca3dmm_engine_exec_host: host buffers in and out, copies overlapped with the
 * computation band by band (see struct host_exec). */

static int hx_create(ca3dmm_engine_p e, struct host_exec **out)
{
    plan_t *pl = (plan_t *) e->impl;
    if (pl->hx) { *out = pl->hx; return CA3DMM_OK; }
    struct host_exec *x = (struct host_exec *) calloc(1, sizeof(struct host_exec));
    if (!x) return CA3DMM_ENOMEM;
    pl->hx = x;
    x->built_mode = -1;
    const int a_rows = e->trans_A ? e->k : e->m, a_cols = e->trans_A ? e->m : e->k;
    const int b_rows = e->trans_B ? e->n : e->k, b_cols = e->trans_B ? e->k : e->n;
    x->lda = ca3dmm_round_up(a_rows > 0 ? a_rows : 1, 2);
    x->ldb = ca3dmm_round_up(b_rows > 0 ? b_rows : 1, 2);
    x->ldc = ca3dmm_round_up(pl->dst_nrow > 0 ? pl->dst_nrow : 1, 2);
    if (!e->is_BTB &&
        cudaMalloc((void **) &x->dA, sizeof(double) * (size_t) x->lda * (size_t) (a_cols > 0 ? a_cols : 1)) != cudaSuccess)
        return CA3DMM_ENOMEM;
    if (cudaMalloc((void **) &x->dB, sizeof(double) * (size_t) x->ldb * (size_t) (b_cols > 0 ? b_cols : 1)) != cudaSuccess)
        return CA3DMM_ENOMEM;
    if (cudaMalloc((void **) &x->dC, sizeof(double) * (size_t) x->ldc * (size_t) (pl->dst_ncol > 0 ? pl->dst_ncol : 1)) != cudaSuccess)
        return CA3DMM_ENOMEM;
    if (cudaStreamCreateWithFlags(&x->s_in, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&x->s_out, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&x->ev_b, cudaEventDisableTiming) != cudaSuccess)
        return CA3DMM_ECUDA;
    for (int i = 0; i < HX_MAX_BANDS; i++)
        if (cudaEventCreateWithFlags(&x->ev_a[i], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&x->ev_c[i], cudaEventDisableTiming) != cudaSuccess)
            return CA3DMM_ECUDA;
    x->ok = 1;
    *out = x;
    return CA3DMM_OK;
}

/* Output row bands and, per band, the GEMM tile ranges and the descriptors
 * that pack or slice its op(A) rows.  Returns the band count (0 or 1: no
 * pipelining for this layout). */
/* Bands of the modular mode: one group over all of C (a single k slab), whose
 * work list numbers its items in bands of `raster` tile rows, so a band of
 * output rows is one range; per band the residue descriptors of its op(A)
 * rows. */
static int hx_build_bands_crt(ca3dmm_engine_p e, struct host_exec *x, cudaStream_t st)
{
    plan_t *pl = (plan_t *) e->impl;
    const int whole = pl->has_dst && pl->dst_srow == 0 && pl->dst_scol == 0 &&
                      pl->dst_nrow == e->m && pl->dst_ncol == e->n;
    if (e->is_BTB || !whole || pl->crt_nsl != 1 || e->m <= 0) return 0;
    const int raster = e->raster > 0 ? e->raster : 8;
    int band_rows = raster * 128;
    while ((e->m + band_rows - 1) / band_rows > HX_MAX_BANDS) band_rows *= 2;
    const size_t one = ca3dmm_oz_desc_bytes();
    x->ndesc = 1;
    x->desc_stride = align_up(one);
    if (!x->desc_h) {
        const size_t p1 = align_up(sizeof(ca3dmm_pack_desc_t) * (size_t) e->kp);
        const size_t p2 = align_up(one * (size_t) e->kp);
        const size_t cap = (p1 > p2 ? p1 : p2) * HX_MAX_BANDS;
        if (cudaMallocHost(&x->desc_h, cap) != cudaSuccess) { x->desc_h = NULL; return 0; }
        if (cudaMalloc(&x->desc_d, cap) != cudaSuccess) { x->desc_d = NULL; return 0; }
    }
    const char *hp = (const char *) pl->stage + pl->off_crtplan;
    for (int r = 0; r < e->m; r += band_rows) {
        const int c = x->nband++;
        const int rend = r + band_rows < e->m ? r + band_rows : e->m;
        x->r0[c] = r;
        x->r1[c] = rend;
        int begin = 0, count = 0, blk = 0;
        if (ca3dmm_crt_group_items(hp, 0, r / 128, (rend + 127) / 128, &begin, &count) ||
            ca3dmm_crt_encode_rows(hp, 1, &blk, 1, r, rend,
                                   (char *) x->desc_h + (size_t) c * x->desc_stride, x->ntile[c])) {
            x->nband = 0;
            return 0;
        }
        ca3dmm_tile_ranges_t *rg = &x->rng[c];
        memset(rg, 0, sizeof(*rg));
        rg->n = 1;
        rg->begin[0] = begin;
        rg->len[0] = count;
    }
    if (cudaMemcpyAsync(x->desc_d, x->desc_h, x->desc_stride * (size_t) x->nband,
                        cudaMemcpyHostToDevice, st) != cudaSuccess) {
        x->nband = 0;
        return 0;
    }
    return x->nband;
}

static int hx_build_bands(ca3dmm_engine_p e, struct host_exec *x, cudaStream_t st)
{
    plan_t *pl = (plan_t *) e->impl;
    const int tmn = pl->tmn, tnn = pl->tnn;
    const int whole = pl->has_dst && pl->dst_srow == 0 && pl->dst_scol == 0 &&
                      pl->dst_nrow == e->m && pl->dst_ncol == e->n;
    const int ozaki = e->gemm_mode == CA3DMM_GEMM_OZAKI;
    x->nband = 0;
    x->built_mode = e->gemm_mode;
    x->built_slices = e->ozaki_slices;
    x->built_raster = e->raster;
    if (e->gemm_mode == CA3DMM_GEMM_CRT) return hx_build_bands_crt(e, x, st);
    if (e->is_BTB || !whole || ((ozaki && pl->oz_fused) ? 1 : e->kp) * tnn > CA3DMM_MAX_RANGES ||
        (!ozaki && pl->ksplit > 1))
        return 0;
    const int raster = e->raster > 0 ? e->raster : 8;
    const int bn = ozaki ? 64 : pl->plain_tile_n;
    /* tile numbering of the GEMM plans: per group (plain) or per unit of
     * (task_m, task_n) with its kp slabs chained (split precision) */
    int *tb = (int *) malloc(sizeof(int) * (size_t) pl->ngroup);
    if (!tb) return 0;
    const int chained = ozaki && pl->oz_fused;
    const int nnum = chained ? tmn * tnn : pl->ngroup;
    for (int g = 0, t = 0; g < nnum; g++) {
        const group_t *gg = &pl->groups[g];
        tb[g] = t;
        if (gg->mz > 0 && gg->nz > 0) t += ((gg->mz + 127) / 128) * ((gg->nz + bn - 1) / bn);
    }
    int band_rows = raster * 128;
    for (;;) {
        int cnt = 0;
        for (int tm = 0; tm < tmn; tm++) cnt += (pl->A[tm].rows + band_rows - 1) / band_rows;
        if (cnt <= HX_MAX_BANDS) break;
        band_rows *= 2;
    }
    const size_t one = ozaki ? ca3dmm_oz_desc_bytes() : sizeof(ca3dmm_pack_desc_t);
    x->ndesc = e->kp;
    x->desc_stride = align_up(one * (size_t) e->kp);
    if (!x->desc_h) {
        /* room for either mode's descriptors */
        const size_t p1 = align_up(sizeof(ca3dmm_pack_desc_t) * (size_t) e->kp);
        const size_t p2 = align_up(ca3dmm_oz_desc_bytes() * (size_t) e->kp);
        const size_t cap = (p1 > p2 ? p1 : p2) * HX_MAX_BANDS;
        if (cudaMallocHost(&x->desc_h, cap) != cudaSuccess) { x->desc_h = NULL; free(tb); return 0; }
        if (cudaMalloc(&x->desc_d, cap) != cudaSuccess) { x->desc_d = NULL; free(tb); return 0; }
    }
    int *blocks = (int *) malloc(sizeof(int) * (size_t) e->kp);
    if (!blocks) { free(tb); return 0; }
    int bad = 0;
    for (int tm = 0; tm < tmn && !bad; tm++) {
        const blk_t *a0 = &pl->A[tm];              /* the same rows in every slab */
        for (int r = 0; r < a0->rows && !bad; r += band_rows) {
            const int c = x->nband++;
            const int rend = r + band_rows < a0->rows ? r + band_rows : a0->rows;
            x->r0[c] = a0->r0 + r;
            x->r1[c] = a0->r0 + rend;
            ca3dmm_tile_ranges_t *rg = &x->rng[c];
            memset(rg, 0, sizeof(*rg));
            const int row_lo = r / 128, nrow_t = band_rows / 128;
            for (int tk = 0; tk < ((chained || (!ozaki && pl->plain_merged)) ? 1 : e->kp); tk++)
                for (int tn = 0; tn < tnn; tn++) {
                    const int g = (tk * tmn + tm) * tnn + tn;
                    const group_t *gg = &pl->groups[g];
                    if (gg->mz <= 0 || gg->nz <= 0) continue;
                    const int tiles_m = (gg->mz + 127) / 128, tiles_n = (gg->nz + bn - 1) / bn;
                    const int row_hi = row_lo + nrow_t < tiles_m ? row_lo + nrow_t : tiles_m;
                    if (row_hi <= row_lo) continue;
                    rg->begin[rg->n] = tb[g] + row_lo * tiles_n;
                    rg->len[rg->n] = (row_hi - row_lo) * tiles_n;
                    rg->n++;
                }
            char *dh = (char *) x->desc_h + (size_t) c * x->desc_stride;
            for (int tk = 0; tk < e->kp; tk++) blocks[tk] = tk * tmn + tm;
            if (ozaki) {
                bad = ca3dmm_oz_encode_rows((char *) pl->stage + pl->off_ozplan, pl->ngroup, blocks,
                                            e->kp, r, rend, dh, x->ntile[c]);
            } else {
                ca3dmm_pack_desc_t *pd = (ca3dmm_pack_desc_t *) dh;
                for (int tk = 0; tk < e->kp; tk++) {
                    const blk_t *b = &pl->A[blocks[tk]];
                    ca3dmm_pack_desc_t *d = &pd[tk];
                    memset(d, 0, sizeof(*d));
                    /* read in place by the GEMM, or a slab the merged plain GEMM skips */
                    if (b->direct || (pl->plain_merged && tk > 0)) continue;
                    a_pack_desc(e, pl, b, r, rend, x->lda, d);
                }
                x->ntile[c][0] = ca3dmm_pack_tiles(pd, e->kp);
            }
        }
    }
    free(blocks);
    free(tb);
    if (bad) { x->nband = 0; return 0; }
    if (cudaMemcpyAsync(x->desc_d, x->desc_h, x->desc_stride * (size_t) x->nband,
                        cudaMemcpyHostToDevice, st) != cudaSuccess) {
        x->nband = 0;
        return 0;
    }
    return x->nband;
}

static int hx_copy_in_B(ca3dmm_engine_p e, struct host_exec *x, const void *B_h, int ldB)
{
    const int b_rows = e->trans_B ? e->n : e->k, b_cols = e->trans_B ? e->k : e->n;
    if (b_rows > 0 && b_cols > 0)
        CA3DMM_CUDA_TRY(cudaMemcpy2DAsync(x->dB, sizeof(double) * (size_t) x->ldb, B_h,
                                          sizeof(double) * (size_t) ldB, sizeof(double) * (size_t) b_rows,
                                          (size_t) b_cols, cudaMemcpyHostToDevice, x->s_in));
    return CA3DMM_OK;
}

/* op(A) rows [r0, r1) into the staging copy of A. */
static int hx_copy_in_A_rows(ca3dmm_engine_p e, struct host_exec *x, const double *A_h, int ldA,
                             int r0, int r1)
{
    if (r1 <= r0 || e->k <= 0) return CA3DMM_OK;
    if (e->trans_A)     /* A is k x m: op(A) rows are columns of A */
        CA3DMM_CUDA_TRY(cudaMemcpy2DAsync(x->dA + (size_t) r0 * x->lda, sizeof(double) * (size_t) x->lda,
                                          A_h + (size_t) r0 * ldA, sizeof(double) * (size_t) ldA,
                                          sizeof(double) * (size_t) e->k, (size_t) (r1 - r0),
                                          cudaMemcpyHostToDevice, x->s_in));
    else
        CA3DMM_CUDA_TRY(cudaMemcpy2DAsync(x->dA + r0, sizeof(double) * (size_t) x->lda, A_h + r0,
                                          sizeof(double) * (size_t) ldA, sizeof(double) * (size_t) (r1 - r0),
                                          (size_t) e->k, cudaMemcpyHostToDevice, x->s_in));
    return CA3DMM_OK;
}

/* B^T B from host memory, pipelined over the kp k-slabs: slab j of B (its
 * rows [k0_j, k0_j + kz_j)) is copied in while slab j - 1 is sliced (split
 * precision) and multiplied into its C slab buffer; the slab sum (and the
 * mirror of the symmetric option) and the copy out of C follow.  Used when
 * kp > 1, the whole C is the destination and every operand block is read in
 * place (plain) -- returns 1 to ask for the serial path otherwise. */
static int hx_btb_slabs(ca3dmm_engine_p e, struct host_exec *x, const void *B_h, int ldB,
                        void *C_h, int ldC, cudaStream_t st)
{
    plan_t *pl = (plan_t *) e->impl;
    const int crt = e->gemm_mode == CA3DMM_GEMM_CRT;
    /* split precision (slices or residues) slices each arriving slab itself */
    const int ozaki = e->gemm_mode == CA3DMM_GEMM_OZAKI || crt;
    const int kp = e->kp, n = e->n, ks = ozaki ? 1 : pl->ksplit;
    const int whole = pl->has_dst && pl->dst_srow == 0 && pl->dst_scol == 0 &&
                      pl->dst_nrow == e->m && pl->dst_ncol == e->n;
    if (!e->is_BTB || kp < 2 || kp > HX_MAX_BANDS || !whole || (!crt && ozaki && pl->oz_fused) ||
        (crt && pl->crt_nsl != kp))
        return 1;
    for (int i = 0; !ozaki && i < pl->nA; i++)
        if (!pl->A[i].direct) return 1;
    for (int i = 0; !ozaki && i < pl->nB; i++)
        if (!pl->B[i].direct) return 1;
    const int gps = pl->ngroup / kp;        /* groups of one slab (consecutive) */
    if (ozaki && !x->slab_built) {
        /* one slicing descriptor per slab: its B block (op(A) reuses its slices) */
        const size_t one = ca3dmm_oz_desc_bytes();
        x->desc_stride = align_up(one);
        if (!x->desc_h) {
            const size_t p1 = align_up(sizeof(ca3dmm_pack_desc_t) * (size_t) kp);
            const size_t p2 = align_up(one * (size_t) kp);
            const size_t cap = (p1 > p2 ? p1 : p2) * HX_MAX_BANDS;
            if (cudaMallocHost(&x->desc_h, cap) != cudaSuccess) { x->desc_h = NULL; return 1; }
            if (cudaMalloc(&x->desc_d, cap) != cudaSuccess) { x->desc_d = NULL; return 1; }
        }
        for (int j = 0; j < kp; j++) {
            char *dj = (char *) x->desc_h + (size_t) j * x->desc_stride;
            const int idx = crt ? pl->crt_nsl + j : pl->nA + j;
            if (crt ? ca3dmm_crt_encode_blocks((char *) pl->stage + pl->off_crtplan, pl->crt_nsl,
                                               &idx, 1, dj, x->ntile[j])
                    : ca3dmm_oz_encode_blocks((char *) pl->stage + pl->off_ozplan, pl->ngroup,
                                              &idx, 1, dj, x->ntile[j]))
                return 1;
        }
        CA3DMM_CUDA_TRY(cudaMemcpyAsync(x->desc_d, x->desc_h, x->desc_stride * (size_t) kp,
                                        cudaMemcpyHostToDevice, st));
        x->slab_built = 1;
    }
    char *w = (char *) e->workbuf_d;
    int *status_d = (int *) (w + pl->off_status);
    CA3DMM_CUDA_TRY(cudaMemsetAsync(status_d, 0, 64, st));
    /* copies in: B slab by slab */
    for (int j = 0; j < kp; j++) {
        int k0, kz;
        calc_block_spos_size(e->k, kp, j, &k0, &kz);
        if (kz > 0 && n > 0)
            CA3DMM_CUDA_TRY(cudaMemcpy2DAsync(x->dB + k0, sizeof(double) * (size_t) x->ldb,
                                              (const double *) B_h + k0, sizeof(double) * (size_t) ldB,
                                              sizeof(double) * (size_t) kz, (size_t) n,
                                              cudaMemcpyHostToDevice, x->s_in));
        CA3DMM_CUDA_TRY(cudaEventRecord(x->ev_a[j], x->s_in));
    }
    int rc = crt ? ca3dmm_crt_clear(&pl->crt, st) : ozaki ? ca3dmm_oz_clear(&pl->oz, st) : CA3DMM_OK;
    if (rc) return rc;
    int tile0 = 0;
    for (int j = 0; j < kp; j++) {
        /* the tiles of slab j's groups (and k sub-slabs): consecutive in both GEMM plans */
        int count = 0;
        for (int g = j * gps; g < (j + 1) * gps; g++) {
            const group_t *gg = &pl->groups[g];
            if (gg->mz <= 0 || gg->nz <= 0) continue;
            const int bn = ozaki ? 64 : pl->plain_tile_n;
            count += ks * ((gg->mz + 127) / 128) * ((gg->nz + bn - 1) / bn);
        }
        ca3dmm_tile_ranges_t rg;
        memset(&rg, 0, sizeof(rg));
        rg.n = 1;
        rg.begin[0] = tile0;
        rg.len[0] = count;
        tile0 += count;
        CA3DMM_CUDA_TRY(cudaStreamWaitEvent(st, x->ev_a[j], 0));
        if (crt) {
            const void *dd = (const char *) x->desc_d + (size_t) j * x->desc_stride;
            int ib = 0, ic = 0;
            rc = ca3dmm_crt_group_items((char *) pl->stage + pl->off_crtplan, j, 0, INT32_MAX, &ib,
                                        &ic);
            rg.begin[0] = ib;
            rg.len[0] = ic;
            if (!rc) rc = ca3dmm_crt_pack_descs(&pl->crt, x->dB, dd, 1, x->ntile[j], st);
            if (!rc) rc = ca3dmm_crt_run_gemm(&pl->crt, &rg, status_d, 5.0, st);
            if (!rc) rc = ca3dmm_crt_run_reconstruct(&pl->crt, j, j + 1, 0, INT32_MAX, st);
            if (!rc) rc = ca3dmm_crt_run_nonfinite(&pl->crt, j, j + 1, 0, INT32_MAX, x->dB, x->dB, st);
        } else if (ozaki) {
            const void *dd = (const char *) x->desc_d + (size_t) j * x->desc_stride;
            rc = ca3dmm_oz_slice_descs(&pl->oz, x->dB, dd, 1, x->ntile[j], st);
            if (!rc) rc = ca3dmm_oz_run_gemm_ranges(&pl->oz, &rg, status_d, 5.0, st);
            if (!rc) rc = ca3dmm_oz_run_nonfinite(&pl->oz, &rg, x->dB, x->dB, st);
        } else {
            rc = ca3dmm_dgemm_launch_ranges_tn(w + pl->off_gemm, pl->ngroup * pl->ksplit, &rg,
                                               pl->a_kmajor, status_d, 5.0, st, pl->plain_tile_n);
        }
        if (rc) return rc;
    }
    const int nred = kp * ks;
    rc = ca3dmm_reduce_slabs_launch((const double *) (w + pl->off_slab), (long long) pl->slab_stride,
                                    pl->slab_ld, nred, e->m, e->n, x->dC, x->ldc, st);
    if (!rc && pl->sym) rc = ca3dmm_mirror_upper_launch(x->dC, x->ldc, e->m, st);
    if (rc) return rc;
    CA3DMM_CUDA_TRY(cudaMemcpy2DAsync(C_h, sizeof(double) * (size_t) ldC, x->dC,
                                      sizeof(double) * (size_t) x->ldc, sizeof(double) * (size_t) e->m,
                                      (size_t) e->n, cudaMemcpyDeviceToHost, st));
    rc = launch_guard_check(e, pl, status_d, st);
    if (rc) return rc;
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(pl->status_h, status_d, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                                    st));
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
    return device_status_error(pl);
}

static int exec_host(ca3dmm_engine_p e, const void *A_h, int ldA, const void *B_h, int ldB,
                     void *C_h, int ldC)
{
    plan_t *pl = (plan_t *) e->impl;
    const int a_rows = e->trans_A ? e->k : e->m, b_rows = e->trans_B ? e->n : e->k;
    if (!B_h || ldB < b_rows || (!e->is_BTB && (!A_h || ldA < a_rows))) {
        ERROR_PRINTF("Invalid host operands: ldA = %d (>= %d), ldB = %d (>= %d)\n", ldA, a_rows, ldB,
                     b_rows);
        return CA3DMM_EINVAL;
    }
    if (!pl->has_dst || C_h == NULL || ldC < pl->dst_nrow) {
        ERROR_PRINTF("exec_host needs a dst_C block and a host C with ldC >= %d\n", pl->dst_nrow);
        return CA3DMM_EINVAL;
    }
    struct host_exec *x;
    int rc = hx_create(e, &x);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t) e->stream;
    const double *dAsrc = e->is_BTB ? x->dB : x->dA;
    const long long ldAsrc = e->is_BTB ? x->ldb : x->lda;
    if (e->gemm_auto == 1) {
        /* CA3DMM_GEMM_AUTO: tune on device copies of the whole operands */
        const int a_cols = e->trans_A ? e->m : e->k, b_cols = e->trans_B ? e->k : e->n;
        if (!e->is_BTB)
            CA3DMM_CUDA_TRY(cudaMemcpy2DAsync(x->dA, sizeof(double) * x->lda, A_h,
                                              sizeof(double) * (size_t) ldA,
                                              sizeof(double) * (size_t) a_rows, a_cols,
                                              cudaMemcpyHostToDevice, st));
        CA3DMM_CUDA_TRY(cudaMemcpy2DAsync(x->dB, sizeof(double) * x->ldb, B_h,
                                          sizeof(double) * (size_t) ldB,
                                          sizeof(double) * (size_t) b_rows, b_cols,
                                          cudaMemcpyHostToDevice, st));
        CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
        rc = ca3dmm_engine_autotune_env(e, dAsrc, (int) ldAsrc, x->dB, (int) x->ldb, x->dC,
                                        (int) x->ldc);
        if (rc) return rc;
        pl->plan_valid = 0;   /* the row-band pipeline needs its own plan */
    }
    /* device plan for the staging buffers (rebuilt only when they change) */
    if (!pl->plan_valid || pl->c_A != dAsrc || pl->c_B != x->dB || pl->c_ldA != ldAsrc ||
        pl->c_ldB != x->ldb || pl->c_dst != x->dC || pl->c_ldC != x->ldc) {
        pl->upload_for_host = 1;
        rc = plan_upload(e, dAsrc, (int) ldAsrc, x->dB, (int) x->ldb, x->dC, (int) x->ldc, st);
        pl->upload_for_host = 0;
        if (rc) return rc;
        x->built_mode = -1;
        x->slab_built = 0;
    }
    if (x->built_mode != e->gemm_mode || x->built_slices != e->ozaki_slices ||
        x->built_raster != e->raster)
        hx_build_bands(e, x, st);
    /* the inputs may not be overwritten before the previous exec's reads are done */
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (e->is_BTB) {
        const int r = hx_btb_slabs(e, x, B_h, ldB, C_h, ldC, st);
        if (r != 1) return r;
    }
    const int dn = pl->dst_nrow, dc = pl->dst_ncol;
    if (x->nband < 2) {
        /* serial: copy in, the device exec, copy out */
        rc = hx_copy_in_B(e, x, B_h, ldB);
        if (!rc && !e->is_BTB) rc = hx_copy_in_A_rows(e, x, (const double *) A_h, ldA, 0, e->m);
        if (rc) return rc;
        CA3DMM_CUDA_TRY(cudaEventRecord(x->ev_b, x->s_in));
        CA3DMM_CUDA_TRY(cudaStreamWaitEvent(st, x->ev_b, 0));
        const int sync = e->sync_exec;
        e->sync_exec = 1;
        rc = exec_device(e, dAsrc, (int) ldAsrc, x->dB, (int) x->ldb, x->dC, (int) x->ldc, st);
        e->sync_exec = sync;
        if (rc) return rc;
        if (dn > 0 && dc > 0)
            CA3DMM_CUDA_TRY(cudaMemcpy2DAsync(C_h, sizeof(double) * (size_t) ldC, x->dC,
                                              sizeof(double) * (size_t) x->ldc, sizeof(double) * (size_t) dn,
                                              (size_t) dc, cudaMemcpyDeviceToHost, st));
        CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
        return CA3DMM_OK;
    }
    char *w = (char *) e->workbuf_d;
    int *status_d = (int *) (w + pl->off_status);
    CA3DMM_CUDA_TRY(cudaMemsetAsync(status_d, 0, 64, st));
    /* copies in: all of B, then the op(A) rows band by band */
    rc = hx_copy_in_B(e, x, B_h, ldB);
    if (rc) return rc;
    CA3DMM_CUDA_TRY(cudaEventRecord(x->ev_b, x->s_in));
    for (int c = 0; c < x->nband; c++) {
        rc = hx_copy_in_A_rows(e, x, (const double *) A_h, ldA, x->r0[c], x->r1[c]);
        if (rc) return rc;
        CA3DMM_CUDA_TRY(cudaEventRecord(x->ev_a[c], x->s_in));
    }
    const int ozaki = e->gemm_mode == CA3DMM_GEMM_OZAKI;
    const int crt = e->gemm_mode == CA3DMM_GEMM_CRT;
    CA3DMM_CUDA_TRY(cudaStreamWaitEvent(st, x->ev_b, 0));
    if (crt) {
        rc = ca3dmm_crt_clear(&pl->crt, st);
        if (!rc) rc = ca3dmm_crt_pack_side(&pl->crt, 1, x->dB, st);
    } else if (ozaki) {
        rc = ca3dmm_oz_clear(&pl->oz, st);
        if (!rc) rc = ca3dmm_oz_slice_side(&pl->oz, 1, x->dB, st);
    } else {
        rc = launch_pack_side(e, 1, x->dB, st);
    }
    if (rc) return rc;
    for (int c = 0; c < x->nband; c++) {
        const void *dd = (const char *) x->desc_d + (size_t) c * x->desc_stride;
        CA3DMM_CUDA_TRY(cudaStreamWaitEvent(st, x->ev_a[c], 0));
        if (crt) {
            rc = ca3dmm_crt_pack_descs(&pl->crt, x->dA, dd, 1, x->ntile[c], st);
            if (!rc) rc = ca3dmm_crt_run_gemm(&pl->crt, &x->rng[c], status_d, 5.0, st);
            if (!rc) rc = ca3dmm_crt_run_reconstruct(&pl->crt, 0, 1, x->r0[c], x->r1[c], st);
            if (!rc) rc = ca3dmm_crt_run_nonfinite(&pl->crt, 0, 1, x->r0[c], x->r1[c], x->dA, x->dB, st);
        } else if (ozaki) {
            rc = ca3dmm_oz_slice_descs(&pl->oz, x->dA, dd, x->ndesc, x->ntile[c], st);
            if (!rc) rc = ca3dmm_oz_run_gemm_ranges(&pl->oz, &x->rng[c], status_d, 5.0, st);
            if (!rc) rc = ca3dmm_oz_run_nonfinite(&pl->oz, &x->rng[c], x->dA, x->dB, st);
        } else {
            rc = ca3dmm_pack_launch(x->dA, (double *) w, (const ca3dmm_pack_desc_t *) dd, x->ndesc,
                                    x->ntile[c][0], st);
            if (!rc)
                rc = ca3dmm_dgemm_launch_ranges_tn(w + pl->off_gemm, pl->ngroup, &x->rng[c],
                                                   pl->a_kmajor, status_d, 5.0, st,
                                                   pl->plain_tile_n);
        }
        if (!rc && !crt && e->kp > 1 && !(ozaki && pl->oz_fused) && !(!ozaki && pl->plain_merged))
            rc = ca3dmm_reduce_slabs_launch((const double *) (w + pl->off_slab) + x->r0[c],
                                            (long long) pl->slab_stride, pl->slab_ld, e->kp,
                                            x->r1[c] - x->r0[c], e->n, x->dC + x->r0[c], x->ldc, st);
        if (rc) return rc;
        CA3DMM_CUDA_TRY(cudaEventRecord(x->ev_c[c], st));
        CA3DMM_CUDA_TRY(cudaStreamWaitEvent(x->s_out, x->ev_c[c], 0));
        CA3DMM_CUDA_TRY(cudaMemcpy2DAsync((double *) C_h + x->r0[c], sizeof(double) * (size_t) ldC,
                                          x->dC + x->r0[c], sizeof(double) * (size_t) x->ldc,
                                          sizeof(double) * (size_t) (x->r1[c] - x->r0[c]), (size_t) e->n,
                                          cudaMemcpyDeviceToHost, x->s_out));
    }
    rc = launch_guard_check(e, pl, status_d, st);
    if (rc) return rc;
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(pl->status_h, status_d, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                                    st));
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(x->s_out));
    return device_status_error(pl);
}

int ca3dmm_engine_exec_host(ca3dmm_engine_p e, const void *A_h, int ldA, const void *B_h, int ldB,
                            void *C_h, int ldC)
{
    if (e == NULL) {
        ERROR_PRINTF("ca3dmm_engine not initialized\n");
        return CA3DMM_EINVAL;
    }
    if (e->workbuf_d == NULL || ((plan_t *) e->impl)->stage == NULL) {
        ERROR_PRINTF("ca3dmm_engine has no device work buffer attached\n");
        e->last_error = CA3DMM_EINVAL;
        return CA3DMM_EINVAL;
    }
    double t0 = ca3dmm_wtime_sec();
    nvtxRangePushA("ca3dmm_engine_exec_host");
    int rc = exec_host(e, A_h, ldA, B_h, ldB, C_h, ldC);
    nvtxRangePop();
    e->last_error = rc;
    if (rc) {
        ERROR_PRINTF("ca3dmm_engine_exec_host failed (error %d)\n", rc);
        return rc;
    }
    double ms = 1000.0 * (ca3dmm_wtime_sec() - t0);
    e->exec_ms += ms;
    e->n_exec++;
    if (e->print_timing) INFO_PRINTF("CA3DMM exec (host buffers) time = %.2f ms\n\n", ms);
    return CA3DMM_OK;
}

void ca3dmm_engine_reset_stat(ca3dmm_engine_p e)
{
    if (e == NULL) return;
    cannon_engine_reset_stat(e->cannon_engine);
    e->redist_ms = 0.0;
    e->agvAB_ms = 0.0;
    e->cannon_ms = 0.0;
    e->reduce_ms = 0.0;
    e->hd_trans_ms = 0.0;
    e->exec_ms = 0.0;
    e->n_exec = 0;
}

void ca3dmm_engine_print_stat(ca3dmm_engine_p e)
{
    if (e == NULL) return;
    if (e->n_exec == 0) {
        WARNING_PRINTF("No ca3dmm_engine statistic data to print\n");
        return;
    }
    printf("================== CA3DMM algorithm engine =================\n");
    printf("* Initialization         : %.2f ms\n", e->init_ms);
    printf("* Number of executions   : %d\n", e->n_exec);
    printf("* Execution time (avg)   : %.2f ms\n", e->exec_ms / e->n_exec);
    printf("  * Redistribute A, B, C : %.2f ms\n", e->redist_ms / e->n_exec);
    printf("  * Allgather A or B     : %.2f ms\n", e->agvAB_ms / e->n_exec);
    printf("  * 2D Cannon execution  : %.2f ms\n", e->cannon_ms / e->n_exec);
    printf("  * Reduce-scatter C     : %.2f ms\n", e->reduce_ms / e->n_exec);
    double gf = 2.0 * (double) e->m * (double) e->n * (double) e->k / (e->cannon_ms / e->n_exec) /
                1e6;
    printf("* GEMM throughput        : %.2f GFlops (%s)\n", gf,
           e->gemm_mode == CA3DMM_GEMM_OZAKI ? "split precision"
           : e->gemm_mode == CA3DMM_GEMM_CRT ? "split precision, modular" : "FP64 DMMA");
    if (e->gemm_auto == 2) {
        ca3dmm_tune_cfg_t c;
        ca3dmm_engine_get_tune(e, &c);
        printf("* Tuned (auto mode)      : mode %d, %d slices / moduli, raster %d, tile %d "
               "(%.0f ms to tune)\n", c.gemm_mode, c.slices, c.raster, c.tile_n, e->tune_ms);
    }
    printf("============================================================\n");
}

int ca3dmm_engine_last_error(ca3dmm_engine_p e) { return e ? e->last_error : CA3DMM_EINVAL; }

void ca3dmm_engine_set_stream(ca3dmm_engine_p e, void *stream, int sync)
{
    if (!e) return;
    e->stream = stream;
    e->sync_exec = sync ? 1 : 0;
}

/* Make the work buffer at least `need` bytes: the engine's own buffer is
 * replaced, a caller's buffer that is too small is an error. */
static int grow_workbuf(ca3dmm_engine_p e, plan_t *pl, size_t need, size_t have)
{
    if (e->workbuf_d == NULL || need <= have) return CA3DMM_OK;
    if (!e->alloc_workbuf) return CA3DMM_ENOMEM;
    void *nw = dev_type_malloc(need, DEV_TYPE_CUDA);
    if (!nw) return CA3DMM_ENOMEM;
    dev_type_free(e->workbuf_d, DEV_TYPE_CUDA);
    pl->total = need;
    ca3dmm_engine_attach_workbuf(e, NULL, nw);
    return CA3DMM_OK;
}

int ca3dmm_engine_set_gemm_mode(ca3dmm_engine_p e, int mode, int slices)
{
    if (!e) return CA3DMM_EINVAL;
    plan_t *pl = (plan_t *) e->impl;
    if (mode == CA3DMM_GEMM_AUTO) {
        const size_t old_total = pl->total, need = auto_bytes(e);
        if (pl->total < need) pl->total = need;
        int rc = grow_workbuf(e, pl, pl->total, old_total);
        if (rc) {
            pl->total = old_total;
            return rc;
        }
        e->workbuf_bytes = pl->total;
        e->gemm_auto = 1;
        return CA3DMM_OK;
    }
    if (mode != CA3DMM_GEMM_PLAIN && mode != CA3DMM_GEMM_OZAKI && mode != CA3DMM_GEMM_CRT)
        return CA3DMM_EINVAL;
    if (mode == CA3DMM_GEMM_OZAKI && (slices < 2 || slices > 8)) return CA3DMM_EINVAL;
    int nmod = 0;
    if (mode == CA3DMM_GEMM_CRT && (nmod = crt_resolve(e, slices)) == 0) return CA3DMM_EINVAL;
    int old_mode = e->gemm_mode, old_sl = e->ozaki_slices, old_nm = e->crt_moduli;
    e->gemm_mode = mode;
    if (mode == CA3DMM_GEMM_OZAKI) e->ozaki_slices = slices;
    if (mode == CA3DMM_GEMM_CRT) e->crt_moduli = nmod;
    size_t old_total = pl->total;
    plan_layout(e, pl);
    int rc = grow_workbuf(e, pl, pl->total, old_total);
    if (rc) {
        /* the caller's buffer is too small, or no memory: keep the old mode */
        e->gemm_mode = old_mode;
        e->ozaki_slices = old_sl;
        e->crt_moduli = old_nm;
        plan_layout(e, pl);
        if (pl->total < old_total) pl->total = old_total;
        return rc;
    }
    if (pl->total < old_total) pl->total = old_total;   /* keep the larger layout's size */
    e->workbuf_bytes = pl->total;
    e->gemm_auto = 0;
    pl->plan_valid = 0;
    return CA3DMM_OK;
}

int ca3dmm_engine_set_tune(ca3dmm_engine_p e, const ca3dmm_tune_cfg_t *c)
{
    if (!e || !c) return CA3DMM_EINVAL;
    plan_t *pl = (plan_t *) e->impl;
    if (c->gemm_mode == CA3DMM_GEMM_CRT) {
        if ((c->tile_n != 0 && c->tile_n != 128 && c->tile_n != 256) || c->raster < 0 ||
            c->raster > 1024)
            return CA3DMM_EINVAL;
    } else if (c->raster != 0 && c->raster != 4 && c->raster != 8 && c->raster != 16) {
        return CA3DMM_EINVAL;
    } else if (c->gemm_mode == CA3DMM_GEMM_PLAIN) {
        /* 128- or 64-column DMMA tiles; the symmetric B^T B plan takes 128 */
        if ((c->tile_n != 0 && c->tile_n != 64 && c->tile_n != 128) || (c->tile_n == 64 && pl->sym))
            return CA3DMM_EINVAL;
    } else if (c->tile_n != 0) {
        return CA3DMM_EINVAL;
    }
    int rc = ca3dmm_engine_set_gemm_mode(e, c->gemm_mode, c->slices);
    if (rc) return rc;
    if (c->gemm_mode == CA3DMM_GEMM_CRT) {
        pl->crt_band = c->raster ? c->raster : pl->crt_band_env;
        pl->crt_tile_n = c->tile_n ? c->tile_n : 256;
    } else {
        e->raster = c->raster ? c->raster : 8;
        if (c->gemm_mode == CA3DMM_GEMM_PLAIN)
            pl->plain_tile_n = c->tile_n ? c->tile_n : pl->plain_tile_n_env;
    }
    pl->plan_valid = 0;
    return CA3DMM_OK;
}

int ca3dmm_engine_get_tune(ca3dmm_engine_p e, ca3dmm_tune_cfg_t *c)
{
    if (!e || !c) return CA3DMM_EINVAL;
    const plan_t *pl = (const plan_t *) e->impl;
    c->gemm_mode = e->gemm_mode;
    c->slices = e->gemm_mode == CA3DMM_GEMM_OZAKI ? e->ozaki_slices
                : e->gemm_mode == CA3DMM_GEMM_CRT ? e->crt_moduli : 0;
    c->kp = e->kp;
    c->raster = e->gemm_mode == CA3DMM_GEMM_CRT ? pl->crt_band : e->raster;
    c->tile_n = e->gemm_mode == CA3DMM_GEMM_CRT ? pl->crt_tile_n
                : (e->gemm_mode == CA3DMM_GEMM_PLAIN && pl->plain_tile_n != 128) ? pl->plain_tile_n
                : 0;
    return CA3DMM_OK;
}

ca3dmm_tune_report_t *ca3dmm_engine_report_slot(ca3dmm_engine_p e)
{
    return e && e->impl ? &((plan_t *) e->impl)->report : NULL;
}

int ca3dmm_engine_tune_report(ca3dmm_engine_p e, ca3dmm_tune_cfg_t *cfgs, float *ms, float *err,
                              int max)
{
    const ca3dmm_tune_report_t *r = ca3dmm_engine_report_slot(e);
    if (!r) return -1;
    for (int i = 0; i < r->n && i < max; i++) {
        if (cfgs) cfgs[i] = r->cfg[i];
        if (ms) ms[i] = r->ms[i];
        if (err) err[i] = r->err[i];
    }
    return r->n;
}

static int exec_device(ca3dmm_engine_p e, const void *src_A, int ldA, const void *src_B, int ldB,
                       void *dst_C, int ldC, cudaStream_t st);

int ca3dmm_engine_exec_reps(ca3dmm_engine_p e, const void *A, int ldA, const void *B, int ldB,
                            void *C, int ldC, int reps, float *ms)
{
    const int sync = e->sync_exec;
    e->sync_exec = 1;
    const double t0 = e->redist_ms + e->cannon_ms + e->reduce_ms;
    int rc = CA3DMM_OK;
    for (int r = 0; r < reps && !rc; r++)
        rc = exec_device(e, A, ldA, B, ldB, C, ldC, (cudaStream_t) e->stream);
    e->sync_exec = sync;
    if (!rc && ms && reps > 0)
        *ms = (float) ((e->redist_ms + e->cannon_ms + e->reduce_ms - t0) / reps);
    return rc;
}

int ca3dmm_engine_full_c(ca3dmm_engine_p e, void *dst_C, int ldC, const double **C,
                         long long *ld)
{
    const plan_t *pl = (const plan_t *) e->impl;
    const int whole = pl->has_dst && pl->dst_srow == 0 && pl->dst_scol == 0 &&
                      pl->dst_nrow == e->m && pl->dst_ncol == e->n;
    *C = whole ? (const double *) dst_C : (const double *) ((char *) e->workbuf_d + pl->off_cout);
    *ld = whole ? ldC : e->m;
    return CA3DMM_OK;
}

size_t ca3dmm_engine_workbuf_bytes(ca3dmm_engine_p e) { return e ? e->workbuf_bytes : 0; }

int ca3dmm_engine_set_raster(ca3dmm_engine_p e, int raster)
{
    if (!e || (raster != 4 && raster != 8 && raster != 16)) return CA3DMM_EINVAL;
    e->raster = raster;
    ((plan_t *) e->impl)->plan_valid = 0;
    return CA3DMM_OK;
}

int ca3dmm_engine_vrank_info(ca3dmm_engine_p e, int vrank, int *out34)
{
    if (!e || !out34 || vrank < 0 || vrank >= e->n_proc) return CA3DMM_EINVAL;
    vrank_geometry(e->m, e->n, e->k, e->mp, e->np, e->kp, vrank, e->is_BTB, out34);
    return CA3DMM_OK;
}

int ca3dmm_engine_guard_bands(ca3dmm_engine_p e, long long *offsets, int max)
{
    if (!e || !e->impl) return -1;
    const plan_t *pl = (const plan_t *) e->impl;
    for (int i = 0; i < pl->ncanary && i < max && offsets; i++) offsets[i] = pl->canary[i];
    return pl->ncanary;
}
