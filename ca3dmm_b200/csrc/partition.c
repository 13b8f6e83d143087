/* 3D process-grid planner and balanced split.
 *
 * The grid decision is part of the drop-in contract (it fixes every virtual
 * rank's cuboid), so this follows the reference's search step for step and
 * with the same floating-point expressions: src/partition.c:9-231 (sort the
 * three dimensions, one / two / three "large dimension" regimes, the
 * fixed-ratio neighbourhood search with the 1.25 volume and 4.0 aspect
 * filters, and the n x n x k variant).  Parity with the reference's own
 * compiled partition.c is tested over thousands of (p, m, n, k). */
#include <math.h>
#include "ca3dmm_util.h"
#include "partition.h"
#include <sys/time.h>

double ca3dmm_wtime_sec(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + (double) tv.tv_usec / 1000000.0;
}

/* src/utils.c:26-48 */
void calc_block_spos_size(const int len, const int nblk, const int iblk, int *blk_spos,
                          int *blk_size)
{
    if (iblk < 0 || iblk > nblk) {
        *blk_spos = -1;
        *blk_size = 0;
        return;
    }
    int small = len / nblk, nbig = len % nblk;
    if (iblk < nbig) {
        *blk_spos = (small + 1) * iblk;
        *blk_size = small + 1;
    } else {
        *blk_spos = small * iblk + nbig;
        *blk_size = small;
    }
}

static double spread3(const double *v)
{
    double hi = v[0], lo = v[0];
    for (int i = 1; i < 3; i++) {
        if (v[i] > hi) hi = v[i];
        if (v[i] < lo) lo = v[i];
    }
    return hi / lo;
}

/* Search (src/partition.c:21-94) around the ideal real-valued grid with the
 * pair (i0, i1) tied by an integer ratio so that max/min divides. */
static void search_tied_pair(int p, int i0, int i1, const double *dims, const double *ideal,
                             int *grid)
{
    const int i2 = 3 - i0 - i1;
    const double ratio = ideal[i1] / ideal[i0];
    const double pd = p;
    double ideal_vol = 1.0;
    for (int d = 0; d < 3; d++) ideal_vol *= dims[d] / ideal[d];

    grid[i0] = (int) floor(ideal[i0]);
    grid[i1] = (int) floor(ratio) * grid[i0];
    grid[i2] = (int) (floor(pd / (double) (grid[i0] * grid[i1])));
    double blk[3], best_vol = 1.0;
    for (int d = 0; d < 3; d++) {
        blk[d] = dims[d] / (double) grid[d];
        best_vol *= blk[d];
    }
    double best_surf = (blk[0] * blk[1] + blk[0] * blk[2] + blk[1] * blk[2]) * (double) grid[0] *
                       (double) grid[1] * (double) grid[2];

    const int a_lo = (int) ceil(ideal[i0] * 0.3), a_hi = (int) floor(ideal[i0] * 3.3);
    const int r_lo = (int) ceil(ratio * 0.3), r_hi = (int) floor(ratio * 3.3);
    for (int a = a_lo; a <= a_hi; a++) {
        for (int r = r_lo; r <= r_hi; r++) {
            int cand[3];
            cand[i0] = a;
            cand[i1] = r * a;
            cand[i2] = (int) floor(pd / (double) (cand[i0] * cand[i1]));
            double cb[3], vol = 1.0, nproc = 1.0;
            for (int d = 0; d < 3; d++) {
                cb[d] = dims[d] / (double) cand[d];
                vol *= cb[d];
                nproc *= (double) cand[d];
            }
            double surf = nproc * (cb[0] * cb[1] + cb[0] * cb[2] + cb[1] * cb[2]);
            if (cand[0] < 1 || cand[1] < 1 || cand[2] < 1) continue;
            if (vol / ideal_vol > 1.25) continue;
            if (spread3(cb) >= 4.0) continue;
            if (vol < best_vol) {
                best_vol = vol;
                best_surf = surf;
                grid[0] = cand[0]; grid[1] = cand[1]; grid[2] = cand[2];
            }
            if ((vol < best_vol * 1.05) && (surf < best_surf)) {
                best_vol = vol;
                best_surf = surf;
                grid[0] = cand[0]; grid[1] = cand[1]; grid[2] = cand[2];
            }
        }
    }
}

void calc_3d_decomposition_cannon(const int p, const int m, const int n, const int k, int *mp,
                                  int *np, int *kp, int *rp)
{
    /* order[] lists which of (m, n, k) = (0, 1, 2) is smallest .. largest;
     * later matching branches win on ties, as in src/partition.c:104-133. */
    int order[3] = {0, 1, 2};
    if (m <= n && n <= k) { order[0] = 0; order[1] = 1; order[2] = 2; }
    if (m <= k && k <= n) { order[0] = 0; order[1] = 2; order[2] = 1; }
    if (n <= m && m <= k) { order[0] = 1; order[1] = 0; order[2] = 2; }
    if (n <= k && k <= m) { order[0] = 1; order[1] = 2; order[2] = 0; }
    if (k <= m && m <= n) { order[0] = 2; order[1] = 0; order[2] = 1; }
    if (k <= n && n <= m) { order[0] = 2; order[1] = 1; order[2] = 0; }
    const int mnk[3] = {m, n, k};
    double dims[3];
    for (int d = 0; d < 3; d++) dims[d] = mnk[order[d]];
    /* position of m, n, k inside the sorted order */
    int pos[3];
    for (int d = 0; d < 3; d++) pos[order[d]] = d;

    int grid[3] = {1, 1, 1};
    const double pd = p, d0 = dims[0], d1 = dims[1], d2 = dims[2];
    const double r21 = d2 / d1;
    if (r21 > pd) grid[2] = p;                               /* one large dimension */

    const double two_large = d1 * d2 / (d0 * d0);
    if ((r21 <= pd) && (pd <= two_large)) {                 /* two large dimensions */
        double best = 1.0;
        int lo = (int) ceil(r21 * 0.5), hi = (int) floor(r21 * 2);
        for (int r = lo; r <= hi; r++) {
            int g1 = (int) floor(sqrt(pd / (double) r));
            int g2 = ((double) k == d0) ? (g1 * r) : (int) floor(pd / (double) g1);
            double prod = (double) g1 * g2;
            if (prod > best) {
                best = prod;
                grid[1] = g1;
                grid[2] = g2;
            }
        }
    }
    if (pd > two_large) {                                   /* three large dimensions */
        double r20 = d2 / d0, r10 = d1 / d0;
        double g0 = cbrt(pd / (r20 * r10));
        double ideal[3] = {g0, g0 * r10, g0 * r20};
        /* tie the two dimensions that become the Cannon plane (m and n) */
        int k_pos = pos[2];
        if (k_pos == 0) search_tied_pair(p, 1, 2, dims, ideal, grid);
        if (k_pos == 1) search_tied_pair(p, 0, 2, dims, ideal, grid);
        if (k_pos == 2) search_tied_pair(p, 0, 1, dims, ideal, grid);
    }
    *mp = grid[pos[0]];
    *np = grid[pos[1]];
    *kp = grid[pos[2]];
    *rp = p - (*mp) * (*np) * (*kp);
    if (*rp * 10 > p)
        WARNING_PRINTF("Failed to find a good solution, current: %d * %d * %d + %d\n", *mp, *np,
                       *kp, *rp);
}

void calc_3d_decomposition_nk(const int p, const int n, const int k, int *np, int *kp, int *rp)
{
    const double ratio = (double) k / (double) n;
    int side = (int) ceil(cbrt((double) p / ratio));
    int depth = p / (side * side);
    *np = side;
    *kp = depth;
    *rp = p - side * side * depth;
    while (side > 1) {
        side--;
        depth = p / (side * side);
        int idle = p - side * side * depth;
        if ((double) depth / (double) side >= 4.0 * ratio) break;
        if (idle < *rp) {
            *np = side;
            *kp = depth;
            *rp = idle;
        }
    }
    if (*rp * 10 > p)
        WARNING_PRINTF("Failed to find a good solution, current: %d * %d * %d + %d\n", *np, *np,
                       *kp, *rp);
}
