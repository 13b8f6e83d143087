/* 3D process-grid planner.  Same names, arguments and results as
 * src/partition.h:16-31 (algorithm of src/partition.c:9-231). */
#ifndef CA3DMM_PARTITION_H
#define CA3DMM_PARTITION_H

#ifdef __cplusplus
extern "C" {
#endif

/* src/partition.h:16-19: near-optimal mp x np x kp (+ rp idle) for an
 * m x n x k cuboid on p ranks with max(mp,np) % min(mp,np) == 0. */
void calc_3d_decomposition_cannon(const int p, const int m, const int n, const int k, int *mp,
                                  int *np, int *kp, int *rp);

/* src/partition.h:27-30: np x np x kp (+ rp idle) for an n x n x k cuboid. */
void calc_3d_decomposition_nk(const int p, const int n, const int k, int *np, int *kp, int *rp);

/* src/utils.h:130-133 (src/utils.c:26-48): balanced 1D split. */
void calc_block_spos_size(const int len, const int nblk, const int iblk, int *blk_spos,
                          int *blk_size);

#ifdef __cplusplus
}
#endif
#endif
