// Split-precision (Ozaki INT8) GEMM -- placeholder until the tcgen05 kernel lands.
#include <cuda_runtime.h>
#include "ca3dmm_kernels.h"
#include "ca3dmm_ozaki.h"

extern "C" size_t ca3dmm_oz_plan_bytes(int ngroup) { return 256 + (size_t) ngroup * 512; }
extern "C" size_t ca3dmm_oz_work_bytes(int, const int *, const int *, int, const int *,
                                       const int *, int) { return 256; }
extern "C" int ca3dmm_oz_plan_encode(ca3dmm_oz_plan_t *, int, int, const ca3dmm_oz_blk_t *, int,
                                     const ca3dmm_oz_blk_t *, int, const ca3dmm_oz_group_t *,
                                     void *, size_t, void *, void *) { return CA3DMM_EINVAL; }
extern "C" int ca3dmm_oz_run_pack(const ca3dmm_oz_plan_t *, const void *, int, int, const void *,
                                  int, int, cudaStream_t) { return CA3DMM_EINVAL; }
extern "C" int ca3dmm_oz_run_gemm(const ca3dmm_oz_plan_t *, int *, double, cudaStream_t)
{ return CA3DMM_EINVAL; }
