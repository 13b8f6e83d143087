// Redistribution kernels of the virtual process grid, HBM-bound:
//   * batched block pack (copy or transpose) of column-major matrices --
//     the on-device form of mat_redist's pack -> alltoallv -> unpack
//     (src/mat_redist.c:327-348, :395-416) fused with the operand transpose
//     the reference does with cublasDgeam (src/ca3dmm.c:1036-1058);
//   * the kp-slab FP64 reduction -- the on-device form of the C
//     reduce-scatter with mpi_op_omp_sum (src/ca3dmm.c:1287-1343,
//     src/mpi_op_omp.c:6-23), summing slabs in rank order.
#include <cuda_runtime.h>
#include "k_common.cuh"
#include "ca3dmm_kernels.h"

namespace {

constexpr int TT = 32;   // transpose tile edge

// One CTA per (descriptor, 2D tile).  blockIdx.z = descriptor index.
// Copy path: tile of 256 rows x 8 columns, 256 threads, thread = row.
// Transpose path: 32 x 32 tile through shared memory (+1 pad), 32 x 8 threads.
__global__ void __launch_bounds__(256)
pack_kernel(const double *__restrict__ src_base, double *__restrict__ dst_base,
            const ca3dmm_pack_desc_t *__restrict__ descs)
{
    const ca3dmm_pack_desc_t d = descs[blockIdx.z];
    const double *src = src_base + d.src_off;
    double *dst = dst_base + d.dst_off;
    if (!d.trans) {
        const int r = blockIdx.x * 256 + threadIdx.x;
        const int c0 = blockIdx.y * 8;
        if (r >= d.rows || c0 >= d.cols) return;
        const int cn = min(8, d.cols - c0);
        double v[8];
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (c < cn) v[c] = __ldg(src + r + (long long) (c0 + c) * d.lds);
#pragma unroll
        for (int c = 0; c < 8; ++c)
            if (c < cn) dst[r + (long long) (c0 + c) * d.ldd] = v[c];
        return;
    }
    // dst (rows x cols) = transpose of the src block (cols x rows).
    __shared__ double tile[TT][TT + 1];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;   // 32 x 8
    const int r0 = blockIdx.x * TT, c0 = blockIdx.y * TT;     // in dst coordinates
    if (r0 >= d.rows || c0 >= d.cols) return;
    // Reads run along the source's contiguous index (dst column c), writes
    // along the destination's (dst row r); both are coalesced.
#pragma unroll
    for (int k = 0; k < TT; k += 8) {
        const int c = c0 + tx, r = r0 + ty + k;
        if (c < d.cols && r < d.rows) tile[ty + k][tx] = __ldg(src + c + (long long) r * d.lds);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < TT; k += 8) {
        const int r = r0 + tx, c = c0 + ty + k;
        if (r < d.rows && c < d.cols) dst[r + (long long) c * d.ldd] = tile[tx][ty + k];
    }
}

// out = sum of nslab slabs, column-major, 2 doubles per thread when aligned.
__global__ void __launch_bounds__(256)
reduce_slabs_kernel(const double *__restrict__ slab, long long slab_stride, long long lds,
                    int nslab, int m, int n, double *__restrict__ out, long long ldo, int vec)
{
    const long long mh = vec ? (m + 1) / 2 : m;
    const long long total = mh * n;
    for (long long idx = blockIdx.x * (long long) blockDim.x + threadIdx.x; idx < total;
         idx += (long long) gridDim.x * blockDim.x) {
        const long long j = idx / mh;
        const long long i = (idx - j * mh) * (vec ? 2 : 1);
        if (vec && i + 1 < m) {
            const double *p = slab + i + j * lds;
            double2 s = *reinterpret_cast<const double2 *>(p);
            for (int q = 1; q < nslab; ++q) {
                double2 v = *reinterpret_cast<const double2 *>(p + q * slab_stride);
                s.x += v.x;
                s.y += v.y;
            }
            *reinterpret_cast<double2 *>(out + i + j * ldo) = s;
        } else {
            const double *p = slab + i + j * lds;
            double s = p[0];
            for (int q = 1; q < nslab; ++q) s += p[q * slab_stride];
            out[i + j * ldo] = s;
        }
    }
}

}  // namespace

extern "C" int ca3dmm_pack_launch(const double *src_base, double *dst_base,
                                  const ca3dmm_pack_desc_t *dev_descs, int ndesc, int max_rows,
                                  int max_cols, int any_trans, cudaStream_t stream)
{
    if (ndesc <= 0 || max_rows <= 0 || max_cols <= 0) return CA3DMM_OK;
    if (ndesc > 65535) return CA3DMM_EINVAL;
    // grid covers the larger of the copy tiling (256 x 8) and the transpose
    // tiling (32 x 32); blocks outside a descriptor's extent exit at once.
    unsigned gx = (unsigned) ((max_rows + 255) / 256), gy = (unsigned) ((max_cols + 7) / 8);
    if (any_trans) {
        unsigned tx = (unsigned) ((max_rows + TT - 1) / TT), ty = (unsigned) ((max_cols + TT - 1) / TT);
        if (tx > gx) gx = tx;
        if (ty > gy) gy = ty;
    }
    if (gy > 65535) return CA3DMM_EINVAL;
    dim3 grid(gx, gy, (unsigned) ndesc);
    pack_kernel<<<grid, 256, 0, stream>>>(src_base, dst_base, dev_descs);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    return CA3DMM_OK;
}

extern "C" int ca3dmm_reduce_slabs_launch(const double *slab, long long slab_stride,
                                          long long lds, int nslab, int m, int n, double *out,
                                          long long ldo, cudaStream_t stream)
{
    if (m <= 0 || n <= 0 || nslab <= 0) return CA3DMM_OK;
    int vec = ((reinterpret_cast<uintptr_t>(slab) | reinterpret_cast<uintptr_t>(out)) & 15) == 0 &&
              (lds % 2 == 0) && (ldo % 2 == 0) && (slab_stride % 2 == 0);
    long long work = (vec ? (m + 1LL) / 2 : (long long) m) * n;
    long long blocks = (work + 255) / 256;
    int cap = ca3dmm_device_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    reduce_slabs_kernel<<<(unsigned) blocks, 256, 0, stream>>>(slab, slab_stride, lds, nslab, m, n,
                                                             out, ldo, vec);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    return CA3DMM_OK;
}
