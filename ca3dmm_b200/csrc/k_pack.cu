// Redistribution kernels of the virtual process grid, HBM-bound:
//   * batched block pack (copy or transpose) of column-major matrices --
//     the on-device form of mat_redist's pack -> alltoallv -> unpack
//     (src/mat_redist.c:327-348, :395-416) fused with the operand transpose
//     the reference does with cublasDgeam (src/ca3dmm.c:1036-1058);
//   * the kp-slab FP64 reduction -- the on-device form of the C
//     reduce-scatter with mpi_op_omp_sum (src/ca3dmm.c:1287-1343,
//     src/mpi_op_omp.c:6-23), summing slabs in rank order.
#include <atomic>
#include <cuda_runtime.h>
#include "k_common.cuh"
#include "ca3dmm_kernels.h"

namespace {

constexpr int PT = 64;   // pack tile edge

__device__ __forceinline__ int find_desc(const ca3dmm_pack_desc_t *d, int n, int tile)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (d[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Persistent over the flat list of 64 x 64 tiles of every descriptor.
// Copy: thread -> (row, 16 columns), reads and writes run down the columns.
// Transpose: through a padded shared tile; reads run along the source's
// contiguous index, writes along the destination's.
__global__ void __launch_bounds__(256)
pack_kernel(const double *__restrict__ src_base, double *__restrict__ dst_base,
            const ca3dmm_pack_desc_t *__restrict__ descs, int ndesc, int total_tiles)
{
    __shared__ double tile[PT][PT + 1];
    for (int t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const ca3dmm_pack_desc_t d = descs[find_desc(descs, ndesc, t)];
        const int local = t - d.tile_begin;
        const int tx = (d.rows + PT - 1) / PT;
        const int r0 = (local % tx) * PT, c0 = (local / tx) * PT;
        const double *src = reinterpret_cast<const double *>(
            reinterpret_cast<uintptr_t>(src_base) + (uintptr_t) d.src_off * sizeof(double));
        double *dst = reinterpret_cast<double *>(reinterpret_cast<uintptr_t>(dst_base) +
                                                 (uintptr_t) d.dst_off * sizeof(double));
        if (!d.trans) {
            const int r = r0 + (threadIdx.x & 63), cb = c0 + (threadIdx.x >> 6) * 16;
            if (r < d.rows) {
                double v[16];
#pragma unroll
                for (int c = 0; c < 16; ++c)
                    if (cb + c < d.cols) v[c] = __ldg(src + r + (long long) (cb + c) * d.lds);
#pragma unroll
                for (int c = 0; c < 16; ++c)
                    if (cb + c < d.cols) dst[r + (long long) (cb + c) * d.ldd] = v[c];
            }
            continue;
        }
        // dst (rows x cols) = transpose of the source block (cols x rows)
        __syncthreads();
        for (int e = threadIdx.x; e < PT * PT; e += blockDim.x) {
            const int c = c0 + (e & 63), r = r0 + (e >> 6);
            if (c < d.cols && r < d.rows) tile[e >> 6][e & 63] = __ldg(src + c + (long long) r * d.lds);
        }
        __syncthreads();
        for (int e = threadIdx.x; e < PT * PT; e += blockDim.x) {
            const int r = r0 + (e & 63), c = c0 + (e >> 6);
            if (r < d.rows && c < d.cols) dst[r + (long long) c * d.ldd] = tile[e & 63][e >> 6];
        }
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

static std::atomic<unsigned long long> g_kernel_launches{0};

extern "C" void ca3dmm_note_launch(int n)
{
    g_kernel_launches.fetch_add((unsigned long long) n, std::memory_order_relaxed);
}

extern "C" unsigned long long ca3dmm_kernel_launches(void)
{
    return g_kernel_launches.load(std::memory_order_relaxed);
}

extern "C" int ca3dmm_pack_tiles(ca3dmm_pack_desc_t *descs, int ndesc)
{
    int tiles = 0;
    for (int j = 0; j < ndesc; ++j) {
        descs[j].tile_begin = tiles;
        if (descs[j].rows > 0 && descs[j].cols > 0)
            tiles += ((descs[j].rows + PT - 1) / PT) * ((descs[j].cols + PT - 1) / PT);
    }
    return tiles;
}

extern "C" int ca3dmm_pack_launch(const double *src_base, double *dst_base,
                                  const ca3dmm_pack_desc_t *dev_descs, int ndesc, int total_tiles,
                                  cudaStream_t stream)
{
    if (ndesc <= 0 || total_tiles <= 0) return CA3DMM_OK;
    int grid = ca3dmm_device_sm_count() * 8;
    if (grid > total_tiles) grid = total_tiles;
    pack_kernel<<<grid, 256, 0, stream>>>(src_base, dst_base, dev_descs, ndesc, total_tiles);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
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
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}

// Diagnostic of the bounded device wait every kernel of the library uses:
// thread 0 waits on an mbarrier that is completed (arrive != 0) or that
// nothing ever completes; the wait returns by itself after limit_ns.
__global__ void wait_check_kernel(int *status, unsigned long long limit_ns, int arrive)
{
    __shared__ uint64_t bar;
    __shared__ volatile int abort_flag;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        abort_flag = 0;
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (arrive) mbar_arrive(&bar);
        if (mbar_wait_bounded(&bar, 0, &abort_flag, status, CA3DMM_DEV_TIMEOUT_QUEUE, limit_ns))
            status[1] = 1;
    }
}

extern "C" int ca3dmm_device_wait_check(double timeout_s, int arrive)
{
    if (!(timeout_s >= 0.0) || timeout_s > 60.0) return CA3DMM_EINVAL;
    int *d = nullptr, h[2] = {0, 0};
    CA3DMM_CUDA_TRY(cudaMalloc(&d, 2 * sizeof(int)));
    int rc = CA3DMM_OK;
    if (cudaMemset(d, 0, 2 * sizeof(int)) != cudaSuccess) rc = CA3DMM_ECUDA;
    if (!rc) {
        wait_check_kernel<<<1, 32>>>(d, (unsigned long long) (timeout_s * 1e9), arrive ? 1 : 0);
        ca3dmm_note_launch(1);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
            cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess)
            rc = CA3DMM_ECUDA;
    }
    cudaFree(d);
    if (rc) return rc;
    if (h[0] != 0) return CA3DMM_ETIMEOUT;
    return h[1] ? CA3DMM_OK : CA3DMM_ECUDA;
}
