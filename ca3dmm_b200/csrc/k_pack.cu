// Redistribution kernels of the virtual process grid, HBM-bound:
//   * batched block pack (copy or transpose) of column-major matrices --
//     the on-device form of mat_redist's pack -> alltoallv -> unpack
//     (src/mat_redist.c:327-348, :395-416) fused with the operand transpose
//     the reference does with cublasDgeam (src/ca3dmm.c:1036-1058);
//   * the kp-slab FP64 reduction -- the on-device form of the C
//     reduce-scatter with mpi_op_omp_sum (src/ca3dmm.c:1287-1343,
//     src/mpi_op_omp.c:6-23), summing slabs in rank order.
#include <atomic>
#include <cstring>
#include <cuda.h>
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
__global__ void __launch_bounds__(256, 3)
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
        // dst (rows x cols) = transpose of the source block (cols x rows); the
        // 16 loads of a thread are all in flight before the shared stores
        double v[PT * PT / 256];
#pragma unroll
        for (int i = 0; i < PT * PT / 256; ++i) {
            const int e = threadIdx.x + 256 * i;
            const int c = c0 + (e & 63), r = r0 + (e >> 6);
            v[i] = (c < d.cols && r < d.rows) ? __ldg(src + c + (long long) r * d.lds) : 0.0;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < PT * PT / 256; ++i) {
            const int e = threadIdx.x + 256 * i;
            tile[e >> 6][e & 63] = v[i];
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < PT * PT / 256; ++i) {
            const int e = threadIdx.x + 256 * i;
            const int r = r0 + (e & 63), c = c0 + (e >> 6);
            if (r < d.rows && c < d.cols) dst[r + (long long) c * d.ldd] = tile[e & 63][e >> 6];
        }
    }
}

// Transposing pack staged through shared memory by TMA: tiles of 64
// destination rows x 64 destination columns arrive as four 16 x 64 boxes of
// the source (16 contiguous doubles = one 128-byte box row, so 512
// contiguous source bytes per row and tile) with the 128-byte swizzle,
// TT_STAGES tiles ahead of the threads that write them out.  A thread reads
// 16-byte chunks (two destination columns of one row): 32 threads of
// consecutive rows hit eight distinct swizzled chunks, the minimum four
// wavefronts; the writes run down the destination columns.
constexpr int TT_R = 64, TT_BOX = 16, TT_NBOX = 4, TT_C = TT_BOX * TT_NBOX, TT_STAGES = 4;
constexpr int TT_BOX_BYTES = TT_R * TT_BOX * (int) sizeof(double);   // 8 KB
constexpr int TT_BYTES = TT_BOX_BYTES * TT_NBOX;                       // 32 KB
constexpr int TT_SMEM = TT_STAGES * TT_BYTES + 1024;

__device__ __forceinline__ void tt_tile(const ca3dmm_pack_desc_t &d, int t, int &r0, int &c0)
{
    const int local = t - d.tile_begin, tr = (d.rows + TT_R - 1) / TT_R;
    r0 = (local % tr) * TT_R;
    c0 = (local / tr) * TT_C;
}

__global__ void __launch_bounds__(256)
pack_transpose_tma_kernel(const CUtensorMap *__restrict__ tmaps,
                          const ca3dmm_pack_desc_t *__restrict__ descs, int ndesc, int total_tiles,
                          double *__restrict__ dst_base, int *status, unsigned long long limit_ns)
{
    extern __shared__ unsigned char tt_raw[];
    unsigned char *sm = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(tt_raw) + 1023) & ~uintptr_t(1023));
    __shared__ uint64_t full[TT_STAGES];
    __shared__ volatile int abort_flag;
    if (threadIdx.x == 0) {
        for (int s = 0; s < TT_STAGES; ++s) mbar_init(&full[s], 1);
        abort_flag = 0;
        fence_barrier_init();
    }
    __syncthreads();
    const int mine = blockIdx.x < total_tiles ? (total_tiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    int issued = 0;
    auto issue = [&](int i) {
        const int t = blockIdx.x + i * gridDim.x;
        const int j = find_desc(descs, ndesc, t);
        int r0, c0;
        tt_tile(descs[j], t, r0, c0);
        tmap_acquire(tmaps + j);
        const int s = i % TT_STAGES;
        mbar_arrive_expect_tx(&full[s], TT_BYTES);
#pragma unroll
        for (int b = 0; b < TT_NBOX; ++b)
            tma_load_2d(sm + s * TT_BYTES + b * TT_BOX_BYTES, tmaps + j, c0 + b * TT_BOX, r0, &full[s]);
    };
    if (threadIdx.x == 0)
        for (; issued < mine && issued < TT_STAGES; ++issued) issue(issued);
    const int r = threadIdx.x & (TT_R - 1), q0 = threadIdx.x >> 6;
    bool ok = true;
    for (int i = 0; i < mine && ok; ++i) {
        const int s = i % TT_STAGES;
        if (!mbar_wait_bounded(&full[s], (uint32_t) (i / TT_STAGES) & 1u, &abort_flag, status,
                               CA3DMM_DEV_TIMEOUT_CONSUME, limit_ns)) {
            ok = false;
            break;
        }
        const int t = blockIdx.x + i * gridDim.x;
        const ca3dmm_pack_desc_t d = descs[find_desc(descs, ndesc, t)];
        int r0, c0;
        tt_tile(d, t, r0, c0);
        double *dst = reinterpret_cast<double *>(reinterpret_cast<uintptr_t>(dst_base) +
                                                 (uintptr_t) d.dst_off * sizeof(double));
        const unsigned char *row = sm + s * TT_BYTES + r * 128;
#pragma unroll
        for (int h = 0; h < TT_C / 8; ++h) {
            const int q = q0 + 4 * h;                       // chunk: columns 2q, 2q + 1
            const double2 v = *reinterpret_cast<const double2 *>(
                row + (q >> 3) * TT_BOX_BYTES + (((q & 7) ^ (r & 7)) << 4));
            const int gr = r0 + r, gc = c0 + 2 * q;
            if (gr < d.rows) {
                if (gc < d.cols) dst[gr + (long long) gc * d.ldd] = v.x;
                if (gc + 1 < d.cols) dst[gr + (long long) (gc + 1) * d.ldd] = v.y;
            }
        }
        __syncthreads();                                     // stage s read by every thread
        if (threadIdx.x == 0 && issued < mine) issue(issued++);
    }
    if (threadIdx.x == 0 && !ok) {
        // let the copies this CTA issued land before its shared memory is released
        for (int i = 0; i < issued; ++i) {
            const uint64_t t0 = global_timer_ns();
            while (!mbar_try_wait(&full[i % TT_STAGES], (uint32_t) (i / TT_STAGES) & 1u))
                if (global_timer_ns() - t0 > limit_ns) break;
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

// One block copy with its geometry passed by value (no descriptor in device
// memory): thread (row, 16 columns) of a 128 x 16 tile, the grid's y extent
// walking further column tiles when there are more than 65535 of them.
__global__ void __launch_bounds__(128)
copy_block_kernel(const double *__restrict__ src, long long lds, double *__restrict__ dst,
                  long long ldd, int rows, int cols)
{
    const int r = blockIdx.x * 128 + threadIdx.x;
    if (r >= rows) return;
    for (long long c0 = (long long) blockIdx.y * 16; c0 < cols; c0 += (long long) gridDim.y * 16) {
        double v[16];
#pragma unroll
        for (int c = 0; c < 16; ++c)
            if (c0 + c < cols) v[c] = __ldg(src + r + (c0 + c) * lds);
#pragma unroll
        for (int c = 0; c < 16; ++c)
            if (c0 + c < cols) dst[r + (c0 + c) * ldd] = v[c];
    }
}

extern "C" int ca3dmm_copy_block_launch(const double *src, long long lds, double *dst,
                                        long long ldd, int rows, int cols, cudaStream_t stream)
{
    if (rows <= 0 || cols <= 0) return CA3DMM_OK;
    const long long ty = ((long long) cols + 15) / 16;
    dim3 grid((unsigned) ((rows + 127) / 128), (unsigned) (ty < 65535 ? ty : 65535));
    copy_block_kernel<<<grid, 128, 0, stream>>>(src, lds, dst, ldd, rows, cols);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}

// Guard bands of a work buffer: one block, each thread compares its bytes of
// every band with the fill pattern.
__global__ void __launch_bounds__(256)
guard_check_kernel(const unsigned char *__restrict__ base, const ca3dmm_guard_bands_t g,
                   int *status)
{
    for (int b = 0; b < g.n; ++b) {
        const unsigned char *band = base + g.off[b];
        bool bad = false;
        for (int i = threadIdx.x; i < g.bytes; i += blockDim.x)
            bad = bad || band[i] != (unsigned char) g.pattern;
        if (__syncthreads_or(bad) && threadIdx.x == 0 &&
            atomicCAS(status, 0, CA3DMM_DEV_CANARY) == 0)
            status[1] = b;
    }
}

extern "C" int ca3dmm_guard_check_launch(const void *base, const ca3dmm_guard_bands_t *bands,
                                         int *dev_status, cudaStream_t stream)
{
    if (!bands || bands->n <= 0) return CA3DMM_OK;
    if (bands->n > CA3DMM_MAX_CANARIES) return CA3DMM_EINVAL;
    guard_check_kernel<<<1, 256, 0, stream>>>(static_cast<const unsigned char *>(base), *bands,
                                              dev_status);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
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

extern "C" int ca3dmm_encode_tmap_2d(void *tmap, int dtype_bytes, const void *base,
                                     unsigned long long dim0, unsigned long long dim1,
                                     unsigned long long stride1_bytes, unsigned box0,
                                     unsigned box1, int swizzle128);

extern "C" int ca3dmm_pack_tma_prepare(ca3dmm_pack_desc_t *descs, int ndesc, const double *src_base,
                                       void *host_tmaps, int *total_tiles)
{
    CUtensorMap *tm = static_cast<CUtensorMap *>(host_tmaps);
    int tiles = 0;
    for (int j = 0; j < ndesc; ++j) {
        ca3dmm_pack_desc_t &d = descs[j];
        memset(&tm[j], 0, sizeof(CUtensorMap));
        d.tile_begin = tiles;
        if (d.rows <= 0 || d.cols <= 0) continue;
        const double *b = src_base + d.src_off;
        if (!d.trans || (d.lds & 1) || (reinterpret_cast<uintptr_t>(b) & 15)) return CA3DMM_EINVAL;
        // source block: cols contiguous doubles per row, rows rows lds apart
        const int rc = ca3dmm_encode_tmap_2d(&tm[j], 8, b, (unsigned long long) d.cols,
                                             (unsigned long long) d.rows,
                                             (unsigned long long) d.lds * 8, TT_BOX, TT_R, 1);
        if (rc) return rc;
        tiles += ((d.rows + TT_R - 1) / TT_R) * ((d.cols + TT_C - 1) / TT_C);
    }
    *total_tiles = tiles;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_pack_tma_launch(const void *dev_tmaps, const ca3dmm_pack_desc_t *dev_descs,
                                      int ndesc, int total_tiles, double *dst_base,
                                      int *dev_status, double timeout_s, cudaStream_t stream)
{
    if (ndesc <= 0 || total_tiles <= 0) return CA3DMM_OK;
    static std::atomic<unsigned long long> attr_done{0};     // one bit per device
    int dev = 0;
    CA3DMM_CUDA_TRY(cudaGetDevice(&dev));
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (!(attr_done.load(std::memory_order_acquire) & bit) || !bit) {
        CA3DMM_CUDA_TRY(cudaFuncSetAttribute(pack_transpose_tma_kernel,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, TT_SMEM));
        attr_done.fetch_or(bit, std::memory_order_release);
    }
    int grid = ca3dmm_device_sm_count();
    if (grid > total_tiles) grid = total_tiles;
    pack_transpose_tma_kernel<<<grid, 256, TT_SMEM, stream>>>(
        static_cast<const CUtensorMap *>(dev_tmaps), dev_descs, ndesc, total_tiles, dst_base,
        dev_status, (unsigned long long) (timeout_s * 1e9));
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

// C(i, j) = C(j, i) for i > j: the strictly lower triangle of an n x n C
// rewritten from the upper one, through 32 x 32 shared-memory tiles (block
// (bi, bj), bi > bj, reads the upper tile (bj, bi) transposed).
__global__ void __launch_bounds__(256)
mirror_upper_kernel(double *__restrict__ C, long long ldc, int n)
{
    __shared__ double t[32][33];
    const int nb = (n + 31) / 32;
    const long long ntile = (long long) nb * (nb + 1) / 2;       // blocks with bi >= bj
    for (long long idx = blockIdx.x; idx < ntile; idx += gridDim.x) {
        // idx -> (bi, bj), bj <= bi, row-major over the lower block triangle
        int bi = (int) ((sqrt(8.0 * (double) idx + 1.0) - 1.0) * 0.5);
        while ((long long) (bi + 1) * (bi + 2) / 2 <= idx) ++bi;
        while ((long long) bi * (bi + 1) / 2 > idx) --bi;
        const int bj = (int) (idx - (long long) bi * (bi + 1) / 2);
        const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
        __syncthreads();                             // t of the previous tile is read
        // read the upper tile: rows 32 bj.., columns 32 bi.. (element (r, c) at r + c ldc)
        for (int y = ty; y < 32; y += 8) {
            const int r = 32 * bj + tx, c = 32 * bi + y;
            t[y][tx] = (r < n && c < n) ? C[r + (long long) c * ldc] : 0.0;
        }
        __syncthreads();
        // write the lower tile: rows 32 bi + tx, columns 32 bj + y, only strictly below the diagonal
        for (int y = ty; y < 32; y += 8) {
            const int r = 32 * bi + tx, c = 32 * bj + y;
            if (r < n && c < n && r > c) C[r + (long long) c * ldc] = t[tx][y];
        }
    }
}

extern "C" int ca3dmm_mirror_upper_launch(double *C, long long ldc, int n, cudaStream_t stream)
{
    if (n <= 1) return CA3DMM_OK;
    const int nb = (n + 31) / 32;
    long long tiles = (long long) nb * (nb + 1) / 2;
    const long long cap = (long long) ca3dmm_device_sm_count() * 8;
    mirror_upper_kernel<<<(unsigned) (tiles < cap ? tiles : cap), 256, 0, stream>>>(C, ldc, n);
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
