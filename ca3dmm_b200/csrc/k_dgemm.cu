// Plain FP64 GEMM on the sm_100a FP64 tensor path (DMMA, mma.sync m16n8k4 f64),
// fed by TMA through a multi-stage mbarrier pipeline, as one persistent
// grouped launch over every tile of every problem.
//
// Replaces the reference's per-Cannon-step cublasDgemm + stream sync
// (src/cannon.c:410-418, :651-676; src/cuda_proxy.cu:211-230).  All virtual
// ranks' cuboid GEMMs of one ca3dmm exec run in this single launch.
//
// Layout (per stage, 32 KiB for 128-column tiles or 24 KiB for 64-column
// ones, 1024-byte aligned):
//   A tile: 128 (m) x 16 (k) doubles as 8 TMA boxes of 16 m x 16 k, each box
//           16 rows (k) of 128 B (m), SWIZZLE_128B -- or, for a K-major A
//           (a transposed operand read in place), 1 box of 128 rows (m) of
//           128 B (k), like B.
//   B tile: TBN (n) x 16 (k) doubles as 1 TMA box, TBN rows (n) of 128 B (k),
//           SWIZZLE_128B (TBN = 128 or 64 output columns per tile).
// Fragment ownership is permuted so every fragment load is one conflict-free
// 128-bit LDS:
//   * MMA row r of an m16 tile  -> tile row 2r (r < 8) or 2(r-8)+1, so a0/a1 of
//     m16n8k4 are the two doubles of one 16-byte chunk;
//   * MMA column c of n8 tile j -> warp column 4c + j;
//   * MMA k index t of k-step (q, b) -> tile k row 8q + 2t + b, so one 16-byte
//     chunk of a B row holds the b0 fragments of two consecutive k-steps.
// With the 128B swizzle (16-byte chunk index XOR row % 8) these choices put
// every quarter-warp of a 128-bit load on 8 distinct chunks.
// K-major A: a 16-byte chunk of a tile row holds that row's a0 (or a1) of two
// consecutive k-steps, as for B.  MMA rows g and g + 8 of m16 tile i are tile
// rows 16i + 2 sigma(g) and 16i + 2 sigma(g) + 1, sigma swapping the two low
// bits of g, so the two rows of a quarter-warp differ by 4 (mod 8) and hit
// disjoint chunk sets, and the C pairs (m, m+1) stay adjacent.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include <atomic>
#include "k_common.cuh"
#include "ca3dmm_kernels.h"

namespace {

constexpr int BM = 128, BK = 16;
constexpr int A_BYTES = BM * BK * 8;                 // 16 KiB
constexpr int CONSUMER_WARPS = 8;
constexpr int THREADS = CONSUMER_WARPS * 32;         // thread 0 also issues the TMA loads
constexpr int GROUP_M = 8;

// The output tile is BM x TBN, TBN = 128 or 64 columns.  Each warp computes
// 16 MI rows x 32 columns (MI m16 tiles x 4 n8 tiles): the 8 warps stand
// WM x WN = 2 x 4 over a 128-column tile and 4 x 2 over a 64-column one, so
// the fragment layout of a warp is the same for both widths.
template <int TBN>
struct DTile {
    static_assert(TBN == 128 || TBN == 64, "tile width");
    static constexpr int WN = TBN / 32, WM = CONSUMER_WARPS / WN, MI = BM / (16 * WM);
    static constexpr int STAGE_BYTES = A_BYTES + TBN * BK * 8;   // 32 or 24 KiB
    static constexpr int STAGES = TBN == 128 ? 5 : 6;
    static constexpr size_t SMEM_BYTES = (size_t) STAGES * STAGE_BYTES + 2 * STAGES * 8 + 1024;
};

struct alignas(16) DProb {
    double *C;
    long long ldc;
    int m, n, k;
    int tiles_m, tiles_n, tile_begin;
    double alpha, beta;
    int vec_ok, raster;
};

// The problem holding tile `tile`.  sb: a shared-memory copy of the problems'
// first tiles (nullptr when there are more than PROB_CACHE problems), so that a
// batch of small GEMMs does not pay a chain of dependent global loads per tile.
constexpr int PROB_CACHE = 1024;
__device__ __forceinline__ int find_problem(const int *sb, const DProb *probs, int nprob, int tile)
{
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if ((sb ? sb[mid] : probs[mid].tile_begin) <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void tile_coords(const DProb &p, int tile, int &tm, int &tn)
{
    int t = tile - p.tile_begin;
    int group_size = p.raster * p.tiles_n;
    int group = t / group_size;
    int first_m = group * p.raster;
    int gm = min(p.tiles_m - first_m, p.raster);
    int r = t % group_size;
    tm = first_m + r % gm;
    tn = r / gm;
}

__device__ __forceinline__ void dmma(double (&d)[4], double a0, double a1, double b0)
{
    asm volatile(
        "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a0), "d"(a1), "d"(b0));
}

__device__ __forceinline__ void store_pair(const DProb &p, int m, int n, double v0, double v1)
{
    if (n >= p.n || m >= p.m) return;
    double *c = p.C + (long long) m + (long long) n * p.ldc;
    if (p.vec_ok && m + 1 < p.m) {
        double2 o;
        if (p.beta != 0.0) {
            double2 old = *reinterpret_cast<const double2 *>(c);
            o.x = p.alpha * v0 + p.beta * old.x;
            o.y = p.alpha * v1 + p.beta * old.y;
        } else {
            o.x = p.alpha * v0;
            o.y = p.alpha * v1;
        }
        *reinterpret_cast<double2 *>(c) = o;
    } else {
        c[0] = p.beta != 0.0 ? p.alpha * v0 + p.beta * c[0] : p.alpha * v0;
        if (m + 1 < p.m) c[1] = p.beta != 0.0 ? p.alpha * v1 + p.beta * c[1] : p.alpha * v1;
    }
}

// Iterator over this CTA's (tile, k-tile) load sequence, used by the
// producer thread.  Tiles with k == 0 carry no loads and are skipped.
template <int TBN>
struct LoadCursor {
    int tile, kt, ktiles, pi, m0, n0;   // tile: virtual index into the launch's ranges
    bool valid;
    __device__ void seek(const int *sb, const DProb *probs, int nprob,
                         const ca3dmm_tile_ranges_t &rg, int total_tiles, int stride)
    {
        while (tile < total_tiles) {
            const int t = range_tile(rg, tile);
            pi = find_problem(sb, probs, nprob, t);
            const DProb &p = probs[pi];
            ktiles = (p.k + BK - 1) / BK;
            if (ktiles > 0) {
                int tm, tn;
                tile_coords(p, t, tm, tn);
                m0 = tm * BM;
                n0 = tn * TBN;
                valid = true;
                return;
            }
            tile += stride;
        }
        valid = false;
    }
    __device__ void advance(const int *sb, const DProb *probs, int nprob,
                            const ca3dmm_tile_ranges_t &rg,
                            int total_tiles, int stride)
    {
        if (++kt < ktiles) return;
        kt = 0;
        tile += stride;
        seek(sb, probs, nprob, rg, total_tiles, stride);
    }
};

// sigma: swap the two low bits of g (0..7)
__device__ __forceinline__ int sigma_row(int g) { return (g & 4) | ((g & 1) << 1) | ((g >> 1) & 1); }

// The k loop of one output tile: wait for each stage, run the 16-k block's
// DMMAs, release the stage and (thread 0) refill it.  AK: A tile K-major.
template <bool AK, int TBN, class Issue>
__device__ __forceinline__ bool k_loop(const uint8_t *smem, uint64_t *full, uint64_t *empty,
                                       int ktiles, uint32_t &it,
                                       double (&acc)[DTile<TBN>::MI][4][4],
                                       volatile int *abort_flag, int *status,
                                       unsigned long long limit_ns, bool producer,
                                       Issue &issue_one, int wm, int wn, int g, int t, int lane)
{
    using T = DTile<TBN>;
    constexpr int MI = T::MI;
    for (int kt = 0; kt < ktiles; ++kt, ++it) {
        const uint32_t stage = it % T::STAGES, phase = (it / T::STAGES) & 1u;
        if (!mbar_wait_bounded(&full[stage], phase, abort_flag, status,
                               CA3DMM_DEV_TIMEOUT_CONSUME, limit_ns))
            return false;
        const uint8_t *sA = smem + stage * T::STAGE_BYTES;
        const uint8_t *sB = sA + A_BYTES;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            double2 bf[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int nl = wn * 32 + 4 * g + j;
                bf[j] = *reinterpret_cast<const double2 *>(
                    sB + nl * 128 + (((4 * q + t) ^ (nl & 7)) << 4));
            }
            if (AK) {
#pragma unroll
                for (int ip = 0; ip < MI / 2; ++ip) {
                    double2 alo[2], ahi[2];
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        // K-major A: tile row of MMA row g of m16 tile i
                        const int ra = wm * 16 * MI + 2 * sigma_row(g) + 16 * (2 * ip + h);
                        alo[h] = *reinterpret_cast<const double2 *>(
                            sA + ra * 128 + (((4 * q + t) ^ (ra & 7)) << 4));
                        ahi[h] = *reinterpret_cast<const double2 *>(
                            sA + (ra + 1) * 128 + (((4 * q + t) ^ ((ra + 1) & 7)) << 4));
                    }
#pragma unroll
                    for (int b = 0; b < 2; ++b)
#pragma unroll
                        for (int h = 0; h < 2; ++h)
#pragma unroll
                            for (int j = 0; j < 4; ++j)
                                dmma(acc[2 * ip + h][j], b ? alo[h].y : alo[h].x,
                                     b ? ahi[h].y : ahi[h].x, b ? bf[j].y : bf[j].x);
                    
                }
            } else {
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    const int kr = 8 * q + 2 * t + b;
                    double2 af[MI];
#pragma unroll
                    for (int i = 0; i < MI; ++i)
                        af[i] = *reinterpret_cast<const double2 *>(
                            sA + (wm * MI + i) * 2048 + kr * 128 + ((g ^ (kr & 7)) << 4));
#pragma unroll
                    for (int i = 0; i < MI; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            dmma(acc[i][j], af[i].x, af[i].y, b ? bf[j].y : bf[j].x);
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[stage]);
        if (producer && !issue_one()) return false;
    }
    return true;
}

// All 8 warps compute; thread 0 also drives the TMA pipeline.  Load L lands
// in stage L % STAGES; before issuing it the producer waits for the release
// of load L - STAGES.  Loads are issued STAGES-1 ahead of consumption, and the
// refill after consuming load `it` waits on the release of load it - 1, which
// every warp has usually finished, so the producer thread rarely stalls.
template <bool AK, int TBN>
__global__ void __launch_bounds__(THREADS, 1)
dgemm_dmma_grouped(const CUtensorMap *__restrict__ tmaps, const DProb *__restrict__ probs,
                   int nprob, const ca3dmm_tile_ranges_t rg, int total_tiles, int *status,
                   unsigned long long limit_ns)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    using T = DTile<TBN>;
    constexpr int STAGES = T::STAGES, STAGE_BYTES = T::STAGE_BYTES, MI = T::MI;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    __shared__ volatile int abort_flag;
    __shared__ int s_pbeg[PROB_CACHE];
    // the search table: rematerialised at each use (a kernel parameter and a
    // shared address), not held in a register across the main loop
#define CA3DMM_PB (nprob <= PROB_CACHE ? s_pbeg : nullptr)
    if (nprob <= PROB_CACHE)
        for (int i = threadIdx.x; i < nprob; i += blockDim.x) s_pbeg[i] = probs[i].tile_begin;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool producer = threadIdx.x == 0;
    if (producer) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], CONSUMER_WARPS);
        }
        abort_flag = 0;
        fence_barrier_init();
    }
    __syncthreads();

    LoadCursor<TBN> lc = {};
    uint32_t issued = 0;
    int last_p = -1;
    // Issue load number `issued` at the cursor (producer thread only).
    auto issue_one = [&]() -> bool {
        if (!lc.valid) return true;
        const uint32_t s = issued % STAGES, ph = (issued / STAGES) & 1u;
        if (!mbar_wait_bounded(&empty[s], ph ^ 1u, &abort_flag, status,
                               CA3DMM_DEV_TIMEOUT_PRODUCE, limit_ns))
            return false;
        const CUtensorMap *ta = tmaps + 2 * lc.pi, *tb = ta + 1;
        if (lc.pi != last_p) {
            tmap_acquire(ta);
            tmap_acquire(tb);
            last_p = lc.pi;
        }
        uint8_t *sA = smem + s * STAGE_BYTES;
        uint8_t *sB = sA + A_BYTES;
        mbar_arrive_expect_tx(&full[s], STAGE_BYTES);
        if (AK) {
            tma_load_2d(sA, ta, lc.kt * BK, lc.m0, &full[s]);
        } else {
#pragma unroll
            for (int j = 0; j < BM / 16; ++j)
                tma_load_2d(sA + j * 2048, ta, lc.m0 + 16 * j, lc.kt * BK, &full[s]);
        }
        tma_load_2d(sB, tb, lc.kt * BK, lc.n0, &full[s]);
        ++issued;
        lc.advance(CA3DMM_PB, probs, nprob, rg, total_tiles, gridDim.x);
        return true;
    };
    if (producer) {
        lc.tile = blockIdx.x;
        lc.kt = 0;
        lc.seek(CA3DMM_PB, probs, nprob, rg, total_tiles, gridDim.x);
        for (int s = 0; s < STAGES - 1; ++s)
            if (!issue_one()) break;
    }

    const int g = lane >> 2, t = lane & 3;
    const int wm = warp / T::WN, wn = warp % T::WN;
    uint32_t it = 0;   // loads consumed so far
    double acc[MI][4][4];
    bool ok = true;

    for (int v = blockIdx.x; v < total_tiles && ok; v += gridDim.x) {
        const int tile = range_tile(rg, v);
        int pi = find_problem(CA3DMM_PB, probs, nprob, tile);
        const DProb &p = probs[pi];
        int tm, tn;
        tile_coords(p, tile, tm, tn);
        const int ktiles = (p.k + BK - 1) / BK;
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0;

        ok = k_loop<AK, TBN>(smem, full, empty, ktiles, it, acc, &abort_flag, status, limit_ns,
                        producer, issue_one, wm, wn, g, t, lane);
        if (!ok) break;

        const int mb = tm * BM + wm * 16 * MI + 2 * (AK ? sigma_row(g) : g);
        const int nb = tn * TBN + wn * 32 + 8 * t;
#pragma unroll
        for (int i = 0; i < MI; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                store_pair(p, mb + 16 * i, nb + j, acc[i][j][0], acc[i][j][2]);
                store_pair(p, mb + 16 * i, nb + 4 + j, acc[i][j][1], acc[i][j][3]);
            }
    }

    if (producer) {
        // Wait (bounded, ignoring the abort flag) for every copy still in
        // flight so no TMA write lands in shared memory after exit.
        const uint32_t first = issued > STAGES ? issued - STAGES : 0;
        for (uint32_t L = first; L < issued; ++L) {
            const uint32_t s = L % STAGES, ph = (L / STAGES) & 1u;
            uint64_t t0 = global_timer_ns();
            while (!mbar_try_wait(&full[s], ph)) {
                if (global_timer_ns() - t0 > limit_ns) {
                    atomicCAS(status, 0, CA3DMM_DEV_TIMEOUT_PRODUCE);
                    break;
                }
            }
        }
    }
}
#undef CA3DMM_PB

typedef CUresult (*encode_tiled_fn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                    const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                    const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

encode_tiled_fn get_encode()
{
    // resolved once; the initialisation of a function-local static is thread-safe
    static const encode_tiled_fn fn = []() -> encode_tiled_fn {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        return reinterpret_cast<encode_tiled_fn>(p);
    }();
    return fn;
}

// cuTensorMapEncodeTiled is a driver call: it fails in a host thread that has
// no current context, which a thread that has made no runtime call yet lacks
// (the runtime binds the primary context lazily).  cudaSetDevice binds the
// current device's primary context to the calling thread without waiting on
// any stream.
void bind_device_context()
{
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaSetDevice(dev);
}

}  // namespace

extern "C" int ca3dmm_encode_tmap_2d(void *tmap, int dtype_bytes, const void *base,
                                     unsigned long long dim0, unsigned long long dim1,
                                     unsigned long long stride1_bytes, unsigned box0,
                                     unsigned box1, int swizzle128)
{
    encode_tiled_fn enc = get_encode();
    if (!enc) return CA3DMM_ENODEV;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (stride1_bytes & 15)) return CA3DMM_EINVAL;
    bind_device_context();
    CUtensorMapDataType dt =
        dtype_bytes == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_UINT8;
    cuuint64_t dims[2] = {dim0, dim1};
    cuuint64_t strides[1] = {stride1_bytes};
    cuuint32_t box[2] = {box0, box1};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(reinterpret_cast<CUtensorMap *>(tmap), dt, 2, const_cast<void *>(base), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     swizzle128 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CA3DMM_OK : CA3DMM_EINVAL;
}

extern "C" int ca3dmm_encode_tmap_u8(void *tmap, int rank, const void *base,
                                     const unsigned long long *dims,
                                     const unsigned long long *strides_bytes,
                                     const unsigned *box)
{
    encode_tiled_fn enc = get_encode();
    if (!enc) return CA3DMM_ENODEV;
    if (rank < 1 || rank > 5 || (reinterpret_cast<uintptr_t>(base) & 15)) return CA3DMM_EINVAL;
    bind_device_context();
    cuuint64_t d[5], st[4];
    cuuint32_t bx[5], es[5];
    for (int i = 0; i < rank; ++i) {
        d[i] = dims[i];
        bx[i] = box[i];
        es[i] = 1;
        if (i > 0) {
            if (strides_bytes[i - 1] & 15) return CA3DMM_EINVAL;
            st[i - 1] = strides_bytes[i - 1];
        }
    }
    CUresult r = enc(reinterpret_cast<CUtensorMap *>(tmap), CU_TENSOR_MAP_DATA_TYPE_UINT8,
                     (cuuint32_t) rank, const_cast<void *>(base), d, st, bx, es,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CA3DMM_OK : CA3DMM_EINVAL;
}

extern "C" size_t ca3dmm_dgemm_plan_bytes(int nprob)
{
    return (size_t) nprob * 2 * sizeof(CUtensorMap) + (size_t) nprob * sizeof(DProb);
}

extern "C" int ca3dmm_dgemm_plan_encode(const ca3dmm_dgemm_desc_t *probs, int nprob,
                                        void *host_plan, int *total_tiles)
{
    return ca3dmm_dgemm_plan_encode_tn(probs, nprob, host_plan, total_tiles, 128);
}

extern "C" int ca3dmm_dgemm_plan_encode_tn(const ca3dmm_dgemm_desc_t *probs, int nprob,
                                           void *host_plan, int *total_tiles, int tile_n)
{
    if (tile_n != 128 && tile_n != 64) return CA3DMM_EINVAL;
    CUtensorMap *tm = reinterpret_cast<CUtensorMap *>(host_plan);
    DProb *dp = reinterpret_cast<DProb *>(tm + 2 * nprob);
    int tiles = 0;
    for (int i = 0; i < nprob; ++i) {
        const ca3dmm_dgemm_desc_t &q = probs[i];
        if (q.m < 0 || q.n < 0 || q.k < 0) return CA3DMM_EINVAL;
        if ((q.a_kmajor != 0) != (probs[0].a_kmajor != 0)) return CA3DMM_EINVAL;
        if ((q.lda & 1) || (q.ldb & 1) || q.lda < (q.a_kmajor ? q.k : q.m) || q.ldb < q.k)
            return CA3DMM_EINVAL;
        memset(&tm[2 * i], 0, 2 * sizeof(CUtensorMap));
        if (q.m > 0 && q.n > 0 && q.k > 0) {
            int r = q.a_kmajor
                        ? ca3dmm_encode_tmap_2d(&tm[2 * i], 8, q.A, (unsigned long long) q.k,
                                                (unsigned long long) q.m,
                                                (unsigned long long) q.lda * 8, 16, BM, 1)
                        : ca3dmm_encode_tmap_2d(&tm[2 * i], 8, q.A, (unsigned long long) q.m,
                                                (unsigned long long) q.k,
                                                (unsigned long long) q.lda * 8, 16, 16, 1);
            if (r) return r;
            r = ca3dmm_encode_tmap_2d(&tm[2 * i + 1], 8, q.B, (unsigned long long) q.k,
                                      (unsigned long long) q.n, (unsigned long long) q.ldb * 8,
                                      16, (unsigned) tile_n, 1);
            if (r) return r;
        }
        DProb &d = dp[i];
        memset(&d, 0, sizeof(d));
        d.C = q.C;
        d.ldc = q.ldc;
        d.m = q.m; d.n = q.n; d.k = q.k;
        d.alpha = q.alpha; d.beta = q.beta;
        // k == 0 still needs the beta-scaling pass; give it one tile per block
        // through the normal path (ktiles == 0 -> acc stays 0).
        d.tiles_m = (q.m > 0 && q.n > 0) ? (q.m + BM - 1) / BM : 0;
        d.tiles_n = (q.m > 0 && q.n > 0) ? (q.n + tile_n - 1) / tile_n : 0;
        d.tile_begin = tiles;
        d.vec_ok = ((reinterpret_cast<uintptr_t>(q.C) & 15) == 0) && ((q.ldc & 1) == 0);
        d.raster = q.raster > 0 ? q.raster : GROUP_M;
        tiles += d.tiles_m * d.tiles_n;
    }
    *total_tiles = tiles;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_dgemm_launch(const void *dev_plan, int nprob, int total_tiles, int a_kmajor,
                                   int *dev_status, double timeout_s, cudaStream_t stream)
{
    return ca3dmm_dgemm_launch_tn(dev_plan, nprob, total_tiles, a_kmajor, dev_status, timeout_s,
                                  stream, 128);
}

extern "C" int ca3dmm_dgemm_launch_tn(const void *dev_plan, int nprob, int total_tiles,
                                      int a_kmajor, int *dev_status, double timeout_s,
                                      cudaStream_t stream, int tile_n)
{
    ca3dmm_tile_ranges_t rg;
    memset(&rg, 0, sizeof(rg));
    rg.n = 1;
    rg.len[0] = total_tiles;
    return ca3dmm_dgemm_launch_ranges_tn(dev_plan, nprob, &rg, a_kmajor, dev_status, timeout_s,
                                         stream, tile_n);
}

extern "C" int ca3dmm_dgemm_launch_ranges(const void *dev_plan, int nprob,
                                          const ca3dmm_tile_ranges_t *ranges, int a_kmajor,
                                          int *dev_status, double timeout_s, cudaStream_t stream)
{
    return ca3dmm_dgemm_launch_ranges_tn(dev_plan, nprob, ranges, a_kmajor, dev_status, timeout_s,
                                         stream, 128);
}

namespace {
// the shared-memory limit of one instantiation, raised once per device (a bit
// per device ordinal; two threads may both set it, which is harmless)
template <bool AK, int TBN>
cudaError_t dgemm_attr_once()
{
    static std::atomic<unsigned long long> done{0};
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (!bit || !(done.load(std::memory_order_acquire) & bit)) {
        err = cudaFuncSetAttribute(dgemm_dmma_grouped<AK, TBN>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int) DTile<TBN>::SMEM_BYTES);
        if (err != cudaSuccess) return err;
        done.fetch_or(bit, std::memory_order_release);
    }
    return cudaSuccess;
}

template <bool AK, int TBN>
cudaError_t dgemm_launch_one(int grid, const CUtensorMap *tm, const DProb *dp, int nprob,
                             const ca3dmm_tile_ranges_t &rg, int total_tiles, int *status,
                             unsigned long long limit, cudaStream_t stream)
{
    cudaError_t err = dgemm_attr_once<AK, TBN>();
    if (err != cudaSuccess) return err;
    dgemm_dmma_grouped<AK, TBN><<<grid, THREADS, DTile<TBN>::SMEM_BYTES, stream>>>(
        tm, dp, nprob, rg, total_tiles, status, limit);
    return cudaGetLastError();
}
}  // namespace

extern "C" int ca3dmm_dgemm_launch_ranges_tn(const void *dev_plan, int nprob,
                                             const ca3dmm_tile_ranges_t *ranges, int a_kmajor,
                                             int *dev_status, double timeout_s,
                                             cudaStream_t stream, int tile_n)
{
    if (!ranges || ranges->n < 0 || ranges->n > CA3DMM_MAX_RANGES) return CA3DMM_EINVAL;
    if (tile_n != 128 && tile_n != 64) return CA3DMM_EINVAL;
    const int total_tiles = range_total(*ranges);
    if (total_tiles <= 0) return CA3DMM_OK;
    const CUtensorMap *tm = reinterpret_cast<const CUtensorMap *>(dev_plan);
    const DProb *dp = reinterpret_cast<const DProb *>(tm + 2 * nprob);
    int grid = ca3dmm_device_sm_count();
    if (grid > total_tiles) grid = total_tiles;
    const unsigned long long limit = (unsigned long long) (timeout_s * 1e9);
    cudaError_t err;
    if (tile_n == 128)
        err = a_kmajor ? dgemm_launch_one<true, 128>(grid, tm, dp, nprob, *ranges, total_tiles,
                                                      dev_status, limit, stream)
                       : dgemm_launch_one<false, 128>(grid, tm, dp, nprob, *ranges, total_tiles,
                                                       dev_status, limit, stream);
    else
        err = a_kmajor ? dgemm_launch_one<true, 64>(grid, tm, dp, nprob, *ranges, total_tiles,
                                                     dev_status, limit, stream)
                       : dgemm_launch_one<false, 64>(grid, tm, dp, nprob, *ranges, total_tiles,
                                                      dev_status, limit, stream);
    CA3DMM_CUDA_TRY(err);
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}

extern "C" int ca3dmm_device_sm_count(void)
{
    static std::atomic<int> sms[64];        // zero-initialised (static storage)
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int v = sms[dev].load(std::memory_order_relaxed);
    if (!v) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        sms[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}
