// Split-precision FP64 GEMM (Ozaki scheme with INT8 slices) for sm_100a.
//
//  1. oz_exp_kernel    -- per row of op(A) / column of op(B) over the block's k
//                         range: E = frexp exponent of max|x| (max|x| < 2^E).
//  2. oz_slice_kernel  -- x = sum_t q_t 2^(E-6-7t) + r with q_t = rint(...) in
//                         [-64, 64]; writes the s slices K-major (k contiguous),
//                         transposing through shared memory when the source is
//                         k-strided.  HBM-bound.
//  3. oz_gemm_kernel   -- tcgen05.mma kind::i8, M=128 x N=64 x K=32, all s
//                         diagonal accumulators D_d = sum_{t+u=d} Aq_t Bq_u^T held
//                         in TMEM at once (s*64 <= 512 columns), so every 64-byte
//                         k-block of every slice is loaded once (one 3D TMA box
//                         per operand, SWIZZLE_64B) and feeds all s(s+1)/2 slice
//                         products.  INT32 accumulation is exact while
//                         (d+1) k 64^2 < 2^31.  The epilogue recombines
//                         C = sum_{d=s-1..0} 2^(E_i+F_j-12-7d) D_d in FP64 from the
//                         least significant diagonal up.
// Warp roles of the GEMM: warp 0 TMA producer, warp 1 TMEM owner + MMA issuer,
// warps 2..5 epilogue (warp w reads TMEM lanes 32*(w%4)..+31).  All waits are
// bounded; on timeout the kernel records a status, drains, frees TMEM, returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <climits>
#include <cstdio>
#include <cstring>
#include "k_common.cuh"
#include "ca3dmm_kernels.h"
#include "ca3dmm_ozaki.h"

extern "C" int ca3dmm_encode_tmap_2d(void *tmap, int dtype_bytes, const void *base,
                                     unsigned long long dim0, unsigned long long dim1,
                                     unsigned long long stride1_bytes, unsigned box0,
                                     unsigned box1, int swizzle128);

namespace {

constexpr int OBM = 128, OBN = 64, OKB = 64;    // tile rows, tile cols, k bytes per stage
constexpr int OTHREADS = 192;
constexpr int MAX_SLICES = 8;
constexpr int A_SLICE_BYTES = OBM * OKB;        // 8 KiB
constexpr int B_SLICE_BYTES = OBN * OKB;        // 4 KiB
constexpr int SMEM_BUDGET = 200 * 1024;
constexpr int GROUP_M = 8;
constexpr int EXP_BIAS = 2048;                   // stored exponent = E + bias, 0 = all-zero row

// Slicing descriptor: block rows r in [0,rows), k index l in [0,kz);
// element (r,l) at src[src_off + r*rs + l*ls].
struct SliceDesc {
    long long src_off, rs, ls;
    long long q_off;        // byte offset of slice 0 in the work region
    long long e_off;        // int offset of the exponents in the work region
    int rows, kz, kpad, pad;
};

struct OzGroup {
    double *C;
    long long ldc;
    int m, n, k;
    int a_blk, b_blk;       // tensor map indices (B maps follow the A maps)
    int tiles_m, tiles_n, tile_begin;
    long long ea_off, eb_off;   // exponent offsets (ints) of the A rows / B columns
};

struct PlanHeader {
    int nA, nB, ngroup, slices;
    int nslice_desc, tiles, pad0, pad1;
};

// ------------------------------------------------------------------ slicing
constexpr int ST = 64;   // slicing tile edge (rows x k)

__global__ void __launch_bounds__(256)
oz_exp_kernel(const double *__restrict__ src, const SliceDesc *__restrict__ descs,
              unsigned *__restrict__ ework)
{
    const SliceDesc d = descs[blockIdx.z];
    const int r0 = blockIdx.x * ST, l0 = blockIdx.y * ST;
    if (r0 >= d.rows || l0 >= d.kz) return;
    __shared__ int smax[ST];
    if (threadIdx.x < ST) smax[threadIdx.x] = 0;
    __syncthreads();
    const double *base = src + d.src_off;
    const bool rfast = d.rs == 1;   // consecutive threads walk the contiguous index
    for (int e = threadIdx.x; e < ST * ST; e += blockDim.x) {
        const int a = e % ST, b = e / ST;
        const int r = rfast ? a : b, l = rfast ? b : a;
        const int gr = r0 + r, gl = l0 + l;
        if (gr < d.rows && gl < d.kz) {
            const double v = fabs(__ldg(base + gr * d.rs + gl * d.ls));
            if (v != 0.0) {
                int ex;
                frexp(v, &ex);
                atomicMax(&smax[r], ex + EXP_BIAS);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x < ST && r0 + threadIdx.x < d.rows && smax[threadIdx.x] > 0)
        atomicMax(ework + d.e_off + r0 + threadIdx.x, (unsigned) smax[threadIdx.x]);
}

__global__ void __launch_bounds__(256)
oz_slice_kernel(const double *__restrict__ src, const SliceDesc *__restrict__ descs,
                unsigned char *__restrict__ work, int slices)
{
    const SliceDesc d = descs[blockIdx.z];
    const int r0 = blockIdx.x * ST, l0 = blockIdx.y * ST;
    if (r0 >= d.rows || l0 >= d.kpad) return;
    __shared__ double tile[ST][ST + 1];
    const double *base = src + d.src_off;
    const bool rfast = d.rs == 1;
    for (int e = threadIdx.x; e < ST * ST; e += blockDim.x) {
        const int a = e % ST, b = e / ST;
        const int r = rfast ? a : b, l = rfast ? b : a;
        const int gr = r0 + r, gl = l0 + l;
        tile[r][l] = (gr < d.rows && gl < d.kz) ? __ldg(base + gr * d.rs + gl * d.ls) : 0.0;
    }
    __syncthreads();
    // thread -> (row r, 16 consecutive k)
    const int r = threadIdx.x >> 2, c = (threadIdx.x & 3) * 16;
    const int gr = r0 + r, gl = l0 + c;
    if (gr >= d.rows || gl >= d.kpad) return;
    const unsigned eb = reinterpret_cast<const unsigned *>(work)[d.e_off + gr];
    const int E = eb ? (int) eb - EXP_BIAS : 0;
    double up[MAX_SLICES], dn[MAX_SLICES];
#pragma unroll
    for (int t = 0; t < MAX_SLICES; ++t) {
        up[t] = ldexp(1.0, 6 + 7 * t - E);
        dn[t] = ldexp(1.0, E - 6 - 7 * t);
    }
    uint32_t q[MAX_SLICES][4];
#pragma unroll
    for (int t = 0; t < MAX_SLICES; ++t)
#pragma unroll
        for (int w = 0; w < 4; ++w) q[t][w] = 0;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        double x = tile[r][c + j];
#pragma unroll
        for (int t = 0; t < MAX_SLICES; ++t) {
            if (t < slices) {
                const double qq = rint(x * up[t]);
                x -= qq * dn[t];
                const uint32_t byte = (uint32_t) ((int) qq) & 0xffu;
                q[t][j >> 2] |= byte << (8 * (j & 3));
            }
        }
    }
    unsigned char *dst = work + d.q_off + (long long) gr * d.kpad + gl;
    const long long slice_bytes = (long long) d.rows * d.kpad;
#pragma unroll
    for (int t = 0; t < MAX_SLICES; ++t)
        if (t < slices)
            *reinterpret_cast<uint4 *>(dst + t * slice_bytes) =
                make_uint4(q[t][0], q[t][1], q[t][2], q[t][3]);
}

// ------------------------------------------------------------------ tcgen05 GEMM
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, int x, int y, int z,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

// K-major, SWIZZLE_64B shared-memory operand descriptor: rows of 64 bytes,
// 8-row groups 512 bytes apart (SBO), version 1, layout type 4.
__device__ __forceinline__ uint64_t sdesc_k64(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t) ((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t) 1 << 16;                 // LBO (unused for swizzled K-major)
    d |= (uint64_t) (512 >> 4) << 32;        // SBO
    d |= (uint64_t) 1 << 46;                 // descriptor version (sm_100)
    d |= (uint64_t) 4 << 61;                 // SWIZZLE_64B
    return d;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 2^e as a double: built from the exponent bits in the normal range (exact),
// ldexp outside it.
__device__ __forceinline__ double pow2(int e)
{
    if (e >= -1022 && e <= 1023) return __longlong_as_double((long long) (e + 1023) << 52);
    return ldexp(1.0, e);
}

__device__ __forceinline__ int find_group(const OzGroup *g, int n, int tile)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (g[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void group_tile(const OzGroup &p, int tile, int &tm, int &tn)
{
    int t = tile - p.tile_begin;
    int gs = GROUP_M * p.tiles_n;
    int first = (t / gs) * GROUP_M;
    int gm = min(p.tiles_m - first, GROUP_M);
    int r = t % gs;
    tm = first + r % gm;
    tn = r / gm;
}

__global__ void __launch_bounds__(OTHREADS, 1)
oz_gemm_kernel(const CUtensorMap *__restrict__ tmaps, const OzGroup *__restrict__ groups,
               int ngroup, int total_tiles, int slices, int nstage, const int *__restrict__ ework,
               int *status, unsigned long long limit_ns)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int a_bytes = slices * A_SLICE_BYTES;
    const int stage_bytes = slices * (A_SLICE_BYTES + B_SLICE_BYTES);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + nstage * stage_bytes);
    uint64_t *empty = full + nstage;
    uint64_t *acc_full = empty + nstage;
    uint64_t *acc_empty = acc_full + 1;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tmem_cols = slices * OBN <= 256 ? 256u : 512u;
    if (threadIdx.x == 0) {
        for (int s = 0; s < nstage; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, 4);
        abort_flag = 0;
        fence_barrier_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(tmem_cols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = tmem_slot;

    if (warp == 0) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            uint32_t it = 0;
            int last_g = -1;
            for (int tile = blockIdx.x; tile < total_tiles && !abort_flag; tile += gridDim.x) {
                const int gi = find_group(groups, ngroup, tile);
                const OzGroup &p = groups[gi];
                const CUtensorMap *ta = tmaps + p.a_blk, *tb = tmaps + p.b_blk;
                if (gi != last_g) {
                    tmap_acquire(ta);
                    tmap_acquire(tb);
                    last_g = gi;
                }
                int tm, tn;
                group_tile(p, tile, tm, tn);
                const int kblocks = (p.k + OKB - 1) / OKB;
                bool ok = true;
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const uint32_t s = it % nstage, ph = (it / nstage) & 1u;
                    if (!mbar_wait_bounded(&empty[s], ph ^ 1u, &abort_flag, status,
                                           CA3DMM_DEV_TIMEOUT_PRODUCE, limit_ns)) {
                        ok = false;
                        break;
                    }
                    uint8_t *sA = smem + s * stage_bytes;
                    mbar_arrive_expect_tx(&full[s], stage_bytes);
                    tma_load_3d(sA, ta, kb * OKB, tm * OBM, 0, &full[s]);
                    tma_load_3d(sA + a_bytes, tb, kb * OKB, tn * OBN, 0, &full[s]);
                }
                if (!ok) break;
            }
            // drain copies in flight (bounded, abort flag ignored)
            const uint32_t first = it > (uint32_t) nstage ? it - nstage : 0;
            for (uint32_t L = first; L < it; ++L) {
                uint64_t t0 = global_timer_ns();
                while (!mbar_try_wait(&full[L % nstage], (L / nstage) & 1u))
                    if (global_timer_ns() - t0 > limit_ns) break;
            }
        }
    } else if (warp == 1) {
        // ---------------------------------------------------------- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) |
                                   ((uint32_t) (OBN >> 3) << 17) | ((uint32_t) (OBM >> 4) << 24);
            uint32_t it = 0, ti = 0;
            bool ok = true;
            for (int tile = blockIdx.x; tile < total_tiles && ok; tile += gridDim.x, ++ti) {
                const OzGroup &p = groups[find_group(groups, ngroup, tile)];
                if (!mbar_wait_bounded(acc_empty, (ti & 1u) ^ 1u, &abort_flag, status,
                                       CA3DMM_DEV_TIMEOUT_ACCUM, limit_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const int kblocks = (p.k + OKB - 1) / OKB;
                for (int kb = 0; kb < kblocks; ++kb, ++it) {
                    const uint32_t s = it % nstage, ph = (it / nstage) & 1u;
                    if (!mbar_wait_bounded(&full[s], ph, &abort_flag, status,
                                           CA3DMM_DEV_TIMEOUT_CONSUME, limit_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sA = smem_u32(smem + s * stage_bytes);
                    const uint32_t sB = sA + a_bytes;
#pragma unroll
                    for (int ks = 0; ks < OKB / 32; ++ks) {
                        for (int t = 0; t < slices; ++t) {
                            const uint64_t ad = sdesc_k64(sA + t * A_SLICE_BYTES + ks * 32);
                            for (int u = 0; u + t < slices; ++u) {
                                const uint64_t bd = sdesc_k64(sB + u * B_SLICE_BYTES + ks * 32);
                                const uint32_t acc = (kb > 0 || ks > 0 || t > 0) ? 1u : 0u;
                                tc_mma_i8(tmem_base + (uint32_t) ((t + u) * OBN), ad, bd, idesc,
                                          acc);
                            }
                        }
                    }
                    tc_commit(&empty[s]);
                }
                if (!ok) break;
                tc_commit(acc_full);
            }
            if (!ok) {
                // let every MMA already issued finish before TMEM is freed
                tc_commit(acc_full);
                uint64_t t0 = global_timer_ns();
                while (!mbar_try_wait(acc_full, ti & 1u))
                    if (global_timer_ns() - t0 > limit_ns) break;
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- epilogue
        const int q = warp & 3;                       // TMEM lane quarter of this warp
        const int row = q * 32 + lane;
        uint32_t ti = 0;
        for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x, ++ti) {
            const OzGroup &p = groups[find_group(groups, ngroup, tile)];
            int tm, tn;
            group_tile(p, tile, tm, tn);
            if (!mbar_wait_bounded(acc_full, ti & 1u, &abort_flag, status, CA3DMM_DEV_TIMEOUT_EPI,
                                   limit_ns))
                break;
            tc_fence_after();
            const int gr = tm * OBM + row;
            const int ebase = gr < p.m ? ework[p.ea_off + gr] : 0;
            const int Ei = ebase ? ebase - EXP_BIAS : 0;
            for (int c0 = 0; c0 < OBN; c0 += 16) {
                double acc[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) acc[j] = 0.0;
                int Fj[16];
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int gc = tn * OBN + c0 + j;
                    const int fb = gc < p.n ? ework[p.eb_off + gc] : 0;
                    Fj[j] = fb ? fb - EXP_BIAS : 0;
                }
                for (int d = slices - 1; d >= 0; --d) {
                    uint32_t v[16];
                    tmem_ld16(tmem_base + ((uint32_t) (q * 32) << 16) + (uint32_t) (d * OBN + c0), v);
                    if (p.k > 0) {
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            // |v| < 2^31, so v * 2^e is exact unless it leaves the
                            // normal range, where ldexp rounds it once
                            const int e = Ei + Fj[j] - 12 - 7 * d;
                            const double x = (double) (int) v[j];
                            acc[j] += (e >= -1022 + 31 && e <= 1023 - 31) ? x * pow2(e)
                                                                          : ldexp(x, e);
                        }
                    }
                }
                if (gr < p.m) {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int gc = tn * OBN + c0 + j;
                        if (gc < p.n) p.C[(long long) gr + (long long) gc * p.ldc] = acc[j];
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(acc_empty);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(tmem_cols)
                     : "memory");
    }
}

typedef CUresult (*encode_tiled_fn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                    const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                    const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                    CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

encode_tiled_fn get_encode()
{
    static encode_tiled_fn fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
                cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return nullptr;
        fn = reinterpret_cast<encode_tiled_fn>(p);
    }
    return fn;
}

// 3D map over one block's slices: dims {kz bytes, rows, slices}.
int encode_slices(CUtensorMap *tm, const void *base, int kz, int rows, int kpad, int slices,
                  int box_rows)
{
    encode_tiled_fn enc = get_encode();
    if (!enc) return CA3DMM_ENODEV;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (kpad & 15)) return CA3DMM_EINVAL;
    cuuint64_t dims[3] = {(cuuint64_t) kz, (cuuint64_t) rows, (cuuint64_t) slices};
    cuuint64_t strides[2] = {(cuuint64_t) kpad, (cuuint64_t) kpad * (cuuint64_t) rows};
    cuuint32_t box[3] = {(cuuint32_t) OKB, (cuuint32_t) box_rows, (cuuint32_t) slices};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, const_cast<void *>(base), dims, strides,
                     box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? CA3DMM_OK : CA3DMM_EINVAL;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }
int kpad_of(int kz) { return (kz + OKB - 1) / OKB * OKB; }


// Device plan layout for g groups (at most 2g operand blocks):
// [header 256 B][2g slice descriptors][2g tensor maps, 64-byte aligned][g groups]
struct PlanLayout {
    size_t sd, tm, gr, total;
    explicit PlanLayout(int g)
    {
        sd = 256;
        tm = (sd + (size_t) 2 * g * sizeof(SliceDesc) + 127) / 128 * 128;
        gr = tm + (size_t) 2 * g * sizeof(CUtensorMap);
        total = gr + (size_t) g * sizeof(OzGroup);
    }
};

}  // namespace

extern "C" size_t ca3dmm_oz_plan_bytes(int ngroup) { return PlanLayout(ngroup).total; }

extern "C" size_t ca3dmm_oz_work_bytes(int nA, const int *a_rows, const int *a_k, int nB,
                                       const int *b_k, const int *b_cols, int slices)
{
    size_t e = 0, q = 0;
    for (int i = 0; i < nA; ++i) {
        e += (size_t) a_rows[i];
        q += align256((size_t) slices * a_rows[i] * kpad_of(a_k[i] > 0 ? a_k[i] : 1));
    }
    for (int i = 0; i < nB; ++i) {
        e += (size_t) b_cols[i];
        q += align256((size_t) slices * b_cols[i] * kpad_of(b_k[i] > 0 ? b_k[i] : 1));
    }
    return align256(e * sizeof(int)) + q + 256;
}

extern "C" int ca3dmm_oz_plan_encode(ca3dmm_oz_plan_t *oz, int slices, int nA,
                                     const ca3dmm_oz_blk_t *A, int nB, const ca3dmm_oz_blk_t *B,
                                     int ngroup, const ca3dmm_oz_group_t *G, long long ldA,
                                     int transA, long long ldB, int transB, void *dev_work,
                                     size_t work_bytes, void *host_plan, void *dev_plan)
{
    if (slices < 2 || slices > MAX_SLICES || nA + nB > 2 * ngroup) return CA3DMM_EINVAL;
    const PlanLayout L(ngroup);
    unsigned char *h = static_cast<unsigned char *>(host_plan);
    memset(h, 0, L.total);
    PlanHeader *hd = reinterpret_cast<PlanHeader *>(h);
    SliceDesc *sd = reinterpret_cast<SliceDesc *>(h + L.sd);
    CUtensorMap *tm = reinterpret_cast<CUtensorMap *>(h + L.tm);
    OzGroup *gr = reinterpret_cast<OzGroup *>(h + L.gr);
    unsigned char *w = static_cast<unsigned char *>(dev_work);
    // exponents first: one int array, cleared before each run
    size_t ne = 0;
    for (int i = 0; i < nA; ++i) ne += A[i].rows;
    for (int i = 0; i < nB; ++i) ne += B[i].cols;
    size_t qoff = align256(ne * sizeof(int));
    long long eoff = 0;
    int max_rows = 1, max_kpad = 1;
    for (int i = 0; i < nA + nB; ++i) {
        const bool isA = i < nA;
        const ca3dmm_oz_blk_t &b = isA ? A[i] : B[i - nA];
        const int rows = isA ? b.rows : b.cols;   // A: rows of op(A); B: columns of op(B)
        const int kz = isA ? b.cols : b.rows;
        const int kpad = kpad_of(kz > 0 ? kz : 1);
        SliceDesc &d = sd[i];
        d.rows = rows;
        d.kz = kz;
        d.kpad = kpad;
        d.q_off = (long long) qoff;
        d.e_off = eoff;
        if (isA) {
            // op(A)(r, l) = transA ? A[l + r ldA] : A[r + l ldA]; block at (b.r0, b.c0)
            d.rs = transA ? ldA : 1;
            d.ls = transA ? 1 : ldA;
            d.src_off = (long long) b.r0 * d.rs + (long long) b.c0 * d.ls;
        } else {
            // column j of op(B) over l: transB ? B[j + l ldB] : B[l + j ldB]; block at (l0 = b.r0, j0 = b.c0)
            d.rs = transB ? 1 : ldB;
            d.ls = transB ? ldB : 1;
            d.src_off = (long long) b.c0 * d.rs + (long long) b.r0 * d.ls;
        }
        if (rows > 0 && kz > 0) {
            int rc = encode_slices(&tm[i], w + qoff, kz, rows, kpad, slices, isA ? OBM : OBN);
            if (rc) return rc;
        }
        qoff += align256((size_t) slices * rows * kpad);
        eoff += rows;
        if (rows > max_rows) max_rows = rows;
        if (kpad > max_kpad) max_kpad = kpad;
    }
    if (qoff > work_bytes) return CA3DMM_ENOMEM;
    int tiles = 0;
    for (int g = 0; g < ngroup; ++g) {
        OzGroup &o = gr[g];
        o.C = G[g].C; o.ldc = G[g].ldc;
        o.m = G[g].m; o.n = G[g].n; o.k = G[g].k;
        if ((long long) G[g].k * slices >= (1LL << 19)) {
            fprintf(stderr, "[ERROR] split-precision GEMM: k = %d with %d slices exceeds the exact "
                            "INT32 range (k * slices < 2^19); use more k slabs\n", G[g].k, slices);
            return CA3DMM_EINVAL;
        }
        o.a_blk = G[g].a_blk;
        o.b_blk = nA + G[g].b_blk;
        o.ea_off = sd[o.a_blk].e_off;
        o.eb_off = sd[o.b_blk].e_off;
        o.tiles_m = (o.m > 0 && o.n > 0) ? (o.m + OBM - 1) / OBM : 0;
        o.tiles_n = (o.m > 0 && o.n > 0) ? (o.n + OBN - 1) / OBN : 0;
        o.tile_begin = tiles;
        tiles += o.tiles_m * o.tiles_n;
    }
    hd->nA = nA; hd->nB = nB; hd->ngroup = ngroup; hd->slices = slices;
    hd->nslice_desc = nA + nB; hd->tiles = tiles;
    oz->slices = slices; oz->nA = nA; oz->nB = nB; oz->ngroup = ngroup; oz->tiles = tiles;
    oz->max_rows = max_rows; oz->max_kpad = max_kpad;
    oz->n_exp = (long long) ne;
    oz->dev_plan = dev_plan;
    oz->dev_work = dev_work;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_oz_run_pack(const ca3dmm_oz_plan_t *oz, const void *A, const void *B,
                                  cudaStream_t stream)
{
    const PlanLayout L(oz->ngroup);
    const SliceDesc *sd =
        reinterpret_cast<const SliceDesc *>(static_cast<const unsigned char *>(oz->dev_plan) + L.sd);
    unsigned char *w = static_cast<unsigned char *>(oz->dev_work);
    CA3DMM_CUDA_TRY(cudaMemsetAsync(w, 0, (size_t) oz->n_exp * sizeof(int), stream));
    const int nd = oz->nA + oz->nB;
    dim3 ge((unsigned) ((oz->max_rows + ST - 1) / ST), (unsigned) ((oz->max_kpad + ST - 1) / ST),
            (unsigned) nd);
    if (ge.y > 65535 || nd > 65535) return CA3DMM_EINVAL;
    // A blocks then B blocks: the kernels read their source from the right base
    if (oz->nA > 0) {
        dim3 ga(ge.x, ge.y, (unsigned) oz->nA);
        oz_exp_kernel<<<ga, 256, 0, stream>>>(static_cast<const double *>(A), sd,
                                              reinterpret_cast<unsigned *>(w));
        CA3DMM_CUDA_TRY(cudaGetLastError());
    }
    if (oz->nB > 0) {
        dim3 gb(ge.x, ge.y, (unsigned) oz->nB);
        oz_exp_kernel<<<gb, 256, 0, stream>>>(static_cast<const double *>(B), sd + oz->nA,
                                              reinterpret_cast<unsigned *>(w));
        CA3DMM_CUDA_TRY(cudaGetLastError());
    }
    if (oz->nA > 0) {
        dim3 ga(ge.x, ge.y, (unsigned) oz->nA);
        oz_slice_kernel<<<ga, 256, 0, stream>>>(static_cast<const double *>(A), sd, w, oz->slices);
        CA3DMM_CUDA_TRY(cudaGetLastError());
    }
    if (oz->nB > 0) {
        dim3 gb(ge.x, ge.y, (unsigned) oz->nB);
        oz_slice_kernel<<<gb, 256, 0, stream>>>(static_cast<const double *>(B), sd + oz->nA, w,
                                                oz->slices);
        CA3DMM_CUDA_TRY(cudaGetLastError());
    }
    return CA3DMM_OK;
}

extern "C" int ca3dmm_oz_run_gemm(const ca3dmm_oz_plan_t *oz, int *dev_status, double timeout_s,
                                  cudaStream_t stream)
{
    if (oz->tiles <= 0) return CA3DMM_OK;
    const PlanLayout L(oz->ngroup);
    const unsigned char *pl = static_cast<const unsigned char *>(oz->dev_plan);
    const int stage_bytes = oz->slices * (A_SLICE_BYTES + B_SLICE_BYTES);
    int nstage = SMEM_BUDGET / stage_bytes;
    if (nstage > 4) nstage = 4;
    if (nstage < 2) return CA3DMM_EINVAL;
    const size_t smem = (size_t) nstage * stage_bytes + (2 * nstage + 2) * 8 + 1024;
    CA3DMM_CUDA_TRY(cudaFuncSetAttribute(oz_gemm_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    int grid = ca3dmm_device_sm_count();
    if (grid > oz->tiles) grid = oz->tiles;
    const unsigned long long limit = (unsigned long long) (timeout_s * 1e9);
    oz_gemm_kernel<<<grid, OTHREADS, smem, stream>>>(
        reinterpret_cast<const CUtensorMap *>(pl + L.tm),
        reinterpret_cast<const OzGroup *>(pl + L.gr), oz->ngroup, oz->tiles, oz->slices, nstage,
        static_cast<const int *>(oz->dev_work), dev_status, limit);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    return CA3DMM_OK;
}
