// Split-precision FP64 GEMM (Ozaki scheme with INT8 slices) for sm_100a.
//
//  1. oz_exp_kernel    -- per row of op(A) / column of op(B) over the block's k
//                         range: E = frexp exponent of max|x| (max|x| < 2^E).
//  2. slice_kc/rc_kernel<SliceWriter<S>> -- x = sum_t q_t 2^(E-7-8t) + r with |r| <= 2^(E-8s): the
//                         integer N = rint(x 2^(8s-1-E)) written in balanced
//                         base-256 digits q_t in [-128, 127] (E chosen so that
//                         max|x| <= 2^E 127/128, which keeps the top digit in range).
//                         The slices are written straight into the GEMM's shared
//                         memory image: per 128-row (A) / 64-row (B) tile and
//                         32-byte k-block, the s slices are contiguous, each a
//                         K-major rows x 32-byte tile with the 32-byte swizzle
//                         (16-byte chunk ^= (row >> 2) & 1) already applied.
//                         HBM-bound; reads k-contiguous sources with 16-byte
//                         loads per thread, transposes rows-contiguous ones
//                         through shared memory.
//  3. oz_gemm_kernel   -- tcgen05.mma kind::i8 (signed x signed), M=128 x K=32,
//                         N = 64 per slice pair, up to four pairs of one A slice
//                         fused into one N <= 256 MMA.  All s diagonal accumulators
//                         D_d = sum_{t+u=d} Aq_t Bq_u^T live in TMEM at once
//                         (s*64 <= 512 columns), so each 32-byte k-block of every
//                         slice is brought in once -- two contiguous bulk copies
//                         per stage -- and feeds all s(s+1)/2 slice products.
//                         The k range is processed in chunks short enough for the
//                         INT32 sums to stay exact (s kc 2^14 < 2^31); after each
//                         chunk the epilogue adds 2^(-14-8d) D_d, d = s-1 down
//                         to 0, into FP64 registers, and stores 2^(E_i+F_j) times
//                         that sum after the last chunk.
//  4. oz_nonfinite_kernel -- rows / columns holding an Inf or a NaN were sliced as
//                         zero rows; writes the IEEE value of their C entries.
// Warp roles of the GEMM: warp 0 copy producer, warps 1, 6, 7 MMA issuers, each
// owning a set of A slices (warp 1 also owns the TMEM allocation), warps 2..5
// and 8..11 epilogue (warp w reads TMEM lanes 32*(w%4)..+31, columns 0-31 of
// each 64-column accumulator for w <= 5, 32-63 for w >= 8: two warps per lane
// quarter halve the time the MMAs wait for the accumulators to drain).  Each issuing thread needs
// ~150-190 cycles per tcgen05.mma, so one issuer cannot keep the tensor core
// busy; the A slices are dealt out so that no issuer has more than four MMAs
// per k-block (s <= 8).  Issuers of different slices add into
// the same diagonal accumulators, so every MMA accumulates and the epilogue
// zeroes each accumulator after reading it.  All waits are bounded; on
// timeout the kernel records a status, drains, frees TMEM, returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <climits>
#include <cstdio>
#include <cstring>
#include "k_common.cuh"
#include "k_split.cuh"
#include "ca3dmm_kernels.h"
#include "ca3dmm_ozaki.h"

extern "C" int ca3dmm_encode_tmap_2d(void *tmap, int dtype_bytes, const void *base,
                                     unsigned long long dim0, unsigned long long dim1,
                                     unsigned long long stride1_bytes, unsigned box0,
                                     unsigned box1, int swizzle128);
extern "C" int ca3dmm_encode_tmap_u8(void *tmap, int rank, const void *base,
                                     const unsigned long long *dims,
                                     const unsigned long long *strides_bytes,
                                     const unsigned *box);

namespace {

constexpr int OBM = 128, OBN = 64, OKB = 32;    // tile rows, tile cols, k bytes per stage
constexpr int OTHREADS = 384;                    // 12 warps
constexpr int EPI_WARPS = 8;                     // two per TMEM lane quarter
constexpr int MAX_ISSUERS = 3;                   // MMA issuer warps 1, 6, 7
constexpr int MAX_SLICES = 8;
constexpr int MAX_STAGES = 8;
constexpr int A_SLICE_BYTES = OBM * OKB;        // 4 KiB
constexpr int B_SLICE_BYTES = OBN * OKB;        // 2 KiB
constexpr int SMEM_BUDGET = 200 * 1024;
constexpr int GROUP_M = 8;

struct OzGroup {
    double *C;
    long long ldc;
    int m, n, k;
    int nkb;                    // 32-byte k-blocks
    int tiles_m, tiles_n, tile_begin, raster;
    int a_from_b;               // A slices stored in the B layout (64-row tiles): B^T B
    int a_tmap;                 // a_from_b: the group's 5D tensor map gathers a whole A stage
    long long ea_off, eb_off;   // exponent offsets (ints) of the A rows / B columns
    long long qa_off, qb_off;   // byte offsets of the tiled slices
    int a_desc, b_desc;         // slicing descriptors of the operand blocks (A: a B block when aliased)
    int row0, col0;             // first row / column of the group inside those blocks
};

// A work unit is a chain of nsub groups (group, group + sub_stride, ...) that
// write the same C block: the kp k-slabs of one (task_m, task_n) block.  Its
// tiles are numbered once and every CTA owns a fixed set of tile numbers; the
// CTA runs all its tiles for slab 0 (storing C), then all for slab 1 (adding
// to the C it wrote), and so on -- the reference's slab-sum order, with the
// operand locality of slab-by-slab processing.
struct OzUnit {
    int tile_begin, tiles_m, tiles_n, raster;
    int group, nsub, sub_stride, pad;
};

struct PlanHeader {
    int nA, nB, ngroup, slices;
    int nslice_desc, tiles, nunit, pad1;
};

// Pass 2 for one (row, 16 consecutive k): N = rint(x 2^(8S-1-E)) per element;
// the balanced digits q_t in [-128, 127] of N (least significant first:
// q = ((N + 128) mod 256) - 128, N = (N - q) / 256) are exactly the bytes of
// N + 0x80..80 (S bytes of 0x80) with the top bit flipped, because adding 128
// to every digit of a balanced representation gives the unsigned base-256
// representation of N + 0x80..80 (|N| < 2^(8S-1) 127/128 keeps it in range).
// Slice t holds digit S-1-t.  The 16 bytes of each slice are gathered with
// byte permutes and stored with the 32-byte swizzle of the GEMM's operand tile.
template <int S>
__device__ __forceinline__ void slice16(const SliceDesc &d, unsigned char *__restrict__ work,
                                        const unsigned long long *__restrict__ mwork, int gr,
                                        int gl, const double (&x)[16])
{
    // a row holding an Inf or a NaN is sliced as a zero row; oz_nonfinite_kernel
    // writes the IEEE result of its C entries after the GEMM
    const unsigned long long mr = gr < d.rows ? mwork[d.e_off + gr] : 0ull;
    const bool fin = mr < INF_BITS;
    const unsigned long long mb = fin ? mr : 0ull;
    int E = 0;
    if (mb) {
        int ex;
        const double mant = frexp(__longlong_as_double((long long) mb), &ex);
        E = ex + (mant > 0.9921875 ? 1 : 0);
    }
    if (gl == 0 && gr < d.rows) reinterpret_cast<int *>(work)[d.e_off + gr] = mb ? E + EXP_BIAS : 0;
    // x 2^(8S-1-E) as two exact power-of-two factors (each inside the normal range)
    const int sh = 8 * S - 1 - E;
    const double up1 = ldexp(1.0, sh / 2), up2 = ldexp(1.0, sh - sh / 2);
    constexpr unsigned long long BIAS = 0x8080808080808080ull >> (64 - 8 * S);
    uint32_t lo[16], hi[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const long long N = __double2ll_rn((fin ? x[j] : 0.0) * up1 * up2);
        const unsigned long long U = (unsigned long long) N + BIAS;
        lo[j] = (uint32_t) U;
        hi[j] = (uint32_t) (U >> 32);
    }
    const int rt = gr / d.tile_rows, rr = gr % d.tile_rows;
    const int kb = gl / OKB, chunk = (gl % OKB) >> 4;
    const long long tile_bytes = (long long) d.tile_rows * OKB;
    unsigned char *dst = work + d.q_off + ((long long) rt * d.nkb + kb) * S * tile_bytes +
                         rr * OKB + ((chunk ^ ((rr >> 2) & 1)) << 4);
#pragma unroll
    for (int t = 0; t < S; ++t) {
        const int b = S - 1 - t, bb = b & 3;
        const uint32_t *w = b < 4 ? lo : hi;
        const uint32_t sel = (uint32_t) bb | ((uint32_t) (bb + 4) << 4);
        uint32_t out[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t p01 = __byte_perm(w[4 * q], w[4 * q + 1], sel);
            const uint32_t p23 = __byte_perm(w[4 * q + 2], w[4 * q + 3], sel);
            out[q] = __byte_perm(p01, p23, 0x5410) ^ 0x80808080u;
        }
        *reinterpret_cast<uint4 *>(dst + t * tile_bytes) = make_uint4(out[0], out[1], out[2], out[3]);
    }
}

template <int S>
struct SliceWriter {
    static constexpr int kMinBlocks = 4;
    static __device__ __forceinline__ void write16(const SliceDesc &d, unsigned char *__restrict__ work,
                                                   const unsigned long long *__restrict__ mwork,
                                                   int gr, int gl, const double (&x)[16])
    {
        slice16<S>(d, work, mwork, gr, gl, x);
    }
};

// ------------------------------------------------------------------ tcgen05 GEMM
// The unit holding tile `tile`.  sb: a shared-memory copy of the units' first
// tiles (nullptr when there are more than UNIT_CACHE units), so that a batch of
// small GEMMs does not pay a chain of dependent global loads per tile.
constexpr int UNIT_CACHE = 1024;
__device__ __forceinline__ int find_unit(const int *sb, const OzUnit *u, int n, int tile)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if ((sb ? sb[mid] : u[mid].tile_begin) <= tile) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void unit_tile(const OzUnit &p, int tile, int &tm, int &tn)
{
    int t = tile - p.tile_begin;
    int gs = p.raster * p.tiles_n;
    int first = (t / gs) * p.raster;
    int gm = min(p.tiles_m - first, p.raster);
    int r = t % gs;
    tm = first + r % gm;
    tn = r / gm;
}

// number of exactly-accumulated k chunks of a tile with nkb k-blocks
__device__ __forceinline__ int nchunks(int nkb, int kb_per_chunk)
{
    return nkb > 0 ? (nkb + kb_per_chunk - 1) / kb_per_chunk : 1;
}

// The slice count is a template parameter: with compile-time loops the MMA
// descriptors of a k-block are formed without per-MMA loop bookkeeping, which
// measured 1.45x faster than the same loops over a runtime count.
template <int S>
__global__ void __launch_bounds__(OTHREADS, 1)
oz_gemm_kernel(const OzGroup *__restrict__ groups, const OzUnit *__restrict__ units,
               const unsigned char *__restrict__ tmaps, int nunit,
               int nsub_max, const ca3dmm_tile_ranges_t rg,
               int total_tiles, int nstage,
               int kb_per_chunk, int4 tsplit, const unsigned char *__restrict__ work,
               int *status, unsigned long long limit_ns)
{
    constexpr int slices = S;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int a_bytes = slices * A_SLICE_BYTES;
    const int b_bytes = slices * B_SLICE_BYTES;
    const int stage_bytes = a_bytes + b_bytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + nstage * stage_bytes);
    uint64_t *empty = full + nstage;
    uint64_t *acc_full = empty + nstage;
    uint64_t *acc_empty = acc_full + 1;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    __shared__ int col_exp_all[OTHREADS / 32][32];      // F_j per epilogue warp (no cross-warp barrier)
    __shared__ int s_ubeg[UNIT_CACHE];
    const int *ework = reinterpret_cast<const int *>(work);
    const int *ub = nunit <= UNIT_CACHE ? s_ubeg : nullptr;
    if (ub)
        for (int i = threadIdx.x; i < nunit; i += blockDim.x) s_ubeg[i] = units[i].tile_begin;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t tmem_cols = slices * OBN <= 256 ? 256u : 512u;
    if (threadIdx.x == 0) {
        for (int s = 0; s < nstage; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], MAX_ISSUERS);     // one commit per MMA issuer
        }
        mbar_init(acc_full, MAX_ISSUERS);
        mbar_init(acc_empty, EPI_WARPS);
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
    // the MMAs only ever accumulate: the epilogue warps clear the accumulators
    // here and again after draining each chunk
    if (warp >= 2 && warp <= 5) {
        const uint32_t lane_base = (uint32_t) ((warp & 3) * 32) << 16;
        for (int c = 0; c < slices * OBN; c += 32) tmem_zero32(tmem_base + lane_base + (uint32_t) c);
        tmem_wait_st();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    if (warp == 0) {
        // ---------------------------------------------------------- producer
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            int last_g = -1;
          for (int sub = 0; sub < nsub_max && ok; ++sub)
            for (int v = blockIdx.x; v < total_tiles && ok && !abort_flag; v += gridDim.x) {
                const int tile = range_tile(rg, v);
                const OzUnit &U = units[find_unit(ub, units, nunit, tile)];
                int tm, tn;
                unit_tile(U, tile, tm, tn);
              if (sub < U.nsub) {
                const int gi = U.group + sub * U.sub_stride;
                const OzGroup &p = groups[gi];
                const unsigned char *tm5 = tmaps + (size_t) gi * 128;
                if (p.a_tmap && gi != last_g) {
                    tmap_acquire(tm5);
                    last_g = gi;
                }
                const unsigned char *qa =
                    p.a_from_b ? work + p.qa_off + (long long) (2 * tm) * p.nkb * b_bytes
                               : work + p.qa_off + (long long) tm * p.nkb * a_bytes;
                const unsigned char *qb =
                    work + p.qb_off + (long long) tn * p.nkb * b_bytes;
                for (int kb = 0; kb < p.nkb; ++kb, ++it) {
                    const uint32_t s = it % nstage, ph = (it / nstage) & 1u;
                    if (!mbar_wait_bounded(&empty[s], ph ^ 1u, &abort_flag, status,
                                           CA3DMM_DEV_TIMEOUT_PRODUCE, limit_ns)) {
                        ok = false;
                        break;
                    }
                    uint8_t *sA = smem + s * stage_bytes;
                    mbar_arrive_expect_tx(&full[s], stage_bytes);
                    if (p.a_tmap) {
                        tma_load_5d(sA, tm5, 0, 0, 2 * tm, 0, kb, &full[s]);
                    } else if (p.a_from_b) {
                        // rows 0-63 / 64-127 of each A slice: the same slice of the
                        // 64-row tiles 2 tm and 2 tm + 1 of the B layout
                        const unsigned char *h0 = qa + (long long) kb * b_bytes;
                        const unsigned char *h1 = h0 + (long long) p.nkb * b_bytes;
                        for (int t = 0; t < slices; ++t) {
                            bulk_load(sA + t * A_SLICE_BYTES, h0 + t * B_SLICE_BYTES,
                                      B_SLICE_BYTES, &full[s]);
                            bulk_load(sA + t * A_SLICE_BYTES + B_SLICE_BYTES,
                                      h1 + t * B_SLICE_BYTES, B_SLICE_BYTES, &full[s]);
                        }
                    } else {
                        bulk_load(sA, qa + (long long) kb * a_bytes, a_bytes, &full[s]);
                    }
                    bulk_load(sA + a_bytes, qb + (long long) kb * b_bytes, b_bytes, &full[s]);
                }
              }
            }
            // drain copies in flight (bounded, abort flag ignored)
            const uint32_t first = it > (uint32_t) nstage ? it - nstage : 0;
            for (uint32_t L = first; L < it; ++L) {
                uint64_t t0 = global_timer_ns();
                while (!mbar_try_wait(&full[L % nstage], (L / nstage) & 1u))
                    if (global_timer_ns() - t0 > limit_ns) break;
            }
        }
    } else if (warp == 1 || warp == 6 || warp == 7) {
        // ---------------------------------------------------------- MMA issuers
        if (lane == 0) {
            // this issuer's A slices (bit t of the mask; possibly none: an idle
            // issuer still commits, keeping the barrier counts)
            const int ii = warp == 1 ? 0 : warp - 5;
            const unsigned tmask = (unsigned) (ii == 0 ? tsplit.x : (ii == 1 ? tsplit.y : tsplit.z));
            uint32_t it = 0, ci = 0;
            bool ok = true;
          for (int sub = 0; sub < nsub_max && ok; ++sub)
            for (int v = blockIdx.x; v < total_tiles && ok; v += gridDim.x) {
                const OzUnit &U = units[find_unit(ub, units, nunit, range_tile(rg, v))];
              if (sub < U.nsub) {
                const OzGroup &p = groups[U.group + sub * U.sub_stride];
                const int nch = nchunks(p.nkb, kb_per_chunk);
                for (int ch = 0; ch < nch && ok; ++ch, ++ci) {
                    if (!mbar_wait_bounded(acc_empty, (ci & 1u) ^ 1u, &abort_flag, status,
                                           CA3DMM_DEV_TIMEOUT_ACCUM, limit_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const int kb0 = ch * kb_per_chunk;
                    const int kb1 = min(p.nkb, kb0 + kb_per_chunk);
                    (void) kb0;
                    for (int kb = kb0; kb < kb1; ++kb, ++it) {
                        const uint32_t s = it % nstage, ph = (it / nstage) & 1u;
                        if (!mbar_wait_bounded(&full[s], ph, &abort_flag, status,
                                               CA3DMM_DEV_TIMEOUT_CONSUME, limit_ns)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t sA = smem_u32(smem + s * stage_bytes);
                        const uint32_t sB = sA + a_bytes;
                        // For slice t of A the partner slices u = 0 .. s-1-t of B are
                        // adjacent 64-row tiles in shared memory and their
                        // accumulators D_{t+u} adjacent 64-column blocks in TMEM, so
                        // one MMA with N = 64 * (#u) (<= 256) covers up to four slice
                        // products.  Issuers of different A slices add into the same
                        // diagonals; integer accumulation makes the order immaterial.
#pragma unroll
                        for (int t = 0; t < slices; ++t) {
                            if (!((tmask >> t) & 1u)) continue;
                            const uint64_t ad = sdesc_k32(sA + t * A_SLICE_BYTES);
#pragma unroll
                            for (int u = 0; u < slices - t; u += 4) {
                                const int nu = min(4, slices - t - u);
                                const uint64_t bd = sdesc_k32(sB + u * B_SLICE_BYTES);
                                tc_mma_i8(tmem_base + (uint32_t) ((t + u) * OBN), ad, bd,
                                          idesc_i8(nu * OBN), 1u);
                            }
                        }
                        tc_commit(&empty[s]);
                    }
                    if (!ok) break;
                    tc_commit(acc_full);
                }
              }
            }
            if (!ok) {
                // let every MMA this thread issued finish before TMEM is freed
                tc_commit(acc_full);
                uint64_t t0 = global_timer_ns();
                while (!mbar_try_wait(acc_full, ci & 1u))
                    if (global_timer_ns() - t0 > limit_ns) break;
            }
        }
        __syncwarp();
    } else {
        // ---------------------------------------------------------- epilogue
        const int q = warp & 3;                       // TMEM lane quarter of this warp
        const int c0 = warp >= 8 ? 32 : 0;            // its 32 columns of each accumulator
        const int row = q * 32 + lane;
        int *col_exp = col_exp_all[warp];
        uint32_t ci = 0;
        bool ok = true;
      for (int sub = 0; sub < nsub_max && ok; ++sub)
        for (int v = blockIdx.x; v < total_tiles && ok; v += gridDim.x) {
            const int tile = range_tile(rg, v);
            const OzUnit &U = units[find_unit(ub, units, nunit, tile)];
            int tm, tn;
            unit_tile(U, tile, tm, tn);
          if (sub < U.nsub) {
            const OzGroup &p = groups[U.group + sub * U.sub_stride];
            const int gr = tm * OBM + row;
            const int gm = p.m, gn = p.n;
            const long long ldc = p.ldc;
            double *const Cg = p.C;
            const int eb = gr < gm ? ework[p.ea_off + gr] : 0;
            const int Ei = eb ? eb - EXP_BIAS : 0;
            // column exponents F_j of this tile into this warp's shared slots
            __syncwarp();
            {
                const int gc = tn * OBN + c0 + lane;
                const int fb = gc < gn ? ework[p.eb_off + gc] : 0;
                col_exp[lane] = fb ? fb - EXP_BIAS : 0;
            }
            __syncwarp();
            double acc[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) acc[j] = 0.0;
            const int nch = nchunks(p.nkb, kb_per_chunk);
            for (int ch = 0; ch < nch; ++ch, ++ci) {
                if (!mbar_wait_bounded(acc_full, ci & 1u, &abort_flag, status,
                                       CA3DMM_DEV_TIMEOUT_EPI, limit_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                if (p.nkb > 0) {
                    for (int d = slices - 1; d >= 0; --d) {
                        // acc_j += D_d 2^(-14 - 8d), the term exact (|D_d| < 2^31,
                        // power-of-two scale), one rounding per addition; the factor
                        // 2^(E_i + F_j) is applied once at the store (one rounding,
                        // only where the result leaves the normal range), as the
                        // oracle's ldexp(sum_d ldexp(D_d, -14 - 8d), E_i + F_j).
                        const double rs = pow2(-14 - 8 * d);
                        uint32_t v[32];
                        const uint32_t ta = tmem_base + ((uint32_t) (q * 32) << 16) +
                                            (uint32_t) (d * OBN + c0);
                        tmem_ld32(ta, v);
                        tmem_zero32(ta);
#pragma unroll
                        for (int j = 0; j < 32; ++j) acc[j] = fma(i32_to_f64(v[j]), rs, acc[j]);
                    }
                    tmem_wait_st();
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(acc_empty);
            }
            if (!ok) break;
            if (gr < gm) {
                // slab 0 stores; later slabs of the chain add in slab order (this
                // thread wrote the value it reads)
                double *crow = Cg + gr + (long long) (tn * OBN + c0) * ldc;
                const int nj = min(32, gn - tn * OBN - c0);
                if (sub == 0) {
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (j < nj) crow[(long long) j * ldc] = scale2(acc[j], Ei + col_exp[j]);
                } else {
#pragma unroll
                    for (int j0 = 0; j0 < 32; j0 += 8) {
                        double c[8];
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            c[j] = j0 + j < nj ? crow[(long long) (j0 + j) * ldc] : 0.0;
#pragma unroll
                        for (int j = 0; j < 8; ++j)
                            if (j0 + j < nj)
                                crow[(long long) (j0 + j) * ldc] =
                                    c[j] + scale2(acc[j0 + j], Ei + col_exp[j0 + j]);
                    }
                }
            }
          }
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

// ------------------------------------------------------------------ non-finite inputs
// A row of op(A) or a column of op(B) that holds an Inf or a NaN was sliced
// as a zero row, so the GEMM wrote the finite entries of C exactly as without
// it.  Every C entry in such a row or column is non-finite under IEEE
// arithmetic -- each of its products with a non-finite factor is an Inf or a
// NaN -- and which one does not depend on the summation order: NaN when some
// product is NaN (a NaN factor, or Inf times 0) or products of both infinite
// signs occur, else the infinity of the products' sign.  This pass writes that
// value over the tiles of a launch, after the GEMM over the same tiles and
// before any slab sum (which then carries it through IEEE additions).  It
// returns at once when the exponent passes flagged nothing.
constexpr int NF_THREADS = 256;

__global__ void __launch_bounds__(NF_THREADS)
oz_nonfinite_kernel(const double *__restrict__ srcA, const double *__restrict__ srcB,
                    const SliceDesc *__restrict__ descs, int nA, const OzGroup *__restrict__ groups,
                    const OzUnit *__restrict__ units, int nunit, const ca3dmm_tile_ranges_t rg,
                    int total_tiles, const unsigned long long *__restrict__ mwork,
                    const unsigned long long *__restrict__ nonfinite)
{
    if (*nonfinite == 0ull) return;
    __shared__ unsigned char row_bad[OBM], col_bad[OBN];
    for (int v = blockIdx.x; v < total_tiles; v += gridDim.x) {
        const int tile = range_tile(rg, v);
        const OzUnit &U = units[find_unit(nullptr, units, nunit, tile)];
        int tm, tn;
        unit_tile(U, tile, tm, tn);
        const OzGroup &g0 = groups[U.group];
        // rows and columns of this tile flagged in any k-slab of the unit
        __syncthreads();                              // the previous tile's flags are read
        if (threadIdx.x < OBM + OBN) {
            const bool isrow = threadIdx.x < OBM;
            const int idx = isrow ? tm * OBM + threadIdx.x : tn * OBN + threadIdx.x - OBM;
            bool bad = false;
            if (idx < (isrow ? g0.m : g0.n))
                for (int sub = 0; sub < U.nsub; ++sub) {
                    const OzGroup &g = groups[U.group + sub * U.sub_stride];
                    bad = bad || mwork[(isrow ? g.ea_off : g.eb_off) + idx] >= INF_BITS;
                }
            (isrow ? row_bad[threadIdx.x] : col_bad[threadIdx.x - OBM]) = bad ? 1 : 0;
        }
        const int any = __syncthreads_or(threadIdx.x < OBM + OBN &&
                                         (threadIdx.x < OBM ? row_bad[threadIdx.x]
                                                            : col_bad[threadIdx.x - OBM]));
        if (!any) continue;
        for (int e = threadIdx.x; e < OBM * OBN; e += blockDim.x) {
            const int r = e % OBM, c = e / OBM;
            const int i = tm * OBM + r, j = tn * OBN + c;
            if (i >= g0.m || j >= g0.n || !(row_bad[r] || col_bad[c])) continue;
            int cls = 0;
            for (int sub = 0; sub < U.nsub && !(cls & 1); ++sub) {
                const OzGroup &g = groups[U.group + sub * U.sub_stride];
                const unsigned long long ma = mwork[g.ea_off + i], mb = mwork[g.eb_off + j];
                if (ma < INF_BITS && mb < INF_BITS) continue;      // all products finite
                if (ma > INF_BITS || mb > INF_BITS) { cls |= 1; break; }   // a NaN factor
                const SliceDesc &da = descs[g.a_desc], &db = descs[g.b_desc];
                const double *pa = slice_src(g.a_desc < nA ? srcA : srcB, da.src_off) +
                                   (long long) (g.row0 + i) * da.rs;
                const double *pb = slice_src(srcB, db.src_off) + (long long) (g.col0 + j) * db.rs;
                for (int l = 0; l < g.k; ++l)
                    cls |= product_class(__ldg(pa + (long long) l * da.ls),
                                         __ldg(pb + (long long) l * db.ls));
            }
            double out;
            if ((cls & 1) || (cls & 6) == 6) out = __longlong_as_double(0x7ff8000000000000ll);
            else if (cls & 2) out = __longlong_as_double(0x7ff0000000000000ll);
            else if (cls & 4) out = __longlong_as_double((long long) 0xfff0000000000000ull);
            else continue;
            g0.C[i + (long long) j * g0.ldc] = out;
        }
    }
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }
int kpad_of(int kz) { return (kz + OKB - 1) / OKB * OKB; }
int rows_pad_of(int rows, int tr) { return (rows + tr - 1) / tr * tr; }

// k chunk (bytes) over which every diagonal sum stays exact in INT32:
// s * kc * 2^14 < 2^31 (|q| <= 128), rounded down to the 32-byte k step (the
// oracle's orc_ozaki_kchunk uses the same rule).
int kchunk_of(int s) { return (int) ((2147483647L / 16384L) / s / OKB * OKB); }

// A slices of the three MMA issuers (bit masks): slice t needs
// ceil((s - t) / 4) MMAs per k-block; minimise the largest per-issuer MMA count
// (each issuing thread needs ~150-190 cycles per tcgen05.mma), then the spread
// of slice products.
int4 slice_split(int s)
{
    int best_m[3] = {0, 0, 0}, best_instr = 1 << 30, best_gap = 1 << 30;
    int pow3 = 1;
    for (int t = 0; t < s; ++t) pow3 *= 3;
    for (int code = 0; code < pow3; ++code) {
        int m[3] = {0, 0, 0}, n[3] = {0, 0, 0}, u[3] = {0, 0, 0}, c = code;
        for (int t = 0; t < s; ++t, c /= 3) {
            const int w = c % 3;
            m[w] |= 1 << t;
            n[w] += (s - t + 3) / 4;
            u[w] += s - t;
        }
        const int mi = n[0] > n[1] ? (n[0] > n[2] ? n[0] : n[2]) : (n[1] > n[2] ? n[1] : n[2]);
        const int umax = u[0] > u[1] ? (u[0] > u[2] ? u[0] : u[2]) : (u[1] > u[2] ? u[1] : u[2]);
        const int umin = u[0] < u[1] ? (u[0] < u[2] ? u[0] : u[2]) : (u[1] < u[2] ? u[1] : u[2]);
        if (mi < best_instr || (mi == best_instr && umax - umin < best_gap)) {
            best_instr = mi;
            best_gap = umax - umin;
            best_m[0] = m[0]; best_m[1] = m[1]; best_m[2] = m[2];
        }
    }
    return make_int4(best_m[0], best_m[1], best_m[2], 0);
}

// Device plan layout for g groups (at most 2g operand blocks, g units):
// [header 256 B][2g slice descriptors][g groups][g units]
struct PlanLayout {
    size_t sd, gr, un, tm, total;
    explicit PlanLayout(int g)
    {
        sd = 256;
        gr = (sd + (size_t) 2 * g * sizeof(SliceDesc) + 127) / 128 * 128;
        un = (gr + (size_t) g * sizeof(OzGroup) + 127) / 128 * 128;
        tm = (un + (size_t) g * sizeof(OzUnit) + 127) / 128 * 128;
        total = tm + (size_t) g * 128;          // one 128-byte tensor map per group
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
        q += align256((size_t) slices * rows_pad_of(a_rows[i], OBM) *
                      kpad_of(a_k[i] > 0 ? a_k[i] : 1));
    }
    for (int i = 0; i < nB; ++i) {
        e += (size_t) b_cols[i];
        q += align256((size_t) slices * rows_pad_of(b_cols[i], OBN) *
                      kpad_of(b_k[i] > 0 ? b_k[i] : 1));
    }
    return exp_bytes((long long) e) + maxbits_bytes((long long) e + 1) + q + 256;
}

extern "C" int ca3dmm_oz_plan_encode(ca3dmm_oz_plan_t *oz, int slices, int nA,
                                     const ca3dmm_oz_blk_t *A, const ca3dmm_oz_src_t *srcA,
                                     int nB, const ca3dmm_oz_blk_t *B,
                                     const ca3dmm_oz_src_t *srcB, int ngroup,
                                     const ca3dmm_oz_group_t *G, int nunit,
                                     const ca3dmm_oz_unit_t *units, void *dev_work,
                                     size_t work_bytes, void *host_plan, void *dev_plan)
{
    if (slices < 2 || slices > MAX_SLICES || nA + nB > 2 * ngroup) return CA3DMM_EINVAL;
    if (units && (nunit < 1 || nunit > ngroup)) return CA3DMM_EINVAL;
    const PlanLayout L(ngroup);
    unsigned char *h = static_cast<unsigned char *>(host_plan);
    memset(h, 0, L.total);
    PlanHeader *hd = reinterpret_cast<PlanHeader *>(h);
    SliceDesc *sd = reinterpret_cast<SliceDesc *>(h + L.sd);
    OzGroup *gr = reinterpret_cast<OzGroup *>(h + L.gr);
    // exponents first: one int array, cleared before each run
    size_t ne = 0;
    for (int i = 0; i < nA; ++i) ne += A[i].rows;
    for (int i = 0; i < nB; ++i) ne += B[i].cols;
    size_t qoff = exp_bytes((long long) ne) + maxbits_bytes((long long) ne + 1);
    // B blocks whose slices an A block reuses get 128-row padding, so that both
    // 64-row halves of every 128-row A tile exist
    for (int i = 0; i < nA; ++i)
        if (A[i].alias >= nB) return CA3DMM_EINVAL;
    long long eoff = 0;
    int max_rows = 1, max_kpad = 1;
    for (int side = 0; side < 2; ++side) oz->kc_tiles[side] = oz->rc_tiles[side] = oz->exp_items[side] = 0;
    for (int i = 0; i < nA + nB; ++i) {
        const bool isA = i < nA;
        const ca3dmm_oz_blk_t &b = isA ? A[i] : B[i - nA];
        const bool aliased = isA && b.alias >= 0;   // sliced as its B block
        bool target = false;
        for (int a = 0; !isA && a < nA; ++a) target = target || A[a].alias == i - nA;
        const int rows = aliased ? 0 : (isA ? b.rows : b.cols);   // A: rows of op(A); B: columns of op(B)
        const int kz = isA ? b.cols : b.rows;
        SliceDesc &d = sd[i];
        d.rows = rows;
        d.kz = kz;
        d.kpad = kpad_of(kz > 0 ? kz : 1);
        d.tile_rows = isA ? OBM : OBN;
        d.rows_pad = rows_pad_of(rows, target ? OBM : d.tile_rows);
        d.nkb = d.kpad / OKB;
        d.q_off = (long long) qoff;
        d.e_off = eoff;
        const ca3dmm_oz_src_t &src = isA ? srcA[i] : srcB[i - nA];
        if (isA) {
            // op(A)(r, l) = trans ? A[l + r ld] : A[r + l ld]; block at (b.r0, b.c0)
            d.rs = src.trans ? src.ld : 1;
            d.ls = src.trans ? 1 : src.ld;
            d.src_off = (long long) b.r0 * d.rs + (long long) b.c0 * d.ls;
        } else {
            // column j of op(B) over l: trans ? B[j + l ld] : B[l + j ld]; block at (l0 = b.r0, j0 = b.c0)
            d.rs = src.trans ? 1 : src.ld;
            d.ls = src.trans ? src.ld : 1;
            d.src_off = (long long) b.c0 * d.rs + (long long) b.r0 * d.ls;
        }
        if (src.base) d.src_off += (long long) (reinterpret_cast<uintptr_t>(src.base) / sizeof(double));
        if (d.ls != 1 && d.rs != 1) return CA3DMM_EINVAL;
        d.shape = d.ls == 1 ? SHAPE_KC : SHAPE_RC;
        const int side = isA ? 0 : 1;
        d.kc_begin = oz->kc_tiles[side];
        d.rc_begin = oz->rc_tiles[side];
        d.xbegin = oz->exp_items[side];
        (d.shape == SHAPE_KC ? oz->kc_tiles : oz->rc_tiles)[side] += slice_tiles_of(d);
        oz->exp_items[side] += exp_items_of(d);
        qoff += align256((size_t) slices * d.rows_pad * d.kpad);
        eoff += rows;
        if (d.rows_pad > max_rows) max_rows = d.rows_pad;
        if (d.kpad > max_kpad) max_kpad = d.kpad;
    }
    if (qoff > work_bytes) return CA3DMM_ENOMEM;
    int tiles = 0;
    for (int g = 0; g < ngroup; ++g) {
        OzGroup &o = gr[g];
        const int al = A[G[g].a_blk].alias;
        const SliceDesc &da = al >= 0 ? sd[nA + al] : sd[G[g].a_blk], &db = sd[nA + G[g].b_blk];
        const int row0 = G[g].row0, col0 = G[g].col0;
        if (row0 < 0 || col0 < 0 || row0 % OBM || col0 % OBN) return CA3DMM_EINVAL;
        o.a_from_b = al >= 0 ? 1 : 0;
        o.C = G[g].C; o.ldc = G[g].ldc;
        o.m = G[g].m; o.n = G[g].n; o.k = G[g].k;
        o.nkb = G[g].k > 0 ? da.nkb : 0;
        // a group may start inside its blocks: 128-row A tiles (aliased: two
        // 64-row B tiles, the same bytes) and 64-column B tiles further on
        o.ea_off = da.e_off + row0;
        o.eb_off = db.e_off + col0;
        o.a_desc = al >= 0 ? nA + al : G[g].a_blk;
        o.b_desc = nA + G[g].b_blk;
        o.row0 = row0;
        o.col0 = col0;
        o.qa_off = da.q_off + (long long) (row0 / OBM) * da.nkb * slices * A_SLICE_BYTES;
        o.qb_off = db.q_off + (long long) (col0 / OBN) * db.nkb * slices * B_SLICE_BYTES;
        o.a_tmap = 0;
        if (o.a_from_b && da.rows_pad % OBM == 0 && da.nkb > 0 && da.rows_pad > row0) {
            // One 5D box gathers an A stage from the B layout: (32 k bytes, 64 rows,
            // 64-row tile 2 tm and 2 tm + 1, slice, k-block); in shared memory the
            // box lands as [slice][tile][row][32 B], the 128-row A slices in turn.
            const unsigned long long dims[5] = {(unsigned long long) OKB, (unsigned long long) OBN,
                                                (unsigned long long) ((da.rows_pad - row0) / OBN),
                                                (unsigned long long) slices,
                                                (unsigned long long) da.nkb};
            const unsigned long long strides[4] = {
                (unsigned long long) OKB, (unsigned long long) da.nkb * slices * B_SLICE_BYTES,
                (unsigned long long) B_SLICE_BYTES, (unsigned long long) slices * B_SLICE_BYTES};
            const unsigned box[5] = {(unsigned) OKB, (unsigned) OBN, 2u, (unsigned) slices, 1u};
            o.a_tmap = ca3dmm_encode_tmap_u8(h + L.tm + (size_t) g * 128, 5,
                                             static_cast<unsigned char *>(dev_work) + o.qa_off,
                                             dims, strides, box) == CA3DMM_OK ? 1 : 0;
        }
        o.tiles_m = (o.m > 0 && o.n > 0) ? (o.m + OBM - 1) / OBM : 0;
        o.tiles_n = (o.m > 0 && o.n > 0) ? (o.n + OBN - 1) / OBN : 0;
        o.tile_begin = tiles;
        o.raster = G[g].raster > 0 ? G[g].raster : GROUP_M;
        tiles += o.tiles_m * o.tiles_n;
    }
    // work units: one per group, or the caller's chains of equal-shaped groups
    OzUnit *un = reinterpret_cast<OzUnit *>(h + L.un);
    const int nu = units ? nunit : ngroup;
    tiles = 0;
    for (int u = 0; u < nu; ++u) {
        const int g0 = units ? units[u].group : u;
        const int ns = units ? units[u].nsub : 1, st = units ? units[u].sub_stride : 0;
        if (g0 < 0 || ns < 1 || g0 + (ns - 1) * st >= ngroup || (ns > 1 && st < 1))
            return CA3DMM_EINVAL;
        for (int j = 1; j < ns; ++j)
            if (gr[g0 + j * st].m != gr[g0].m || gr[g0 + j * st].n != gr[g0].n)
                return CA3DMM_EINVAL;
        OzUnit &w = un[u];
        w.group = g0; w.nsub = ns; w.sub_stride = st; w.pad = 0;
        w.tiles_m = gr[g0].tiles_m;
        w.tiles_n = gr[g0].tiles_n;
        w.raster = gr[g0].raster;
        w.tile_begin = tiles;
        tiles += w.tiles_m * w.tiles_n;
    }
    hd->nA = nA; hd->nB = nB; hd->ngroup = ngroup; hd->slices = slices;
    hd->nslice_desc = nA + nB; hd->tiles = tiles; hd->nunit = nu;
    oz->slices = slices; oz->nA = nA; oz->nB = nB; oz->ngroup = ngroup; oz->tiles = tiles;
    oz->nunit = nu;
    oz->max_nsub = 1;
    for (int u = 0; u < nu; ++u) oz->max_nsub = un[u].nsub > oz->max_nsub ? un[u].nsub : oz->max_nsub;
    oz->max_rows = max_rows; oz->max_kpad = max_kpad;
    oz->n_exp = (long long) ne;
    oz->dev_plan = dev_plan;
    oz->dev_work = dev_work;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_oz_clear(const ca3dmm_oz_plan_t *oz, cudaStream_t stream)
{
    CA3DMM_CUDA_TRY(cudaMemsetAsync(oz->dev_work, 0,
                                    exp_bytes(oz->n_exp) + maxbits_bytes(oz->n_exp + 1), stream));
    return CA3DMM_OK;
}

static int launch_exp(const ca3dmm_oz_plan_t *oz, const void *src, const SliceDesc *descs,
                      int ndesc, int nitems, cudaStream_t stream)
{
    if (ndesc <= 0 || nitems <= 0) return CA3DMM_OK;
    unsigned char *w = static_cast<unsigned char *>(oz->dev_work);
    unsigned long long *mwork = reinterpret_cast<unsigned long long *>(w + exp_bytes(oz->n_exp));
    const int cap = ca3dmm_device_sm_count() * 8;
    oz_exp_kernel<<<nitems < cap ? nitems : cap, 256, 0, stream>>>(
        static_cast<const double *>(src), descs, ndesc, nitems, mwork, mwork + oz->n_exp);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}

static int launch_slice(const ca3dmm_oz_plan_t *oz, const void *src, const SliceDesc *descs,
                        int ndesc, int nkc, int nrc, cudaStream_t stream)
{
    if (ndesc <= 0) return CA3DMM_OK;
    unsigned char *w = static_cast<unsigned char *>(oz->dev_work);
    const unsigned long long *mwork =
        reinterpret_cast<const unsigned long long *>(w + exp_bytes(oz->n_exp));
    const int cap = ca3dmm_device_sm_count() * 4;
    const double *x = static_cast<const double *>(src);
    for (int shape = SHAPE_KC; shape <= SHAPE_RC; ++shape) {
        const int nt = shape == SHAPE_KC ? nkc : nrc;
        if (nt <= 0) continue;
        const unsigned grid = nt < cap ? nt : cap;
        switch (oz->slices) {
#define CA3DMM_SLICE_CASE(S)                                                                       \
    case S:                                                                                        \
        if (shape == SHAPE_KC)                                                                     \
            slice_kc_kernel<SliceWriter<S>><<<grid, 256, 0, stream>>>(x, descs, ndesc, nt, w, mwork);       \
        else                                                                                       \
            slice_rc_kernel<SliceWriter<S>><<<grid, 256, 0, stream>>>(x, descs, ndesc, nt, w, mwork);       \
        break;
            CA3DMM_SLICE_CASE(2) CA3DMM_SLICE_CASE(3) CA3DMM_SLICE_CASE(4) CA3DMM_SLICE_CASE(5)
            CA3DMM_SLICE_CASE(6) CA3DMM_SLICE_CASE(7) CA3DMM_SLICE_CASE(8)
#undef CA3DMM_SLICE_CASE
            default: return CA3DMM_EINVAL;
        }
        CA3DMM_CUDA_TRY(cudaGetLastError());
        ca3dmm_note_launch(1);
    }
    return CA3DMM_OK;
}

extern "C" int ca3dmm_oz_run_pack(const ca3dmm_oz_plan_t *oz, const void *A, const void *B,
                                  cudaStream_t stream)
{
    const PlanLayout L(oz->ngroup);
    const SliceDesc *sd =
        reinterpret_cast<const SliceDesc *>(static_cast<const unsigned char *>(oz->dev_plan) + L.sd);
    int rc = ca3dmm_oz_clear(oz, stream);
    if (!rc) rc = launch_exp(oz, A, sd, oz->nA, oz->exp_items[0], stream);
    if (!rc) rc = launch_exp(oz, B, sd + oz->nA, oz->nB, oz->exp_items[1], stream);
    if (!rc) rc = launch_slice(oz, A, sd, oz->nA, oz->kc_tiles[0], oz->rc_tiles[0], stream);
    if (!rc) rc = launch_slice(oz, B, sd + oz->nA, oz->nB, oz->kc_tiles[1], oz->rc_tiles[1], stream);
    return rc;
}

extern "C" int ca3dmm_oz_slice_side(const ca3dmm_oz_plan_t *oz, int which, const void *src,
                                    cudaStream_t stream)
{
    const PlanLayout L(oz->ngroup);
    const SliceDesc *sd =
        reinterpret_cast<const SliceDesc *>(static_cast<const unsigned char *>(oz->dev_plan) + L.sd);
    const SliceDesc *d = which ? sd + oz->nA : sd;
    const int nd = which ? oz->nB : oz->nA;
    const int side = which ? 1 : 0;
    int rc = launch_exp(oz, src, d, nd, oz->exp_items[side], stream);
    if (!rc) rc = launch_slice(oz, src, d, nd, oz->kc_tiles[side], oz->rc_tiles[side], stream);
    return rc;
}

extern "C" size_t ca3dmm_oz_desc_bytes(void) { return sizeof(SliceDesc); }

extern "C" int ca3dmm_oz_encode_rows(const void *host_plan, int ngroup, const int *blocks,
                                     int count, int r0, int r1, void *out_descs, int ntiles[3])
{
    const PlanLayout L(ngroup);
    const unsigned char *h = static_cast<const unsigned char *>(host_plan);
    const PlanHeader *hd = reinterpret_cast<const PlanHeader *>(h);
    const SliceDesc *sd = reinterpret_cast<const SliceDesc *>(h + L.sd);
    SliceDesc *out = static_cast<SliceDesc *>(out_descs);
    if (!blocks || count < 0 || r0 < 0 || r1 < r0) return CA3DMM_EINVAL;
    int kc = 0, rct = 0, items = 0;
    for (int i = 0; i < count; ++i) {
        if (blocks[i] < 0 || blocks[i] >= hd->nA) return CA3DMM_EINVAL;
        const SliceDesc &d = sd[blocks[i]];
        if (r0 % d.tile_rows) return CA3DMM_EINVAL;
        SliceDesc c = d;
        const int hi = r1 < d.rows ? r1 : d.rows;
        c.rows = hi > r0 ? hi - r0 : 0;
        c.rows_pad = rows_pad_of(c.rows, d.tile_rows);
        c.src_off = d.src_off + (long long) r0 * d.rs;
        c.q_off = d.q_off + (long long) (r0 / d.tile_rows) * d.nkb * hd->slices * d.tile_rows * OKB;
        c.e_off = d.e_off + r0;
        c.kc_begin = kc;
        c.rc_begin = rct;
        c.xbegin = items;
        (c.shape == SHAPE_KC ? kc : rct) += slice_tiles_of(c);
        items += exp_items_of(c);
        out[i] = c;
    }
    ntiles[0] = items;
    ntiles[1] = kc;
    ntiles[2] = rct;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_oz_encode_blocks(const void *host_plan, int ngroup, const int *descs,
                                       int count, void *out_descs, int ntiles[3])
{
    const PlanLayout L(ngroup);
    const unsigned char *h = static_cast<const unsigned char *>(host_plan);
    const PlanHeader *hd = reinterpret_cast<const PlanHeader *>(h);
    const SliceDesc *sd = reinterpret_cast<const SliceDesc *>(h + L.sd);
    SliceDesc *out = static_cast<SliceDesc *>(out_descs);
    if (!descs || count < 0) return CA3DMM_EINVAL;
    int kc = 0, rct = 0, items = 0;
    for (int i = 0; i < count; ++i) {
        if (descs[i] < 0 || descs[i] >= hd->nA + hd->nB) return CA3DMM_EINVAL;
        SliceDesc c = sd[descs[i]];
        c.kc_begin = kc;
        c.rc_begin = rct;
        c.xbegin = items;
        (c.shape == SHAPE_KC ? kc : rct) += slice_tiles_of(c);
        items += exp_items_of(c);
        out[i] = c;
    }
    ntiles[0] = items;
    ntiles[1] = kc;
    ntiles[2] = rct;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_oz_slice_descs(const ca3dmm_oz_plan_t *oz, const void *src,
                                     const void *dev_descs, int ndesc, const int ntiles[3],
                                     cudaStream_t stream)
{
    const SliceDesc *d = static_cast<const SliceDesc *>(dev_descs);
    int rc = launch_exp(oz, src, d, ndesc, ntiles[0], stream);
    if (!rc) rc = launch_slice(oz, src, d, ndesc, ntiles[1], ntiles[2], stream);
    return rc;
}

extern "C" int ca3dmm_oz_run_gemm(const ca3dmm_oz_plan_t *oz, int *dev_status, double timeout_s,
                                  cudaStream_t stream)
{
    ca3dmm_tile_ranges_t rg;
    memset(&rg, 0, sizeof(rg));
    rg.n = 1;
    rg.len[0] = oz->tiles;
    return ca3dmm_oz_run_gemm_ranges(oz, &rg, dev_status, timeout_s, stream);
}

extern "C" int ca3dmm_oz_run_gemm_ranges(const ca3dmm_oz_plan_t *oz, const ca3dmm_tile_ranges_t *rg,
                                         int *dev_status, double timeout_s, cudaStream_t stream)
{
    if (!rg || rg->n < 0 || rg->n > CA3DMM_MAX_RANGES) return CA3DMM_EINVAL;
    const int vtiles = range_total(*rg);
    if (vtiles <= 0) return CA3DMM_OK;
    const PlanLayout L(oz->ngroup);
    const unsigned char *pl = static_cast<const unsigned char *>(oz->dev_plan);
    const int stage_bytes = oz->slices * (A_SLICE_BYTES + B_SLICE_BYTES);
    int nstage = SMEM_BUDGET / stage_bytes;
    if (nstage > MAX_STAGES) nstage = MAX_STAGES;
    if (nstage < 2) return CA3DMM_EINVAL;
    const size_t smem = (size_t) nstage * stage_bytes + (2 * nstage + 2) * 8 + 1024;
    int grid = ca3dmm_device_sm_count();
    if (grid > vtiles) grid = vtiles;
    const unsigned long long limit = (unsigned long long) (timeout_s * 1e9);
    const int kb_per_chunk = kchunk_of(oz->slices) / OKB;
    const OzGroup *groups = reinterpret_cast<const OzGroup *>(pl + L.gr);
    const OzUnit *units = reinterpret_cast<const OzUnit *>(pl + L.un);
    const unsigned char *work = static_cast<const unsigned char *>(oz->dev_work);
    const int4 split = slice_split(oz->slices);
    switch (oz->slices) {
#define CA3DMM_GEMM_CASE(S)                                                                        \
    case S:                                                                                        \
        CA3DMM_CUDA_TRY(cudaFuncSetAttribute(oz_gemm_kernel<S>,                                    \
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,          \
                                             (int) smem));                                         \
        oz_gemm_kernel<S><<<grid, OTHREADS, smem, stream>>>(groups, units, pl + L.tm, oz->nunit,  \
                                                           oz->max_nsub, *rg, vtiles,              \
                                                           nstage,                                 \
                                                           kb_per_chunk, split, work, dev_status,  \
                                                           limit);                                 \
        break;
        CA3DMM_GEMM_CASE(2) CA3DMM_GEMM_CASE(3) CA3DMM_GEMM_CASE(4) CA3DMM_GEMM_CASE(5)
        CA3DMM_GEMM_CASE(6) CA3DMM_GEMM_CASE(7) CA3DMM_GEMM_CASE(8)
#undef CA3DMM_GEMM_CASE
        default: return CA3DMM_EINVAL;
    }
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}

extern "C" int ca3dmm_oz_run_nonfinite(const ca3dmm_oz_plan_t *oz, const ca3dmm_tile_ranges_t *rg,
                                       const void *A, const void *B, cudaStream_t stream)
{
    ca3dmm_tile_ranges_t all;
    if (!rg) {
        memset(&all, 0, sizeof(all));
        all.n = 1;
        all.len[0] = oz->tiles;
        rg = &all;
    }
    if (rg->n < 0 || rg->n > CA3DMM_MAX_RANGES) return CA3DMM_EINVAL;
    const int vtiles = range_total(*rg);
    if (vtiles <= 0) return CA3DMM_OK;
    const PlanLayout L(oz->ngroup);
    const unsigned char *pl = static_cast<const unsigned char *>(oz->dev_plan);
    const unsigned long long *mwork = reinterpret_cast<const unsigned long long *>(
        static_cast<const unsigned char *>(oz->dev_work) + exp_bytes(oz->n_exp));
    int grid = ca3dmm_device_sm_count() * 4;
    if (grid > vtiles) grid = vtiles;
    oz_nonfinite_kernel<<<grid, NF_THREADS, 0, stream>>>(
        static_cast<const double *>(A), static_cast<const double *>(B),
        reinterpret_cast<const SliceDesc *>(pl + L.sd), oz->nA,
        reinterpret_cast<const OzGroup *>(pl + L.gr), reinterpret_cast<const OzUnit *>(pl + L.un),
        oz->nunit, *rg, vtiles, mwork, mwork + oz->n_exp);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}
