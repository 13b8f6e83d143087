// Split-precision FP64 GEMM by the modular (CRT) scheme for sm_100a.
//
//  1. oz_exp_kernel (k_split.cuh) -- per row of op(A) / column of op(B): the
//                         largest |x| as its bit pattern.
//  2. slice_kc/rc_kernel<ResidueWriter> -- E = frexp exponent of the row max,
//                         a' = rint(x 2^(P-E)) (|a'| <= 2^P), and for every
//                         modulus p_t the residue a' mod p_t as a signed byte in
//                         [-floor(p/2), ceil(p/2) - 1] (computed in FP64), written
//                         straight into the GEMM's shared-memory image: per
//                         modulus, 128-row (A) /
//                         256-row (B) tile and 128-byte k block, a K-major tile
//                         with the 128-byte swizzle (16-byte chunk ^= row & 7).
//  3. crt_gemm_kernel<TN> -- per modulus, the INT8 product of the residues on the
//                         tcgen05 tensor cores: 128 x TN output tiles (TN = 256 or
//                         128), K = 32 per MMA, S32 accumulators in TMEM (two
//                         TN-column buffers, so the epilogue of one tile overlaps
//                         the next tile's MMAs).
//                         The sums are exact (k 2^14 < 2^31); the epilogue reduces
//                         each mod p_t into a byte plane of C's residues.
//  4. crt_reconstruct_kernel<N, L> -- per C entry, C' from its N residues by the
//                         Chinese remainder theorem: limb sums of the weights (in
//                         constant memory), an FP64 quotient estimate, the low 128
//                         bits exact; rounded once to double and scaled by
//                         2^(E_i + F_j - 2P).
//  5. crt_nonfinite_kernel -- rows / columns holding an Inf or a NaN were zero rows;
//                         writes their entries' IEEE value.
// Warp roles of the GEMM: warp 0 bulk-copy producer, warps 1-2 MMA issuers (two
// of the four k steps of each stage each: one issuing thread alone does not keep
// the tensor pipe busy), warps 3-10 epilogue (warp w reads TMEM lanes
// 32 (w % 4) .. +31, columns 0 .. TN/2-1 or TN/2 .. TN-1 of the accumulator).  The MMAs only
// accumulate; the epilogue zeroes each accumulator after reading it.  Every wait
// is bounded; on timeout the kernel records a status, drains, frees TMEM, returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include "k_common.cuh"
#include "k_split.cuh"
#include "ca3dmm_kernels.h"
#include "ca3dmm_crt.h"

namespace {

constexpr int MAXMOD = CA3DMM_CRT_MAX_MODULI;
// B residue blocks are stored in 256-column tiles (CBN); a GEMM tile is CBM rows
// by TN = 256 or 128 columns (a 128-column tile reads one half of a stored
// 256-row block, 16 KiB per k block, as the A side of B^T B already does).
constexpr int CBM = 128, CBN = 256, CKB = 128;   // tile rows, stored B tile rows, k bytes per stage
constexpr int CA_BYTES = CBM * CKB;              // 16 KiB
constexpr int CB_BYTES = CBN * CKB;              // 32 KiB

template <int TN>
struct CrtTile {
    static constexpr int kBBytes = TN * CKB;                    // B bytes per stage
    static constexpr int kStageBytes = CA_BYTES + kBBytes;
    static constexpr int kStages = TN == 256 ? 4 : 6;          // 192 KiB of stages either way
    static constexpr int kTmemCols = 2 * TN;                    // two accumulators
    static constexpr size_t kSmem = (size_t) kStages * kStageBytes + (2 * kStages + 4) * 8 + 1024;
};
constexpr int C_THREADS = 352;                   // 11 warps
constexpr int C_ISSUERS = 2;
constexpr int C_EPI_WARPS = 8;
constexpr int GROUP_CACHE = 512;
constexpr int DEFAULT_BAND = 8;

// ------------------------------------------------------------------ moduli
// Pairwise coprime moduli <= 256, largest first (256 = 2^8 and odd numbers
// with disjoint prime factors), and per modulus the constants of the GEMM
// epilogue's reduction (2^16 mod p, floor(2^32 / p), a bias) and of the
// residue pass (2^27 mod p and 1/p in FP64).
constexpr int kModList[MAXMOD] = {256, 255, 253, 251, 247, 241, 239, 233, 229,
                                  227, 223, 217, 211, 199, 197, 193, 191, 181};
static_assert(kModList[0] == 256, "the residue pass takes modulus 0 as the byte of the integer");

struct ModConst {
    int p, c16;          // p, 2^16 mod p
    unsigned int mrec;   // floor(2^32 / p): floor(y mrec / 2^32) is floor(y / p) or one less (y < 2^28)
    int bias;            // a multiple of p above 2^15 * 255 (keeps the epilogue's sums >= 0)
    double c27;      // 2^27 mod p (the residue pass, in FP64)
    double inv;      // 1 / p rounded to double
};

constexpr ModConst make_mod(int p)
{
    return ModConst{p,
                    (int) ((1LL << 16) % p),
                    (unsigned int) ((1ULL << 32) / (unsigned long long) p),
                    (int) (((8650752LL + p - 1) / p) * p),   // a multiple of p >= 2^23 + 2^18
                    (double) ((1LL << 27) % p),
                    1.0 / (double) p};
}

struct ModTable {
    ModConst m[MAXMOD];
};

constexpr ModTable make_mod_table()
{
    ModTable t{};
    for (int i = 0; i < MAXMOD; ++i) t.m[i] = make_mod(kModList[i]);
    return t;
}

// CRT weights, exact, for every modulus count N: M_N = prod_{t<N} p_t,
// W_t = (M_N / p_t) ((M_N / p_t)^-1 mod p_t), so that sum_t u_t W_t = C' (mod M_N)
// for residues u_t = C' mod p_t.  Little-endian 32-bit limbs.
constexpr int LIMBS = 5;                        // M_18 < 2^141, W_t < M_N
struct Big {
    unsigned int w[6];
};

constexpr Big big_small(unsigned int v)
{
    Big b{};
    b.w[0] = v;
    return b;
}

constexpr Big big_mul(Big a, unsigned int m)
{
    unsigned long long c = 0;
    for (int i = 0; i < 6; ++i) {
        unsigned long long t = (unsigned long long) a.w[i] * m + c;
        a.w[i] = (unsigned int) t;
        c = t >> 32;
    }
    return a;
}

constexpr Big big_div(Big a, unsigned int d)
{
    unsigned long long r = 0;
    for (int i = 5; i >= 0; --i) {
        unsigned long long cur = (r << 32) | a.w[i];
        a.w[i] = (unsigned int) (cur / d);
        r = cur % d;
    }
    return a;
}

constexpr unsigned int big_mod(Big a, unsigned int d)
{
    unsigned long long r = 0;
    for (int i = 5; i >= 0; --i) r = ((r << 32) | a.w[i]) % d;
    return (unsigned int) r;
}

constexpr unsigned int inv_mod(unsigned int a, unsigned int p)
{
    for (unsigned int x = 1; x < p; ++x)
        if ((a * x) % p == 1) return x;
    return 0;
}

struct CrtTable {
    unsigned int W[MAXMOD + 1][MAXMOD][LIMBS];
    unsigned int M[MAXMOD + 1][LIMBS + 1];
    unsigned int H[MAXMOD + 1][LIMBS + 1];      // M / 2 (M is even: 256 is a modulus)
    double Md[MAXMOD + 1], invM[MAXMOD + 1];
};

constexpr CrtTable make_crt_table()
{
    CrtTable T{};
    for (int n = 2; n <= MAXMOD; ++n) {
        Big M = big_small(1);
        for (int t = 0; t < n; ++t) M = big_mul(M, (unsigned int) kModList[t]);
        for (int t = 0; t < n; ++t) {
            const unsigned int p = (unsigned int) kModList[t];
            Big Mt = big_div(M, p);
            const Big W = big_mul(Mt, inv_mod(big_mod(Mt, p), p));
            for (int q = 0; q < LIMBS; ++q) T.W[n][t][q] = W.w[q];
        }
        const Big H = big_div(M, 2);
        double md = 0.0;
        for (int q = 5; q >= 0; --q) md = md * 4294967296.0 + (double) M.w[q];
        for (int q = 0; q <= LIMBS; ++q) {
            T.M[n][q] = M.w[q];
            T.H[n][q] = H.w[q];
        }
        T.Md[n] = md;
        T.invM[n] = 1.0 / md;
    }
    return T;
}

__constant__ ModTable kMod = make_mod_table();
__constant__ CrtTable kCrt = make_crt_table();

double log2_modprod(int nmod)
{
    double s = 0.0;
    for (int t = 0; t < nmod && t < MAXMOD; ++t) s += std::log2((double) kModList[t]);
    return s;
}

// ------------------------------------------------------------------ residues
// The residues of the row / column integers a' = rint(a 2^(P - E)) (|a'| <=
// 2^53), as signed bytes in [-(p-1)/2, (p-1)/2] (p odd) and [-128, 127]
// (p = 256).  a' = h 2^27 + l with |h|, |l| <= 2^26 (h by rounding with
// 1.5 2^52 added), then per odd modulus yb = h (2^27 mod p) + l + 1.5 2^52
// (one FMA, exact: |y| < 2^35) and q = the nearest integer to y / p, from
// y = yb - 1.5 2^52 and one FMA with 1.5 2^52 added (y (1/p) is within 2^-23
// of y / p, which is never closer than 1 / (2p) to a half-integer for odd p).
// The low words of yb and of that FMA are y and q modulo 2^32 (the low bits of
// x + 1.5 2^52 are the integer x in two's complement), and r = y - q p is
// small, so it is one 32-bit integer multiply-add modulo 2^32: three FP64
// operations and one on the integer pipe per modulus (five FP64 operations
// when r was formed in FP64: 119 -> 99 us per 4000 x 4000 operand).  For
// p = 256 the byte is the low byte of l (a' = l mod 256).  Every value is the
// unique representative of a' mod p in that range, so the bytes equal the
// integer formulation's.
// NM: the modulus count, a template argument so that the modulus loop unrolls
// (the constants become immediate operands and consecutive moduli interleave).
template <int NM>
struct ResidueWriter {
    static constexpr int kMinBlocks = 2;
    static __device__ __forceinline__ void write16(const SliceDesc &d, unsigned char *__restrict__ work,
                                                   const unsigned long long *__restrict__ mwork,
                                                   int gr, int gl, const double (&x)[16])
    {
        const unsigned long long mr = gr < d.rows ? mwork[d.e_off + gr] : 0ull;
        const bool fin = mr < INF_BITS;
        int E = 0;
        if (fin && mr) frexp(__longlong_as_double((long long) mr), &E);
        if (gl == 0 && gr < d.rows)
            reinterpret_cast<int *>(work)[d.e_off + gr] = (fin && mr) ? E + EXP_BIAS : 0;
        const int sh = d.p_bits - E;
        const double up1 = ldexp(1.0, sh / 2), up2 = ldexp(1.0, sh - sh / 2);
        constexpr double MAGIC = 6755399441055744.0;          // 1.5 2^52
        double hh[16], lm[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const double a = rint((fin ? x[j] : 0.0) * up1 * up2);
            const double h = (a * 0x1p-27 + MAGIC) - MAGIC;   // nearest integer, |h| <= 2^26
            hh[j] = h;
            lm[j] = fma(-h, 0x1p27, a) + MAGIC;              // l + 1.5 2^52, exact
        }
        const int rt = gr / d.tile_rows, rr = gr % d.tile_rows;
        const int kb = gl >> 7, chunk = (gl & 127) >> 4;
        unsigned char *dst = work + d.q_off + ((long long) rt * d.nkb + kb) * d.tile_rows * CKB +
                             rr * CKB + ((chunk ^ (rr & 7)) << 4);
        // modulus 0 is 256 (kModList), the others are odd
#pragma unroll
        for (int t = 0; t < NM; ++t) {
            unsigned int r[16];
            if (t == 0) {
#pragma unroll
                for (int j = 0; j < 16; ++j) r[j] = (unsigned int) __double2loint(lm[j]);
            } else {
                const double c27 = kMod.m[t].c27, inv = kMod.m[t].inv;
                const unsigned int p = (unsigned int) kMod.m[t].p;
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const double yb = fma(hh[j], c27, lm[j]);      // y + 1.5 2^52
                    const double qm = fma(yb - MAGIC, inv, MAGIC);  // q + 1.5 2^52
                    r[j] = (unsigned int) __double2loint(yb) - (unsigned int) __double2loint(qm) * p;
                }
            }
            uint32_t out[4];
#pragma unroll
            for (int w = 0; w < 4; ++w) {
                const uint32_t lo = __byte_perm(r[4 * w], r[4 * w + 1], 0x7740);
                const uint32_t hi = __byte_perm(r[4 * w + 2], r[4 * w + 3], 0x7740);
                out[w] = __byte_perm(lo, hi, 0x5410);
            }
            *reinterpret_cast<uint4 *>(dst + (long long) t * d.t_stride) =
                make_uint4(out[0], out[1], out[2], out[3]);
        }
    }
};

// ------------------------------------------------------------------ plan
struct CrtGroup {
    double *C;
    long long ldc;
    int m, n, k;
    int a_desc, b_desc, a_from_b;   // a_from_b: A tile tm is half tm % 2 of the B block's tile tm / 2
    int tiles_m, tiles_n, item_begin, band;
    int tile_n, pad_;               // GEMM tile columns (128 or 256; the same in every group)
    long long rc_begin;             // first reconstruction item (4 rows x 1 column) of the group
    int P, nkb;                     // integer width, 128-byte k blocks
    long long ea_off, eb_off;       // exponents of the A rows / B columns
    long long qa_off, qb_off;       // residue bytes of the operand blocks
    long long qa_tstride, qb_tstride;
    long long pl_off, pl_ld, pl_bytes;   // residue planes of C: [t][tiles_n * 256][pl_ld]
};

struct CrtHeader {
    int nmod, nA, nB, ngroup;
    int items, pad[3];
};

struct CrtLayout {
    size_t sd, gr, total;
    CrtLayout(int nblk, int ngroup)
    {
        sd = 256;
        gr = (sd + (size_t) nblk * sizeof(SliceDesc) + 127) / 128 * 128;
        total = (gr + (size_t) ngroup * sizeof(CrtGroup) + 255) / 256 * 256;
    }
};

size_t align256(size_t x) { return (x + 255) / 256 * 256; }
int round_up(int x, int a) { return (x + a - 1) / a * a; }

__device__ __forceinline__ int find_group(const int *sb, const CrtGroup *g, int n, int item)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if ((sb ? sb[mid] : g[mid].item_begin) <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// work item -> (modulus t, tile row tm, tile column tn) of its group: bands of
// `band` tile rows; inside a band the moduli in turn, each over the band's
// tiles with the tile row fastest
__device__ __forceinline__ void item_decode(const CrtGroup &G, int nmod, int item, int &t, int &tm,
                                            int &tn)
{
    const int local = item - G.item_begin;
    const int full = nmod * G.band * G.tiles_n;
    const int b = local / full;
    const int rem = local - b * full;
    const int rows = min(G.band, G.tiles_m - b * G.band);
    const int per_t = rows * G.tiles_n;
    t = rem / per_t;
    const int r2 = rem - t * per_t;
    tm = b * G.band + r2 % rows;
    tn = r2 / rows;
}

// Columns of tile tn that the MMAs compute: TN, or for the last tile of a
// group the columns of C it holds rounded up to 16 (an MMA N with M = 128);
// the B rows past them are neither loaded nor multiplied.
__device__ __forceinline__ int tile_cols(const CrtGroup &G, int tn, int TN)
{
    const int left = G.n - tn * TN;
    return left >= TN ? TN : (left + 15) & ~15;
}

// K-major, SWIZZLE_128B shared-memory operand descriptor: rows of 128 bytes,
// 8-row groups 1024 bytes apart (SBO), descriptor version 1, layout type 2.
__device__ __forceinline__ uint64_t sdesc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t) ((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t) 1 << 16;                 // LBO (unused for swizzled K-major)
    d |= (uint64_t) (1024 >> 4) << 32;       // SBO
    d |= (uint64_t) 1 << 46;                 // descriptor version (sm_100)
    d |= (uint64_t) 2 << 61;                 // SWIZZLE_128B
    return d;
}

// int32 sum -> its residue mod p in [0, p): v = 2^16 h + l (h signed), so
// y = h (2^16 mod p) + l + bias >= 0 is below 2^25 and congruent to v; the
// quotient floor(y floor(2^32/p) / 2^32) is short by at most one.
__device__ __forceinline__ unsigned int mod_i32(uint32_t vbits, const ModConst &mc)
{
    const int v = (int) vbits;
    const int h = v >> 16;
    const unsigned int y = (unsigned int) (h * mc.c16 + (int) (vbits & 0xffffu) + mc.bias);
    const unsigned int q = __umulhi(y, mc.mrec);
    const unsigned int r0 = y - q * (unsigned int) mc.p;
    const unsigned int r1 = r0 - (unsigned int) mc.p;
    return r0 < r1 ? r0 : r1;
}

// ------------------------------------------------------------------ GEMM
template <int TN>
__global__ void __launch_bounds__(C_THREADS, 1)
crt_gemm_kernel(const CrtGroup *__restrict__ groups, int ngroup, int nmod,
                const ca3dmm_tile_ranges_t rg, int total_items,
                unsigned char *__restrict__ work, int *status, unsigned long long limit_ns)
{
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    using T = CrtTile<TN>;
    constexpr int CNSTAGE = T::kStages, CSTAGE_BYTES = T::kStageBytes;
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + CNSTAGE * CSTAGE_BYTES);
    uint64_t *empty = full + CNSTAGE;
    uint64_t *acc_full = empty + CNSTAGE;       // [2]
    uint64_t *acc_empty = acc_full + 2;         // [2]
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    __shared__ int s_gbeg[GROUP_CACHE];
    const int *gb = ngroup <= GROUP_CACHE ? s_gbeg : nullptr;
    if (gb)
        for (int i = threadIdx.x; i < ngroup; i += blockDim.x) s_gbeg[i] = groups[i].item_begin;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < CNSTAGE; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], C_ISSUERS);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], C_ISSUERS);
            mbar_init(&acc_empty[b], C_EPI_WARPS);
        }
        abort_flag = 0;
        fence_barrier_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_slot)),
                     "r"(T::kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = tmem_slot;
    if (warp >= 3 && warp <= 6) {
        // zero both accumulators (the MMAs only accumulate)
        const uint32_t lane_base = (uint32_t) ((warp & 3) * 32) << 16;
        for (int c = 0; c < T::kTmemCols; c += 32) tmem_zero32(tmem_base + lane_base + (uint32_t) c);
        tmem_wait_st();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    if (warp == 0) {
        // ------------------------------------------------------ producer
        if (lane == 0) {
            uint32_t it = 0;
            bool ok = true;
            for (int v = blockIdx.x; v < total_items && ok && !abort_flag; v += gridDim.x) {
                const int item = range_tile(rg, v);
                const CrtGroup &G = groups[find_group(gb, groups, ngroup, item)];
                int t, tm, tn;
                item_decode(G, nmod, item, t, tm, tn);
                const unsigned char *qa =
                    G.a_from_b ? work + G.qa_off + t * G.qa_tstride +
                                     (long long) (tm >> 1) * G.nkb * CB_BYTES + (tm & 1) * CA_BYTES
                               : work + G.qa_off + t * G.qa_tstride + (long long) tm * G.nkb * CA_BYTES;
                const long long a_step = G.a_from_b ? CB_BYTES : CA_BYTES;
                const uint32_t b_bytes = (uint32_t) tile_cols(G, tn, TN) * CKB;
                // a 128-column tile: half tn % 2 of stored 256-row tile tn / 2
                const unsigned char *qb =
                    TN == CBN ? work + G.qb_off + t * G.qb_tstride + (long long) tn * G.nkb * CB_BYTES
                              : work + G.qb_off + t * G.qb_tstride +
                                    (long long) (tn >> 1) * G.nkb * CB_BYTES + (tn & 1) * T::kBBytes;
                for (int kb = 0; kb < G.nkb; ++kb, ++it) {
                    const uint32_t s = it % CNSTAGE, ph = (it / CNSTAGE) & 1u;
                    if (!mbar_wait_bounded(&empty[s], ph ^ 1u, &abort_flag, status,
                                           CA3DMM_DEV_TIMEOUT_PRODUCE, limit_ns)) {
                        ok = false;
                        break;
                    }
                    uint8_t *sA = smem + s * CSTAGE_BYTES;
                    mbar_arrive_expect_tx(&full[s], CA_BYTES + b_bytes);
                    bulk_load(sA, qa + (long long) kb * a_step, CA_BYTES, &full[s]);
                    bulk_load(sA + CA_BYTES, qb + (long long) kb * CB_BYTES, b_bytes, &full[s]);
                }
            }
            // drain copies in flight (bounded, abort flag ignored)
            const uint32_t first = it > (uint32_t) CNSTAGE ? it - CNSTAGE : 0;
            for (uint32_t L = first; L < it; ++L) {
                uint64_t t0 = global_timer_ns();
                while (!mbar_try_wait(&full[L % CNSTAGE], (L / CNSTAGE) & 1u))
                    if (global_timer_ns() - t0 > limit_ns) break;
            }
        }
    } else if (warp == 1 || warp == 2) {
        // ------------------------------------------------------ MMA issuers
        if (lane == 0) {
            const int half = warp - 1;          // k steps 2 half, 2 half + 1 of each stage
            uint32_t it = 0, ai = 0;
            bool ok = true;
            for (int v = blockIdx.x; v < total_items && ok; v += gridDim.x, ++ai) {
                const int item = range_tile(rg, v);
                const CrtGroup &G = groups[find_group(gb, groups, ngroup, item)];
                int t, tm, tn;
                item_decode(G, nmod, item, t, tm, tn);
                const uint32_t idesc = idesc_i8(tile_cols(G, tn, TN), CBM);
                const uint32_t buf = ai & 1u;
                if (!mbar_wait_bounded(&acc_empty[buf], ((ai >> 1) & 1u) ^ 1u, &abort_flag, status,
                                       CA3DMM_DEV_TIMEOUT_ACCUM, limit_ns)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t tacc = tmem_base + buf * TN;
                for (int kb = 0; kb < G.nkb; ++kb, ++it) {
                    const uint32_t s = it % CNSTAGE, ph = (it / CNSTAGE) & 1u;
                    if (!mbar_wait_bounded(&full[s], ph, &abort_flag, status,
                                           CA3DMM_DEV_TIMEOUT_CONSUME, limit_ns)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sA = smem_u32(smem + s * CSTAGE_BYTES);
                    const uint32_t sB = sA + CA_BYTES;
                    // k steps past the group's k hold zero residues: not issued
                    const int kleft = G.k - kb * CKB;
#pragma unroll
                    for (int kk = 2 * half; kk < 2 * half + 2; ++kk)
                        if (kk * 32 < kleft)
                            tc_mma_i8(tacc, sdesc_sw128(sA + kk * 32), sdesc_sw128(sB + kk * 32),
                                      idesc, 1u);
                    tc_commit(&empty[s]);
                }
                if (!ok) break;
                tc_commit(&acc_full[buf]);
            }
            if (!ok) {
                // let every MMA this thread issued finish before TMEM is freed
                tc_commit(&acc_full[ai & 1u]);
                uint64_t t0 = global_timer_ns();
                while (!mbar_try_wait(&acc_full[ai & 1u], (ai >> 1) & 1u))
                    if (global_timer_ns() - t0 > limit_ns) break;
            }
        }
        __syncwarp();
    } else {
        // ------------------------------------------------------ epilogue
        const int q = warp & 3;                       // TMEM lane quarter of this warp
        const int h = (warp - 3) >> 2;                // accumulator columns TN/2 h .. TN/2 (h + 1) - 1
        uint32_t ai = 0;
        for (int v = blockIdx.x; v < total_items; v += gridDim.x, ++ai) {
            const int item = range_tile(rg, v);
            const CrtGroup &G = groups[find_group(gb, groups, ngroup, item)];
            int t, tm, tn;
            item_decode(G, nmod, item, t, tm, tn);
            const uint32_t buf = ai & 1u;
            if (!mbar_wait_bounded(&acc_full[buf], (ai >> 1) & 1u, &abort_flag, status,
                                   CA3DMM_DEV_TIMEOUT_EPI, limit_ns))
                break;
            tc_fence_after();
            const ModConst mc = kMod.m[t];
            const int row = tm * CBM + q * 32 + lane;
            unsigned char *plane = work + G.pl_off + (long long) t * G.pl_bytes + row;
            // columns past tile_cols were not accumulated (still zero) and lie
            // past the group's n (never read): skipped
            const int ncols = tile_cols(G, tn, TN);
#pragma unroll 1
            for (int cb = 0; cb < TN / 64; ++cb) {
                const int c0 = h * (TN / 2) + cb * 32;
                if (c0 >= ncols) break;
                uint32_t vv[32];
                const uint32_t ta = tmem_base + ((uint32_t) (q * 32) << 16) + buf * TN + (uint32_t) c0;
                tmem_ld32(ta, vv);
                tmem_zero32(ta);
                unsigned char *pc = plane + (long long) (tn * TN + c0) * G.pl_ld;
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    pc[(long long) j * G.pl_ld] = (unsigned char) mod_i32(vv[j], mc);
            }
            tmem_wait_st();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[buf]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(T::kTmemCols)
                     : "memory");
    }
}

// ------------------------------------------------------------------ reconstruction
// |x| < 2^127 given as two 64-bit halves -> double rounded to nearest even,
// with *sh the power of two it is to be scaled by: a 64-bit window with the
// leading bit at 63 and the bits below it ORed into bit 0, converted once.
__device__ __forceinline__ double u128_to_double(unsigned long long hi, unsigned long long lo,
                                                 int *sh)
{
    if (hi == 0ull) {
        *sh = 0;
        return __ull2double_rn(lo);
    }
    const int lz = __clzll((long long) hi);
    unsigned long long w = lz ? (hi << lz) | (lo >> (64 - lz)) : hi;
    const unsigned long long rest = lo << lz;
    w |= rest ? 1ull : 0ull;
    *sh = 64 - lz;
    return __ull2double_rn(w);
}

// 32-bit limbs that the modulus product M_N needs (known at compile time)
constexpr int crt_limbs(int n)
{
    const CrtTable T = make_crt_table();
    int l = LIMBS + 1;
    while (l > 1 && T.M[n][l - 1] == 0u) --l;
    return l;
}

// C' from its residues: S = sum_t u_t W_t (column sums of 32-bit limb
// products), q = rint(S / M) from an FP64 estimate of S (|C'| < M / 2, and the
// estimate is off by far less than the gap to a half-integer), then
// C' = S - q M taken modulo 2^128, which holds it exactly in two's complement
// because |C'| <= k 2^(2P) <= 2^123.  Only the limbs below 2^128 of S and q M
// are formed; all W_t and M fit in L = crt_limbs(N) limbs (a template
// argument, computed on the host).
// Work items are 4 rows x 1 column of C.  One group: the rows [r0, r1) of
// group g0; several: every row of groups [g0, g1), numbered by the groups'
// rc_begin prefix (found by a search over a shared copy), so that the grid
// is spread by size over a batch of uneven groups.
template <int N, int L>
__global__ void __launch_bounds__(256)
crt_reconstruct_kernel(const CrtGroup *__restrict__ groups, int g0, int g1, int r0, int r1,
                       long long total, const unsigned char *__restrict__ work)
{
    static_assert(L >= 2 && L <= LIMBS, "modulus product outside the limb range");
    __shared__ long long s_rb[GROUP_CACHE];
    const int ng = g1 - g0;
    const bool cached = ng > 1 && ng <= GROUP_CACHE;
    if (cached)
        for (int i = threadIdx.x; i < ng; i += blockDim.x) s_rb[i] = groups[g0 + i].rc_begin;
    __syncthreads();
    const int *ework = reinterpret_cast<const int *>(work);
    const long long base = ng > 1 ? groups[g0].rc_begin : 0;
    for (long long it = blockIdx.x * (long long) blockDim.x + threadIdx.x; it < total;
         it += (long long) gridDim.x * blockDim.x) {
        int gi = 0;
        if (ng > 1) {
            const long long a = base + it;
            int lo = 0, hi = ng - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if ((cached ? s_rb[mid] : groups[g0 + mid].rc_begin) <= a) lo = mid; else hi = mid - 1;
            }
            gi = lo;
        }
        const CrtGroup &G = groups[g0 + gi];
        const int rb = ng > 1 ? 0 : max(r0, 0), re = ng > 1 ? G.m : min(r1, G.m);
        if (re <= rb) continue;
        const int nq = (re - rb + 3) >> 2;
        const long long local = ng > 1 ? base + it - G.rc_begin : it;
        if (local >= (long long) nq * G.n) continue;
        const int j = (int) (local / nq), i0 = rb + 4 * (int) (local % nq);
        const int fb = ework[G.eb_off + j];
        const int Fj = fb ? fb - EXP_BIAS : 0;
        uint32_t u4[N];
#pragma unroll
        for (int t = 0; t < N; ++t)
            u4[t] = __ldg(reinterpret_cast<const unsigned int *>(
                work + G.pl_off + (long long) t * G.pl_bytes + (long long) j * G.pl_ld + i0));
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int i = i0 + e;
            if (i < re) {
                unsigned long long a[L];
#pragma unroll
                for (int q = 0; q < L; ++q) a[q] = 0ull;
#pragma unroll
                for (int t = 0; t < N; ++t) {
                    const unsigned int u = __byte_perm(u4[t], 0u, 0x4440u | (unsigned int) e);
#pragma unroll
                    for (int q = 0; q < L; ++q) a[q] += (unsigned long long) u * kCrt.W[N][t][q];
                }
                // quotient: S = sum_q a_q 2^(32 q) in FP64 (each a_q < 2^46 exact)
                double sd = (double) a[L - 1];
#pragma unroll
                for (int q = L - 2; q >= 0; --q) sd = fma(sd, 4294967296.0, (double) a[q]);
                const unsigned int qe = (unsigned int) __double2int_rn(sd * kCrt.invM[N]);
                // low 128 bits of S and of q M, then C' = S - q M mod 2^128
                unsigned int s4[4];
                unsigned long long c = 0ull;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const unsigned long long x = (q < L ? a[q] : 0ull) + c;
                    s4[q] = (unsigned int) x;
                    c = x >> 32;
                }
                unsigned int t4[4];
                unsigned long long pc = 0ull;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const unsigned long long pm = (unsigned long long) qe * kCrt.M[N][q] + pc;
                    t4[q] = (unsigned int) pm;
                    pc = pm >> 32;
                }
                const unsigned long long slo = ((unsigned long long) s4[1] << 32) | s4[0];
                const unsigned long long shi = ((unsigned long long) s4[3] << 32) | s4[2];
                const unsigned long long tlo = ((unsigned long long) t4[1] << 32) | t4[0];
                const unsigned long long thi = ((unsigned long long) t4[3] << 32) | t4[2];
                unsigned long long lo = slo - tlo;
                unsigned long long hi = shi - thi - (slo < tlo ? 1ull : 0ull);
                const bool neg = (long long) hi < 0;
                if (neg) {
                    lo = ~lo + 1ull;
                    hi = ~hi + (lo == 0ull ? 1ull : 0ull);
                }
                int sh;
                const double dv = u128_to_double(hi, lo, &sh);
                const int eb = ework[G.ea_off + i];
                const int Ei = eb ? eb - EXP_BIAS : 0;
                const double val = scale2(dv, sh + Ei + Fj - 2 * G.P);
                G.C[i + (long long) j * G.ldc] = neg ? -val : val;
            }
        }
    }
}

// ------------------------------------------------------------------ non-finite inputs
__global__ void __launch_bounds__(256)
crt_nonfinite_kernel(const double *__restrict__ srcA, const double *__restrict__ srcB,
                     const SliceDesc *__restrict__ descs, int nA, const CrtGroup *__restrict__ groups,
                     int g0, int r0, int r1, const unsigned long long *__restrict__ mwork,
                     const unsigned long long *__restrict__ nonfinite)
{
    if (*nonfinite == 0ull) return;
    const CrtGroup &G = groups[g0 + blockIdx.y];
    const int rb = max(r0, 0), re = min(r1, G.m);
    if (re <= rb) return;
    const SliceDesc &da = descs[G.a_desc], &db = descs[G.b_desc];
    const double *baseA = slice_src(G.a_desc < nA ? srcA : srcB, da.src_off);
    const double *baseB = slice_src(srcB, db.src_off);
    const int lines = (re - rb) + G.n;
    for (int line = blockIdx.x; line < lines; line += gridDim.x) {
        const bool isrow = line < re - rb;
        const int fixed = isrow ? rb + line : line - (re - rb);
        if (mwork[(isrow ? G.ea_off : G.eb_off) + fixed] < INF_BITS) continue;
        const int count = isrow ? G.n : re - rb;
        for (int x = threadIdx.x; x < count; x += blockDim.x) {
            const int i = isrow ? fixed : rb + x, j = isrow ? x : fixed;
            const unsigned long long ma = mwork[G.ea_off + i], mb = mwork[G.eb_off + j];
            int cls = 0;
            if (ma > INF_BITS || mb > INF_BITS) {
                cls = 1;                                   // a NaN factor
            } else {
                const double *pa = baseA + (long long) i * da.rs;
                const double *pb = baseB + (long long) j * db.rs;
                for (int l = 0; l < G.k && !(cls & 1); ++l)
                    cls |= product_class(__ldg(pa + (long long) l * da.ls),
                                         __ldg(pb + (long long) l * db.ls));
            }
            double out;
            if ((cls & 1) || (cls & 6) == 6) out = __longlong_as_double(0x7ff8000000000000ll);
            else if (cls & 2) out = __longlong_as_double(0x7ff0000000000000ll);
            else if (cls & 4) out = __longlong_as_double((long long) 0xfff0000000000000ull);
            else continue;
            G.C[i + (long long) j * G.ldc] = out;
        }
    }
}

}  // namespace

// ------------------------------------------------------------------ host side
extern "C" int ca3dmm_crt_modulus(int t) { return (t >= 0 && t < MAXMOD) ? kModList[t] : 0; }

extern "C" int ca3dmm_crt_bits(int nmod, long long k)
{
    if (nmod < 2 || nmod > MAXMOD) return 0;
    const double lk = std::log2((double) (k > 1 ? k : 1));
    const int P = (int) std::floor((log2_modprod(nmod) - 1.0 - lk - 1e-9) / 2.0);
    return P > 53 ? 53 : P;
}

extern "C" size_t ca3dmm_crt_plan_bytes(int nblk, int ngroup) { return CrtLayout(nblk, ngroup).total; }

static size_t crt_block_bytes(int rows, int k, int tile_rows, int nmod)
{
    return align256((size_t) nmod * (size_t) round_up(rows > 0 ? rows : 1, tile_rows) *
                    (size_t) round_up(k > 0 ? k : 1, CKB));
}

static size_t crt_plane_bytes(int m, int n)
{
    return (size_t) round_up(m > 0 ? m : 1, CBM) * (size_t) round_up(n > 0 ? n : 1, CBN);
}

extern "C" size_t ca3dmm_crt_work_bytes(int nA, const int *a_rows, const int *a_k, int nB,
                                        const int *b_k, const int *b_cols, int ngroup,
                                        const int *g_m, const int *g_n, int nmod)
{
    size_t e = 0, q = 0;
    for (int i = 0; i < nA; ++i) {
        e += (size_t) a_rows[i];
        q += crt_block_bytes(a_rows[i], a_k[i], CBM, nmod);
    }
    for (int i = 0; i < nB; ++i) {
        e += (size_t) b_cols[i];
        q += crt_block_bytes(b_cols[i], b_k[i], CBN, nmod);
    }
    for (int g = 0; g < ngroup; ++g) q += align256((size_t) nmod * crt_plane_bytes(g_m[g], g_n[g]));
    return exp_bytes((long long) e) + maxbits_bytes((long long) e + 1) + q + 256;
}

extern "C" int ca3dmm_crt_plan_encode(ca3dmm_crt_plan_t *pl, int nmod, int nA,
                                      const ca3dmm_oz_blk_t *A, const ca3dmm_oz_src_t *srcA, int nB,
                                      const ca3dmm_oz_blk_t *B, const ca3dmm_oz_src_t *srcB,
                                      int ngroup, const ca3dmm_crt_group_t *G, void *dev_work,
                                      size_t work_bytes, void *host_plan, void *dev_plan)
{
    if (nmod < 2 || nmod > MAXMOD || ngroup < 1) return CA3DMM_EINVAL;
    const CrtLayout L(nA + nB, ngroup);
    unsigned char *h = static_cast<unsigned char *>(host_plan);
    memset(h, 0, L.total);
    CrtHeader *hd = reinterpret_cast<CrtHeader *>(h);
    SliceDesc *sd = reinterpret_cast<SliceDesc *>(h + L.sd);
    CrtGroup *gr = reinterpret_cast<CrtGroup *>(h + L.gr);
    size_t ne = 0;
    for (int i = 0; i < nA; ++i) ne += A[i].rows;
    for (int i = 0; i < nB; ++i) ne += B[i].cols;
    size_t qoff = exp_bytes((long long) ne) + maxbits_bytes((long long) ne + 1);
    for (int i = 0; i < nA; ++i)
        if (A[i].alias >= nB) return CA3DMM_EINVAL;
    for (int side = 0; side < 2; ++side) pl->kc_tiles[side] = pl->rc_tiles[side] = pl->exp_items[side] = 0;
    long long eoff = 0;
    for (int i = 0; i < nA + nB; ++i) {
        const bool isA = i < nA;
        const ca3dmm_oz_blk_t &b = isA ? A[i] : B[i - nA];
        const bool aliased = isA && b.alias >= 0;
        const int rows = aliased ? 0 : (isA ? b.rows : b.cols);
        const int kz = isA ? b.cols : b.rows;
        if (kz > CA3DMM_CRT_MAX_K) return CA3DMM_EINVAL;
        SliceDesc &d = sd[i];
        d.rows = rows;
        d.kz = kz;
        d.kpad = round_up(kz > 0 ? kz : 1, CKB);
        d.tile_rows = isA ? CBM : CBN;
        d.rows_pad = round_up(rows > 0 ? rows : 1, d.tile_rows);
        d.nkb = d.kpad / CKB;
        d.q_off = (long long) qoff;
        d.e_off = eoff;
        d.t_stride = (long long) d.rows_pad * d.kpad;
        d.nmod = nmod;
        d.p_bits = ca3dmm_crt_bits(nmod, kz);
        if (rows > 0 && d.p_bits < 2) return CA3DMM_EINVAL;
        const ca3dmm_oz_src_t &src = isA ? srcA[i] : srcB[i - nA];
        if (isA) {
            d.rs = src.trans ? src.ld : 1;
            d.ls = src.trans ? 1 : src.ld;
            d.src_off = (long long) b.r0 * d.rs + (long long) b.c0 * d.ls;
        } else {
            d.rs = src.trans ? 1 : src.ld;
            d.ls = src.trans ? src.ld : 1;
            d.src_off = (long long) b.c0 * d.rs + (long long) b.r0 * d.ls;
        }
        if (src.base) d.src_off += (long long) (reinterpret_cast<uintptr_t>(src.base) / sizeof(double));
        if (d.ls != 1 && d.rs != 1) return CA3DMM_EINVAL;
        d.shape = d.ls == 1 ? SHAPE_KC : SHAPE_RC;
        const int side = isA ? 0 : 1;
        d.kc_begin = pl->kc_tiles[side];
        d.rc_begin = pl->rc_tiles[side];
        d.xbegin = pl->exp_items[side];
        (d.shape == SHAPE_KC ? pl->kc_tiles : pl->rc_tiles)[side] += slice_tiles_of(d);
        pl->exp_items[side] += exp_items_of(d);
        qoff += rows > 0 ? align256((size_t) nmod * d.t_stride) : 0;
        eoff += rows;
    }
    int items = 0, pmin = 64, pmax = 0;
    long long recon = 0;
    for (int g = 0; g < ngroup; ++g) {
        CrtGroup &o = gr[g];
        if (G[g].a_blk < 0 || G[g].a_blk >= nA || G[g].b_blk < 0 || G[g].b_blk >= nB)
            return CA3DMM_EINVAL;
        const int al = A[G[g].a_blk].alias;
        const SliceDesc &da = al >= 0 ? sd[nA + al] : sd[G[g].a_blk], &db = sd[nA + G[g].b_blk];
        if (da.kz != db.kz || da.kz != G[g].k) return CA3DMM_EINVAL;
        o.C = G[g].C;
        o.ldc = G[g].ldc;
        o.m = G[g].m; o.n = G[g].n; o.k = G[g].k;
        o.a_desc = al >= 0 ? nA + al : G[g].a_blk;
        o.b_desc = nA + G[g].b_blk;
        o.a_from_b = al >= 0 ? 1 : 0;
        o.tiles_m = (o.m > 0 && o.n > 0) ? (o.m + CBM - 1) / CBM : 0;
        o.tile_n = G[g].tile_n == 128 ? 128 : CBN;
        if (o.tile_n != (G[0].tile_n == 128 ? 128 : CBN)) return CA3DMM_EINVAL;
        o.tiles_n = (o.m > 0 && o.n > 0) ? (o.n + o.tile_n - 1) / o.tile_n : 0;
        o.band = G[g].band > 0 ? G[g].band : DEFAULT_BAND;
        o.item_begin = items;
        o.rc_begin = recon;
        recon += (long long) ((o.m + 3) / 4) * (o.n > 0 ? o.n : 0);
        o.P = db.p_bits;
        o.nkb = o.k > 0 ? db.nkb : 0;
        o.ea_off = da.e_off;
        o.eb_off = db.e_off;
        o.qa_off = da.q_off;
        o.qb_off = db.q_off;
        o.qa_tstride = da.t_stride;
        o.qb_tstride = db.t_stride;
        o.pl_ld = round_up(o.m > 0 ? o.m : 1, CBM);
        o.pl_bytes = (long long) crt_plane_bytes(o.m, o.n);
        o.pl_off = (long long) qoff;
        qoff += align256((size_t) nmod * (size_t) o.pl_bytes);
        items += nmod * o.tiles_m * o.tiles_n;
        if (o.tiles_m > 0) {
            pmin = o.P < pmin ? o.P : pmin;
            pmax = o.P > pmax ? o.P : pmax;
        }
    }
    if (qoff > work_bytes) return CA3DMM_ENOMEM;
    hd->nmod = nmod; hd->nA = nA; hd->nB = nB; hd->ngroup = ngroup; hd->items = items;
    pl->nmod = nmod; pl->nA = nA; pl->nB = nB; pl->ngroup = ngroup; pl->items = items;
    pl->p_min = pmin > pmax ? 0 : pmin;
    pl->p_max = pmax;
    pl->n_exp = (long long) ne;
    pl->recon_items = recon;
    pl->tile_n = G[0].tile_n == 128 ? 128 : CBN;
    pl->group_m = ngroup == 1 ? gr[0].m : 0;
    pl->group_n = ngroup == 1 ? gr[0].n : 0;
    pl->dev_plan = dev_plan;
    pl->dev_work = dev_work;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_crt_group_items(const void *host_plan, int g, int tile_lo, int tile_hi,
                                      int *begin, int *count)
{
    const CrtHeader *hd = static_cast<const CrtHeader *>(host_plan);
    if (g < 0 || g >= hd->ngroup) return CA3DMM_EINVAL;
    const CrtLayout L(hd->nA + hd->nB, hd->ngroup);
    const CrtGroup &o = reinterpret_cast<const CrtGroup *>(static_cast<const unsigned char *>(host_plan) + L.gr)[g];
    const int lo = tile_lo < 0 ? 0 : tile_lo, hi = tile_hi > o.tiles_m ? o.tiles_m : tile_hi;
    if (hi <= lo) { *begin = o.item_begin; *count = 0; return CA3DMM_OK; }
    // a range of whole bands: tile_lo a multiple of the band (or the group's start)
    if (lo % o.band || (hi % o.band && hi != o.tiles_m)) return CA3DMM_EINVAL;
    *begin = o.item_begin + (lo / o.band) * hd->nmod * o.band * o.tiles_n;
    *count = hd->nmod * (hi - lo) * o.tiles_n;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_crt_clear(const ca3dmm_crt_plan_t *pl, cudaStream_t stream)
{
    CA3DMM_CUDA_TRY(cudaMemsetAsync(pl->dev_work, 0,
                                    exp_bytes(pl->n_exp) + maxbits_bytes(pl->n_exp + 1), stream));
    return CA3DMM_OK;
}

static int crt_exp(const ca3dmm_crt_plan_t *pl, const void *src, const SliceDesc *descs, int ndesc,
                   int nitems, cudaStream_t stream)
{
    if (ndesc <= 0 || nitems <= 0) return CA3DMM_OK;
    unsigned char *w = static_cast<unsigned char *>(pl->dev_work);
    unsigned long long *mwork = reinterpret_cast<unsigned long long *>(w + exp_bytes(pl->n_exp));
    const int cap = ca3dmm_device_sm_count() * 8;
    oz_exp_kernel<<<nitems < cap ? nitems : cap, 256, 0, stream>>>(
        static_cast<const double *>(src), descs, ndesc, nitems, mwork, mwork + pl->n_exp);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}

static int crt_residues(const ca3dmm_crt_plan_t *pl, const void *src, const SliceDesc *descs,
                        int ndesc, int nkc, int nrc, cudaStream_t stream)
{
    if (ndesc <= 0) return CA3DMM_OK;
    unsigned char *w = static_cast<unsigned char *>(pl->dev_work);
    const unsigned long long *mwork =
        reinterpret_cast<const unsigned long long *>(w + exp_bytes(pl->n_exp));
    const int cap = ca3dmm_device_sm_count() * 4;
    const double *x = static_cast<const double *>(src);
    switch (pl->nmod) {
#define CA3DMM_RES_CASE(N)                                                                          \
    case N:                                                                                         \
        if (nkc > 0) {                                                                              \
            slice_kc_kernel<ResidueWriter<N>><<<nkc < cap ? nkc : cap, 256, 0, stream>>>(          \
                x, descs, ndesc, nkc, w, mwork);                                                    \
            CA3DMM_CUDA_TRY(cudaGetLastError());                                                    \
            ca3dmm_note_launch(1);                                                                  \
        }                                                                                           \
        if (nrc > 0) {                                                                              \
            slice_rc_kernel<ResidueWriter<N>><<<nrc < cap ? nrc : cap, 256, 0, stream>>>(          \
                x, descs, ndesc, nrc, w, mwork);                                                    \
            CA3DMM_CUDA_TRY(cudaGetLastError());                                                    \
            ca3dmm_note_launch(1);                                                                  \
        }                                                                                           \
        break;
        CA3DMM_RES_CASE(8) CA3DMM_RES_CASE(9) CA3DMM_RES_CASE(10) CA3DMM_RES_CASE(11)
        CA3DMM_RES_CASE(12) CA3DMM_RES_CASE(13) CA3DMM_RES_CASE(14) CA3DMM_RES_CASE(15)
        CA3DMM_RES_CASE(16) CA3DMM_RES_CASE(17) CA3DMM_RES_CASE(18)
#undef CA3DMM_RES_CASE
        default: return CA3DMM_EINVAL;
    }
    return CA3DMM_OK;
}

static const SliceDesc *crt_descs(const ca3dmm_crt_plan_t *pl)
{
    const CrtLayout L(pl->nA + pl->nB, pl->ngroup);
    return reinterpret_cast<const SliceDesc *>(static_cast<const unsigned char *>(pl->dev_plan) + L.sd);
}

extern "C" int ca3dmm_crt_pack_side(const ca3dmm_crt_plan_t *pl, int which, const void *src,
                                    cudaStream_t stream)
{
    const SliceDesc *sd = crt_descs(pl);
    const SliceDesc *d = which ? sd + pl->nA : sd;
    const int nd = which ? pl->nB : pl->nA, side = which ? 1 : 0;
    int rc = crt_exp(pl, src, d, nd, pl->exp_items[side], stream);
    if (!rc) rc = crt_residues(pl, src, d, nd, pl->kc_tiles[side], pl->rc_tiles[side], stream);
    return rc;
}

extern "C" int ca3dmm_crt_run_pack(const ca3dmm_crt_plan_t *pl, const void *A, const void *B,
                                   cudaStream_t stream)
{
    const SliceDesc *sd = crt_descs(pl);
    int rc = ca3dmm_crt_clear(pl, stream);
    if (!rc) rc = crt_exp(pl, A, sd, pl->nA, pl->exp_items[0], stream);
    if (!rc) rc = crt_exp(pl, B, sd + pl->nA, pl->nB, pl->exp_items[1], stream);
    if (!rc) rc = crt_residues(pl, A, sd, pl->nA, pl->kc_tiles[0], pl->rc_tiles[0], stream);
    if (!rc) rc = crt_residues(pl, B, sd + pl->nA, pl->nB, pl->kc_tiles[1], pl->rc_tiles[1], stream);
    return rc;
}

static int crt_encode_list(const unsigned char *h, const SliceDesc *sd, int nsel,
                           const SliceDesc *sel_src, SliceDesc *out, int ntiles[3])
{
    (void) h; (void) sd;
    int kc = 0, rct = 0, items = 0;
    for (int i = 0; i < nsel; ++i) {
        SliceDesc c = sel_src[i];
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

extern "C" int ca3dmm_crt_encode_rows(const void *host_plan, int ngroup, const int *blocks,
                                      int count, int r0, int r1, void *out_descs, int ntiles[3])
{
    const CrtHeader *hd = static_cast<const CrtHeader *>(host_plan);
    (void) ngroup;
    const CrtLayout L(hd->nA + hd->nB, hd->ngroup);
    const unsigned char *h = static_cast<const unsigned char *>(host_plan);
    const SliceDesc *sd = reinterpret_cast<const SliceDesc *>(h + L.sd);
    if (!blocks || count < 0 || count > 64 || r0 < 0 || r1 < r0) return CA3DMM_EINVAL;
    SliceDesc sel[64];
    for (int i = 0; i < count; ++i) {
        if (blocks[i] < 0 || blocks[i] >= hd->nA) return CA3DMM_EINVAL;
        const SliceDesc &d = sd[blocks[i]];
        if (r0 % d.tile_rows) return CA3DMM_EINVAL;
        SliceDesc c = d;
        const int hi = r1 < d.rows ? r1 : d.rows;
        c.rows = hi > r0 ? hi - r0 : 0;
        c.rows_pad = round_up(c.rows > 0 ? c.rows : 1, d.tile_rows);
        if (c.rows == 0) c.rows_pad = 0;
        c.src_off = d.src_off + (long long) r0 * d.rs;
        c.q_off = d.q_off + (long long) (r0 / d.tile_rows) * d.nkb * d.tile_rows * CKB;
        c.e_off = d.e_off + r0;
        sel[i] = c;
    }
    return crt_encode_list(h, sd, count, sel, static_cast<SliceDesc *>(out_descs), ntiles);
}

extern "C" int ca3dmm_crt_encode_blocks(const void *host_plan, int ngroup, const int *descs,
                                        int count, void *out_descs, int ntiles[3])
{
    const CrtHeader *hd = static_cast<const CrtHeader *>(host_plan);
    (void) ngroup;
    const CrtLayout L(hd->nA + hd->nB, hd->ngroup);
    const unsigned char *h = static_cast<const unsigned char *>(host_plan);
    const SliceDesc *sd = reinterpret_cast<const SliceDesc *>(h + L.sd);
    if (!descs || count < 0 || count > 64) return CA3DMM_EINVAL;
    SliceDesc sel[64];
    for (int i = 0; i < count; ++i) {
        if (descs[i] < 0 || descs[i] >= hd->nA + hd->nB) return CA3DMM_EINVAL;
        sel[i] = sd[descs[i]];
    }
    return crt_encode_list(h, sd, count, sel, static_cast<SliceDesc *>(out_descs), ntiles);
}

extern "C" int ca3dmm_crt_pack_descs(const ca3dmm_crt_plan_t *pl, const void *src,
                                     const void *dev_descs, int ndesc, const int ntiles[3],
                                     cudaStream_t stream)
{
    const SliceDesc *d = static_cast<const SliceDesc *>(dev_descs);
    int rc = crt_exp(pl, src, d, ndesc, ntiles[0], stream);
    if (!rc) rc = crt_residues(pl, src, d, ndesc, ntiles[1], ntiles[2], stream);
    return rc;
}

extern "C" int ca3dmm_crt_run_gemm(const ca3dmm_crt_plan_t *pl, const ca3dmm_tile_ranges_t *rg_in,
                                   int *dev_status, double timeout_s, cudaStream_t stream)
{
    ca3dmm_tile_ranges_t rg;
    if (rg_in) {
        rg = *rg_in;
    } else {
        memset(&rg, 0, sizeof(rg));
        rg.n = 1;
        rg.len[0] = pl->items;
    }
    if (rg.n < 0 || rg.n > CA3DMM_MAX_RANGES) return CA3DMM_EINVAL;
    const int vitems = range_total(rg);
    if (vitems <= 0) return CA3DMM_OK;
    const CrtLayout L(pl->nA + pl->nB, pl->ngroup);
    const CrtGroup *groups =
        reinterpret_cast<const CrtGroup *>(static_cast<const unsigned char *>(pl->dev_plan) + L.gr);
    int grid = ca3dmm_device_sm_count();
    if (grid > vitems) grid = vitems;
    unsigned char *w = static_cast<unsigned char *>(pl->dev_work);
    const unsigned long long lim = (unsigned long long) (timeout_s * 1e9);
    if (pl->tile_n == 128) {
        const size_t smem = CrtTile<128>::kSmem;
        CA3DMM_CUDA_TRY(cudaFuncSetAttribute(crt_gemm_kernel<128>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        crt_gemm_kernel<128><<<grid, C_THREADS, smem, stream>>>(groups, pl->ngroup, pl->nmod, rg,
                                                                vitems, w, dev_status, lim);
    } else {
        const size_t smem = CrtTile<256>::kSmem;
        CA3DMM_CUDA_TRY(cudaFuncSetAttribute(crt_gemm_kernel<256>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        crt_gemm_kernel<256><<<grid, C_THREADS, smem, stream>>>(groups, pl->ngroup, pl->nmod, rg,
                                                                vitems, w, dev_status, lim);
    }
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}

extern "C" int ca3dmm_crt_run_reconstruct(const ca3dmm_crt_plan_t *pl, int g0, int g1, int r0,
                                          int r1, cudaStream_t stream)
{
    return ca3dmm_crt_run_reconstruct_capped(pl, g0, g1, r0, r1, 0, stream);
}

extern "C" int ca3dmm_crt_run_reconstruct_capped(const ca3dmm_crt_plan_t *pl, int g0, int g1,
                                                 int r0, int r1, int max_blocks,
                                                 cudaStream_t stream)
{
    if (g0 < 0) g0 = 0;
    if (g1 > pl->ngroup) g1 = pl->ngroup;
    if (g1 <= g0) return CA3DMM_OK;
    // several groups: all their rows; one group: a row window of it, the
    // items of the whole plan as the bound (the kernel skips the others)
    if (g1 - g0 > 1 && (g0 != 0 || g1 != pl->ngroup || r0 > 0 || r1 < 0x7fffffff))
        return CA3DMM_EINVAL;
    long long total = pl->recon_items;
    if (g1 - g0 == 1 && pl->ngroup == 1) {
        const long long hi = r1 < pl->group_m ? r1 : pl->group_m, lo = r0 > 0 ? r0 : 0;
        total = hi > lo ? ((hi - lo + 3) / 4) * pl->group_n : 0;
    }
    const CrtLayout L(pl->nA + pl->nB, pl->ngroup);
    const CrtGroup *groups =
        reinterpret_cast<const CrtGroup *>(static_cast<const unsigned char *>(pl->dev_plan) + L.gr);
    const unsigned char *w = static_cast<const unsigned char *>(pl->dev_work);
    if (total <= 0) return CA3DMM_OK;
    long long blocks = (total + 255) / 256;
    const long long cap = max_blocks > 0 ? max_blocks : (long long) ca3dmm_device_sm_count() * 8;
    if (blocks > cap) blocks = cap;
    // the same shared-memory carveout as the GEMM, so that blocks of this
    // kernel can share an SM with a GEMM CTA running beside it (a kernel
    // attribute of each device: set once per instantiation, device and
    // process; a bit per device ordinal below 64, set atomically, as ranks
    // that are threads of one process may drive several devices)
    static unsigned long long carveout_set[MAXMOD + 1] = {};
    int dev = 0;
    CA3DMM_CUDA_TRY(cudaGetDevice(&dev));
    const unsigned long long dbit = dev < 64 ? 1ull << dev : 0ull;
    switch (pl->nmod) {
#define CA3DMM_CRT_CASE(N)                                                                          \
    case N:                                                                                         \
        if (!(__atomic_load_n(&carveout_set[N], __ATOMIC_ACQUIRE) & dbit)) {                        \
            CA3DMM_CUDA_TRY(cudaFuncSetAttribute(crt_reconstruct_kernel<N, crt_limbs(N)>,          \
                                                 cudaFuncAttributePreferredSharedMemoryCarveout,  \
                                                 (int) cudaSharedmemCarveoutMaxShared));          \
            __atomic_fetch_or(&carveout_set[N], dbit, __ATOMIC_RELEASE);                            \
        }                                                                                           \
        crt_reconstruct_kernel<N, crt_limbs(N)><<<(unsigned) blocks, 256, 0, stream>>>(            \
            groups, g0, g1, r0, r1, total, w);                                                     \
        break;
        CA3DMM_CRT_CASE(8) CA3DMM_CRT_CASE(9) CA3DMM_CRT_CASE(10) CA3DMM_CRT_CASE(11)
        CA3DMM_CRT_CASE(12) CA3DMM_CRT_CASE(13) CA3DMM_CRT_CASE(14) CA3DMM_CRT_CASE(15)
        CA3DMM_CRT_CASE(16) CA3DMM_CRT_CASE(17) CA3DMM_CRT_CASE(18)
#undef CA3DMM_CRT_CASE
        default: return CA3DMM_EINVAL;
    }
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}

extern "C" int ca3dmm_crt_run_nonfinite(const ca3dmm_crt_plan_t *pl, int g0, int g1, int r0,
                                        int r1, const void *A, const void *B, cudaStream_t stream)
{
    if (g0 < 0) g0 = 0;
    if (g1 > pl->ngroup) g1 = pl->ngroup;
    if (g1 <= g0) return CA3DMM_OK;
    if (g1 - g0 > 65535) return CA3DMM_EINVAL;
    const CrtLayout L(pl->nA + pl->nB, pl->ngroup);
    const unsigned char *p = static_cast<const unsigned char *>(pl->dev_plan);
    const unsigned long long *mwork = reinterpret_cast<const unsigned long long *>(
        static_cast<const unsigned char *>(pl->dev_work) + exp_bytes(pl->n_exp));
    const int per = (ca3dmm_device_sm_count() * 2 + (g1 - g0) - 1) / (g1 - g0);
    dim3 grid((unsigned) (per > 1 ? per : 1), (unsigned) (g1 - g0));
    crt_nonfinite_kernel<<<grid, 256, 0, stream>>>(
        static_cast<const double *>(A), static_cast<const double *>(B),
        reinterpret_cast<const SliceDesc *>(p + L.sd), pl->nA,
        reinterpret_cast<const CrtGroup *>(p + L.gr), g0, r0, r1, mwork, mwork + pl->n_exp);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    return CA3DMM_OK;
}
