// Device code shared by the two split-precision GEMMs (k_ozaki.cu: INT8
// slices, k_crt.cu: INT8 residues of a modular scheme): the slicing
// descriptor, the per-row exponent pass, the two slicing kernels (templated on
// the writer that turns 16 consecutive elements of a row into operand bytes)
// and the tcgen05 / TMEM helpers.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>
#include "k_common.cuh"

namespace {

constexpr int EXP_BIAS = 2048;                   // stored exponent = E + bias, 0 = all-zero row
// |x| bit patterns at or above this are Inf (equal) or NaN (above)
constexpr unsigned long long INF_BITS = 0x7ff0000000000000ull;

// Slicing descriptor: block rows r in [0,rows), k index l in [0,kz);
// element (r,l) at src[src_off + r*rs + l*ls].  Exactly one of rs, ls is 1
// for a column-major source (both when ld = 1): shape KC reads along k, RC
// along rows.
struct SliceDesc {
    long long src_off, rs, ls;
    long long q_off;        // byte offset of the block's tiled slices in the work region
    long long e_off;        // int offset of the exponents in the work region
    int rows, kz, kpad;     // kpad = kz rounded up to the GEMM's k block (32 or 128 bytes)
    int rows_pad, tile_rows, nkb;   // rows rounded up to tile_rows (slices: 128 for A, 64 for B;
                                    // residues: 128 for A, 256 for B)
    int kc_begin, rc_begin; // first slicing tile of this block among the KC / RC tiles of its operand
    int xbegin;             // first exponent work item of this block (per operand)
    int shape;              // SHAPE_KC or SHAPE_RC
    // modular scheme only: bytes per modulus of the block's residues, integer width, moduli
    long long t_stride;
    int p_bits, nmod;
};

// ------------------------------------------------------------------ slicing
constexpr int ST = 64;   // exponent tile edge of the RC shape (rows x k)
constexpr int SHAPE_KC = 1, SHAPE_RC = 2;
// KC (k contiguous): exponent items of 8 rows x 512 k (a warp reads 4 KB of one
// row), slicing tiles of 16 rows x 256 k (a thread reads its own 16 k).
// RC (rows contiguous): exponent tiles of 64 rows x 64 k, slicing tiles of
// 128 rows x 32 k (one k-block) transposed through shared memory.
// Long contiguous runs per warp matter on B200: 512-byte row pieces 8 MB apart
// read at half the rate of 4 KB runs.
constexpr int KC_XR = 8, KC_XK = 512, KC_SR = 16, KC_SK = 256;
constexpr int RC_SR = 128, RC_SK = 32;

__host__ __device__ inline int exp_items_of(const SliceDesc &d)
{
    if (d.rows <= 0 || d.kz <= 0) return 0;
    if (d.shape == SHAPE_KC) return ((d.rows + KC_XR - 1) / KC_XR) * ((d.kz + KC_XK - 1) / KC_XK);
    return ((d.rows + ST - 1) / ST) * ((d.kz + ST - 1) / ST);
}

__host__ __device__ inline int slice_tiles_of(const SliceDesc &d)
{
    if (d.rows <= 0 || d.kz <= 0) return 0;
    if (d.shape == SHAPE_KC) return ((d.rows_pad + KC_SR - 1) / KC_SR) * ((d.kpad + KC_SK - 1) / KC_SK);
    return ((d.rows_pad + RC_SR - 1) / RC_SR) * ((d.kpad + RC_SK - 1) / RC_SK);
}

// Which numbering a search runs over: exponent items, KC or RC slicing tiles.
constexpr int FIND_EXP = 0;

__device__ __forceinline__ int desc_begin(const SliceDesc &d, int which)
{
    return which == SHAPE_KC ? d.kc_begin : which == SHAPE_RC ? d.rc_begin : d.xbegin;
}

// The descriptor holding flat item t: the last one whose first item is <= t
// (blocks without items in this numbering share their first item with the next).
// The slicing kernels copy the first items of up to DESC_CACHE descriptors
// into shared memory once, so that the search per tile is not a chain of
// dependent global loads (a batch of 256 GEMMs has 256 descriptors per side).
constexpr int DESC_CACHE = 1024;

struct DescFinder {
    int *begin;      // shared copy, or nullptr when there are more descriptors than DESC_CACHE
    __device__ __forceinline__ int operator()(const SliceDesc *d, int n, int t, int which) const
    {
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if ((begin ? begin[mid] : desc_begin(d[mid], which)) <= t) lo = mid; else hi = mid - 1;
        }
        return lo;
    }
};

// Fill the shared copy (every thread of the block calls this once, before its loop).
__device__ __forceinline__ DescFinder make_finder(int *sbeg, const SliceDesc *d, int n, int which)
{
    DescFinder f;
    f.begin = n <= DESC_CACHE ? sbeg : nullptr;
    if (f.begin)
        for (int i = threadIdx.x; i < n; i += blockDim.x) sbeg[i] = desc_begin(d[i], which);
    __syncthreads();
    return f;
}

__device__ __forceinline__ const double *slice_src(const double *base, long long off)
{
    // with a NULL base the offset is an absolute address / 8 (batched sources)
    return reinterpret_cast<const double *>(reinterpret_cast<uintptr_t>(base) +
                                            (uintptr_t) off * sizeof(double));
}

// Work region: [E + EXP_BIAS per row, int][max |x| per row as its IEEE bit
// pattern, u64; then one u64 set when any row holds an Inf or a NaN][tiled
// slices].  Both prefix arrays are cleared before a run.
__host__ __device__ inline size_t exp_bytes(long long n_exp)
{
    return ((size_t) n_exp * sizeof(int) + 255) / 256 * 256;
}
__host__ __device__ inline size_t maxbits_bytes(long long n_exp)
{
    return ((size_t) n_exp * sizeof(unsigned long long) + 255) / 256 * 256;
}

__device__ __forceinline__ unsigned long long abs_bits(double x)
{
    return (unsigned long long) __double_as_longlong(x) & 0x7fffffffffffffffull;
}

// Pass 1, persistent over the flat list of exponent items of every block: per
// row, the largest |x| as its bit pattern (for non-negative doubles the bit
// pattern orders like the value).  The effective exponent
// E(x) = min{E : |x| <= 2^E 127/128} is non-decreasing in |x|, so the row's
// exponent max_l E(x_l) is E(max_l |x_l|), formed once per row in pass 2.
__global__ void __launch_bounds__(256)
oz_exp_kernel(const double *__restrict__ src, const SliceDesc *__restrict__ descs, int ndesc,
              int total_items, unsigned long long *__restrict__ mwork,
              unsigned long long *__restrict__ nonfinite)
{
    __shared__ unsigned long long part[4][ST];
    __shared__ int sbeg[DESC_CACHE];
    const DescFinder find = make_finder(sbeg, descs, ndesc, FIND_EXP);
    for (int item = blockIdx.x; item < total_items; item += gridDim.x) {
        const SliceDesc &d = descs[find(descs, ndesc, item, FIND_EXP)];
        const int local = item - d.xbegin;
        if (d.shape == SHAPE_KC) {
            // warp w: row r0 + w, k [l0, l0 + 512) as 16-byte loads (scalar when unaligned)
            const int nkr = (d.kz + KC_XK - 1) / KC_XK, lane = threadIdx.x & 31;
            const int r = (local / nkr) * KC_XR + (threadIdx.x >> 5), l0 = (local % nkr) * KC_XK;
            unsigned long long m = 0;
            if (r < d.rows) {
                const double *row = slice_src(src, d.src_off) + (long long) r * d.rs + l0;
                const int ln = d.kz - l0;
                if (!(reinterpret_cast<uintptr_t>(row) & 15) && ln >= KC_XK) {
                    double2 v[KC_XK / 64];
#pragma unroll
                    for (int i = 0; i < KC_XK / 64; ++i)
                        v[i] = __ldg(reinterpret_cast<const double2 *>(row) + lane + 32 * i);
#pragma unroll
                    for (int i = 0; i < KC_XK / 64; ++i) {
                        const unsigned long long a = abs_bits(v[i].x), b = abs_bits(v[i].y);
                        m = a > m ? a : m;
                        m = b > m ? b : m;
                    }
                } else {
                    double v[KC_XK / 32];
#pragma unroll
                    for (int i = 0; i < KC_XK / 32; ++i) {
                        const int l = lane + 32 * i;
                        v[i] = l < ln ? __ldg(row + l) : 0.0;
                    }
#pragma unroll
                    for (int i = 0; i < KC_XK / 32; ++i) {
                        const unsigned long long a = abs_bits(v[i]);
                        m = a > m ? a : m;
                    }
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long w = __shfl_xor_sync(0xffffffffu, m, o);
                m = w > m ? w : m;
            }
            if (lane == 0 && r < d.rows && m) {
                atomicMax(mwork + d.e_off + r, m);
                if (m >= INF_BITS) *nonfinite = 1ull;
            }
            continue;
        }
        // RC: 64 x 64 tile, thread (row r, k phase g) walks k = g, g + 4, ...
        const int tx = (d.rows + ST - 1) / ST;
        const int r0 = (local % tx) * ST, l0 = (local / tx) * ST;
        const int rn = min(ST, d.rows - r0), ln = min(ST, d.kz - l0);
        const double *base = slice_src(src, d.src_off) + r0 + (long long) l0 * d.ls;
        const int r = threadIdx.x & (ST - 1), g = threadIdx.x >> 6;
        unsigned long long m = 0;
        if (r < rn) {
#pragma unroll
            for (int j = 0; j < ST / 4; ++j) {
                const int l = g + 4 * j;
                if (l < ln) {
                    const unsigned long long v = abs_bits(__ldg(base + r + (long long) l * d.ls));
                    m = v > m ? v : m;
                }
            }
        }
        __syncthreads();                             // part[] of the previous tile is read
        part[g][r] = m;
        __syncthreads();
        if (threadIdx.x < rn) {
            unsigned long long v = part[0][threadIdx.x];
#pragma unroll
            for (int q = 1; q < 4; ++q) v = part[q][threadIdx.x] > v ? part[q][threadIdx.x] : v;
            if (v) atomicMax(mwork + d.e_off + r0 + threadIdx.x, v);
            if (v >= INF_BITS) *nonfinite = 1ull;
        }
    }
}

// Pass 2 over the flat list of slicing tiles of one shape (padding rows and k
// included: they hold zero digits).  W::write16 turns one row's 16
// consecutive k elements into the operand bytes of the GEMM that follows
// (INT8 slices, or residues modulo the moduli of the modular scheme);
// W::kMinBlocks is the occupancy the kernel is compiled for.
//
// KC: 16 rows x 256 k per tile.  Warp w loads rows 2w and 2w + 1 with
// coalesced 16-byte loads (512 contiguous bytes per instruction), the tile is
// staged in shared memory as 16-k chunks (slots 144 bytes apart, rows padded by
// 32 bytes, so the 16-byte accesses of every quarter-warp hit distinct banks),
// and warp w slices k-block w: lane (row lane / 2, chunk 2w + lane % 2), so each
// slice's stores from a warp cover 512 contiguous bytes.  Measured 15 % faster
// than each thread loading its own 128 bytes from global memory, and another 6 %
// over slicing one chunk per thread in row order.
constexpr int KC_SLOT = 18;                           // doubles per staged chunk (16 + 2 of padding)
constexpr int KC_ROW = (KC_SK / 16) * KC_SLOT + 4;    // doubles per staged row
template <class W>
__global__ void __launch_bounds__(256, W::kMinBlocks)
slice_kc_kernel(const double *__restrict__ src, const SliceDesc *__restrict__ descs, int ndesc,
                   int total_tiles, unsigned char *__restrict__ work,
                   const unsigned long long *__restrict__ mwork)
{
    __shared__ __align__(16) double sm[KC_SR * KC_ROW];
    __shared__ int sbeg[DESC_CACHE];
    const DescFinder find = make_finder(sbeg, descs, ndesc, SHAPE_KC);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
        const SliceDesc &d = descs[find(descs, ndesc, tile, SHAPE_KC)];
        const int local = tile - d.kc_begin;
        const int nkt = (d.kpad + KC_SK - 1) / KC_SK;
        const int r0 = (local / nkt) * KC_SR, l0 = (local % nkt) * KC_SK;
        const double *base = slice_src(src, d.src_off);
        // 16-byte piece q = lane + 32 j (j < 4) of row 2w + h: k offset 2q
        double2 v[8];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = r0 + 2 * w + h;
            const double *row = base + (long long) r * d.rs + l0;
            const bool al = !(reinterpret_cast<uintptr_t>(row) & 15);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int l = 2 * (lane + 32 * j);
                if (r < d.rows && al && l0 + l + 1 < d.kz) {
                    v[4 * h + j] = __ldg(reinterpret_cast<const double2 *>(row + l));
                } else {
                    v[4 * h + j].x = (r < d.rows && l0 + l < d.kz) ? __ldg(row + l) : 0.0;
                    v[4 * h + j].y = (r < d.rows && l0 + l + 1 < d.kz) ? __ldg(row + l + 1) : 0.0;
                }
            }
        }
        __syncthreads();                             // sm of the previous tile is read
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int q = lane + 32 * j;
                *reinterpret_cast<double2 *>(
                    &sm[(2 * w + h) * KC_ROW + (q >> 3) * KC_SLOT + 2 * (q & 7)]) = v[4 * h + j];
            }
        __syncthreads();
        const int rr = lane >> 1, c = 2 * w + (lane & 1);
        const int gr = r0 + rr, gl = l0 + 16 * c;
        if (gr >= d.rows_pad || gl >= d.kpad) continue;
        const double2 *slot = reinterpret_cast<const double2 *>(&sm[rr * KC_ROW + c * KC_SLOT]);
        double x[16];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const double2 t = slot[i];
            x[2 * i] = t.x;
            x[2 * i + 1] = t.y;
        }
        W::write16(d, work, mwork, gr, gl, x);
    }
}

template <class W>
__global__ void __launch_bounds__(256, W::kMinBlocks)
slice_rc_kernel(const double *__restrict__ src, const SliceDesc *__restrict__ descs, int ndesc,
                   int total_tiles, unsigned char *__restrict__ work,
                   const unsigned long long *__restrict__ mwork)
{
    __shared__ __align__(16) double tl[RC_SK][RC_SR];
    __shared__ int sbeg[DESC_CACHE];
    const DescFinder find = make_finder(sbeg, descs, ndesc, SHAPE_RC);
    for (int tile = blockIdx.x; tile < total_tiles; tile += gridDim.x) {
        const SliceDesc &d = descs[find(descs, ndesc, tile, SHAPE_RC)];
        const int local = tile - d.rc_begin;
        // 128 rows x 32 k; thread (row pair tid % 64, k column tid / 64 + 4 i)
        // loads 16 bytes of a column, the tile is transposed through shared memory
        const int ntr = (d.rows_pad + RC_SR - 1) / RC_SR;
        const int r0 = (local % ntr) * RC_SR, l0 = (local / ntr) * RC_SK;
        const int rp = threadIdx.x & 63, cg = threadIdx.x >> 6;
        const double *base = slice_src(src, d.src_off) + r0 + (long long) l0 * d.ls;
        const int rn = d.rows - r0, ln = d.kz - l0;
        double2 v[8];
        if (!(reinterpret_cast<uintptr_t>(base) & 15) && !(d.ls & 1) && rn >= RC_SR && ln >= RC_SK) {
#pragma unroll
            for (int i = 0; i < 8; ++i)
                v[i] = __ldg(reinterpret_cast<const double2 *>(base + (long long) (cg + 4 * i) * d.ls) + rp);
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int l = cg + 4 * i;
                const double *c = base + (long long) l * d.ls + 2 * rp;
                v[i].x = (l < ln && 2 * rp < rn) ? __ldg(c) : 0.0;
                v[i].y = (l < ln && 2 * rp + 1 < rn) ? __ldg(c + 1) : 0.0;
            }
        }
        __syncthreads();                             // tl of the previous tile is read
#pragma unroll
        for (int i = 0; i < 8; ++i) reinterpret_cast<double2 *>(&tl[cg + 4 * i][0])[rp] = v[i];
        __syncthreads();
        // warp w: rows 16 w .. 16 w + 15, both 16-k chunks (lane: row lane / 2,
        // chunk lane % 2): each slice's stores from a warp cover 512 contiguous bytes
        const int r = 16 * (threadIdx.x >> 5) + ((threadIdx.x & 31) >> 1), c = (threadIdx.x & 1) * 16;
        const int gr = r0 + r, gl = l0 + c;
        if (gr >= d.rows_pad || gl >= d.kpad) continue;
        double x[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) x[j] = tl[c + j][r];
        W::write16(d, work, mwork, gr, gl, x);
    }
}

// Contiguous global -> shared bulk copy completing on an mbarrier.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
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

// K-major, SWIZZLE_32B shared-memory operand descriptor: rows of 32 bytes,
// 8-row groups 256 bytes apart (SBO), descriptor version 1, layout type 6.
__device__ __forceinline__ uint64_t sdesc_k32(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t) ((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t) 1 << 16;                 // LBO (unused for swizzled K-major)
    d |= (uint64_t) (256 >> 4) << 32;        // SBO
    d |= (uint64_t) 1 << 46;                 // descriptor version (sm_100)
    d |= (uint64_t) 6 << 61;                 // SWIZZLE_32B
    return d;
}

// Instruction descriptor: S32 accumulator, A and B signed 8-bit, both
// K-major, M = m (128 per CTA), N = n.
__device__ __forceinline__ uint32_t idesc_i8(int n, int m = 128)
{
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (n >> 3) << 17) |
           ((uint32_t) (m >> 4) << 24);
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
          "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]),
          "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]),
          "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Zero 32 consecutive TMEM columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_zero32(uint32_t taddr)
{
    const uint32_t z = 0;
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
        "%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
        "r"(z)
        : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Exact int32 -> double without the conversion unit: the double with high word
// 0x43300000 and low word v ^ 2^31 is 2^52 + v + 2^31.
__device__ __forceinline__ double i32_to_f64(uint32_t v)
{
    return __hiloint2double(0x43300000, (int) (v ^ 0x80000000u)) - 4503601774854144.0;
}

// 2^e as a double: built from the exponent bits in the normal range (exact),
// ldexp outside it.
__device__ __forceinline__ double pow2(int e)
{
    if (e >= -1022 && e <= 1023) return __longlong_as_double((long long) (e + 1023) << 52);
    return ldexp(1.0, e);
}

// x 2^e with one rounding (exact unless the result leaves the normal range):
// a multiplication by the exact power of two where 2^e is a normal double,
// ldexp beyond that.
__device__ __forceinline__ double scale2(double x, int e)
{
    if (e >= -1022 && e <= 1023) return x * __longlong_as_double((long long) (e + 1023) << 52);
    return ldexp(x, e);
}

// Which IEEE value a product a * b takes when a factor is not finite:
// 1 NaN, 2 +Inf, 4 -Inf, 0 finite.
__device__ __forceinline__ int product_class(double a, double b)
{
    if (isnan(a) || isnan(b)) return 1;
    if (isinf(a) || isinf(b)) {
        if (a == 0.0 || b == 0.0) return 1;
        return signbit(a) != signbit(b) ? 4 : 2;
    }
    return 0;
}

}  // namespace
