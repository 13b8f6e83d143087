// Accuracy guard of the autotuner: the error of a candidate's C on a sample
// of entries, against a Dot2 (compensated, twice-working-precision) value of
// each sampled entry computed from the operands.
//
// Sample: half of the rows of op(A) (columns of op(B)) are the ones whose
// largest entry stands furthest above their mean magnitude -- the rows where
// rounding the operands to P bits below the row maximum loses the most --
// and half are evenly spaced over the matrix.  Per entry the guard keeps the
// Dot2 value T and sum_l |a_il| |b_lj|, so that a candidate's C gives
//   normwise     sum |C - T| / sum |T|,
//   componentwise max |C - T| / (|A| |B|)_ij
// over the sample.  Dot2 is the compensated dot product of Ogita, Rump and
// Oishi (SIAM J. Sci. Comput. 26(6), 2005): TwoProduct by FMA, TwoSum of the
// running sum, the error terms summed separately.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include "k_common.cuh"
#include "ca3dmm_kernels.h"
#include "ca3dmm_tune_guard.h"

namespace {

constexpr int STAT_CHUNK = 2048;   // k per statistics thread

// per row r of X (element (r, l) at X[r rs + l ls]) and k chunk c:
// max |x|, sum |x|, min nonzero |x|
__global__ void __launch_bounds__(256)
guard_stats_kernel(const double *__restrict__ X, long long rs, long long ls, int R, int K,
                   double *__restrict__ pmax, double *__restrict__ psum,
                   double *__restrict__ pmin, int *__restrict__ nonfinite)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const int c = blockIdx.y;
    if (r >= R) return;
    const int l0 = c * STAT_CHUNK, l1 = min(K, l0 + STAT_CHUNK);
    double mx = 0.0, sm = 0.0, mn = INFINITY;
    bool bad = false;
    const double *x = X + (long long) r * rs;
#pragma unroll 4
    for (int l = l0; l < l1; ++l) {
        const double v = fabs(x[(long long) l * ls]);
        bad |= !(v <= 1.79769313486231570815e308);   // Inf or NaN
        mx = v > mx ? v : mx;
        sm += v;
        if (v > 0.0 && v < mn) mn = v;
    }
    const long long o = (long long) c * R + r;
    pmax[o] = mx;
    psum[o] = sm;
    pmin[o] = mn;
    if (bad) atomicOr(nonfinite, 1);
}

// partial statistics over the k chunks, in chunk order (deterministic)
__global__ void guard_stats_reduce(const double *__restrict__ pmax, const double *__restrict__ psum,
                                   const double *__restrict__ pmin, int R, int nchunk,
                                   double *__restrict__ out)   // [3][R]
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= R) return;
    double mx = 0.0, sm = 0.0, mn = INFINITY;
    for (int c = 0; c < nchunk; ++c) {
        const long long o = (long long) c * R + r;
        mx = pmax[o] > mx ? pmax[o] : mx;
        sm += psum[o];
        mn = pmin[o] < mn ? pmin[o] : mn;
    }
    out[r] = mx;
    out[R + r] = sm;
    out[2 * R + r] = mn;
}

__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e)
{
    s = a + b;
    const double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

// one warp per sampled entry: lanes take every 32nd l, then the lanes'
// (sum, error) pairs are added with TwoSum
__global__ void __launch_bounds__(256)
guard_truth_kernel(const double *__restrict__ A, long long a_rs, long long a_ls,
                   const double *__restrict__ B, long long b_rs, long long b_ls, int K,
                   const int *__restrict__ rows, int nr, const int *__restrict__ cols, int nc,
                   double *__restrict__ truth, double *__restrict__ absprod)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= nr * nc) return;
    const int i = rows[warp % nr], j = cols[warp / nr];
    const double *a = A + (long long) i * a_rs;
    const double *b = B + (long long) j * b_rs;
    double s = 0.0, c = 0.0, ab = 0.0;
    for (int l = lane; l < K; l += 32) {
        const double x = a[(long long) l * a_ls], y = b[(long long) l * b_ls];
        const double p = x * y;
        const double pe = fma(x, y, -p);
        double t, te;
        two_sum(s, p, t, te);
        s = t;
        c += te + pe;
        ab += fabs(p);
    }
    for (int off = 16; off > 0; off >>= 1) {
        const double s2 = __shfl_down_sync(0xffffffffu, s, off);
        const double c2 = __shfl_down_sync(0xffffffffu, c, off);
        const double ab2 = __shfl_down_sync(0xffffffffu, ab, off);
        double t, te;
        two_sum(s, s2, t, te);
        s = t;
        c += c2 + te;
        ab += ab2;
    }
    if (lane == 0) {
        truth[warp] = s + c;
        absprod[warp] = ab;
    }
}

// out[0] = sum |C - T|, out[1] = max |C - T| / (|A||B|), out[2] = 1 if any
// difference is not finite (one block)
__global__ void __launch_bounds__(256)
guard_error_kernel(const double *__restrict__ C, long long ldc, const int *__restrict__ rows,
                   int nr, const int *__restrict__ cols, int nc, const double *__restrict__ truth,
                   const double *__restrict__ absprod, double *__restrict__ out)
{
    __shared__ double s_sum[256], s_max[256];
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    double sm = 0.0, mx = 0.0;
    bool bad = false;
    for (int e = threadIdx.x; e < nr * nc; e += blockDim.x) {
        const int i = rows[e % nr], j = cols[e / nr];
        const double d = fabs(C[i + (long long) j * ldc] - truth[e]);
        if (!(d <= 1.79769313486231570815e308)) {
            bad = true;
            continue;
        }
        sm += d;
        const double ap = absprod[e];
        const double r = ap > 0.0 ? d / ap : (d > 0.0 ? INFINITY : 0.0);
        mx = r > mx ? r : mx;
    }
    if (bad) atomicOr(&s_bad, 1);
    s_sum[threadIdx.x] = sm;
    s_max[threadIdx.x] = mx;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int) threadIdx.x < w) {
            s_sum[threadIdx.x] += s_sum[threadIdx.x + w];
            s_max[threadIdx.x] = fmax(s_max[threadIdx.x], s_max[threadIdx.x + w]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s_sum[0];
        out[1] = s_max[0];
        out[2] = s_bad ? 1.0 : 0.0;
    }
}

// rows of X (R rows over K): statistics to the host
int row_stats(const double *X, long long rs, long long ls, int R, int K, std::vector<double> &st,
              int *d_flag, cudaStream_t stream)
{
    const int nchunk = (K + STAT_CHUNK - 1) / STAT_CHUNK;
    double *d = nullptr;
    const size_t np = (size_t) nchunk * R;
    CA3DMM_CUDA_TRY(cudaMalloc(&d, sizeof(double) * (3 * np + 3 * (size_t) R)));
    double *out = d + 3 * np;
    dim3 grid((R + 255) / 256, nchunk);
    guard_stats_kernel<<<grid, 256, 0, stream>>>(X, rs, ls, R, K, d, d + np, d + 2 * np, d_flag);
    guard_stats_reduce<<<(R + 255) / 256, 256, 0, stream>>>(d, d + np, d + 2 * np, R, nchunk, out);
    ca3dmm_note_launch(2);
    st.resize(3 * (size_t) R);
    cudaError_t err = cudaMemcpyAsync(st.data(), out, sizeof(double) * 3 * R,
                                      cudaMemcpyDeviceToHost, stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(stream);
    cudaFree(d);
    CA3DMM_CUDA_TRY(err);
    return CA3DMM_OK;
}

// the sample: the `half` highest scores (max |x| K / sum |x|), then evenly
// spaced indices, distinct, ascending
std::vector<int> pick(const std::vector<double> &st, int R, int K, int want)
{
    std::vector<int> idx;
    if (want >= R) {
        for (int i = 0; i < R; ++i) idx.push_back(i);
        return idx;
    }
    std::vector<std::pair<double, int>> sc((size_t) R);
    for (int i = 0; i < R; ++i) {
        const double mx = st[i], sm = st[R + i];
        sc[i] = {sm > 0.0 ? mx * (double) K / sm : 0.0, i};
    }
    const int half = want / 2;
    std::partial_sort(sc.begin(), sc.begin() + half, sc.end(),
                      [](const std::pair<double, int> &x, const std::pair<double, int> &y) {
                          return x.first > y.first || (x.first == y.first && x.second < y.second);
                      });
    std::vector<char> used((size_t) R, 0);
    for (int h = 0; h < half; ++h) {
        idx.push_back(sc[h].second);
        used[sc[h].second] = 1;
    }
    const int rest = want - half;
    for (int t = 0; t < rest; ++t) {
        const int i = (int) (((long long) (2 * t + 1) * R) / (2LL * rest));
        if (!used[i]) {
            idx.push_back(i);
            used[i] = 1;
        }
    }
    for (int q = 0; (int) idx.size() < want && q < R; ++q)
        if (!used[q]) {
            idx.push_back(q);
            used[q] = 1;
        }
    std::sort(idx.begin(), idx.end());
    return idx;
}

}  // namespace

static int guard_build(ca3dmm_guard_t *g, int m, int n, int k, int trans_A, int trans_B,
                       const double *A, int ldA, const double *B, int ldB, int samples,
                       void *stream_);

extern "C" int ca3dmm_guard_create(ca3dmm_guard_t *g, int m, int n, int k, int trans_A,
                                   int trans_B, const double *A, int ldA, const double *B,
                                   int ldB, int samples, void *stream_)
{
    if (!g) return CA3DMM_EINVAL;
    memset(g, 0, sizeof(*g));
    const int rc = guard_build(g, m, n, k, trans_A, trans_B, A, ldA, B, ldB, samples, stream_);
    if (rc) ca3dmm_guard_free(g);        /* nothing half-made stays allocated */
    return rc;
}

static int guard_build(ca3dmm_guard_t *g, int m, int n, int k, int trans_A, int trans_B,
                       const double *A, int ldA, const double *B, int ldB, int samples,
                       void *stream_)
{
    if (m < 1 || n < 1 || k < 1 || !A || !B || samples < 2) return CA3DMM_EINVAL;
    cudaStream_t stream = (cudaStream_t) stream_;
    g->m = m; g->n = n; g->k = k;
    // op(A)(i, l) and op(B)(l, j) as rows of a strided matrix
    const long long a_rs = trans_A ? ldA : 1, a_ls = trans_A ? 1 : ldA;
    const long long b_rs = trans_B ? 1 : ldB, b_ls = trans_B ? ldB : 1;
    int *d_flag = nullptr;
    CA3DMM_CUDA_TRY(cudaMalloc(&d_flag, sizeof(int)));
    CA3DMM_CUDA_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int), stream));
    std::vector<double> sa, sb;
    int rc = row_stats(A, a_rs, a_ls, m, k, sa, d_flag, stream);
    if (!rc) rc = row_stats(B, b_rs, b_ls, n, k, sb, d_flag, stream);
    int flag = 0;
    if (!rc && cudaMemcpy(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        rc = CA3DMM_ECUDA;
    cudaFree(d_flag);
    if (rc) return rc;
    g->nonfinite = flag;
    double mx = 0.0, mn = INFINITY;
    for (int i = 0; i < m; ++i) { mx = std::max(mx, sa[i]); mn = std::min(mn, sa[2 * (size_t) m + i]); }
    for (int j = 0; j < n; ++j) { mx = std::max(mx, sb[j]); mn = std::min(mn, sb[2 * (size_t) n + j]); }
    g->spread = (mx > 0.0 && mn < INFINITY) ? (float) std::log2(mx / mn) : 0.f;
    const std::vector<int> ri = pick(sa, m, k, samples), ci = pick(sb, n, k, samples);
    g->nr = (int) ri.size();
    g->nc = (int) ci.size();
    const size_t ne = (size_t) g->nr * g->nc;
    void *mem = nullptr;
    CA3DMM_CUDA_TRY(cudaMalloc(&mem, sizeof(int) * (ri.size() + ci.size()) + sizeof(double) * (2 * ne + 4) + 64));
    g->mem = mem;
    g->d_out = static_cast<double *>(mem);
    g->d_truth = g->d_out + 4;
    g->d_absprod = g->d_truth + ne;
    g->d_rows = reinterpret_cast<int *>(g->d_absprod + ne);
    g->d_cols = g->d_rows + g->nr;
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(g->d_rows, ri.data(), sizeof(int) * ri.size(),
                                    cudaMemcpyHostToDevice, stream));
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(g->d_cols, ci.data(), sizeof(int) * ci.size(),
                                    cudaMemcpyHostToDevice, stream));
    const long long warps = (long long) ne;
    guard_truth_kernel<<<(unsigned) ((warps * 32 + 255) / 256), 256, 0, stream>>>(
        A, a_rs, a_ls, B, b_rs, b_ls, k, g->d_rows, g->nr, g->d_cols, g->nc, g->d_truth,
        g->d_absprod);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    std::vector<double> t(ne);
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(t.data(), g->d_truth, sizeof(double) * ne,
                                    cudaMemcpyDeviceToHost, stream));
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(stream));
    double tn = 0.0;
    for (size_t e = 0; e < ne; ++e) tn += std::fabs(t[e]);
    g->truth_norm = tn;
    return CA3DMM_OK;
}

extern "C" int ca3dmm_guard_error(const ca3dmm_guard_t *g, const double *C, long long ldC,
                                  double *normwise, double *componentwise, void *stream_)
{
    if (!g || !g->mem || !C) return CA3DMM_EINVAL;
    cudaStream_t stream = (cudaStream_t) stream_;
    guard_error_kernel<<<1, 256, 0, stream>>>(C, ldC, g->d_rows, g->nr, g->d_cols, g->nc,
                                              g->d_truth, g->d_absprod, g->d_out);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(1);
    double h[3];
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(h, g->d_out, sizeof(h), cudaMemcpyDeviceToHost, stream));
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(stream));
    const double bad = h[2] != 0.0 ? NAN : 0.0;
    if (normwise) *normwise = (g->truth_norm > 0.0 ? h[0] / g->truth_norm : h[0]) + bad;
    if (componentwise) *componentwise = h[1] + bad;
    return CA3DMM_OK;
}

extern "C" void ca3dmm_guard_free(ca3dmm_guard_t *g)
{
    if (g && g->mem) cudaFree(g->mem);
    if (g) memset(g, 0, sizeof(*g));
}
