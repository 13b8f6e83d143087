// Cost-model MLP: nin -> h1 (ReLU) -> h2 (ReLU) -> 1, FP32, trained with Adam
// on mean-squared error, with hand-written forward / backward / update kernels.
// Every batch reduction runs in a fixed order per thread (no atomics), so
// training is bit-reproducible.
//
// Parameter layout (one contiguous float array): W1[h1][nin], b1[h1],
// W2[h2][h1], b2[h2], W3[h2], b3[1].
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include "k_common.cuh"
#include "ca3dmm_kernels.h"
#include "ca3dmm_tune.h"

struct ca3dmm_mlp {
    int nin, h1, h2, np;
    int cap;                  // batch capacity of the activation buffers
    float *params, *grads, *m1, *m2;   // device
    float *a1, *a2, *out, *d1, *d2, *dout;   // device activations / deltas [cap x h]
    float *X, *y;             // device batch staging
    float *loss;              // device scalar
    float *feat_mean, *feat_std;   // host feature normalisation (nin each)
    int step;
};

namespace {

__global__ void dense_fwd(const float *__restrict__ X, const float *__restrict__ W,
                          const float *__restrict__ b, float *__restrict__ Y, int B, int nin,
                          int nout, int relu)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * nout) return;
    const int r = idx / nout, o = idx % nout;
    float s = b[o];
    for (int i = 0; i < nin; ++i) s += W[o * nin + i] * X[r * nin + i];
    Y[idx] = relu ? fmaxf(s, 0.f) : s;
}

// dout = (out - y) / B, loss = mean 0.5 (out - y)^2 (one block, fixed order)
__global__ void mse_grad(const float *__restrict__ out, const float *__restrict__ y,
                         float *__restrict__ dout, float *__restrict__ loss, int B)
{
    __shared__ float part[256];
    float s = 0.f;
    for (int r = threadIdx.x; r < B; r += blockDim.x) {
        const float g = out[r] - y[r];
        dout[r] = g / (float) B;
        s += 0.5f * g * g;
    }
    part[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *loss = part[0] / (float) B;
}

// dW[o][i] = sum_r dY[r][o] X[r][i], db[o] = sum_r dY[r][o].  Block (o, group of
// 32 columns; column nin is the bias, X = 1): warp w sums the rows r = w, w + 8,
// ... of its lane's column, then the 8 partial sums are added in warp order --
// a fixed order, so the gradient does not depend on scheduling.
constexpr int WG_WARPS = 8;
__global__ void __launch_bounds__(WG_WARPS * 32)
dense_wgrad(const float *__restrict__ dY, const float *__restrict__ X, float *__restrict__ dW,
            float *__restrict__ db, int B, int nin, int nout)
{
    __shared__ float part[WG_WARPS][32];
    const int o = blockIdx.x, lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int i = blockIdx.y * 32 + lane;
    float s = 0.f;
    if (i <= nin)
        for (int r = w; r < B; r += WG_WARPS) s += dY[r * nout + o] * (i < nin ? X[r * nin + i] : 1.f);
    part[w][lane] = s;
    __syncthreads();
    if (w == 0 && i <= nin) {
        float t = 0.f;
#pragma unroll
        for (int q = 0; q < WG_WARPS; ++q) t += part[q][lane];
        if (i < nin) dW[o * nin + i] = t; else db[o] = t;
    }
}

inline dim3 wgrad_grid(int nin, int nout) { return dim3(nout, (nin + 1 + 31) / 32); }

// dX[r][i] = (sum_o dY[r][o] W[o][i]) * (A[r][i] > 0)   (ReLU of the layer below)
__global__ void dense_xgrad(const float *__restrict__ dY, const float *__restrict__ W,
                            const float *__restrict__ A, float *__restrict__ dX, int B, int nin,
                            int nout)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= B * nin) return;
    const int r = idx / nin, i = idx % nin;
    float s = 0.f;
    for (int o = 0; o < nout; ++o) s += dY[r * nout + o] * W[o * nin + i];
    dX[idx] = A[idx] > 0.f ? s : 0.f;
}

__global__ void adam_step(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                          float *__restrict__ v, int n, float lr, float b1, float b2, float eps,
                          float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline int blocks(long long n) { return (int) ((n + 255) / 256); }

int ensure_capacity(ca3dmm_mlp *m, int B)
{
    if (B <= m->cap) return CA3DMM_OK;
    cudaFree(m->a1); cudaFree(m->a2); cudaFree(m->out); cudaFree(m->d1); cudaFree(m->d2);
    cudaFree(m->dout); cudaFree(m->X); cudaFree(m->y);
    const size_t f = sizeof(float);
    CA3DMM_CUDA_TRY(cudaMalloc(&m->a1, f * B * m->h1));
    CA3DMM_CUDA_TRY(cudaMalloc(&m->a2, f * B * m->h2));
    CA3DMM_CUDA_TRY(cudaMalloc(&m->out, f * B));
    CA3DMM_CUDA_TRY(cudaMalloc(&m->d1, f * B * m->h1));
    CA3DMM_CUDA_TRY(cudaMalloc(&m->d2, f * B * m->h2));
    CA3DMM_CUDA_TRY(cudaMalloc(&m->dout, f * B));
    CA3DMM_CUDA_TRY(cudaMalloc(&m->X, f * B * m->nin));
    CA3DMM_CUDA_TRY(cudaMalloc(&m->y, f * B));
    m->cap = B;
    return CA3DMM_OK;
}

// forward on m->X (device, B rows) into m->out
int forward(ca3dmm_mlp *m, int B)
{
    float *W1 = m->params, *b1 = W1 + m->h1 * m->nin, *W2 = b1 + m->h1, *b2 = W2 + m->h2 * m->h1;
    float *W3 = b2 + m->h2, *b3 = W3 + m->h2;
    dense_fwd<<<blocks((long long) B * m->h1), 256>>>(m->X, W1, b1, m->a1, B, m->nin, m->h1, 1);
    dense_fwd<<<blocks((long long) B * m->h2), 256>>>(m->a1, W2, b2, m->a2, B, m->h1, m->h2, 1);
    dense_fwd<<<blocks(B), 256>>>(m->a2, W3, b3, m->out, B, m->h2, 1, 0);
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(3);
    return CA3DMM_OK;
}

// loss and gradients for the batch in m->X / m->y
int fwd_bwd(ca3dmm_mlp *m, int B)
{
    int rc = forward(m, B);
    if (rc) return rc;
    float *W1 = m->params, *b1 = W1 + m->h1 * m->nin, *W2 = b1 + m->h1, *b2 = W2 + m->h2 * m->h1;
    float *W3 = b2 + m->h2;
    (void) b2;
    float *gW1 = m->grads, *gb1 = gW1 + m->h1 * m->nin, *gW2 = gb1 + m->h1,
          *gb2 = gW2 + m->h2 * m->h1, *gW3 = gb2 + m->h2, *gb3 = gW3 + m->h2;
    mse_grad<<<1, 256>>>(m->out, m->y, m->dout, m->loss, B);
    dense_wgrad<<<wgrad_grid(m->h2, 1), WG_WARPS * 32>>>(m->dout, m->a2, gW3, gb3, B, m->h2, 1);
    dense_xgrad<<<blocks((long long) B * m->h2), 256>>>(m->dout, W3, m->a2, m->d2, B, m->h2, 1);
    dense_wgrad<<<wgrad_grid(m->h1, m->h2), WG_WARPS * 32>>>(m->d2, m->a1, gW2, gb2, B, m->h1,
                                                             m->h2);
    dense_xgrad<<<blocks((long long) B * m->h1), 256>>>(m->d2, W2, m->a1, m->d1, B, m->h1, m->h2);
    dense_wgrad<<<wgrad_grid(m->nin, m->h1), WG_WARPS * 32>>>(m->d1, m->X, gW1, gb1, B, m->nin,
                                                              m->h1);
    (void) W1;
    CA3DMM_CUDA_TRY(cudaGetLastError());
    ca3dmm_note_launch(6);
    return CA3DMM_OK;
}

// xorshift-based deterministic initialisation (He-uniform scaled)
float urand(unsigned long long &s)
{
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    return (float) ((s >> 11) * (1.0 / 9007199254740992.0));
}

void normalise(const ca3dmm_mlp *m, const float *X, int n, float *out)
{
    for (int r = 0; r < n; ++r)
        for (int i = 0; i < m->nin; ++i)
            out[r * m->nin + i] = (X[r * m->nin + i] - m->feat_mean[i]) / m->feat_std[i];
}

}  // namespace

extern "C" int ca3dmm_mlp_create(int nin, int h1, int h2, unsigned long long seed,
                                 ca3dmm_mlp_p *out)
{
    if (!out || nin < 1 || h1 < 1 || h2 < 1 || nin > 256 || h1 > 1024 || h2 > 1024)
        return CA3DMM_EINVAL;
    *out = nullptr;
    ca3dmm_mlp *m = (ca3dmm_mlp *) calloc(1, sizeof(ca3dmm_mlp));
    if (!m) return CA3DMM_ENOMEM;
    m->nin = nin; m->h1 = h1; m->h2 = h2;
    m->np = h1 * nin + h1 + h2 * h1 + h2 + h2 + 1;
    const size_t pb = sizeof(float) * m->np;
    if (cudaMalloc(&m->params, pb) != cudaSuccess || cudaMalloc(&m->grads, pb) != cudaSuccess ||
        cudaMalloc(&m->m1, pb) != cudaSuccess || cudaMalloc(&m->m2, pb) != cudaSuccess ||
        cudaMalloc(&m->loss, sizeof(float)) != cudaSuccess) {
        ca3dmm_mlp_free(&m);
        return CA3DMM_ENOMEM;
    }
    m->feat_mean = (float *) calloc(nin, sizeof(float));
    m->feat_std = (float *) malloc(sizeof(float) * nin);
    for (int i = 0; i < nin; ++i) m->feat_std[i] = 1.f;
    float *h = (float *) malloc(pb);
    unsigned long long s = seed * 0x9E3779B97F4A7C15ull + 1;
    float *W1 = h, *b1 = W1 + h1 * nin, *W2 = b1 + h1, *b2 = W2 + h2 * h1, *W3 = b2 + h2;
    for (int i = 0; i < h1 * nin; ++i) W1[i] = (2.f * urand(s) - 1.f) * sqrtf(6.f / nin);
    for (int i = 0; i < h1; ++i) b1[i] = 0.f;
    for (int i = 0; i < h2 * h1; ++i) W2[i] = (2.f * urand(s) - 1.f) * sqrtf(6.f / h1);
    for (int i = 0; i < h2; ++i) b2[i] = 0.f;
    for (int i = 0; i < h2; ++i) W3[i] = (2.f * urand(s) - 1.f) * sqrtf(3.f / h2);
    W3[h2] = 0.f;
    cudaMemcpy(m->params, h, pb, cudaMemcpyHostToDevice);
    free(h);
    cudaMemset(m->m1, 0, pb);
    cudaMemset(m->m2, 0, pb);
    *out = m;
    return CA3DMM_OK;
}

extern "C" void ca3dmm_mlp_free(ca3dmm_mlp_p *mp)
{
    if (!mp || !*mp) return;
    ca3dmm_mlp *m = *mp;
    cudaFree(m->params); cudaFree(m->grads); cudaFree(m->m1); cudaFree(m->m2); cudaFree(m->loss);
    cudaFree(m->a1); cudaFree(m->a2); cudaFree(m->out); cudaFree(m->d1); cudaFree(m->d2);
    cudaFree(m->dout); cudaFree(m->X); cudaFree(m->y);
    free(m->feat_mean); free(m->feat_std);
    free(m);
    *mp = nullptr;
}

extern "C" int ca3dmm_mlp_nparams(ca3dmm_mlp_p m) { return m ? m->np : 0; }

extern "C" int ca3dmm_mlp_inputs(ca3dmm_mlp_p m) { return m ? m->nin : 0; }

extern "C" int ca3dmm_mlp_get_params(ca3dmm_mlp_p m, float *host)
{
    if (!m || !host) return CA3DMM_EINVAL;
    CA3DMM_CUDA_TRY(cudaMemcpy(host, m->params, sizeof(float) * m->np, cudaMemcpyDeviceToHost));
    return CA3DMM_OK;
}

extern "C" int ca3dmm_mlp_set_params(ca3dmm_mlp_p m, const float *host)
{
    if (!m || !host) return CA3DMM_EINVAL;
    CA3DMM_CUDA_TRY(cudaMemcpy(m->params, host, sizeof(float) * m->np, cudaMemcpyHostToDevice));
    return CA3DMM_OK;
}

extern "C" int ca3dmm_mlp_set_normalisation(ca3dmm_mlp_p m, const float *mean, const float *stdv)
{
    if (!m || !mean || !stdv) return CA3DMM_EINVAL;
    for (int i = 0; i < m->nin; ++i) {
        m->feat_mean[i] = mean[i];
        m->feat_std[i] = stdv[i] > 0.f ? stdv[i] : 1.f;
    }
    return CA3DMM_OK;
}

// One forward + backward on raw (already normalised) inputs; returns the
// loss and, when grads is not NULL, the parameter gradients (host).
extern "C" int ca3dmm_mlp_fwd_bwd(ca3dmm_mlp_p m, const float *X, const float *y, int B,
                                  float *loss, float *grads)
{
    if (!m || !X || !y || B < 1) return CA3DMM_EINVAL;
    int rc = ensure_capacity(m, B);
    if (rc) return rc;
    CA3DMM_CUDA_TRY(cudaMemcpy(m->X, X, sizeof(float) * B * m->nin, cudaMemcpyHostToDevice));
    CA3DMM_CUDA_TRY(cudaMemcpy(m->y, y, sizeof(float) * B, cudaMemcpyHostToDevice));
    rc = fwd_bwd(m, B);
    if (rc) return rc;
    if (loss) CA3DMM_CUDA_TRY(cudaMemcpy(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    if (grads)
        CA3DMM_CUDA_TRY(cudaMemcpy(grads, m->grads, sizeof(float) * m->np, cudaMemcpyDeviceToHost));
    return CA3DMM_OK;
}

// Train on n samples (features X [n x nin] raw, targets y), full-batch
// shuffled minibatches of `batch`, `epochs` passes, Adam(lr).  The feature
// normalisation (mean / std over X) is computed here and kept with the model.
extern "C" int ca3dmm_mlp_train(ca3dmm_mlp_p m, const float *X, const float *y, int n, int epochs,
                                int batch, float lr, unsigned long long seed, float *final_loss)
{
    if (!m || !X || !y || n < 1 || epochs < 1 || batch < 1) return CA3DMM_EINVAL;
    if (batch > n) batch = n;
    for (int i = 0; i < m->nin; ++i) {
        double s = 0, q = 0;
        for (int r = 0; r < n; ++r) s += X[r * m->nin + i];
        const double mu = s / n;
        for (int r = 0; r < n; ++r) q += (X[r * m->nin + i] - mu) * (X[r * m->nin + i] - mu);
        m->feat_mean[i] = (float) mu;
        const double sd = sqrt(q / n);
        m->feat_std[i] = sd > 1e-6 ? (float) sd : 1.f;
    }
    float *Xn = (float *) malloc(sizeof(float) * n * m->nin);
    float *xb = (float *) malloc(sizeof(float) * batch * m->nin), *yb = (float *) malloc(sizeof(float) * batch);
    int *perm = (int *) malloc(sizeof(int) * n);
    if (!Xn || !xb || !yb || !perm) { free(Xn); free(xb); free(yb); free(perm); return CA3DMM_ENOMEM; }
    normalise(m, X, n, Xn);
    int rc = ensure_capacity(m, batch);
    unsigned long long s = seed * 0x2545F4914F6CDD1Dull + 7;
    float loss = 0.f;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int r = 0; r < n; ++r) perm[r] = r;
    for (int ep = 0; ep < epochs && !rc; ++ep) {
        for (int r = n - 1; r > 0; --r) {
            int j = (int) (urand(s) * (r + 1));
            if (j > r) j = r;
            int t = perm[r]; perm[r] = perm[j]; perm[j] = t;
        }
        for (int b0 = 0; b0 < n && !rc; b0 += batch) {
            const int B = n - b0 < batch ? n - b0 : batch;
            for (int r = 0; r < B; ++r) {
                memcpy(xb + r * m->nin, Xn + (size_t) perm[b0 + r] * m->nin, sizeof(float) * m->nin);
                yb[r] = y[perm[b0 + r]];
            }
            if (cudaMemcpy(m->X, xb, sizeof(float) * B * m->nin, cudaMemcpyHostToDevice) != cudaSuccess ||
                cudaMemcpy(m->y, yb, sizeof(float) * B, cudaMemcpyHostToDevice) != cudaSuccess) {
                rc = CA3DMM_ECUDA;
                break;
            }
            rc = fwd_bwd(m, B);
            if (rc) break;
            ++m->step;
            const float c1 = 1.f - powf(b1, (float) m->step), c2 = 1.f - powf(b2, (float) m->step);
            adam_step<<<blocks(m->np), 256>>>(m->params, m->grads, m->m1, m->m2, m->np, lr, b1, b2,
                                              eps, c1, c2);
            if (cudaGetLastError() != cudaSuccess) rc = CA3DMM_ECUDA;
            ca3dmm_note_launch(1);
        }
    }
    if (!rc) {
        // final full-data loss
        float *yy = (float *) malloc(sizeof(float) * n);
        rc = ca3dmm_mlp_predict(m, X, n, yy);
        double q = 0;
        for (int r = 0; r < n && !rc; ++r) q += 0.5 * (yy[r] - y[r]) * (yy[r] - y[r]);
        loss = (float) (q / n);
        free(yy);
    }
    if (final_loss) *final_loss = loss;
    free(Xn); free(xb); free(yb); free(perm);
    return rc;
}

// Predict for n raw feature rows (normalised with the model's statistics).
extern "C" int ca3dmm_mlp_predict(ca3dmm_mlp_p m, const float *X, int n, float *out)
{
    if (!m || !X || !out || n < 1) return CA3DMM_EINVAL;
    int rc = ensure_capacity(m, n);
    if (rc) return rc;
    float *Xn = (float *) malloc(sizeof(float) * n * m->nin);
    if (!Xn) return CA3DMM_ENOMEM;
    normalise(m, X, n, Xn);
    cudaError_t e = cudaMemcpy(m->X, Xn, sizeof(float) * n * m->nin, cudaMemcpyHostToDevice);
    free(Xn);
    if (e != cudaSuccess) return CA3DMM_ECUDA;
    rc = forward(m, n);
    if (rc) return rc;
    CA3DMM_CUDA_TRY(cudaMemcpy(out, m->out, sizeof(float) * n, cudaMemcpyDeviceToHost));
    return CA3DMM_OK;
}

// Versioned text file: "ca3dmm-mlp v1 nin h1 h2", mean, std, params.
extern "C" int ca3dmm_mlp_save(ca3dmm_mlp_p m, const char *path)
{
    if (!m || !path) return CA3DMM_EINVAL;
    float *p = (float *) malloc(sizeof(float) * m->np);
    int rc = ca3dmm_mlp_get_params(m, p);
    if (rc) { free(p); return rc; }
    FILE *f = fopen(path, "w");
    if (!f) { free(p); return CA3DMM_EINVAL; }
    fprintf(f, "ca3dmm-mlp v1 %d %d %d\n", m->nin, m->h1, m->h2);
    for (int i = 0; i < m->nin; ++i) fprintf(f, "%.9g ", m->feat_mean[i]);
    fprintf(f, "\n");
    for (int i = 0; i < m->nin; ++i) fprintf(f, "%.9g ", m->feat_std[i]);
    fprintf(f, "\n");
    for (int i = 0; i < m->np; ++i) fprintf(f, "%.9g\n", p[i]);
    fclose(f);
    free(p);
    return CA3DMM_OK;
}

extern "C" int ca3dmm_mlp_load(const char *path, ca3dmm_mlp_p *out)
{
    if (!path || !out) return CA3DMM_EINVAL;
    *out = nullptr;
    FILE *f = fopen(path, "r");
    if (!f) return CA3DMM_EINVAL;
    int nin, h1, h2;
    if (fscanf(f, "ca3dmm-mlp v1 %d %d %d", &nin, &h1, &h2) != 3) { fclose(f); return CA3DMM_EINVAL; }
    ca3dmm_mlp_p m;
    int rc = ca3dmm_mlp_create(nin, h1, h2, 1, &m);
    if (rc) { fclose(f); return rc; }
    float *p = (float *) malloc(sizeof(float) * m->np);
    bool ok = true;
    for (int i = 0; i < nin && ok; ++i) ok = fscanf(f, "%f", &m->feat_mean[i]) == 1;
    for (int i = 0; i < nin && ok; ++i) ok = fscanf(f, "%f", &m->feat_std[i]) == 1;
    for (int i = 0; i < m->np && ok; ++i) ok = fscanf(f, "%f", &p[i]) == 1;
    fclose(f);
    if (ok) rc = ca3dmm_mlp_set_params(m, p);
    free(p);
    if (!ok || rc) { ca3dmm_mlp_free(&m); return ok ? rc : CA3DMM_EINVAL; }
    *out = m;
    return CA3DMM_OK;
}
