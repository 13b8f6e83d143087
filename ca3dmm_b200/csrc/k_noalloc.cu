// k-slab FP64 GEMM that allocates no memory.
//
// Some callers cannot call cudaMalloc: code hosted inside a process whose
// device memory is owned by another allocator (a serving framework's pool, a
// memory-capped MPS client) and may not take memory behind that allocator's
// back, or code that must not let an allocation fail half-way through a job.
// ca3dmm_dgemm_kslab_noalloc serves them: the caller passes A, B and C, and
// the partial k-slab results, the tensor maps and the status word live in one
// fixed, file-scope device array instead of an engine work buffer.
//
// The array is part of the library image, so every GPU that loads the library
// holds CA3DMM_NOALLOC_SCRATCH_BYTES of it until the process exits.  All
// calls share it: two calls that overlap on the GPU (different streams or
// host threads without ordering) race on it.  It keeps whatever the last call
// left there; this entry point clears the one part that must start at zero
// (the status word) itself, and every partial slab it reads back is fully
// rewritten by the GEMM first.  The call is synchronous: it copies its plan
// from host memory and waits for the stream before returning the status.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdio>
#include <cstring>
#include "k_common.cuh"
#include "ca3dmm_kernels.h"

#define CA3DMM_NOALLOC_SCRATCH_BYTES (32ull << 20)
#define CA3DMM_NOALLOC_MAX_SLABS 64

static __device__ __align__(256) unsigned char g_kslab_scratch[CA3DMM_NOALLOC_SCRATCH_BYTES];

namespace {

// Device address of g_kslab_scratch on the current device.  In host code the
// array's name is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress with that device current.  It is looked up on every
// call (the lookup allocates nothing): a cached address would go stale after
// a cudaDeviceReset or under another context.
int scratch_address(void **out)
{
    void *p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_kslab_scratch);
    if (err != cudaSuccess || p == nullptr) {
        fprintf(stderr, "[ERROR] %s, %d: cudaGetSymbolAddress(g_kslab_scratch) failed: %s\n",
                __FILE__, __LINE__, cudaGetErrorString(err));
        return CA3DMM_ECUDA;
    }
    *out = p;
    return CA3DMM_OK;
}

size_t round256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace

extern "C" size_t ca3dmm_dgemm_kslab_noalloc_scratch_bytes(void)
{
    return CA3DMM_NOALLOC_SCRATCH_BYTES;
}

// C = A * B (column-major, no transposes) computed as kp k-slabs, like the kp
// planes of the CA3DMM grid: slab s multiplies A[:, ks] by B[ks, :] (ks the
// balanced split of k) with the FP64 DMMA kernel into a partial C held in the
// fixed scratch array, then the partials are summed in slab order into C.
// Every call looks up the scratch address (no allocation).  Synchronous on
// `stream` (it waits for the stream), so it must not be called while the
// stream is being captured; returns 0 or a CA3DMM_E* code.
extern "C" int ca3dmm_dgemm_kslab_noalloc(int m, int n, int k, int kp, const double *A, int ldA,
                                          const double *B, int ldB, double *C, int ldC,
                                          void *stream)
{
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (m < 1 || n < 1 || k < 1 || kp < 1 || kp > CA3DMM_NOALLOC_MAX_SLABS || kp > k) {
        fprintf(stderr, "[ERROR] ca3dmm_dgemm_kslab_noalloc: invalid sizes m=%d n=%d k=%d kp=%d "
                        "(need 1 <= kp <= min(k, %d))\n", m, n, k, kp, CA3DMM_NOALLOC_MAX_SLABS);
        return CA3DMM_EINVAL;
    }
    if (!A || !B || !C || ldA < m || ldB < k || ldC < m ||
        (reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15) ||
        (ldA & 1) || (ldB & 1)) {
        fprintf(stderr, "[ERROR] ca3dmm_dgemm_kslab_noalloc: A and B must be 16-byte aligned "
                        "with even leading dimensions ldA >= m, ldB >= k, and ldC >= m\n");
        return CA3DMM_EINVAL;
    }
    const long long ldp = (m + 1) / 2 * 2;
    const size_t plan_bytes = ca3dmm_dgemm_plan_bytes(kp);
    const size_t off_plan = 256;
    const size_t off_slab = round256(off_plan + plan_bytes);
    const size_t slab_elems = (size_t) ldp * (size_t) n;
    const size_t need = kp > 1 ? off_slab + slab_elems * sizeof(double) * (size_t) kp : off_slab;
    if (need > CA3DMM_NOALLOC_SCRATCH_BYTES) {
        fprintf(stderr, "[ERROR] ca3dmm_dgemm_kslab_noalloc: m=%d n=%d kp=%d needs %zu bytes of "
                        "scratch; the fixed scratch array holds %llu bytes\n", m, n, kp, need,
                CA3DMM_NOALLOC_SCRATCH_BYTES);
        return CA3DMM_EINVAL;
    }
    void *base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    unsigned char *scratch = static_cast<unsigned char *>(base);
    int *status = reinterpret_cast<int *>(scratch);
    double *slabs = reinterpret_cast<double *>(scratch + off_slab);

    // Plan (tensor maps + problem records) built in host memory on the stack
    // and copied into the scratch array.
    alignas(64) unsigned char host_plan[(128 * 2 + 128) * CA3DMM_NOALLOC_MAX_SLABS];
    if (plan_bytes > sizeof(host_plan)) return CA3DMM_EINVAL;
    ca3dmm_dgemm_desc_t probs[CA3DMM_NOALLOC_MAX_SLABS];
    for (int s = 0; s < kp; ++s) {
        const int rem = k % kp, bs = k / kp;
        const int k0 = s < rem ? (bs + 1) * s : bs * s + rem;
        const int kz = s < rem ? bs + 1 : bs;
        ca3dmm_dgemm_desc_t &q = probs[s];
        memset(&q, 0, sizeof(q));
        // slab s reads A columns [k0, k0+kz) and B rows [k0, k0+kz); the TMA
        // base of B + k0 must be 16-byte aligned, so every k0 must be even.
        q.A = A + (size_t) k0 * ldA;
        q.lda = ldA;
        q.B = B + k0;
        q.ldb = ldB;
        q.m = m; q.n = n; q.k = kz;
        q.alpha = 1.0; q.beta = 0.0;
        if (kp > 1) {
            q.C = slabs + (size_t) s * slab_elems;
            q.ldc = ldp;
        } else {
            q.C = C;
            q.ldc = ldC;
        }
        if (reinterpret_cast<uintptr_t>(q.B) & 15) {
            fprintf(stderr, "[ERROR] ca3dmm_dgemm_kslab_noalloc: slab %d starts at odd k = %d; "
                            "choose kp so that every slab start k0 is even\n", s, k0);
            return CA3DMM_EINVAL;
        }
    }
    int tiles = 0;
    rc = ca3dmm_dgemm_plan_encode(probs, kp, host_plan, &tiles);
    if (rc) return rc;
    CA3DMM_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int), st));
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(scratch + off_plan, host_plan, plan_bytes,
                                    cudaMemcpyHostToDevice, st));
    rc = ca3dmm_dgemm_launch(scratch + off_plan, kp, tiles, 0, status, 5.0, st);
    if (rc) return rc;
    if (kp > 1) {
        rc = ca3dmm_reduce_slabs_launch(slabs, (long long) slab_elems, ldp, kp, m, n, C, ldC, st);
        if (rc) return rc;
    }
    int status_h = 0;
    CA3DMM_CUDA_TRY(cudaMemcpyAsync(&status_h, status, sizeof(int), cudaMemcpyDeviceToHost, st));
    CA3DMM_CUDA_TRY(cudaStreamSynchronize(st));
    if (status_h) {
        fprintf(stderr, "[ERROR] ca3dmm_dgemm_kslab_noalloc: device status %d (a bounded wait "
                        "ran out)\n", status_h);
        return CA3DMM_ETIMEOUT;
    }
    return CA3DMM_OK;
}
