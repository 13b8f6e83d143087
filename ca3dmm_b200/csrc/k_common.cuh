// Device-side helpers shared by the sm_100a kernels: mbarriers, TMA tile
// loads, bounded waits and the device status word.
//
// Every spin-wait in this library is bounded by a wall-clock limit read from
// %globaltimer; a wait that runs out records a status code in the launch's
// status word, raises the CTA-local abort flag and returns false, so the
// kernel winds down instead of hanging the GPU.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <cstdio>

#define CA3DMM_DEV __device__ __forceinline__

// Status codes written to the device status word (first writer wins).
enum {
    CA3DMM_DEV_OK              = 0,
    CA3DMM_DEV_TIMEOUT_PRODUCE = 1,   // producer gave up waiting for a free stage
    CA3DMM_DEV_TIMEOUT_CONSUME = 2,   // consumer gave up waiting for a full stage
    CA3DMM_DEV_TIMEOUT_ACCUM   = 3,   // MMA issuer gave up waiting for a drained accumulator
    CA3DMM_DEV_TIMEOUT_EPI     = 4,   // epilogue gave up waiting for an accumulator
    CA3DMM_DEV_TIMEOUT_QUEUE   = 5,   // persistent work queue wait ran out
    CA3DMM_DEV_CANARY          = 6,   // a work-buffer guard band was overwritten
};

// Virtual tile v of a persistent launch -> tile index of the plan: v walks the
// ranges in order (a launch over the whole list is one range [0, total)).
// (fully unrolled over the fixed capacity, so the parameter struct is read
// with constant indices and never copied to local memory)
template <typename R>
CA3DMM_DEV int range_tile(const R &r, int v)
{
    int t = -1;
#pragma unroll
    for (int i = 0; i < (int) (sizeof(r.len) / sizeof(r.len[0])); ++i) {
        if (t < 0 && i < r.n) {
            if (v < r.len[i]) t = r.begin[i] + v;
            else v -= r.len[i];
        }
    }
    return t;
}

template <typename R>
inline int range_total(const R &r)
{
    int t = 0;
    for (int i = 0; i < r.n; ++i) t += r.len[i];
    return t;
}

CA3DMM_DEV uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

CA3DMM_DEV uint64_t global_timer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

CA3DMM_DEV void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

CA3DMM_DEV void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

CA3DMM_DEV void fence_proxy_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

CA3DMM_DEV void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

CA3DMM_DEV void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

CA3DMM_DEV bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase.  Returns false (and records `code` in
// *status, sets *abort) when `limit_ns` passes or another role aborted.
CA3DMM_DEV bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, volatile int *abort,
                                  int *status, int code, uint64_t limit_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    uint64_t t0 = global_timer_ns();
    for (uint32_t it = 1;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63u) == 0) {
            if (*abort) return false;
            if (global_timer_ns() - t0 > limit_ns) {
                atomicCAS(status, 0, code);
                *abort = 1;
                return false;
            }
        }
    }
}

// 2D tiled TMA load into shared memory, completing on `bar` (tx bytes).
// The tensor map lives in global memory (64-byte aligned, written by the
// host before the launch).
CA3DMM_DEV void tma_load_2d(void *smem_dst, const void *tmap, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

// 5D tiled TMA load (coordinates innermost first), completing on `bar`.
CA3DMM_DEV void tma_load_5d(void *smem_dst, const void *tmap, int c0, int c1, int c2, int c3,
                            int c4, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(smem_dst)),
        "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

CA3DMM_DEV void tmap_prefetch(const void *tmap)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(tmap) : "memory");
}

// Tensor maps written by the host through a plain copy are read by the TMA
// unit through the tensormap proxy; acquire them once per CTA before use.
CA3DMM_DEV void tmap_acquire(const void *tmap)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmap) : "memory");
}

// Host: report a failed CUDA call with its error string, return CA3DMM_ECUDA.
#define CA3DMM_CUDA_TRY(call)                                                              \
    do {                                                                                   \
        cudaError_t err_ = (call);                                                         \
        if (err_ != cudaSuccess) {                                                         \
            fprintf(stderr, "[ERROR] %s, %d: %s failed: %s\n", __FILE__, __LINE__, #call,   \
                    cudaGetErrorString(err_));                                             \
            return 2;                                                                      \
        }                                                                                  \
    } while (0)

CA3DMM_DEV int lane_id() { return threadIdx.x & 31; }
