// bulk.cuh -- asynchronous bulk copies from global to shared memory (cp.async.bulk, executed by the
// TMA engine) completed on shared-memory mbarriers, with bounded waits.
//
// A stencil tile is a contiguous run of cells (plus a halo of one block row on each side), so one
// untiled bulk copy per array moves it: no tensor map is needed.  A bulk copy needs 16-byte aligned
// global and shared addresses and a size that is a multiple of 16 bytes; BulkRun rounds the start of a
// run down to the 16-byte boundary (the array's base must be 16-byte aligned, which the host checks) and
// ends the bulk part at the last boundary inside the run, so no byte outside [base, base + end of the
// run) is read; the few elements after the last boundary are loaded with plain loads.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace pict {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes the initialised mbarriers visible to the asynchronous proxy (the bulk copies)
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// one arrival that also announces `bytes` of transactions for the current phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the completion of phase `parity`; false after `limit` unsuccessful tries.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
    for (long long k = 0; k < limit; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// orders this thread's earlier generic-proxy accesses of shared memory before later bulk copies into it
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Elements [g0, g0 + n) of the array at `base` (16-byte aligned), staged at dst[lead .. lead + n):
// the bulk part covers elements [g0 - lead, g0 - lead + bytes / sizeof(T)) and the plain-load tail the
// dst indices [tail0, tail1) (at most 16 / sizeof(T) - 1 elements).
template <typename T>
struct BulkRun {
    const T* src;
    uint32_t bytes;
    int lead;
    int tail0, tail1;
};

template <typename T>
__device__ __forceinline__ BulkRun<T> bulk_run(const T* base, long long g0, int n) {
    constexpr long long V = 16 / sizeof(T);
    const long long ga = g0 - (g0 % V);
    const long long g1 = g0 + n;
    const long long gb = ga + ((g1 - ga) / V) * V;
    BulkRun<T> r;
    r.src = base + ga;
    r.bytes = static_cast<uint32_t>((gb - ga) * (long long)sizeof(T));
    r.lead = static_cast<int>(g0 - ga);
    r.tail0 = static_cast<int>(gb - ga);
    r.tail1 = static_cast<int>(g1 - ga);
    return r;
}

// issue the bulk part of a run (thread that owns the mbarrier's arrival)
template <typename T>
__device__ __forceinline__ void bulk_issue(const BulkRun<T>& r, T* dst, uint64_t* bar) {
    if (r.bytes) bulk_copy_g2s(dst, r.src, r.bytes, bar);
}

// plain loads of a run's tail, spread over the CTA
template <typename T>
__device__ __forceinline__ void bulk_tail(const BulkRun<T>& r, T* dst) {
    const int k = r.tail0 + (int)threadIdx.x;
    if (k < r.tail1) dst[k] = r.src[k];
}

}  // namespace pict
