// Small sm_100a device helpers written as inline PTX: 1-D TMA bulk copies
// into shared memory completed through an mbarrier, acquire/release
// accesses for inter-CTA flags, and bounded waits.
#pragma once

#include <cstdint>

namespace gpj {

// Error bits a kernel ORs into its status word (never traps).
enum DeviceError : unsigned long long {
    kErrLookbackTimeout = 1ull << 0,  // a predecessor tile never published
    kErrCopyTimeout = 1ull << 1,      // a TMA copy never completed
    kErrIrregular = 1ull << 3,        // a line does not end outside strings at level -1
    kErrLongLine = 1ull << 4,         // a line runs further past its tile than the bound
    kErrDeferred = 1ull << 5,         // some lines were not evaluated by the fused queries
    kErrOutOverflow = 1ull << 6,      // a line index beyond the result buffer's capacity
};

// Errors after which waiting for other tiles is pointless (the others are
// notes for the host: take another path for part or all of the input).
constexpr unsigned long long kFatalErrors = kErrLookbackTimeout | kErrCopyTimeout;

// Poll budgets of the bounded waits (each poll also sleeps briefly).
constexpr unsigned kMaxPolls = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// Makes the barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// 1-D bulk copy global -> shared of `bytes` (multiple of 16, both addresses
// 16-byte aligned), completing on `bar`.  No multicast.
__device__ __forceinline__ void tma_load_1d(void* dst, const void* src, uint32_t bytes,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return done != 0;
}

// Bounded wait for phase `phase` of `bar`; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase) {
    for (unsigned i = 0; i < kMaxPolls; i++) {
        if (mbar_try_wait(bar, phase)) return true;
    }
    return false;
}

// The same for warps that may wait long (a whole pipeline stage): backs off
// with growing sleeps so idle warps leave the issue slots to working ones.
__device__ __forceinline__ bool mbar_wait_idle(uint64_t* bar, uint32_t phase) {
    unsigned sleep_ns = 32;
    for (unsigned i = 0; i < kMaxPolls; i++) {
        if (mbar_try_wait(bar, phase)) return true;
        __nanosleep(sleep_ns);
        if (sleep_ns < 1024) sleep_ns <<= 1;
    }
    return false;
}

__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
    asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

}  // namespace gpj
