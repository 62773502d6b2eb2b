// tma.cuh -- Blackwell/Hopper async-copy primitives used by the pipelined
// gather kernels: mbarriers in shared memory, 1-D bulk copies
// (cp.async.bulk, the TMA engine's untiled form) with L2 cache hints, and
// bounded waits.  Inline PTX, sm_90+ (built for sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace daspmm {

// Device-side error word: set by a kernel whose bounded wait expired.  Read and
// cleared by daspmm_device_error() (api.cu, the one file that includes this).
static __device__ int g_device_error = 0;

constexpr int kErrWaitExpired = 1;
// An mbarrier wait gives up after this many polls (each poll may suspend the
// thread for a short, hardware-chosen time); the normal wait is a few
// microseconds, this bound is far above any legitimate one.
constexpr int kWaitPolls = 1 << 21;

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Make initialised barriers visible to the async proxy (the copy engine).
__device__ __forceinline__ void mbar_init_fence()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of the barrier; false (and the error word set) if
// the bound (`polls` polls) expires.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int polls = kWaitPolls)
{
    for (int i = 0; i < polls; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    atomicExch(&g_device_error, kErrWaitExpired);
    return false;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_inval(uint32_t bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start before the previous kernel of its stream has
// finished; pdl_wait() blocks until that kernel has completed and its writes
// are visible (a no-op for a kernel launched the ordinary way), and
// pdl_trigger() lets the next kernel of the stream be scheduled early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;"); }

// Order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) writes to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ uint64_t policy_evict_last()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t policy_evict_first()
{
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global to this CTA's shared memory; completion is signalled on `bar` as
// transaction bytes.  No multicast.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes,
                                         uint32_t bar, uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar), "l"(policy)
        : "memory");
}

// Per-thread asynchronous 16-byte copy global -> shared (LDGSTS), bypassing
// L1, with an L2 hint; completion tracked by commit/wait groups of this thread.
__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, uint64_t pol)
{
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(dst),
                 "l"(src), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Global loads / stores with an L2 eviction-priority hint.
__device__ __forceinline__ void st_hint_v4(float *p, float a, float b, float c, float d, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(a),
                 "f"(b), "f"(c), "f"(d), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void st_hint_v2(float *p, float a, float b, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(a), "f"(b),
                 "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void st_hint_f32(float *p, float a, uint64_t pol)
{
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(a), "l"(pol)
                 : "memory");
}
template <int V>
__device__ __forceinline__ void st_hint(float *p, const float (&r)[V], uint64_t pol)
{
    if constexpr (V == 4) st_hint_v4(p, r[0], r[1], r[2], r[3], pol);
    else if constexpr (V == 2) st_hint_v2(p, r[0], r[1], pol);
    else st_hint_f32(p, r[0], pol);
}
// (not volatile: pure loads of read-only data, free to schedule)
template <int V>
__device__ __forceinline__ void ld_nc_hint(float (&r)[V], const float *p, uint64_t pol)
{
    if constexpr (V == 4) {
        asm("ld.global.nc.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
            : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3])
            : "l"(p), "l"(pol));
    } else if constexpr (V == 2) {
        asm("ld.global.nc.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
            : "=f"(r[0]), "=f"(r[1])
            : "l"(p), "l"(pol));
    } else {
        asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(r[0]) : "l"(p), "l"(pol));
    }
}
__device__ __forceinline__ int ld_hint_s32(const int *p, uint64_t pol)
{
    int v;
    asm("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_hint_f32(const float *p, uint64_t pol)
{
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}

}  // namespace daspmm
