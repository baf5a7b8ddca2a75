// Shared device helpers: D2Q9 lattice, storage formats, mbarrier / TMA wrappers.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "lbm_b200.h"

namespace lbm {

// D2Q9 velocity set and opposite directions, the reference's ordering
// (lbm_core4.cu:1-3): q = 0 rest, 1 E, 2 N, 3 W, 4 S, 5 NE, 6 NW, 7 SW, 8 SE.
__host__ __device__ constexpr int cx(int q)
{
    return (q == 1 || q == 5 || q == 8) ? 1 : ((q == 3 || q == 6 || q == 7) ? -1 : 0);
}
__host__ __device__ constexpr int cy(int q)
{
    return (q == 2 || q == 5 || q == 6) ? 1 : ((q == 4 || q == 7 || q == 8) ? -1 : 0);
}
__host__ __device__ constexpr int opp(int q)
{
    return q == 0 ? 0 : (q <= 4 ? ((q + 1) % 4 + 1) : ((q - 5 + 2) % 4 + 5));
}
__host__ __device__ constexpr float wgt(int q)
{
    return q == 0 ? 4.0f / 9.0f : (q <= 4 ? 1.0f / 9.0f : 1.0f / 36.0f);
}
static_assert(opp(1) == 3 && opp(2) == 4 && opp(3) == 1 && opp(4) == 2, "opp");
static_assert(opp(5) == 7 && opp(6) == 8 && opp(7) == 5 && opp(8) == 6, "opp");

// ---------------------------------------------------------------------------
// Storage formats of the population planes in HBM.  Arithmetic is FP32 (R) for
// the kernels of the hot path; F16DEV/BF16DEV store the deviation f_q - w_q,
// which keeps the ~1e-3 relative resolution of a 16-bit float on the small
// departures from rest.  F64 (double storage and arithmetic) is the judge format
// of general_f64.cu and of the format-generic helpers (initialisation,
// conversion, reductions).
// ---------------------------------------------------------------------------
struct StoreF32 {
    using T = float;
    using R = float;
    static constexpr int kind = LBM_STORE_F32;
    __device__ __forceinline__ static float load(T v, int)
    {
        return v;
    }
    __device__ __forceinline__ static T store(float f, int)
    {
        return f;
    }
};
struct StoreF16Dev {
    using T = __half;
    using R = float;
    static constexpr int kind = LBM_STORE_F16DEV;
    __device__ __forceinline__ static float load(T v, int q)
    {
        return __half2float(v) + wgt(q);
    }
    __device__ __forceinline__ static T store(float f, int q)
    {
        return __float2half_rn(f - wgt(q));
    }
};
struct StoreBF16Dev {
    using T = __nv_bfloat16;
    using R = float;
    static constexpr int kind = LBM_STORE_BF16DEV;
    __device__ __forceinline__ static float load(T v, int q)
    {
        return __bfloat162float(v) + wgt(q);
    }
    __device__ __forceinline__ static T store(float f, int q)
    {
        return __float2bfloat16_rn(f - wgt(q));
    }
};
struct StoreF64 {
    using T = double;
    using R = double;
    static constexpr int kind = LBM_STORE_F64;
    __device__ __forceinline__ static double load(T v, int)
    {
        return v;
    }
    __device__ __forceinline__ static T store(double f, int)
    {
        return f;
    }
};

// ---------------------------------------------------------------------------
// mbarrier and TMA (cp.async.bulk.tensor) wrappers.  Every load lands in the issuing CTA's own shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Give-up limit of every spin-wait on an mbarrier: 2^31 SM cycles, about a
// second at the B200's clocks.
constexpr long long kWaitLimitCycles = 1ll << 31;

// Bounded wait: gives up after `limit` SM cycles and returns false (the callers
// then set the device error word, wait with the same bound for their own copies
// in flight and return).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity,
                                                  long long limit = kWaitLimitCycles)
{
    if (mbar_try_wait(bar, parity))
        return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > limit)
            return false;
    }
    return true;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, uint64_t *bar, int x, int y, int z)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Programmatic dependent launch: let the next kernel of the stream be scheduled
// (pdl_trigger), and wait until the previous one has completed with its memory
// visible (pdl_wait; a no-op for a kernel launched without the attribute).
__device__ __forceinline__ void pdl_trigger()
{
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

__host__ __device__ constexpr int round_up(int a, int b)
{
    return (a + b - 1) / b * b;
}

// Floor division / modulo for possibly negative integers.
__host__ __device__ __forceinline__ int floor_div(int a, int b)
{
    return (a >= 0) ? a / b : -((-a + b - 1) / b);
}
__host__ __device__ __forceinline__ int wrap(int a, int n)
{
    int r = a % n;
    return r < 0 ? r + n : r;
}

} // namespace lbm
