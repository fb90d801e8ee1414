// Device-side primitives for the Cahn-Hilliard step kernels (sm_100a):
// PTX wrappers for mbarriers and TMA tensor loads, the exact-rounding FP64
// arithmetic used by the drop-in path, and compensated-sum helpers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mg {

// ------------------------------------------------------------------ PTX glue
__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make mbarrier initialisation visible to the TMA (async) proxy
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
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

// Bounded wait with a 32-bit poll count (limits up to 2^31 - 1).
__device__ __forceinline__ bool mbar_wait_bounded32(uint64_t* bar, uint32_t parity, int limit)
{
    for (int n = 0; n < limit; ++n)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Bounded wait: gives up after `limit` polls and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit)
{
    for (long long n = 0; n < limit; ++n)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// 3-D tiled TMA load (no multicast), completion counted on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y,
                                            int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// --------------------------------------------------------------- arithmetic
// FP64: every operation rounded on its own (no contraction into FMA), in the
// order the reference writes it, so results are bit-identical to the
// reference's x86-64 build.  FP32: contraction allowed.
template <typename T>
struct Arith;

template <>
struct Arith<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};

template <>
struct Arith<float> {
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float div(float a, float b) { return a / b; }
};

// ------------------------------------------------------- compensated sums
// Knuth's TwoSum: s + e == a + b exactly.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e)
{
    s = __dadd_rn(a, b);
    double bp = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bp)), __dsub_rn(b, bp));
}

// (s1,e1) + (s2,e2) as an unevaluated pair
__device__ __forceinline__ double2 pair_add(double2 x, double2 y)
{
    double s, e;
    two_sum(x.x, y.x, s, e);
    e = __dadd_rn(e, __dadd_rn(x.y, y.y));
    double s2, e2;
    two_sum(s, e, s2, e2);
    return make_double2(s2, e2);
}

__device__ __forceinline__ double2 shfl_down_pair(double2 v, int off)
{
    v.x = __shfl_down_sync(0xffffffffu, v.x, off);
    v.y = __shfl_down_sync(0xffffffffu, v.y, off);
    return v;
}

// Fixed-shape block reduction of pairs; result valid in thread 0.
// `scratch` holds blockDim/32 pairs.  Same tree for every call with the same
// blockDim, so the result does not depend on timing.
__device__ __forceinline__ double2 block_pair_sum(double2 v, double2* scratch)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        double2 o = shfl_down_pair(v, off);
        if (lane + off < 32) v = pair_add(v, o);
    }
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double2 r = make_double2(0.0, 0.0);
    if (warp == 0) {
        r = lane < nwarps ? scratch[lane] : make_double2(0.0, 0.0);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            double2 o = shfl_down_pair(r, off);
            if (lane + off < 32) r = pair_add(r, o);
        }
    }
    __syncthreads();
    return r;
}

}  // namespace mg
