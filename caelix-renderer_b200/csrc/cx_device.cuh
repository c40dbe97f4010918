// Small device helpers shared by the kernels of libcaelix_b200: relaxed device-scope atomics for
// the look-back state words, warp and block scans, and the order-preserving float encoding used
// by the min/max reductions.
#pragma once
#include <cuda/atomic>
#include <cstdint>

namespace cx {

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p)
{
    return cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(*const_cast<uint32_t*>(p))
        .load(cuda::memory_order_relaxed);
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v)
{
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device>(*p).store(v, cuda::memory_order_relaxed);
}

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Inclusive warp scan of a u32.
__device__ __forceinline__ uint32_t warp_inclusive_sum(uint32_t v)
{
    const uint32_t lane = threadIdx.x & 31u;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Exclusive scan over a block of kThreads threads (a multiple of 32, at most 1024); `total`
// receives the block sum. `scratch` holds kThreads / 32 words. Every thread must call it.
template <int kThreads>
__device__ __forceinline__ uint32_t block_exclusive_sum(uint32_t v, uint32_t* scratch, uint32_t& total)
{
    constexpr int kWarps = kThreads / 32;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t inc = warp_inclusive_sum(v);
    if (lane == 31) scratch[warp] = inc;
    __syncthreads();
    uint32_t prefix = 0;
    total = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
        const uint32_t s = scratch[w];
        prefix += (uint32_t)w < warp ? s : 0u;
        total += s;
    }
    __syncthreads();
    return prefix + inc - v;
}

// Order-preserving encoding of a non-NaN float as u32 (-0 below +0): min/max over the codes are
// exact and independent of the order of a reduction.
__device__ __host__ __forceinline__ uint32_t float_order(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __host__ __forceinline__ float float_unorder(uint32_t u)
{
    const uint32_t b = (u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

// A bounded spin: returns false once `iteration` reaches the limit (the caller records the
// failure in its status word and gives up instead of waiting for ever).
constexpr uint32_t kSpinLimit = 1u << 22;
__device__ __forceinline__ bool spin_wait(uint32_t& iteration, uint32_t limit = kSpinLimit)
{
    if (++iteration >= limit) return false;
    if (iteration > 64) __nanosleep(64);
    return true;
}

}  // namespace cx
