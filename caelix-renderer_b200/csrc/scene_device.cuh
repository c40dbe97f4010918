// Device functions of the brick hash table shared by the scene build and the trace kernels.
//
// The key slot layout and the fingerprint are the reference's hash module
// (lib/src/rhi/hash_table_layout.h:24-34: 16-byte slots key_lo, key_hi, payload, pad;
// shaders/common/caelix_hash_table.hlsl:102-128: splitmix64 rounds over the key words, key_lo >= 1,
// key_hi != 0). The table is built canonically (scene.cu): the home slot of a key is
// floor(key_lo * capacity / 2^32) (capacity = 2 x keys: load factor 0.5), keys are placed in the
// order (home, brick index) at the first free slot at or after the home, and no probe wraps (a
// tail follows the table). A lookup probes from the home until the key or an empty slot, at most
// max_probe + 1 slots.
#pragma once
#include <cstdint>

namespace cx {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__host__ __device__ __forceinline__ void hash_fingerprint(int32_t x, int32_t y, int32_t z, uint32_t& lo, uint32_t& hi)
{
    uint64_t h = splitmix64(0ull ^ (((uint64_t)(uint32_t)y << 32) | (uint32_t)x));
    h = splitmix64(h ^ (uint64_t)(uint32_t)z);
    const uint32_t l = (uint32_t)h;
    const uint32_t u = (uint32_t)(h >> 32);
    lo = l > 1u ? l : 1u;
    hi = u != 0u ? u : 1u;
}

__host__ __device__ __forceinline__ uint32_t hash_home(uint32_t key_lo, uint32_t capacity)
{
    return (uint32_t)(((uint64_t)key_lo * capacity) >> 32);
}

// The record of brick (x, y, z), or 0xFFFFFFFF.
__device__ __forceinline__ uint32_t hash_lookup(const uint4* __restrict__ slots, uint32_t capacity, uint32_t max_probe,
                                                int32_t x, int32_t y, int32_t z)
{
    uint32_t lo, hi;
    hash_fingerprint(x, y, z, lo, hi);
    const uint32_t home = hash_home(lo, capacity);
    for (uint32_t p = home; p <= home + max_probe; ++p) {
        const uint4 s = __ldg(slots + p);
        if (s.x == 0u) return 0xFFFFFFFFu;
        if (s.x == lo && s.y == hi) return s.z;
    }
    return 0xFFFFFFFFu;
}

}  // namespace cx
