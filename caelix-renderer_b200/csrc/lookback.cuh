// The decoupled look-back of the single-pass scans, by one warp: the 32 lanes read the states of
// 128 predecessor tiles at once, so a tile waits one round trip per 128 predecessors instead of one
// per predecessor.
#pragma once
#include <cstdint>

#include "cx_device.cuh"
#include "cx_layout.h"
#include "radix_sort.cuh"

namespace cx {

// Called by every lane of one warp for tile `tile` with its aggregate `agg` (30-bit values; kMax:
// running maximum, else sum): lane 0 publishes the aggregate, the warp walks back window by window
// (the nearest tile with an inclusive prefix ends the walk; a window with an unpublished tile
// before that one is read again, a bounded number of times, after which kStatusLookbackTimeout is
// set in *status), lane 0 publishes the inclusive prefix. Returns the exclusive prefix in every lane.
template <bool kMax>
__device__ __forceinline__ uint32_t warp_lookback(uint32_t* states, uint32_t tile, uint32_t agg, uint32_t* status)
{
    constexpr int kPerLane = 4;  // a window of 128 predecessors: lane l reads tiles j - l - 32 q
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t* state = states + tile;
    if (tile == 0) {
        if (lane == 0) st_relaxed(state, kTileFlagPrefix | (agg & kTileValueMask));
        return 0;
    }
    if (lane == 0) st_relaxed(state, kTileFlagAggregate | (agg & kTileValueMask));
    uint32_t prefix = 0;
    int64_t j = (int64_t)tile - 1;  // the nearest tile of the window
    uint32_t spins = 0;
    while (j >= 0) {
        uint32_t s[kPerLane];
#pragma unroll
        for (int q = 0; q < kPerLane; ++q) {
            const int64_t t = j - (int64_t)lane - 32 * q;
            s[q] = t >= 0 ? ld_relaxed(states + t) : kTileFlagPrefix;  // before tile 0: a prefix of 0
        }
        // The nearest tile with an inclusive prefix (offset `stop` from j), and whether every tile
        // nearer than it (and it) has published.
        uint32_t stop = 32u * kPerLane - 1u;
        bool found = false, ready = true;
#pragma unroll
        for (int q = 0; q < kPerLane; ++q) {
            if (!found) {
                const uint32_t f = __ballot_sync(0xFFFFFFFFu, (s[q] & kTileFlagPrefix) != 0u);
                const uint32_t r = __ballot_sync(0xFFFFFFFFu, (s[q] & ~kTileValueMask) != 0u);
                const uint32_t last = f ? (uint32_t)(__ffs(f) - 1) : 31u;
                const uint32_t need = (2u << last) - 1u;  // lanes 0 .. last
                ready = ready && (r & need) == need;
                if (f) {
                    found = true;
                    stop = 32u * q + last;
                }
            }
        }
        if (!ready) {
            if (!spin_wait(spins)) {
                if (lane == 0) atomicOr(status, kStatusLookbackTimeout);
                break;
            }
            continue;
        }
        uint32_t v = 0;
#pragma unroll
        for (int q = 0; q < kPerLane; ++q) {
            const uint32_t off = 32u * q + lane;
            const uint32_t x = off <= stop ? (s[q] & kTileValueMask) : 0u;
            v = kMax ? max(v, x) : v + x;
        }
        const uint32_t w = kMax ? __reduce_max_sync(0xFFFFFFFFu, v) : __reduce_add_sync(0xFFFFFFFFu, v);
        prefix = kMax ? max(prefix, w) : prefix + w;
        if (found) break;
        j -= 32 * kPerLane;
    }
    const uint32_t incl = kMax ? max(prefix, agg) : prefix + agg;
    if (lane == 0) st_relaxed(state, kTileFlagPrefix | (incl & kTileValueMask));
    return prefix;
}

}  // namespace cx
