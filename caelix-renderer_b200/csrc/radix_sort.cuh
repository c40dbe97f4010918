// Onesweep LSD radix sort of (u32 key, u32 value) pairs: 8-bit digits, 4 passes over 32-bit keys.
//
// Replaces the reference's sort (shaders/light/bvh/caelix_light_bvh_sort.hlsl,
// caelix_light_bvh_sort_histogram.hlsl:8-38, caelix_light_bvh_sort_scatter.hlsl:10-78, driven by
// lib/src/light/light_tree_record.cpp:282-302: 4-bit digits, 8 passes of histogram + one-workgroup
// scan + scatter). Both are stable LSD sorts of the same keys, so the permutation is the same.
//
// One pass is one kernel (no separate histogram or scan launch):
//   * the digit counts of all four passes come from one upsweep (the caller's key producer, or
//     radix_histogram_kernel), so a pass only needs its own 256 global counts;
//   * a CTA takes the next tile id from an atomic counter, loads a tile of keys warp-striped
//     (coalesced 128-byte rows), ranks them stably inside each warp (the lanes of equal digits
//     from eight ballots, the warp's running digit count from one shared atomic per digit group),
//     and publishes its per-digit counts in the tile status words;
//   * the per-digit exclusive prefix over earlier tiles comes from a decoupled look-back over
//     those status words (one thread per digit, bounded spin: a timeout sets a status bit instead
//     of hanging);
//   * the tile is staged in shared memory in digit order and written out in runs per digit.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

#include "cx_layout.h"

namespace cx {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortKeysPerThread = 16;  // the default tile: 4096 keys
constexpr int kSortMinKeysPerThread = 4;  // the smallest tile a caller may pick: 1024 keys
constexpr uint32_t kSmallSortKeys = 4096;  // up to this many pairs, one CTA sorts in shared memory
constexpr int kRadix = 256;
constexpr uint32_t kTileFlagAggregate = 1u << 30;
constexpr uint32_t kTileFlagPrefix = 2u << 30;
constexpr uint32_t kTileValueMask = (1u << 30) - 1u;

// The tile sizes a sort may use: 256 threads x 4, 8 or 16 keys.
__host__ __device__ constexpr bool sort_keys_per_thread_ok(uint32_t kpt)
{
    return kpt == 4 || kpt == 8 || kpt == 16;
}

__host__ __device__ constexpr uint32_t sort_tiles(uint32_t n, uint32_t kpt = kSortKeysPerThread)
{
    return (n + kSortThreads * kpt - 1) / (kSortThreads * kpt);
}

// Scratch words one sort of n elements with tiles of 256 * kpt keys needs (all of them zero
// before the first pass):
//   histogram  4 * 256 digit counts
//   counters   4 tile-id counters (one per pass)
//   states     4 * tiles * 256 look-back status words
// sort_scratch_words(n, kSortMinKeysPerThread) covers every tile size.
__host__ __device__ constexpr uint64_t sort_scratch_words(uint32_t n, uint32_t kpt = kSortKeysPerThread)
{
    return 4ull * kRadix + 4ull + 4ull * sort_tiles(n, kpt) * kRadix;
}

// The tile for a sort of n pairs chosen by the sort's callers: 4096 keys when that gives at least
// kPipeMinTiles tiles (the persistent pipelined pass), else 1024 (more tiles for a small sort, and
// a quarter of the ranking work in each tile's critical path).
constexpr uint32_t kPipeMinTiles = 64;
__host__ __device__ constexpr uint32_t sort_keys_per_thread_for(uint32_t n)
{
    return sort_tiles(n, kSortKeysPerThread) >= kPipeMinTiles ? (uint32_t)kSortKeysPerThread
                                                             : (uint32_t)kSortMinKeysPerThread;
}

// The number of SMs of the current CUDA device (looked up once per device), for grid sizing.
uint32_t current_sm_count();

// Accumulates the 256-bin histograms of all four digits of keys[0 .. n) into hist[4][256].
void radix_histogram(const uint32_t* keys, uint32_t n, uint32_t* hist, uint32_t grid, cudaStream_t stream);

// An optional gather fused into the last pass: the 48-byte row at rows_in + rows_in_stride * value
// (in uint4 units) of every element is copied to rows_out[destination] (48-byte rows), and, when
// inverse is not null, inverse[value] = destination.
struct SortGather
{
    const uint4* rows_in;
    uint32_t rows_in_stride;
    uint4* rows_out;
    uint32_t* inverse;
};

// A failure injected into the look-back of the first pass, for tests of the bounded waits: tile
// `silent_tile` never publishes its status words, and every look-back wait gives up after
// `spin_limit` polls (setting kStatusLookbackTimeout) instead of the default limit.
struct SortWaitTest
{
    uint32_t silent_tile;
    uint32_t spin_limit;
};

// Launches the four passes: keys_a/values_a hold the input and, after the even number of passes,
// the output; keys_b/values_b are the ping-pong buffers. `identity_values`: the input values are
// 0 .. n-1 and are not read (values_a is still written). `scratch` holds sort_scratch_words(n)
// words, already zero, with the histograms of all four digits in its first 1024 words
// (radix_histogram or a fused producer).
// `keys_per_thread` (4, 8 or 16) sets the tile (256 * keys_per_thread keys); `scratch` then holds
// sort_scratch_words(n, keys_per_thread) words. Up to kSmallSortKeys pairs one CTA does all four
// passes in shared memory (one launch; the same permutation; scratch and histograms unused).
// `key_bits`: every key is below 2^key_bits, so only the passes of its low ceil(key_bits / 8) digits
// run (an odd count of passes ends with a copy of the result back into keys_a / values_a).
void onesweep_sort(uint32_t* keys_a, uint32_t* values_a, uint32_t* keys_b, uint32_t* values_b, uint32_t n,
                   bool identity_values, uint32_t* scratch, uint32_t* status, cudaStream_t stream,
                   const SortGather* gather = nullptr, uint32_t keys_per_thread = kSortKeysPerThread,
                   const SortWaitTest* wait_test = nullptr, uint32_t key_bits = 32);

// The number of bits of the values below `bound` (0 for bound <= 1).
inline uint32_t bits_below(uint64_t bound)
{
    uint32_t b = 0;
    while (b < 64 && (1ull << b) < bound) ++b;
    return b;
}

}  // namespace cx
