// Kernels of the onesweep radix sort (radix_sort.cuh describes the algorithm).
#include <algorithm>
#include <atomic>

#include "cx_device.cuh"
#include "radix_sort.cuh"

namespace cx {

uint32_t current_sm_count()
{
    constexpr int kDevices = 64;
    static std::atomic<uint32_t> cache[kDevices];
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return 1;
    if (device >= 0 && device < kDevices) {
        const uint32_t known = cache[device].load(std::memory_order_relaxed);
        if (known) return known;
    }
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0) return 1;
    if (device >= 0 && device < kDevices) cache[device].store((uint32_t)sms, std::memory_order_relaxed);
    return (uint32_t)sms;
}

struct SortPass
{
    const uint32_t* keys_in;
    const uint32_t* values_in;  // nullptr: the value of element i is i
    uint32_t* keys_out;
    uint32_t* values_out;
    uint32_t n;
    uint32_t shift;
    const uint32_t* counts;  // the 256 global digit counts of this pass
    uint32_t* tile_counter;
    uint32_t* tile_states;  // tiles * 256 words, zero
    uint32_t* status;
    const uint4* rows_in;  // gathering pass: 48-byte rows by value (stride rows_in_stride uint4), else nullptr
    uint32_t rows_in_stride;
    uint4* rows_out;       // 48-byte rows by destination
    uint32_t* inverse;     // inverse[value] = destination (null: not written)
    uint32_t silent_tile;  // a tile that publishes no status (SortWaitTest), else 0xFFFFFFFF
    uint32_t spin_limit;   // polls of a look-back wait before it gives up
};

namespace {

__global__ void __launch_bounds__(256) radix_histogram_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                              uint32_t* __restrict__ hist)
{
    __shared__ uint32_t s_hist[4][kRadix];
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) (&s_hist[0][0])[i] = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
#pragma unroll
        for (int p = 0; p < 4; ++p) atomicAdd(&s_hist[p][(k >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) {
        const uint32_t c = (&s_hist[0][0])[i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// Position p of tile element k, two 16-bit positions per register (a tile holds at most 4096).
template <int KPT>
struct TilePositions
{
    uint32_t w[KPT / 2];
    __device__ __forceinline__ uint32_t get(int k) const { return (w[k >> 1] >> (16 * (k & 1))) & 0xFFFFu; }
    __device__ __forceinline__ void add(int k, uint32_t v) { w[k >> 1] += v << (16 * (k & 1)); }
};

// Stable ranks inside the warp of its KPT x 32 warp-striped keys (element k of lane l is tile
// element warp_base + 32k + l; elements at or above n take no part): pos.add(k, the number of the
// warp's earlier keys of the same digit), counts[digit] += the warp's keys of each digit. The lanes
// of equal digits come from eight ballots; the lowest of them adds their count with one shared
// atomic and broadcasts the old value.
template <int KPT>
__device__ __forceinline__ void warp_rank(const uint32_t (&key)[KPT], uint32_t warp_base, uint32_t n, uint32_t shift,
                                          uint32_t* counts, TilePositions<KPT>& pos)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = lanemask_lt();
#pragma unroll
    for (int k = 0; k < KPT; ++k) {
        const bool valid = warp_base + k * 32u + lane < n;
        const uint32_t digit = (key[k] >> shift) & 255u;
        uint32_t peers = __ballot_sync(0xFFFFFFFFu, valid);  // invalid lanes have no peers
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, (digit >> b) & 1u);
            peers &= ((digit >> b) & 1u) ? m : ~m;
        }
        const uint32_t before = __popc(peers & lt);
        uint32_t running = 0;
        if (valid && before == 0) running = atomicAdd(&counts[digit], __popc(peers));
        running = __shfl_sync(0xFFFFFFFFu, running, valid ? __ffs(peers) - 1 : lane);
        pos.add(k, running + before);
    }
}

// One onesweep pass over a tile of 256 * KPT elements. Phases:
//   1. keys (warp-striped, coalesced) -> digits -> stable rank inside the warp: the lanes of
//      equal digits from eight ballots, the warp's running count of the digit from one shared
//      atomic of the lowest such lane;
//   2. per-digit warp offsets and tile counts; the tile's counts are published at once (the
//      look-back of later tiles can proceed), then the keys go to the shared staging area in
//      tile-sorted order (their key registers are free from here on);
//   3. decoupled look-back per digit (one thread per digit, bounded spin);
//   4. values (and, on the gathering pass, the 48-byte rows) are staged by the same positions and
//      the tile is written out in runs per digit.
// The exclusive prefix of digit d over the tiles before `tile` (decoupled look-back): the states of
// kLookbackWindow predecessors are read at once, so a long walk over tiles that have published
// only their aggregates costs one round trip per window; the walk resumes at the first tile of a
// window that has published nothing yet (a bounded wait, after which kStatusLookbackTimeout is set).
constexpr int kLookbackWindow = 8;

__device__ __forceinline__ uint32_t digit_lookback(const SortPass& a, uint32_t tile, uint32_t d)
{
    uint32_t exclusive = 0;
    int64_t j = (int64_t)tile - 1;
    uint32_t spins = 0;
    while (j >= 0) {
        uint32_t st[kLookbackWindow];
#pragma unroll
        for (int w = 0; w < kLookbackWindow; ++w)
            st[w] = j - w >= 0 ? ld_relaxed(a.tile_states + (uint64_t)(j - w) * kRadix + d) : kTileFlagPrefix;
        bool done = false, stalled = false;
        int used = 0;
#pragma unroll
        for (int w = 0; w < kLookbackWindow; ++w) {
            if (!done && !stalled) {
                if ((st[w] & ~kTileValueMask) == 0) {
                    stalled = true;
                } else {
                    exclusive += st[w] & kTileValueMask;
                    used = w + 1;
                    done = (st[w] & kTileFlagPrefix) != 0;
                }
            }
        }
        if (done) break;
        j -= used;
        if (stalled && !spin_wait(spins, a.spin_limit)) {
            atomicOr(a.status, kStatusLookbackTimeout);
            break;
        }
    }
    return exclusive;
}

template <int KPT>
__global__ void __launch_bounds__(kSortThreads, 4) onesweep_pass_kernel(const SortPass a)
{
    constexpr int kTile = kSortThreads * KPT;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp_counts[kSortWarps][kRadix];  // counts, then exclusive offsets per warp
    __shared__ uint32_t s_local[kRadix];                    // tile-local exclusive offset of each digit
    __shared__ uint32_t s_dest[kRadix];                     // global destination base minus s_local
    __shared__ uint32_t s_scan[kSortWarps];
    __shared__ uint32_t s_keys[kTile];
    __shared__ uint32_t s_values[kTile];

    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1u);
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) s_warp_counts[w][tid] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * kTile;
    const uint32_t warp_base = base + warp * 32u * KPT;

    // Phase 1.
    uint32_t key[KPT];
    TilePositions<KPT> pos;  // rank in the warp, then position in the tile
#pragma unroll
    for (int k = 0; k < KPT / 2; ++k) pos.w[k] = 0;
#pragma unroll
    for (int k = 0; k < KPT; ++k) {
        const uint32_t i = warp_base + k * 32u + lane;
        key[k] = i < a.n ? __ldg(a.keys_in + i) : 0u;
    }
    warp_rank<KPT>(key, warp_base, a.n, a.shift, s_warp_counts[warp], pos);
    __syncthreads();

    // Phase 2: thread d owns digit d.
    const uint32_t d = tid;
    uint32_t total = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
        const uint32_t c = s_warp_counts[w][d];
        s_warp_counts[w][d] = total;
        total += c;
    }
    uint32_t* state = a.tile_states + (uint64_t)tile * kRadix + d;
    const bool publish = tile != a.silent_tile;
    if (publish) st_relaxed(state, (tile == 0 ? kTileFlagPrefix : kTileFlagAggregate) | total);
    uint32_t tile_total;
    const uint32_t local = block_exclusive_sum<kSortThreads>(total, s_scan, tile_total);
    s_local[d] = local;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < KPT; ++k) {
        const uint32_t i = warp_base + k * 32u + lane;
        if (i < a.n) {
            const uint32_t digit = (key[k] >> a.shift) & 255u;
            pos.add(k, s_local[digit] + s_warp_counts[warp][digit]);
            s_keys[pos.get(k)] = key[k];
        }
    }

    // Phase 3: the exclusive prefix of digit d over the earlier tiles.
    uint32_t exclusive = 0;
    if (tile != 0) {
        exclusive = digit_lookback(a, tile, d);
        if (publish) st_relaxed(state, kTileFlagPrefix | (exclusive + total));
    }
    uint32_t digit_total;
    const uint32_t global_base = block_exclusive_sum<kSortThreads>(a.counts[d], s_scan, digit_total);
    s_dest[d] = global_base + exclusive - local;

    // Phase 4.
#pragma unroll
    for (int k = 0; k < KPT; ++k) {
        const uint32_t i = warp_base + k * 32u + lane;
        if (i < a.n) s_values[pos.get(k)] = a.values_in ? __ldg(a.values_in + i) : i;
    }
    __syncthreads();
    const uint32_t count = a.n - base < (uint32_t)kTile ? a.n - base : (uint32_t)kTile;
    for (uint32_t j = tid; j < count; j += kSortThreads) {
        const uint32_t k = s_keys[j];
        const uint32_t v = s_values[j];
        const uint32_t dest = s_dest[(k >> a.shift) & 255u] + j;
        a.keys_out[dest] = k;
        a.values_out[dest] = v;
        if (a.rows_in) {
            const uint4* src = a.rows_in + (uint64_t)a.rows_in_stride * v;
            uint4* dst = a.rows_out + 3ull * dest;
            const uint4 r0 = __ldg(src);
            const uint4 r1 = __ldg(src + 1);
            const uint4 r2 = __ldg(src + 2);
            dst[0] = r0;
            dst[1] = r1;
            dst[2] = r2;
            if (a.inverse) a.inverse[v] = dest;
        }
    }
}

// ---------------------------------------------------------------------------------------------
// The persistent, software-pipelined pass: a CTA stays resident and takes tile after tile. While
// it ranks, looks back and writes one tile, the keys and values of its next tile come into shared
// memory by 1-D bulk copies (cp.async.bulk, completion counted on an mbarrier of the CTA; the
// source is this GPU's own memory), so the loads of a tile overlap the look-back and the stores of
// the tile before, and the values are in shared memory before the look-back ends. The ranking, the
// look-back and the output are the plain pass's (the same stable permutation). Two CTAs per SM.
constexpr uint32_t kPipeTile = kSortThreads * kSortKeysPerThread;  // 4096

struct PipeShared
{
    uint32_t raw_keys[2][kPipeTile];
    uint32_t raw_values[2][kPipeTile];
    uint32_t keys[kPipeTile];
    uint32_t values[kPipeTile];
    uint32_t warp_counts[kSortWarps][kRadix];
    uint32_t local[kRadix];
    uint32_t dest[kRadix];
    uint32_t base[kRadix];
    uint32_t scan[kSortWarps];
    uint32_t tile[2];
    unsigned long long bar[2];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t arrivals)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(arrivals) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, unsigned long long* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Thread 0: the bulk copies of tile t into stage `stage` (its whole 16-byte units; the tail of a
// last tile is loaded by plain loads after the wait).
__device__ __forceinline__ void pipe_issue(const SortPass& a, PipeShared& S, uint32_t t, uint32_t stage)
{
    const uint32_t base = t * kPipeTile;
    const uint32_t count = min(a.n - base, kPipeTile);
    const uint32_t bytes = (count * 4u) & ~15u;
    const bool values = a.values_in != nullptr;
    // Reads of this buffer by the generic proxy (the tile two steps back) come before the copy.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&S.bar[stage], values ? 2u * bytes : bytes);
    if (bytes) {
        bulk_load(S.raw_keys[stage], a.keys_in + base, bytes, &S.bar[stage]);
        if (values) bulk_load(S.raw_values[stage], a.values_in + base, bytes, &S.bar[stage]);
    }
}

__global__ void __launch_bounds__(kSortThreads, 2) onesweep_pipe_kernel(const SortPass a, uint32_t tiles)
{
    extern __shared__ __align__(128) unsigned char pipe_smem[];
    PipeShared& S = *reinterpret_cast<PipeShared*>(pipe_smem);
    constexpr int KPT = kSortKeysPerThread;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const uint32_t d = tid;  // the digit of this thread in the per-digit phases
    {
        uint32_t digit_total;
        S.base[d] = block_exclusive_sum<kSortThreads>(a.counts[d], S.scan, digit_total);
    }
    if (tid == 0) {
        mbar_init(&S.bar[0], 1);
        mbar_init(&S.bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        const uint32_t t = atomicAdd(a.tile_counter, 1u);
        S.tile[0] = t;
        if (t < tiles) pipe_issue(a, S, t, 0);
    }
    __syncthreads();
    uint32_t stage = 0, parity = 0;  // parity bit s: the phase of stage s's barrier to wait for
    for (;;) {
        const uint32_t tile = S.tile[stage];
        if (tile >= tiles) break;
        if (tid == 0) {
            const uint32_t next = atomicAdd(a.tile_counter, 1u);
            S.tile[stage ^ 1u] = next;
            if (next < tiles) pipe_issue(a, S, next, stage ^ 1u);
        }
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) S.warp_counts[w][tid] = 0;
        // This tile's copies (a bounded wait: a copy that never lands sets a status bit).
        {
            const uint32_t ph = (parity >> stage) & 1u;
            uint32_t spins = 0;
            while (!mbar_try_wait(&S.bar[stage], ph)) {
                if (!spin_wait(spins)) {
                    if (tid == 0) atomicOr(a.status, kStatusCopyTimeout);
                    break;
                }
            }
            parity ^= 1u << stage;
        }
        const uint32_t base = tile * kPipeTile;
        const uint32_t count = min(a.n - base, kPipeTile);
        const uint32_t bulk = ((count * 4u) & ~15u) / 4u;
        if (tid < count - bulk) {  // the last tile's tail (under 4 elements)
            S.raw_keys[stage][bulk + tid] = __ldg(a.keys_in + base + bulk + tid);
            if (a.values_in) S.raw_values[stage][bulk + tid] = __ldg(a.values_in + base + bulk + tid);
        }
        __syncthreads();
        const uint32_t warp_base = base + warp * 32u * KPT;
        const uint32_t local_base = warp * 32u * KPT;
        uint32_t key[KPT];
        TilePositions<KPT> pos;
#pragma unroll
        for (int k = 0; k < KPT / 2; ++k) pos.w[k] = 0;
#pragma unroll
        for (int k = 0; k < KPT; ++k) {
            const uint32_t e = local_base + k * 32u + lane;
            key[k] = e < count ? S.raw_keys[stage][e] : 0u;
        }
        warp_rank<KPT>(key, warp_base, a.n, a.shift, S.warp_counts[warp], pos);
        __syncthreads();
        uint32_t total = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = S.warp_counts[w][d];
            S.warp_counts[w][d] = total;
            total += c;
        }
        uint32_t* state = a.tile_states + (uint64_t)tile * kRadix + d;
        const bool publish = tile != a.silent_tile;
        if (publish) st_relaxed(state, (tile == 0 ? kTileFlagPrefix : kTileFlagAggregate) | total);
        uint32_t tile_total;
        const uint32_t local = block_exclusive_sum<kSortThreads>(total, S.scan, tile_total);
        S.local[d] = local;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < KPT; ++k) {
            const uint32_t e = local_base + k * 32u + lane;
            if (e < count) {
                const uint32_t digit = (key[k] >> a.shift) & 255u;
                pos.add(k, S.local[digit] + S.warp_counts[warp][digit]);
                const uint32_t p = pos.get(k);
                S.keys[p] = key[k];
                S.values[p] = a.values_in ? S.raw_values[stage][e] : base + e;
            }
        }
        uint32_t exclusive = 0;
        if (tile != 0) {
            exclusive = digit_lookback(a, tile, d);
            if (publish) st_relaxed(state, kTileFlagPrefix | (exclusive + total));
        }
        S.dest[d] = S.base[d] + exclusive - local;
        __syncthreads();
        for (uint32_t j = tid; j < count; j += kSortThreads) {
            const uint32_t k = S.keys[j];
            const uint32_t v = S.values[j];
            const uint32_t dest = S.dest[(k >> a.shift) & 255u] + j;
            a.keys_out[dest] = k;
            a.values_out[dest] = v;
            if (a.rows_in) {
                const uint4* src = a.rows_in + (uint64_t)a.rows_in_stride * v;
                uint4* dst = a.rows_out + 3ull * dest;
                const uint4 r0 = __ldg(src);
                const uint4 r1 = __ldg(src + 1);
                const uint4 r2 = __ldg(src + 2);
                dst[0] = r0;
                dst[1] = r1;
                dst[2] = r2;
                if (a.inverse) a.inverse[v] = dest;
            }
        }
        __syncthreads();
        stage ^= 1u;
    }
}

// A whole sort of n <= kSmallSortKeys pairs by one CTA: the passes of the onesweep ranking that the
// keys' digits need, over one tile held in shared memory (a stable LSD sort: the same permutation
// as the onesweep passes), then the output with the optional row gather of the last pass. One
// launch instead of four for the small sorts of small light trees.
constexpr int kSmallSortKeysPerThread = 16;
static_assert(kSmallSortKeys == kSortThreads * kSmallSortKeysPerThread, "one tile");

template <bool kIdentity>
__global__ void __launch_bounds__(kSortThreads) small_sort_kernel(uint32_t* __restrict__ keys,
                                                                  uint32_t* __restrict__ values, uint32_t n,
                                                                  uint32_t passes, const SortGather gather)
{
    constexpr int KPT = kSmallSortKeysPerThread;
    __shared__ uint32_t s_warp_counts[kSortWarps][kRadix];
    __shared__ uint32_t s_local[kRadix];
    __shared__ uint32_t s_scan[kSortWarps];
    __shared__ uint32_t s_keys[kSmallSortKeys];
    __shared__ uint32_t s_values[kSmallSortKeys];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    for (uint32_t i = tid; i < n; i += kSortThreads) {
        s_keys[i] = keys[i];
        s_values[i] = kIdentity ? i : values[i];
    }
    const uint32_t warp_base = warp * 32u * KPT;
    for (uint32_t pass = 0; pass < passes; ++pass) {
        const uint32_t shift = 8 * pass;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) s_warp_counts[w][tid] = 0;
        __syncthreads();
        uint32_t key[KPT], val[KPT];
#pragma unroll
        for (int k = 0; k < KPT; ++k) {
            const uint32_t i = warp_base + k * 32u + lane;
            key[k] = i < n ? s_keys[i] : 0u;
            val[k] = i < n ? s_values[i] : 0u;
        }
        TilePositions<KPT> pos;
#pragma unroll
        for (int k = 0; k < KPT / 2; ++k) pos.w[k] = 0;
        warp_rank<KPT>(key, warp_base, n, shift, s_warp_counts[warp], pos);
        __syncthreads();
        // Thread d owns digit d: the warps' exclusive offsets and the tile offset of the digit.
        const uint32_t d = tid;
        uint32_t total = 0;
#pragma unroll
        for (int w = 0; w < kSortWarps; ++w) {
            const uint32_t c = s_warp_counts[w][d];
            s_warp_counts[w][d] = total;
            total += c;
        }
        uint32_t tile_total;
        s_local[d] = block_exclusive_sum<kSortThreads>(total, s_scan, tile_total);
        __syncthreads();
#pragma unroll
        for (int k = 0; k < KPT; ++k) {
            if (warp_base + k * 32u + lane < n) {
                const uint32_t digit = (key[k] >> shift) & 255u;
                const uint32_t p = pos.get(k) + s_local[digit] + s_warp_counts[warp][digit];
                s_keys[p] = key[k];
                s_values[p] = val[k];
            }
        }
        __syncthreads();
    }
    for (uint32_t i = tid; i < n; i += kSortThreads) {
        const uint32_t v = s_values[i];
        keys[i] = s_keys[i];
        values[i] = v;
        if (gather.rows_in) {
            const uint4* src = gather.rows_in + (uint64_t)gather.rows_in_stride * v;
            uint4* dst = gather.rows_out + 3ull * i;
            dst[0] = __ldg(src);
            dst[1] = __ldg(src + 1);
            dst[2] = __ldg(src + 2);
            if (gather.inverse) gather.inverse[v] = i;
        }
    }
}

// A whole sort of n <= kRankSortKeys pairs by one CTA without passes: each element's place is the
// count of smaller keys plus the count of equal keys before it (the stable order), counted over the
// keys in shared memory; the optional row gather as in small_sort_kernel.
constexpr uint32_t kRankSortKeys = 512;

template <bool kIdentity>
__global__ void __launch_bounds__(kSortThreads) rank_sort_kernel(uint32_t* __restrict__ keys,
                                                                 uint32_t* __restrict__ values, uint32_t n,
                                                                 const SortGather gather)
{
    __shared__ uint32_t s_keys[kRankSortKeys];
    __shared__ uint32_t s_values[kRankSortKeys];
    const uint32_t tid = threadIdx.x;
    for (uint32_t i = tid; i < n; i += kSortThreads) {
        s_keys[i] = keys[i];
        s_values[i] = kIdentity ? i : values[i];
    }
    __syncthreads();
    for (uint32_t i = tid; i < n; i += kSortThreads) {
        const uint32_t k = s_keys[i];
        uint32_t r = 0;
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t kj = s_keys[j];
            r += (kj < k || (kj == k && j < i)) ? 1u : 0u;
        }
        const uint32_t v = s_values[i];
        keys[r] = k;
        values[r] = v;
        if (gather.rows_in) {
            const uint4* src = gather.rows_in + (uint64_t)gather.rows_in_stride * v;
            uint4* dst = gather.rows_out + 3ull * r;
            dst[0] = __ldg(src);
            dst[1] = __ldg(src + 1);
            dst[2] = __ldg(src + 2);
            if (gather.inverse) gather.inverse[v] = r;
        }
    }
}

}  // namespace

void radix_histogram(const uint32_t* keys, uint32_t n, uint32_t* hist, uint32_t grid, cudaStream_t stream)
{
    if (n == 0) return;
    radix_histogram_kernel<<<grid, 256, 0, stream>>>(keys, n, hist);
}

void onesweep_sort(uint32_t* keys_a, uint32_t* values_a, uint32_t* keys_b, uint32_t* values_b, uint32_t n,
                   bool identity_values, uint32_t* scratch, uint32_t* status, cudaStream_t stream,
                   const SortGather* gather, uint32_t keys_per_thread, const SortWaitTest* wait_test,
                   uint32_t key_bits)
{
    if (n == 0) return;
    const uint32_t passes = key_bits >= 32 ? 4u : std::max(1u, (key_bits + 7u) / 8u);
    if (n <= kSmallSortKeys) {
        const SortGather g = gather ? *gather : SortGather{nullptr, 0, nullptr, nullptr};
        if (n <= kRankSortKeys) {
            if (identity_values) rank_sort_kernel<true><<<1, kSortThreads, 0, stream>>>(keys_a, values_a, n, g);
            else rank_sort_kernel<false><<<1, kSortThreads, 0, stream>>>(keys_a, values_a, n, g);
        } else if (identity_values) {
            small_sort_kernel<true><<<1, kSortThreads, 0, stream>>>(keys_a, values_a, n, passes, g);
        } else {
            small_sort_kernel<false><<<1, kSortThreads, 0, stream>>>(keys_a, values_a, n, passes, g);
        }
        return;
    }
    if (!sort_keys_per_thread_ok(keys_per_thread)) keys_per_thread = kSortKeysPerThread;
    const uint32_t tiles = sort_tiles(n, keys_per_thread);
    // The pipelined pass for sorts of at least kPipeMinTiles tiles of 4096 pairs whose arrays start
    // on 16-byte boundaries (the bulk copies' rule); the plain pass otherwise.
    const auto aligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    const bool pipe = keys_per_thread == (uint32_t)kSortKeysPerThread && tiles >= kPipeMinTiles && aligned(keys_a) &&
                      aligned(keys_b) && aligned(values_a) && aligned(values_b);
    uint32_t pipe_grid = 0;
    if (pipe) {
        static int per_sm = 0;
        if (per_sm == 0) {
            cudaFuncSetAttribute(onesweep_pipe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)sizeof(PipeShared));
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, onesweep_pipe_kernel, kSortThreads,
                                                          sizeof(PipeShared));
            per_sm = per_sm > 0 ? per_sm : 1;
        }
        pipe_grid = std::min<uint32_t>(tiles, current_sm_count() * (uint32_t)per_sm);
    }
    uint32_t* hist = scratch;
    uint32_t* counters = scratch + 4 * kRadix;
    uint32_t* states = counters + 4;
    uint32_t* kin = keys_a;
    uint32_t* vin = values_a;
    uint32_t* kout = keys_b;
    uint32_t* vout = values_b;
    for (uint32_t pass = 0; pass < passes; ++pass) {
        SortPass p;
        p.keys_in = kin;
        p.values_in = (pass == 0 && identity_values) ? nullptr : vin;
        p.keys_out = kout;
        p.values_out = vout;
        p.n = n;
        p.shift = 8 * pass;
        p.counts = hist + kRadix * pass;
        p.tile_counter = counters + pass;
        p.tile_states = states + (uint64_t)pass * tiles * kRadix;
        p.status = status;
        const bool last = pass + 1 == passes;
        p.rows_in = (last && gather) ? gather->rows_in : nullptr;
        p.rows_in_stride = gather ? gather->rows_in_stride : 0;
        p.rows_out = (last && gather) ? gather->rows_out : nullptr;
        p.inverse = (last && gather) ? gather->inverse : nullptr;
        p.silent_tile = (pass == 0 && wait_test) ? wait_test->silent_tile : 0xFFFFFFFFu;
        p.spin_limit = wait_test ? wait_test->spin_limit : kSpinLimit;
        if (pipe) onesweep_pipe_kernel<<<pipe_grid, kSortThreads, sizeof(PipeShared), stream>>>(p, tiles);
        else if (keys_per_thread == 4) onesweep_pass_kernel<4><<<tiles, kSortThreads, 0, stream>>>(p);
        else if (keys_per_thread == 8) onesweep_pass_kernel<8><<<tiles, kSortThreads, 0, stream>>>(p);
        else onesweep_pass_kernel<16><<<tiles, kSortThreads, 0, stream>>>(p);
        uint32_t* t = kin;
        kin = kout;
        kout = t;
        t = vin;
        vin = vout;
        vout = t;
    }
    if (passes & 1u) {  // the result is in keys_b / values_b
        cudaMemcpyAsync(keys_a, keys_b, 4ull * n, cudaMemcpyDeviceToDevice, stream);
        cudaMemcpyAsync(values_a, values_b, 4ull * n, cudaMemcpyDeviceToDevice, stream);
    }
}

}  // namespace cx
