// Device-resident brick staging: the bricks a host uploads stay on the device in upload slots, so
// a flush sorts and gathers them on the device instead of re-sending every brick. Replaces, for
// the path here, the reference's staging of uploaded records (lib/src/scene/scene_flush.cpp:797-857:
// uploaded records copied to the record pages on the device).
#include <algorithm>

#include "radix_sort.cuh"
#include "scene.cuh"
#include "scene_device.cuh"

namespace cx {

namespace {

constexpr uint32_t kStageThreads = 256;

// One uint4 (8 voxels) per thread: brick src_index[j] of the upload to staging slot slots[j].
__global__ void __launch_bounds__(kStageThreads)
    staging_scatter_kernel(const uint4* __restrict__ src, const uint32_t* __restrict__ src_index,
                           const uint32_t* __restrict__ slots, uint32_t count, uint4* __restrict__ stage)
{
    const uint64_t u = (uint64_t)blockIdx.x * kStageThreads + threadIdx.x;
    if (u >= 64ull * count) return;
    const uint32_t j = (uint32_t)(u >> 6), w = (uint32_t)(u & 63u);
    stage[64ull * __ldg(slots + j) + w] = __ldg(src + 64ull * __ldg(src_index + j) + w);
}

// Compaction after a removal: slot moves[2j] takes the key and the block values of slot
// moves[2j + 1]. No destination is also a source, so the moves run in any order.
__global__ void __launch_bounds__(kStageThreads)
    staging_move_kernel(int32_t* __restrict__ keys, uint4* __restrict__ stage, const uint32_t* __restrict__ moves,
                        uint32_t count)
{
    const uint64_t u = (uint64_t)blockIdx.x * kStageThreads + threadIdx.x;
    if (u >= 64ull * count) return;
    const uint32_t j = (uint32_t)(u >> 6), w = (uint32_t)(u & 63u);
    const uint32_t dst = __ldg(moves + 2 * j), src = __ldg(moves + 2 * j + 1);
    stage[64ull * dst + w] = stage[64ull * src + w];
    if (w < 3) keys[3ull * dst + w] = keys[3ull * src + w];
}

// The linear index of a slot's brick in the grid (origin o, extents gx, gy): below 2^32 for every
// grid the flush accepts.
__global__ void __launch_bounds__(kStageThreads)
    staging_linear_kernel(const int32_t* __restrict__ keys, uint32_t n, int32_t ox, int32_t oy, int32_t oz,
                          uint32_t gx, uint32_t gy, uint32_t* __restrict__ lin)
{
    const uint32_t s = blockIdx.x * kStageThreads + threadIdx.x;
    if (s >= n) return;
    lin[s] = (uint32_t)(keys[3 * s] - ox) +
             gx * ((uint32_t)(keys[3 * s + 1] - oy) + gy * (uint32_t)(keys[3 * s + 2] - oz));
}

__global__ void __launch_bounds__(kStageThreads)
    staging_gather_kernel(const uint32_t* __restrict__ order, uint32_t n, const int32_t* __restrict__ stage_keys,
                          const uint4* __restrict__ stage_voxels, const float* __restrict__ slot_power,
                          int32_t* __restrict__ keys, uint4* __restrict__ voxels, float* __restrict__ power,
                          uint32_t* __restrict__ record_of_slot)
{
    const uint64_t u = (uint64_t)blockIdx.x * kStageThreads + threadIdx.x;
    if (u >= 64ull * n) return;
    const uint32_t i = (uint32_t)(u >> 6), w = (uint32_t)(u & 63u);
    const uint32_t s = __ldg(order + i);
    voxels[u] = __ldg(stage_voxels + 64ull * s + w);
    if (w < 3) keys[3ull * i + w] = __ldg(stage_keys + 3ull * s + w);
    if (w == 3) power[i] = slot_power ? __ldg(slot_power + s) : 0.0f;
    if (w == 4) record_of_slot[s] = i;
}

// One warp per edited slot: its values and power to its brick, then the brick and its six
// neighbours listed once each (the first warp to stamp a brick with this epoch lists it).
__global__ void __launch_bounds__(kStageThreads)
    staging_update_kernel(const uint4* __restrict__ stage_voxels, const uint32_t* __restrict__ slots,
                          const float* __restrict__ slot_power, uint32_t count,
                          const uint32_t* __restrict__ record_of_slot, const int32_t* __restrict__ keys,
                          uint4* __restrict__ voxels, float* __restrict__ power, const uint4* __restrict__ hash_slots,
                          uint32_t hash_capacity, uint32_t hash_max_probe, uint32_t* __restrict__ marks,
                          uint32_t epoch, uint32_t* __restrict__ list, uint32_t* __restrict__ list_count)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t j = (blockIdx.x * kStageThreads + threadIdx.x) >> 5;
    if (j >= count) return;
    const uint32_t s = __ldg(slots + j);
    const uint32_t r = __ldg(record_of_slot + s);
    voxels[64ull * r + lane] = __ldg(stage_voxels + 64ull * s + lane);
    voxels[64ull * r + 32 + lane] = __ldg(stage_voxels + 64ull * s + 32 + lane);
    if (lane == 0) power[r] = __ldg(slot_power + j);
    uint32_t target = 0xFFFFFFFFu;
    if (lane == 6) {
        target = r;
    } else if (lane < 6) {
        const int dx = lane == 0 ? 1 : (lane == 1 ? -1 : 0);
        const int dy = lane == 2 ? 1 : (lane == 3 ? -1 : 0);
        const int dz = lane == 4 ? 1 : (lane == 5 ? -1 : 0);
        target = hash_lookup(hash_slots, hash_capacity, hash_max_probe, keys[3ull * r] + dx, keys[3ull * r + 1] + dy,
                             keys[3ull * r + 2] + dz);
    }
    if (target != 0xFFFFFFFFu && atomicExch(marks + target, epoch) != epoch)
        list[atomicAdd(list_count, 1u)] = target;
}

uint32_t blocks(uint64_t items) { return (uint32_t)((items + kStageThreads - 1) / kStageThreads); }

}  // namespace

cudaError_t staging_scatter(const uint16_t* src, const uint32_t* src_index, const uint32_t* slots, uint32_t count,
                            uint16_t* stage_voxels, cudaStream_t stream)
{
    if (count == 0) return cudaSuccess;
    staging_scatter_kernel<<<blocks(64ull * count), kStageThreads, 0, stream>>>(
        reinterpret_cast<const uint4*>(src), src_index, slots, count, reinterpret_cast<uint4*>(stage_voxels));
    return cudaGetLastError();
}

cudaError_t staging_move(int32_t* stage_keys, uint16_t* stage_voxels, const uint32_t* moves, uint32_t count,
                         cudaStream_t stream)
{
    if (count == 0) return cudaSuccess;
    staging_move_kernel<<<blocks(64ull * count), kStageThreads, 0, stream>>>(
        stage_keys, reinterpret_cast<uint4*>(stage_voxels), moves, count);
    return cudaGetLastError();
}

uint64_t staging_sort_words(uint32_t n)
{
    const uint64_t c = std::max(n, 1u);
    return 4 * c + sort_scratch_words((uint32_t)c, kSortMinKeysPerThread);
}

cudaError_t staging_gather(const int32_t* stage_keys, const uint16_t* stage_voxels, const float* slot_power,
                           uint32_t n, const int32_t origin[3], const uint32_t grid[3], uint32_t* scratch,
                           uint32_t* status, int32_t* keys, uint16_t* voxels, float* power, uint32_t* record_of_slot,
                           cudaStream_t stream)
{
    if (n == 0) return cudaSuccess;
    uint32_t* lin = scratch;
    uint32_t* order = scratch + n;
    uint32_t* lin_alt = scratch + 2ull * n;
    uint32_t* order_alt = scratch + 3ull * n;
    uint32_t* sortw = scratch + 4ull * n;
    staging_linear_kernel<<<blocks(n), kStageThreads, 0, stream>>>(stage_keys, n, origin[0], origin[1], origin[2],
                                                                    grid[0], grid[1], lin);
    const uint32_t kpt = sort_keys_per_thread_for(n);
    CX_TRY(cudaMemsetAsync(sortw, 0, 4 * sort_scratch_words(n, kpt), stream));
    radix_histogram(lin, n, sortw, std::min<uint32_t>((n + 2047) / 2048, current_sm_count() * 4), stream);
    // A stable sort of the linear indices (unique: one slot per key), values = the slots.
    onesweep_sort(lin, order, lin_alt, order_alt, n, true, sortw, status, stream, nullptr, kpt, nullptr,
                  bits_below((uint64_t)grid[0] * grid[1] * grid[2]));
    staging_gather_kernel<<<blocks(64ull * n), kStageThreads, 0, stream>>>(
        order, n, stage_keys, reinterpret_cast<const uint4*>(stage_voxels), slot_power, keys,
        reinterpret_cast<uint4*>(voxels), power, record_of_slot);
    return cudaGetLastError();
}

cudaError_t staging_update(const uint16_t* stage_voxels, const uint32_t* slots, const float* power, uint32_t count,
                           const uint32_t* record_of_slot, DeviceScene& s, uint32_t* marks, uint32_t epoch,
                           uint32_t* list, uint32_t* list_count, cudaStream_t stream)
{
    if (count == 0) return cudaSuccess;
    staging_update_kernel<<<blocks(32ull * count), kStageThreads, 0, stream>>>(
        reinterpret_cast<const uint4*>(stage_voxels), slots, power, count, record_of_slot, s.keys,
        reinterpret_cast<uint4*>(s.voxels), s.power, s.hash_slots, s.hash_capacity, s.hash_max_probe, marks, epoch,
        list, list_count);
    return cudaGetLastError();
}

}  // namespace cx
