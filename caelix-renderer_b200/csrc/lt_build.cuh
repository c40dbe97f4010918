// The light BVH build on the GPU: brick light records -> world leaves -> Morton codes -> onesweep
// radix sort -> Karras binary radix tree -> depth parity + scan -> bottom-up aggregation with the
// 4-wide collapse -> header.
//
// Replaces the reference's per-tree dispatch sequence LightTree::RecordTree
// (lib/src/light/light_tree_record.cpp:230-309, about 35 dependent dispatches with a barrier after
// each) with 14 kernels and one memset at 4,097 leaves and more (one small-sort CTA in place of
// the four sort passes below that), all on one stream (capturable in a CUDA graph):
//   lt_emit_kernel        gather emit (caelix_light_gather_emit.hlsl:11-86) fused with the centre
//                         bounds (caelix_light_bvh_bounds.hlsl:10-53): warp max-reductions of
//                         order-preserving codes instead of a one-workgroup reduction
//   lt_morton_kernel      Morton codes (caelix_light_bvh_morton.hlsl:6-28) fused with the digit
//                         histograms of all four sort passes and the clear of the arrival counters
//   onesweep_pipe_kernel  x4 (radix_sort.cuh); later kernels read a sorted leaf through the
//                         permutation
//   lt_karras_kernel      caelix_light_bvh_karras.hlsl:8-96, plus the range-count differences
//   lt_cover_scan_kernel  the depths (caelix_light_bvh_depth.hlsl:7-30) without walking to the
//   lt_flags_scan_kernel  root: depth(i) + 1 = the number of binary nodes whose range spans node i's
//                         split boundary (node i and its ancestors), a prefix sum of +1/-1 range
//                         ends; then the even-depth flags scanned into 4-wide indices (single-pass
//                         decoupled look-back scans instead of the one-workgroup scan)
//   lt_tile_kernel        by tiles of 256 sorted leaves in shared memory: the aggregation
//                         (caelix_light_bvh_aggregate.hlsl:30-55) of the nodes inside the tile and
//                         the 4-wide nodes over them (caelix_light_bvh_wide.hlsl:10-100)
//   lt_aggregate_upper_kernel  the aggregation of the nodes that cross tiles (acq_rel arrivals; two
//                         variants, one CTA for up to 1,024 walks or a persistent grid)
//   lt_wide_upper_kernel  the 4-wide nodes over the nodes that cross tiles
//   lt_finish_kernel      caelix_light_bvh_finish.hlsl:8-63
// Every float operation is a single IEEE fp32 operation in the order of the HLSL source (the
// library is compiled with --fmad=false), so the tree is bit-identical to the oracle's.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "cx_layout.h"
#include "radix_sort.cuh"

namespace cx {

// Per-tree build state, persistent across builds (LightTreeState, light_tree_layout.h:123-148).
struct alignas(16) LightTreeState
{
    uint32_t building;
    uint32_t leaves_found;
    uint32_t leaves_dropped;
    uint32_t builds;
    uint32_t node_overflow;
    uint32_t status;  // cx::kStatus* bits of the newest build
    uint32_t pad0[2];
    float bounds[6];  // centre bounds lo[3], hi[3]
    uint32_t pad1[2];
};
static_assert(sizeof(LightTreeState) == 64);

// The control words a build zeroes before its first kernel.
struct BuildControl
{
    uint32_t bounds_code[6];  // [0..2] ~order(min centre), [3..5] order(max centre): atomicMax from 0
    uint32_t status;
    uint32_t node_count;         // the scan total of the even-depth flags
    uint32_t scan_tile_counter;  // unused
    uint32_t upper_count;        // walks the tile kernel hands to lt_aggregate_upper_kernel
    uint32_t crossing_count;     // even-depth nodes the tile kernel hands to lt_wide_upper_kernel
    uint32_t pad[5];
};
static_assert(sizeof(BuildControl) == 64);

// A binary node's summary padded to 64 bytes, so that every aggregate write covers two whole
// 32-byte sectors.
struct alignas(16) AggregateSlot
{
    LightSummary summary;
    uint32_t pad[4];
};
static_assert(sizeof(AggregateSlot) == 64);

// Device arrays of one tree and its build scratch (the kLtScratch* arrays of
// light_tree_layout.h:392-423, here separate arrays).
struct LightBvhBuffers
{
    uint32_t leaf_capacity = 0;
    uint32_t node_capacity = 0;
    LightBvhLeaf* leaves = nullptr;
    LightBvhNode* nodes = nullptr;
    LightTreeHeader* header = nullptr;  // header then LightTreeState, 128 bytes
    LightTreeState* state = nullptr;
    uint32_t* keys = nullptr;  // sorted Morton codes after the build
    uint32_t* values = nullptr;
    uint32_t* keys_alt = nullptr;
    uint32_t* values_alt = nullptr;
    uint32_t* left = nullptr;
    uint32_t* right = nullptr;
    uint32_t* parent = nullptr;
    uint32_t* leaf_parent = nullptr;
    uint32_t* counter = nullptr;
    uint32_t* depth = nullptr;
    uint32_t* wide = nullptr;
    uint32_t* cover = nullptr;      // range-count differences, then the nodes over each leaf boundary
    AggregateSlot* aggregates = nullptr;
    LightSummary* sorted = nullptr;  // leaf summaries in sorted order
    BuildControl* control = nullptr;  // followed by the sort scratch, then the scan states
    uint32_t* sort_scratch = nullptr;
};

// Input of one build: `count` records (device), optional per-record group and entry words and
// group_count per-group frames (device; null: group 0, entry = record index, identity frame at
// origin 0).
struct LightBvhInput
{
    const BrickLightRecord* records;
    uint32_t count;
    const uint32_t* record_group;
    const uint32_t* record_entry;
    const GroupFrame* group_frames;
    uint32_t group_count;
    uint32_t sort_keys_per_thread = kSortKeysPerThread;  // the radix sort's tile: 256 x 4, 8 or 16 keys (0: by size)
};

constexpr int kScanThreads = 256;

// Bytes of device memory for a leaf capacity (one allocation, carved by lt_carve).
uint64_t lt_buffer_bytes(uint32_t leaf_capacity);
// Carves the arrays of `leaf_capacity` leaves out of `base` (lt_buffer_bytes bytes, 256-aligned).
LightBvhBuffers lt_carve(void* base, uint32_t leaf_capacity);
// Stages of a build that lt_build can bracket with events: stage[k] is recorded after stage k - 1
// (stage[0] before the first command): emit+bounds, morton+histograms, sort (4 passes and the
// gather), karras, depth+scan, tile aggregation and collapse + upper aggregation, upper collapse +
// finish.
constexpr int kBuildStages = 7;
// Records the build into `stream`; `stage` (null, or kBuildStages + 1 events) brackets its stages.
// Returns the first CUDA launch error.
cudaError_t lt_build(const LightBvhBuffers& b, const LightBvhInput& in, cudaStream_t stream, cudaEvent_t* stage);
// Kernels one build of n leaves launches.
uint32_t lt_kernel_launches(uint32_t n);

}  // namespace cx
