// The scene on the device: brick records, the brick hash table, the brick occupancy bitmap, the
// light records (group light blocks) and the light tree. Built by scene_build (scene.cu) from
// raw bricks; read by the trace kernels (trace.cu).
//
// Replaces, for the trace path, the reference's scene tables and acceleration structures
// (lib/src/scene/scene_bricks.cpp, scene_accel.cpp: page table, slot rows, BLAS/TLAS) with a
// brick-keyed hash table and a brick occupancy bitmap, and the light tree's group pass
// (shaders/light/records/*.hlsl) with a one-shot record producer (every light brick recomputed).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "cx_layout.h"
#include "lt_build.cuh"

namespace cx {

constexpr uint32_t kOpaqueBit = 0x8000u;  // block-ID encoding
constexpr uint32_t kMaterialSlots = 128;  // albedo table rows (material id = value & 0x7F)

// Everything the trace kernels read, passed by value.
struct SceneView
{
    uint32_t grid[3];
    uint32_t group_shift;
    uint32_t groups[3];
    uint32_t brick_count;
    const uint32_t* records;  // [brick_count][kRecordWords]
    const uint4* hash_slots;  // key_lo, key_hi, record, 0
    uint32_t hash_capacity;
    uint32_t hash_max_probe;
    const uint32_t* bitmap;  // brick occupancy by linear brick index
    const float* power;      // per-brick emitter power
    const float* albedo;     // [kMaterialSlots][3]
    const uint32_t* heap;    // group light blocks, 16-byte units
    const uint32_t* group_rows;  // [group_count][8]
    const GroupFrame* frames;    // [group_count]
    const LightBvhLeaf* leaves;
    const LightBvhNode* nodes;
    const LightTreeHeader* header;
    uint32_t light_count;
    uint32_t group_count;
};

// Host-side owner of the device scene.
struct DeviceScene
{
    uint32_t grid[3] = {0, 0, 0};
    uint32_t group_shift = 4;
    uint32_t groups[3] = {0, 0, 0};
    uint32_t group_count = 0;
    uint32_t brick_count = 0;
    uint32_t hash_capacity = 0;
    uint32_t hash_slot_count = 0;
    uint32_t hash_max_probe = 0;
    uint32_t light_count = 0;
    uint32_t heap_words = 0;
    uint64_t light_faces = 0;
    // Device buffers (cudaMalloc'd, owned).
    int32_t* keys = nullptr;
    uint16_t* voxels = nullptr;
    float* power = nullptr;
    uint32_t* records = nullptr;
    uint4* hash_slots = nullptr;
    uint32_t* bitmap = nullptr;
    float* albedo = nullptr;
    uint32_t* heap = nullptr;
    uint32_t* group_rows = nullptr;
    GroupFrame* frames = nullptr;
    BrickLightRecord* light_headers = nullptr;
    uint32_t* light_group = nullptr;
    uint32_t* light_entry = nullptr;
    uint32_t* light_brick = nullptr;
    uint32_t* scratch = nullptr;  // build scratch (sort, scans)
    uint64_t scratch_words = 0;
    void* tree_memory = nullptr;
    LightBvhBuffers tree;
    uint32_t tree_capacity = 0;
    uint32_t* status = nullptr;  // device status word of the build
};

// Builds the device scene from host bricks (keys in increasing linear brick index, every
// coordinate in [0, grid)), voxels (512 block values per brick), per-brick power and the albedo
// table (kMaterialSlots x 3). Synchronous on `stream`. Returns the first CUDA error.
cudaError_t scene_build(DeviceScene& s, const uint32_t grid[3], uint32_t group_shift, uint32_t brick_count,
                        const int32_t* keys, const uint16_t* voxels, const float* power, const float* albedo,
                        cudaStream_t stream, uint32_t* device_status_out);
// Rebuilds the light tree of a built scene from its light records (asynchronous on `stream`, no
// allocation: the tree buffers were sized by scene_build). The reference's per-flush light BVH
// rebuild (lib/src/light/light_tree_record.cpp:230-302, RecordTree).
cudaError_t scene_build_light_tree(const DeviceScene& s, cudaStream_t stream,
                                   uint32_t sort_keys_per_thread = kSortKeysPerThread);
// Reads the scene's and its light tree's device status words (synchronises `stream`).
cudaError_t scene_read_status(const DeviceScene& s, cudaStream_t stream, uint32_t* device_status_out);
void scene_release(DeviceScene& s);
SceneView scene_view(const DeviceScene& s);

}  // namespace cx
