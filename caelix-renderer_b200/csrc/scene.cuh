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

// Block encodings (caelix_record.hlsl:180-212, include/caelix/caelix.h:243-249): which bits of a
// 16-bit block value make it opaque, the id of a transparent value and where its face bits go.
struct Encoding
{
    uint32_t opaque_mask;  // opaque when (value & opaque_mask) != 0
    uint32_t id_mask;      // the id of a transparent value
    uint32_t face_shift;   // its six face bits start here
};
__host__ __device__ constexpr Encoding encoding_of(uint32_t e)
{
    return e == kEncodingPacked ? Encoding{0xC000u, 0xFFu, 8u} : Encoding{0x8000u, 0x1FFu, 9u};
}
// The material table index of a raw block value (BlockMaterialCode): opaque values as they are,
// transparent ones without their face bits.
__host__ __device__ __forceinline__ uint32_t material_code(uint32_t v, const Encoding& e)
{
    return (v & e.opaque_mask) ? v : (v & e.id_mask);
}

// The material table on the device: one entry per 16-bit block code, two float4 (albedo rgb, 0;
// emission rgb, 0), fp32. The light code set: one bit per code whose emission luminance reaches
// the scene's min_emission.
constexpr uint32_t kMaterialCodes = 65536;
constexpr uint32_t kLightCodeWords = kMaterialCodes / 32;

struct EntityView;

// A node of the BVH over a scene's entities (their bounding-sphere boxes, world space): lo, then
// the left child (or kEntityLeaf | entity index) as a float's bits; hi, then the right child.
struct EntityNode
{
    float lo[3];
    uint32_t first;
    float hi[3];
    uint32_t second;
};
constexpr uint32_t kEntityLeaf = 0x80000000u;

// Everything the trace kernels read, passed by value.
struct SceneView
{
    uint32_t grid[3];     // bricks of the grid per axis from `origin`
    uint32_t group_shift;
    uint32_t groups[3];
    uint32_t brick_count;
    int32_t origin[3];    // brick key of grid cell 0 (a multiple of the group edge)
    Encoding enc;
    const uint32_t* records;  // [brick_count][kRecordWords]
    const uint4* hash_slots;  // key_lo, key_hi, record, 0
    uint32_t hash_capacity;
    uint32_t hash_max_probe;
    const uint32_t* bitmap;  // brick occupancy by linear brick index
    const float* power;      // per-brick emitter power (a factor of the material emission)
    const float4* materials;  // [kMaterialCodes][2]: albedo, emission
    const uint32_t* light_codes;  // [kLightCodeWords]: the light code set
    const int32_t* keys;          // [brick_count][3]: the key of every record
    // The light set of tree 0: the world's own, or, with lights in static entities, the static
    // light set (the world's light blocks, group rows, frames, power and light records first, at
    // the same indices, then the static entities' appended as for `dyn`) with tree 0 built over it.
    const uint32_t* heap;    // group light blocks, 16-byte units
    const uint32_t* group_rows;  // [group_count][8]
    const GroupFrame* frames;    // [group_count]
    const LightBvhLeaf* leaves;
    const LightBvhNode* nodes;
    const LightTreeHeader* header;
    uint32_t light_count;
    uint32_t group_count;
    // Entities beside the scene's own bricks (the static world): each traversed in its frame
    // after the world; the lights of static entities are in tree 0's light set, those of dynamic
    // ones in `dyn`.
    const EntityView* entities;  // device, entity_count of them
    uint32_t entity_count;
    const EntityNode* entity_nodes;  // the BVH over the entities (root 0), or null: test every entity
    // The dynamic entities' lights (null: none), a light set of its own in device memory (its
    // heap, group rows, frames, power and the dynamic light tree; the tree of the reference's
    // dynamic entities): entity e's groups from its group_base, its light blocks' brick words after
    // the earlier entities' bricks, every index entry's leaf word 0x80000000 | its leaf in that tree.
    const SceneView* dyn;
};

// An entity on the device: its bricks' tables (a scene of their own, entity-local block
// coordinates from 0; no lights, no entities) and its object-to-world transform,
// world = rot * local + pos (rot row-major). Replaces, for the trace, the reference's TLAS
// instance of an entity's groups (shaders/render/caelix_scene_trace.hlsl:104-131: the object ray
// of an instance, the committed object-to-world normal).
struct EntityView
{
    SceneView scene;
    float rot[9];
    float pos[3];
    uint32_t group_base;  // its first group in the light set of its tree
    float sphere[4];      // world centre and radius of a sphere holding its brick grid (inflated)
    uint32_t id;          // its entity id (the voxel id target's entity word)
    uint32_t tree;        // the tree holding its lights: 0 (static), 1 (dynamic), kNone (no light set has it)
};

// The attribute bit of an entity hit (bits 0..5 face flags, 6..14 cell, 16..31 block: bit 15 is
// free); the hit's group is then entity << 24 | the group in the entity, its normal the rotated
// face normal and its object_hit the entity-local point.
constexpr uint32_t kEntityHit = 0x8000u;
constexpr uint32_t kEntityShift = 24;
constexpr uint32_t kEntityGroupMask = (1u << kEntityShift) - 1u;

// Host-side owner of the device scene.
struct DeviceScene
{
    uint32_t grid[3] = {0, 0, 0};
    int32_t origin[3] = {0, 0, 0};
    uint32_t encoding = kEncodingBlockId;
    // The material table and the light code set the build reads (device, owned by the scene
    // object that sets them; an entity's bricks use their scene's).
    const float4* materials = nullptr;
    const uint32_t* light_codes = nullptr;
    bool lights = true;  // build the light records and the light tree (the scene's light tree is enabled)
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
    // Pinned host words the build reads back into (a read into pageable memory waits for the
    // device at every copy): [0] light count, [1] heap units, [2] [3] status words, [4] free.
    uint32_t* pinned = nullptr;
    // The group frames on the device were made for this origin, group grid and group edge.
    int32_t frames_origin[3] = {0, 0, 0};
    uint32_t frames_groups[3] = {0, 0, 0};
    uint32_t frames_shift = ~0u;
    // The light records kept for the next rebuild over the same bricks: the first unit of every
    // brick's light record in `heap` (0xFFFFFFFF: none), and the previous heap and map (the
    // buffers a rebuild over the same bricks copies unchanged records from, then swaps).
    uint32_t* unit_of_brick = nullptr;
    uint32_t* unit_of_brick_prev = nullptr;
    uint32_t* heap_prev = nullptr;
    // Group generations (GroupLightRow::generation, lib/src/light/light_tree_layout.h:217-254): per
    // group its generation (life << 16 | version) and the flags the next build compares against,
    // kept across builds for the grid they were made for (gen_count groups).
    uint32_t* group_gen = nullptr;
    uint32_t* group_flag = nullptr;
    uint32_t gen_count = 0;
    int32_t gen_origin[3] = {0, 0, 0};
    uint32_t gen_groups[3] = {0, 0, 0};
    uint32_t gen_shift = ~0u;
    // Element capacities of the buffers above: a rebuild reallocates a buffer only to grow it.
    struct
    {
        uint64_t keys, voxels, power, scratch, hash_slots, bitmap, records, group_rows, light_headers,
            light_group, light_entry, light_brick, frames, heap, heap_prev, unit_of_brick, unit_of_brick_prev, group_gen,
            group_flag;
    } capacity{};
};

// The grid of a set of brick keys: `origin` = the smallest key per axis rounded down to a multiple
// of the group edge, `grid` = the bricks from there to the largest key. False when the grid is
// larger than the tables allow (more than 2^32 cells once rounded to whole groups).
bool scene_grid(const int32_t key_min[3], const int32_t key_max[3], uint32_t group_shift, int32_t origin[3],
                uint32_t grid[3]);
// Scene build for inputs produced on the device: scene_alloc_inputs sizes s.keys, s.voxels,
// s.power for n bricks (and clears the status words); the caller fills them (keys in increasing
// linear brick index of the grid), sets s.encoding, s.materials and s.light_codes;
// scene_build_device builds everything else.
cudaError_t scene_alloc_inputs(DeviceScene& s, uint32_t n, cudaStream_t stream);
cudaError_t scene_build_device(DeviceScene& s, const int32_t origin[3], const uint32_t grid[3], uint32_t group_shift,
                               uint32_t brick_count, cudaStream_t stream, uint32_t* device_status_out);
// The parts of a rebuild whose brick set is unchanged (same keys, same order): the records of the
// bricks list[0 .. *list_count) (device; at most max_count) finalized again from s.voxels, then
// (scene_build_lights) the light records and the light tree. Synchronous.
cudaError_t scene_refinalize(DeviceScene& s, const uint32_t* list, const uint32_t* list_count, uint32_t max_count,
                             cudaStream_t stream);
// The light records of every light brick and the light tree. With `marks` (a rebuild over the
// same bricks as the previous one), a light brick b with marks[b] != epoch keeps its previous
// record (copied); the others are recomputed.
cudaError_t scene_build_lights(DeviceScene& s, cudaStream_t stream, uint32_t* device_status_out,
                               const uint32_t* marks = nullptr, uint32_t epoch = 0);

// ---- device-resident brick staging (staging.cu) ----
// Copies brick src_index[j] of an upload (src, device, 512 values per brick) to staging slot
// slots[j], j < count (the slots distinct).
cudaError_t staging_scatter(const uint16_t* src, const uint32_t* src_index, const uint32_t* slots, uint32_t count,
                            uint16_t* stage_voxels, cudaStream_t stream);
// Compaction of the staging after a removal: for j < count, slot moves[2j] takes the key and the
// block values of slot moves[2j + 1] (moves: device, no destination also a source).
cudaError_t staging_move(int32_t* stage_keys, uint16_t* stage_voxels, const uint32_t* moves, uint32_t count,
                         cudaStream_t stream);
// The staging slots in increasing linear brick index of the grid (origin, grid), gathered into the
// scene's input arrays (power zero when `power` is null). `scratch`: staging_sort_words(n) words.
uint64_t staging_sort_words(uint32_t n);
// Also writes record_of_slot[slot] = the slot's brick index in the scene.
cudaError_t staging_gather(const int32_t* stage_keys, const uint16_t* stage_voxels, const float* slot_power,
                           uint32_t n, const int32_t origin[3], const uint32_t grid[3], uint32_t* scratch,
                           uint32_t* status, int32_t* keys, uint16_t* voxels, float* power, uint32_t* record_of_slot,
                           cudaStream_t stream);
// An edit of a built scene that adds no brick: the `count` edited slots (slots[i], with power
// power[i], both device) copied to their bricks in the scene (values and power), and the list of
// the bricks whose records depend on them (each edited brick and its six neighbours, each once)
// written to list[0 .. *list_count) (list: 7 * count words; `marks`: one word per brick, holding
// `epoch` once listed, never equal to a new epoch before; *list_count zero on entry).
cudaError_t staging_update(const uint16_t* stage_voxels, const uint32_t* slots, const float* power, uint32_t count,
                           const uint32_t* record_of_slot, DeviceScene& s, uint32_t* marks, uint32_t epoch,
                           uint32_t* list, uint32_t* list_count, cudaStream_t stream);
// A merged light set (SceneView::dyn, or tree 0's static set): a part's light blocks, group rows,
// frames, power and light records copied after the earlier parts' (dst_*: device arrays sized for
// all) and their indices moved: group rows by unit_base heap units, the index entries' brick words
// by record_base, their leaf words to leaf_flag | (light_base + leaf) (0x80000000 in the dynamic
// tree, 0 in tree 0), the frames set to the part's transform, the light records' groups by
// group_base. The world as the first part of the static set (bases 0, identity transform) is a
// plain copy.
struct DynPart
{
    uint32_t group_base, unit_base, record_base, light_base;
    float rot[9], pos[3];
    uint32_t leaf_flag;
};
cudaError_t dyn_append(const DeviceScene& e, const DynPart& part, uint32_t* dst_heap, uint32_t* dst_rows,
                       GroupFrame* dst_frames, float* dst_power, BrickLightRecord* dst_headers, uint32_t* dst_group,
                       uint32_t* dst_entry, cudaStream_t stream);
// Rebuilds the light tree of a built scene from its light records (asynchronous on `stream`, no
// allocation: the tree buffers were sized by scene_build). The reference's per-flush light BVH
// rebuild (lib/src/light/light_tree_record.cpp:230-302, RecordTree).
cudaError_t scene_build_light_tree(const DeviceScene& s, cudaStream_t stream, uint32_t sort_keys_per_thread = 0);
// Reads the scene's and its light tree's device status words (synchronises `stream`).
cudaError_t scene_read_status(const DeviceScene& s, cudaStream_t stream, uint32_t* device_status_out);
void scene_release(DeviceScene& s);
SceneView scene_view(const DeviceScene& s);

}  // namespace cx
