// The scene and renderer objects behind the C ABI, shared by abi_scene.cu and abi_batch.cu.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <unordered_map>
#include <vector>

#include "../../include/caelix_b200.h"
#include "abi_internal.h"
#include "scene.cuh"
#include "trace.cuh"

// A merged light set on the device (the dynamic entities' lights, or tree 0's static set: the
// world's lights and the static entities'): its arrays, its light tree, the device copy of its
// SceneView (the dynamic set's), the tree's build input and the view itself (null pointers when
// not live).
struct LightSet
{
    cx::GrowBuffer arrays;
    cx::GrowBuffer tree;
    cx::GrowBuffer view;
    uint32_t tree_capacity = 0;
    bool live = false;
    cx::LightBvhInput input{};
    cx::SceneView v{};
    void release()
    {
        arrays.release();
        tree.release();
        view.release();
        tree_capacity = 0;
        live = false;
    }
};

struct CaelixScene
{
    CaelixDevice* device = nullptr;
    uint32_t group_shift = 4;
    uint32_t encoding = cx::kEncodingPacked;
    // An entity's bricks are a scene of their own under the scene that holds the entity (`parent`):
    // they use its material table, light code set and light options.
    CaelixScene* parent = nullptr;
    // Brick staging. Slot s holds the brick keys[3s .. 3s+2]; its 512 block values stay on the
    // device (stage_voxels[512s ..], copied there by the upload that wrote them), its key in
    // stage_keys[3s ..] and its power in slot_power[s].
    std::unordered_map<uint64_t, uint32_t> slot_of;
    std::vector<int32_t> keys;
    std::vector<float> slot_power;
    std::unordered_map<uint64_t, float> pending_power;  // power of keys not uploaded yet (default 1)
    int32_t key_min[3] = {0, 0, 0};
    int32_t key_max[3] = {0, 0, 0};
    uint32_t stage_capacity = 0;  // slots
    int32_t* stage_keys = nullptr;
    uint16_t* stage_voxels = nullptr;
    cudaStream_t upload_stream = nullptr;
    cx::GrowBuffer upload;         // one upload's block values and slot lists
    cx::GrowBuffer flush_scratch;  // slot powers, linear indices and the sort of a flush
    std::vector<uint32_t> upload_mark;  // per slot: the last upload that wrote it
    uint32_t upload_epoch = 0;
    // Edits since the last flush. A full rebuild follows a new key (or the first flush, or a
    // light-tree toggle); otherwise only the edited slots are copied to their bricks and their
    // records (and their neighbours') finalized again.
    bool full_rebuild = true;
    std::vector<uint32_t> dirty_slots;
    std::vector<uint8_t> slot_dirty;
    bool materials_dirty = true;  // the device table and light code set are stale
    cx::GrowBuffer record_of_slot;  // device: the brick index of every slot (the last full build)
    cx::GrowBuffer marks;           // device: one word per brick (staging_update)
    uint32_t mark_epoch = 0;
    cx::GrowBuffer update;          // device: edited slots, their power, the refinalize list
    uint32_t* edit_host = nullptr;  // pinned host: an edit flush's slots and their power
    uint64_t edit_host_words = 0;
    uint32_t last_update_records = 0;  // records finalized again by the last incremental flush
    // The material table (host copy, one entry per 16-bit code), its device form (two float4 per
    // code: albedo, emission) and the light code set (codes whose emission luminance reaches
    // min_emission), host and device.
    std::vector<CaelixMaterial> materials;
    std::vector<uint32_t> light_codes;
    cx::GrowBuffer materials_dev;
    cx::GrowBuffer light_codes_dev;
    CaelixLightOptions light_options{0, 20.0f, 16ull << 20};
    bool light_tree_dirty = false;  // the light tree is stale (a light-options change)
    uint64_t last_frame = 0;
    cx::DeviceScene dev;
    bool built = false;
    uint64_t generation = 0;  // full builds so far (the device tables move on each)
    cudaEvent_t start = nullptr;
    cudaEvent_t stop = nullptr;
    float flush_ms = 0.0f;
    // Entities 1, 2, ... (entities[id - 1]; `bricks` null: a free id). Each holds its bricks in a
    // scene of its own (no lights); the device keeps one EntityView per live entity, in id order
    // (the index a hit reports), rewritten by the flush after a change and by a removal.
    struct Entity
    {
        CaelixScene* bricks = nullptr;
        uint8_t guid[16] = {};
        float position[3] = {0.0f, 0.0f, 0.0f};
        float rotation[4] = {0.0f, 0.0f, 0.0f, 1.0f};
        float rot[9] = {1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f};
        uint32_t motion = CAELIX_ENTITY_STATIC;
        uint64_t generation = ~0ull;  // the generation of `bricks` the device view was made from
    };
    std::vector<Entity> entities;
    cx::GrowBuffer entity_views;  // device EntityView per live entity
    cx::GrowBuffer entity_nodes;  // device EntityNode: the BVH over the live entities
    bool entity_nodes_used = false;
    uint32_t entity_view_count = 0;
    bool entity_views_dirty = false;
    // The dynamic entities' light set (SceneView::dyn) and tree 0's static set (the world's lights
    // then the static entities'; live only while a static entity has lights), rebuilt with the
    // views; the static set also after every change of the world's lights.
    LightSet dyn;
    LightSet stat;
    bool stat_dirty = false;
    std::vector<uint32_t> view_entity;     // the entity index of every device view
    std::vector<cx::EntityView> host_views;  // the host copy of the device views
    uint64_t entity_generation = 0;  // uploads of the entity views so far (the device views move)
};

struct CaelixRenderer
{
    CaelixDevice* device = nullptr;
    CaelixScene* scene = nullptr;
    CaelixLightNeeOptions nee{1, 0, 0, 0};
    unsigned long long* counts = nullptr;
    cudaEvent_t start = nullptr;
    cudaEvent_t stop = nullptr;
    cudaStream_t last_stream = nullptr;
    uint64_t frame_number = 0;
    bool rendered = false;
    uint32_t trace_mode = 0;        // CAELIX_TRACE_WAVEFRONT or CAELIX_TRACE_MEGAKERNEL
    uint32_t wave_capacity = 0;     // 0 = every pixel of a sample in one wave
    cx::GrowBuffer wave_memory;     // path state and queues of the wavefront trace
    cx::GrowBuffer wave_views;      // the device copy of the view and its wave table
    uint32_t launches = 0;          // kernels of the newest render
};


// The scene as the trace kernels see it: the world's tables and the entities' device views.
cx::SceneView render_view(const CaelixScene* scene);

// The trace parameters of a render call (caelix_renderer_render's checks): INVALID_ARGUMENT for a
// bad target, camera or options, or a scene that was never flushed.
CaelixResult render_params(const CaelixRenderer* renderer, const CaelixRenderTargets* targets,
                           const CaelixCamera* camera, const CaelixRenderOptions* options, const char* what,
                           cx::TraceParams* out);
