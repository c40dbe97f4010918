// The scene and renderer parts of the C ABI (include/caelix_b200.h): device-resident brick
// staging, the flush (staging_gather + scene_build_device) and the render call. Replaces the entry points of the
// reference's lib/src/abi/caelix.cpp for the scene (:296-700) and the renderer (:700-953).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <unordered_map>
#include <new>
#include <vector>

#include "../../include/caelix_b200.h"
#include "abi_internal.h"
#include "abi_scene_internal.h"
#include "materials.h"
#include "scene.cuh"
#include "trace.cuh"

using cx::log;

namespace {

// Brick keys per axis in [-2^20, 2^20) (include/caelix/caelix.h:334).
constexpr int32_t kKeyLimit = 1 << 20;

bool key_ok(const CaelixBrickKey& k)
{
    return k.x >= -kKeyLimit && k.y >= -kKeyLimit && k.z >= -kKeyLimit && k.x < kKeyLimit && k.y < kKeyLimit &&
           k.z < kKeyLimit;
}

// 21 bits per axis (the key moved to [0, 2^21)).
uint64_t pack_key(const CaelixBrickKey& k)
{
    return (uint64_t)(uint32_t)(k.x + kKeyLimit) | ((uint64_t)(uint32_t)(k.y + kKeyLimit) << 21) |
           ((uint64_t)(uint32_t)(k.z + kKeyLimit) << 42);
}

// The scene whose material table, light code set and light options a scene uses: its own, or for
// an entity's bricks the scene that holds the entity.
const CaelixScene* owner_of(const CaelixScene* scene) { return scene->parent ? scene->parent : scene; }

// The smallest and largest key of the staged bricks, per axis (0 without bricks).
void key_bounds(CaelixScene* scene)
{
    const size_t n = scene->slot_power.size();
    for (int a = 0; a < 3; ++a) {
        scene->key_min[a] = n ? scene->keys[a] : 0;
        scene->key_max[a] = n ? scene->keys[a] : 0;
    }
    for (size_t slot = 1; slot < n; ++slot)
        for (int a = 0; a < 3; ++a) {
            scene->key_min[a] = std::min(scene->key_min[a], scene->keys[3 * slot + a]);
            scene->key_max[a] = std::max(scene->key_max[a], scene->keys[3 * slot + a]);
        }
}

// The device form of a scene's material table and its light code set, after a change of either
// (materials or min_emission): uploaded on `stream`; *codes_changed when the light code set is
// not the one the scene's tables were built with.
CaelixResult upload_materials(CaelixScene* scene, cudaStream_t stream, bool* codes_changed)
{
    *codes_changed = false;
    if (!scene->materials_dirty) return CAELIX_OK;
    std::vector<uint32_t> codes;
    cx::light_code_set(scene->materials, scene->encoding, scene->light_options.min_emission, codes);
    *codes_changed = codes != scene->light_codes;
    std::vector<float> table;
    cx::pack_materials(scene->materials, scene->encoding, table);
    CaelixResult r = scene->materials_dev.reserve(4ull * table.size(), "caelix_scene_flush");
    if (r == CAELIX_OK) r = scene->light_codes_dev.reserve(4ull * codes.size(), "caelix_scene_flush");
    if (r != CAELIX_OK) return r;
    cudaError_t e = cudaMemcpyAsync(scene->materials_dev.ptr, table.data(), 4ull * table.size(),
                                    cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scene->light_codes_dev.ptr, codes.data(), 4ull * codes.size(), cudaMemcpyHostToDevice,
                            stream);
    // The host vectors are released on return: the copies finish first.
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
    scene->light_codes = std::move(codes);
    scene->materials_dirty = false;
    return CAELIX_OK;
}

// Object-to-world rotation rows of a quaternion (x, y, z, w), normalised, in double, then rounded.
bool entity_rows(const float q[4], float rot[9])
{
    for (int i = 0; i < 4; ++i)
        if (!std::isfinite(q[i])) return false;
    const double n = std::sqrt((double)q[0] * q[0] + (double)q[1] * q[1] + (double)q[2] * q[2] + (double)q[3] * q[3]);
    if (!(n > 0.0) || !std::isfinite(n)) return false;
    const double x = q[0] / n, y = q[1] / n, z = q[2] / n, w = q[3] / n;
    const double r[9] = {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * w), 2.0 * (x * z + y * w),
                         2.0 * (x * y + z * w), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * w),
                         2.0 * (x * z - y * w), 2.0 * (y * z + x * w), 1.0 - 2.0 * (x * x + y * y)};
    for (int i = 0; i < 9; ++i) rot[i] = (float)r[i];
    return true;
}

// The scene holding the bricks of `entity` (0: the scene itself), or null for an unknown id.
CaelixScene* entity_bricks(CaelixScene* scene, uint32_t entity)
{
    if (entity == 0) return scene;
    if (entity > scene->entities.size()) return nullptr;
    return scene->entities[entity - 1].bricks;
}

uint64_t align256(uint64_t v) { return (v + 255) & ~255ull; }

// Scenes with at least this many entities trace them through the entity BVH.
constexpr size_t kEntityBvhMin = 4;

// A merged light set over `parts` (each a built scene's light tables under a transform: rows
// null for the world part, whose frames are kept), their light blocks, group rows, frames, power
// and light records appended in order (cx::dyn_append moves their indices; leaf words get
// `leaf_flag`), then the light tree built over them. group_base[i] receives part i's first group.
// With no light in any part the set is left not live.
uint32_t entity_bvh_build(std::vector<cx::EntityNode>& nodes, std::vector<uint32_t>& order, size_t first, size_t last,
                          const std::vector<cx::EntityView>& views);

struct LightPart
{
    const cx::DeviceScene* d;
    const float* rot;  // null: identity, no translation
    const float* pos;
};

CaelixResult build_light_set(CaelixScene* scene, LightSet& set, const std::vector<LightPart>& parts,
                             uint32_t leaf_flag, std::vector<uint32_t>& group_base, cudaStream_t stream)
{
    set.live = false;
    group_base.assign(parts.size(), 0);
    uint64_t units = 0, groups = 0, bricks = 0, lights = 0;
    for (size_t i = 0; i < parts.size(); ++i) {
        const cx::DeviceScene& d = *parts[i].d;
        group_base[i] = (uint32_t)groups;
        units += d.heap_words / 4;
        groups += d.group_count;
        bricks += d.brick_count;
        lights += d.light_count;
    }
    if (lights == 0) return CAELIX_OK;
    if (units * 4 >= (1ull << 32) || groups >= (1ull << 32) || bricks >= (1ull << 32) || lights >= (1ull << 31))
        return CAELIX_ERROR_OUT_OF_MEMORY;
    // One allocation, carved: heap, rows, frames, power, records, record groups, record entries.
    const uint64_t o_rows = align256(16 * units), o_frames = o_rows + align256(32 * groups),
                   o_power = o_frames + align256(sizeof(cx::GroupFrame) * groups),
                   o_hdr = o_power + align256(4 * bricks), o_group = o_hdr + align256(sizeof(cx::BrickLightRecord) * lights),
                   o_entry = o_group + align256(4 * lights), total = o_entry + align256(4 * lights);
    CaelixResult r = set.arrays.reserve_grow(total, "caelix_scene_flush");
    if (r != CAELIX_OK) return r;
    uint8_t* base = static_cast<uint8_t*>(set.arrays.ptr);
    uint32_t* heap = reinterpret_cast<uint32_t*>(base);
    uint32_t* rows = reinterpret_cast<uint32_t*>(base + o_rows);
    cx::GroupFrame* frames = reinterpret_cast<cx::GroupFrame*>(base + o_frames);
    float* power = reinterpret_cast<float*>(base + o_power);
    cx::BrickLightRecord* hdr = reinterpret_cast<cx::BrickLightRecord*>(base + o_hdr);
    uint32_t* lgroup = reinterpret_cast<uint32_t*>(base + o_group);
    uint32_t* lentry = reinterpret_cast<uint32_t*>(base + o_entry);
    if (lights > set.tree_capacity) {
        const uint32_t cap = (uint32_t)std::max<uint64_t>(lights + lights / 8, 64);
        r = set.tree.reserve(cx::lt_buffer_bytes(cap), "caelix_scene_flush");
        if (r != CAELIX_OK) return r;
        set.tree_capacity = cap;
    }
    const cx::LightBvhBuffers tree = cx::lt_carve(set.tree.ptr, set.tree_capacity);
    cudaError_t e = cudaSuccess;
    cx::DynPart part{0, 0, 0, 0, {1.0f, 0.0f, 0.0f, 0.0f, 1.0f, 0.0f, 0.0f, 0.0f, 1.0f}, {0.0f, 0.0f, 0.0f}, leaf_flag};
    for (size_t i = 0; i < parts.size() && e == cudaSuccess; ++i) {
        const cx::DeviceScene& d = *parts[i].d;
        part.group_base = group_base[i];
        if (parts[i].rot) {
            std::memcpy(part.rot, parts[i].rot, sizeof(part.rot));
            std::memcpy(part.pos, parts[i].pos, sizeof(part.pos));
        }
        e = cx::dyn_append(d, part, heap, rows, frames, power, hdr, lgroup, lentry, stream);
        part.unit_base += d.heap_words / 4;
        part.record_base += d.brick_count;
        part.light_base += d.light_count;
    }
    cx::LightBvhInput in;
    in.records = hdr;
    in.count = (uint32_t)lights;
    in.record_group = lgroup;
    in.record_entry = lentry;
    in.group_frames = frames;
    in.group_count = (uint32_t)groups;
    in.sort_keys_per_thread = 0;  // the tile for the light count (sort_keys_per_thread_for)
    set.input = in;
    if (e == cudaSuccess) e = cx::lt_build(tree, in, stream, nullptr);
    cx::SceneView& v = set.v;
    std::memset(&v, 0, sizeof(v));
    v.group_shift = scene->group_shift;
    v.enc = cx::encoding_of(scene->encoding);
    v.materials = static_cast<const float4*>(scene->materials_dev.ptr);
    v.light_codes = static_cast<const uint32_t*>(scene->light_codes_dev.ptr);
    v.power = power;
    v.heap = heap;
    v.group_rows = rows;
    v.frames = frames;
    v.leaves = tree.leaves;
    v.nodes = tree.nodes;
    v.header = tree.header;
    v.light_count = (uint32_t)lights;
    v.group_count = (uint32_t)groups;
    if (e == cudaSuccess) {
        r = set.view.reserve_grow(sizeof(v), "caelix_scene_flush");
        if (r != CAELIX_OK) return r;
        e = cudaMemcpyAsync(set.view.ptr, &v, sizeof(v), cudaMemcpyHostToDevice, stream);
    }
    uint32_t status = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&status, &tree.state->status, 4, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
    if (status & ~cx::kStatusNodeOverflow) return cx::status_result(status, "caelix_scene_flush");
    set.live = true;
    return CAELIX_OK;
}

// The dynamic entities' light set (SceneView::dyn) over the live dynamic entities, in view order.
CaelixResult build_dynamic_lights(CaelixScene* scene, cudaStream_t stream)
{
    std::vector<LightPart> parts;
    std::vector<size_t> which;
    for (size_t i = 0; i < scene->host_views.size(); ++i) {
        const CaelixScene::Entity& ent = scene->entities[scene->view_entity[i]];
        if (ent.motion != CAELIX_ENTITY_DYNAMIC) continue;
        parts.push_back({&ent.bricks->dev, ent.rot, ent.position});
        which.push_back(i);
    }
    std::vector<uint32_t> base;
    CaelixResult r = build_light_set(scene, scene->dyn, parts, 0x80000000u, base, stream);
    for (size_t j = 0; j < which.size(); ++j) {
        scene->host_views[which[j]].group_base = base[j];
        scene->host_views[which[j]].tree = scene->dyn.live ? 1u : cx::kNone;
    }
    return r;
}

// Tree 0's static set: the world's light tables first (so every world index stays valid), then
// the live static entities' in view order, with tree 0 built over them. Only while a static
// entity has lights (and the world's tables exist); otherwise tree 0 is the world's own.
CaelixResult build_static_lights(CaelixScene* scene, cudaStream_t stream)
{
    std::vector<LightPart> parts;
    std::vector<size_t> which;
    bool lit = false;
    if (scene->built) {
        parts.push_back({&scene->dev, nullptr, nullptr});
        for (size_t i = 0; i < scene->host_views.size(); ++i) {
            const CaelixScene::Entity& ent = scene->entities[scene->view_entity[i]];
            if (ent.motion != CAELIX_ENTITY_STATIC) continue;
            parts.push_back({&ent.bricks->dev, ent.rot, ent.position});
            which.push_back(i);
            lit = lit || ent.bricks->dev.light_count != 0;
        }
    }
    scene->stat_dirty = false;
    std::vector<uint32_t> base;
    CaelixResult r = CAELIX_OK;
    if (lit) {
        r = build_light_set(scene, scene->stat, parts, 0u, base, stream);
    } else {
        scene->stat.live = false;
        base.assign(parts.size(), 0);
    }
    for (size_t j = 0; j < which.size(); ++j) {
        scene->host_views[which[j]].group_base = base[j + 1];
        scene->host_views[which[j]].tree = scene->stat.live ? 0u : cx::kNone;
    }
    return r;
}

// The device copies of the entity views (host_views) and the entity BVH.
CaelixResult write_entity_views(CaelixScene* scene, cudaStream_t stream)
{
    const std::vector<cx::EntityView>& views = scene->host_views;
    scene->entity_nodes_used = false;
    if (!views.empty()) {
        CaelixResult r = scene->entity_views.reserve(sizeof(cx::EntityView) * views.size(), "caelix_scene_flush");
        if (r != CAELIX_OK) return r;
        cudaError_t e = cudaMemcpyAsync(scene->entity_views.ptr, views.data(), sizeof(cx::EntityView) * views.size(),
                                        cudaMemcpyHostToDevice, stream);
        // With several entities a ray tests only those whose box it meets (trace_entities).
        std::vector<cx::EntityNode> nodes;
        if (e == cudaSuccess && views.size() >= kEntityBvhMin) {
            std::vector<uint32_t> order(views.size());
            for (uint32_t i = 0; i < order.size(); ++i) order[i] = i;
            nodes.reserve(2 * views.size());
            entity_bvh_build(nodes, order, 0, order.size(), views);
            r = scene->entity_nodes.reserve(sizeof(cx::EntityNode) * nodes.size(), "caelix_scene_flush");
            if (r != CAELIX_OK) return r;
            e = cudaMemcpyAsync(scene->entity_nodes.ptr, nodes.data(), sizeof(cx::EntityNode) * nodes.size(),
                                cudaMemcpyHostToDevice, stream);
            scene->entity_nodes_used = true;
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
    }
    scene->entity_view_count = (uint32_t)views.size();
    scene->entity_generation += 1;
    return CAELIX_OK;
}

// The BVH over the entities' bounding spheres (world space, boxes rounded outwards): binary, one
// entity per leaf, split at the median of the longest axis of the centres. Node 0 is the root.
uint32_t entity_bvh_build(std::vector<cx::EntityNode>& nodes, std::vector<uint32_t>& order, size_t first, size_t last,
                          const std::vector<cx::EntityView>& views)
{
    const uint32_t index = (uint32_t)nodes.size();
    nodes.emplace_back();
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    double clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (size_t i = first; i < last; ++i) {
        const float* sp = views[order[i]].sphere;
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], std::nextafter(sp[k] - sp[3], -INFINITY));
            hi[k] = std::max(hi[k], std::nextafter(sp[k] + sp[3], INFINITY));
            clo[k] = std::min(clo[k], (double)sp[k]);
            chi[k] = std::max(chi[k], (double)sp[k]);
        }
    }
    cx::EntityNode n;
    for (int k = 0; k < 3; ++k) {
        n.lo[k] = lo[k];
        n.hi[k] = hi[k];
    }
    if (last - first == 1) {
        n.first = cx::kEntityLeaf | order[first];
        n.second = 0;
    } else {
        int axis = 0;
        for (int k = 1; k < 3; ++k)
            if (chi[k] - clo[k] > chi[axis] - clo[axis]) axis = k;
        const size_t mid = first + (last - first) / 2;
        std::nth_element(order.begin() + first, order.begin() + mid, order.begin() + last, [&](uint32_t a, uint32_t b) {
            return views[a].sphere[axis] < views[b].sphere[axis] ||
                   (views[a].sphere[axis] == views[b].sphere[axis] && a < b);
        });
        n.first = entity_bvh_build(nodes, order, first, mid, views);
        n.second = entity_bvh_build(nodes, order, mid, last, views);
    }
    nodes[index] = n;
    return index;
}

// Rewrites the device views of the live entities and their light sets (after waiting for the
// device: renders may read the old ones) and returns when they are in place. An entity whose
// bricks were never flushed has no tables yet and joins at the flush that builds them.
CaelixResult upload_entity_views(CaelixScene* scene, cudaStream_t stream)
{
    std::vector<cx::EntityView>& views = scene->host_views;
    views.clear();
    scene->view_entity.clear();
    for (size_t id = 0; id < scene->entities.size(); ++id) {
        CaelixScene::Entity& e = scene->entities[id];
        if (!e.bricks || !e.bricks->built) continue;
        cx::EntityView v;
        std::memset(&v, 0, sizeof(v));
        v.scene = cx::scene_view(e.bricks->dev);
        std::memcpy(v.rot, e.rot, sizeof(v.rot));
        std::memcpy(v.pos, e.position, sizeof(v.pos));
        v.group_base = 0;
        v.id = (uint32_t)id + 1;
        v.tree = cx::kNone;
        // The sphere round the entity's brick grid [8 origin, 8 (origin + grid)) in world space
        // (double, inflated).
        {
            const cx::DeviceScene& d = e.bricks->dev;
            double c[3], r2 = 0.0, mid[3];
            for (int a = 0; a < 3; ++a) {
                const double h = 4.0 * d.grid[a];
                r2 += h * h;
                mid[a] = 8.0 * d.origin[a] + h;
            }
            for (int i = 0; i < 3; ++i) {
                c[i] = e.position[i];
                for (int j = 0; j < 3; ++j) c[i] += (double)e.rot[3 * i + j] * mid[j];
                v.sphere[i] = (float)c[i];
            }
            v.sphere[3] = (float)(std::sqrt(r2) * 1.001 + 0.01);
        }
        views.push_back(v);
        scene->view_entity.push_back((uint32_t)id);
        e.generation = e.bricks->generation;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
    scene->entity_view_count = 0;
    CaelixResult r = build_dynamic_lights(scene, stream);
    if (r == CAELIX_OK) r = build_static_lights(scene, stream);
    if (r != CAELIX_OK) return r;
    r = write_entity_views(scene, stream);
    if (r != CAELIX_OK) return r;
    scene->entity_views_dirty = false;
    return CAELIX_OK;
}

// After a change of the world's light tables: tree 0's static set again (with the static
// entities' views, whose group bases follow the world's group count), when static entities exist.
CaelixResult refresh_static_lights(CaelixScene* scene, cudaStream_t stream)
{
    if (!scene->stat_dirty) return CAELIX_OK;
    scene->stat_dirty = false;
    bool any = false;
    for (uint32_t id : scene->view_entity) any = any || scene->entities[id].motion == CAELIX_ENTITY_STATIC;
    if (!any) return CAELIX_OK;
    cudaError_t e = cudaDeviceSynchronize();  // renders may read the old set
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
    CaelixResult r = build_static_lights(scene, stream);
    if (r == CAELIX_OK) r = write_entity_views(scene, stream);
    return r;
}

}  // namespace

cx::SceneView render_view(const CaelixScene* scene)
{
    cx::SceneView v = cx::scene_view(scene->dev);
    if (scene->entity_view_count) {
        v.entities = static_cast<const cx::EntityView*>(scene->entity_views.ptr);
        v.entity_count = scene->entity_view_count;
        if (scene->entity_nodes_used) v.entity_nodes = static_cast<const cx::EntityNode*>(scene->entity_nodes.ptr);
        if (scene->dyn.live) v.dyn = static_cast<const cx::SceneView*>(scene->dyn.view.ptr);
        if (scene->stat.live) {
            // Tree 0 and its light set: the static set, the world's tables at their own indices.
            const cx::SceneView& t = scene->stat.v;
            v.power = t.power;
            v.heap = t.heap;
            v.group_rows = t.group_rows;
            v.frames = t.frames;
            v.leaves = t.leaves;
            v.nodes = t.nodes;
            v.header = t.header;
            v.light_count = t.light_count;
            v.group_count = t.group_count;
        }
    }
    return v;
}

CaelixResult render_params(const CaelixRenderer* renderer, const CaelixRenderTargets* targets,
                           const CaelixCamera* camera, const CaelixRenderOptions* options, const char* what,
                           cx::TraceParams* out)
{
    if (!renderer || !targets || !camera || !options || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    if (!targets->radiance || targets->width == 0 || targets->height == 0 || options->mode != 1 ||
        options->bounce_count > 14 || camera->jitter[0] != 0.0f || camera->jitter[1] != 0.0f ||
        !std::isfinite(options->voxel_id_tmax) || options->voxel_id_tmax < 0.0f)
        return CAELIX_ERROR_INVALID_ARGUMENT;
    for (uint32_t r : options->reserved)
        if (r) return CAELIX_ERROR_INVALID_ARGUMENT;
    const CaelixScene* scene = renderer->scene;
    if (!scene->built) {
        log(CAELIX_LOG_ERROR, "%s: the scene has not been flushed", what);
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    cx::TraceParams& p = *out;
    for (int k = 0; k < 3; ++k) {
        p.position[k] = camera->position[k];
        p.right[k] = camera->right[k];
        p.up[k] = camera->up[k];
        p.forward[k] = camera->forward[k];
    }
    p.tan_half_fov_y = camera->tan_half_fov_y;
    p.aspect = camera->aspect;
    p.width = targets->width;
    p.height = targets->height;
    p.spp = options->spp ? options->spp : 1;
    p.bounce_count = options->bounce_count;
    p.frame_seed = options->frame_seed;
    p.light_nee = (renderer->nee.enabled && scene->light_options.enabled && scene->dev.light_count) ? 1u : 0u;
    p.voxel_id = reinterpret_cast<uint32_t*>(targets->voxel_id);
    p.voxel_id_tmax = options->voxel_id_tmax;
    return CAELIX_OK;
}

extern "C" {

CAELIX_API CaelixResult caelix_scene_create(CaelixDevice* device, const CaelixSceneDesc* desc, CaelixScene** out_scene)
{
    CAELIX_GUARD_BEGIN
    if (!device || !out_scene) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out_scene = nullptr;
    uint32_t shift = 4, encoding = cx::kEncodingPacked;
    if (desc) {
        // The reference's checks (include/caelix/caelix.h:274-294), then what this version implements.
        if ((desc->staging_bytes != 0 && desc->staging_bytes < (4ull << 20)) ||
            (desc->records_per_page & (desc->records_per_page - 1u)) != 0 || desc->group_shift > 8 ||
            (desc->block_bytes != 0 && desc->block_bytes != 2 && desc->block_bytes != 4) || desc->encoding > 1) {
            log(CAELIX_LOG_ERROR, "caelix_scene_create: invalid scene description");
            return CAELIX_ERROR_INVALID_ARGUMENT;
        }
        shift = desc->group_shift ? desc->group_shift : 4;
        if (shift > 4 || desc->block_bytes == 4) {
            log(CAELIX_LOG_ERROR, "caelix_scene_create: group_shift %u above 4 or 4-byte blocks are not implemented",
                shift);
            return CAELIX_ERROR_UNSUPPORTED;
        }
        encoding = desc->encoding;
    }
    cudaSetDevice(device->ordinal);
    CaelixScene* s = new CaelixScene();
    s->device = device;
    s->group_shift = shift;
    s->encoding = encoding;
    s->materials.resize(cx::kMaterialCodes);
    for (uint32_t c = 0; c < cx::kMaterialCodes; ++c) s->materials[c] = cx::builtin_material(c, encoding);
    cudaError_t e = cudaEventCreate(&s->start);
    if (e == cudaSuccess) e = cudaEventCreate(&s->stop);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->upload_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        caelix_scene_destroy(s);
        return cx::cuda_result(e, "caelix_scene_create");
    }
    *out_scene = s;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API void caelix_scene_destroy(CaelixScene* scene)
{
    if (!scene) return;
    cudaSetDevice(scene->device->ordinal);
    for (auto& e : scene->entities) caelix_scene_destroy(e.bricks);
    scene->entities.clear();
    scene->entity_views.release();
    scene->entity_nodes.release();
    scene->dyn.release();
    scene->stat.release();
    scene->materials_dev.release();
    scene->light_codes_dev.release();
    cx::scene_release(scene->dev);
    if (scene->upload_stream) cudaStreamSynchronize(scene->upload_stream);
    if (scene->stage_keys) cudaFree(scene->stage_keys);
    if (scene->stage_voxels) cudaFree(scene->stage_voxels);
    scene->upload.release();
    scene->flush_scratch.release();
    scene->record_of_slot.release();
    scene->marks.release();
    scene->update.release();
    if (scene->edit_host) cudaFreeHost(scene->edit_host);
    if (scene->upload_stream) cudaStreamDestroy(scene->upload_stream);
    if (scene->start) cudaEventDestroy(scene->start);
    if (scene->stop) cudaEventDestroy(scene->stop);
    delete scene;
}

CAELIX_API CaelixResult caelix_scene_upload_bricks(CaelixScene* scene, uint32_t entity, uint32_t count,
                                                   const CaelixBrickKey* keys, const void* blocks, uint32_t* consumed)
{
    CAELIX_GUARD_BEGIN
    if (consumed) *consumed = 0;
    if (!scene || (count && (!keys || !blocks))) return CAELIX_ERROR_INVALID_ARGUMENT;
    if (entity != 0) {
        CaelixScene* bricks = entity_bricks(scene, entity);
        return bricks ? caelix_scene_upload_bricks(bricks, 0, count, keys, blocks, consumed)
                      : CAELIX_ERROR_INVALID_ARGUMENT;
    }
    for (uint32_t i = 0; i < count; ++i) {
        if (!key_ok(keys[i])) {
            log(CAELIX_LOG_ERROR, "caelix_scene_upload_bricks: key (%d, %d, %d) outside [-%d, %d)", keys[i].x,
                keys[i].y, keys[i].z, kKeyLimit, kKeyLimit);
            return CAELIX_ERROR_INVALID_ARGUMENT;
        }
    }
    if (count == 0) return CAELIX_OK;
    cudaSetDevice(scene->device->ordinal);
    cudaStream_t st = scene->upload_stream;
    // Slots: new keys take the next slots (with any power set before their upload). A failure
    // below gives the new slots back, so the scene stays as it was before the call.
    const uint32_t old_slots = (uint32_t)scene->slot_power.size();
    const int32_t old_max[3] = {scene->key_max[0], scene->key_max[1], scene->key_max[2]};
    const int32_t old_min[3] = {scene->key_min[0], scene->key_min[1], scene->key_min[2]};
    std::vector<std::pair<uint64_t, float>> taken_power;
    std::vector<uint32_t> slot(count);
    for (uint32_t i = 0; i < count; ++i) {
        const uint64_t packed = pack_key(keys[i]);
        const auto ins = scene->slot_of.emplace(packed, (uint32_t)scene->slot_power.size());
        slot[i] = ins.first->second;
        if (ins.second) {
            const int32_t k3[3] = {keys[i].x, keys[i].y, keys[i].z};
            const bool first = scene->slot_power.empty();
            scene->keys.insert(scene->keys.end(), {k3[0], k3[1], k3[2]});
            for (int a = 0; a < 3; ++a) {
                scene->key_max[a] = first ? k3[a] : std::max(scene->key_max[a], k3[a]);
                scene->key_min[a] = first ? k3[a] : std::min(scene->key_min[a], k3[a]);
            }
            const auto p = scene->pending_power.find(packed);
            scene->slot_power.push_back(p != scene->pending_power.end() ? p->second : 1.0f);
            if (p != scene->pending_power.end()) {
                taken_power.emplace_back(p->first, p->second);
                scene->pending_power.erase(p);
            }
        }
    }
    const uint32_t slots = (uint32_t)scene->slot_power.size();
    auto give_back = [&](CaelixResult r) {
        for (uint32_t s = old_slots; s < slots; ++s) {
            const CaelixBrickKey k{scene->keys[3ull * s], scene->keys[3ull * s + 1], scene->keys[3ull * s + 2]};
            scene->slot_of.erase(pack_key(k));
        }
        scene->keys.resize(3ull * old_slots);
        scene->slot_power.resize(old_slots);
        for (int a = 0; a < 3; ++a) {
            scene->key_max[a] = old_max[a];
            scene->key_min[a] = old_min[a];
        }
        for (const auto& kv : taken_power) scene->pending_power.insert(kv);
        return r;
    };
    // Staging growth (doubling), the resident slots carried over.
    if (slots > scene->stage_capacity) {
        const uint32_t cap = std::max<uint32_t>(slots, std::max<uint32_t>(2 * scene->stage_capacity, 1024));
        int32_t* nk = nullptr;
        uint16_t* nv = nullptr;
        cudaError_t e = cudaMalloc(&nk, 12ull * cap);
        if (e == cudaSuccess) e = cudaMalloc(&nv, 1024ull * cap);
        if (e == cudaSuccess && old_slots) {
            e = cudaMemcpyAsync(nk, scene->stage_keys, 12ull * old_slots, cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(nv, scene->stage_voxels, 1024ull * old_slots, cudaMemcpyDeviceToDevice, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        }
        if (e != cudaSuccess) {
            if (nk) cudaFree(nk);
            if (nv) cudaFree(nv);
            return give_back(cx::cuda_result(e, "caelix_scene_upload_bricks"));
        }
        if (scene->stage_keys) cudaFree(scene->stage_keys);
        if (scene->stage_voxels) cudaFree(scene->stage_voxels);
        scene->stage_keys = nk;
        scene->stage_voxels = nv;
        scene->stage_capacity = cap;
    }
    // One copy per slot: the last upload of a key in this call wins.
    scene->upload_mark.resize(slots, 0);
    if (++scene->upload_epoch == 0) {
        std::fill(scene->upload_mark.begin(), scene->upload_mark.end(), 0u);
        scene->upload_epoch = 1;
    }
    std::vector<uint32_t> lists;  // [src index][slot], `unique` entries each
    lists.reserve(2ull * count);
    std::vector<uint32_t> dst;
    dst.reserve(count);
    for (uint32_t i = count; i-- > 0;) {
        if (scene->upload_mark[slot[i]] == scene->upload_epoch) continue;
        scene->upload_mark[slot[i]] = scene->upload_epoch;
        lists.push_back(i);
        dst.push_back(slot[i]);
    }
    const uint32_t unique = (uint32_t)dst.size();
    lists.insert(lists.end(), dst.begin(), dst.end());
    CaelixResult r = scene->upload.reserve(1024ull * count + 4ull * lists.size(), "caelix_scene_upload_bricks");
    if (r != CAELIX_OK) return give_back(r);
    uint16_t* d_blocks = static_cast<uint16_t*>(scene->upload.ptr);
    uint32_t* d_lists = reinterpret_cast<uint32_t*>(d_blocks + 512ull * count);
    cudaError_t e = cudaMemcpyAsync(d_blocks, blocks, 1024ull * count, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_lists, lists.data(), 4ull * lists.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && slots > old_slots)
        e = cudaMemcpyAsync(scene->stage_keys + 3ull * old_slots, scene->keys.data() + 3ull * old_slots,
                            12ull * (slots - old_slots), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cx::staging_scatter(d_blocks, d_lists, d_lists + unique, unique, scene->stage_voxels, st);
    // The caller may reuse its buffers on return, and the next flush reads the staging.
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return give_back(cx::cuda_result(e, "caelix_scene_upload_bricks"));
    // The call's slots are edits of the next flush (a new key: a full rebuild).
    if (slots > old_slots) scene->full_rebuild = true;
    scene->slot_dirty.resize(slots, 0);
    for (uint32_t s : dst) {
        if (!scene->slot_dirty[s]) {
            scene->slot_dirty[s] = 1;
            scene->dirty_slots.push_back(s);
        }
    }
    if (consumed) *consumed = count;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_scene_remove_bricks(CaelixScene* scene, uint32_t entity, uint32_t count,
                                                   const CaelixBrickKey* keys)
{
    CAELIX_GUARD_BEGIN
    if (!scene || (count && !keys)) return CAELIX_ERROR_INVALID_ARGUMENT;
    if (entity != 0) {
        CaelixScene* bricks = entity_bricks(scene, entity);
        return bricks ? caelix_scene_remove_bricks(bricks, 0, count, keys) : CAELIX_ERROR_INVALID_ARGUMENT;
    }
    if (count == 0) return CAELIX_OK;
    // Room for the compaction's moves (one per removed key), taken before any state changes.
    CaelixResult r = scene->upload.reserve(8ull * count, "caelix_scene_remove_bricks");
    if (r != CAELIX_OK) return r;
    // The slots stay dense: the last slot moves into the removed one. A dry run over the original
    // slots first: `source` maps a slot that takes another brick to the slot that brick had
    // before this call, `moved` a key to its slot after such a move, `gone` the removed keys. The
    // host state changes only after the moves have been checked.
    const uint32_t old_slots = (uint32_t)scene->slot_power.size();
    uint32_t n = old_slots;
    std::unordered_map<uint32_t, uint32_t> source;
    std::unordered_map<uint64_t, uint32_t> moved;
    std::unordered_map<uint64_t, uint32_t> gone;
    auto original = [&](uint32_t slot) {
        const auto m = source.find(slot);
        return m != source.end() ? m->second : slot;
    };
    auto key_of = [&](uint32_t slot) {
        const uint32_t o = original(slot);
        return pack_key(CaelixBrickKey{scene->keys[3ull * o], scene->keys[3ull * o + 1], scene->keys[3ull * o + 2]});
    };
    for (uint32_t i = 0; i < count; ++i) {
        if (!key_ok(keys[i])) continue;
        const uint64_t k = pack_key(keys[i]);
        if (gone.count(k)) continue;
        uint32_t slot;
        if (const auto m = moved.find(k); m != moved.end()) {
            slot = m->second;
            moved.erase(m);
        } else if (const auto it = scene->slot_of.find(k); it != scene->slot_of.end()) {
            slot = it->second;
        } else {
            continue;
        }
        gone.emplace(k, slot);
        const uint32_t last = n - 1;
        if (slot != last) {
            moved[key_of(last)] = slot;
            source[slot] = original(last);
        }
        source.erase(last);
        n = last;
    }
    if (n == old_slots) return CAELIX_OK;
    // Every destination is a remaining slot and every source a slot past the end, so the moves
    // (on the host arrays and on the device) never overlap.
    std::vector<uint32_t> moves;
    moves.reserve(2 * source.size());
    for (const auto& kv : source) {
        if (kv.first >= n || kv.second < n || kv.second >= old_slots) {
            log(CAELIX_LOG_ERROR, "caelix_scene_remove_bricks: bad staging move %u <- %u (nothing removed)", kv.first,
                kv.second);
            return CAELIX_ERROR_INVALID_ARGUMENT;
        }
        moves.push_back(kv.first);
        moves.push_back(kv.second);
    }
    for (const auto& kv : gone) scene->slot_of.erase(kv.first);
    for (const auto& kv : moved) scene->slot_of[kv.first] = kv.second;
    for (const auto& kv : source) {
        for (int a = 0; a < 3; ++a) scene->keys[3ull * kv.first + a] = scene->keys[3ull * kv.second + a];
        scene->slot_power[kv.first] = scene->slot_power[kv.second];
    }
    scene->keys.resize(3ull * n);
    scene->slot_power.resize(n);
    scene->slot_dirty.assign(n, 0);
    scene->dirty_slots.clear();
    scene->upload_mark.resize(n, 0);
    key_bounds(scene);
    // The key set changed: the next flush rebuilds the tables from the remaining slots.
    scene->full_rebuild = true;
    if (moves.empty()) return CAELIX_OK;
    cudaSetDevice(scene->device->ordinal);
    cudaStream_t st = scene->upload_stream;
    uint32_t* d_moves = static_cast<uint32_t*>(scene->upload.ptr);
    cudaError_t e = cudaMemcpyAsync(d_moves, moves.data(), 4ull * moves.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cx::staging_move(scene->stage_keys, scene->stage_voxels, d_moves, (uint32_t)(moves.size() / 2), st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? CAELIX_OK : cx::cuda_result(e, "caelix_scene_remove_bricks");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_scene_add_entity(CaelixScene* scene, const CaelixEntityDesc* desc, CaelixEntityId* out_id)
{
    CAELIX_GUARD_BEGIN
    if (out_id) *out_id = CAELIX_INVALID_ENTITY;
    if (!scene || !desc || !out_id) return CAELIX_ERROR_INVALID_ARGUMENT;
    float rot[9];
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(desc->position[k])) return CAELIX_ERROR_INVALID_ARGUMENT;
    if (!entity_rows(desc->rotation, rot)) return CAELIX_ERROR_INVALID_ARGUMENT;
    CaelixSceneDesc sd{0, 0, scene->group_shift, 0, scene->encoding, 0};
    CaelixScene* bricks = nullptr;
    CaelixResult r = caelix_scene_create(scene->device, &sd, &bricks);
    if (r != CAELIX_OK) return r;
    bricks->parent = scene;
    bricks->materials.clear();  // the scene's table is used
    bricks->materials_dirty = false;
    bricks->last_frame = scene->last_frame;
    uint32_t slot = 0;
    while (slot < scene->entities.size() && scene->entities[slot].bricks) ++slot;
    if (slot == scene->entities.size()) scene->entities.emplace_back();
    CaelixScene::Entity& e = scene->entities[slot];
    e = CaelixScene::Entity();
    e.bricks = bricks;
    std::memcpy(e.guid, desc->guid, sizeof(e.guid));
    std::memcpy(e.position, desc->position, sizeof(e.position));
    std::memcpy(e.rotation, desc->rotation, sizeof(e.rotation));
    std::memcpy(e.rot, rot, sizeof(rot));
    scene->entity_views_dirty = true;
    *out_id = slot + 1;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_scene_remove_entity(CaelixScene* scene, CaelixEntityId entity)
{
    CAELIX_GUARD_BEGIN
    if (!scene || entity == 0 || !entity_bricks(scene, entity)) return CAELIX_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(scene->device->ordinal);
    // Renders that read its bricks finish first; the device views drop it before its tables go.
    CaelixScene* bricks = scene->entities[entity - 1].bricks;
    scene->entities[entity - 1] = CaelixScene::Entity();
    CaelixResult r = upload_entity_views(scene, scene->upload_stream);
    caelix_scene_destroy(bricks);
    return r;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_scene_set_entity_transform(CaelixScene* scene, CaelixEntityId entity,
                                                          const float position[3], const float rotation[4])
{
    CAELIX_GUARD_BEGIN
    if (!scene || entity == 0 || !entity_bricks(scene, entity) || !position || !rotation)
        return CAELIX_ERROR_INVALID_ARGUMENT;
    float rot[9];
    for (int k = 0; k < 3; ++k)
        if (!std::isfinite(position[k])) return CAELIX_ERROR_INVALID_ARGUMENT;
    if (!entity_rows(rotation, rot)) return CAELIX_ERROR_INVALID_ARGUMENT;
    CaelixScene::Entity& e = scene->entities[entity - 1];
    std::memcpy(e.position, position, sizeof(e.position));
    std::memcpy(e.rotation, rotation, sizeof(e.rotation));
    std::memcpy(e.rot, rot, sizeof(rot));
    scene->entity_views_dirty = true;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_scene_set_entity_motion(CaelixScene* scene, CaelixEntityId entity, uint32_t motion)
{
    if (!scene || entity == 0 || !entity_bricks(scene, entity) ||
        (motion != CAELIX_ENTITY_STATIC && motion != CAELIX_ENTITY_DYNAMIC))
        return CAELIX_ERROR_INVALID_ARGUMENT;
    CaelixScene::Entity& e = scene->entities[entity - 1];
    if (e.motion != motion) scene->entity_views_dirty = true;  // its lights change trees at the next flush
    e.motion = motion;
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_scene_set_brick_power(CaelixScene* scene, uint32_t entity, uint32_t count,
                                                     const CaelixBrickKey* keys, const float* power)
{
    CAELIX_GUARD_BEGIN
    if (!scene || (count && (!keys || !power))) return CAELIX_ERROR_INVALID_ARGUMENT;
    if (entity != 0) {
        CaelixScene* bricks = entity_bricks(scene, entity);
        return bricks ? caelix_scene_set_brick_power(bricks, 0, count, keys, power) : CAELIX_ERROR_INVALID_ARGUMENT;
    }
    for (uint32_t i = 0; i < count; ++i)
        if (!key_ok(keys[i]) || !std::isfinite(power[i]) || power[i] < 0.0f) return CAELIX_ERROR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < count; ++i) {
        const uint64_t packed = pack_key(keys[i]);
        const auto it = scene->slot_of.find(packed);
        if (it != scene->slot_of.end()) {
            const uint32_t slot = it->second;
            scene->slot_power[slot] = power[i];
            scene->slot_dirty.resize(scene->slot_power.size(), 0);
            if (!scene->slot_dirty[slot]) {
                scene->slot_dirty[slot] = 1;
                scene->dirty_slots.push_back(slot);
            }
        } else {
            scene->pending_power[packed] = power[i];
        }
    }
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_scene_set_materials(CaelixScene* scene, const CaelixMaterial* entries, uint32_t count)
{
    CAELIX_GUARD_BEGIN
    if (!scene || scene->parent || (count && !entries) || count > cx::kMaterialCodes)
        return CAELIX_ERROR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < count; ++i) {
        const char* reason = nullptr;
        if (!cx::material_valid(entries[i], &reason)) {
            log(CAELIX_LOG_ERROR, "caelix_scene_set_materials: entry %u: %s", i, reason);
            return CAELIX_ERROR_INVALID_ARGUMENT;
        }
    }
    for (uint32_t c = 0; c < cx::kMaterialCodes; ++c) {
        scene->materials[c] = c < count ? entries[c] : cx::builtin_material(c, scene->encoding);
        scene->materials[c].reserved = 0;
    }
    scene->materials_dirty = true;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_scene_set_material_entries(CaelixScene* scene, const CaelixMaterialEntry* entries,
                                                          uint32_t count)
{
    CAELIX_GUARD_BEGIN
    if (!scene || scene->parent || (count && !entries)) return CAELIX_ERROR_INVALID_ARGUMENT;
    for (uint32_t i = 0; i < count; ++i) {
        const char* reason = "code above 0xFFFF";
        if (entries[i].code > 0xFFFFu || !cx::material_valid(entries[i].material, &reason)) {
            log(CAELIX_LOG_ERROR, "caelix_scene_set_material_entries: entry %u: %s", i, reason);
            return CAELIX_ERROR_INVALID_ARGUMENT;
        }
    }
    for (uint32_t i = 0; i < count; ++i) {
        scene->materials[entries[i].code] = entries[i].material;
        scene->materials[entries[i].code].reserved = 0;
    }
    if (count) scene->materials_dirty = true;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_scene_get_material(const CaelixScene* scene, uint32_t code, CaelixMaterial* out)
{
    if (!scene || !out || code > 0xFFFFu) return CAELIX_ERROR_INVALID_ARGUMENT;
    const CaelixScene* o = owner_of(scene);
    *out = o->materials[cx::canonical_code(code, o->encoding)];
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_scene_set_light_options(CaelixScene* scene, const CaelixLightOptions* options)
{
    if (!scene || scene->parent || !options || options->enabled > 1 || !std::isfinite(options->min_emission) ||
        options->min_emission < 0.0f || options->heap_bytes > (16ull << 32))
        return CAELIX_ERROR_INVALID_ARGUMENT;
    CaelixLightOptions o = *options;
    if (o.min_emission == 0.0f) o.min_emission = 20.0f;
    // Toggling the tree rebuilds the tables (the light records come and go); a new min_emission
    // may change the light code set (checked at the flush, which then rebuilds the tables); any
    // other change takes effect as a light-tree rebuild at the next flush, as in the reference.
    if (o.enabled != scene->light_options.enabled || !scene->built) scene->full_rebuild = true;
    else scene->light_tree_dirty = true;
    if (o.min_emission != scene->light_options.min_emission) scene->materials_dirty = true;
    scene->light_options = o;
    return CAELIX_OK;
}

static CaelixResult scene_flush_body(CaelixScene* scene, const CaelixFrameDesc* desc)
{
    if (!scene || !desc) return CAELIX_ERROR_INVALID_ARGUMENT;
    if (desc->frame_number <= scene->last_frame || desc->safe_frame_number >= desc->frame_number) {
        log(CAELIX_LOG_ERROR, "caelix_scene_flush: frame %llu after %llu (safe %llu) breaks the frame contract",
            (unsigned long long)desc->frame_number, (unsigned long long)scene->last_frame,
            (unsigned long long)desc->safe_frame_number);
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    scene->last_frame = desc->frame_number;
    cudaSetDevice(scene->device->ordinal);
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(desc->command_buffer);
    const CaelixScene* owner = owner_of(scene);
    const bool lit = owner->light_options.enabled != 0;
    // The material table and the light code set first (an entity's bricks use its scene's). The
    // trace reads the table at draw time; a change of the light code set rebuilds the tables, as the
    // reference finalizes every resident brick again (include/caelix/caelix.h:625-629).
    if (!scene->parent) {
        bool codes_changed = false;
        CaelixResult r = upload_materials(scene, stream, &codes_changed);
        if (r != CAELIX_OK) return r;
        if (codes_changed) {
            scene->full_rebuild = true;
            for (auto& ent : scene->entities)
                if (ent.bricks) ent.bricks->full_rebuild = true;
        }
    }
    if (scene->built && scene->dev.lights != lit) scene->full_rebuild = true;
    scene->dev.encoding = scene->encoding;
    scene->dev.materials = static_cast<const float4*>(owner->materials_dev.ptr);
    scene->dev.light_codes = static_cast<const uint32_t*>(owner->light_codes_dev.ptr);
    scene->dev.lights = lit;
    // The entities' bricks (their own flushes), then their device views when any moved, changed,
    // came or went.
    for (auto& ent : scene->entities) {
        if (!ent.bricks) continue;
        CaelixResult r = caelix_scene_flush(ent.bricks, desc);
        if (r != CAELIX_OK) return r;
        if (ent.bricks->generation != ent.generation) scene->entity_views_dirty = true;
    }
    if (scene->entity_views_dirty) {
        CaelixResult r = upload_entity_views(scene, stream);
        if (r != CAELIX_OK) return r;
    }
    if (!scene->built) scene->full_rebuild = true;
    const bool edits = !scene->dirty_slots.empty();
    if (!scene->full_rebuild && !edits && !scene->light_tree_dirty) return CAELIX_OK;
    scene->stat_dirty = true;  // the world's light tables change
    uint32_t status = 0;
    cudaError_t e = cudaSuccess;
    if (!scene->full_rebuild) {
        // The brick set is unchanged: the tables stay; the edited bricks are copied into the
        // scene and their records and their neighbours' finalized again, then the light records
        // and the light tree are rebuilt. A light-options change alone rebuilds the light tree.
        if (edits) {
            // Rewritten in place: renders of the scene, on any stream, finish first.
            e = cudaDeviceSynchronize();
            if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
        }
        cudaEventRecord(scene->start, stream);
        if (edits) {
            const uint32_t c = (uint32_t)scene->dirty_slots.size();
            // The slots and their power go up from pinned memory (a copy from pageable memory
            // waits for the stream first); the previous flush has finished with the buffer.
            if (scene->edit_host_words < 2ull * c) {
                if (scene->edit_host) cudaFreeHost(scene->edit_host);
                scene->edit_host = nullptr;
                scene->edit_host_words = 0;
                const uint64_t words = 2ull * c + c / 4;
                e = cudaHostAlloc(reinterpret_cast<void**>(&scene->edit_host), 4ull * words, cudaHostAllocDefault);
                if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
                scene->edit_host_words = words;
            }
            uint32_t* host = scene->edit_host;
            for (uint32_t i = 0; i < c; ++i) {
                const uint32_t slot = scene->dirty_slots[i];
                const float p = scene->slot_power[slot];
                host[i] = slot;
                std::memcpy(&host[c + i], &p, 4);
            }
            CaelixResult r = scene->update.reserve(4ull * (9ull * c + 1), "caelix_scene_flush");
            if (r != CAELIX_OK) return r;
            uint32_t* d_slots = static_cast<uint32_t*>(scene->update.ptr);
            const float* d_power = reinterpret_cast<const float*>(d_slots + c);
            uint32_t* d_list = d_slots + 2ull * c;
            uint32_t* d_count = d_list + 7ull * c;
            if (++scene->mark_epoch == 0) {
                e = cudaMemsetAsync(scene->marks.ptr, 0, 4ull * scene->dev.brick_count, stream);
                scene->mark_epoch = 1;
            }
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(d_slots, host, 8ull * c, cudaMemcpyHostToDevice, stream);
            if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, 4, stream);
            // The build's status words and counters start from zero, as in a full build.
            if (e == cudaSuccess) e = cudaMemsetAsync(scene->dev.status, 0, 64, stream);
            if (e == cudaSuccess)
                e = cx::staging_update(scene->stage_voxels, d_slots, d_power, c,
                                       static_cast<const uint32_t*>(scene->record_of_slot.ptr), scene->dev,
                                       static_cast<uint32_t*>(scene->marks.ptr), scene->mark_epoch, d_list, d_count,
                                       stream);
            if (e == cudaSuccess) e = cx::scene_refinalize(scene->dev, d_list, d_count, 7 * c, stream);
            // The refinalized record count, read back with the build's own reads (which wait for
            // the stream).
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(scene->dev.pinned + 4, d_count, 4, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess)
                e = cx::scene_build_lights(scene->dev, stream, &status, static_cast<const uint32_t*>(scene->marks.ptr),
                                           scene->mark_epoch);
            if (e == cudaSuccess) scene->last_update_records = scene->dev.pinned[4];
        } else if (scene->light_tree_dirty) {
            e = cx::scene_build_light_tree(scene->dev, stream);
            if (e == cudaSuccess) e = cx::scene_read_status(scene->dev, stream, &status);
        }
        cudaEventRecord(scene->stop, stream);
        if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
        cudaEventSynchronize(scene->stop);
        cudaEventElapsedTime(&scene->flush_ms, scene->start, scene->stop);
        for (uint32_t slot : scene->dirty_slots) scene->slot_dirty[slot] = 0;
        scene->dirty_slots.clear();
        scene->light_tree_dirty = false;
        if (edits) scene->generation += 1;
        return cx::status_result(status & ~cx::kStatusNodeOverflow, "caelix_scene_flush");
    }
    // A full rebuild: the staged bricks in increasing linear brick index of the box spanned by the
    // keys (rounded to whole groups), sorted and gathered on the device, then the build.
    const uint32_t n = (uint32_t)scene->slot_power.size();
    int32_t origin[3];
    uint32_t grid[3];
    if (!cx::scene_grid(scene->key_min, scene->key_max, scene->group_shift, origin, grid)) {
        log(CAELIX_LOG_ERROR,
            "caelix_scene_flush: the box of the keys (%d, %d, %d) .. (%d, %d, %d) holds more than 2^32 brick cells",
            scene->key_min[0], scene->key_min[1], scene->key_min[2], scene->key_max[0], scene->key_max[1],
            scene->key_max[2]);
        return CAELIX_ERROR_UNSUPPORTED;
    }
    CaelixResult r = scene->flush_scratch.reserve_grow(4ull * n + 4 * cx::staging_sort_words(n), "caelix_scene_flush");
    if (r == CAELIX_OK) r = scene->record_of_slot.reserve_grow(4ull * std::max(n, 1u), "caelix_scene_flush");
    if (r == CAELIX_OK) r = scene->marks.reserve_grow(4ull * std::max(n, 1u), "caelix_scene_flush");
    // The edit lists of later flushes, sized for edits of up to 1/32 of the bricks.
    if (r == CAELIX_OK) r = scene->update.reserve_grow(4ull * (9ull * std::max(n / 32, 1024u) + 1), "caelix_scene_flush");
    if (r != CAELIX_OK) return r;
    float* d_power = static_cast<float*>(scene->flush_scratch.ptr);
    uint32_t* sort_scratch = reinterpret_cast<uint32_t*>(d_power + n);
    // The build rewrites the device tables in place: renders of the previous build, on any
    // stream, finish first.
    e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
    cudaEventRecord(scene->start, stream);
    e = cx::scene_alloc_inputs(scene->dev, n, stream);
    if (e == cudaSuccess && n)
        e = cudaMemcpyAsync(d_power, scene->slot_power.data(), 4ull * n, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(scene->marks.ptr, 0, 4ull * std::max(n, 1u), stream);
    if (e == cudaSuccess)
        e = cx::staging_gather(scene->stage_keys, scene->stage_voxels, d_power, n, origin, grid, sort_scratch,
                               scene->dev.status, scene->dev.keys, scene->dev.voxels, scene->dev.power,
                               static_cast<uint32_t*>(scene->record_of_slot.ptr), stream);
    if (e == cudaSuccess) e = cx::scene_build_device(scene->dev, origin, grid, scene->group_shift, n, stream, &status);
    cudaEventRecord(scene->stop, stream);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_scene_flush");
    cudaEventSynchronize(scene->stop);
    cudaEventElapsedTime(&scene->flush_ms, scene->start, scene->stop);
    for (uint32_t slot : scene->dirty_slots) scene->slot_dirty[slot] = 0;
    scene->dirty_slots.clear();
    scene->mark_epoch = 0;
    scene->full_rebuild = false;
    scene->light_tree_dirty = false;
    scene->built = true;
    scene->generation += 1;
    return cx::status_result(status & ~cx::kStatusNodeOverflow, "caelix_scene_flush");
}

CAELIX_API CaelixResult caelix_scene_flush(CaelixScene* scene, const CaelixFrameDesc* desc)
{
    CAELIX_GUARD_BEGIN
    CaelixResult r = scene_flush_body(scene, desc);
    // Tree 0's static set follows the world's light tables.
    if (r == CAELIX_OK) r = refresh_static_lights(scene, reinterpret_cast<cudaStream_t>(desc->command_buffer));
    return r;
    CAELIX_GUARD_END
}

CAELIX_API void caelix_scene_get_light_stats(const CaelixScene* scene, CaelixLightStats* out)
{
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    if (!scene || !scene->built || !scene->light_options.enabled) return;
    const cx::DeviceScene& d = scene->dev;
    unsigned char host[128];
    cudaSetDevice(scene->device->ordinal);
    // Tree 0: the static set's tree while static entities have lights, else the world's own.
    const bool stat = scene->stat.live && scene->entity_view_count;
    const void* tree0 = stat ? static_cast<const void*>(scene->stat.v.header) : static_cast<const void*>(d.tree.header);
    if (cudaMemcpy(host, tree0, 128, cudaMemcpyDeviceToHost) != cudaSuccess) return;
    cx::LightTreeHeader h;
    cx::LightTreeState st;
    std::memcpy(&h, host, 64);
    std::memcpy(&st, host + 64, 64);
    out->enabled = 1;
    out->light_bricks = d.light_count;
    out->heap_bytes_used = 4ull * d.heap_words;
    out->heap_bytes_capacity = 4ull * d.heap_words;
    out->passes = 1;
    out->records_recomputed = d.light_count;
    out->gpu_ms = scene->flush_ms;
    out->tree_leaves[0] = h.leaf_count;
    out->tree_nodes[0] = h.node_count;
    out->tree_builds[0] = st.builds;
    out->tree_leaves_dropped[0] = st.leaves_dropped;
    if (scene->dyn.live && scene->entity_view_count &&
        cudaMemcpy(host, scene->dyn.v.header, 128, cudaMemcpyDeviceToHost) == cudaSuccess) {
        std::memcpy(&h, host, 64);
        std::memcpy(&st, host + 64, 64);
        out->tree_leaves[1] = h.leaf_count;
        out->tree_nodes[1] = h.node_count;
        out->tree_builds[1] = st.builds;
        out->tree_leaves_dropped[1] = st.leaves_dropped;
    }
    std::vector<uint32_t> rows(8ull * d.group_count);
    if (d.group_count &&
        cudaMemcpy(rows.data(), d.group_rows, 32ull * d.group_count, cudaMemcpyDeviceToHost) == cudaSuccess) {
        for (uint32_t g = 0; g < d.group_count; ++g) out->light_groups += rows[8ull * g + 5] ? 1u : 0u;
    }
    if (d.light_count) {
        std::vector<cx::BrickLightRecord> hdr(d.light_count);
        if (cudaMemcpy(hdr.data(), d.light_headers, sizeof(cx::BrickLightRecord) * d.light_count,
                       cudaMemcpyDeviceToHost) == cudaSuccess)
            for (const auto& r : hdr) out->light_faces += r.entry_count;
    }
}

CAELIX_API CaelixResult caelix_scene_get_view(const CaelixScene* scene, CaelixSceneView* out)
{
    if (!scene || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (!scene->built) return CAELIX_OK;
    const cx::DeviceScene& d = scene->dev;
    for (int k = 0; k < 3; ++k) {
        out->grid[k] = d.grid[k];
        out->groups[k] = d.groups[k];
        out->origin[k] = d.origin[k];
    }
    out->encoding = d.encoding;
    out->group_shift = d.group_shift;
    out->brick_count = d.brick_count;
    out->hash_capacity = d.hash_capacity;
    out->hash_slot_count = d.hash_slot_count;
    out->hash_max_probe = d.hash_max_probe;
    out->light_count = d.light_count;
    out->heap_words = d.heap_words;
    out->group_count = d.group_count;
    out->keys = reinterpret_cast<uint64_t>(d.keys);
    out->records = reinterpret_cast<uint64_t>(d.records);
    out->hash_slots = reinterpret_cast<uint64_t>(d.hash_slots);
    out->bitmap = reinterpret_cast<uint64_t>(d.bitmap);
    out->heap = reinterpret_cast<uint64_t>(d.heap);
    out->group_rows = reinterpret_cast<uint64_t>(d.group_rows);
    out->light_headers = reinterpret_cast<uint64_t>(d.light_headers);
    out->light_group = reinterpret_cast<uint64_t>(d.light_group);
    out->light_entry = reinterpret_cast<uint64_t>(d.light_entry);
    out->light_brick = reinterpret_cast<uint64_t>(d.light_brick);
    out->tree_header = reinterpret_cast<uint64_t>(d.tree.header);
    out->tree_nodes = reinterpret_cast<uint64_t>(d.tree.nodes);
    out->tree_leaves = reinterpret_cast<uint64_t>(d.tree.leaves);
    return CAELIX_OK;
}

CAELIX_API uint64_t caelix_scene_get_light_tree(const CaelixScene* scene)
{
    if (!scene || !scene->built || !scene->light_options.enabled) return 0;
    return reinterpret_cast<uint64_t>(scene->dev.tree.header);
}

CAELIX_API CaelixResult caelix_renderer_create(CaelixDevice* device, CaelixScene* scene, CaelixRenderer** out_renderer)
{
    CAELIX_GUARD_BEGIN
    if (!device || !scene || !out_renderer || scene->device != device) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out_renderer = nullptr;
    cudaSetDevice(device->ordinal);
    CaelixRenderer* r = new CaelixRenderer();
    r->device = device;
    r->scene = scene;
    cudaError_t e = cudaMalloc(&r->counts, 64);
    if (e == cudaSuccess) e = cudaEventCreate(&r->start);
    if (e == cudaSuccess) e = cudaEventCreate(&r->stop);
    if (e != cudaSuccess) {
        if (r->counts) cudaFree(r->counts);
        delete r;
        return cx::cuda_result(e, "caelix_renderer_create");
    }
    *out_renderer = r;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API void caelix_renderer_destroy(CaelixRenderer* renderer)
{
    if (!renderer) return;
    cudaSetDevice(renderer->device->ordinal);
    if (renderer->rendered) cudaStreamSynchronize(renderer->last_stream);
    if (renderer->counts) cudaFree(renderer->counts);
    if (renderer->start) cudaEventDestroy(renderer->start);
    if (renderer->stop) cudaEventDestroy(renderer->stop);
    renderer->wave_memory.release();
    renderer->wave_views.release();
    delete renderer;
}

CAELIX_API CaelixResult caelix_renderer_render(CaelixRenderer* renderer, const CaelixFrameDesc* frame,
                                               const CaelixRenderTargets* targets, const CaelixCamera* camera,
                                               const CaelixRenderOptions* options)
{
    CAELIX_GUARD_BEGIN
    if (!renderer || !frame) return CAELIX_ERROR_INVALID_ARGUMENT;
    cx::TraceParams p;
    const CaelixResult r = render_params(renderer, targets, camera, options, "caelix_renderer_render", &p);
    if (r != CAELIX_OK) return r;
    CaelixScene* scene = renderer->scene;
    cudaSetDevice(renderer->device->ordinal);
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(frame->command_buffer);
    cudaError_t e = cudaMemsetAsync(renderer->counts, 0, 24, stream);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_renderer_render");
    if (renderer->trace_mode == CAELIX_TRACE_MEGAKERNEL) {
        cudaEventRecord(renderer->start, stream);
        e = cx::trace_launch(render_view(scene), p, reinterpret_cast<float*>(targets->radiance),
                             renderer->counts, stream);
        cudaEventRecord(renderer->stop, stream);
        renderer->launches = 1;
    } else {
        // The wavefront trace of the one view: its path state sized for one sample of every pixel
        // (or the set capacity), the view and its wave table uploaded ahead of the kernels.
        cx::WaveView view;
        std::memset(&view, 0, sizeof(view));
        view.scene = render_view(scene);
        view.params = p;
        view.radiance = reinterpret_cast<float*>(targets->radiance);
        view.ray_counts = renderer->counts;
        constexpr uint32_t kBlockWidth = 8;  // 8 x 4 pixel blocks per warp
        view.blocks_x = (p.width + kBlockWidth - 1) / kBlockWidth;
        const cx::WavePlan plan = cx::wave_plan(&view, 1, kBlockWidth);
        const uint32_t items = plan.items.empty() ? 0 : plan.items[0];
        const uint32_t capacity = renderer->wave_capacity ? std::min(renderer->wave_capacity, items) : items;
        CaelixResult r2 = renderer->wave_memory.reserve(cx::wave_buffer_bytes(capacity), "caelix_renderer_render");
        const uint64_t view_bytes = (sizeof(cx::WaveView) + 255) & ~uint64_t{255};
        if (r2 == CAELIX_OK)
            r2 = renderer->wave_views.reserve(view_bytes + 4ull * plan.table.size(), "caelix_renderer_render");
        if (r2 != CAELIX_OK) return r2;
        char* vbase = static_cast<char*>(renderer->wave_views.ptr);
        cx::WaveView* d_view = reinterpret_cast<cx::WaveView*>(vbase);
        uint32_t* d_table = reinterpret_cast<uint32_t*>(vbase + view_bytes);
        e = cudaMemcpyAsync(d_view, &view, sizeof(view), cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_table, plan.table.data(), 4 * plan.table.size(), cudaMemcpyHostToDevice, stream);
        if (e != cudaSuccess) return cx::cuda_result(e, "caelix_renderer_render");
        const cx::WaveBuffers wb = cx::wave_carve(renderer->wave_memory.ptr, capacity);
        renderer->launches = 0;
        cudaEventRecord(renderer->start, stream);
        e = cx::wave_trace(&view, d_view, 1, plan, d_table, wb, kBlockWidth, renderer->device->sm_count, stream,
                           &renderer->launches);
        cudaEventRecord(renderer->stop, stream);
    }
    renderer->last_stream = stream;
    renderer->frame_number = frame->frame_number;
    renderer->rendered = true;
    return cx::cuda_result(e, "caelix_renderer_render");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_renderer_backward(CaelixRenderer* renderer, const CaelixFrameDesc* frame,
                                                 const CaelixRenderTargets* targets, const CaelixCamera* camera,
                                                 const CaelixRenderOptions* options, const float* d_radiance,
                                                 float* d_albedo, float* d_power)
{
    CAELIX_GUARD_BEGIN
    if (!renderer || !frame || !d_radiance || !d_albedo || !d_power) return CAELIX_ERROR_INVALID_ARGUMENT;
    cx::TraceParams p;
    // The forward image is optional here: a zero radiance pointer passes the target checks with a
    // stand-in and is not written.
    CaelixRenderTargets t = targets ? *targets : CaelixRenderTargets{0, 0, 0};
    const uint64_t image = t.radiance;
    if (!t.radiance) t.radiance = 1;
    const CaelixResult r = render_params(renderer, &t, camera, options, "caelix_renderer_backward", &p);
    if (r != CAELIX_OK) return r;
    CaelixScene* scene = renderer->scene;
    cudaSetDevice(renderer->device->ordinal);
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(frame->command_buffer);
    cudaError_t e = cudaMemsetAsync(d_albedo, 0, sizeof(float) * cx::kMaterialCodes * 3, stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_power, 0, sizeof(float) * std::max(scene->dev.brick_count, 1u), stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(renderer->counts, 0, 24, stream);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_renderer_backward");
    const CaelixResult r2 =
        renderer->wave_memory.reserve(cx::adjoint_bytes(p, renderer->wave_capacity), "caelix_renderer_backward");
    if (r2 != CAELIX_OK) return r2;
    renderer->launches = 0;
    cudaEventRecord(renderer->start, stream);
    e = cx::adjoint_launch(render_view(scene), p, d_radiance, reinterpret_cast<float*>(image), d_albedo,
                           d_power, renderer->counts, renderer->wave_memory.ptr, renderer->wave_capacity,
                           renderer->device->sm_count, stream, &renderer->launches);
    cudaEventRecord(renderer->stop, stream);
    renderer->last_stream = stream;
    renderer->frame_number = frame->frame_number;
    renderer->rendered = true;
    return cx::cuda_result(e, "caelix_renderer_backward");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_renderer_set_trace_mode(CaelixRenderer* renderer, uint32_t mode, uint32_t wave_capacity)
{
    if (!renderer || (mode != CAELIX_TRACE_WAVEFRONT && mode != CAELIX_TRACE_MEGAKERNEL) ||
        (wave_capacity != 0 && wave_capacity < 32))
        return CAELIX_ERROR_INVALID_ARGUMENT;
    renderer->trace_mode = mode;
    renderer->wave_capacity = wave_capacity;
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_renderer_set_light_nee_options(CaelixRenderer* renderer, const CaelixLightNeeOptions* options)
{
    if (!renderer || !options || options->enabled > 1 || options->flags != 0 || options->reserved != 0 ||
        (options->hint_patch != 0 && options->hint_patch != 1 && options->hint_patch != 2 && options->hint_patch != 4)) {
        log(CAELIX_LOG_ERROR, "caelix_renderer_set_light_nee_options: invalid options");
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    renderer->nee = *options;
    return CAELIX_OK;
}

CAELIX_API void caelix_renderer_get_gpu_timings(const CaelixRenderer* renderer, CaelixGpuTimings* out)
{
    if (!out) return;
    std::memset(out, 0, sizeof(*out));
    if (!renderer) return;
    cudaSetDevice(renderer->device->ordinal);
    out->flush_ms = renderer->scene->flush_ms;
    if (!renderer->rendered) return;
    cudaEventSynchronize(renderer->stop);
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, renderer->start, renderer->stop) == cudaSuccess) out->trace_ms = ms;
    out->frame_number = renderer->frame_number;
}

CAELIX_API CaelixResult caelix_renderer_get_stats(CaelixRenderer* renderer, CaelixRenderStats* out)
{
    CAELIX_GUARD_BEGIN
    if (!renderer || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (!renderer->rendered) return CAELIX_OK;
    cudaSetDevice(renderer->device->ordinal);
    cudaError_t e = cudaStreamSynchronize(renderer->last_stream);
    unsigned long long c[3] = {0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpy(c, renderer->counts, 24, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_renderer_get_stats");
    out->primary_rays = c[0];
    out->bounce_rays = c[1];
    out->shadow_rays = c[2];
    out->kernel_launches = renderer->launches;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

}  // extern "C"
