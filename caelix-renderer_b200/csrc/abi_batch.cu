// The batch part of the C ABI (include/caelix_b200.h): many views of many scenes in one CUDA graph
// launch (per-scene light-tree rebuilds as parallel graph branches, then the trace of every view:
// the persistent kernel of trace_batch.cu or the wavefront kernels of wave.cu), and the autotuner
// of its launch parameters with a JSON cache.
// No counterpart in the reference, which renders one scene per renderer call
// (lib/src/abi/caelix.cpp:700-953).
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/caelix_b200.h"
#include "abi_internal.h"
#include "abi_scene_internal.h"
#include "lt_build.cuh"
#include "scene.cuh"
#include "trace.cuh"

using cx::log;

namespace {

constexpr uint32_t kMaxBranches = 8;  // parallel streams of the light-tree builds in the graph

CaelixBatchTuning default_tuning()
{
    CaelixBatchTuning t;
    std::memset(&t, 0, sizeof(t));
    t.min_blocks = 6;
    t.wavefront = 0;
    t.block_width = 16;
    t.refill_min = 4;
    t.sort_keys_per_thread = 16;
    t.order = 1;
    return t;
}

constexpr uint32_t kDefaultWaveSlots = 1u << 22;

bool tuning_ok(const CaelixBatchTuning& t)
{
    return cx::trace_batch_variant_ok(t.min_blocks) &&
           (t.block_width == 8 || t.block_width == 16 || t.block_width == 32) && t.refill_min >= 1 &&
           t.refill_min <= 32 && cx::sort_keys_per_thread_ok(t.sort_keys_per_thread) && t.order <= 1 &&
           t.kernel <= CAELIX_BATCH_WAVEFRONT && (t.kernel != CAELIX_BATCH_WAVEFRONT || t.wavefront == 0 ||
                                                   t.wavefront >= 32) &&
           t.reserved == 0;
}

bool same_tuning(const CaelixBatchTuning& a, const CaelixBatchTuning& b)
{
    return std::memcmp(&a, &b, sizeof(a)) == 0;
}

}  // namespace

struct CaelixBatch
{
    CaelixDevice* device = nullptr;
    std::vector<CaelixBatchView> views;
    bool rebuild = true;
    std::vector<CaelixScene*> scenes;       // distinct scenes, in order of first appearance
    std::vector<uint64_t> generations;      // of the scenes when the graph was captured
    std::vector<uint64_t> entity_generations;  // of the scenes' entity views then
    CaelixBatchTuning tuning = default_tuning();
    cx::BatchView* d_views = nullptr;
    cx::WaveView* d_wave_views = nullptr;
    cx::GrowBuffer wave_table;               // the wave plan's view tables
    cx::GrowBuffer wave_memory;              // path state and queues of the wavefront kernels
    cx::WavePlan plan;                       // of the uploaded view order
    std::vector<cx::WaveView> wave_views;    // host copy, in the uploaded order
    unsigned long long* d_counts = nullptr;  // [view][3]
    uint32_t* d_next = nullptr;
    cudaStream_t capture = nullptr;
    cudaStream_t branches[kMaxBranches] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t joins[kMaxBranches] = {};
    cudaGraphExec_t exec = nullptr;
    CaelixBatchTuning exec_tuning{};  // the tuning `exec` was captured with
    uint32_t captures = 0;
    uint32_t kernel_nodes = 0;
    uint32_t wavefront = 0;
    cudaEvent_t start = nullptr;
    cudaEvent_t stop = nullptr;
    cudaStream_t last_stream = nullptr;
    bool ran = false;
};

namespace {

// The kernel organisation a run uses: the tuning's, except that views of scenes with entities are
// traced by the wavefront kernels (the persistent kernel traces world bricks only).
uint32_t run_kernel(const CaelixBatch* b, const CaelixBatchTuning& t)
{
    for (const CaelixScene* s : b->scenes)
        if (s->entity_view_count) return CAELIX_BATCH_WAVEFRONT;
    return t.kernel;
}

void release(CaelixBatch* b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->d_views) cudaFree(b->d_views);
    if (b->d_wave_views) cudaFree(b->d_wave_views);
    b->wave_table.release();
    b->wave_memory.release();
    if (b->d_counts) cudaFree(b->d_counts);
    if (b->d_next) cudaFree(b->d_next);
    if (b->capture) cudaStreamDestroy(b->capture);
    for (uint32_t i = 0; i < kMaxBranches; ++i) {
        if (b->branches[i]) cudaStreamDestroy(b->branches[i]);
        if (b->joins[i]) cudaEventDestroy(b->joins[i]);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->start) cudaEventDestroy(b->start);
    if (b->stop) cudaEventDestroy(b->stop);
}

// The device view table for a tuning: views ordered as the tuning says, consecutive item ranges,
// counters by the caller's view index. Uploaded synchronously (outside any capture).
cudaError_t upload_views(CaelixBatch* b, const CaelixBatchTuning& t, uint32_t* item_count)
{
    const uint32_t n = (uint32_t)b->views.size();
    std::vector<uint32_t> order(n);
    for (uint32_t i = 0; i < n; ++i) order[i] = i;
    if (t.order == 1) {
        auto work = [&](uint32_t i) {
            const CaelixBatchView& v = b->views[i];
            return (uint64_t)v.target.width * v.target.height * (v.options.spp ? v.options.spp : 1);
        };
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return work(x) > work(y); });
    }
    const uint32_t bw = t.block_width;
    const uint32_t bh = 32u / bw;
    std::vector<cx::BatchView> host(n);
    b->wave_views.assign(n, cx::WaveView{});
    uint64_t items = 0;
    for (uint32_t j = 0; j < n; ++j) {
        const uint32_t i = order[j];
        const CaelixBatchView& v = b->views[i];
        cx::BatchView& h = host[j];
        std::memset(&h, 0, sizeof(h));
        h.scene = render_view(v.renderer->scene);
        const CaelixResult r = render_params(v.renderer, &v.target, &v.camera, &v.options, "caelix_batch_run", &h.params);
        if (r != CAELIX_OK) return cudaErrorInvalidValue;
        h.radiance = reinterpret_cast<float*>(v.target.radiance);
        h.ray_counts = b->d_counts + 3ull * i;
        h.item_base = (uint32_t)items;
        h.blocks_x = (v.target.width + bw - 1) / bw;
        cx::WaveView& wv = b->wave_views[j];
        std::memset(&wv, 0, sizeof(wv));
        wv.scene = h.scene;
        wv.params = h.params;
        wv.radiance = h.radiance;
        wv.ray_counts = h.ray_counts;
        wv.blocks_x = h.blocks_x;
        const uint64_t blocks_y = (v.target.height + bh - 1) / bh;
        items += 32ull * h.blocks_x * blocks_y;
        // The work counter runs past the last item by at most 32 per warp: keep clear of 2^32.
        if (items >= (1ull << 32) - (1ull << 24)) return cudaErrorInvalidValue;
    }
    *item_count = (uint32_t)items;
    CX_TRY(cudaMemcpy(b->d_views, host.data(), sizeof(cx::BatchView) * n, cudaMemcpyHostToDevice));
    if (run_kernel(b, t) != CAELIX_BATCH_WAVEFRONT) return cudaSuccess;
    // The wavefront organisation: its view table, wave plan and path state.
    CX_TRY(cudaMemcpy(b->d_wave_views, b->wave_views.data(), sizeof(cx::WaveView) * n, cudaMemcpyHostToDevice));
    b->plan = cx::wave_plan(b->wave_views.data(), n, bw);
    if (b->wave_table.reserve(4ull * std::max<size_t>(b->plan.table.size(), 1), "caelix_batch_run") != CAELIX_OK)
        return cudaErrorMemoryAllocation;
    CX_TRY(cudaMemcpy(b->wave_table.ptr, b->plan.table.data(), 4 * b->plan.table.size(), cudaMemcpyHostToDevice));
    uint32_t largest = 0;
    for (uint32_t w : b->plan.items) largest = std::max(largest, w);
    const uint32_t slots = std::min(largest, t.wavefront ? t.wavefront : kDefaultWaveSlots);
    if (b->wave_memory.reserve(cx::wave_buffer_bytes(slots), "caelix_batch_run") != CAELIX_OK)
        return cudaErrorMemoryAllocation;
    return cudaSuccess;
}

uint32_t wave_slots(const CaelixBatch* b, const CaelixBatchTuning& t)
{
    uint32_t largest = 0;
    for (uint32_t w : b->plan.items) largest = std::max(largest, w);
    return std::max(32u, std::min(largest, t.wavefront ? t.wavefront : kDefaultWaveSlots));
}

uint32_t trace_grid(const CaelixBatch* b, const CaelixBatchTuning& t)
{
    const int per_sm = cx::trace_batch_blocks_per_sm(t.min_blocks);
    const uint32_t resident = b->device->sm_count * (uint32_t)std::max(per_sm, 1);
    if (t.wavefront == 0) return resident;
    return std::max(1u, std::min(resident, t.wavefront / cx::kBatchThreads));
}

// Records the work of a run (builds and/or trace) into `s`.
cudaError_t record(CaelixBatch* b, const CaelixBatchTuning& t, uint32_t item_count, uint32_t grid, bool builds,
                   bool trace, cudaStream_t s)
{
    if (builds && b->rebuild && !b->scenes.empty()) {
        CX_TRY(cudaEventRecord(b->fork, s));
        const uint32_t used = std::min<uint32_t>(kMaxBranches, (uint32_t)b->scenes.size());
        for (uint32_t j = 0; j < used; ++j) CX_TRY(cudaStreamWaitEvent(b->branches[j], b->fork, 0));
        uint32_t branch = 0;
        for (size_t i = 0; i < b->scenes.size(); ++i) {
            CaelixScene* sc = b->scenes[i];
            // Tree 0: the world's own, or the static set's (world and static entities' lights).
            if (sc->stat.live && sc->entity_view_count) {
                cx::LightBvhInput in = sc->stat.input;
                in.sort_keys_per_thread = t.sort_keys_per_thread;
                CX_TRY(cx::lt_build(cx::lt_carve(sc->stat.tree.ptr, sc->stat.tree_capacity), in,
                                    b->branches[branch++ % used], nullptr));
            } else {
                CX_TRY(cx::scene_build_light_tree(sc->dev, b->branches[branch++ % used], t.sort_keys_per_thread));
            }
            if (sc->dyn.live && sc->entity_view_count) {  // the dynamic entities' light tree
                cx::LightBvhInput in = sc->dyn.input;
                in.sort_keys_per_thread = t.sort_keys_per_thread;
                CX_TRY(cx::lt_build(cx::lt_carve(sc->dyn.tree.ptr, sc->dyn.tree_capacity), in,
                                    b->branches[branch++ % used], nullptr));
            }
        }
        for (uint32_t j = 0; j < used; ++j) {
            CX_TRY(cudaEventRecord(b->joins[j], b->branches[j]));
            CX_TRY(cudaStreamWaitEvent(s, b->joins[j], 0));
        }
    }
    if (trace && run_kernel(b, t) == CAELIX_BATCH_WAVEFRONT) {
        CX_TRY(cudaMemsetAsync(b->d_counts, 0, 24ull * b->views.size(), s));
        const cx::WaveBuffers wb = cx::wave_carve(b->wave_memory.ptr, wave_slots(b, t));
        return cx::wave_trace(b->wave_views.data(), b->d_wave_views, (uint32_t)b->views.size(), b->plan,
                              static_cast<const uint32_t*>(b->wave_table.ptr), wb, t.block_width, b->device->sm_count,
                              s, nullptr);
    }
    if (trace) {
        CX_TRY(cudaMemsetAsync(b->d_counts, 0, 24ull * b->views.size(), s));
        CX_TRY(cudaMemsetAsync(b->d_next, 0, 4, s));
        cx::BatchLaunch L;
        L.views = b->d_views;
        L.view_count = (uint32_t)b->views.size();
        L.item_count = item_count;
        L.block_width = t.block_width;
        L.refill_min = t.refill_min;
        L.next_item = b->d_next;
        CX_TRY(cx::trace_batch_launch(L, t.min_blocks, grid, s));
    }
    return cudaSuccess;
}

// Captures the work of a run into an executable graph.
cudaError_t capture_graph(CaelixBatch* b, const CaelixBatchTuning& t, bool builds, bool trace, cudaGraphExec_t* out,
                          uint32_t* kernel_nodes)
{
    uint32_t items = 0;
    CX_TRY(upload_views(b, t, &items));
    const uint32_t grid = trace_grid(b, t);  // (an occupancy query: before the capture)
    cudaGraph_t graph = nullptr;
    CX_TRY(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
    const cudaError_t e = record(b, t, items, grid, builds, trace, b->capture);
    const cudaError_t end = cudaStreamEndCapture(b->capture, &graph);
    if (e != cudaSuccess || end != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return e != cudaSuccess ? e : end;
    }
    size_t count = 0;
    cudaError_t g = cudaGraphGetNodes(graph, nullptr, &count);
    if (g == cudaSuccess && kernel_nodes) {
        std::vector<cudaGraphNode_t> nodes(count);
        g = cudaGraphGetNodes(graph, nodes.data(), &count);
        uint32_t kernels = 0;
        for (size_t i = 0; g == cudaSuccess && i < count; ++i) {
            cudaGraphNodeType type;
            if (cudaGraphNodeGetType(nodes[i], &type) == cudaSuccess && type == cudaGraphNodeTypeKernel) ++kernels;
        }
        *kernel_nodes = kernels;
    }
    if (g == cudaSuccess) g = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    return g;
}

bool scenes_moved(const CaelixBatch* b)
{
    for (size_t i = 0; i < b->scenes.size(); ++i)
        if (b->scenes[i]->generation != b->generations[i] ||
            b->scenes[i]->entity_generation != b->entity_generations[i])
            return true;
    return false;
}

// The graph of a full run with the batch's tuning, captured again when needed.
cudaError_t ensure_graph(CaelixBatch* b)
{
    if (b->exec && same_tuning(b->exec_tuning, b->tuning) && !scenes_moved(b)) return cudaSuccess;
    for (CaelixScene* s : b->scenes)
        if (!s->built) return cudaErrorInvalidValue;
    // The view table is rewritten below: the previous run must have finished reading it.
    if (b->ran) CX_TRY(cudaStreamSynchronize(b->last_stream));
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    uint32_t kernels = 0;
    CX_TRY(capture_graph(b, b->tuning, true, true, &b->exec, &kernels));
    b->exec_tuning = b->tuning;
    b->kernel_nodes = kernels;
    b->wavefront = run_kernel(b, b->tuning) == CAELIX_BATCH_WAVEFRONT ? wave_slots(b, b->tuning)
                                                               : trace_grid(b, b->tuning) * cx::kBatchThreads;
    for (size_t i = 0; i < b->scenes.size(); ++i) {
        b->generations[i] = b->scenes[i]->generation;
        b->entity_generations[i] = b->scenes[i]->entity_generation;
    }
    b->captures += 1;
    return cudaSuccess;
}

// ---- the autotuner ----

uint64_t fnv1a(uint64_t h, const void* p, size_t n)
{
    const unsigned char* c = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; ++i) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

// The cache key: the GPU (name, SM count) and the workload's shape (views' sizes and options,
// scenes' brick and light counts).
std::string tuning_key(const CaelixBatch* b)
{
    cudaDeviceProp prop;
    std::memset(&prop, 0, sizeof(prop));
    cudaGetDeviceProperties(&prop, b->device->ordinal);
    uint64_t h = 1469598103934665603ull;
    for (const CaelixBatchView& v : b->views) {
        const uint32_t w[5] = {v.target.width, v.target.height, v.options.spp ? v.options.spp : 1,
                               v.options.bounce_count, v.renderer->nee.enabled};
        h = fnv1a(h, w, sizeof(w));
        size_t scene = 0;
        while (b->scenes[scene] != v.renderer->scene) ++scene;
        const uint32_t sc = (uint32_t)scene;
        h = fnv1a(h, &sc, sizeof(sc));
    }
    for (const CaelixScene* s : b->scenes) {
        const uint32_t w[2] = {s->dev.brick_count, s->dev.light_count};
        h = fnv1a(h, w, sizeof(w));
    }
    std::string name = prop.name;
    for (char& c : name)
        if (c == '"' || c == '\\' || c == '|') c = '_';
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s|sm%d|views%zu|rebuild%d|%016llx", name.c_str(), prop.multiProcessorCount,
                  b->views.size(), b->rebuild ? 1 : 0, (unsigned long long)h);
    return buf;
}

// The cache file: one JSON object, one entry per line:
//   {"format": "caelix-batch-tuning/1", "entries": [
//   {"key": "...", "min_blocks": 6, "wavefront": 0, "block_width": 16, "refill_min": 4, "sort_keys_per_thread": 16, "order": 1, "kernel": 1, "ms": 12.5},
//   ...
//   ]}
bool read_field(const std::string& line, const char* name, double* out)
{
    const std::string tag = std::string("\"") + name + "\": ";
    const size_t at = line.find(tag);
    if (at == std::string::npos) return false;
    const char* p = line.c_str() + at + tag.size();
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(p, &end);
    if (end == p || errno != 0) return false;
    *out = v;
    return true;
}

std::vector<std::string> cache_entries(const char* path)
{
    std::vector<std::string> out;
    std::ifstream in(path);
    std::string line;
    while (std::getline(in, line))
        if (line.find("{\"key\": \"") != std::string::npos) {
            while (!line.empty() && (line.back() == ',' || line.back() == ' ' || line.back() == '\r')) line.pop_back();
            out.push_back(line);
        }
    return out;
}

bool cache_lookup(const char* path, const std::string& key, CaelixBatchTuning* t)
{
    const std::string tag = "{\"key\": \"" + key + "\",";
    for (const std::string& line : cache_entries(path)) {
        if (line.compare(0, tag.size(), tag) != 0) continue;
        CaelixBatchTuning c = default_tuning();
        double v;
        const char* names[7] = {"min_blocks", "wavefront",  "block_width", "refill_min", "sort_keys_per_thread",
                                "order",      "kernel"};
        uint32_t* fields[7] = {&c.min_blocks, &c.wavefront, &c.block_width, &c.refill_min, &c.sort_keys_per_thread,
                               &c.order,      &c.kernel};
        bool ok = true;
        for (int i = 0; i < 7; ++i) {
            if (!read_field(line, names[i], &v) || v < 0 || v > 4294967295.0) {
                ok = false;
                break;
            }
            *fields[i] = (uint32_t)v;
        }
        if (ok && tuning_ok(c)) {
            *t = c;
            return true;
        }
    }
    return false;
}

bool cache_store(const char* path, const std::string& key, const CaelixBatchTuning& t, float ms)
{
    std::vector<std::string> entries = cache_entries(path);
    const std::string tag = "{\"key\": \"" + key + "\",";
    entries.erase(std::remove_if(entries.begin(), entries.end(),
                                 [&](const std::string& l) { return l.compare(0, tag.size(), tag) == 0; }),
                  entries.end());
    char buf[1024];
    std::snprintf(buf, sizeof(buf),
                  "{\"key\": \"%s\", \"min_blocks\": %u, \"wavefront\": %u, \"block_width\": %u, \"refill_min\": %u, "
                  "\"sort_keys_per_thread\": %u, \"order\": %u, \"kernel\": %u, \"ms\": %.4f}",
                  key.c_str(), t.min_blocks, t.wavefront, t.block_width, t.refill_min, t.sort_keys_per_thread, t.order,
                  t.kernel, (double)ms);
    entries.push_back(buf);
    const std::string tmp = std::string(path) + ".tmp";
    {
        std::ofstream out(tmp, std::ios::trunc);
        if (!out) return false;
        out << "{\"format\": \"caelix-batch-tuning/1\", \"entries\": [\n";
        for (size_t i = 0; i < entries.size(); ++i) out << entries[i] << (i + 1 < entries.size() ? ",\n" : "\n");
        out << "]}\n";
        if (!out) return false;
    }
    return std::rename(tmp.c_str(), path) == 0;
}

// Minimum over `repeats` timed launches of a graph of the given part of a run, after one warm-up.
cudaError_t time_part(CaelixBatch* b, const CaelixBatchTuning& t, bool builds, bool trace, cudaStream_t s,
                      uint32_t repeats, float* best_ms)
{
    cudaGraphExec_t exec = nullptr;
    CX_TRY(capture_graph(b, t, builds, trace, &exec, nullptr));
    cudaError_t e = cudaGraphLaunch(exec, s);
    float best = INFINITY;
    for (uint32_t r = 0; e == cudaSuccess && r < repeats; ++r) {
        e = cudaEventRecord(b->start, s);
        if (e == cudaSuccess) e = cudaGraphLaunch(exec, s);
        if (e == cudaSuccess) e = cudaEventRecord(b->stop, s);
        if (e == cudaSuccess) e = cudaEventSynchronize(b->stop);
        float ms = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b->start, b->stop);
        if (e == cudaSuccess) best = std::min(best, ms);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaGraphExecDestroy(exec);
    *best_ms = best;
    return e;
}

}  // namespace

extern "C" {

CAELIX_API CaelixResult caelix_batch_create(CaelixDevice* device, const CaelixBatchDesc* desc, CaelixBatch** out_batch)
{
    CAELIX_GUARD_BEGIN
    if (!device || !desc || !out_batch || !desc->views || desc->view_count == 0 ||
        desc->view_count > cx::kMaxBatchViews || desc->rebuild_light_trees > 1)
        return CAELIX_ERROR_INVALID_ARGUMENT;
    *out_batch = nullptr;
    for (uint32_t r : desc->reserved)
        if (r) return CAELIX_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(device->ordinal);
    CaelixBatch* b = new CaelixBatch();
    b->device = device;
    b->rebuild = desc->rebuild_light_trees == 1;
    b->views.assign(desc->views, desc->views + desc->view_count);
    for (uint32_t i = 0; i < desc->view_count; ++i) {
        const CaelixBatchView& v = b->views[i];
        cx::TraceParams p;
        CaelixResult r = v.renderer ? CAELIX_OK : CAELIX_ERROR_INVALID_ARGUMENT;
        if (r == CAELIX_OK && v.renderer->device != device) r = CAELIX_ERROR_INVALID_ARGUMENT;
        if (r == CAELIX_OK) r = render_params(v.renderer, &v.target, &v.camera, &v.options, "caelix_batch_create", &p);
        if (r == CAELIX_OK) {
            cudaPointerAttributes attr;
            if (cudaPointerGetAttributes(&attr, reinterpret_cast<const void*>(v.target.radiance)) != cudaSuccess ||
                (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) ||
                attr.device != device->ordinal) {
                cudaGetLastError();
                log(CAELIX_LOG_ERROR, "caelix_batch_create: view %u: the target is not device memory of this device", i);
                r = CAELIX_ERROR_INVALID_ARGUMENT;
            }
        }
        if (r != CAELIX_OK) {
            log(CAELIX_LOG_ERROR, "caelix_batch_create: view %u is invalid", i);
            delete b;
            return r;
        }
        CaelixScene* s = v.renderer->scene;
        if (std::find(b->scenes.begin(), b->scenes.end(), s) == b->scenes.end()) b->scenes.push_back(s);
    }
    b->generations.assign(b->scenes.size(), ~0ull);
    b->entity_generations.assign(b->scenes.size(), ~0ull);
    const uint32_t n = desc->view_count;
    cudaError_t e = cudaMalloc(&b->d_views, sizeof(cx::BatchView) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_wave_views, sizeof(cx::WaveView) * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_counts, 24ull * n);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_next, 64);
    if (e == cudaSuccess) e = cudaMemset(b->d_counts, 0, 24ull * n);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking);
    for (uint32_t i = 0; e == cudaSuccess && i < kMaxBranches; ++i) {
        e = cudaStreamCreateWithFlags(&b->branches[i], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->joins[i], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreate(&b->start);
    if (e == cudaSuccess) e = cudaEventCreate(&b->stop);
    if (e != cudaSuccess) {
        release(b);
        delete b;
        return cx::cuda_result(e, "caelix_batch_create");
    }
    *out_batch = b;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API void caelix_batch_destroy(CaelixBatch* batch)
{
    if (!batch) return;
    cudaSetDevice(batch->device->ordinal);
    if (batch->ran) cudaStreamSynchronize(batch->last_stream);
    release(batch);
    delete batch;
}

CAELIX_API CaelixResult caelix_batch_run(CaelixBatch* batch, const CaelixFrameDesc* frame)
{
    CAELIX_GUARD_BEGIN
    if (!batch || !frame) return CAELIX_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(batch->device->ordinal);
    cudaError_t e = ensure_graph(batch);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_batch_run");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(frame->command_buffer);
    e = cudaEventRecord(batch->start, s);
    if (e == cudaSuccess) e = cudaGraphLaunch(batch->exec, s);
    if (e == cudaSuccess) e = cudaEventRecord(batch->stop, s);
    batch->last_stream = s;
    batch->ran = e == cudaSuccess;
    return cx::cuda_result(e, "caelix_batch_run");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_batch_set_tuning(CaelixBatch* batch, const CaelixBatchTuning* tuning)
{
    if (!batch || !tuning || !tuning_ok(*tuning)) return CAELIX_ERROR_INVALID_ARGUMENT;
    batch->tuning = *tuning;
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_batch_get_tuning(const CaelixBatch* batch, CaelixBatchTuning* out)
{
    if (!batch || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out = batch->tuning;
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_batch_autotune(CaelixBatch* batch, const CaelixFrameDesc* frame, const char* cache_path,
                                              uint32_t repeats, CaelixBatchTuning* out)
{
    CAELIX_GUARD_BEGIN
    if (!batch || !frame) return CAELIX_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(batch->device->ordinal);
    for (CaelixScene* s : batch->scenes)
        if (!s->built) return CAELIX_ERROR_INVALID_ARGUMENT;
    const std::string key = tuning_key(batch);
    CaelixBatchTuning t = batch->tuning;
    if (cache_path && cache_lookup(cache_path, key, &t)) {
        batch->tuning = t;
        if (out) *out = t;
        return CAELIX_OK;
    }
    if (repeats == 0) repeats = 2;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(frame->command_buffer);
    cudaError_t e = batch->ran ? cudaStreamSynchronize(batch->last_stream) : cudaSuccess;
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_batch_autotune");
    // The sort tile on the builds alone.
    if (batch->rebuild && !batch->scenes.empty()) {
        float best = INFINITY;
        uint32_t best_kpt = t.sort_keys_per_thread;
        for (uint32_t kpt : {4u, 8u, 16u}) {
            CaelixBatchTuning c = t;
            c.sort_keys_per_thread = kpt;
            float ms = 0.0f;
            e = time_part(batch, c, true, false, s, repeats, &ms);
            if (e != cudaSuccess) return cx::cuda_result(e, "caelix_batch_autotune");
            if (ms < best) {
                best = ms;
                best_kpt = kpt;
            }
        }
        t.sort_keys_per_thread = best_kpt;
    }
    // The trace parameters on the trace alone: for each kernel organisation a coordinate descent
    // over its own parameters; the best of the two.
    struct Axis
    {
        uint32_t CaelixBatchTuning::*field;
        std::vector<uint32_t> values;
    };
    const uint32_t full = batch->device->sm_count * 8u * cx::kBatchThreads;
    const std::vector<Axis> persistent_axes = {
        {&CaelixBatchTuning::min_blocks, {4u, 6u, 8u}},
        {&CaelixBatchTuning::block_width, {8u, 16u, 32u}},
        {&CaelixBatchTuning::refill_min, {1u, 4u, 16u}},
        {&CaelixBatchTuning::order, {0u, 1u}},
        {&CaelixBatchTuning::wavefront, {0u, full / 4u, full / 2u}},
    };
    const std::vector<Axis> wave_axes = {
        {&CaelixBatchTuning::block_width, {8u, 16u, 32u}},
        {&CaelixBatchTuning::order, {0u, 1u}},
        {&CaelixBatchTuning::wavefront, {0u, 1u << 20, 1u << 24}},
    };
    float best = INFINITY;
    CaelixBatchTuning best_t = t;
    for (uint32_t kernel : {CAELIX_BATCH_PERSISTENT, CAELIX_BATCH_WAVEFRONT}) {
        if (run_kernel(batch, CaelixBatchTuning{0, 0, 0, 0, 0, 0, kernel, 0}) != kernel) continue;
        CaelixBatchTuning k = t;
        k.kernel = kernel;
        k.wavefront = 0;
        float k_best = 0.0f;
        e = time_part(batch, k, false, true, s, repeats, &k_best);
        if (e != cudaSuccess) return cx::cuda_result(e, "caelix_batch_autotune");
        for (const Axis& axis : kernel == CAELIX_BATCH_WAVEFRONT ? wave_axes : persistent_axes) {
            for (uint32_t value : axis.values) {
                if (k.*(axis.field) == value) continue;
                CaelixBatchTuning c = k;
                c.*(axis.field) = value;
                float ms = 0.0f;
                e = time_part(batch, c, false, true, s, repeats, &ms);
                if (e != cudaSuccess) return cx::cuda_result(e, "caelix_batch_autotune");
                if (ms < k_best) {
                    k_best = ms;
                    k = c;
                }
            }
        }
        if (k_best < best) {
            best = k_best;
            best_t = k;
        }
    }
    t = best_t;
    batch->tuning = t;
    if (cache_path && !cache_store(cache_path, key, t, best))
        log(CAELIX_LOG_WARNING, "caelix_batch_autotune: could not write the cache %s", cache_path);
    if (out) *out = t;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_batch_get_stats(CaelixBatch* batch, CaelixBatchStats* out)
{
    CAELIX_GUARD_BEGIN
    if (!batch || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    out->graph_captures = batch->captures;
    if (!batch->ran) return CAELIX_OK;
    cudaSetDevice(batch->device->ordinal);
    cudaError_t e = cudaEventSynchronize(batch->stop);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&out->gpu_ms, batch->start, batch->stop);
    std::vector<unsigned long long> c(3 * batch->views.size());
    if (e == cudaSuccess) e = cudaMemcpy(c.data(), batch->d_counts, 8 * c.size(), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_batch_get_stats");
    for (size_t i = 0; i < batch->views.size(); ++i) {
        out->primary_rays += c[3 * i];
        out->bounce_rays += c[3 * i + 1];
        out->shadow_rays += c[3 * i + 2];
    }
    out->kernel_launches = batch->kernel_nodes;
    out->light_tree_builds = batch->rebuild ? (uint32_t)batch->scenes.size() : 0u;
    out->wavefront = batch->wavefront;
    uint32_t status = 0;
    for (CaelixScene* s : batch->scenes) {
        uint32_t st = 0;
        e = cx::scene_read_status(s->dev, batch->last_stream, &st);
        if (e != cudaSuccess) return cx::cuda_result(e, "caelix_batch_get_stats");
        status |= st;
    }
    return cx::status_result(status & ~cx::kStatusNodeOverflow, "caelix_batch_get_stats");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_batch_get_view_stats(CaelixBatch* batch, uint32_t view, CaelixRenderStats* out)
{
    CAELIX_GUARD_BEGIN
    if (!batch || !out || view >= batch->views.size()) return CAELIX_ERROR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (!batch->ran) return CAELIX_OK;
    cudaSetDevice(batch->device->ordinal);
    unsigned long long c[3] = {0, 0, 0};
    cudaError_t e = cudaEventSynchronize(batch->stop);
    if (e == cudaSuccess) e = cudaMemcpy(c, batch->d_counts + 3ull * view, 24, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_batch_get_view_stats");
    out->primary_rays = c[0];
    out->bounce_rays = c[1];
    out->shadow_rays = c[2];
    out->kernel_launches = 1;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

}  // extern "C"
