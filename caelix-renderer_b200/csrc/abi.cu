// The C ABI shim (include/caelix_b200.h): handle objects, argument checks, CUDA errors and device
// status words -> CaelixResult, logging through the host callback. Replaces the reference's
// lib/src/abi/caelix.cpp (TranslateException :79-110 and the entry points it guards).
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <algorithm>
#include <new>

#include "../../include/caelix_b200.h"
#include "abi_internal.h"
#include "cx_device.cuh"
#include "lt_build.cuh"
#include "radix_sort.cuh"

namespace {

std::mutex g_log_mutex;
CaelixLogCallback g_log = nullptr;
void* g_log_user = nullptr;

}  // namespace

namespace cx {

void log(CaelixLogLevel level, const char* fmt, ...)
{
    CaelixLogCallback cb;
    void* user;
    {
        std::lock_guard<std::mutex> lock(g_log_mutex);
        cb = g_log;
        user = g_log_user;
    }
    if (!cb) return;
    char buffer[1024];
    va_list args;
    va_start(args, fmt);
    vsnprintf(buffer, sizeof(buffer), fmt, args);
    va_end(args);
    cb(level, buffer, user);
}

CaelixResult cuda_result(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return CAELIX_OK;
    log(CAELIX_LOG_ERROR, "%s: %s", what, cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? CAELIX_ERROR_OUT_OF_MEMORY : CAELIX_ERROR_CUDA;
}

CaelixResult status_result(uint32_t status, const char* what)
{
    if (status == 0) return CAELIX_OK;
    log(CAELIX_LOG_ERROR, "%s: device status 0x%x%s%s%s%s%s%s%s", what, status,
        (status & kStatusLookbackTimeout) ? " lookback-timeout" : "",
        (status & kStatusDepthGuard) ? " depth-guard" : "", (status & kStatusNodeOverflow) ? " node-overflow" : "",
        (status & kStatusHashProbeLimit) ? " hash-probe-limit" : "",
        (status & kStatusRecordOverflow) ? " record-overflow" : "", (status & kStatusBadGroup) ? " bad-group" : "",
        (status & kStatusCopyTimeout) ? " copy-timeout" : "");
    return CAELIX_ERROR_DEVICE_STATUS;
}

// Device memory grown on demand (never shrunk).
CaelixResult GrowBuffer::reserve(uint64_t want, const char* what)
{
    if (want <= bytes) return CAELIX_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    const cudaError_t e = cudaMalloc(&ptr, want);
    if (e != cudaSuccess) return cuda_result(e, what);
    bytes = want;
    return CAELIX_OK;
}

void GrowBuffer::release()
{
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
}

}  // namespace cx

struct CaelixLightBvh
{
    CaelixDevice* device = nullptr;
    void* memory = nullptr;
    cx::LightBvhBuffers buffers;
    cudaStream_t last_stream = nullptr;
    cudaEvent_t start = nullptr;
    cudaEvent_t stop = nullptr;
    cudaEvent_t stage[cx::kBuildStages + 1] = {};
    bool profiling = false;
    bool built = false;
    bool profiled = false;
    uint32_t launches = 0;
    // The build as a CUDA graph, replayed while the inputs stay the same (one submission instead
    // of a launch per kernel: a small build is bound by launch latency, not by its work).
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    cx::LightBvhInput graph_input{};
};

namespace {

bool same_input(const cx::LightBvhInput& a, const cx::LightBvhInput& b)
{
    return a.records == b.records && a.count == b.count && a.record_group == b.record_group &&
           a.record_entry == b.record_entry && a.group_frames == b.group_frames && a.group_count == b.group_count &&
           a.sort_keys_per_thread == b.sort_keys_per_thread;
}

// The build of `in` as an instantiated graph (captured on the object's own stream).
cudaError_t capture_build(CaelixLightBvh* bvh, const cx::LightBvhInput& in)
{
    if (bvh->graph) {
        cudaGraphExecDestroy(bvh->graph);
        bvh->graph = nullptr;
    }
    if (!bvh->capture_stream) CX_TRY(cudaStreamCreateWithFlags(&bvh->capture_stream, cudaStreamNonBlocking));
    CX_TRY(cudaStreamBeginCapture(bvh->capture_stream, cudaStreamCaptureModeThreadLocal));
    const cudaError_t built = cx::lt_build(bvh->buffers, in, bvh->capture_stream, nullptr);
    cudaGraph_t graph = nullptr;
    const cudaError_t ended = cudaStreamEndCapture(bvh->capture_stream, &graph);
    if (built != cudaSuccess || ended != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return built != cudaSuccess ? built : ended;
    }
    const cudaError_t e = cudaGraphInstantiate(&bvh->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
        bvh->graph = nullptr;
        return e;
    }
    bvh->graph_input = in;
    return cudaSuccess;
}

}  // namespace

using cx::log;

extern "C" {

CAELIX_API void caelix_get_version(CaelixVersion* out)
{
    if (!out) return;
    out->major = 0;
    out->minor = 1;
    out->patch = 0;
    out->abi = CAELIX_ABI_VERSION;
}

CAELIX_API const char* caelix_version_string(void) { return "0.1.0-b200"; }

CAELIX_API void caelix_set_log_callback(CaelixLogCallback callback, void* user_data)
{
    std::lock_guard<std::mutex> lock(g_log_mutex);
    g_log = callback;
    g_log_user = user_data;
}

CAELIX_API CaelixResult caelix_device_create(const CaelixDeviceDesc* desc, CaelixDevice** out_device)
{
    CAELIX_GUARD_BEGIN
    if (!desc || !out_device || desc->reserved != 0) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out_device = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_device_create");
    if (desc->cuda_device < 0 || desc->cuda_device >= count) {
        log(CAELIX_LOG_ERROR, "caelix_device_create: no CUDA device %d", desc->cuda_device);
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, desc->cuda_device);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_device_create");
    if (prop.major != 10) {
        log(CAELIX_LOG_ERROR, "caelix_device_create: %s is sm_%d%d; this library is built for sm_100a",
            prop.name, prop.major, prop.minor);
        return CAELIX_ERROR_UNSUPPORTED;
    }
    e = cudaSetDevice(desc->cuda_device);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_device_create");
    CaelixDevice* d = new CaelixDevice();
    d->ordinal = desc->cuda_device;
    d->sm_count = (uint32_t)prop.multiProcessorCount;
    e = cudaMalloc(&d->status, 256);
    if (e == cudaSuccess) e = cudaMemset(d->status, 0, 256);
    if (e != cudaSuccess) {
        if (d->status) cudaFree(d->status);
        delete d;
        return cx::cuda_result(e, "caelix_device_create");
    }
    *out_device = d;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API void caelix_device_destroy(CaelixDevice* device)
{
    if (!device) return;
    cudaSetDevice(device->ordinal);
    device->sort_scratch.release();
    if (device->status) cudaFree(device->status);
    delete device;
}

CAELIX_API CaelixResult caelix_light_bvh_create(CaelixDevice* device, uint32_t leaf_capacity, CaelixLightBvh** out_bvh)
{
    CAELIX_GUARD_BEGIN
    if (!device || !out_bvh || leaf_capacity == 0 || leaf_capacity > (1u << 28)) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out_bvh = nullptr;
    cudaSetDevice(device->ordinal);
    CaelixLightBvh* b = new CaelixLightBvh();
    b->device = device;
    const uint64_t bytes = cx::lt_buffer_bytes(leaf_capacity);
    cudaError_t e = cudaMalloc(&b->memory, bytes);
    if (e != cudaSuccess) {
        delete b;
        return cx::cuda_result(e, "caelix_light_bvh_create");
    }
    b->buffers = cx::lt_carve(b->memory, leaf_capacity);
    e = cudaMemset(b->buffers.header, 0, 128);
    if (e == cudaSuccess) e = cudaEventCreate(&b->start);
    if (e == cudaSuccess) e = cudaEventCreate(&b->stop);
    if (e != cudaSuccess) {
        cudaFree(b->memory);
        delete b;
        return cx::cuda_result(e, "caelix_light_bvh_create");
    }
    *out_bvh = b;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API void caelix_light_bvh_destroy(CaelixLightBvh* bvh)
{
    if (!bvh) return;
    cudaSetDevice(bvh->device->ordinal);
    if (bvh->start) cudaEventDestroy(bvh->start);
    if (bvh->stop) cudaEventDestroy(bvh->stop);
    for (cudaEvent_t ev : bvh->stage)
        if (ev) cudaEventDestroy(ev);
    if (bvh->last_stream) cudaStreamSynchronize(bvh->last_stream);
    if (bvh->graph) cudaGraphExecDestroy(bvh->graph);
    if (bvh->capture_stream) cudaStreamDestroy(bvh->capture_stream);
    cudaFree(bvh->memory);
    delete bvh;
}

CAELIX_API CaelixResult caelix_light_bvh_build(CaelixLightBvh* bvh, const CaelixLightBvhInput* input, uint64_t stream)
{
    CAELIX_GUARD_BEGIN
    if (!bvh || !input || (input->count > 0 && !input->records) || (input->group_count > 0) != (input->group_frames != nullptr))
        return CAELIX_ERROR_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(input->records) & 15u) != 0) {
        log(CAELIX_LOG_ERROR, "caelix_light_bvh_build: records must be 16-byte aligned");
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    if (input->group_frames && !input->record_group) {
        log(CAELIX_LOG_ERROR, "caelix_light_bvh_build: group_frames needs record_group");
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    cudaSetDevice(bvh->device->ordinal);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cx::LightBvhInput in;
    in.records = reinterpret_cast<const cx::BrickLightRecord*>(input->records);
    in.count = input->count;
    in.record_group = input->record_group;
    in.record_entry = input->record_entry;
    in.group_frames = reinterpret_cast<const cx::GroupFrame*>(input->group_frames);
    in.group_count = input->group_count;
    // Profiled builds run kernel by kernel (their stage events sit between the launches); others
    // replay the graph of the same inputs, captured on first use.
    cudaError_t e = cudaSuccess;
    if (!bvh->profiling && !(bvh->graph && same_input(bvh->graph_input, in))) e = capture_build(bvh, in);
    cudaEventRecord(bvh->start, s);
    if (e == cudaSuccess) {
        if (bvh->profiling) e = cx::lt_build(bvh->buffers, in, s, bvh->stage);
        else e = cudaGraphLaunch(bvh->graph, s);
    }
    cudaEventRecord(bvh->stop, s);
    bvh->last_stream = s;
    bvh->built = true;
    bvh->profiled = bvh->profiling;
    bvh->launches = cx::lt_kernel_launches(std::min(input->count, bvh->buffers.leaf_capacity));
    return cx::cuda_result(e, "caelix_light_bvh_build");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_light_bvh_set_profiling(CaelixLightBvh* bvh, uint32_t enabled)
{
    CAELIX_GUARD_BEGIN
    if (!bvh || enabled > 1) return CAELIX_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(bvh->device->ordinal);
    if (enabled && !bvh->stage[0]) {
        for (cudaEvent_t& ev : bvh->stage) {
            const cudaError_t e = cudaEventCreate(&ev);
            if (e != cudaSuccess) return cx::cuda_result(e, "caelix_light_bvh_set_profiling");
        }
    }
    bvh->profiling = enabled != 0;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_light_bvh_get_view(const CaelixLightBvh* bvh, CaelixLightBvhView* out)
{
    if (!bvh || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    const cx::LightBvhBuffers& b = bvh->buffers;
    out->leaves = reinterpret_cast<uint64_t>(b.leaves);
    out->nodes = reinterpret_cast<uint64_t>(b.nodes);
    out->header = reinterpret_cast<uint64_t>(b.header);
    out->keys = reinterpret_cast<uint64_t>(b.keys);
    out->values = reinterpret_cast<uint64_t>(b.values);
    out->left = reinterpret_cast<uint64_t>(b.left);
    out->right = reinterpret_cast<uint64_t>(b.right);
    out->parent = reinterpret_cast<uint64_t>(b.parent);
    out->leaf_parent = reinterpret_cast<uint64_t>(b.leaf_parent);
    out->depth = reinterpret_cast<uint64_t>(b.depth);
    out->wide = reinterpret_cast<uint64_t>(b.wide);
    out->aggregates = reinterpret_cast<uint64_t>(b.aggregates);
    out->leaf_capacity = b.leaf_capacity;
    out->node_capacity = b.node_capacity;
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_light_bvh_get_stats(CaelixLightBvh* bvh, CaelixLightBvhStats* out)
{
    CAELIX_GUARD_BEGIN
    if (!bvh || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    cudaSetDevice(bvh->device->ordinal);
    if (!bvh->built) return CAELIX_OK;
    cudaError_t e = cudaStreamSynchronize(bvh->last_stream);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_light_bvh_get_stats");
    unsigned char host[128];
    e = cudaMemcpy(host, bvh->buffers.header, 128, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_light_bvh_get_stats");
    cx::LightTreeHeader h;
    cx::LightTreeState st;
    std::memcpy(&h, host, 64);
    std::memcpy(&st, host + 64, 64);
    out->leaves = h.leaf_count;
    out->nodes = h.node_count;
    out->root = h.root;
    out->builds = st.builds;
    out->leaves_found = st.leaves_found;
    out->leaves_dropped = st.leaves_dropped;
    out->node_overflow = st.node_overflow;
    out->status = st.status;
    std::memcpy(out->bounds, st.bounds, sizeof(out->bounds));
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, bvh->start, bvh->stop) == cudaSuccess) out->gpu_ms = ms;
    out->kernel_launches = bvh->launches;
    if (bvh->profiled) {
        for (int k = 0; k < cx::kBuildStages; ++k)
            if (cudaEventElapsedTime(&ms, bvh->stage[k], bvh->stage[k + 1]) == cudaSuccess) out->stage_ms[k] = ms;
    }
    return cx::status_result(st.status & ~cx::kStatusNodeOverflow, "caelix_light_bvh_build");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_radix_sort_pairs(CaelixDevice* device, uint32_t* keys, uint32_t* values, uint32_t count,
                                                uint32_t identity_values, uint64_t stream)
{
    CAELIX_GUARD_BEGIN
    if (!device || (count > 0 && (!keys || !values)) || identity_values > 1 || count >= (1u << 30))
        return CAELIX_ERROR_INVALID_ARGUMENT;
    if (count == 0) return CAELIX_OK;
    cudaSetDevice(device->ordinal);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // Scratch: ping-pong keys and values, then the onesweep words (for the tile chosen by size).
    const uint32_t kpt = cx::sort_keys_per_thread_for(count);
    const uint64_t words = 2ull * count + cx::sort_scratch_words(count, kpt);
    CaelixResult r = device->sort_scratch.reserve(words * 4, "caelix_radix_sort_pairs");
    if (r != CAELIX_OK) return r;
    uint32_t* base = static_cast<uint32_t*>(device->sort_scratch.ptr);
    uint32_t* keys_b = base;
    uint32_t* values_b = base + count;
    uint32_t* scratch = base + 2ull * count;
    cudaError_t e = cudaMemsetAsync(scratch, 0, cx::sort_scratch_words(count, kpt) * 4, s);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_radix_sort_pairs");
    const uint32_t grid = std::min<uint32_t>((count + 2047) / 2048, device->sm_count * 4);
    cx::radix_histogram(keys, count, scratch, grid, s);
    cx::onesweep_sort(keys, values, keys_b, values_b, count, identity_values != 0, scratch, device->status, s, nullptr,
                      kpt);
    e = cudaGetLastError();
    return cx::cuda_result(e, "caelix_radix_sort_pairs");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_radix_sort_pairs_wait_test(CaelixDevice* device, uint32_t* keys, uint32_t* values,
                                                          uint32_t count, uint32_t silent_tile, uint32_t spin_limit,
                                                          uint64_t stream)
{
    CAELIX_GUARD_BEGIN
    const uint32_t tiles = cx::sort_tiles(count);
    if (!device || !keys || !values || count <= cx::kSmallSortKeys || count >= (1u << 30) || silent_tile == 0 ||
        silent_tile >= tiles || spin_limit == 0 || spin_limit > cx::kSpinLimit)
        return CAELIX_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(device->ordinal);
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t words = 2ull * count + cx::sort_scratch_words(count);
    CaelixResult r = device->sort_scratch.reserve(words * 4, "caelix_radix_sort_pairs_wait_test");
    if (r != CAELIX_OK) return r;
    uint32_t* base = static_cast<uint32_t*>(device->sort_scratch.ptr);
    uint32_t* scratch = base + 2ull * count;
    cudaError_t e = cudaMemsetAsync(scratch, 0, cx::sort_scratch_words(count) * 4, s);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_radix_sort_pairs_wait_test");
    const uint32_t grid = std::min<uint32_t>((count + 2047) / 2048, device->sm_count * 4);
    cx::radix_histogram(keys, count, scratch, grid, s);
    const cx::SortWaitTest test{silent_tile, spin_limit};
    cx::onesweep_sort(keys, values, base, base + count, count, false, scratch, device->status, s, nullptr,
                      cx::kSortKeysPerThread, &test);
    return cx::cuda_result(cudaGetLastError(), "caelix_radix_sort_pairs_wait_test");
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_device_check(CaelixDevice* device, uint32_t* out_status)
{
    CAELIX_GUARD_BEGIN
    if (!device) return CAELIX_ERROR_INVALID_ARGUMENT;
    cudaSetDevice(device->ordinal);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_device_check");
    uint32_t status = 0;
    e = cudaMemcpy(&status, device->status, 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemset(device->status, 0, 4);
    if (e != cudaSuccess) return cx::cuda_result(e, "caelix_device_check");
    if (out_status) *out_status = status;
    return cx::status_result(status, "caelix_device_check");
    CAELIX_GUARD_END
}

}  // extern "C"
