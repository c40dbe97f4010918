// The trace kernel's launch interface (trace.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "scene.cuh"

namespace cx {

// One render call: the pinhole camera (caelix.h CaelixCamera, without jitter) and the lighting
// options of the path tracer.
struct TraceParams
{
    float position[3];
    float right[3];
    float up[3];
    float forward[3];
    float tan_half_fov_y;
    float aspect;
    uint32_t width;
    uint32_t height;
    uint32_t spp;           // samples per pixel: frame seeds frame_seed .. frame_seed + spp - 1, averaged
    uint32_t bounce_count;  // stochastic bounces after the primary hit
    uint32_t frame_seed;
    uint32_t light_nee;  // 1: light-tree NEE with MIS
    uint32_t* voxel_id;   // optional: width * height uint2, the camera ray's first hit (first sample)
    float voxel_id_tmax;  // hits farther than this are misses of the voxel id (0: no limit)
};

// radiance: width * height fp32 RGB; ray_counts (may be null): u64 primary, bounce, shadow rays,
// accumulated.
cudaError_t trace_launch(const SceneView& s, const TraceParams& p, float* radiance, unsigned long long* ray_counts,
                         cudaStream_t stream);

// The adjoint of a frame (backward.cu): d_radiance = dL/d(radiance), width * height RGB;
// d_albedo (kMaterialCodes x 3, per material code) and d_power (one per brick, the scene's order) are accumulated
// into (zero them first); image (may be null) receives the forward radiance; ray_counts (may be
// null) the rays of the recording pass. `memory`: adjoint_bytes(p, wave_capacity) bytes of device
// memory, 256-aligned (wave_capacity 0 = one path per pixel).
uint64_t adjoint_bytes(const TraceParams& p, uint32_t wave_capacity);
cudaError_t adjoint_launch(const SceneView& s, const TraceParams& p, const float* d_radiance, float* image,
                           float* d_albedo, float* d_power, unsigned long long* ray_counts, void* memory,
                           uint32_t wave_capacity, uint32_t sm_count, cudaStream_t stream, uint32_t* launches);

// ---- the wavefront trace (wave.cu) ----
//
// Paths live in HBM (structure of arrays, one slot per path); a wave is every pixel of one sample
// index of the views that have it, split into sub-waves of at most `capacity` slots. Per bounce
// two kernels run over compacted queues: wave_trace_kernel traces every queued ray (extension
// and shadow rays alike, one DDA code path) and wave_shade_kernel advances every live path by
// one vertex (shadow result, emission and MIS, albedo, light-tree NEE, Russian roulette),
// queueing its next rays. Each kernel is small, and its warps start full.

struct WaveView
{
    SceneView scene;
    TraceParams params;
    float* radiance;                 // width * height fp32 RGB (accumulated over the samples)
    unsigned long long* ray_counts;  // u64 primary, bounce, shadow rays of this view
    uint32_t blocks_x;               // pixel blocks per row (block_width x 32 / block_width pixels)
    uint32_t pad;
};

struct WaveBuffers
{
    uint32_t capacity = 0;  // slots
    uint32_t* item = nullptr;   // pixel index within the view (y * width + x)
    uint32_t* vs = nullptr;     // view | sample << 16
    uint32_t* flags = nullptr;
    uint32_t* rng = nullptr;
    uint32_t* light_rng = nullptr;
    float4* org = nullptr;
    float4* dir = nullptr;
    float4* throughput = nullptr;
    float4* radiance = nullptr;
    float4* seg_n = nullptr;
    float4* a0 = nullptr;    // primary albedo
    float4* e0 = nullptr;    // primary emission
    float4* sdir = nullptr;  // pending shadow ray: direction, t_max
    float4* sadd = nullptr;  // pending shadow contribution
    uint4* hit = nullptr;    // t bits, attrib (0 = miss), record, group
    uint32_t* occluded = nullptr;
    uint32_t* rayq[2] = {nullptr, nullptr};   // 2 * capacity entries: slot | kind << 30
    uint32_t* pathq[2] = {nullptr, nullptr};  // capacity entries
    uint32_t* counts = nullptr;               // [parity][2]: rays, paths; then the trace fetch counters
    // The adjoint's per-slot state (wave_adjoint): dL/dR of the sample, its radiance R, the power
    // gradient of a pending NEE lamp (brick, value; applied if its shadow ray is unoccluded).
    float4* adj_g = nullptr;
    float4* adj_r = nullptr;
    uint2* adj_nee = nullptr;
};

// The arrays of an adjoint (wave_adjoint, one view): dL/d(pixel), the radiance of every pixel
// sample (spp x width x height x 3, written by the recording pass, read by the replay), and the
// gradients (accumulated into).
struct WaveAdjoint
{
    const float* d_radiance;
    float* sample_radiance;
    float* d_albedo;  // [kMaterialCodes][3]
    float* d_power;   // [brick_count]
};

uint64_t wave_buffer_bytes(uint32_t capacity);
WaveBuffers wave_carve(void* base, uint32_t capacity);

// The wave plan of a set of views: for every sample index s below the largest spp, the views
// with spp > s and their first item (pixel blocks x 32 per view) in that wave.
struct WavePlan
{
    std::vector<uint32_t> table;     // per wave: view indices, then item bases (n_views each)
    std::vector<uint32_t> offset;    // per wave: first word of its views in `table`
    std::vector<uint32_t> views;     // per wave: number of views
    std::vector<uint32_t> items;     // per wave: items
    std::vector<uint32_t> bounces;   // per wave: the largest bounce count of its views
};
WavePlan wave_plan(const WaveView* views, uint32_t view_count, uint32_t block_width);

// Records the trace of every sample of every view into `stream` (no host synchronisation):
// d_views the device copy of `views`, d_table the device copy of plan.table. The views'
// radiance buffers receive the averaged radiance (the per-frame kernel's result, bit for bit).
// Kernel launches recorded are added to *launches (may be null).
// A single view of a scene of at most kWaveResidentBricks bricks (records about 72 MB: they stay
// in the 126 MB L2) runs the shade kernels at 5 CTAs per SM, anything larger or a batch at 8.
constexpr uint32_t kWaveResidentBricks = 65536;
cudaError_t wave_trace(const WaveView* views, const WaveView* d_views, uint32_t view_count, const WavePlan& plan,
                       const uint32_t* d_table, const WaveBuffers& b, uint32_t block_width, uint32_t sm_count,
                       cudaStream_t stream, uint32_t* launches);

// The adjoint of wave_trace for one view (path replay, sampling held fixed; backward.cu states the
// estimator and its derivative): a recording pass (the trace of d_record: radiance into its
// radiance buffer when not null, every sample's R into adj.sample_radiance), then the replay of
// every path (d_replay: the same view without radiance buffer or ray counters) gathering dL/dalbedo
// and dL/dpower. Gradients are accumulated into (zero them first).
cudaError_t wave_adjoint(const SceneView& scene, const WaveView* d_record, const WaveView* d_replay,
                         const WavePlan& plan, const uint32_t* d_table, const WaveBuffers& b, uint32_t block_width,
                         uint32_t sm_count, const WaveAdjoint& adj, cudaStream_t stream, uint32_t* launches);

// ---- the batched persistent trace (trace_batch.cu) ----

constexpr uint32_t kMaxBatchViews = 256;  // views of one persistent launch
constexpr uint32_t kBatchThreads = 128;

// One viewport of a batch, device-resident: its scene, camera and options, output and counters.
// Work items are pixels: item_base + 32 * block + lane, blocks of block_width x (32 / block_width)
// pixels in row-major order over the viewport (blocks_x per row).
struct BatchView
{
    SceneView scene;
    TraceParams params;
    float* radiance;                  // width * height fp32 RGB
    unsigned long long* ray_counts;   // u64 primary, bounce, shadow rays of this view, accumulated
    uint32_t item_base;
    uint32_t blocks_x;
};

struct BatchLaunch
{
    const BatchView* views;
    uint32_t view_count;     // <= kMaxBatchViews
    uint32_t item_count;     // total work items of the views
    uint32_t block_width;    // 8, 16 or 32
    uint32_t refill_min;     // a warp takes new pixels once this many of its lanes are idle (1..32)
    uint32_t* next_item;     // the work counter, zero before the launch
};

// The register-cap variants of the persistent kernel: `min_blocks` CTAs of 128 threads resident
// per SM (4: 128 registers, 6: 80, 8: 64).
bool trace_batch_variant_ok(uint32_t min_blocks);
// Resident CTAs per SM of a variant (the occupancy calculator), 0 for an unknown variant.
int trace_batch_blocks_per_sm(uint32_t min_blocks);
cudaError_t trace_batch_launch(const BatchLaunch& launch, uint32_t min_blocks, uint32_t grid, cudaStream_t stream);

}  // namespace cx
