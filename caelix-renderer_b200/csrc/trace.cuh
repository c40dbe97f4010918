// The trace kernel's launch interface (trace.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

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
};

// radiance: width * height fp32 RGB; ray_counts (may be null): u64 primary, bounce, shadow rays,
// accumulated.
cudaError_t trace_launch(const SceneView& s, const TraceParams& p, float* radiance, unsigned long long* ray_counts,
                         cudaStream_t stream);

// The adjoint of trace_launch (backward.cu): d_radiance = dL/d(radiance), width * height RGB;
// d_albedo (kMaterialSlots x 3) and d_power (one per brick, the scene's order) are accumulated
// into (zero them first); image (may be null) receives the forward radiance.
cudaError_t adjoint_launch(const SceneView& s, const TraceParams& p, const float* d_radiance, float* image,
                           float* d_albedo, float* d_power, unsigned long long* ray_counts, cudaStream_t stream);

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
