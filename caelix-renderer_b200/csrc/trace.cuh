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

}  // namespace cx
