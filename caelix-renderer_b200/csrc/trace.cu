// The per-frame trace kernel: one thread per pixel runs the path tracer (trace_device.cuh) with
// light-tree NEE over the brick scene; the integrator loop restates
// shaders/render/caelix_path_trace.hlsl:737-978 (primary hit, NEE, bounces, MIS, Russian roulette).
#include <cstdint>

#include "trace.cuh"
#include "trace_device.cuh"

namespace cx {

namespace {

__device__ __noinline__ void next_event(const SceneView& s, const float x[3], const float n[3], uint32_t& light_rng,
                                        float out[3], Counters& rays)
{
    out[0] = out[1] = out[2] = 0.0f;
    ShadowRay r;
    if (!nee_prepare(s, x, n, light_rng, r)) return;
    ++rays.shadow;
    const Hit h = trace_scene(s, x, r.dir, 0.0f, r.t_max, true);  // occlusion only
    if (!h.hit) {
        out[0] = r.value[0];
        out[1] = r.value[1];
        out[2] = r.value[2];
    }
}

__device__ void trace_pixel(const SceneView& s, const TraceParams& P, uint32_t px, uint32_t py, uint32_t seed,
                            float rgb[3], Counters& rays)
{
    rgb[0] = rgb[1] = rgb[2] = 0.0f;
    const float sx = (float)px + 0.5f + 0.0f;
    const float sy = (float)py + 0.5f + 0.0f;
    const float ndc_x = sx / (float)P.width * 2.0f - 1.0f;
    const float ndc_y = 1.0f - sy / (float)P.height * 2.0f;
    const float a = ndc_x * P.tan_half_fov_y * P.aspect;
    const float b = ndc_y * P.tan_half_fov_y;
    float d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = P.right[k] * a + P.up[k] * b + P.forward[k];
    const float inv_len = 1.0f / sqrtf(dot3(d, d));
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = d[k] * inv_len;
    ++rays.primary;
    const Hit primary = trace_scene(s, P.position, d, 0.0f, kRayTMax);
    if (P.voxel_id && seed == P.frame_seed)
        write_voxel_id<true>(s, P, py * P.width + px, primary.hit, primary.t, primary.attrib, primary.record, primary.group);
    if (!primary.hit) return;
    uint32_t rng = init_random(px, py, seed);
    uint32_t light_rng = init_random(px, py, seed ^ 0x7F4A7C15u);
    float a0[3], e0[3], org[3], dir[3];
    shade(s, primary, P.position, d, rng, a0, e0, org, dir);
    float seg_n[3] = {primary.normal[0], primary.normal[1], primary.normal[2]};
    float radiance[3] = {0.0f, 0.0f, 0.0f};
    const float t0 = 1.0f / hmax(0.001f, 1.0f);
    float throughput[3] = {t0, t0, t0};
    uint32_t segment_light = 0;
    if (P.light_nee && P.bounce_count >= 1) {
        float nee[3];
        next_event(s, org, primary.normal, light_rng, nee, rays);
#pragma unroll
        for (int k = 0; k < 3; ++k) radiance[k] += nee[k] * throughput[k];
        segment_light = 3u;
    }
    uint32_t bounce_index = 1;
    while (bounce_index <= P.bounce_count) {
        ++rays.bounce;
        const Hit h = trace_scene(s, org, dir, 0.0f, kBounceTMax);
        if (!h.hit) break;
        float al[3], em[3], o2[3], d2[3];
        shade(s, h, org, dir, rng, al, em, o2, d2);
        bounce_index += 1;
        float ew = 1.0f;
        if (segment_light != 0u && (em[0] > 0.0f || em[1] > 0.0f || em[2] > 0.0f))
            ew = lamp_hit_weight(s, segment_light, h, org, dir, seg_n);
#pragma unroll
        for (int k = 0; k < 3; ++k) radiance[k] += em[k] * (throughput[k] * ew);
#pragma unroll
        for (int k = 0; k < 3; ++k) throughput[k] *= al[k] / hmax(0.001f, 1.0f);
        segment_light = 0u;
        if (P.light_nee && bounce_index <= P.bounce_count) {
            segment_light = 3u;
            float nee[3];
            next_event(s, o2, h.normal, light_rng, nee, rays);
#pragma unroll
            for (int k = 0; k < 3; ++k) radiance[k] += nee[k] * (throughput[k] * (1.0f / 1.0f));
        }
        const float cp = hmax(throughput[0], hmax(throughput[1], throughput[2]));
        if (cp <= 0.0f || cp < random01(rng)) break;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            throughput[k] *= 1.0f / cp;
            org[k] = o2[k];
            dir[k] = d2[k];
            seg_n[k] = h.normal[k];
        }
    }
    bool bad = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) bad |= isnan(radiance[k]) || isinf(radiance[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float sr = hmin(bad ? 0.0f : radiance[k], 65504.0f);
        rgb[k] = e0[k] + a0[k] * sr;
    }
}

// One thread per pixel; blocks of 128 threads cover 16 x 8 pixel tiles. The traversal, the light-tree
// walks and the NEE are out-of-line functions (one copy each: the megakernel's instruction footprint
// was its bound), and 8 blocks per SM cap the registers at 64.
__global__ void __launch_bounds__(128, 8) trace_kernel(const SceneView s, const TraceParams P, float* __restrict__ radiance,
                                                    unsigned long long* __restrict__ ray_counts)
{
    const uint32_t tiles_x = (P.width + 15) / 16;
    const uint32_t tile = blockIdx.x;
    const uint32_t px = (tile % tiles_x) * 16 + (threadIdx.x & 15u);
    const uint32_t py = (tile / tiles_x) * 8 + (threadIdx.x >> 4);
    Counters rays = {0, 0, 0};
    if (px < P.width && py < P.height) {
        float acc[3] = {0.0f, 0.0f, 0.0f};
        for (uint32_t sp = 0; sp < P.spp; ++sp) {
            float rgb[3];
            trace_pixel(s, P, px, py, P.frame_seed + sp, rgb, rays);
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[k] += rgb[k];
        }
        float* out = radiance + 3ull * ((uint64_t)py * P.width + px);
#pragma unroll
        for (int k = 0; k < 3; ++k) out[k] = acc[k] / (float)P.spp;
    }
    // Per-warp sums of the ray counters, one atomic per warp and counter.
    const uint32_t p = __reduce_add_sync(0xFFFFFFFFu, rays.primary);
    const uint32_t b = __reduce_add_sync(0xFFFFFFFFu, rays.bounce);
    const uint32_t sh = __reduce_add_sync(0xFFFFFFFFu, rays.shadow);
    if ((threadIdx.x & 31u) == 0 && ray_counts) {
        atomicAdd(ray_counts, (unsigned long long)p);
        atomicAdd(ray_counts + 1, (unsigned long long)b);
        atomicAdd(ray_counts + 2, (unsigned long long)sh);
    }
}

}  // namespace

cudaError_t trace_launch(const SceneView& s, const TraceParams& P, float* radiance, unsigned long long* ray_counts,
                         cudaStream_t stream)
{
    const uint32_t tiles = ((P.width + 15) / 16) * ((P.height + 7) / 8);
    if (tiles == 0) return cudaSuccess;
    trace_kernel<<<tiles, 128, 0, stream>>>(s, P, radiance, ray_counts);
    return cudaGetLastError();
}

}  // namespace cx
