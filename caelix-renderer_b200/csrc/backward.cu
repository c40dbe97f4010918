// The adjoint of the trace (path replay): gradients of an image loss with respect to the albedo
// of every material and the emitter power of every brick.
//
// The forward estimator is the per-frame kernel's (trace.cu trace_pixel, the reference's
// shaders/render/caelix_path_trace.hlsl:737-978 integrator). Its parameter-dependent factors are
//   * the primary albedo a0 and emission e0: pixel sample = e0 + a0 * sanitize(R);
//   * the albedo of every bounce vertex, a factor of the throughput of everything after it;
//   * the power of every emitting brick the path reaches: an emitter hit adds
//     power * throughput * w_mis, an NEE vertex adds power * s * throughput (s: the geometry,
//     pdf and MIS factors of the light sample).
// The sampling quantities (pdfs, MIS weights, Russian-roulette probabilities, every discrete
// decision) are held fixed (detached), so a sample is a polynomial in the parameters and
//   dL/da0[c]          = g[c] * sanitize(R)[c]
//   dL/de0             = g[0] + g[1] + g[2]
//   dL/dR[c]           = G[c] = g[c] * a0[c] (0 where sanitize clamps)
//   dL/dalbedo_j[c]    = G[c] * (R[c] - R_before_j[c]) / albedo_j[c]
//   dL/dpower_b        = sum_c G[c] * (throughput[c] * w_mis  or  s * throughput[c])
// with g = dL/d(pixel) / spp and R_before_j the radiance gathered before vertex j's albedo
// multiplies the throughput. Each thread runs a pixel's samples twice: once to get R (the
// forward pass, bit-identical to trace_pixel), once more (the replay) to gather the gradients;
// nothing of the path is stored. Albedo gradients are summed per CTA in shared memory, power
// gradients with global atomics.
#include <cstdint>

#include "trace.cuh"
#include "trace_device.cuh"

namespace cx {

namespace {

struct Grad
{
    float* albedo;  // shared: [kMaterialSlots][3]
    float* power;   // global: [brick_count]
    float G[3];     // dL/dR of the sample
    float R[3];     // the sample's radiance from the forward pass
};

struct Sample
{
    bool hit;
    float radiance[3];
    float rgb[3];
    float a0[3];
    uint32_t material0;
    uint32_t record0;
    bool emits0;  // the primary emission is the primary brick's power
};

__device__ __forceinline__ float gsum3(const float G[3], const float t[3], float s)
{
    return G[0] * (t[0] * s) + G[1] * (t[1] * s) + G[2] * (t[2] * s);
}

// One path sample: the forward pass (kReplay false) or the replay that gathers the gradients
// (kReplay true, gr set). The arithmetic of the estimator is trace_pixel's, operation for
// operation.
template <bool kReplay>
__device__ __forceinline__ void path_sample(const SceneView& s, const TraceParams& P, uint32_t px, uint32_t py,
                                            uint32_t seed, Sample& out, Counters& rays, Grad* gr)
{
    out.hit = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) out.radiance[k] = out.rgb[k] = out.a0[k] = 0.0f;
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
    if (!kReplay) ++rays.primary;
    float cam[3] = {P.position[0], P.position[1], P.position[2]};
    const Hit primary = trace_ray(s, cam, d, 0.0f, kRayTMax);
    if (!primary.hit) return;
    out.hit = true;
    uint32_t rng = init_random(px, py, seed);
    uint32_t light_rng = init_random(px, py, seed ^ 0x7F4A7C15u);
    float a0[3], e0, org[3], dir[3];
    shade(s, primary, cam, d, rng, a0, e0, org, dir);
    const uint32_t block0 = (primary.attrib >> 16) & 0xFFFFu;
    out.material0 = block0 & (kMaterialSlots - 1);
    out.record0 = primary.record;
    out.emits0 = (block0 & kOpaqueBit) != 0;
    float seg_n[3] = {primary.normal[0], primary.normal[1], primary.normal[2]};
    float radiance[3] = {0.0f, 0.0f, 0.0f};
    const float t0 = 1.0f / hmax(0.001f, 1.0f);
    float throughput[3] = {t0, t0, t0};
    uint32_t segment_light = 0;
    if (P.light_nee && P.bounce_count >= 1) {
        ShadowRay r;
        float nee = 0.0f;
        if (nee_prepare(s, org, primary.normal, light_rng, r)) {
            if (!kReplay) ++rays.shadow;
            const Hit h = trace_ray(s, org, r.dir, 0.0f, r.t_max);
            if (!h.hit) {
                nee = r.value;
                if (kReplay && r.brick != kNone) atomicAdd(gr->power + r.brick, gsum3(gr->G, throughput, r.dvalue_de));
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) radiance[k] += nee * throughput[k];
        segment_light = 3u;
    }
    uint32_t bounce_index = 1;
    while (bounce_index <= P.bounce_count) {
        if (!kReplay) ++rays.bounce;
        const Hit h = trace_ray(s, org, dir, 0.0f, kBounceTMax);
        if (!h.hit) break;
        float al[3], em, o2[3], d2[3];
        shade(s, h, org, dir, rng, al, em, o2, d2);
        bounce_index += 1;
        float ew = 1.0f;
        if (segment_light != 0u && em > 0.0f) ew = lamp_hit_weight(s, segment_light, h, org, dir, seg_n);
#pragma unroll
        for (int k = 0; k < 3; ++k) radiance[k] += em * (throughput[k] * ew);
        const uint32_t block = (h.attrib >> 16) & 0xFFFFu;
        if (kReplay) {
            if (block & kOpaqueBit) atomicAdd(gr->power + h.record, gsum3(gr->G, throughput, ew));
            // Everything gathered from here on carries this vertex's albedo as a factor.
            float* ga = gr->albedo + 3 * (block & (kMaterialSlots - 1));
#pragma unroll
            for (int k = 0; k < 3; ++k)
                if (al[k] > 0.0f && gr->G[k] != 0.0f) atomicAdd(ga + k, gr->G[k] * (gr->R[k] - radiance[k]) / al[k]);
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) throughput[k] *= al[k] / hmax(0.001f, 1.0f);
        segment_light = 0u;
        if (P.light_nee && bounce_index <= P.bounce_count) {
            segment_light = 3u;
            ShadowRay r;
            float nee = 0.0f;
            if (nee_prepare(s, o2, h.normal, light_rng, r)) {
                if (!kReplay) ++rays.shadow;
                const Hit hs = trace_ray(s, o2, r.dir, 0.0f, r.t_max);
                if (!hs.hit) {
                    nee = r.value;
                    if (kReplay && r.brick != kNone)
                        atomicAdd(gr->power + r.brick, gsum3(gr->G, throughput, r.dvalue_de));
                }
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) radiance[k] += nee * (throughput[k] * (1.0f / 1.0f));
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
        out.rgb[k] = e0 + a0[k] * sr;
        out.radiance[k] = radiance[k];
        out.a0[k] = a0[k];
    }
}

// One thread per pixel, 16 x 8 pixel tiles (trace_kernel's layout).
__global__ void __launch_bounds__(128, 4)
    adjoint_kernel(const SceneView s, const TraceParams P, const float* __restrict__ d_radiance,
                   float* __restrict__ image, float* __restrict__ d_albedo, float* __restrict__ d_power,
                   unsigned long long* __restrict__ ray_counts)
{
    __shared__ float s_albedo[kMaterialSlots * 3];
    for (uint32_t i = threadIdx.x; i < kMaterialSlots * 3; i += blockDim.x) s_albedo[i] = 0.0f;
    __syncthreads();
    const uint32_t tiles_x = (P.width + 15) / 16;
    const uint32_t tile = blockIdx.x;
    const uint32_t px = (tile % tiles_x) * 16 + (threadIdx.x & 15u);
    const uint32_t py = (tile / tiles_x) * 8 + (threadIdx.x >> 4);
    Counters rays = {0, 0, 0};
    if (px < P.width && py < P.height) {
        const uint64_t pix = (uint64_t)py * P.width + px;
        float g[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) g[k] = d_radiance[3 * pix + k] / (float)P.spp;
        float acc[3] = {0.0f, 0.0f, 0.0f};
        for (uint32_t sp = 0; sp < P.spp; ++sp) {
            Sample fw;
            path_sample<false>(s, P, px, py, P.frame_seed + sp, fw, rays, nullptr);
#pragma unroll
            for (int k = 0; k < 3; ++k) acc[k] += fw.rgb[k];
            if (!fw.hit) continue;
            bool bad = false;
#pragma unroll
            for (int k = 0; k < 3; ++k) bad |= isnan(fw.radiance[k]) || isinf(fw.radiance[k]);
            Grad gr;
            gr.albedo = s_albedo;
            gr.power = d_power;
            bool any = false;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float sr = hmin(bad ? 0.0f : fw.radiance[k], 65504.0f);
                atomicAdd(s_albedo + 3 * fw.material0 + k, g[k] * sr);
                const bool pass = !bad && fw.radiance[k] <= 65504.0f;
                gr.G[k] = pass ? g[k] * fw.a0[k] : 0.0f;
                gr.R[k] = fw.radiance[k];
                any |= gr.G[k] != 0.0f;
            }
            if (fw.emits0) atomicAdd(d_power + fw.record0, g[0] + g[1] + g[2]);
            if (any) {
                Sample rp;
                path_sample<true>(s, P, px, py, P.frame_seed + sp, rp, rays, &gr);
            }
        }
        if (image) {
#pragma unroll
            for (int k = 0; k < 3; ++k) image[3 * pix + k] = acc[k] / (float)P.spp;
        }
    }
    const uint32_t p = __reduce_add_sync(0xFFFFFFFFu, rays.primary);
    const uint32_t b = __reduce_add_sync(0xFFFFFFFFu, rays.bounce);
    const uint32_t sh = __reduce_add_sync(0xFFFFFFFFu, rays.shadow);
    if ((threadIdx.x & 31u) == 0 && ray_counts) {
        atomicAdd(ray_counts, (unsigned long long)p);
        atomicAdd(ray_counts + 1, (unsigned long long)b);
        atomicAdd(ray_counts + 2, (unsigned long long)sh);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kMaterialSlots * 3; i += blockDim.x)
        if (s_albedo[i] != 0.0f) atomicAdd(d_albedo + i, s_albedo[i]);
}

}  // namespace

cudaError_t adjoint_launch(const SceneView& s, const TraceParams& p, const float* d_radiance, float* image,
                           float* d_albedo, float* d_power, unsigned long long* ray_counts, cudaStream_t stream)
{
    const uint32_t tiles = ((p.width + 15) / 16) * ((p.height + 7) / 8);
    if (tiles == 0) return cudaSuccess;
    adjoint_kernel<<<tiles, 128, 0, stream>>>(s, p, d_radiance, image, d_albedo, d_power, ray_counts);
    return cudaGetLastError();
}

}  // namespace cx
