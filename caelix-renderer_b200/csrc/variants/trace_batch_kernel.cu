// The batched persistent trace kernel, compiled once per register-cap variant
// (-DCX_BATCH_MIN_BLOCKS=4, 6 or 8: that many 128-thread CTAs resident per SM). Many viewports of
// many scenes are traced by one launch of one resident CTA set (the "wavefront": every thread
// carries one path), fed from one work counter over the pixels of all views.
//
// Each thread is a small state machine over the path of one pixel sample. Every iteration of the
// loop traces exactly one ray per busy lane, from one call site, whatever the ray is for (the
// primary ray, a bounce, or the NEE shadow ray of the last vertex), then advances the path to its
// next ray. Lanes whose pixel is finished take new pixels (a warp fetches for all its idle lanes
// with one atomic once refill_min of them are idle), so a warp's lanes stay busy when paths end
// at different depths, and shadow and extension rays share the traversal instead of running it
// one after the other.
//
// The per-pixel arithmetic is the per-frame kernel's (trace.cu trace_pixel: the reference's
// shaders/render/caelix_path_trace.hlsl:737-978 integrator) in the same order, so each pixel is
// bit-identical to a plain render of its view: the NEE of a vertex is split into nee_prepare
// (the light draw, before the shadow ray) and the addition of its contribution when the shadow
// ray is found unoccluded, and no other addition to the path radiance happens in between.
#include <cstdint>

#include "../trace.cuh"
#include "../trace_device.cuh"

#ifndef CX_BATCH_MIN_BLOCKS
#error "CX_BATCH_MIN_BLOCKS must be defined (4, 6 or 8)"
#endif

#define CX_CAT2(a, b) a##b
#define CX_CAT(a, b) CX_CAT2(a, b)

namespace cx {

namespace {

enum : uint32_t
{
    kPhasePrimary = 0,
    kPhaseBounce = 1,
    kPhaseShadow = 2,
};

__global__ void __launch_bounds__(kBatchThreads, CX_BATCH_MIN_BLOCKS) trace_batch_kernel(const BatchLaunch L)
{
    __shared__ uint32_t s_base[kMaxBatchViews + 1];
    __shared__ uint32_t s_rays[kMaxBatchViews][3];
    for (uint32_t i = threadIdx.x; i < L.view_count; i += kBatchThreads) {
        s_base[i] = L.views[i].item_base;
        s_rays[i][0] = s_rays[i][1] = s_rays[i][2] = 0;
    }
    if (threadIdx.x == 0) s_base[L.view_count] = L.item_count;
    __syncthreads();

    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = lanemask_lt();
    const uint32_t bw = L.block_width;
    const uint32_t bh = 32u / bw;

    // Lane state: the view, the pixel and sample, the path.
    bool active = false;
    uint32_t view = kNone;
    const BatchView* V = nullptr;
    uint32_t px = 0, py = 0, sp = 0;
    uint32_t phase = kPhasePrimary;
    uint32_t bounce_index = 0, segment_light = 0;
    bool alive_after_shadow = false;
    uint32_t rng = 0, light_rng = 0;
    float acc[3], e0[3] = {0.0f, 0.0f, 0.0f}, a0[3], radiance[3], throughput[3], seg_n[3];
    float org[3], dir[3], sdir[3], stmax = 0.0f, sadd[3];
    Counters rays = {0, 0, 0};  // of `view`, not yet in s_rays
    bool exhausted = false;     // warp-uniform: the work counter has passed the last item

#pragma unroll
    for (int k = 0; k < 3; ++k) acc[k] = a0[k] = radiance[k] = throughput[k] = seg_n[k] = org[k] = dir[k] = sdir[k] =
        sadd[k] = 0.0f;

    // The primary ray of sample `sp` of the lane's pixel (trace_pixel's camera ray).
    auto start_sample = [&]() {
        const TraceParams& P = V->params;
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
        for (int k = 0; k < 3; ++k) {
            dir[k] = d[k] * inv_len;
            org[k] = P.position[k];
        }
        phase = kPhasePrimary;
    };

    // The end of a sample: its pixel value (trace_pixel's tail) into the accumulator; the next
    // sample, or the pixel written and the lane idle.
    auto finish_sample = [&]() {
        bool bad = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) bad |= isnan(radiance[k]) || isinf(radiance[k]);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float sr = hmin(bad ? 0.0f : radiance[k], 65504.0f);
            acc[k] += e0[k] + a0[k] * sr;
        }
        sp += 1;
        if (sp < V->params.spp) {
            start_sample();
            return;
        }
        float* out = V->radiance + 3ull * ((uint64_t)py * V->params.width + px);
        const float inv = (float)V->params.spp;
#pragma unroll
        for (int k = 0; k < 3; ++k) out[k] = acc[k] / inv;
        active = false;
    };

    // After the vertex's NEE (if any): the next bounce ray, or the end of the sample.
    auto continue_path = [&]() {
        if (bounce_index <= V->params.bounce_count) phase = kPhaseBounce;
        else finish_sample();
    };

    while (true) {
        // Refill idle lanes with the next pixels.
        const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !active);
        if (!exhausted && idle != 0u && (idle == 0xFFFFFFFFu || (uint32_t)__popc(idle) >= L.refill_min)) {
            const uint32_t want = (uint32_t)__popc(idle);
            const uint32_t leader = (uint32_t)__ffs(idle) - 1u;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(L.next_item, want);
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            if (base + want >= L.item_count) exhausted = true;
            if (!active) {
                const uint32_t item = base + (uint32_t)__popc(idle & lt);
                if (item < L.item_count) {
                    // The view of the item: the last view whose first item is <= item.
                    uint32_t lo = 0, hi = L.view_count;
                    while (hi - lo > 1u) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (s_base[mid] <= item) lo = mid;
                        else hi = mid;
                    }
                    if (lo != view) {
                        if (view != kNone) {
                            atomicAdd(&s_rays[view][0], rays.primary);
                            atomicAdd(&s_rays[view][1], rays.bounce);
                            atomicAdd(&s_rays[view][2], rays.shadow);
                        }
                        rays = {0, 0, 0};
                        view = lo;
                        V = L.views + lo;
                    }
                    const uint32_t local = item - s_base[lo];
                    const uint32_t blk = local >> 5;
                    const uint32_t in = local & 31u;
                    const uint32_t bx = blk % V->blocks_x;
                    const uint32_t by = blk / V->blocks_x;
                    px = bx * bw + in % bw;
                    py = by * bh + in / bw;
                    if (px < V->params.width && py < V->params.height) {
                        active = true;
                        sp = 0;
                        acc[0] = acc[1] = acc[2] = 0.0f;
                        start_sample();
                    }
                }
            }
        }
        if (!__any_sync(0xFFFFFFFFu, active)) {
            if (exhausted) break;
            continue;
        }
        if (!active) continue;

        // One ray.
        const SceneView& S = V->scene;
        const TraceParams& P = V->params;
        const float t_max = phase == kPhasePrimary ? kRayTMax : (phase == kPhaseShadow ? stmax : kBounceTMax);
        if (phase == kPhasePrimary) ++rays.primary;
        else if (phase == kPhaseBounce) ++rays.bounce;
        else ++rays.shadow;
        // Copies for the out-of-line calls (the state arrays stay in registers).
        float ray_o[3], ray_d[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            ray_o[k] = org[k];
            ray_d[k] = phase == kPhaseShadow ? sdir[k] : dir[k];
        }
        const Hit h = trace_ray(S, ray_o, ray_d, 0.0f, t_max);
        if (phase == kPhasePrimary && sp == 0 && P.voxel_id)
            write_voxel_id<false>(S, P, py * P.width + px, h.hit, h.t, h.attrib, h.record, h.group);

        if (phase == kPhaseShadow) {
            if (!h.hit) {
#pragma unroll
                for (int k = 0; k < 3; ++k) radiance[k] += sadd[k];
            }
            if (alive_after_shadow) continue_path();
            else finish_sample();
            continue;
        }
        const bool primary = phase == kPhasePrimary;
        if (!h.hit) {
            if (primary) {  // the sample's value is 0
#pragma unroll
                for (int k = 0; k < 3; ++k) e0[k] = a0[k] = radiance[k] = 0.0f;
            }
            finish_sample();
            continue;
        }
        const uint32_t seed = P.frame_seed + sp;
        if (primary) {
            rng = init_random(px, py, seed);
            light_rng = init_random(px, py, seed ^ 0x7F4A7C15u);
        }
        float al[3], em[3], o2[3], d2[3];
        shade<false>(S, h, org, dir, rng, al, em, o2, d2);  // batched scenes have no entities
        bool nee_now;
        if (primary) {
            const float t0 = 1.0f / hmax(0.001f, 1.0f);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                e0[k] = em[k];
                a0[k] = al[k];
                radiance[k] = 0.0f;
                throughput[k] = t0;
            }
            segment_light = 0;
            bounce_index = 1;
            nee_now = P.light_nee && P.bounce_count >= 1;
        } else {
            bounce_index += 1;
            float ew = 1.0f;
            if (segment_light != 0u && (em[0] > 0.0f || em[1] > 0.0f || em[2] > 0.0f)) {
                float n_prev[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) n_prev[k] = seg_n[k];
                ew = lamp_hit_weight(S, segment_light, h, ray_o, ray_d, n_prev);
            }
#pragma unroll
            for (int k = 0; k < 3; ++k) radiance[k] += em[k] * (throughput[k] * ew);
#pragma unroll
            for (int k = 0; k < 3; ++k) throughput[k] *= al[k] / hmax(0.001f, 1.0f);
            segment_light = 0u;
            nee_now = P.light_nee && bounce_index <= P.bounce_count;
        }
        bool shadow = false;
        if (nee_now) {
            segment_light = 3u;
            ShadowRay r;
            shadow = nee_prepare<false>(S, o2, h.normal, light_rng, r);
            if (shadow) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    sdir[k] = r.dir[k];
                    sadd[k] = r.value[k] * throughput[k];
                }
                stmax = r.t_max;
            }
        }
        bool alive = true;
        if (!primary) {
            const float cp = hmax(throughput[0], hmax(throughput[1], throughput[2]));
            alive = !(cp <= 0.0f || cp < random01(rng));
            if (alive) {
#pragma unroll
                for (int k = 0; k < 3; ++k) throughput[k] *= 1.0f / cp;
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            org[k] = o2[k];  // the shadow ray's origin and the next bounce's
            if (alive) {
                dir[k] = d2[k];
                seg_n[k] = h.normal[k];
            }
        }
        alive_after_shadow = alive;
        if (shadow) phase = kPhaseShadow;
        else if (alive) continue_path();
        else finish_sample();
    }

    if (view != kNone) {
        atomicAdd(&s_rays[view][0], rays.primary);
        atomicAdd(&s_rays[view][1], rays.bounce);
        atomicAdd(&s_rays[view][2], rays.shadow);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < L.view_count; i += kBatchThreads) {
#pragma unroll
        for (int k = 0; k < 3; ++k)
            if (s_rays[i][k]) atomicAdd(L.views[i].ray_counts + k, (unsigned long long)s_rays[i][k]);
    }
}

}  // namespace

int CX_CAT(trace_batch_blocks_per_sm_b, CX_BATCH_MIN_BLOCKS)()
{
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, trace_batch_kernel, kBatchThreads, 0) != cudaSuccess)
        return 0;
    return blocks;
}

cudaError_t CX_CAT(trace_batch_launch_b, CX_BATCH_MIN_BLOCKS)(const BatchLaunch& launch, uint32_t grid,
                                                              cudaStream_t stream)
{
    trace_batch_kernel<<<grid, kBatchThreads, 0, stream>>>(launch);
    return cudaGetLastError();
}

}  // namespace cx
