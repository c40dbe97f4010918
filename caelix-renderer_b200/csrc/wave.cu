// The wavefront trace (trace.cuh): path state in HBM, one kernel per stage over compacted queues.
//
// Stages of one sub-wave (a range of the pixels of one sample index):
//   wave_generate_kernel  one slot per pixel: the camera ray (trace_pixel's), queued;
//   then bounce_count + 1 times:
//   wave_trace_kernel     every queued ray: the closest hit (extension rays) or occlusion (shadow
//                         rays) through the brick-grid DDA, written to the slot;
//   wave_shade_kernel     every live path: its shadow result, then its vertex (the per-frame
//                         kernel's integrator step: emission with MIS, albedo, light-tree NEE,
//                         Russian roulette), queueing its shadow ray and its next extension ray;
//                         a finished path adds its sample to the pixel (the last sample divides).
// A path's arithmetic is trace_pixel's in the same order (the shadow contribution of a vertex is
// added before anything of the next vertex), so the radiance is the per-frame kernel's, bit for
// bit. Queues are compacted with warp-aggregated atomics; every kernel reads its queue length on
// the device, so a whole frame is recorded without a host synchronisation (graph-capturable).
#include <algorithm>
#include <cstdint>

#include "trace.cuh"
#include "trace_device.cuh"

namespace cx {

namespace {

constexpr uint32_t kWaveThreads = 128;
constexpr uint32_t kKindPrimary = 0, kKindBounce = 1, kKindShadow = 2;
constexpr uint32_t kSlotMask = 0x3FFFFFFFu;
constexpr uint32_t kFlagBounce = 0xFFu;       // bounce_index
constexpr uint32_t kFlagSegLight = 1u << 8;   // segment_light = 3
constexpr uint32_t kFlagShadow = 1u << 9;     // a shadow ray of the last vertex was queued
constexpr uint32_t kFlagExt = 1u << 10;       // an extension ray was queued
constexpr uint32_t kFlagPrimary = 1u << 11;   // that extension ray is the camera ray
// Words of WaveBuffers::counts: 0..3 the queue lengths of the two parities (rays, paths), then
// the trace and shade launches' fetch counters of the two parities.
constexpr uint32_t kFetchTrace = 4, kFetchShade = 6;

// The next 32-item chunk of a queue for the calling warp, from a fetch counter. A warp that is done
// with its chunk takes the next one, so the work of a launch whose items' costs differ widely
// spreads over the warps until its end. Every lane calls.
__device__ __forceinline__ uint32_t fetch_chunk(uint32_t* counter)
{
    uint32_t base = 0;
    if ((threadIdx.x & 31u) == 0) base = atomicAdd(counter, 32u);
    return __shfl_sync(0xFFFFFFFFu, base, 0);
}

struct WaveGen
{
    const uint32_t* table;  // view indices, then item bases (n_views each)
    uint32_t n_views;
    uint32_t sample;
    uint32_t first_item;
    uint32_t count;
    uint32_t block_width;
};

// Warp-aggregated append: returns this lane's first index in the queue. All lanes of the warp call.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, uint32_t n)
{
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t incl = n;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, incl, d);
        if (lane >= d) incl += t;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    uint32_t base = 0;
    if (lane == 0 && total) base = atomicAdd(counter, total);
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    return base + incl - n;
}

__global__ void __launch_bounds__(kWaveThreads)
    wave_generate_kernel(const WaveView* __restrict__ views, const WaveGen g, const WaveBuffers b)
{
    const uint32_t i = blockIdx.x * kWaveThreads + threadIdx.x;
    const uint32_t bw = g.block_width, bh = 32u / bw;
    bool valid = false;
    if (i < g.count) {
        const uint32_t item = g.first_item + i;
        const uint32_t* bases = g.table + g.n_views;
        uint32_t lo = 0, hi = g.n_views;
        while (hi - lo > 1u) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(bases + mid) <= item) lo = mid;
            else hi = mid;
        }
        const uint32_t v = __ldg(g.table + lo);
        const WaveView& V = views[v];
        const TraceParams& P = V.params;
        const uint32_t local = item - __ldg(bases + lo);
        const uint32_t blk = local >> 5, in = local & 31u;
        const uint32_t px = (blk % V.blocks_x) * bw + in % bw;
        const uint32_t py = (blk / V.blocks_x) * bh + in / bw;
        if (px < P.width && py < P.height) {
            valid = true;
            const float sx = (float)px + 0.5f + 0.0f;
            const float sy = (float)py + 0.5f + 0.0f;
            const float ndc_x = sx / (float)P.width * 2.0f - 1.0f;
            const float ndc_y = 1.0f - sy / (float)P.height * 2.0f;
            const float a = ndc_x * P.tan_half_fov_y * P.aspect;
            const float bb = ndc_y * P.tan_half_fov_y;
            float d[3];
#pragma unroll
            for (int k = 0; k < 3; ++k) d[k] = P.right[k] * a + P.up[k] * bb + P.forward[k];
            const float inv_len = 1.0f / sqrtf(dot3(d, d));
#pragma unroll
            for (int k = 0; k < 3; ++k) d[k] = d[k] * inv_len;
            b.item[i] = py * P.width + px;
            b.vs[i] = v | (g.sample << 16);
            b.flags[i] = kFlagExt | kFlagPrimary;
            b.org[i] = make_float4(P.position[0], P.position[1], P.position[2], 0.0f);
            b.dir[i] = make_float4(d[0], d[1], d[2], 0.0f);
        }
    }
    const uint32_t q = warp_append(&b.counts[1], valid ? 1u : 0u);
    const uint32_t r = warp_append(&b.counts[0], valid ? 1u : 0u);
    if (valid) {
        b.pathq[0][q] = i;
        b.rayq[0][r] = i | (kKindPrimary << 30);
    }
}

// kEntities: the views' scenes have entities (traversed after the world's bricks); the variant
// without them keeps the world-only DDA's registers (no out-of-line call). kDynamic: warps take
// chunks of the queue from a fetch counter (fetch_chunk) instead of a fixed grid stride: faster
// where ray costs spread widely (entities, scenes whose records do not stay in L2), slower on the
// small resident scene, where the fixed stride is kept.
template <bool kEntities, bool kDynamic>
__global__ void __launch_bounds__(kWaveThreads)
    wave_trace_kernel(const WaveView* __restrict__ views, const WaveBuffers b, uint32_t parity)
{
    const uint32_t n = *(volatile uint32_t*)&b.counts[2 * parity];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        b.counts[2 * (parity ^ 1u)] = 0;
        b.counts[2 * (parity ^ 1u) + 1] = 0;
        b.counts[kFetchTrace + (parity ^ 1u)] = 0;  // the next trace launch's fetch counter
    }
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * kWaveThreads;
    uint32_t* const fetch = &b.counts[kFetchTrace + parity];
    for (uint32_t base = kDynamic ? fetch_chunk(fetch) : blockIdx.x * kWaveThreads + (threadIdx.x & ~31u); base < n;
         base = kDynamic ? fetch_chunk(fetch) : base + stride) {
        const uint32_t i = base + lane;
        uint32_t key = 0xFFFFFFFFu;
        if (i < n) {
            const uint32_t e = b.rayq[parity][i];
            const uint32_t slot = e & kSlotMask, kind = e >> 30;
            const uint32_t v = b.vs[slot] & 0xFFFFu;
            const float4 o4 = b.org[slot];
            const float4 d4 = kind == kKindShadow ? b.sdir[slot] : b.dir[slot];
            const float o[3] = {o4.x, o4.y, o4.z};
            const float d[3] = {d4.x, d4.y, d4.z};
            const float t_max = kind == kKindShadow ? d4.w : (kind == kKindPrimary ? kRayTMax : kBounceTMax);
            Hit h;
            if constexpr (kEntities) h = trace_scene_body(views[v].scene, o, d, 0.0f, t_max, kind == kKindShadow);
            else h = trace_ray_body(views[v].scene, o, d, 0.0f, t_max);
            if (kind == kKindShadow) b.occluded[slot] = h.hit ? 1u : 0u;
            else b.hit[slot] = h.hit ? make_uint4(__float_as_uint(h.t), h.attrib, h.record, h.group) : make_uint4(0, 0, 0, 0);
            key = v * 4u + kind;
        }
        // Ray counters: one atomic per (view, kind) group of the warp.
        const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
        if (key != 0xFFFFFFFFu && lane == (uint32_t)__ffs(peers) - 1u) {
            unsigned long long* counts = views[key >> 2].ray_counts;
            if (counts) atomicAdd(counts + (key & 3u), (unsigned long long)__popc(peers));
        }
    }
}

// kMode: kShadeRender (the render), kShadeRecord (the adjoint's recording pass: also every
// sample's radiance R), kShadeReplay (the adjoint's replay: the gradients, no image).
enum : int
{
    kShadeRender = 0,
    kShadeRecord = 1,
    kShadeReplay = 2,
};

// sum_c G[c] (t[c] s) e[c]: the power gradient of an emission e * P gathered with throughput t and
// weight s (e the material emission without the power).
__device__ __forceinline__ float gsum3(const float G[3], const float t[3], float s, const float e[3])
{
    return G[0] * ((t[0] * s) * e[0]) + G[1] * ((t[1] * s) * e[1]) + G[2] * ((t[2] * s) * e[2]);
}

// The replay's albedo gradients per material code: a CTA sums them in shared memory, in a table of
// kAlbedoCache entries indexed by the code's low bits (the first code to reach an entry owns it; a
// code whose entry another code owns goes to global memory directly), added to the global
// gradients once at the end of the CTA.
constexpr uint32_t kAlbedoCache = 128;
struct AlbedoCache
{
    uint32_t* tag;
    float* sum;
    float* global;
    __device__ __forceinline__ void add(uint32_t code, uint32_t c, float v)
    {
        const uint32_t e = code & (kAlbedoCache - 1u);
        uint32_t owner = tag[e];
        if (owner == kNone) {
            const uint32_t old = atomicCAS(tag + e, kNone, code);
            owner = old == kNone ? code : old;
        }
        if (owner == code) atomicAdd(sum + 3 * e + c, v);
        else atomicAdd(global + 3ull * code + c, v);
    }
};

// kMinBlocks CTAs of 128 threads per SM: 5 (96 registers, few spills) for a scene whose records
// stay in L2, 8 (64 registers) where the descent and the record loads go to HBM and more warps
// in flight hide them (measured: 5 is the fastest of 3 .. 8 on the 128^3 world; 8 on the
// 2 M-brick world and the 64-scene batch).
// kEntities: the views' scenes have entities (their hits, their lights); the variant without
// them keeps the world-only shading's registers.
template <int kMode, int kMinBlocks, bool kEntities>
__global__ void __launch_bounds__(kWaveThreads, kMinBlocks)
    wave_shade_kernel(const WaveView* __restrict__ views, const WaveBuffers b, uint32_t parity, const WaveAdjoint adj)
{
    __shared__ float s_albedo[kMode == kShadeReplay ? kAlbedoCache * 3 : 1];
    __shared__ uint32_t s_tag[kMode == kShadeReplay ? kAlbedoCache : 1];
    AlbedoCache cache{s_tag, s_albedo, adj.d_albedo};
    if (kMode == kShadeReplay) {
        for (uint32_t i = threadIdx.x; i < kAlbedoCache * 3; i += kWaveThreads) s_albedo[i] = 0.0f;
        for (uint32_t i = threadIdx.x; i < kAlbedoCache; i += kWaveThreads) s_tag[i] = kNone;
        __syncthreads();
    }
    const uint32_t n = *(volatile uint32_t*)&b.counts[2 * parity + 1];
    const uint32_t out = parity ^ 1u;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * kWaveThreads;
    if (blockIdx.x == 0 && threadIdx.x == 0) b.counts[kFetchShade + out] = 0;  // the next shade launch's
    // Chunks from a fetch counter (as in wave_trace_kernel) for scenes with entities or records that
    // do not stay in L2 (the 8-CTA variants); the fixed stride for the resident scene.
    constexpr bool kDynamic = kEntities || kMinBlocks == 8;
    uint32_t* const fetch = &b.counts[kFetchShade + parity];
    for (uint32_t base = kDynamic ? fetch_chunk(fetch) : blockIdx.x * kWaveThreads + (threadIdx.x & ~31u); base < n;
         base = kDynamic ? fetch_chunk(fetch) : base + stride) {
        const uint32_t i = base + lane;
        uint32_t slot = 0, next_flags = 0;
        bool live = false, shadow = false, ext = false;
        if (i < n) {
            slot = b.pathq[parity][i];
            const uint32_t f = b.flags[slot];
            const uint32_t vs = b.vs[slot];
            const WaveView& V = views[vs & 0xFFFFu];
            const SceneView& S = V.scene;
            const TraceParams& P = V.params;
            const uint32_t sp = vs >> 16;
            const uint32_t item = b.item[slot];
            const bool primary = (f & kFlagPrimary) != 0;
            float rad[3] = {0.0f, 0.0f, 0.0f};
            if (!primary) {
                const float4 r4 = b.radiance[slot];
                rad[0] = r4.x;
                rad[1] = r4.y;
                rad[2] = r4.z;
            }
            if ((f & kFlagShadow) && !b.occluded[slot]) {
                const float4 s4 = b.sadd[slot];
                rad[0] += s4.x;
                rad[1] += s4.y;
                rad[2] += s4.z;
                if (kMode == kShadeReplay) {
                    const uint2 pn = b.adj_nee[slot];  // the lamp's power gradient, now unoccluded
                    if (pn.x != kNone) atomicAdd(adj.d_power + pn.x, __uint_as_float(pn.y));
                }
            }
            float G[3] = {0.0f, 0.0f, 0.0f}, R[3] = {0.0f, 0.0f, 0.0f};
            if (kMode == kShadeReplay && !primary) {
                const float4 g4 = b.adj_g[slot];
                const float4 r4 = b.adj_r[slot];
                G[0] = g4.x;
                G[1] = g4.y;
                G[2] = g4.z;
                R[0] = r4.x;
                R[1] = r4.y;
                R[2] = r4.z;
            }
            bool finish = true, zero = false;
            float e0[3] = {0.0f, 0.0f, 0.0f}, a0[3] = {0.0f, 0.0f, 0.0f};
            if (!primary) {
                const float4 a4 = b.a0[slot];
                const float4 e4 = b.e0[slot];
                a0[0] = a4.x;
                a0[1] = a4.y;
                a0[2] = a4.z;
                e0[0] = e4.x;
                e0[1] = e4.y;
                e0[2] = e4.z;
            }
            if (f & kFlagExt) {
                const uint4 hw = b.hit[slot];
                if (kMode != kShadeReplay && primary && sp == 0 && P.voxel_id)
                    write_voxel_id<kEntities>(S, P, item, hw.y != 0u, __uint_as_float(hw.x), hw.y, hw.z, hw.w);
                const float4 o4 = b.org[slot];
                const float4 d4 = b.dir[slot];
                const float org[3] = {o4.x, o4.y, o4.z};
                const float dir[3] = {d4.x, d4.y, d4.z};
                if (hw.y == 0u) {
                    zero = primary;  // a missed camera ray: the sample is 0
                } else {
                    Hit h;
                    h.hit = true;
                    h.t = __uint_as_float(hw.x);
                    h.attrib = hw.y;
                    h.record = hw.z;
                    h.group = hw.w;
                    const uint32_t fc = (uint32_t)(__ffs(h.attrib & 0x3Fu) - 1);
                    h.normal[0] = fc == 0 ? 1.0f : (fc == 1 ? -1.0f : 0.0f);
                    h.normal[1] = fc == 2 ? 1.0f : (fc == 3 ? -1.0f : 0.0f);
                    h.normal[2] = fc == 4 ? 1.0f : (fc == 5 ? -1.0f : 0.0f);
#pragma unroll
                    for (int k = 0; k < 3; ++k) h.object_hit[k] = org[k] + dir[k] * h.t;
                    if constexpr (kEntities) {
                        if (h.attrib & kEntityHit) {
                            entity_normal(S, h.group >> kEntityShift, h.attrib, h.normal);
                            entity_local_hit(S, h.group >> kEntityShift, org, dir, h.t, h.object_hit);
                        }
                    }
                    const uint32_t px = item % P.width, py = item / P.width;
                    const uint32_t seed = P.frame_seed + sp;
                    uint32_t rng, light_rng;
                    if (primary) {
                        rng = init_random(px, py, seed);
                        light_rng = init_random(px, py, seed ^ 0x7F4A7C15u);
                    } else {
                        rng = b.rng[slot];
                        light_rng = b.light_rng[slot];
                    }
                    float tp[3], seg_n[3];
                    uint32_t bounce_index, seg_light;
                    float al[3], em[3], o2[3], d2[3];
                    shade<kEntities>(S, h, org, dir, rng, al, em, o2, d2);
                    const uint32_t block = (h.attrib >> 16) & 0xFFFFu;
                    // The replay's power gradients need the material emission without the power.
                    float me[3] = {0.0f, 0.0f, 0.0f};
                    if (kMode == kShadeReplay) {
                        float ma[3];
                        material_of(S, block, ma, me);
                    }
                    bool nee_now;
                    if (primary) {
                        const float t0 = 1.0f / hmax(0.001f, 1.0f);
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            e0[k] = em[k];
                            a0[k] = al[k];
                            rad[k] = 0.0f;
                            tp[k] = t0;
                        }
                        seg_light = 0;
                        bounce_index = 1;
                        nee_now = P.light_nee && P.bounce_count >= 1;
                        if (kMode == kShadeReplay) {
                            // The sample's value e0 + a0 * sanitize(R), R from the recording pass.
                            const float* rs = adj.sample_radiance + 3ull * ((uint64_t)sp * P.width * P.height + item);
                            bool bad = false;
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                R[k] = rs[k];
                                bad |= isnan(R[k]) || isinf(R[k]);
                            }
                            const uint32_t code0 = material_code(block, S.enc);
                            float g[3];
                            bool any = false;
#pragma unroll
                            for (int k = 0; k < 3; ++k) {
                                g[k] = adj.d_radiance[3ull * item + k] / (float)P.spp;
                                const float sr = hmin(bad ? 0.0f : R[k], 65504.0f);
                                cache.add(code0, k, g[k] * sr);
                                G[k] = (!bad && R[k] <= 65504.0f) ? g[k] * a0[k] : 0.0f;
                                any |= G[k] != 0.0f;
                            }
                            if (!(h.attrib & kEntityHit))
                                atomicAdd(adj.d_power + h.record, g[0] * me[0] + g[1] * me[1] + g[2] * me[2]);
                            if (!any) nee_now = false, bounce_index = P.bounce_count + 1u;  // nothing flows back
                        }
                    } else {
                        const float4 t4 = b.throughput[slot];
                        const float4 n4 = b.seg_n[slot];
                        tp[0] = t4.x;
                        tp[1] = t4.y;
                        tp[2] = t4.z;
                        seg_n[0] = n4.x;
                        seg_n[1] = n4.y;
                        seg_n[2] = n4.z;
                        seg_light = (f & kFlagSegLight) ? 3u : 0u;
                        bounce_index = (f & kFlagBounce) + 1u;
                        float ew = 1.0f;
                        if (seg_light != 0u && (em[0] > 0.0f || em[1] > 0.0f || em[2] > 0.0f))
                            ew = lamp_hit_weight(S, seg_light, h, org, dir, seg_n);
#pragma unroll
                        for (int k = 0; k < 3; ++k) rad[k] += em[k] * (tp[k] * ew);
                        if (kMode == kShadeReplay) {
                            if (!(h.attrib & kEntityHit)) atomicAdd(adj.d_power + h.record, gsum3(G, tp, ew, me));
                            // Everything gathered from here on carries this vertex's albedo.
                            const uint32_t code = material_code(block, S.enc);
#pragma unroll
                            for (int k = 0; k < 3; ++k)
                                if (al[k] > 0.0f && G[k] != 0.0f) cache.add(code, k, G[k] * (R[k] - rad[k]) / al[k]);
                        }
#pragma unroll
                        for (int k = 0; k < 3; ++k) tp[k] *= al[k] / hmax(0.001f, 1.0f);
                        seg_light = 0u;
                        nee_now = P.light_nee && bounce_index <= P.bounce_count;
                    }
                    ShadowRay r;
                    float sadd[3] = {0.0f, 0.0f, 0.0f};
                    if (nee_now) {
                        seg_light = 3u;
                        shadow = nee_prepare<kEntities>(S, o2, h.normal, light_rng, r);
                        // Added to the radiance when unoccluded as nee * throughput (this vertex's
                        // throughput, before Russian roulette rescales it).
                        if (shadow) {
#pragma unroll
                            for (int k = 0; k < 3; ++k) sadd[k] = r.value[k] * (tp[k] * (1.0f / 1.0f));
                        }
                    }
                    uint2 pending = make_uint2(kNone, 0u);
                    if (kMode == kShadeReplay && shadow && r.brick != kNone) {
                        const float gp =
                            G[0] * (tp[0] * r.dvalue_de[0]) + G[1] * (tp[1] * r.dvalue_de[1]) + G[2] * (tp[2] * r.dvalue_de[2]);
                        pending = make_uint2(r.brick, __float_as_uint(gp));
                    }
                    bool alive = true;
                    if (!primary) {
                        const float cp = hmax(tp[0], hmax(tp[1], tp[2]));
                        alive = !(cp <= 0.0f || cp < random01(rng));
                        if (alive) {
#pragma unroll
                            for (int k = 0; k < 3; ++k) tp[k] *= 1.0f / cp;
                        }
                    }
                    ext = alive && bounce_index <= P.bounce_count;
                    if (shadow || ext) {
                        finish = false;
                        live = true;
                        next_flags = bounce_index | (seg_light ? kFlagSegLight : 0u) | (shadow ? kFlagShadow : 0u) |
                                     (ext ? kFlagExt : 0u);
                        b.flags[slot] = next_flags;
                        b.rng[slot] = rng;
                        b.light_rng[slot] = light_rng;
                        b.org[slot] = make_float4(o2[0], o2[1], o2[2], 0.0f);
                        if (ext) {
                            b.dir[slot] = make_float4(d2[0], d2[1], d2[2], 0.0f);
                            b.seg_n[slot] = make_float4(h.normal[0], h.normal[1], h.normal[2], 0.0f);
                            b.throughput[slot] = make_float4(tp[0], tp[1], tp[2], 0.0f);
                        }
                        if (shadow) {
                            b.sdir[slot] = make_float4(r.dir[0], r.dir[1], r.dir[2], r.t_max);
                            b.sadd[slot] = make_float4(sadd[0], sadd[1], sadd[2], 0.0f);
                        }
                        b.radiance[slot] = make_float4(rad[0], rad[1], rad[2], 0.0f);
                        if (primary) {
                            b.a0[slot] = make_float4(a0[0], a0[1], a0[2], 0.0f);
                            b.e0[slot] = make_float4(e0[0], e0[1], e0[2], 0.0f);
                        }
                        if (kMode == kShadeReplay) {
                            if (primary) {
                                b.adj_g[slot] = make_float4(G[0], G[1], G[2], 0.0f);
                                b.adj_r[slot] = make_float4(R[0], R[1], R[2], 0.0f);
                            }
                            if (shadow) b.adj_nee[slot] = pending;
                        }
                    }
                }
            }
            if (finish && kMode == kShadeRecord) {
                float* rs = adj.sample_radiance + 3ull * ((uint64_t)sp * P.width * P.height + item);
#pragma unroll
                for (int k = 0; k < 3; ++k) rs[k] = zero ? 0.0f : rad[k];
            }
            if (finish && kMode != kShadeReplay && V.radiance) {
                float rgb[3] = {0.0f, 0.0f, 0.0f};
                if (!zero) {
                    bool bad = false;
#pragma unroll
                    for (int k = 0; k < 3; ++k) bad |= isnan(rad[k]) || isinf(rad[k]);
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float sr = hmin(bad ? 0.0f : rad[k], 65504.0f);
                        rgb[k] = e0[k] + a0[k] * sr;
                    }
                }
                float* o = V.radiance + 3ull * item;
                const bool last = sp + 1u == P.spp;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float acc = (sp == 0 ? 0.0f : o[k]) + rgb[k];
                    o[k] = last ? acc / (float)P.spp : acc;
                }
            }
        }
        const uint32_t q = warp_append(&b.counts[2 * out + 1], live ? 1u : 0u);
        const uint32_t nr = (shadow ? 1u : 0u) + (ext ? 1u : 0u);
        const uint32_t r = warp_append(&b.counts[2 * out], nr);
        if (live) {
            b.pathq[out][q] = slot;
            uint32_t k = r;
            if (shadow) b.rayq[out][k++] = slot | (kKindShadow << 30);
            if (ext) b.rayq[out][k] = slot | (kKindBounce << 30);
        }
    }
    if (kMode == kShadeReplay) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < kAlbedoCache * 3; i += kWaveThreads) {
            const uint32_t code = s_tag[i / 3];
            if (code != kNone && s_albedo[i] != 0.0f) atomicAdd(adj.d_albedo + 3ull * code + i % 3, s_albedo[i]);
        }
    }
}

}  // namespace

uint64_t wave_buffer_bytes(uint32_t capacity)
{
    const uint64_t c = std::max<uint32_t>(capacity, 32);
    auto a = [](uint64_t x) { return (x + 255u) & ~uint64_t{255}; };
    return 5 * a(4 * c) + 9 * a(16 * c) + a(16 * c) + a(4 * c) + 2 * a(8 * c) + 2 * a(4 * c) + a(64) +
           2 * a(16 * c) + a(8 * c);
}

WaveBuffers wave_carve(void* base, uint32_t capacity)
{
    const uint64_t c = std::max<uint32_t>(capacity, 32);
    char* p = static_cast<char*>(base);
    auto take = [&](uint64_t bytes) {
        char* q = p;
        p += (bytes + 255u) & ~uint64_t{255};
        return q;
    };
    WaveBuffers b;
    b.capacity = capacity;
    b.item = reinterpret_cast<uint32_t*>(take(4 * c));
    b.vs = reinterpret_cast<uint32_t*>(take(4 * c));
    b.flags = reinterpret_cast<uint32_t*>(take(4 * c));
    b.rng = reinterpret_cast<uint32_t*>(take(4 * c));
    b.light_rng = reinterpret_cast<uint32_t*>(take(4 * c));
    b.org = reinterpret_cast<float4*>(take(16 * c));
    b.dir = reinterpret_cast<float4*>(take(16 * c));
    b.throughput = reinterpret_cast<float4*>(take(16 * c));
    b.radiance = reinterpret_cast<float4*>(take(16 * c));
    b.seg_n = reinterpret_cast<float4*>(take(16 * c));
    b.a0 = reinterpret_cast<float4*>(take(16 * c));
    b.e0 = reinterpret_cast<float4*>(take(16 * c));
    b.sdir = reinterpret_cast<float4*>(take(16 * c));
    b.sadd = reinterpret_cast<float4*>(take(16 * c));
    b.hit = reinterpret_cast<uint4*>(take(16 * c));
    b.occluded = reinterpret_cast<uint32_t*>(take(4 * c));
    b.rayq[0] = reinterpret_cast<uint32_t*>(take(8 * c));
    b.rayq[1] = reinterpret_cast<uint32_t*>(take(8 * c));
    b.pathq[0] = reinterpret_cast<uint32_t*>(take(4 * c));
    b.pathq[1] = reinterpret_cast<uint32_t*>(take(4 * c));
    b.counts = reinterpret_cast<uint32_t*>(take(64));
    b.adj_g = reinterpret_cast<float4*>(take(16 * c));
    b.adj_r = reinterpret_cast<float4*>(take(16 * c));
    b.adj_nee = reinterpret_cast<uint2*>(take(8 * c));
    return b;
}

WavePlan wave_plan(const WaveView* views, uint32_t view_count, uint32_t block_width)
{
    WavePlan plan;
    uint32_t max_spp = 0;
    for (uint32_t v = 0; v < view_count; ++v) max_spp = std::max(max_spp, views[v].params.spp);
    const uint32_t bh = 32u / block_width;
    for (uint32_t s = 0; s < max_spp; ++s) {
        std::vector<uint32_t> ids, bases;
        uint64_t items = 0;
        uint32_t bounces = 0;
        for (uint32_t v = 0; v < view_count; ++v) {
            const TraceParams& p = views[v].params;
            if (p.spp <= s) continue;
            ids.push_back(v);
            bases.push_back((uint32_t)items);
            const uint64_t bx = (p.width + block_width - 1) / block_width, by = (p.height + bh - 1) / bh;
            items += 32ull * bx * by;
            bounces = std::max(bounces, p.bounce_count);
        }
        plan.offset.push_back((uint32_t)plan.table.size());
        plan.views.push_back((uint32_t)ids.size());
        plan.items.push_back((uint32_t)std::min<uint64_t>(items, 0xFFFFFFFFull));
        plan.bounces.push_back(bounces);
        plan.table.insert(plan.table.end(), ids.begin(), ids.end());
        plan.table.insert(plan.table.end(), bases.begin(), bases.end());
    }
    return plan;
}

namespace {

// Every sub-wave of every wave of the plan, its shade kernels in mode kMode with kMinBlocks CTAs
// per SM.
template <int kMode, int kMinBlocks>
cudaError_t wave_run(const WaveView* d_views, const WavePlan& plan, const uint32_t* d_table, const WaveBuffers& b,
                     uint32_t block_width, uint32_t sm_count, const WaveAdjoint& adj, cudaStream_t stream,
                     uint32_t* launches, bool entities = false)
{
    if (b.capacity == 0) return cudaErrorInvalidValue;
    static int trace_blocks[2] = {0, 0}, shade_blocks[2] = {0, 0};
    if (trace_blocks[0] == 0) {
        CX_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&trace_blocks[0], wave_trace_kernel<false, kMinBlocks == 8>,
                                                             kWaveThreads, 0));
        CX_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&trace_blocks[1], wave_trace_kernel<true, true>, kWaveThreads,
                                                             0));
        CX_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shade_blocks[0], wave_shade_kernel<kMode, kMinBlocks, false>,
                                                             kWaveThreads, 0));
        CX_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&shade_blocks[1], wave_shade_kernel<kMode, kMinBlocks, true>,
                                                             kWaveThreads, 0));
        for (int k = 0; k < 2; ++k) {
            trace_blocks[k] = std::max(trace_blocks[k], 1);
            shade_blocks[k] = std::max(shade_blocks[k], 1);
        }
    }
    uint32_t count = 0;
    for (size_t s = 0; s < plan.items.size(); ++s) {
        for (uint32_t first = 0; first < plan.items[s]; first += b.capacity) {
            const uint32_t n = std::min(b.capacity, plan.items[s] - first);
            WaveGen g;
            g.table = d_table + plan.offset[s];
            g.n_views = plan.views[s];
            g.sample = (uint32_t)s;
            g.first_item = first;
            g.count = n;
            g.block_width = block_width;
            CX_TRY(cudaMemsetAsync(b.counts, 0, 32, stream));
            wave_generate_kernel<<<(n + kWaveThreads - 1) / kWaveThreads, kWaveThreads, 0, stream>>>(d_views, g, b);
            ++count;
            const uint32_t ray_grid = std::min<uint32_t>((2 * n + kWaveThreads - 1) / kWaveThreads,
                                                         sm_count * (uint32_t)trace_blocks[entities ? 1 : 0]);
            const uint32_t shade_grid = std::min<uint32_t>((n + kWaveThreads - 1) / kWaveThreads,
                                                           sm_count * (uint32_t)shade_blocks[entities ? 1 : 0]);
            for (uint32_t it = 0; it <= plan.bounces[s]; ++it) {
                const uint32_t parity = it & 1u;
                if (entities) wave_trace_kernel<true, true><<<ray_grid, kWaveThreads, 0, stream>>>(d_views, b, parity);
                else wave_trace_kernel<false, kMinBlocks == 8><<<ray_grid, kWaveThreads, 0, stream>>>(d_views, b, parity);
                if (entities)
                    wave_shade_kernel<kMode, kMinBlocks, true><<<shade_grid, kWaveThreads, 0, stream>>>(d_views, b, parity, adj);
                else
                    wave_shade_kernel<kMode, kMinBlocks, false><<<shade_grid, kWaveThreads, 0, stream>>>(d_views, b, parity, adj);
                count += 2;
            }
            CX_TRY(cudaGetLastError());
        }
    }
    if (launches) *launches += count;
    return cudaSuccess;
}

}  // namespace

bool wave_resident_scene(const SceneView& s) { return s.brick_count <= kWaveResidentBricks; }

cudaError_t wave_trace(const WaveView* views, const WaveView* d_views, uint32_t view_count, const WavePlan& plan,
                       const uint32_t* d_table, const WaveBuffers& b, uint32_t block_width, uint32_t sm_count,
                       cudaStream_t stream, uint32_t* launches)
{
    const WaveAdjoint none{nullptr, nullptr, nullptr, nullptr};
    bool entities = false;
    for (uint32_t v = 0; v < view_count; ++v) entities |= views[v].scene.entity_count != 0;
    if (view_count == 1 && wave_resident_scene(views[0].scene))
        return wave_run<kShadeRender, 5>(d_views, plan, d_table, b, block_width, sm_count, none, stream, launches,
                                         entities);
    return wave_run<kShadeRender, 8>(d_views, plan, d_table, b, block_width, sm_count, none, stream, launches,
                                     entities);
}

cudaError_t wave_adjoint(const SceneView& scene, const WaveView* d_record, const WaveView* d_replay,
                         const WavePlan& plan, const uint32_t* d_table, const WaveBuffers& b, uint32_t block_width,
                         uint32_t sm_count, const WaveAdjoint& adj, cudaStream_t stream, uint32_t* launches)
{
    const bool entities = scene.entity_count != 0;
    if (wave_resident_scene(scene)) {
        CX_TRY((wave_run<kShadeRecord, 5>(d_record, plan, d_table, b, block_width, sm_count, adj, stream,
                                              launches, entities)));
        return wave_run<kShadeReplay, 5>(d_replay, plan, d_table, b, block_width, sm_count, adj, stream, launches,
                                         entities);
    }
    CX_TRY((wave_run<kShadeRecord, 8>(d_record, plan, d_table, b, block_width, sm_count, adj, stream,
                                          launches, entities)));
    return wave_run<kShadeReplay, 8>(d_replay, plan, d_table, b, block_width, sm_count, adj, stream, launches,
                                     entities);
}

}  // namespace cx
