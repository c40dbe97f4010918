// Device functions of the path tracer, shared by the per-frame kernel (trace.cu) and the batched
// persistent kernel (trace_batch.cu); each translation unit compiles its own copy. Restates, as
// device code:
//   brick DDA          shaders/render/caelix_brick_trace.hlsl:177-451
//   scene traversal    shaders/render/caelix_scene_trace.hlsl:57-169, the TLAS replaced by a
//                      front-to-back DDA over the brick grid: the occupancy bitmap, then the brick
//                      hash table, then the brick DDA; the first brick in DDA order with a hit in
//                      [tmin, tmax) is the closest hit
//   light tree draw    shaders/light/caelix_light_tree.hlsl:65-767
//   light tree pdf     caelix_light_tree.hlsl:514-608, 769-777, 853-949
//   integrator parts   shaders/render/caelix_path_trace.hlsl:245-449, :737-978,
//                      caelix_light_nee.hlsl:20-34, caelix_shading.hlsl:267-307,
//                      caelix_random.hlsl, common/caelix_frame.hlsl:164-171
// in the configuration of the benchmark scenes: opaque voxels with a Lambertian lobe (metallic 0,
// smoothness 0), light-tree NEE with MIS over the world's and the entities' light trees, no sun,
// black sky, no fog, bounce NEE probability 1. A voxel's albedo is its material code's table entry;
// its emission is the entry's emission times its brick's emitter power. Every float operation is one IEEE fp32 operation in the reference's order (the library
// is built with --fmad=false); sin/cos of the unit-vector draw use this library's Cody-Waite +
// Taylor polynomials, normalize is v * (1 / sqrt(dot(v, v))).
#pragma once
#include <cstdint>

#include "cx_device.cuh"
#include "scene.cuh"
#include "scene_device.cuh"
#include "trace.cuh"

namespace cx {

namespace {


constexpr float kRayTMax = 1e30f;
constexpr float kBounceTMax = 1e4f;
constexpr float kPushOff = 0.002f;
constexpr float kNearField = 8.0f;
constexpr float kPi = 3.1415926535f;
constexpr float kTwoPi = 6.283185307f;

__device__ __forceinline__ float hmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float hmax(float a, float b) { return b > a ? b : a; }
__device__ __forceinline__ float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// ---- random streams ----
__device__ __forceinline__ uint32_t pcg_hash(uint32_t v)
{
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
__device__ __forceinline__ uint32_t init_random(uint32_t px, uint32_t py, uint32_t seed)
{
    const uint32_t s = pcg_hash(px ^ (py << 16) ^ (seed * 0x9E3779B9u));
    return s != 0u ? s : 0x9E3779B9u;
}
__device__ __forceinline__ uint32_t random_u32(uint32_t& s)
{
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    return s;
}
__device__ __forceinline__ float random01(uint32_t& s) { return (float)(random_u32(s) >> 8) * (1.0f / 16777216.0f); }
__device__ __forceinline__ uint32_t lt_random(uint32_t& rng)
{
    rng = rng * 747796405u + 2891336453u;
    const uint32_t word = ((rng >> ((rng >> 28) + 4u)) ^ rng) * 277803737u;
    return (word >> 22) ^ word;
}
__device__ __forceinline__ float lt_random_float(uint32_t& rng) { return (float)(lt_random(rng) >> 8) * (1.0f / 16777216.0f); }

// sin and cos of a in [0, 2 pi]: Cody-Waite reduction by pi/2, Taylor polynomials (Horner).
__device__ __forceinline__ void sincos_cw(float a, float& s, float& c)
{
    const float k = floorf(a * 0.636619772f + 0.5f);
    const float r = (a - k * 1.57079637f) - k * -4.37113883e-8f;
    const float r2 = r * r;
    const float sp =
        r + r * r2 * (-0.166666667f + r2 * (0.00833333333f + r2 * (-0.000198412698f + r2 * 2.75573192e-6f)));
    const float cp =
        1.0f + r2 * (-0.5f + r2 * (0.0416666667f + r2 * (-0.00138888889f + r2 * (2.48015873e-5f + r2 * -2.75573192e-7f))));
    const int q = ((int)k) & 3;
    s = q == 0 ? sp : (q == 1 ? cp : (q == 2 ? -sp : -cp));
    c = q == 0 ? cp : (q == 1 ? -sp : (q == 2 ? -cp : sp));
}

__device__ __forceinline__ void random_unit_vector(uint32_t& rng, float out[3])
{
    const float u = random01(rng);
    const float v = random01(rng);
    const float a = u * kTwoPi;
    const float y = v * 2.0f - 1.0f;
    const float sy = sqrtf(hmax(1.0f - y * y, 0.0f));
    float sa, ca;
    sincos_cw(a, sa, ca);
    out[0] = sa * sy;
    out[1] = y;
    out[2] = ca * sy;
}

// ---- brick DDA ----
__device__ __forceinline__ float safe_inv_axis(float d)
{
    if (fabsf(d) >= 1e-20f) return 1.0f / d;
    return d < 0.0f ? -1.0f / 1e-20f : 1.0f / 1e-20f;
}

__device__ __forceinline__ void vrt_step(int cell[3], const float t_start[3], const float origin[3], const float dir[3],
                                         const float inv[3])
{
    float side[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) side[k] = t_start[k] + (float)cell[k] * inv[k];
    const float tmin = hmin(hmin(side[0], side[1]), side[2]) + 0.0001f;
#pragma unroll
    for (int k = 0; k < 3; ++k) cell[k] = (int)floorf(origin[k] + tmin * dir[k]);
}

__device__ __forceinline__ float brick_ray(const uint32_t* __restrict__ rec, const float entry[3], const float dir[3],
                                           float entry_t, uint32_t entry_coarse, const Encoding& enc, uint32_t& attrib)
{
    float inv[3], t_start[3], origin[3];
    int cell[3], prev[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        inv[k] = safe_inv_axis(dir[k]);
        t_start[k] = ((dir[k] >= 0.0f ? 1.0f : 0.0f) - entry[k]) * inv[k];
        origin[k] = hmin(hmax(entry[k], 0.0f), 8.0f - 0.0001f);
        cell[k] = (int)floorf(origin[k]);
        prev[k] = cell[k];
    }
    for (uint32_t step = 0; step < 22; ++step) {
        if ((uint32_t)cell[0] >= 8u || (uint32_t)cell[1] >= 8u || (uint32_t)cell[2] >= 8u) break;
        const uint32_t cbit = (uint32_t)((cell[0] >> 2) | ((cell[1] >> 2) << 1) | ((cell[2] >> 2) << 2));
        if ((entry_coarse & (1u << cbit)) == 0u) {
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                cell[k] = dir[k] < 0.0f ? (cell[k] & ~3) : (cell[k] | 3);
                prev[k] = cell[k];
            }
            vrt_step(cell, t_start, origin, dir, inv);
            continue;
        }
        const uint2 occ2 = __ldg(reinterpret_cast<const uint2*>(rec + 2 + 2 * cbit));
        const uint32_t mbit = (uint32_t)((cell[0] & 3) | ((cell[1] & 3) << 2) | ((cell[2] & 3) << 4));
        const uint32_t occ_word = mbit < 32 ? occ2.x : occ2.y;
        if ((occ_word >> (mbit & 31)) & 1u) {
            const uint32_t w = __ldg(rec + 18 + (cell[0] >> 1) + (cell[1] << 2) + (cell[2] << 5));
            const uint32_t blk = (w >> ((cell[0] & 1) << 4)) & 0xFFFFu;
            float T;
            uint32_t nf;
            if (step == 0u) {
                T = 0.0f;
                nf = entry_coarse >> 26;
            } else {
                float side[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) side[k] = t_start[k] + (float)prev[k] * inv[k];
                T = hmin(hmin(side[0], side[1]), side[2]);
                const bool mx = side[0] <= T + 0.0001f;
                const bool my = side[1] <= T + 0.0001f;
                const uint32_t x_use = mx ? 0xFFFFFFFFu : 0u;
                const uint32_t y_use = (my ? 0xFFFFFFFFu : 0u) & ~x_use;
                const uint32_t z_use = ~(x_use | y_use);
                nf = ((dir[0] > 0.0f ? 2u : 1u) & x_use) | ((dir[1] > 0.0f ? 8u : 4u) & y_use) |
                     ((dir[2] > 0.0f ? 32u : 16u) & z_use);
            }
            bool term = (blk & enc.opaque_mask) != 0;
            if (!term) term = (step == 0 && entry_t == 0.0f) ? false : ((((blk >> enc.face_shift) & 63u) & nf) != 0);
            if (term) {
                attrib = (blk << 16) | (((uint32_t)cell[0] | ((uint32_t)cell[1] << 3) | ((uint32_t)cell[2] << 6)) << 6) | nf;
                return entry_t + T;
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) prev[k] = cell[k];
        vrt_step(cell, t_start, origin, dir, inv);
    }
    attrib = 0u;
    return 0.0f;
}

__device__ __forceinline__ float brick_primitive(const uint32_t* __restrict__ rec, const float o[3], const float d[3],
                                                 float t_current, const float bo[3], const Encoding& enc,
                                                 uint32_t& attrib)
{
    const uint2 info = __ldg(reinterpret_cast<const uint2*>(rec));
    const uint32_t tb = info.y;
    const float tmin_v[3] = {(float)(tb & 7u), (float)((tb >> 3) & 7u), (float)((tb >> 6) & 7u)};
    const float tmax_v[3] = {(float)((tb >> 9) & 7u) + 1.0f, (float)((tb >> 12) & 7u) + 1.0f,
                             (float)((tb >> 15) & 7u) + 1.0f};
    float tmin[3], tmax[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float inv = 1.0f / d[k];
        const float t0 = (bo[k] + tmin_v[k] - o[k]) * inv;
        const float t1 = (bo[k] + tmax_v[k] - o[k]) * inv;
        tmin[k] = hmin(t0, t1);
        tmax[k] = hmax(t0, t1);
    }
    const float largest = hmax(hmax(tmin[0], tmin[1]), tmin[2]);
    const float smallest = hmin(hmin(tmax[0], tmax[1]), tmax[2]);
    if (largest > smallest || smallest < 0.0f || largest > t_current) {
        attrib = 0u;
        return 0.0f;
    }
    const float t = hmax(0.0f, largest);
    float entry[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) entry[k] = o[k] + d[k] * t - bo[k];
    uint32_t nf;
    if (largest == tmin[0]) nf = d[0] > 0.0f ? 2u : 1u;
    else if (largest == tmin[1]) nf = d[1] > 0.0f ? 8u : 4u;
    else nf = d[2] > 0.0f ? 32u : 16u;
    return brick_ray(rec, entry, d, t, (nf << 26) | ((info.x >> 16) & 0xFFu), enc, attrib);
}

struct Hit
{
    bool hit;
    float t;
    uint32_t attrib;
    uint32_t record;
    uint32_t group;
    float normal[3];
    float object_hit[3];
};

// Closest hit over the bricks (front-to-back DDA over the brick grid). Cell c of axis k is brick
// key origin[k] + c, voxels [8 (origin[k] + c), 8 (origin[k] + c + 1)).
__device__ __forceinline__ Hit trace_ray_body(const SceneView& s, const float o[3], const float d[3], float tmin_ray, float tmax_ray)
{
    Hit h;
    h.hit = false;
    float inv[3], tnear = -3.0e38f, tfar = 3.0e38f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        inv[k] = safe_inv_axis(d[k]);
        const float t0 = ((float)(8 * s.origin[k]) - o[k]) * inv[k];
        const float t1 = ((float)(8 * (s.origin[k] + (int)s.grid[k])) - o[k]) * inv[k];
        tnear = hmax(tnear, hmin(t0, t1));
        tfar = hmin(tfar, hmax(t0, t1));
    }
    const float t_enter = hmax(tnear, tmin_ray);
    const float t_exit = hmin(tfar, tmax_ray);
    if (!(t_enter <= t_exit)) return h;
    int cell[3], step[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float p = o[k] + d[k] * t_enter;
        int c = (int)floorf(p * 0.125f) - s.origin[k];
        c = c < 0 ? 0 : c;
        c = c > (int)s.grid[k] - 1 ? (int)s.grid[k] - 1 : c;
        cell[k] = c;
        step[k] = d[k] >= 0.0f ? 1 : -1;
    }
    const uint32_t limit = s.grid[0] + s.grid[1] + s.grid[2] + 3;
    for (uint32_t it = 0; it < limit; ++it) {
        const uint64_t lin = (uint64_t)cell[0] + s.grid[0] * ((uint64_t)cell[1] + (uint64_t)s.grid[1] * cell[2]);
        if ((__ldg(s.bitmap + (lin >> 5)) >> (lin & 31)) & 1u) {
            const int32_t key[3] = {s.origin[0] + cell[0], s.origin[1] + cell[1], s.origin[2] + cell[2]};
            const uint32_t r = hash_lookup(s.hash_slots, s.hash_capacity, s.hash_max_probe, key[0], key[1], key[2]);
            if (r != 0xFFFFFFFFu) {
                const float bo[3] = {(float)(key[0] * 8), (float)(key[1] * 8), (float)(key[2] * 8)};
                uint32_t attrib;
                const float t =
                    brick_primitive(s.records + (uint64_t)r * kRecordWords, o, d, tmax_ray, bo, s.enc, attrib);
                if (attrib != 0u && t >= tmin_ray && t < tmax_ray) {
                    h.hit = true;
                    h.t = t;
                    h.attrib = attrib;
                    h.record = r;
                    const uint32_t gs = s.group_shift;
                    h.group = ((uint32_t)cell[0] >> gs) +
                              s.groups[0] * (((uint32_t)cell[1] >> gs) + s.groups[1] * ((uint32_t)cell[2] >> gs));
                    const uint32_t f = (uint32_t)(__ffs(attrib & 0x3Fu) - 1);
                    h.normal[0] = f == 0 ? 1.0f : (f == 1 ? -1.0f : 0.0f);
                    h.normal[1] = f == 2 ? 1.0f : (f == 3 ? -1.0f : 0.0f);
                    h.normal[2] = f == 4 ? 1.0f : (f == 5 ? -1.0f : 0.0f);
#pragma unroll
                    for (int k = 0; k < 3; ++k) h.object_hit[k] = o[k] + d[k] * t;
                    return h;
                }
            }
        }
        float tn[3];
#pragma unroll
        for (int k = 0; k < 3; ++k)
            tn[k] = ((float)((s.origin[k] + cell[k] + (step[k] > 0 ? 1 : 0)) * 8) - o[k]) * inv[k];
        // The axis of the nearest boundary (the first of equals), stepped with selects.
        int axis = 0;
        float t_next = tn[0];
        if (tn[1] < t_next) {
            axis = 1;
            t_next = tn[1];
        }
        if (tn[2] < t_next) {
            axis = 2;
            t_next = tn[2];
        }
        if (t_next > t_exit) break;
        bool out = false;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (axis == k) {
                cell[k] += step[k];
                out = cell[k] < 0 || cell[k] >= (int)s.grid[k];
            }
        }
        if (out) break;
    }
    return h;
}

// The out-of-line copy for kernels that trace from several call sites (one copy of the DDA keeps
// their instruction footprint small); a kernel with one call site inlines trace_ray_body.
__device__ __noinline__ Hit trace_ray(const SceneView& s, const float o[3], const float d[3], float tmin_ray, float tmax_ray)
{
    return trace_ray_body(s, o, d, tmin_ray, tmax_ray);
}

// One entity after the world's bricks: the ray in the entity's frame (local = rot^T (x - pos)),
// its bricks' DDA up to the current hit, a strictly nearer hit taken with the entity bit, the
// entity's index as its group and the rotated face normal (normalised as v * (1 / sqrt(dot(v, v)))).
__device__ __forceinline__ void entity_candidate(const SceneView& s, uint32_t e, const float o[3], const float d[3],
                                                 float tmin_ray, float tmax_ray, Hit& h)
{
    const EntityView& E = s.entities[e];
    // A ray that misses the entity's bounding sphere, or meets it only behind its origin or beyond
    // the current hit, cannot hit it (the margins cover the rounding: the test only skips work, it
    // never changes a hit).
    {
        const float4 sp = make_float4(__ldg(&E.sphere[0]), __ldg(&E.sphere[1]), __ldg(&E.sphere[2]),
                                      __ldg(&E.sphere[3]));
        const float oc[3] = {sp.x - o[0], sp.y - o[1], sp.z - o[2]};
        const float oc2 = dot3(oc, oc);
        const float tc = dot3(oc, d);
        const float t_far = h.hit ? h.t : tmax_ray;
        if (oc2 - tc * tc > sp.w * sp.w + 1e-5f * (oc2 + 1.0f)) return;
        if (tc + sp.w < tmin_ray - 1e-3f * (1.0f + fabsf(tc))) return;
        if (tc - sp.w > t_far + 1e-3f * (1.0f + fabsf(tc))) return;
    }
    float R[9], ol[3], dl[3];
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = __ldg(&E.rot[i]);
    const float q[3] = {o[0] - __ldg(&E.pos[0]), o[1] - __ldg(&E.pos[1]), o[2] - __ldg(&E.pos[2])};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        ol[k] = R[k] * q[0] + R[3 + k] * q[1] + R[6 + k] * q[2];
        dl[k] = R[k] * d[0] + R[3 + k] * d[1] + R[6 + k] * d[2];
    }
    // A hit must be nearer than the current one; at an equal distance the lower entity index wins
    // against an entity hit (the world's hit always wins a tie), so the result does not depend on
    // the order in which the entities are taken.
    const bool tie_wins = h.hit && (h.attrib & kEntityHit) && e < (h.group >> kEntityShift);
    const float t_limit = h.hit ? (tie_wins ? nextafterf(h.t, INFINITY) : h.t) : tmax_ray;
    const Hit he = trace_ray_body(E.scene, ol, dl, tmin_ray, t_limit);
    if (!he.hit) return;
    h = he;
    h.attrib |= kEntityHit;
    h.group = (e << kEntityShift) | he.group;
    const uint32_t f = (uint32_t)(__ffs(he.attrib & 0x3Fu) - 1);
    const float sign = (f & 1u) ? -1.0f : 1.0f;
    float v[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = R[3 * i + (f >> 1)] * sign;
    const float inv = 1.0f / sqrtf(dot3(v, v));
#pragma unroll
    for (int i = 0; i < 3; ++i) h.normal[i] = v[i] * inv;
}

// The entities after the world's bricks (entity_candidate): every entity in index order, or with
// the scene's entity BVH only those whose box the ray meets before the current hit (collected by a
// traversal of the BVH over the entities' bounding-sphere boxes, then taken in order of their boxes'
// entry distance, so that a near hit culls the farther candidates; entity_candidate's tie rule
// makes the hit the one the loop over every entity finds: the nearest, ties to the world and then to
// the lower index). More candidates than the list holds: every entity. `any`: an occlusion test,
// which stops at the first hit (a shadow ray needs only whether something is hit).
constexpr uint32_t kEntityCandidates = 16;
constexpr uint32_t kEntityStack = 32;

__device__ __forceinline__ void trace_entities_body(const SceneView& s, const float o[3], const float d[3], float tmin_ray,
                                            float tmax_ray, Hit& h, bool any = false)
{
    if (s.entity_nodes) {
        float inv[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) inv[k] = safe_inv_axis(d[k]);
        const float t_far = h.hit ? h.t : tmax_ray;
        const float t_lo = tmin_ray - 1e-3f * (1.0f + fabsf(tmin_ray));
        const float t_hi = t_far + 1e-3f * (1.0f + fabsf(t_far));
        uint32_t cand[kEntityCandidates];
        float cand_t[kEntityCandidates];  // the entry distance of each candidate's box
        uint32_t stack[kEntityStack];
        uint32_t n = 0, sp = 0;
        bool overflow = false;
        stack[sp++] = 0;
        while (sp && !overflow) {
            const EntityNode& N = s.entity_nodes[stack[--sp]];
            const float4 a = __ldg(reinterpret_cast<const float4*>(&N));
            const float4 b = __ldg(reinterpret_cast<const float4*>(&N) + 1);
            const float lo[3] = {a.x, a.y, a.z}, hi[3] = {b.x, b.y, b.z};
            float t0 = t_lo, t1 = t_hi;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float ta = (lo[k] - o[k]) * inv[k];
                const float tb = (hi[k] - o[k]) * inv[k];
                t0 = hmax(t0, hmin(ta, tb));
                t1 = hmin(t1, hmax(ta, tb));
            }
            if (!(t0 <= t1)) continue;
            const uint32_t first = __float_as_uint(a.w), second = __float_as_uint(b.w);
            if (first & kEntityLeaf) {
                if (n < kEntityCandidates) {
                    cand[n] = first & ~kEntityLeaf;
                    cand_t[n++] = t0;
                } else {
                    overflow = true;
                }
            } else if (sp + 2 <= kEntityStack) {
                stack[sp++] = second;
                stack[sp++] = first;
            } else {
                overflow = true;
            }
        }
        if (!overflow) {
            // Nearest box first (an insertion sort of at most kEntityCandidates by entry distance,
            // then index).
            for (uint32_t x = 1; x < n; ++x) {
                const uint32_t v = cand[x];
                const float tv = cand_t[x];
                uint32_t y = x;
                for (; y > 0 && (cand_t[y - 1] > tv || (cand_t[y - 1] == tv && cand[y - 1] > v)); --y) {
                    cand[y] = cand[y - 1];
                    cand_t[y] = cand_t[y - 1];
                }
                cand[y] = v;
                cand_t[y] = tv;
            }
            for (uint32_t x = 0; x < n && !(any && h.hit); ++x) entity_candidate(s, cand[x], o, d, tmin_ray, tmax_ray, h);
            return;
        }
    }
    for (uint32_t e = 0; e < s.entity_count && !(any && h.hit); ++e) entity_candidate(s, e, o, d, tmin_ray, tmax_ray, h);
}

// The out-of-line copy for the kernels that trace from several call sites; the wavefront trace
// kernel inlines trace_entities_body (one call site: 93 registers and no call frame instead of 115
// and a 336-byte frame).
__device__ __noinline__ void trace_entities(const SceneView& s, const float o[3], const float d[3], float tmin_ray,
                                            float tmax_ray, Hit& h, bool any = false)
{
    trace_entities_body(s, o, d, tmin_ray, tmax_ray, h, any);
}

// The entity-local hit point of an entity hit (the wavefront keeps a hit as four words): the ray
// in the entity's frame as trace_entities computes it, at t.
__device__ __forceinline__ void entity_local_hit(const SceneView& s, uint32_t entity, const float o[3], const float d[3],
                                                 float t, float out[3])
{
    const EntityView& E = s.entities[entity];
    float R[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) R[i] = __ldg(&E.rot[i]);
    const float q[3] = {o[0] - __ldg(&E.pos[0]), o[1] - __ldg(&E.pos[1]), o[2] - __ldg(&E.pos[2])};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float ol = R[k] * q[0] + R[3 + k] * q[1] + R[6 + k] * q[2];
        const float dl = R[k] * d[0] + R[3 + k] * d[1] + R[6 + k] * d[2];
        out[k] = ol + dl * t;
    }
}

// The world normal of an entity hit from its face flags (the wavefront keeps a hit as four words).
__device__ __forceinline__ void entity_normal(const SceneView& s, uint32_t entity, uint32_t attrib, float n[3])
{
    const EntityView& E = s.entities[entity];
    const uint32_t f = (uint32_t)(__ffs(attrib & 0x3Fu) - 1);
    const float sign = (f & 1u) ? -1.0f : 1.0f;
    float v[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = __ldg(&E.rot[3 * i + (f >> 1)]) * sign;
    const float inv = 1.0f / sqrtf(dot3(v, v));
#pragma unroll
    for (int i = 0; i < 3; ++i) n[i] = v[i] * inv;
}

// Closest hit over the world's bricks and the entities'. `any`: an occlusion test (only h.hit is
// meaningful): a ray that the world occludes skips the entities, and the entities stop at the
// first hit.
__device__ __forceinline__ Hit trace_scene_body(const SceneView& s, const float o[3], const float d[3], float tmin_ray,
                                                float tmax_ray, bool any = false)
{
    Hit h = trace_ray_body(s, o, d, tmin_ray, tmax_ray);
    if (s.entity_count && !(any && h.hit)) trace_entities_body(s, o, d, tmin_ray, tmax_ray, h, any);
    return h;
}

__device__ __noinline__ Hit trace_scene(const SceneView& s, const float o[3], const float d[3], float tmin_ray, float tmax_ray,
                                        bool any = false)
{
    Hit h = trace_ray(s, o, d, tmin_ray, tmax_ray);
    if (s.entity_count && !(any && h.hit)) trace_entities(s, o, d, tmin_ray, tmax_ray, h, any);
    return h;
}

// ---- the voxel id target (shaders/render/caelix_scene_trace.hlsl:171-200) ----
__device__ __forceinline__ uint32_t hash_avalanche(uint32_t v)
{
    v ^= v >> 16;
    v *= 0x7FEB352Du;
    v ^= v >> 15;
    v *= 0x846CA68Bu;
    v ^= v >> 16;
    return v;
}

__device__ __forceinline__ uint32_t voxel_id_word(uint32_t seed, uint32_t entity, const int32_t v[3])
{
    uint32_t h = hash_avalanche(seed ^ entity);
    h = hash_avalanche(h ^ (uint32_t)v[0]);
    h = hash_avalanche(h ^ (uint32_t)v[1]);
    h = hash_avalanche(h ^ (uint32_t)v[2]);
    return h == 0xFFFFFFFFu ? 0xFFFFFFFEu : h;
}

// The voxel id of a hit: two hashes of (entity id, entity-local voxel = 8 brick key + DDA cell).
template <bool kEntities>
__device__ __forceinline__ uint2 voxel_id_of(const SceneView& s, uint32_t attrib, uint32_t record, uint32_t group)
{
    uint32_t entity = 0;
    const int32_t* keys = s.keys;
    if (kEntities && (attrib & kEntityHit)) {
        const EntityView& E = s.entities[group >> kEntityShift];
        entity = __ldg(&E.id);
        keys = E.scene.keys;
    }
    const uint32_t cell = (attrib >> 6) & 0x1FFu;
    int32_t v[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) v[k] = __ldg(keys + 3ull * record + k) * 8 + (int32_t)((cell >> (3 * k)) & 7u);
    return make_uint2(voxel_id_word(0x9E3779B9u, entity, v), voxel_id_word(0x85EBCA6Bu, entity, v));
}

// Writes pixel `item`'s voxel id (VoxelIdOrMiss): the hit's, or the miss value for a miss and for a
// hit farther than the limit.
template <bool kEntities>
__device__ __forceinline__ void write_voxel_id(const SceneView& s, const TraceParams& P, uint32_t item, bool hit, float t,
                                               uint32_t attrib, uint32_t record, uint32_t group)
{
    uint2 id = make_uint2(0xFFFFFFFFu, 0xFFFFFFFFu);
    if (hit && (P.voxel_id_tmax <= 0.0f || t <= P.voxel_id_tmax)) id = voxel_id_of<kEntities>(s, attrib, record, group);
    reinterpret_cast<uint2*>(P.voxel_id)[item] = id;
}

// ---- light tree ----
__device__ __forceinline__ float power6(const float f[6]) { return f[0] + f[1] + f[2] + f[3] + f[4] + f[5]; }

__device__ __forceinline__ void emitter_cosines(const float dlo[3], const float dhi[3], float c[6])
{
    float c2[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float cl = hmin(hmax(0.0f, dlo[k]), dhi[k]);
        c2[k] = cl * cl;
    }
    const float all2 = c2[0] + c2[1] + c2[2];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float others = all2 - c2[a];
        // Both quotients for every lane, then the selects (no divergent branch around them).
        const float ch = dhi[a] / sqrtf(dhi[a] * dhi[a] + others);
        const float cl = -dlo[a] / sqrtf(dlo[a] * dlo[a] + others);
        c[2 * a] = dhi[a] > 0.0f ? ch : 0.0f;
        c[2 * a + 1] = dlo[a] < 0.0f ? cl : 0.0f;
    }
}

// The importance of a light box for the shading point x with normal n (LtImportance,
// caelix_light_tree.hlsl:85-155). Branch-free: every operation of the reference's order is
// computed for every lane and the early exits become selects, so that the lanes of a warp walking
// the tree stay converged (an early-exit branch would leave the others idle while it runs).
__device__ __forceinline__ float importance(const float x[3], const float n[3], const float lo[3], const float hi[3],
                                            const float face[6])
{
    float dlo[3], dhi[3], c[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dlo[k] = x[k] - hi[k];
        dhi[k] = x[k] - lo[k];
    }
    emitter_cosines(dlo, dhi, c);
    float e = 0.0f;
#pragma unroll
    for (int f = 0; f < 6; ++f) e += face[f] * c[f];
    float centre[3], half[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        centre[k] = 0.5f * (lo[k] + hi[k]);
        half[k] = 0.5f * (hi[k] - lo[k]);
    }
    const bool has_n = n[0] != 0.0f || n[1] != 0.0f || n[2] != 0.0f;
    const float cx[3] = {centre[0] - x[0], centre[1] - x[1], centre[2] - x[2]};
    const float an[3] = {fabsf(n[0]), fabsf(n[1]), fabsf(n[2])};
    const float m = dot3(n, cx) + dot3(an, half);
    float q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) q[k] = hmax(hmax(lo[k] - x[k], x[k] - hi[k]), 0.0f);
    const float dmin = sqrtf(dot3(q, q));
    const float ratio = m / dmin;
    const float cr = has_n ? (dmin > 0.0f ? hmin(1.0f, ratio) : 1.0f) : 1.0f;
    const float tc[3] = {x[0] - centre[0], x[1] - centre[1], x[2] - centre[2]};
    const float extent2 = dot3(half, half);
    const float d2 = hmax(dot3(tc, tc), hmax(1.0f, extent2));
    const float value = e * cr / d2;
    return e <= 0.0f ? 0.0f : ((has_n && m <= 0.0f) ? 0.0f : value);
}

struct Pick
{
    float sum_i, sum_p, weight_i, weight_p;
    uint32_t index_i, index_p;
};
__device__ __forceinline__ void pick_add(Pick& p, float imp, float pw, uint32_t index, float u)
{
    if (imp > 0.0f) {
        p.sum_i += imp;
        if (u * p.sum_i < imp) {
            p.weight_i = imp;
            p.index_i = index;
        }
    }
    if (pw > 0.0f) {
        p.sum_p += pw;
        if (u * p.sum_p < pw) {
            p.weight_p = pw;
            p.index_p = index;
        }
    }
}
__device__ __forceinline__ uint32_t pick_end(const Pick& p, float& prob)
{
    if (p.sum_i > 0.0f) {
        prob = p.weight_i / p.sum_i;
        return p.index_i;
    }
    prob = p.sum_p > 0.0f ? p.weight_p / p.sum_p : 0.0f;
    return p.sum_p > 0.0f ? p.index_p : kNone;
}
__device__ __forceinline__ float pick_probability(float sum_i, float sum_p, float imp, float pw)
{
    if (sum_i > 0.0f) return imp / sum_i;
    return sum_p > 0.0f ? pw / sum_p : 0.0f;
}

struct Summary
{
    float face[6], lo[3], hi[3];
};

__device__ __forceinline__ void node_slot(const LightBvhNode* nd, uint32_t s, Summary& out)
{
#pragma unroll
    for (int f = 0; f < 6; ++f) out.face[f] = __ldg(&nd->child_face[s][f]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        out.lo[k] = __ldg(&nd->child_lo[s][k]);
        out.hi[k] = __ldg(&nd->child_hi[s][k]);
    }
}

// Tree 0 is the world's tree; tree 1 the entities' (none without entity lights).
__device__ __forceinline__ void tree_summary(const SceneView& s, uint32_t k, Summary& out, uint32_t& root)
{
#pragma unroll
    for (int f = 0; f < 6; ++f) out.face[f] = 0.0f;
#pragma unroll
    for (int q = 0; q < 3; ++q) out.lo[q] = out.hi[q] = 0.0f;
    root = kNone;
    const LightTreeHeader* h = k == 0 ? s.header : (s.dyn ? s.dyn->header : nullptr);
    if (h) {
        const uint32_t r = __ldg(&h->root);
        if (r != kNone) {
            root = r;
#pragma unroll
            for (int f = 0; f < 6; ++f) out.face[f] = __ldg(&h->summary.face[f]);
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                out.lo[q] = __ldg(&h->summary.lo[q]);
                out.hi[q] = __ldg(&h->summary.hi[q]);
            }
        }
    }
}

__device__ __forceinline__ uint32_t child_count(const uint4 c)
{
    return (c.x != kNone) + (c.y != kNone) + (c.z != kNone) + (c.w != kNone);
}

// The probability of picking tree `target` (LtTreeProbability). An empty tree's box and faces
// are zero, so its importance and power are never positive and it adds nothing to either sum.
__device__ float tree_probability(const SceneView& s, const float x[3], const float n[3], uint32_t target)
{
    float sum_i = 0.0f, sum_p = 0.0f, imp_t = 0.0f, pow_t = 0.0f;
    for (uint32_t k = 0; k < 2; ++k) {
        Summary sm;
        uint32_t root;
        tree_summary(s, k, sm, root);
        if (root == kNone) continue;  // an empty tree adds zero to both sums
        const float imp = importance(x, n, sm.lo, sm.hi, sm.face);
        const float pw = power6(sm.face);
        sum_i += imp > 0.0f ? imp : 0.0f;
        sum_p += pw > 0.0f ? pw : 0.0f;
        if (k == target) {
            imp_t = imp;
            pow_t = pw;
        }
    }
    return pick_probability(sum_i, sum_p, imp_t, pow_t);
}

__device__ float slot_probability(const LightBvhNode* nd, const float x[3], const float n[3], uint32_t slot)
{
    const uint4 ch = __ldg(reinterpret_cast<const uint4*>(nd->child));
    if (child_count(ch) == 1) return 1.0f;
    float sum_i = 0.0f, sum_p = 0.0f, imp_t = 0.0f, pow_t = 0.0f;
    for (uint32_t q = 0; q < 4; ++q) {
        Summary sm;
        node_slot(nd, q, sm);
        const float imp = importance(x, n, sm.lo, sm.hi, sm.face);
        const float pw = power6(sm.face);
        if (__ldg(&nd->child[q]) != kNone) {
            sum_i += imp > 0.0f ? imp : 0.0f;
            sum_p += pw > 0.0f ? pw : 0.0f;
        }
        if (q == slot) {
            imp_t = imp;
            pow_t = pw;
        }
    }
    return pick_probability(sum_i, sum_p, imp_t, pow_t);
}

// The probability of drawing leaf `leaf` of tree k (its light set L): the slot picks up to the
// root, times the pick of tree k.
__device__ __noinline__ float leaf_probability(const SceneView& s, const SceneView& L, uint32_t leaf, const float x[3],
                                              const float n[3], uint32_t k)
{
    if (__ldg(&L.header->root) == kNone) return 0.0f;
    const uint32_t parent = __ldg(&L.leaves[leaf].parent);
    if (parent == kNone) return 0.0f;
    uint32_t node = parent >> kParentSlotBits, slot = parent & kParentSlotMask;
    float probability = 1.0f;
    for (uint32_t depth = 0; depth < 64; ++depth) {
        const LightBvhNode* nd = L.nodes + node;
        probability *= slot_probability(nd, x, n, slot);
        const uint2 up = __ldg(reinterpret_cast<const uint2*>(&nd->parent));
        if (up.x == kNone) return probability * tree_probability(s, x, n, k);
        node = up.x;
        slot = up.y;
    }
    return 0.0f;
}

__device__ float family_weights(const SceneView& s, uint32_t group, const uint32_t* rec, const float x[3], float w[6])
{
    const GroupFrame* fr = s.frames + group;
    float v[3], xg[3], R[9], org[3];
#pragma unroll
    for (int k = 0; k < 9; ++k) R[k] = __ldg(&fr->rot[k]);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        v[k] = x[k] - __ldg(&fr->trans[k]);
        org[k] = __ldg(&fr->origin[k]);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) xg[j] = v[0] * R[0 * 3 + j] + v[1] * R[1 * 3 + j] + v[2] * R[2 * 3 + j] - org[j];
    const uint32_t blo = __ldg(rec + 6), bhi = __ldg(rec + 7);
    const float lo[3] = {(float)(blo & 0x3FFu), (float)((blo >> 10) & 0x3FFu), (float)((blo >> 20) & 0x3FFu)};
    const float hi[3] = {(float)(bhi & 0x3FFu), (float)((bhi >> 10) & 0x3FFu), (float)((bhi >> 20) & 0x3FFu)};
    float dlo[3], dhi[3], c[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dlo[k] = xg[k] - hi[k];
        dhi[k] = xg[k] - lo[k];
    }
    emitter_cosines(dlo, dhi, c);
    float face[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) face[f] = __uint_as_float(__ldg(rec + f));
    float sum = 0.0f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        w[f] = face[f] * c[f];
        sum += w[f];
    }
    if (sum <= 0.0f) {
        sum = 0.0f;
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            w[f] = face[f];
            sum += w[f];
        }
    }
    return sum;
}

struct LightPoint
{
    float position[3];
    float normal[3];
    float pdf;
    uint32_t block;
    uint32_t group;
    uint32_t entry;
    uint32_t tree;  // 0: the world's light set, 1: the entities' (SceneView::dyn)
};

// kEntities: the scene may have a second (entity) light tree; without it only tree 0 is
// evaluated and tree 1's draw is consumed (the same results for a scene without entity lights).
template <bool kEntities = true>
__device__ __forceinline__ bool light_sample(const SceneView& s, const float x[3], const float n[3], uint32_t rng, LightPoint& p)
{
    float pdf_brick = 1.0f;
    // The tree (one draw per tree; an empty tree's importance and power are never positive, so
    // it only consumes its draw).
    uint32_t root, k;
    {
        Pick pk = {0, 0, 0, 0, kNone, kNone};
        uint32_t roots[2] = {kNone, kNone};
#pragma unroll
        for (uint32_t t = 0; t < 2; ++t) {
            Summary sm;
            if (kEntities || t == 0) tree_summary(s, t, sm, roots[t]);
            const float u = lt_random_float(rng);
            if (roots[t] != kNone) pick_add(pk, importance(x, n, sm.lo, sm.hi, sm.face), power6(sm.face), t, u);
        }
        float prob;
        k = pick_end(pk, prob);
        if (k == kNone) return false;
        pdf_brick *= prob;
        root = roots[k];
    }
    const SceneView& L = (kEntities && k != 0) ? *s.dyn : s;
    p.tree = k;
    // Down the 4-wide nodes. Every slot's importance is computed by every lane (empty slots
    // hold zero summaries and are skipped by the pick), so the lanes stay converged.
    uint32_t leaf = kNone;
    uint32_t node = root;
    for (uint32_t depth = 0; depth < 64; ++depth) {
        const LightBvhNode* nd = L.nodes + node;
        const uint4 ch = __ldg(reinterpret_cast<const uint4*>(nd->child));
        uint32_t chosen;
        if (child_count(ch) == 1) {
            chosen = ch.x;
        } else {
            Pick pk = {0, 0, 0, 0, kNone, kNone};
            for (uint32_t q = 0; q < 4; ++q) {
                Summary sm;
                node_slot(nd, q, sm);
                const float imp = importance(x, n, sm.lo, sm.hi, sm.face);
                if (__ldg(&nd->child[q]) != kNone) pick_add(pk, imp, power6(sm.face), q, lt_random_float(rng));
            }
            float prob;
            const uint32_t q = pick_end(pk, prob);
            if (q == kNone) return false;
            pdf_brick *= prob;
            chosen = __ldg(&nd->child[q]);
        }
        if (chosen & kChildLeafBit) {
            leaf = chosen & ~kChildLeafBit;
            break;
        }
        node = chosen;
    }
    if (leaf == kNone) return false;
    const uint2 owner = __ldg(reinterpret_cast<const uint2*>(&L.leaves[leaf].group));
    const uint32_t group = owner.x, entry = owner.y;
    p.group = group;
    p.entry = entry;
    const uint2 row = __ldg(reinterpret_cast<const uint2*>(L.group_rows + 8ull * group));
    if (row.y == 0) return false;
    const uint32_t* block = L.heap + 4ull * row.x;
    const uint32_t* rec = block + 4ull * __ldg(block + 4 + 4 * entry + 2);
    float w[6];
    const float sum = family_weights(L, group, rec, x, w);
    if (sum <= 0.0f) return false;
    const float u = lt_random_float(rng) * sum;
    uint32_t f = kNone, last = 0;
    float cumulative = 0.0f;
#pragma unroll
    for (uint32_t g = 0; g < 6; ++g) {
        if (w[g] > 0.0f) {
            last = g;
            cumulative += w[g];
            if (f == kNone && u < cumulative) f = g;
        }
    }
    f = f == kNone ? last : f;
    // The entries of families before f, the count and weight of f (selects, no local array).
    const uint32_t counts_lo = __ldg(rec + 10), counts_hi = __ldg(rec + 11);
    uint32_t first = 0, count = 0;
    float wf = 0.0f;
#pragma unroll
    for (uint32_t g = 0; g < 6; ++g) {
        const uint32_t c = ((g < 3 ? counts_lo : counts_hi) >> (10 * (g % 3))) & 0x3FFu;
        if (g < f) first += c;
        if (g == f) {
            count = c;
            wf = w[g];
        }
    }
    if (count == 0 || wf <= 0.0f) return false;
    uint32_t ei = (uint32_t)(lt_random_float(rng) * (float)count);
    ei = ei > count - 1u ? count - 1u : ei;
    const uint32_t ent = __ldg(rec + 12 + first + ei);
    const uint32_t vi = ent & 0x1FFu;
    const uint32_t gs = L.group_shift, gm = (1u << gs) - 1u;
    const uint32_t pos = __ldg(rec + 8);
    const uint32_t voxel[3] = {(pos & gm) * 8 + (vi & 7u), ((pos >> gs) & gm) * 8 + ((vi >> 3) & 7u),
                               ((pos >> (2 * gs)) & gm) * 8 + (vi >> 6)};
    const GroupFrame* fr = L.frames + group;
    const uint32_t axis = f >> 1;
    const float a = lt_random_float(rng);
    const float b = lt_random_float(rng);
    // The face's own axis gets the face offset, the next axis a, the one after b.
    const float off = (f & 1) ? 0.0f : 1.0f;
    float local[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        const uint32_t rel = ((uint32_t)q + 3u - axis) % 3u;
        local[q] = (__ldg(&fr->origin[q]) + (float)voxel[q]) + (rel == 0 ? off : (rel == 1 ? a : b));
    }
    const float dn[3] = {f == 0 ? 1.0f : (f == 1 ? -1.0f : 0.0f), f == 2 ? 1.0f : (f == 3 ? -1.0f : 0.0f),
                         f == 4 ? 1.0f : (f == 5 ? -1.0f : 0.0f)};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const float R0 = __ldg(&fr->rot[3 * r]), R1 = __ldg(&fr->rot[3 * r + 1]), R2 = __ldg(&fr->rot[3 * r + 2]);
        p.position[r] = R0 * local[0] + R1 * local[1] + R2 * local[2] + __ldg(&fr->trans[r]);
        p.normal[r] = R0 * dn[0] + R1 * dn[1] + R2 * dn[2];
    }
    p.pdf = wf / sum / (float)count * pdf_brick;
    p.block = ent >> 16;
    return true;
}

// LightTreeFindLightFace (caelix_light_tree.hlsl:853-935): the face of a voxel whose material code
// is in the light code set, in a brick with a light record.
__device__ __noinline__ bool find_light_face(const SceneView& s, const float x[3], uint32_t group, const uint32_t v[3], uint32_t face,
                                uint32_t block_value, uint32_t& entry_out, uint32_t& leaf_out, float& in_brick)
{
    entry_out = kNone;
    leaf_out = kNone;
    in_brick = 0.0f;
    const uint32_t code = material_code(block_value, s.enc);
    if (!((__ldg(s.light_codes + (code >> 5)) >> (code & 31)) & 1u) || face > 5) return false;
    const uint2 row = __ldg(reinterpret_cast<const uint2*>(s.group_rows + 8ull * group));
    if (row.y == 0) return false;
    const uint32_t* block = s.heap + 4ull * row.x;
    const uint32_t count_r = __ldg(block);
    const uint32_t gs = s.group_shift, gm = (1u << gs) - 1u;
    auto morton = [](uint32_t a, uint32_t b, uint32_t c) {
        auto part = [](uint32_t q) {
            q &= 0x3FFu;
            q = (q | (q << 16)) & 0x030000FFu;
            q = (q | (q << 8)) & 0x0300F00Fu;
            q = (q | (q << 4)) & 0x030C30C3u;
            q = (q | (q << 2)) & 0x09249249u;
            return q;
        };
        return part(a) | (part(b) << 1) | (part(c) << 2);
    };
    const uint32_t key = morton(v[0] / 8, v[1] / 8, v[2] / 8);
    uint32_t lo = 0, hi = count_r, entry = kNone;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t pos = __ldg(block + 4 + 4 * mid);
        const uint32_t mk = morton(pos & gm, (pos >> gs) & gm, (pos >> (2 * gs)) & gm);
        if (mk == key) {
            entry = mid;
            break;
        }
        if (mk < key) lo = mid + 1;
        else hi = mid;
    }
    if (entry == kNone) return false;
    entry_out = entry;
    const uint32_t* rec = block + 4ull * __ldg(block + 4 + 4 * entry + 2);
    float w[6];
    const float sum = family_weights(s, group, rec, x, w);
    const uint32_t counts_lo = __ldg(rec + 10), counts_hi = __ldg(rec + 11);
    uint32_t first = 0, count = 0;
    float wf = 0.0f;
#pragma unroll
    for (uint32_t g = 0; g < 6; ++g) {
        const uint32_t c = ((g < 3 ? counts_lo : counts_hi) >> (10 * (g % 3))) & 0x3FFu;
        if (g < face) first += c;
        if (g == face) {
            count = c;
            wf = w[g];
        }
    }
    if (sum <= 0.0f || wf <= 0.0f || count == 0) return false;
    const uint32_t vi = (v[0] % 8) | ((v[1] % 8) << 3) | ((v[2] % 8) << 6);
    uint32_t a = 0, b = count;
    bool found = false;
    while (a < b) {
        const uint32_t mid = (a + b) >> 1;
        const uint32_t ev = __ldg(rec + 12 + first + mid) & 0x1FFu;
        if (ev == vi) {
            found = true;
            break;
        }
        if (ev < vi) a = mid + 1;
        else b = mid;
    }
    if (!found) return false;
    in_brick = (wf / sum) / (float)count;
    const uint32_t bvh_leaf = __ldg(block + 4 + 4 * entry + 3);
    if (bvh_leaf != kNone) {
        const uint32_t leaf = bvh_leaf & 0x7FFFFFFFu;
        const uint2 owner = __ldg(reinterpret_cast<const uint2*>(&s.leaves[leaf].group));
        if (owner.x == group && owner.y == entry) leaf_out = bvh_leaf;
    }
    return true;
}

// The draw probability of entry `entry` of group `group` of light set k (L).
__device__ float brick_pdf(const SceneView& s, const SceneView& L, const float x[3], const float n[3], uint32_t group,
                           uint32_t entry, uint32_t k)
{
    const uint2 row = __ldg(reinterpret_cast<const uint2*>(L.group_rows + 8ull * group));
    if (row.y == 0) return 0.0f;
    const uint32_t* block = L.heap + 4ull * row.x;
    if (entry >= __ldg(block)) return 0.0f;
    const uint32_t bvh_leaf = __ldg(block + 4 + 4 * entry + 3);
    if (bvh_leaf == kNone) return 0.0f;
    const uint32_t leaf = bvh_leaf & 0x7FFFFFFFu;
    const uint2 owner = __ldg(reinterpret_cast<const uint2*>(&L.leaves[leaf].group));
    if (owner.x != group || owner.y != entry) return 0.0f;
    return leaf_probability(s, L, leaf, x, n, k);
}

// ---- integrator ----
__device__ __forceinline__ float mis_weight(float p_area, const float n_r[3], const float w[3], float d, float cos_l,
                                            bool nee_side)
{
    const float p_sa = cos_l > 0.0f ? p_area * (d * d) / cos_l : 0.0f;
    const float p_bsdf = hmax(0.0f, dot3(n_r, w)) * (1.0f / 3.1415926535f);
    if (!(cos_l > 0.0f) || !(p_sa <= 3.0e38f)) return nee_side ? 1.0f : 0.0f;
    const float sum = p_sa + p_bsdf;
    if (!(sum > 0.0f)) return nee_side ? 0.0f : 1.0f;
    return (nee_side ? p_sa : p_bsdf) / sum;
}

struct Counters
{
    uint32_t primary, bounce, shadow;
};

// The part of the light-tree NEE (caelix_light_nee.hlsl:20-34 with caelix_path_trace.hlsl:245-449)
// before its shadow ray: draws a light point, weighs it (MIS balance heuristic, near field) and
// returns true with the shadow ray and the radiance it carries if unoccluded, or false when the
// vertex gets no light (no ray is traced then).
struct ShadowRay
{
    float dir[3];
    float t_max;
    float value[3];      // the contribution if the ray is unoccluded
    float dvalue_de[3];  // d value / d (the lamp brick's power), the sampling factors held fixed
    uint32_t brick;      // the lamp brick of the world (kNone for an entity's lamp)
};

// The material table entry of a block value: albedo and emission (without the brick's power).
__device__ __forceinline__ void material_of(const SceneView& s, uint32_t block, float albedo[3], float emission[3])
{
    const uint32_t code = material_code(block, s.enc);
    const float4 a = __ldg(s.materials + 2ull * code);
    const float4 e = __ldg(s.materials + 2ull * code + 1);
    albedo[0] = a.x;
    albedo[1] = a.y;
    albedo[2] = a.z;
    emission[0] = e.x;
    emission[1] = e.y;
    emission[2] = e.z;
}

template <bool kEntities = true>
__device__ __forceinline__ bool nee_prepare(const SceneView& s, const float x[3], const float n[3], uint32_t& light_rng,
                                            ShadowRay& r)
{
    const uint32_t point_seed = random_u32(light_rng);
    LightPoint p;
    if (!light_sample<kEntities>(s, x, n, point_seed, p) || !(p.pdf > 0.0f)) return false;
    const float d[3] = {p.position[0] - x[0], p.position[1] - x[1], p.position[2] - x[2]};
    const float d2 = dot3(d, d);
    const float dist = sqrtf(d2);
    if (!(dist >= kNearField)) return false;
    const float w[3] = {d[0] / dist, d[1] / dist, d[2] / dist};
    const float cos_r = dot3(n, w);
    const float cos_l = -dot3(p.normal, w);
    if (!(cos_r > 0.0f) || !(cos_l > 0.0f)) return false;
    float scale = (cos_r * (1.0f / kPi)) * (cos_l / d2) / p.pdf;
    scale *= mis_weight(p.pdf, n, w, dist, cos_l, true);
    const SceneView& L = (kEntities && p.tree != 0) ? *s.dyn : s;
    const uint2 row = __ldg(reinterpret_cast<const uint2*>(L.group_rows + 8ull * p.group));
    const uint32_t brick = __ldg(L.heap + 4ull * row.x + 4 + 4 * p.entry + 1);
    // LampEmission: the table's emission of the lamp voxel's code (the scene's table, shared by its
    // entities) times its brick's power.
    float al[3], em[3];
    material_of(s, p.block, al, em);
    const float P = __ldg(L.power + brick);
    float contribution[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) contribution[c] = (em[c] * P) * scale;
    const float lum = contribution[0] * 0.2126f + contribution[1] * 0.7152f + contribution[2] * 0.0722f;
    const float w_lamp = lum * hmax(0.05f, 1.0f);
    const float w_sum = 0.0f + w_lamp;
    if (!(w_sum > 0.0f)) return false;
    const float t_max = dist - 2.0f * kPushOff;
    if (!(t_max > 0.0f)) return false;
    r.dir[0] = w[0];
    r.dir[1] = w[1];
    r.dir[2] = w[2];
    r.t_max = t_max;
    const float k = w_sum / w_lamp;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        r.value[c] = contribution[c] * k;
        r.dvalue_de[c] = em[c] * (scale * k);
    }
    // A world brick's power (tree 0 also holds static entities' bricks, after the world's).
    r.brick = ((!kEntities || p.tree == 0) && brick < s.brick_count) ? brick : kNone;
    return true;
}

__device__ __noinline__ float lamp_hit_weight(const SceneView& s, uint32_t segment_light, const Hit& h, const float origin[3],
                                 const float dir[3], const float seg_n[3])
{
    if (segment_light == 0u || h.t < kNearField) return 1.0f;
    // The light set of the hit: tree 0's for the world and static entities, the dynamic one for
    // dynamic entities (an entity's groups from its group base; the voxel from the entity-local
    // hit point and face normal).
    const uint32_t face = (uint32_t)(__ffs(h.attrib & 0x3Fu) - 1);
    const bool entity = (h.attrib & kEntityHit) != 0;
    const uint32_t tree = entity ? __ldg(&s.entities[h.group >> kEntityShift].tree) : 0u;
    if (tree > 1u || (tree == 1u && !s.dyn)) return 1.0f;
    const SceneView& L = tree == 1u ? *s.dyn : s;
    const uint32_t group = entity ? __ldg(&s.entities[h.group >> kEntityShift].group_base) + (h.group & kEntityGroupMask)
                                  : h.group;
    float nl[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) nl[k] = entity ? ((uint32_t)k == (face >> 1) ? ((face & 1u) ? -1.0f : 1.0f) : 0.0f)
                                               : h.normal[k];
    const GroupFrame* fr = L.frames + group;
    uint32_t vig[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int32_t voxel = (int32_t)floorf(h.object_hit[k] - 0.25f * nl[k]);
        vig[k] = (uint32_t)(voxel - (int32_t)__ldg(&fr->origin[k]));
    }
    const uint32_t block = (h.attrib >> 16) & 0xFFFFu;
    uint32_t entry, leaf;
    float in_brick;
    if (!find_light_face(L, origin, group, vig, face, block, entry, leaf, in_brick) || leaf == kNone) return 1.0f;
    const float cos_l = -dot3(h.normal, dir);
    const float p_area = brick_pdf(s, L, origin, seg_n, group, entry, tree) * in_brick;
    return mis_weight(p_area, seg_n, dir, h.t, cos_l, false);
}

// The vertex of a hit: its material (the scene's table; an entity's bricks share it), its emission
// (the table's times the brick's power) and the Lambertian bounce.
template <bool kEntities = true>
__device__ __forceinline__ void shade(const SceneView& s, const Hit& h, const float ray_o[3], const float ray_d[3],
                                      uint32_t& rng, float albedo[3], float emission[3], float origin[3], float dir[3])
{
    const uint32_t block = (h.attrib >> 16) & 0xFFFFu;
    material_of(s, block, albedo, emission);
    float P;
    if (kEntities && (h.attrib & kEntityHit)) {  // an entity brick's power
        const float* pw = s.entities[h.group >> kEntityShift].scene.power;
        P = pw ? __ldg(pw + h.record) : 0.0f;
    } else {
        P = __ldg(s.power + h.record);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) emission[c] *= P;
    (void)random01(rng);  // the lobe draw (specular chance 0)
    float u[3];
    random_unit_vector(rng, u);
    const float v[3] = {h.normal[0] + u[0], h.normal[1] + u[1], h.normal[2] + u[2]};
    const float dp3 = hmax(1.175494351e-38f, dot3(v, v));
    const float inv = 1.0f / sqrtf(dp3);
    float dd[3] = {v[0] * inv, v[1] * inv, v[2] * inv};
    if (!(dot3(dd, dd) > 0.0f)) {
        dd[0] = h.normal[0];
        dd[1] = h.normal[1];
        dd[2] = h.normal[2];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dir[k] = dd[k];
        origin[k] = (ray_o[k] + ray_d[k] * h.t) + kPushOff * h.normal[k];
    }
}

}  // namespace

}  // namespace cx
