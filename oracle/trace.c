/* Oracle of the trace path (TEST INFRASTRUCTURE ONLY; see oracle.h). Restates:
 *   brick DDA          shaders/render/caelix_brick_trace.hlsl:177-451 (CaelixTraceBrickPrimitiveCore,
 *                      CaelixTraceBrickRay, VRTJump / VRTStep, the normal-flag tie rule)
 *   scene traversal    shaders/render/caelix_scene_trace.hlsl:57-169, with the TLAS replaced by a
 *                      front-to-back DDA over the brick grid (brick occupancy bitmap + hash lookup);
 *                      the first brick in DDA order whose brick DDA reports a hit in [tmin, tmax)
 *                      is the closest hit (ties at a brick boundary go to the brick entered first)
 *   light tree draw    shaders/light/caelix_light_tree.hlsl:65-767 (PCG draws, importance,
 *                      reservoir picks, 4-wide descent, family CDF, entry, point on the face)
 *   light tree pdf     caelix_light_tree.hlsl:514-608, 769-777, 853-949
 *   integrator         shaders/render/caelix_path_trace.hlsl:245-449 (LampCandidate, NextEventAtVertex,
 *                      LampHitWeight), :737-978 (TracePath), caelix_light_nee.hlsl:20-34 (MIS),
 *                      caelix_shading.hlsl:267-307 (ShadeVoxelHit, opaque Lambertian: metallic 0,
 *                      smoothness 0), caelix_random.hlsl (PcgHash, InitRandom, xorshift32,
 *                      RandomUnitVector), common/caelix_frame.hlsl:164-171 (camera ray)
 * in the benchmark scenes' configuration: Lambertian voxels (the material table's albedo; the
 * emission of a voxel = its table emission times its brick's power), light-tree NEE with MIS, no
 * sun, black sky, no fog, bounce NEE probability 1; entities under rigid transforms, their lights
 * in the second light tree (the reference's dynamic tree); either block encoding.
 *
 * Arithmetic: IEEE fp32, no contraction, HLSL operation order. Two definitions are this
 * project's: sin/cos of RandomUnitVector (Cody-Waite reduction by pi/2 and Taylor polynomials to
 * degree 9 / 10, the same operations as the CUDA path) and normalize / SafeNormalize as
 * v * (1 / sqrt(dot(v, v))).
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define RAY_TMAX 1e30f
#define BOUNCE_TMAX 1e4f
#define PUSH_OFF 0.002f
#define NEAR_FIELD 8.0f
#define K_PI 3.1415926535f
#define K_TWO_PI 6.283185307f

static float hmin(float a, float b) { return b < a ? b : a; }
static float hmax(float a, float b) { return b > a ? b : a; }
static float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* ---- random streams (caelix_random.hlsl, caelix_light_tree.hlsl:65-76) ---- */

static uint32_t pcg_hash(uint32_t v)
{
    const uint32_t state = v * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}

static uint32_t init_random(uint32_t px, uint32_t py, uint32_t seed)
{
    const uint32_t s = pcg_hash(px ^ (py << 16) ^ (seed * 0x9E3779B9u));
    return s != 0u ? s : 0x9E3779B9u;
}

static uint32_t random_u32(uint32_t* state)
{
    *state ^= *state << 13;
    *state ^= *state >> 17;
    *state ^= *state << 5;
    return *state;
}

static float random01(uint32_t* state) { return (float)(random_u32(state) >> 8) * (1.0f / 16777216.0f); }

static uint32_t lt_random(uint32_t* rng)
{
    *rng = *rng * 747796405u + 2891336453u;
    const uint32_t word = ((*rng >> ((*rng >> 28) + 4u)) ^ *rng) * 277803737u;
    return (word >> 22) ^ word;
}

static float lt_random_float(uint32_t* rng) { return (float)(lt_random(rng) >> 8) * (1.0f / 16777216.0f); }

/* sin and cos of a in [0, 2 pi]: a = k pi/2 + r (Cody-Waite, two-part pi/2), Taylor polynomials on
 * |r| <= pi/4 (Horner), quadrant selection. */
static void sincos_cw(float a, float* s, float* c)
{
    const float k = floorf(a * 0.636619772f + 0.5f);
    const float r = (a - k * 1.57079637f) - k * -4.37113883e-8f;
    const float r2 = r * r;
    const float sp = r + r * r2 * (-0.166666667f + r2 * (0.00833333333f + r2 * (-0.000198412698f + r2 * 2.75573192e-6f)));
    const float cp = 1.0f + r2 * (-0.5f + r2 * (0.0416666667f + r2 * (-0.00138888889f + r2 * (2.48015873e-5f + r2 * -2.75573192e-7f))));
    const int q = ((int)k) & 3;
    *s = q == 0 ? sp : (q == 1 ? cp : (q == 2 ? -sp : -cp));
    *c = q == 0 ? cp : (q == 1 ? -sp : (q == 2 ? -cp : sp));
}

void oc_sincos(float a, float* s, float* c) { sincos_cw(a, s, c); }

static void random_unit_vector(uint32_t* rng, float out[3])
{
    const float u = random01(rng);
    const float v = random01(rng);
    const float a = u * K_TWO_PI;
    const float y = v * 2.0f - 1.0f;
    const float sy = sqrtf(hmax(1.0f - y * y, 0.0f));
    float sa, ca;
    sincos_cw(a, &sa, &ca);
    out[0] = sa * sy;
    out[1] = y;
    out[2] = ca * sy;
}

/* ---- brick DDA (caelix_brick_trace.hlsl) ---- */

static float safe_inv_axis(float d)
{
    if (fabsf(d) >= 1e-20f) return 1.0f / d;
    return d < 0.0f ? -1.0f / 1e-20f : 1.0f / 1e-20f;
}

static void vrt_step(int cell[3], const float t_start[3], const float origin[3], const float dir[3],
                     const float inv[3])
{
    float side[3];
    for (int k = 0; k < 3; ++k) side[k] = t_start[k] + (float)cell[k] * inv[k];
    const float tmin = hmin(hmin(side[0], side[1]), side[2]) + 0.0001f;
    for (int k = 0; k < 3; ++k) cell[k] = (int)floorf(origin[k] + tmin * dir[k]);
}

static uint32_t normal_flags(uint32_t index, const int cell[3], const float t_start[3], const float dir[3],
                             const float inv[3], uint32_t entry_flags, float* T)
{
    if (index == 0u) {
        *T = 0.0f;
        return entry_flags;
    }
    float side[3];
    for (int k = 0; k < 3; ++k) side[k] = t_start[k] + (float)cell[k] * inv[k];
    const float t = hmin(hmin(side[0], side[1]), side[2]);
    *T = t;
    const int mx = side[0] <= t + 0.0001f;
    const int my = side[1] <= t + 0.0001f;
    const uint32_t x_use = mx ? 0xFFFFFFFFu : 0u;
    const uint32_t y_use = (my ? 0xFFFFFFFFu : 0u) & ~x_use;
    const uint32_t z_use = ~(x_use | y_use);
    const uint32_t xf = dir[0] > 0.0f ? 2u : 1u;
    const uint32_t yf = dir[1] > 0.0f ? 8u : 4u;
    const uint32_t zf = dir[2] > 0.0f ? 32u : 16u;
    return (xf & x_use) | (yf & y_use) | (zf & z_use);
}

static float brick_ray(const uint32_t* rec, const float entry[3], const float dir[3], float entry_t,
                       uint32_t entry_coarse, uint32_t encoding, uint32_t* attrib)
{
    const uint32_t opaque = encoding == OC_ENCODING_PACKED ? 0xC000u : 0x8000u;
    const uint32_t fshift = encoding == OC_ENCODING_PACKED ? 8u : 9u;
    float inv[3], t_start[3], origin[3];
    int cell[3], prev[3];
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
            for (int k = 0; k < 3; ++k) cell[k] = dir[k] < 0.0f ? (cell[k] & ~3) : (cell[k] | 3);
            memcpy(prev, cell, sizeof(prev));
            vrt_step(cell, t_start, origin, dir, inv);
            continue;
        }
        const uint64_t occ = (uint64_t)rec[2 + 2 * cbit] | ((uint64_t)rec[3 + 2 * cbit] << 32);
        const uint32_t mbit = (uint32_t)((cell[0] & 3) | ((cell[1] & 3) << 2) | ((cell[2] & 3) << 4));
        if (occ & (1ull << mbit)) {
            const uint32_t w = rec[18 + (cell[0] >> 1) + (cell[1] << 2) + (cell[2] << 5)];
            const uint32_t blk = (w >> ((cell[0] & 1) << 4)) & 0xFFFFu;
            float T;
            const uint32_t nf = normal_flags(step, prev, t_start, dir, inv, entry_coarse >> 26, &T);
            int term = (blk & opaque) != 0;
            if (!term) term = (step == 0 && entry_t == 0.0f) ? 0 : ((((blk >> fshift) & 63u) & nf) != 0);
            if (term) {
                *attrib = (blk << 16) | (((uint32_t)cell[0] | ((uint32_t)cell[1] << 3) | ((uint32_t)cell[2] << 6)) << 6) | nf;
                return entry_t + T;
            }
        }
        memcpy(prev, cell, sizeof(prev));
        vrt_step(cell, t_start, origin, dir, inv);
    }
    *attrib = 0u;
    return 0.0f;
}

static float brick_primitive(const uint32_t* rec, const float o[3], const float d[3], float t_current,
                             const float brick_origin[3], uint32_t encoding, uint32_t* attrib)
{
    const uint32_t tb = rec[1];
    const float tmin_v[3] = {(float)(tb & 7u), (float)((tb >> 3) & 7u), (float)((tb >> 6) & 7u)};
    const float tmax_v[3] = {(float)((tb >> 9) & 7u) + 1.0f, (float)((tb >> 12) & 7u) + 1.0f,
                             (float)((tb >> 15) & 7u) + 1.0f};
    float tmin[3], tmax[3];
    for (int k = 0; k < 3; ++k) {
        const float inv = 1.0f / d[k];
        const float t0 = (brick_origin[k] + tmin_v[k] - o[k]) * inv;
        const float t1 = (brick_origin[k] + tmax_v[k] - o[k]) * inv;
        tmin[k] = hmin(t0, t1);
        tmax[k] = hmax(t0, t1);
    }
    const float largest = hmax(hmax(tmin[0], tmin[1]), tmin[2]);
    const float smallest = hmin(hmin(tmax[0], tmax[1]), tmax[2]);
    if (largest > smallest || smallest < 0.0f || largest > t_current) {
        *attrib = 0u;
        return 0.0f;
    }
    const float t = hmax(0.0f, largest);
    float entry[3];
    for (int k = 0; k < 3; ++k) entry[k] = o[k] + d[k] * t - brick_origin[k];
    uint32_t nf;
    if (largest == tmin[0]) nf = d[0] > 0.0f ? 2u : 1u;
    else if (largest == tmin[1]) nf = d[1] > 0.0f ? 8u : 4u;
    else nf = d[2] > 0.0f ? 32u : 16u;
    return brick_ray(rec, entry, d, t, (nf << 26) | ((rec[0] >> 16) & 0xFFu), encoding, attrib);
}

/* ---- scene traversal: front-to-back DDA over the brick grid ----
 * Cell c of axis k is brick key origin[k] + c, voxels [8 (origin[k] + c), 8 (origin[k] + c + 1)). */

static oc_hit trace_grid(const oc_scene* s, const float o[3], const float d[3], float tmin_ray, float tmax_ray)
{
    oc_hit h;
    memset(&h, 0, sizeof(h));
    float inv[3], tnear = -3.0e38f, tfar = 3.0e38f;
    for (int k = 0; k < 3; ++k) {
        inv[k] = safe_inv_axis(d[k]);
        const float t0 = ((float)(8 * s->origin[k]) - o[k]) * inv[k];
        const float t1 = ((float)(8 * (s->origin[k] + (int)s->grid[k])) - o[k]) * inv[k];
        tnear = hmax(tnear, hmin(t0, t1));
        tfar = hmin(tfar, hmax(t0, t1));
    }
    const float t_enter = hmax(tnear, tmin_ray);
    const float t_exit = hmin(tfar, tmax_ray);
    if (!(t_enter <= t_exit)) return h;
    int cell[3], step[3];
    for (int k = 0; k < 3; ++k) {
        const float p = o[k] + d[k] * t_enter;
        int c = (int)floorf(p * 0.125f) - s->origin[k];
        if (c < 0) c = 0;
        if (c > (int)s->grid[k] - 1) c = (int)s->grid[k] - 1;
        cell[k] = c;
        step[k] = d[k] >= 0.0f ? 1 : -1;
    }
    const uint32_t limit = s->grid[0] + s->grid[1] + s->grid[2] + 3;
    for (uint32_t it = 0; it < limit; ++it) {
        const uint64_t lin = (uint64_t)cell[0] + s->grid[0] * ((uint64_t)cell[1] + (uint64_t)s->grid[1] * cell[2]);
        if (s->bitmap[lin >> 5] & (1u << (lin & 31))) {
            const int32_t key[3] = {s->origin[0] + cell[0], s->origin[1] + cell[1], s->origin[2] + cell[2]};
            const uint32_t r = oc_hash_lookup(s, key[0], key[1], key[2]);
            if (r != OC_NONE) {
                const float bo[3] = {(float)(key[0] * 8), (float)(key[1] * 8), (float)(key[2] * 8)};
                uint32_t attrib;
                const float t = brick_primitive(s->records + (size_t)r * OC_RECORD_WORDS, o, d, tmax_ray, bo,
                                                s->encoding, &attrib);
                if (attrib != 0u && t >= tmin_ray && t < tmax_ray) {
                    h.hit = 1;
                    h.t = t;
                    h.attrib = attrib;
                    h.record = r;
                    const uint32_t gs = s->group_shift;
                    h.group = ((uint32_t)cell[0] >> gs) +
                              s->groups[0] * (((uint32_t)cell[1] >> gs) + s->groups[1] * ((uint32_t)cell[2] >> gs));
                    const uint32_t f = (uint32_t)__builtin_ctz(attrib & 0x3Fu);
                    h.normal[0] = f == 0 ? 1.0f : (f == 1 ? -1.0f : 0.0f);
                    h.normal[1] = f == 2 ? 1.0f : (f == 3 ? -1.0f : 0.0f);
                    h.normal[2] = f == 4 ? 1.0f : (f == 5 ? -1.0f : 0.0f);
                    for (int k = 0; k < 3; ++k) h.object_hit[k] = o[k] + d[k] * t;
                    return h;
                }
            }
        }
        /* Next cell: the axis whose boundary comes first (ties: x, then y, then z). */
        float tn[3];
        for (int k = 0; k < 3; ++k)
            tn[k] = ((float)((s->origin[k] + cell[k] + (step[k] > 0 ? 1 : 0)) * 8) - o[k]) * inv[k];
        int axis = 0;
        if (tn[1] < tn[axis]) axis = 1;
        if (tn[2] < tn[axis]) axis = 2;
        if (tn[axis] > t_exit) break;
        cell[axis] += step[axis];
        if (cell[axis] < 0 || cell[axis] >= (int)s->grid[axis]) break;
    }
    return h;
}

void oc_entity_rows(const float q[4], float rot[9])
{
    const double n = sqrt((double)q[0] * q[0] + (double)q[1] * q[1] + (double)q[2] * q[2] + (double)q[3] * q[3]);
    const double x = q[0] / n, y = q[1] / n, z = q[2] / n, w = q[3] / n;
    const double r[9] = {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * w), 2.0 * (x * z + y * w),
                         2.0 * (x * y + z * w), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * w),
                         2.0 * (x * z - y * w), 2.0 * (y * z + x * w), 1.0 - 2.0 * (x * x + y * y)};
    for (int i = 0; i < 9; ++i) rot[i] = (float)r[i];
}

oc_hit oc_trace_ray(const oc_scene* s, const float o[3], const float d[3], float tmin_ray, float tmax_ray)
{
    oc_hit h = trace_grid(s, o, d, tmin_ray, tmax_ray);
    for (uint32_t e = 0; e < s->entity_count; ++e) {
        const oc_entity* E = &s->entities[e];
        const float* R = E->rot;
        const float q[3] = {o[0] - E->pos[0], o[1] - E->pos[1], o[2] - E->pos[2]};
        float ol[3], dl[3];
        for (int k = 0; k < 3; ++k) {
            ol[k] = R[k] * q[0] + R[3 + k] * q[1] + R[6 + k] * q[2];
            dl[k] = R[k] * d[0] + R[3 + k] * d[1] + R[6 + k] * d[2];
        }
        const oc_hit he = trace_grid(E->scene, ol, dl, tmin_ray, h.hit ? h.t : tmax_ray);
        if (!he.hit) continue;
        h = he;
        h.attrib |= OC_ENTITY_HIT;
        h.group = (e << 24) | he.group;
        const uint32_t f = (uint32_t)__builtin_ctz(he.attrib & 0x3Fu);
        const float sign = (f & 1u) ? -1.0f : 1.0f;
        float v[3];
        for (int i = 0; i < 3; ++i) v[i] = R[3 * i + (f >> 1)] * sign;
        const float inv = 1.0f / sqrtf(dot3(v, v));
        for (int i = 0; i < 3; ++i) h.normal[i] = v[i] * inv;
    }
    return h;
}

/* ---- light tree device API (caelix_light_tree.hlsl) ---- */

static float power6(const float f[6]) { return f[0] + f[1] + f[2] + f[3] + f[4] + f[5]; }

static void emitter_cosines(const float dlo[3], const float dhi[3], float c[6])
{
    float cl[3], c2[3];
    for (int k = 0; k < 3; ++k) {
        cl[k] = hmin(hmax(0.0f, dlo[k]), dhi[k]);
        c2[k] = cl[k] * cl[k];
    }
    const float all2 = c2[0] + c2[1] + c2[2];
    for (int a = 0; a < 3; ++a) {
        const float others = all2 - c2[a];
        c[2 * a] = dhi[a] > 0.0f ? dhi[a] / sqrtf(dhi[a] * dhi[a] + others) : 0.0f;
        c[2 * a + 1] = dlo[a] < 0.0f ? -dlo[a] / sqrtf(dlo[a] * dlo[a] + others) : 0.0f;
    }
}

float oc_importance(const float x[3], const float n[3], const float lo[3], const float hi[3], const float face[6])
{
    float dlo[3], dhi[3], c[6];
    for (int k = 0; k < 3; ++k) {
        dlo[k] = x[k] - hi[k];
        dhi[k] = x[k] - lo[k];
    }
    emitter_cosines(dlo, dhi, c);
    float e = 0.0f;
    for (int f = 0; f < 6; ++f) e += face[f] * c[f];
    if (e <= 0.0f) return 0.0f;
    float centre[3], half[3];
    for (int k = 0; k < 3; ++k) {
        centre[k] = 0.5f * (lo[k] + hi[k]);
        half[k] = 0.5f * (hi[k] - lo[k]);
    }
    float cr = 1.0f;
    if (n[0] != 0.0f || n[1] != 0.0f || n[2] != 0.0f) {
        const float cx[3] = {centre[0] - x[0], centre[1] - x[1], centre[2] - x[2]};
        const float an[3] = {fabsf(n[0]), fabsf(n[1]), fabsf(n[2])};
        const float m = dot3(n, cx) + dot3(an, half);
        if (m <= 0.0f) return 0.0f;
        float q[3];
        for (int k = 0; k < 3; ++k) q[k] = hmax(hmax(lo[k] - x[k], x[k] - hi[k]), 0.0f);
        const float dmin = sqrtf(dot3(q, q));
        cr = dmin > 0.0f ? hmin(1.0f, m / dmin) : 1.0f;
    }
    const float tc[3] = {x[0] - centre[0], x[1] - centre[1], x[2] - centre[2]};
    const float extent2 = dot3(half, half);
    const float d2 = hmax(dot3(tc, tc), hmax(1.0f, extent2));
    return e * cr / d2;
}

typedef struct pick {
    float sum_i, sum_p, weight_i, weight_p;
    uint32_t index_i, index_p;
} pick;

static void pick_add(pick* p, float importance, float power, uint32_t index, float u)
{
    if (importance > 0.0f) {
        p->sum_i += importance;
        if (u * p->sum_i < importance) {
            p->weight_i = importance;
            p->index_i = index;
        }
    }
    if (power > 0.0f) {
        p->sum_p += power;
        if (u * p->sum_p < power) {
            p->weight_p = power;
            p->index_p = index;
        }
    }
}

static uint32_t pick_end(const pick* p, float* probability)
{
    if (p->sum_i > 0.0f) {
        *probability = p->weight_i / p->sum_i;
        return p->index_i;
    }
    *probability = p->sum_p > 0.0f ? p->weight_p / p->sum_p : 0.0f;
    return p->sum_p > 0.0f ? p->index_p : OC_NONE;
}

static float pick_probability(float sum_i, float sum_p, float importance, float power)
{
    if (sum_i > 0.0f) return importance / sum_i;
    return sum_p > 0.0f ? power / sum_p : 0.0f;
}

static void node_slot(const oc_node* node, uint32_t s, oc_summary* out)
{
    memcpy(out->face, node->child_face[s], 24);
    memcpy(out->lo, node->child_lo[s], 12);
    memcpy(out->hi, node->child_hi[s], 12);
}

static uint32_t child_count(const oc_node* node)
{
    return (node->child[0] != OC_NONE) + (node->child[1] != OC_NONE) + (node->child[2] != OC_NONE) +
           (node->child[3] != OC_NONE);
}

/* The two trees' root summaries: tree 0 is the world's tree, tree 1 the entities' (empty
 * without entity lights). */
static const oc_light_tree* tree_of(const oc_scene* sc, const oc_light_tree* t, uint32_t k)
{
    return k == 0 ? t : sc->dyn_tree;
}

static const oc_scene* lights_of(const oc_scene* sc, uint32_t k) { return k == 0 ? sc : sc->dyn; }

static void tree_summary(const oc_scene* sc, const oc_light_tree* t, uint32_t k, oc_summary* s, uint32_t* root)
{
    memset(s, 0, sizeof(*s));
    *root = OC_NONE;
    const oc_light_tree* tk = k == 0 ? t : (sc->dyn ? sc->dyn_tree : NULL);
    if (tk && tk->header->root != OC_NONE) {
        *root = tk->header->root;
        *s = tk->header->s;
    }
}

static uint32_t choose_tree(const oc_scene* sc, const oc_light_tree* t, const float x[3], const float n[3],
                            uint32_t* rng, float* pdf, uint32_t* root)
{
    pick p = {0, 0, 0, 0, OC_NONE, OC_NONE};
    uint32_t roots[2];
    for (uint32_t k = 0; k < 2; ++k) {
        oc_summary s;
        tree_summary(sc, t, k, &s, &roots[k]);
        pick_add(&p, oc_importance(x, n, s.lo, s.hi, s.face), power6(s.face), k, lt_random_float(rng));
    }
    float prob;
    const uint32_t k = pick_end(&p, &prob);
    *root = k != OC_NONE ? roots[k] : OC_NONE;
    if (k != OC_NONE) *pdf *= prob;
    return k;
}

static float tree_probability(const oc_scene* sc, const oc_light_tree* t, const float x[3], const float n[3],
                              uint32_t target)
{
    float sum_i = 0.0f, sum_p = 0.0f, imp_t = 0.0f, pow_t = 0.0f;
    for (uint32_t k = 0; k < 2; ++k) {
        oc_summary s;
        uint32_t root;
        tree_summary(sc, t, k, &s, &root);
        const float imp = oc_importance(x, n, s.lo, s.hi, s.face);
        const float pw = power6(s.face);
        sum_i += imp > 0.0f ? imp : 0.0f;
        sum_p += pw > 0.0f ? pw : 0.0f;
        if (k == target) {
            imp_t = imp;
            pow_t = pw;
        }
    }
    return pick_probability(sum_i, sum_p, imp_t, pow_t);
}

static uint32_t choose_leaf(const oc_light_tree* t, uint32_t root, const float x[3], const float n[3], uint32_t* rng,
                            float* pdf)
{
    uint32_t node = root;
    for (uint32_t depth = 0; depth < 64; ++depth) {
        const oc_node* nd = &t->nodes[node];
        uint32_t chosen;
        if (child_count(nd) == 1) {
            chosen = nd->child[0];
        } else {
            pick p = {0, 0, 0, 0, OC_NONE, OC_NONE};
            for (uint32_t s = 0; s < 4; ++s) {
                if (nd->child[s] == OC_NONE) continue;
                oc_summary sm;
                node_slot(nd, s, &sm);
                pick_add(&p, oc_importance(x, n, sm.lo, sm.hi, sm.face), power6(sm.face), s, lt_random_float(rng));
            }
            float prob;
            const uint32_t s = pick_end(&p, &prob);
            if (s == OC_NONE) return OC_NONE;
            *pdf *= prob;
            chosen = nd->child[s];
        }
        if (chosen & OC_CHILD_LEAF_BIT) return chosen & ~OC_CHILD_LEAF_BIT;
        node = chosen;
    }
    return OC_NONE;
}

static float slot_probability(const oc_node* nd, const float x[3], const float n[3], uint32_t slot)
{
    if (child_count(nd) == 1) return 1.0f;
    float sum_i = 0.0f, sum_p = 0.0f, imp_t = 0.0f, pow_t = 0.0f;
    for (uint32_t s = 0; s < 4; ++s) {
        if (nd->child[s] == OC_NONE) continue;
        oc_summary sm;
        node_slot(nd, s, &sm);
        const float imp = oc_importance(x, n, sm.lo, sm.hi, sm.face);
        const float pw = power6(sm.face);
        sum_i += imp > 0.0f ? imp : 0.0f;
        sum_p += pw > 0.0f ? pw : 0.0f;
        if (s == slot) {
            imp_t = imp;
            pow_t = pw;
        }
    }
    return pick_probability(sum_i, sum_p, imp_t, pow_t);
}

/* The probability of drawing leaf `leaf` of tree k (T): the slot picks up to its root, times the
 * pick of tree k among the two (t: the world's tree). */
static float leaf_probability(const oc_scene* sc, const oc_light_tree* t, const oc_light_tree* T, uint32_t leaf,
                              const float x[3], const float n[3], uint32_t k)
{
    const oc_light_tree* t_ = T;
    if (t_->header->root == OC_NONE) return 0.0f;
    const uint32_t parent = t_->leaves[leaf].parent;
    if (parent == OC_NONE) return 0.0f;
    uint32_t node = parent >> 2, slot = parent & 3u;
    float probability = 1.0f;
    for (uint32_t depth = 0; depth < 64; ++depth) {
        const oc_node* nd = &t_->nodes[node];
        probability *= slot_probability(nd, x, n, slot);
        if (nd->parent == OC_NONE) return probability * tree_probability(sc, t, x, n, k);
        node = nd->parent;
        slot = nd->parent_slot;
    }
    return 0.0f;
}

/* A light record of the heap (LtLoadEntryRecord, caelix_light_tree_layout.hlsl:377-400). */
static const uint32_t* entry_record(const oc_scene* s, uint32_t group, uint32_t entry, const uint32_t** block_out)
{
    const uint32_t* row = s->group_rows + 8ull * group;
    const uint32_t* block = s->heap + 4ull * row[0];
    if (block_out) *block_out = block;
    const uint32_t* ie = block + 4 + 4ull * entry;
    return block + 4ull * ie[2];
}

static uint32_t family_count(const uint32_t* rec, uint32_t f)
{
    const uint32_t word = f < 3 ? rec[10] : rec[11];
    return (word >> (10 * (f % 3))) & 0x3FFu;
}

/* x_group = R^T (x - t) - origin and the family weights (LtFamilyWeights). */
static float family_weights(const oc_scene* s, uint32_t group, const uint32_t* rec, const float x[3], float w[6])
{
    const oc_frame* fr = &s->group_frames[group];
    float v[3], xg[3];
    for (int k = 0; k < 3; ++k) v[k] = x[k] - fr->trans[k];
    for (int j = 0; j < 3; ++j)
        xg[j] = v[0] * fr->rot[0 * 3 + j] + v[1] * fr->rot[1 * 3 + j] + v[2] * fr->rot[2 * 3 + j] - fr->origin[j];
    const float lo[3] = {(float)(rec[6] & 0x3FFu), (float)((rec[6] >> 10) & 0x3FFu), (float)((rec[6] >> 20) & 0x3FFu)};
    const float hi[3] = {(float)(rec[7] & 0x3FFu), (float)((rec[7] >> 10) & 0x3FFu), (float)((rec[7] >> 20) & 0x3FFu)};
    float dlo[3], dhi[3], c[6];
    for (int k = 0; k < 3; ++k) {
        dlo[k] = xg[k] - hi[k];
        dhi[k] = xg[k] - lo[k];
    }
    emitter_cosines(dlo, dhi, c);
    float face[6];
    memcpy(face, rec, 24);
    float sum = 0.0f;
    for (int f = 0; f < 6; ++f) {
        w[f] = face[f] * c[f];
        sum += w[f];
    }
    if (sum <= 0.0f) {
        sum = 0.0f;
        for (int f = 0; f < 6; ++f) {
            w[f] = face[f];
            sum += w[f];
        }
    }
    return sum;
}

int oc_light_sample(const oc_scene* s, const oc_light_tree* t, const float x[3], const float n[3], uint32_t rng,
                    float out[7], uint32_t words[6])
{
    memset(out, 0, 7 * sizeof(float));
    memset(words, 0, 6 * sizeof(uint32_t));
    float pdf_brick = 1.0f;
    uint32_t root;
    const uint32_t k = choose_tree(s, t, x, n, &rng, &pdf_brick, &root);
    if (k == OC_NONE) return 0;
    const oc_light_tree* T = tree_of(s, t, k);
    const oc_scene* L = lights_of(s, k);
    const uint32_t leaf = choose_leaf(T, root, x, n, &rng, &pdf_brick);
    if (leaf == OC_NONE) return 0;
    const uint32_t group = T->leaves[leaf].group;
    const uint32_t entry = T->leaves[leaf].entry;
    words[3] = group;
    words[4] = entry;
    words[5] = k;
    const uint32_t* row = L->group_rows + 8ull * group;
    if (row[1] == 0) return 0;
    const uint32_t* rec = entry_record(L, group, entry, NULL);
    float w[6];
    const float sum = family_weights(L, group, rec, x, w);
    if (sum <= 0.0f) return 0;
    const float u = lt_random_float(&rng) * sum;
    uint32_t f = OC_NONE, last = 0;
    float cumulative = 0.0f;
    for (uint32_t g = 0; g < 6; ++g) {
        if (w[g] > 0.0f) {
            last = g;
            cumulative += w[g];
            if (f == OC_NONE && u < cumulative) f = g;
        }
    }
    f = f == OC_NONE ? last : f;
    uint32_t first = 0;
    for (uint32_t h = 0; h < f; ++h) first += family_count(rec, h);
    const uint32_t count = family_count(rec, f);
    if (count == 0 || w[f] <= 0.0f) return 0;
    uint32_t ei = (uint32_t)(lt_random_float(&rng) * (float)count);
    if (ei > count - 1u) ei = count - 1u;
    const uint32_t ent = rec[12 + first + ei];
    const uint32_t vi = ent & 0x1FFu;
    const uint32_t gs = L->group_shift, gm = (1u << gs) - 1u;
    const uint32_t pos = rec[8];
    const uint32_t voxel[3] = {(pos & gm) * 8 + (vi & 7u), ((pos >> gs) & gm) * 8 + ((vi >> 3) & 7u),
                               ((pos >> (2 * gs)) & gm) * 8 + (vi >> 6)};
    const oc_frame* fr = &L->group_frames[group];
    const uint32_t axis = f >> 1;
    float local[3];
    for (int q = 0; q < 3; ++q) local[q] = fr->origin[q] + (float)voxel[q];
    const float a = lt_random_float(&rng);
    const float b = lt_random_float(&rng);
    local[axis] += (f & 1) ? 0.0f : 1.0f;
    local[(axis + 1) % 3] += a;
    local[(axis + 2) % 3] += b;
    const float dirn[3] = {f == 0 ? 1.0f : (f == 1 ? -1.0f : 0.0f), f == 2 ? 1.0f : (f == 3 ? -1.0f : 0.0f),
                           f == 4 ? 1.0f : (f == 5 ? -1.0f : 0.0f)};
    for (int r = 0; r < 3; ++r) {
        const float* R = fr->rot + 3 * r;
        out[r] = R[0] * local[0] + R[1] * local[1] + R[2] * local[2] + fr->trans[r];
        out[3 + r] = R[0] * dirn[0] + R[1] * dirn[1] + R[2] * dirn[2];
    }
    out[6] = w[f] / sum / (float)count * pdf_brick;
    words[0] = ent >> 16;
    words[1] = vi;
    words[2] = f;
    return 1;
}

void oc_light_draws(const oc_scene* s, const oc_light_tree* t, const float x[3], const float n[3], uint32_t seed,
                    uint32_t count, uint32_t* out)
{
    uint32_t state = seed != 0u ? seed : 0x9E3779B9u;
    const uint32_t gs = s->group_shift, gm = (1u << gs) - 1u;
    for (uint32_t i = 0; i < count; ++i) {
        float p[7];
        uint32_t words[6];
        uint32_t* o = out + 4ull * i;
        o[0] = o[1] = o[2] = o[3] = 0;
        if (!oc_light_sample(s, t, x, n, random_u32(&state), p, words)) continue;
        const uint32_t pos = entry_record(lights_of(s, words[5]), words[3], words[4], NULL)[8];
        const uint32_t vi = words[1];
        o[0] = words[3];
        o[1] = ((pos & gm) * 8 + (vi & 7u)) | ((((pos >> gs) & gm) * 8 + ((vi >> 3) & 7u)) << 10) |
               ((((pos >> (2 * gs)) & gm) * 8 + (vi >> 6)) << 20);
        o[2] = words[2];
        o[3] = 1u | (words[5] << 1);
    }
}

/* LightTreeFindLightFace (caelix_light_tree.hlsl:853-934): the face of a voxel whose material code
 * is in the light code set, in a brick that has a brick light record. */
static int find_light_face(const oc_scene* s, const oc_light_tree* t, const float x[3], uint32_t group,
                           const uint32_t v[3], uint32_t face, uint32_t block, uint32_t* entry_out,
                           uint32_t* leaf_out, float* in_brick)
{
    *entry_out = OC_NONE;
    *leaf_out = OC_NONE;
    *in_brick = 0.0f;
    const uint32_t code = oc_material_code(block, s->encoding);
    if (!((s->light_codes[code >> 5] >> (code & 31)) & 1u) || face > 5) return 0;
    const uint32_t* row = s->group_rows + 8ull * group;
    if (row[1] == 0) return 0;
    const uint32_t* block_w = s->heap + 4ull * row[0];
    const uint32_t count_r = block_w[0];
    const uint32_t key = oc_morton(v[0] / 8, v[1] / 8, v[2] / 8);
    const uint32_t gs = s->group_shift, gm = (1u << gs) - 1u;
    uint32_t lo = 0, hi = count_r, entry = OC_NONE;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t pos = block_w[4 + 4 * mid];
        const uint32_t mk = oc_morton(pos & gm, (pos >> gs) & gm, (pos >> (2 * gs)) & gm);
        if (mk == key) {
            entry = mid;
            break;
        }
        if (mk < key) lo = mid + 1;
        else hi = mid;
    }
    if (entry == OC_NONE) return 0;
    *entry_out = entry;
    const uint32_t* rec = block_w + 4ull * block_w[4 + 4 * entry + 2];
    float w[6];
    const float sum = family_weights(s, group, rec, x, w);
    const uint32_t count = family_count(rec, face);
    if (sum <= 0.0f || w[face] <= 0.0f || count == 0) return 0;
    uint32_t first = 0;
    for (uint32_t g = 0; g < face; ++g) first += family_count(rec, g);
    const uint32_t vi = (v[0] % 8) | ((v[1] % 8) << 3) | ((v[2] % 8) << 6);
    uint32_t a = 0, b = count;
    int found = 0;
    while (a < b) {
        const uint32_t mid = (a + b) >> 1;
        const uint32_t ev = rec[12 + first + mid] & 0x1FFu;
        if (ev == vi) {
            found = 1;
            break;
        }
        if (ev < vi) a = mid + 1;
        else b = mid;
    }
    if (!found) return 0;
    *in_brick = (w[face] / sum) / (float)count;
    const uint32_t bvh_leaf = block_w[4 + 4 * entry + 3];
    if (bvh_leaf != OC_NONE) {
        const uint32_t leaf = bvh_leaf & 0x7FFFFFFFu;
        if (t->leaves[leaf].group == group && t->leaves[leaf].entry == entry) *leaf_out = bvh_leaf;
    }
    return 1;
}

/* The draw probability of entry `entry` of group `group` of light set k (L, its tree T). */
static float brick_pdf(const oc_scene* sc, const oc_light_tree* t, const oc_scene* L, const oc_light_tree* T,
                       const float x[3], const float n[3], uint32_t group, uint32_t entry, uint32_t k)
{
    const uint32_t* row = L->group_rows + 8ull * group;
    if (row[1] == 0) return 0.0f;
    const uint32_t* block_w = L->heap + 4ull * row[0];
    if (entry >= block_w[0]) return 0.0f;
    const uint32_t bvh_leaf = block_w[4 + 4 * entry + 3];
    if (bvh_leaf == OC_NONE) return 0.0f;
    const uint32_t leaf = bvh_leaf & 0x7FFFFFFFu;
    if (T->leaves[leaf].group != group || T->leaves[leaf].entry != entry) return 0.0f;
    return leaf_probability(sc, t, T, leaf, x, n, k);
}

float oc_light_point_pdf_tree(const oc_scene* s, const oc_light_tree* t, const float x[3], const float n[3],
                              uint32_t tree, uint32_t group, const uint32_t v[3], uint32_t face, uint32_t block)
{
    const oc_scene* L = tree > 1 ? NULL : lights_of(s, tree);
    if (!L) return 0.0f;
    const oc_light_tree* T = tree_of(s, t, tree);
    uint32_t entry, leaf;
    float in_brick;
    if (!find_light_face(L, T, x, group, v, face, block, &entry, &leaf, &in_brick)) return 0.0f;
    return brick_pdf(s, t, L, T, x, n, group, entry, tree) * in_brick;
}

float oc_light_point_pdf(const oc_scene* s, const oc_light_tree* t, const float x[3], const float n[3], uint32_t group,
                         const uint32_t v[3], uint32_t face, uint32_t block)
{
    return oc_light_point_pdf_tree(s, t, x, n, 0, group, v, face, block);
}

/* ---- integrator ---- */

typedef struct ctx {
    const oc_scene* s;
    const oc_light_tree* t;
    const float* albedo;
    const float* power;
    const oc_camera* cam;
    const oc_render_desc* r;
    float* radiance;
    uint64_t rays[3];
} ctx;

static float mis_weight(float p_area, const float n_r[3], const float w[3], float d, float cos_l, int nee_side)
{
    const float p_sa = cos_l > 0.0f ? p_area * (d * d) / cos_l : 0.0f;
    const float p_bsdf = hmax(0.0f, dot3(n_r, w)) * (1.0f / 3.1415926535f);
    if (!(cos_l > 0.0f) || !(p_sa <= 3.0e38f)) return nee_side ? 1.0f : 0.0f;
    const float sum = p_sa + p_bsdf;
    if (!(sum > 0.0f)) return nee_side ? 0.0f : 1.0f;
    return (nee_side ? p_sa : p_bsdf) / sum;
}

float oc_mis_weight(float p_area, const float n_r[3], const float w[3], float d, float cos_l, int nee_side)
{
    return mis_weight(p_area, n_r, w, d, cos_l, nee_side);
}

/* The emission of a voxel: the table's emission of its material code (the scene's table, shared by
 * its entities) times its brick's power p. */
static void emission_of(const ctx* c, float p, uint32_t block, float e[3])
{
    const float* m = c->s->emission + 3ull * oc_material_code(block, c->s->encoding);
    for (int k = 0; k < 3; ++k) e[k] = m[k] * p;
}

/* ---- the voxel id (shaders/render/caelix_scene_trace.hlsl:171-200) ---- */

static uint32_t hash_avalanche(uint32_t v)
{
    v ^= v >> 16;
    v *= 0x7FEB352Du;
    v ^= v >> 15;
    v *= 0x846CA68Bu;
    v ^= v >> 16;
    return v;
}

static uint32_t voxel_id_word(uint32_t seed, uint32_t entity, const int32_t v[3])
{
    uint32_t h = hash_avalanche(seed ^ entity);
    for (int k = 0; k < 3; ++k) h = hash_avalanche(h ^ (uint32_t)v[k]);
    return h == 0xFFFFFFFFu ? 0xFFFFFFFEu : h;
}

void oc_voxel_id(const oc_scene* s, const oc_hit* h, uint32_t out[2])
{
    uint32_t entity = 0;
    const oc_scene* b = s;
    if (h->attrib & OC_ENTITY_HIT) {
        const uint32_t e = h->group >> 24;
        entity = s->entities[e].id;
        b = s->entities[e].scene;
    }
    const uint32_t cell = (h->attrib >> 6) & 0x1FFu;
    int32_t v[3];
    for (int k = 0; k < 3; ++k) v[k] = b->keys[3ull * h->record + k] * 8 + (int32_t)((cell >> (3 * k)) & 7u);
    out[0] = voxel_id_word(0x9E3779B9u, entity, v);
    out[1] = voxel_id_word(0x85EBCA6Bu, entity, v);
}

/* NextEventAtVertex without the sun: the lamp candidate and its shadow ray. */
/* lamp_brick / lamp_code / dvalue: a drawn, unoccluded lamp of the world (its brick, its code and
 * the factor of its power); lamp_fixed: the power of an unoccluded lamp of the entities' light set
 * (not differentiated; -1 for none). */
static void next_event(ctx* c, const float x[3], const float n[3], uint32_t* light_rng, float out[3],
                       uint32_t* lamp_brick, uint32_t* lamp_code, float* dvalue, float* lamp_fixed)
{
    out[0] = out[1] = out[2] = 0.0f;
    *lamp_brick = OC_NONE;
    *lamp_code = 0;
    *dvalue = 0.0f;
    *lamp_fixed = -1.0f;
    const uint32_t point_seed = random_u32(light_rng);
    float p[7];
    uint32_t words[6];
    if (!oc_light_sample(c->s, c->t, x, n, point_seed, p, words) || !(p[6] > 0.0f)) return;
    float d[3] = {p[0] - x[0], p[1] - x[1], p[2] - x[2]};
    const float d2 = dot3(d, d);
    const float dist = sqrtf(d2);
    if (!(dist >= NEAR_FIELD)) return;
    const float w[3] = {d[0] / dist, d[1] / dist, d[2] / dist};
    const float cos_r = dot3(n, w);
    const float cos_l = -dot3(p + 3, w);
    if (!(cos_r > 0.0f) || !(cos_l > 0.0f)) return;
    float scale = (cos_r * (1.0f / K_PI)) * (cos_l / d2) / p[6];
    scale *= mis_weight(p[6], n, w, dist, cos_l, 1);
    /* The lamp's emission: the brick of the sampled light voxel (in the world, or in the entities'
     * merged light set). */
    const oc_scene* L = lights_of(c->s, words[5]);
    const uint32_t* row = L->group_rows + 8ull * words[3];
    const uint32_t* block_w = L->heap + 4ull * row[0];
    const uint32_t brick = block_w[4 + 4 * words[4] + 1];
    float e[3];
    emission_of(c, words[5] == 0 ? c->power[brick] : c->s->dyn_power[brick], words[0], e);
    float contribution[3] = {e[0] * scale, e[1] * scale, e[2] * scale};
    const float lum = contribution[0] * 0.2126f + contribution[1] * 0.7152f + contribution[2] * 0.0722f;
    const float w_lamp = lum * hmax(0.05f, 1.0f);
    const float w_sum = 0.0f + w_lamp;
    if (!(w_sum > 0.0f)) return;
    const float t_max = dist - 2.0f * PUSH_OFF;
    int occluded = 1;
    if (t_max > 0.0f) {
        c->rays[2]++;
        const oc_hit h = oc_trace_ray(c->s, x, w, 0.0f, t_max);
        occluded = h.hit;
    }
    if (t_max > 0.0f && !occluded) {
        const float k = w_sum / w_lamp;
        for (int q = 0; q < 3; ++q) out[q] = contribution[q] * k;
        /* For the adjoint: the contribution is the lamp brick's power times the emission of its
         * code times scale * k. */
        *lamp_code = oc_material_code(words[0], c->s->encoding);
        *dvalue = scale * k;
        /* A world lamp's power is a parameter; a static entity's (tree 0, after the world's
         * bricks) and a dynamic entity's are held fixed. */
        if (words[5] == 0 && brick < c->s->brick_count) *lamp_brick = brick;
        else *lamp_fixed = words[5] == 0 ? c->power[brick] : c->s->dyn_power[brick];
    }
}

static float lamp_hit_weight(ctx* c, uint32_t segment_light, const oc_hit* h, const float origin[3], const float dir[3],
                             const float seg_n[3])
{
    if (segment_light == 0u || h->t < NEAR_FIELD) return 1.0f;
    /* The light set of the hit: the world's, or for an entity hit the entities' (its groups from
     * the entity's group base; the voxel from the entity-local hit point and face normal). */
    const oc_scene* L = c->s;
    const oc_light_tree* T = c->t;
    uint32_t group = h->group, k = 0;
    const uint32_t face = (uint32_t)__builtin_ctz(h->attrib & 0x3Fu);
    float nl[3] = {h->normal[0], h->normal[1], h->normal[2]};
    if (h->attrib & OC_ENTITY_HIT) {
        /* A static entity's lights are in tree 0 (this scene's light set), a dynamic one's in
         * tree 1. */
        const oc_entity* E = &c->s->entities[h->group >> 24];
        if (E->tree > 1u || (E->tree == 1u && !c->s->dyn)) return 1.0f;
        if (E->tree == 1u) {
            L = c->s->dyn;
            T = c->s->dyn_tree;
            k = 1;
        }
        group = E->group_base + (h->group & 0xFFFFFFu);
        for (int q = 0; q < 3; ++q) nl[q] = 0.0f;
        nl[face >> 1] = (face & 1u) ? -1.0f : 1.0f;
    }
    int32_t voxel[3];
    for (int q = 0; q < 3; ++q) voxel[q] = (int32_t)floorf(h->object_hit[q] - 0.25f * nl[q]);
    const oc_frame* fr = &L->group_frames[group];
    uint32_t vig[3];
    for (int q = 0; q < 3; ++q) vig[q] = (uint32_t)(voxel[q] - (int32_t)fr->origin[q]);
    const uint32_t block = (h->attrib >> 16) & 0xFFFFu;
    uint32_t entry, leaf;
    float in_brick;
    if (!find_light_face(L, T, origin, group, vig, face, block, &entry, &leaf, &in_brick) || leaf == OC_NONE)
        return 1.0f;
    const float cos_l = -dot3(h->normal, dir);
    const float p_area = brick_pdf(c->s, c->t, L, T, origin, seg_n, group, entry, k) * in_brick;
    return mis_weight(p_area, seg_n, dir, h->t, cos_l, 0);
}

static void shade(const ctx* c, const oc_hit* h, const float ray_o[3], const float ray_d[3], uint32_t* rng,
                  float albedo[3], float emission[3], float origin[3], float dir[3])
{
    const uint32_t block = (h->attrib >> 16) & 0xFFFFu;
    if (h->attrib & OC_ENTITY_HIT) { /* an entity brick's power */
        const float* pw = c->s->entities[h->group >> 24].power;
        emission_of(c, pw ? pw[h->record] : 0.0f, block, emission);
    } else {
        emission_of(c, c->power[h->record], block, emission);
    }
    const float* a = c->albedo + 3ull * oc_material_code(block, c->s->encoding);
    albedo[0] = a[0];
    albedo[1] = a[1];
    albedo[2] = a[2];
    (void)random01(rng); /* the lobe draw (specular chance 0) */
    float u[3];
    random_unit_vector(rng, u);
    float v[3] = {h->normal[0] + u[0], h->normal[1] + u[1], h->normal[2] + u[2]};
    const float dp3 = hmax(1.175494351e-38f, dot3(v, v));
    const float inv = 1.0f / sqrtf(dp3);
    float dd[3] = {v[0] * inv, v[1] * inv, v[2] * inv};
    if (!(dot3(dd, dd) > 0.0f)) memcpy(dd, h->normal, sizeof(dd));
    memcpy(dir, dd, sizeof(dd));
    for (int k = 0; k < 3; ++k) origin[k] = (ray_o[k] + ray_d[k] * h->t) + PUSH_OFF * h->normal[k];
}

/* ---- the path record of the adjoint reference ----
 * The events of one path sample in order, as the estimator gathers them: an emitter hit adds
 * power[brick] * factor * throughput, an NEE lamp adds power[brick] * factor * throughput, a
 * bounce vertex multiplies the throughput by the albedo of its material, a Russian-roulette
 * survival by factor (1 / cp). The factors are the sampling quantities of the fp32 forward pass
 * (MIS weights, geometry / pdf terms, RR probabilities), held fixed by the adjoint. */
enum { EV_EMIT = 0, EV_ALBEDO = 1, EV_NEE = 2, EV_RR = 3, EV_FIXED = 4 };
#define MAX_EVENTS 64

typedef struct path_event {
    uint32_t kind;
    uint32_t index; /* brick (EMIT, NEE) or material code (ALBEDO) */
    uint32_t code;  /* EMIT, NEE, FIXED: the material code of the emitting voxel */
    float factor;
    float power;    /* FIXED: the power of an entity's emitting brick (held fixed: an entity's power
                       is not differentiated) */
} path_event;

typedef struct path_rec {
    int hit;
    int emits0;         /* the primary emission is power[record0] times the emission of material0 */
    uint32_t material0; /* the primary material code */
    uint32_t record0;
    int bad;            /* the fp32 radiance was not finite (the sample's radiance part is 0) */
    float e0_fixed[3];  /* the primary emission of an entity voxel (held fixed) */
    float radiance[3];  /* the fp32 radiance of the sample */
    uint32_t n;
    path_event ev[MAX_EVENTS];
} path_rec;

static void rec_event_p(path_rec* rec, uint32_t kind, uint32_t index, uint32_t code, float factor, float power)
{
    if (rec && rec->n < MAX_EVENTS) {
        rec->ev[rec->n].kind = kind;
        rec->ev[rec->n].index = index;
        rec->ev[rec->n].code = code;
        rec->ev[rec->n].factor = factor;
        rec->ev[rec->n].power = power;
        rec->n++;
    }
}

static void rec_event(path_rec* rec, uint32_t kind, uint32_t index, uint32_t code, float factor)
{
    rec_event_p(rec, kind, index, code, factor, 0.0f);
}

/* The NEE events of a vertex: a world lamp's power is a parameter, an entity lamp's is fixed. */
static void rec_nee(path_rec* rec, uint32_t lamp, uint32_t code, float dv, float fixed)
{
    if (lamp != OC_NONE) rec_event(rec, EV_NEE, lamp, code, dv);
    else if (fixed >= 0.0f) rec_event_p(rec, EV_FIXED, 0, code, dv, fixed);
}

static void trace_pixel(ctx* c, uint32_t px, uint32_t py, uint32_t seed, float rgb[3], path_rec* rec)
{
    if (rec) memset(rec, 0, sizeof(*rec));
    const oc_camera* cam = c->cam;
    const oc_render_desc* r = c->r;
    rgb[0] = rgb[1] = rgb[2] = 0.0f;
    const float sx = (float)px + 0.5f + 0.0f;
    const float sy = (float)py + 0.5f + 0.0f;
    const float ndc_x = sx / (float)r->width * 2.0f - 1.0f;
    const float ndc_y = 1.0f - sy / (float)r->height * 2.0f;
    const float a = ndc_x * cam->tan_half_fov_y * cam->aspect;
    const float b = ndc_y * cam->tan_half_fov_y;
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = cam->right[k] * a + cam->up[k] * b + cam->forward[k];
    const float inv_len = 1.0f / sqrtf(dot3(d, d));
    for (int k = 0; k < 3; ++k) d[k] = d[k] * inv_len;
    c->rays[0]++;
    const oc_hit primary = oc_trace_ray(c->s, cam->position, d, 0.0f, RAY_TMAX);
    if (r->voxel_id && seed == r->frame_seed) {
        uint32_t* out = r->voxel_id + 2ull * ((uint64_t)py * r->width + px);
        out[0] = out[1] = 0xFFFFFFFFu;
        if (primary.hit && (r->voxel_id_tmax <= 0.0f || primary.t <= r->voxel_id_tmax))
            oc_voxel_id(c->s, &primary, out);
    }
    if (!primary.hit) return;
    uint32_t rng = init_random(px, py, seed);
    uint32_t light_rng = init_random(px, py, seed ^ 0x7F4A7C15u);
    float a0[3], e0[3], org[3], dir[3];
    shade(c, &primary, cam->position, d, &rng, a0, e0, org, dir);
    if (rec) {
        const uint32_t block0 = (primary.attrib >> 16) & 0xFFFFu;
        rec->hit = 1;
        rec->emits0 = !(primary.attrib & OC_ENTITY_HIT);
        if (!rec->emits0) memcpy(rec->e0_fixed, e0, sizeof(rec->e0_fixed));
        rec->material0 = oc_material_code(block0, c->s->encoding);
        rec->record0 = primary.record;
    }
    float seg_n[3];
    memcpy(seg_n, primary.normal, sizeof(seg_n));
    float radiance[3] = {0, 0, 0};
    float throughput[3] = {1.0f / hmax(0.001f, 1.0f), 1.0f / hmax(0.001f, 1.0f), 1.0f / hmax(0.001f, 1.0f)};
    uint32_t segment_light = 0;
    if (r->light_nee && r->bounce_count >= 1) {
        float nee[3], dv, fixed;
        uint32_t lamp, lamp_code;
        next_event(c, org, primary.normal, &light_rng, nee, &lamp, &lamp_code, &dv, &fixed);
        for (int k = 0; k < 3; ++k) radiance[k] += nee[k] * throughput[k];
        rec_nee(rec, lamp, lamp_code, dv, fixed);
        segment_light = 3u; /* lamp NEE with MIS */
    }
    uint32_t bounce_index = 1;
    while (bounce_index <= r->bounce_count) {
        c->rays[1]++;
        const oc_hit h = oc_trace_ray(c->s, org, dir, 0.0f, BOUNCE_TMAX);
        if (!h.hit) break; /* black sky */
        float al[3], em[3], o2[3], d2[3];
        shade(c, &h, org, dir, &rng, al, em, o2, d2);
        bounce_index += 1;
        float ew = 1.0f;
        if (segment_light != 0u && (em[0] > 0.0f || em[1] > 0.0f || em[2] > 0.0f))
            ew = lamp_hit_weight(c, segment_light, &h, org, dir, seg_n);
        for (int k = 0; k < 3; ++k) radiance[k] += em[k] * (throughput[k] * ew);
        const uint32_t code = oc_material_code((h.attrib >> 16) & 0xFFFFu, c->s->encoding);
        if (!(h.attrib & OC_ENTITY_HIT)) {
            rec_event(rec, EV_EMIT, h.record, code, ew);
        } else {
            const float* pw = c->s->entities[h.group >> 24].power;
            rec_event_p(rec, EV_FIXED, 0, code, ew, pw ? pw[h.record] : 0.0f);
        }
        rec_event(rec, EV_ALBEDO, code, 0, 0.0f);
        for (int k = 0; k < 3; ++k) throughput[k] *= al[k] / hmax(0.001f, 1.0f);
        segment_light = 0u;
        if (r->light_nee && bounce_index <= r->bounce_count) {
            segment_light = 3u;
            float nee[3], dv, fixed;
            uint32_t lamp, lamp_code;
            next_event(c, o2, h.normal, &light_rng, nee, &lamp, &lamp_code, &dv, &fixed);
            for (int k = 0; k < 3; ++k) radiance[k] += nee[k] * (throughput[k] * (1.0f / 1.0f));
            rec_nee(rec, lamp, lamp_code, dv, fixed);
        }
        const float cp = hmax(throughput[0], hmax(throughput[1], throughput[2]));
        if (cp <= 0.0f || cp < random01(&rng)) break;
        rec_event(rec, EV_RR, 0, 0, 1.0f / cp);
        for (int k = 0; k < 3; ++k) throughput[k] *= 1.0f / cp;
        memcpy(org, o2, sizeof(org));
        memcpy(dir, d2, sizeof(dir));
        memcpy(seg_n, h.normal, sizeof(seg_n));
    }
    /* SanitizeRadiance (caelix_shading.hlsl:337-341), then the composite's albedo modulation. */
    int bad = 0;
    for (int k = 0; k < 3; ++k) bad |= isnan(radiance[k]) || isinf(radiance[k]);
    for (int k = 0; k < 3; ++k) {
        const float sr = hmin(bad ? 0.0f : radiance[k], 65504.0f);
        rgb[k] = e0[k] + a0[k] * sr;
    }
    if (rec) {
        rec->bad = bad;
        memcpy(rec->radiance, radiance, sizeof(radiance));
    }
}

typedef struct job {
    ctx* c;
    uint32_t y_begin, y_end;
    uint64_t rays[3];
} job;

static void* run_rows(void* arg)
{
    job* j = (job*)arg;
    ctx local = *j->c;
    local.rays[0] = local.rays[1] = local.rays[2] = 0;
    const oc_render_desc* r = local.r;
    for (uint32_t y = j->y_begin; y < j->y_end; ++y)
        for (uint32_t x = r->x0; x < r->x1; ++x) {
            float acc[3] = {0, 0, 0};
            for (uint32_t s = 0; s < r->spp; ++s) {
                float rgb[3];
                trace_pixel(&local, x, y, r->frame_seed + s, rgb, NULL);
                for (int k = 0; k < 3; ++k) acc[k] += rgb[k];
            }
            float* out = local.radiance + 3ull * ((uint64_t)y * r->width + x);
            for (int k = 0; k < 3; ++k) out[k] = acc[k] / (float)r->spp;
        }
    memcpy(j->rays, local.rays, sizeof(j->rays));
    return NULL;
}

void oc_render(const oc_scene* s, const oc_light_tree* t, const float* albedo, const float* power, const oc_camera* cam,
               const oc_render_desc* r, float* radiance, uint64_t* rays, int threads)
{
    ctx c = {s, t, albedo, power, cam, r, radiance, {0, 0, 0}};
    if (threads < 1) threads = 1;
    const uint32_t rows = r->y1 - r->y0;
    if ((uint32_t)threads > rows) threads = (int)(rows ? rows : 1);
    job* jobs = (job*)calloc((size_t)threads, sizeof(job));
    pthread_t* tids = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    for (int i = 0; i < threads; ++i) {
        jobs[i].c = &c;
        jobs[i].y_begin = r->y0 + (uint32_t)((uint64_t)rows * i / threads);
        jobs[i].y_end = r->y0 + (uint32_t)((uint64_t)rows * (i + 1) / threads);
        if (threads == 1) run_rows(&jobs[i]);
        else pthread_create(&tids[i], NULL, run_rows, &jobs[i]);
    }
    for (int i = 0; i < threads; ++i) {
        if (threads > 1) pthread_join(tids[i], NULL);
        for (int k = 0; k < 3; ++k) rays[k] += jobs[i].rays[k];
    }
    free(jobs);
    free(tids);
}

/* ---- the adjoint reference (double precision) ----
 * The adjoint of the estimator with its sampling quantities held fixed (the factors of the path
 * record): a sample is then a polynomial in the albedo table A and the brick powers P,
 *   rgb = E0 + A0 * sanitize(R),  R = sum over the emission events of P[brick] * factor * T,
 * T the product of the albedo and RR factors before the event. The fp32 forward pass (the
 * oracle's trace_pixel, bit-exact with the CUDA path) fixes the path and its factors; the sample
 * is then evaluated and differentiated in double: forward over the events for the throughputs,
 * backward over them for dL/dT (reverse accumulation, no difference of partial sums). sanitize
 * keeps the fp32 decisions: a non-finite fp32 radiance gives 0, a channel above 65504 gives the
 * constant 65504. */

typedef struct adj_job {
    const ctx* c;
    uint32_t y_begin, y_end;
    const double* A;        /* evaluation albedo [65536][3] by material code */
    const double* P;        /* evaluation power [brick_count] */
    const float* d_radiance; /* dL/d(pixel) (gradient mode) */
    double* image;          /* evaluation mode: the double image */
    double* dA;             /* gradient mode: this job's albedo gradient [65536][3] */
    double* dP;             /* gradient mode: this job's power gradient [brick_count] */
} adj_job;

/* E: the material table's emission [65536][3] (held fixed). */
static void eval_sample(const path_rec* rec, const float* E, const double* A, const double* P, double rgb[3],
                        double T_before[][3], double R[3])
{
    double T[3] = {1.0, 1.0, 1.0};
    R[0] = R[1] = R[2] = 0.0;
    for (uint32_t i = 0; i < rec->n; ++i) {
        const path_event* e = &rec->ev[i];
        for (int k = 0; k < 3; ++k) T_before[i][k] = T[k];
        if (e->kind == EV_EMIT || e->kind == EV_NEE || e->kind == EV_FIXED) {
            const double p = e->kind == EV_FIXED ? (double)e->power : P[e->index];
            for (int k = 0; k < 3; ++k) R[k] += p * (double)E[3 * e->code + k] * (double)e->factor * T[k];
        } else if (e->kind == EV_ALBEDO) {
            for (int k = 0; k < 3; ++k) T[k] *= A[3 * e->index + k];
        } else {
            for (int k = 0; k < 3; ++k) T[k] *= (double)e->factor;
        }
    }
    const double p0 = rec->emits0 ? P[rec->record0] : 0.0;
    for (int k = 0; k < 3; ++k) {
        const double sr = rec->bad ? 0.0 : (rec->radiance[k] > 65504.0f ? 65504.0 : R[k]);
        rgb[k] = p0 * (double)E[3 * rec->material0 + k] + (double)rec->e0_fixed[k] + A[3 * rec->material0 + k] * sr;
    }
}

static void* run_adjoint_rows(void* arg)
{
    adj_job* j = (adj_job*)arg;
    ctx local = *j->c;
    const oc_render_desc* r = local.r;
    path_rec* rec = (path_rec*)malloc(sizeof(path_rec));
    double (*T_before)[3] = (double (*)[3])malloc(sizeof(double) * 3 * MAX_EVENTS);
    for (uint32_t y = j->y_begin; y < j->y_end; ++y)
        for (uint32_t x = r->x0; x < r->x1; ++x) {
            const uint64_t pix = (uint64_t)y * r->width + x;
            double acc[3] = {0, 0, 0};
            for (uint32_t s = 0; s < r->spp; ++s) {
                float rgb32[3];
                trace_pixel(&local, x, y, r->frame_seed + s, rgb32, rec);
                if (!rec->hit) continue;
                double rgb[3], R[3];
                eval_sample(rec, local.s->emission, j->A, j->P, rgb, T_before, R);
                for (int k = 0; k < 3; ++k) acc[k] += rgb[k];
                if (!j->dA) continue;
                double g[3], G[3];
                for (int k = 0; k < 3; ++k) g[k] = (double)j->d_radiance[3 * pix + k] / (double)r->spp;
                const double* a0 = j->A + 3 * rec->material0;
                for (int k = 0; k < 3; ++k) {
                    const int pass = !rec->bad && !(rec->radiance[k] > 65504.0f);
                    const double sr = rec->bad ? 0.0 : (pass ? R[k] : 65504.0);
                    j->dA[3 * rec->material0 + k] += g[k] * sr;
                    G[k] = pass ? g[k] * a0[k] : 0.0;
                }
                const float* E0 = local.s->emission + 3 * rec->material0;
                if (rec->emits0) j->dP[rec->record0] += g[0] * E0[0] + g[1] * E0[1] + g[2] * E0[2];
                /* Backward over the events: lambda = dL/dT after the event. */
                double lambda[3] = {0, 0, 0};
                for (int32_t i = (int32_t)rec->n - 1; i >= 0; --i) {
                    const path_event* e = &rec->ev[i];
                    const double* T = T_before[i];
                    if (e->kind == EV_FIXED) {
                        const double f = (double)e->factor;
                        const float* Ee = local.s->emission + 3 * e->code;
                        for (int k = 0; k < 3; ++k) lambda[k] += G[k] * (double)e->power * (double)Ee[k] * f;
                    } else if (e->kind == EV_EMIT || e->kind == EV_NEE) {
                        const double f = (double)e->factor;
                        const float* Ee = local.s->emission + 3 * e->code;
                        j->dP[e->index] += (G[0] * Ee[0] * T[0] + G[1] * Ee[1] * T[1] + G[2] * Ee[2] * T[2]) * f;
                        for (int k = 0; k < 3; ++k) lambda[k] += G[k] * j->P[e->index] * (double)Ee[k] * f;
                    } else if (e->kind == EV_ALBEDO) {
                        for (int k = 0; k < 3; ++k) {
                            j->dA[3 * e->index + k] += lambda[k] * T[k];
                            lambda[k] *= j->A[3 * e->index + k];
                        }
                    } else {
                        for (int k = 0; k < 3; ++k) lambda[k] *= (double)e->factor;
                    }
                }
            }
            if (j->image)
                for (int k = 0; k < 3; ++k) j->image[3 * pix + k] = acc[k] / (double)r->spp;
        }
    free(rec);
    free(T_before);
    return NULL;
}

/* The frozen estimator (image, double) and/or its gradient. The paths and their sampling
 * quantities are those of the fp32 render at (albedo, power); the estimator is evaluated at
 * (A, P) (double; NULL = the fp32 parameters). d_radiance (may be NULL) = dL/d(pixel): then
 * d_albedo [65536][3] and d_power [brick_count] receive dL/dA and dL/dP at (A, P). image (may be
 * NULL) receives the image at (A, P). Per-thread partial gradients are summed in thread order. */
void oc_adjoint(const oc_scene* s, const oc_light_tree* t, const float* albedo, const float* power,
                const oc_camera* cam, const oc_render_desc* r, const double* A, const double* P,
                const float* d_radiance, double* image, double* d_albedo, double* d_power, int threads)
{
    ctx c = {s, t, albedo, power, cam, r, NULL, {0, 0, 0}};
    double* a_own = NULL;
    double* p_own = NULL;
    if (!A) {
        a_own = (double*)malloc(sizeof(double) * OC_MATERIAL_CODES * 3);
        for (int i = 0; i < OC_MATERIAL_CODES * 3; ++i) a_own[i] = albedo[i];
        A = a_own;
    }
    if (!P) {
        p_own = (double*)malloc(sizeof(double) * (s->brick_count ? s->brick_count : 1));
        for (uint32_t i = 0; i < s->brick_count; ++i) p_own[i] = power[i];
        P = p_own;
    }
    if (threads < 1) threads = 1;
    const uint32_t rows = r->y1 - r->y0;
    if ((uint32_t)threads > rows) threads = (int)(rows ? rows : 1);
    adj_job* jobs = (adj_job*)calloc((size_t)threads, sizeof(adj_job));
    pthread_t* tids = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    const size_t nb = s->brick_count ? s->brick_count : 1;
    for (int i = 0; i < threads; ++i) {
        jobs[i].c = &c;
        jobs[i].y_begin = r->y0 + (uint32_t)((uint64_t)rows * i / threads);
        jobs[i].y_end = r->y0 + (uint32_t)((uint64_t)rows * (i + 1) / threads);
        jobs[i].A = A;
        jobs[i].P = P;
        jobs[i].d_radiance = d_radiance;
        jobs[i].image = image;
        if (d_radiance) {
            jobs[i].dA = (double*)calloc(OC_MATERIAL_CODES * 3, sizeof(double));
            jobs[i].dP = (double*)calloc(nb, sizeof(double));
        }
        if (threads == 1) run_adjoint_rows(&jobs[i]);
        else pthread_create(&tids[i], NULL, run_adjoint_rows, &jobs[i]);
    }
    if (d_radiance) {
        memset(d_albedo, 0, sizeof(double) * OC_MATERIAL_CODES * 3);
        memset(d_power, 0, sizeof(double) * nb);
    }
    for (int i = 0; i < threads; ++i) {
        if (threads > 1) pthread_join(tids[i], NULL);
        if (d_radiance) {
            for (int q = 0; q < OC_MATERIAL_CODES * 3; ++q) d_albedo[q] += jobs[i].dA[q];
            for (size_t q = 0; q < nb; ++q) d_power[q] += jobs[i].dP[q];
            free(jobs[i].dA);
            free(jobs[i].dP);
        }
    }
    free(jobs);
    free(tids);
    free(a_own);
    free(p_own);
}
