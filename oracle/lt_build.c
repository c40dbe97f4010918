/* Oracle of the light BVH build (TEST INFRASTRUCTURE ONLY; see oracle.h).
 *
 * Restates, kernel by kernel, the reference's build sequence LightTree::RecordTree
 * (lib/src/light/light_tree_record.cpp:230-309):
 *   gather emit    shaders/light/bvh/caelix_light_gather_emit.hlsl:11-86
 *   bounds         shaders/light/bvh/caelix_light_bvh_bounds.hlsl:10-53
 *   morton         shaders/light/bvh/caelix_light_bvh_morton.hlsl:6-28
 *   radix sort     shaders/light/bvh/caelix_light_bvh_sort_{histogram,scatter}.hlsl (a stable LSD
 *                  sort; the 8-bit-digit restatement gives the same permutation as the 4-bit one)
 *   karras         shaders/light/bvh/caelix_light_bvh_karras.hlsl:8-96
 *   aggregate      shaders/light/bvh/caelix_light_bvh_aggregate.hlsl:30-55
 *   depth + scan   shaders/light/bvh/caelix_light_bvh_depth.hlsl:7-30, caelix_light_bvh_scan.hlsl
 *   wide           shaders/light/bvh/caelix_light_bvh_wide.hlsl:10-100
 *   finish         shaders/light/bvh/caelix_light_bvh_finish.hlsl:8-63
 * Every float operation is a separate IEEE fp32 operation in the HLSL order (no contraction).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---- helpers of shaders/common/caelix_light_tree_layout.hlsl ---- */

static uint32_t part1by2(uint32_t v) /* caelix_light_tree_layout.hlsl:247-255 */
{
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

uint32_t oc_morton(uint32_t x, uint32_t y, uint32_t z) /* :258-261 */
{
    return part1by2(x) | (part1by2(y) << 1) | (part1by2(z) << 2);
}

static float power6(const float f[6]) /* LtPower :271-274 */
{
    return f[0] + f[1] + f[2] + f[3] + f[4] + f[5];
}

static float fminf_h(float a, float b) { return b < a ? b : a; }
static float fmaxf_h(float a, float b) { return b > a ? b : a; }

static oc_summary empty_summary(void)
{
    oc_summary s;
    memset(&s, 0, sizeof(s));
    return s;
}

static oc_summary lt_union(const oc_summary* a, const oc_summary* b) /* LtUnion :315-334 */
{
    if (power6(a->face) <= 0.0f) return *b;
    if (power6(b->face) <= 0.0f) return *a;
    oc_summary s;
    for (int f = 0; f < 6; ++f) s.face[f] = a->face[f] + b->face[f];
    for (int k = 0; k < 3; ++k) {
        s.lo[k] = fminf_h(a->lo[k], b->lo[k]);
        s.hi[k] = fmaxf_h(a->hi[k], b->hi[k]);
    }
    return s;
}

/* Order-preserving map of a float to u32 (non-NaN): the bounds reduction compares through it,
 * so min/max are exact and independent of the reduction order (-0 sorts below +0). */
static uint32_t ordered(float f)
{
    uint32_t u;
    memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

/* LtWorldSummary, caelix_light_gather_emit.hlsl:11-34. */
static oc_summary world_summary(const oc_summary* local, const float r[9], const float t[3])
{
    float centre[3], half[3], wc[3], wh[3];
    for (int k = 0; k < 3; ++k) {
        centre[k] = 0.5f * (local->lo[k] + local->hi[k]);
        half[k] = 0.5f * (local->hi[k] - local->lo[k]);
    }
    for (int row = 0; row < 3; ++row) {
        const float* R = r + 3 * row;
        wc[row] = R[0] * centre[0] + R[1] * centre[1] + R[2] * centre[2] + t[row];
        wh[row] = fabsf(R[0]) * half[0] + fabsf(R[1]) * half[1] + fabsf(R[2]) * half[2];
    }
    oc_summary w = empty_summary();
    for (int k = 0; k < 3; ++k) {
        w.lo[k] = wc[k] - wh[k];
        w.hi[k] = wc[k] + wh[k];
    }
    for (int f = 0; f < 6; ++f) {
        const int axis = f >> 1;
        const float sign = (f & 1) ? -1.0f : 1.0f;
        const float d[3] = {sign * r[0 * 3 + axis], sign * r[1 * 3 + axis], sign * r[2 * 3 + axis]};
        for (int b = 0; b < 3; ++b) {
            w.face[2 * b] += local->face[f] * fmaxf_h(0.0f, d[b]);
            w.face[2 * b + 1] += local->face[f] * fmaxf_h(0.0f, -d[b]);
        }
    }
    return w;
}

/* ---- the radix sort ---- */

void oc_radix_sort_pairs(uint32_t* keys, uint32_t* values, uint32_t n)
{
    if (n < 2) return;
    uint32_t* k2 = (uint32_t*)malloc((size_t)n * 4);
    uint32_t* v2 = (uint32_t*)malloc((size_t)n * 4);
    uint32_t* ks = keys;
    uint32_t* vs = values;
    uint32_t* kd = k2;
    uint32_t* vd = v2;
    for (int pass = 0; pass < 4; ++pass) {
        const int shift = 8 * pass;
        uint32_t count[256];
        memset(count, 0, sizeof(count));
        for (uint32_t i = 0; i < n; ++i) ++count[(ks[i] >> shift) & 255u];
        uint32_t run = 0;
        for (int d = 0; d < 256; ++d) {
            const uint32_t c = count[d];
            count[d] = run;
            run += c;
        }
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t at = count[(ks[i] >> shift) & 255u]++;
            kd[at] = ks[i];
            vd[at] = vs[i];
        }
        uint32_t* t = ks; ks = kd; kd = t;
        t = vs; vs = vd; vd = t;
    }
    /* After 4 passes the result is back in the caller's arrays (even pass count). */
    free(k2);
    free(v2);
}

/* ---- Karras (caelix_light_bvh_karras.hlsl:8-96) ---- */

static uint32_t clz32(uint32_t x) { return x == 0 ? 32u : (uint32_t)__builtin_clz(x); }

static int delta(const uint32_t* keys, int i, int j, int n, uint32_t key_i)
{
    if (j < 0 || j >= n) return -1;
    const uint32_t key_j = keys[j];
    if (key_i == key_j) return 32 + (int)clz32((uint32_t)i ^ (uint32_t)j);
    return (int)clz32(key_i ^ key_j);
}

static void karras_node(const uint32_t* keys, int n, int i, uint32_t* left, uint32_t* right,
                        uint32_t* parent, uint32_t* leaf_parent)
{
    const uint32_t key_i = keys[i];
    const int d = delta(keys, i, i + 1, n, key_i) - delta(keys, i, i - 1, n, key_i) >= 0 ? 1 : -1;
    const int delta_min = delta(keys, i, i - d, n, key_i);
    int length_max = 2;
    while (delta(keys, i, i + length_max * d, n, key_i) > delta_min) length_max *= 2;
    int length = 0;
    for (int step = length_max / 2; step >= 1; step /= 2)
        if (delta(keys, i, i + (length + step) * d, n, key_i) > delta_min) length += step;
    const int j = i + length * d;
    const int delta_node = delta(keys, i, j, n, key_i);
    int split = 0;
    int divisor = 2;
    int step2 = (length + divisor - 1) / divisor;
    for (;;) {
        if (delta(keys, i, i + (split + step2) * d, n, key_i) > delta_node) split += step2;
        if (step2 == 1) break;
        divisor *= 2;
        step2 = (length + divisor - 1) / divisor;
    }
    const int gamma = i + split * d + (d < 0 ? d : 0);
    const int mn = i < j ? i : j;
    const int mx = i < j ? j : i;
    const uint32_t l = mn == gamma ? (OC_CHILD_LEAF_BIT | (uint32_t)gamma) : (uint32_t)gamma;
    const uint32_t r = mx == gamma + 1 ? (OC_CHILD_LEAF_BIT | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
    left[i] = l;
    right[i] = r;
    if (l & OC_CHILD_LEAF_BIT) leaf_parent[l & ~OC_CHILD_LEAF_BIT] = (uint32_t)i;
    else parent[l] = (uint32_t)i;
    if (r & OC_CHILD_LEAF_BIT) leaf_parent[r & ~OC_CHILD_LEAF_BIT] = (uint32_t)i;
    else parent[r] = (uint32_t)i;
}

/* LtBinaryChildSummary (caelix_light_bvh_common.hlsl:94-121). */
static oc_summary child_summary(uint32_t child, const oc_build_out* o)
{
    if (child & OC_CHILD_LEAF_BIT) return o->leaves[o->values[child & ~OC_CHILD_LEAF_BIT]].s;
    return o->aggregates[child];
}

int oc_lt_build(const oc_record* records, uint32_t n_found, const uint32_t* rec_group,
                const uint32_t* rec_entry, const oc_frame* group_frames, uint32_t leaf_capacity,
                uint32_t node_capacity, const oc_build_out* o)
{
    static const float identity[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    static const float zero3[3] = {0, 0, 0};
    int status = 0;
    const uint32_t n = n_found < leaf_capacity ? n_found : leaf_capacity;

    /* Gather emit: leaf i = record i moved to world space. */
    for (uint32_t i = 0; i < n; ++i) {
        const oc_record* r = &records[i];
        const uint32_t g = rec_group ? rec_group[i] : 0u;
        const float* origin = group_frames ? group_frames[g].origin : zero3;
        const float* rot = group_frames ? group_frames[g].rot : identity;
        const float* trans = group_frames ? group_frames[g].trans : zero3;
        oc_summary local;
        memcpy(local.face, r->face, sizeof(local.face));
        const uint32_t bl[3] = {r->box_lo & 0x3FFu, (r->box_lo >> 10) & 0x3FFu, (r->box_lo >> 20) & 0x3FFu};
        const uint32_t bh[3] = {r->box_hi & 0x3FFu, (r->box_hi >> 10) & 0x3FFu, (r->box_hi >> 20) & 0x3FFu};
        for (int k = 0; k < 3; ++k) {
            local.lo[k] = origin[k] + (float)bl[k];
            local.hi[k] = origin[k] + (float)bh[k];
        }
        oc_leaf* leaf = &o->leaves[i];
        leaf->s = world_summary(&local, rot, trans);
        leaf->group = g;
        leaf->entry = rec_entry ? rec_entry[i] : i;
        leaf->pad = 0;
        leaf->parent = OC_NONE;
    }

    /* Bounds of the leaf box centres. */
    uint32_t blo[3], bhi[3];
    for (int k = 0; k < 3; ++k) {
        blo[k] = ordered(3.0e38f);
        bhi[k] = ordered(-3.0e38f);
    }
    for (uint32_t i = 0; i < n; ++i) {
        for (int k = 0; k < 3; ++k) {
            const float c = 0.5f * (o->leaves[i].s.lo[k] + o->leaves[i].s.hi[k]);
            const uint32_t u = ordered(c);
            if (u < blo[k]) blo[k] = u;
            if (u > bhi[k]) bhi[k] = u;
        }
    }
    float lo[3], hi[3];
    for (int k = 0; k < 3; ++k) {
        uint32_t u = (blo[k] & 0x80000000u) ? (blo[k] & 0x7FFFFFFFu) : ~blo[k];
        memcpy(&lo[k], &u, 4);
        u = (bhi[k] & 0x80000000u) ? (bhi[k] & 0x7FFFFFFFu) : ~bhi[k];
        memcpy(&hi[k], &u, 4);
        o->bounds[k] = lo[k];
        o->bounds[3 + k] = hi[k];
    }

    /* Morton codes. */
    float extent[3];
    for (int k = 0; k < 3; ++k) extent[k] = fmaxf_h(hi[k] - lo[k], 1e-6f);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t cell[3];
        for (int k = 0; k < 3; ++k) {
            const float c = 0.5f * (o->leaves[i].s.lo[k] + o->leaves[i].s.hi[k]);
            float q = (c - lo[k]) / extent[k] * 1024.0f;
            q = fminf_h(fmaxf_h(q, 0.0f), 1023.0f);
            cell[k] = (uint32_t)q;
        }
        o->keys[i] = oc_morton(cell[0], cell[1], cell[2]);
        o->values[i] = i;
    }
    oc_radix_sort_pairs(o->keys, o->values, n);

    /* Karras binary radix tree. */
    if (n >= 2) {
        o->parent[0] = OC_NONE;
        for (uint32_t i = 0; i + 1 < n; ++i)
            karras_node(o->keys, (int)n, (int)i, o->left, o->right, o->parent, o->leaf_parent);
    }

    /* Aggregation: a node's summary is the union of its children's, computed bottom-up (the GPU
     * order of arrival does not change the value). Children of node i have larger indices or are
     * leaves except for the root's chain, so a post-order walk is used. */
    if (n >= 2) {
        uint32_t* stack = (uint32_t*)malloc((size_t)n * 2 * sizeof(uint32_t));
        uint8_t* expanded = (uint8_t*)calloc(n, 1);
        uint32_t top = 0;
        stack[top++] = 0;
        while (top) {
            const uint32_t node = stack[top - 1];
            if (!expanded[node]) {
                expanded[node] = 1;
                if (!(o->right[node] & OC_CHILD_LEAF_BIT)) stack[top++] = o->right[node];
                if (!(o->left[node] & OC_CHILD_LEAF_BIT)) stack[top++] = o->left[node];
                continue;
            }
            --top;
            const oc_summary a = child_summary(o->left[node], o);
            const oc_summary b = child_summary(o->right[node], o);
            o->aggregates[node] = lt_union(&a, &b);
        }
        free(stack);
        free(expanded);
    }

    /* Depth (walk to the root, guard 128) and the even-depth flags, scanned to 4-wide indices. */
    uint32_t node_count_scan = 0;
    for (uint32_t i = 0; i < leaf_capacity; ++i) {
        uint32_t flag = 0;
        if (i + 1 < n) {
            uint32_t d = 0;
            uint32_t node = o->parent[i];
            uint32_t guard = 0;
            for (; guard < 128 && node != OC_NONE; ++guard) {
                ++d;
                node = o->parent[node];
            }
            if (node != OC_NONE) status = -1;
            o->depth[i] = d;
            flag = (d & 1u) == 0 ? 1u : 0u;
        }
        o->wide[i] = node_count_scan;
        node_count_scan += flag;
    }

    /* Wide collapse. */
    for (uint32_t i = 0; i + 1 < n; ++i) {
        if (o->depth[i] & 1u) continue;
        const uint32_t w = o->wide[i];
        if (w >= node_capacity) continue;
        uint32_t slots[4] = {OC_NONE, OC_NONE, OC_NONE, OC_NONE};
        uint32_t count = 0;
        const uint32_t children[2] = {o->left[i], o->right[i]};
        for (int c = 0; c < 2; ++c) {
            const uint32_t child = children[c];
            if (child & OC_CHILD_LEAF_BIT) {
                slots[count++] = child;
            } else {
                slots[count++] = o->left[child];
                slots[count++] = o->right[child];
            }
        }
        oc_node* node = &o->nodes[w];
        for (uint32_t s = 0; s < 4; ++s) {
            oc_summary sm = empty_summary();
            uint32_t word = OC_NONE;
            if (s < count) {
                const uint32_t slot = slots[s];
                sm = child_summary(slot, o);
                if (slot & OC_CHILD_LEAF_BIT) {
                    const uint32_t leaf = o->values[slot & ~OC_CHILD_LEAF_BIT];
                    word = OC_CHILD_LEAF_BIT | leaf;
                    o->leaves[leaf].parent = (w << 2) | s;
                } else {
                    const uint32_t child_node = o->wide[slot];
                    word = child_node;
                    if (child_node < node_capacity) {
                        o->nodes[child_node].parent = w;
                        o->nodes[child_node].parent_slot = s;
                    }
                }
            }
            memcpy(node->child_face[s], sm.face, sizeof(sm.face));
            memcpy(node->child_lo[s], sm.lo, sizeof(sm.lo));
            memcpy(node->child_hi[s], sm.hi, sizeof(sm.hi));
            node->child[s] = word;
        }
        if (i == 0) {
            node->parent = OC_NONE;
            node->parent_slot = 0;
        }
    }

    /* Finish: the header. */
    oc_header* h = o->header;
    oc_summary root = empty_summary();
    uint32_t root_index = OC_NONE, node_count = 0, overflow = 0;
    if (n == 1) {
        root = o->leaves[0].s;
        oc_node* node = &o->nodes[0];
        memset(node->child_face, 0, sizeof(node->child_face));
        memset(node->child_lo, 0, sizeof(node->child_lo));
        memset(node->child_hi, 0, sizeof(node->child_hi));
        memcpy(node->child_face[0], root.face, sizeof(root.face));
        memcpy(node->child_lo[0], root.lo, sizeof(root.lo));
        memcpy(node->child_hi[0], root.hi, sizeof(root.hi));
        node->child[0] = OC_CHILD_LEAF_BIT | 0u;
        node->child[1] = node->child[2] = node->child[3] = OC_NONE;
        node->parent = OC_NONE;
        node->parent_slot = 0;
        o->leaves[0].parent = 0;
        root_index = 0;
        node_count = 1;
    } else if (n >= 2) {
        node_count = node_count_scan;
        if (node_count > node_capacity) overflow = 1;
        else {
            root = o->aggregates[0];
            root_index = 0;
        }
    }
    h->s = root;
    h->root = root_index;
    h->leaf_count = overflow ? 0u : n;
    h->node_count = node_count;
    h->pad = 0;
    o->node_overflow[0] = overflow;
    return status;
}
