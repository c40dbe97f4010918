/* Oracle of the scene side of the trace path (TEST INFRASTRUCTURE ONLY; see oracle.h):
 *   - brick records from raw bricks, restating the finalize kernel
 *     (shaders/scene/caelix_finalize.hlsl:110-340; its CPU twin is the reference's
 *     tests/finalize_test.cpp:74) in either block encoding (caelix_record.hlsl:180-212): per voxel
 *     "alive" (not all six neighbours opaque, an absent brick is air), occupied = alive && value
 *     != 0 && (opaque || a face bit), micro occupancy, coarse byte, tight bounds; opaque-only
 *     payloads are kept as uploaded;
 *   - the brick hash table: the reference's fingerprint (splitmix64 over the key words,
 *     shaders/common/caelix_hash_table.hlsl:102-128) and 16-byte key slots (key_lo, key_hi,
 *     payload, pad: lib/src/rhi/hash_table_layout.h:24-34), linear probing from the home slot.
 *     The build is canonical: keys are placed in the order (home slot, brick index), each at the
 *     first free slot at or after its home (a history-independent layout; no wrap, a tail of
 *     slots follows the table);
 *   - the brick light records and group light blocks, restating the group pass's record build
 *     (shaders/light/records/caelix_light_tree_build.hlsl:93-285): a light voxel is a voxel whose
 *     material code is in the light code set (LtOpenFaces), in a brick with emitter power above 0
 *     (a factor of its voxels' emission); its open faces (neighbour not opaque) are the face
 *     entries, sorted per family by voxel index; face sums = the sum over the entries of the
 *     luminance of the emission times the power (per lane of 16 voxels, then lanes folded 16, 8,
 *     4, 2, 1); box = tight box of the voxels with entries. Index
 *     entries in Morton order of the brick position (caelix_light_tree_layout.hlsl:338-361), the
 *     block layout of light_tree_layout.h:260-323.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

static uint32_t opaque_mask(uint32_t encoding) { return encoding == OC_ENCODING_PACKED ? 0xC000u : 0x8000u; }
static uint32_t id_mask(uint32_t encoding) { return encoding == OC_ENCODING_PACKED ? 0xFFu : 0x1FFu; }
static uint32_t face_shift(uint32_t encoding) { return encoding == OC_ENCODING_PACKED ? 8u : 9u; }

uint32_t oc_material_code(uint32_t value, uint32_t encoding)
{
    value &= 0xFFFFu;
    return (value & opaque_mask(encoding)) ? value : (value & id_mask(encoding));
}

void oc_light_codes(const float* emission, uint32_t encoding, float min_emission, uint32_t* out)
{
    memset(out, 0, 4 * (OC_MATERIAL_CODES / 32));
    for (uint32_t c = 0; c < OC_MATERIAL_CODES; ++c) {
        const float* e = emission + 3ull * oc_material_code(c, encoding);
        const float lum = 0.2126f * e[0] + 0.7152f * e[1] + 0.0722f * e[2];
        if (lum >= min_emission) out[c >> 5] |= 1u << (c & 31);
    }
}

static int is_light_code(const oc_scene* s, uint32_t value)
{
    const uint32_t c = oc_material_code(value, s->encoding);
    return (s->light_codes[c >> 5] >> (c & 31)) & 1u;
}

static uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

void oc_hash_fingerprint(int32_t x, int32_t y, int32_t z, uint32_t* key_lo, uint32_t* key_hi)
{
    uint64_t h = 0;
    h = splitmix64(h ^ (((uint64_t)(uint32_t)y << 32) | (uint32_t)x));
    h = splitmix64(h ^ (uint64_t)(uint32_t)z);
    const uint32_t lo = (uint32_t)h;
    const uint32_t hi = (uint32_t)(h >> 32);
    *key_lo = lo > 1u ? lo : 1u;
    *key_hi = hi != 0u ? hi : 1u;
}

uint32_t oc_hash_home(uint32_t key_lo, uint32_t capacity)
{
    return (uint32_t)(((uint64_t)key_lo * capacity) >> 32);
}

uint32_t oc_hash_lookup(const oc_scene* s, int32_t x, int32_t y, int32_t z)
{
    uint32_t lo, hi;
    oc_hash_fingerprint(x, y, z, &lo, &hi);
    const uint32_t home = oc_hash_home(lo, s->hash_capacity);
    for (uint32_t p = home; p <= home + s->hash_max_probe; ++p) {
        const uint32_t* slot = s->hash_slots + 4ull * p;
        if (slot[0] == 0) return OC_NONE;
        if (slot[0] == lo && slot[1] == hi) return slot[2];
    }
    return OC_NONE;
}

static uint16_t voxel_at(const oc_scene_desc* d, const oc_scene* s, int32_t bx, int32_t by, int32_t bz, int vx,
                         int vy, int vz)
{
    /* Voxel (vx, vy, vz) relative to brick (bx, by, bz), possibly in a neighbour brick. */
    while (vx < 0) { vx += 8; --bx; }
    while (vx > 7) { vx -= 8; ++bx; }
    while (vy < 0) { vy += 8; --by; }
    while (vy > 7) { vy -= 8; ++by; }
    while (vz < 0) { vz += 8; --bz; }
    while (vz > 7) { vz -= 8; ++bz; }
    const uint32_t r = oc_hash_lookup(s, bx, by, bz);
    if (r == OC_NONE) return 0; /* an absent brick is air */
    return d->voxels[512ull * r + (uint32_t)(vx + 8 * vy + 64 * vz)];
}

static void build_hash(const oc_scene_desc* d, oc_scene* s)
{
    const uint32_t n = d->brick_count;
    uint32_t cap = 2 * n;
    if (cap < 2) cap = 2;
    s->hash_capacity = cap;
    s->hash_slot_count = cap + n + 1;
    s->hash_slots = (uint32_t*)calloc(4ull * s->hash_slot_count, 4);
    uint32_t* lo = (uint32_t*)malloc(4ull * (n ? n : 1));
    uint32_t* hi = (uint32_t*)malloc(4ull * (n ? n : 1));
    uint32_t* home = (uint32_t*)malloc(4ull * (n ? n : 1));
    uint32_t* order = (uint32_t*)malloc(4ull * (n ? n : 1));
    for (uint32_t i = 0; i < n; ++i) {
        oc_hash_fingerprint(d->keys[3 * i], d->keys[3 * i + 1], d->keys[3 * i + 2], &lo[i], &hi[i]);
        home[i] = oc_hash_home(lo[i], cap);
        order[i] = i;
    }
    /* Stable order by home slot (ties: brick index). */
    oc_radix_sort_pairs(home, order, n);
    uint32_t max_probe = 0;
    int64_t prev = -1;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t b = order[k];
        int64_t pos = home[k];
        if (pos <= prev) pos = prev + 1;
        prev = pos;
        uint32_t* slot = s->hash_slots + 4ull * (uint64_t)pos;
        slot[0] = lo[b];
        slot[1] = hi[b];
        slot[2] = b;
        slot[3] = 0;
        if ((uint32_t)(pos - home[k]) > max_probe) max_probe = (uint32_t)(pos - home[k]);
    }
    s->hash_max_probe = max_probe;
    free(lo);
    free(hi);
    free(home);
    free(order);
}

static void build_records(const oc_scene_desc* d, oc_scene* s)
{
    const uint32_t n = d->brick_count;
    const uint32_t gshift = d->group_shift;
    const uint32_t gmask = (1u << gshift) - 1u;
    const uint32_t OPAQUE = opaque_mask(d->encoding), IDS = id_mask(d->encoding), FSHIFT = face_shift(d->encoding);
    s->records = (uint32_t*)calloc((size_t)n * OC_RECORD_WORDS, 4);
    for (uint32_t b = 0; b < n; ++b) {
        const int32_t bx = d->keys[3 * b], by = d->keys[3 * b + 1], bz = d->keys[3 * b + 2];
        const uint16_t* vox = d->voxels + 512ull * b;
        uint32_t* rec = s->records + (size_t)b * OC_RECORD_WORDS;
        uint32_t occ[16] = {0};
        int mn[3] = {8, 8, 8}, mx[3] = {-1, -1, -1};
        for (int z = 0; z < 8; ++z)
            for (int y = 0; y < 8; ++y)
                for (int x = 0; x < 8; ++x) {
                    const uint32_t v = vox[x + 8 * y + 64 * z];
                    const uint32_t code = oc_material_code(v, d->encoding);
                    static const int dx[6] = {1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, 1, -1, 0, 0},
                                     dz[6] = {0, 0, 0, 0, 1, -1};
                    uint32_t opaque_count = 0, faces = 0;
                    for (int f = 0; f < 6; ++f) {
                        const uint32_t nv = voxel_at(d, s, bx, by, bz, x + dx[f], y + dy[f], z + dz[f]);
                        const int nop = (nv & OPAQUE) != 0;
                        opaque_count += nop;
                        if (!nop && (nv & IDS) != code) faces |= 1u << f;
                    }
                    const int alive = opaque_count < 6;
                    const uint32_t result = (code & OPAQUE) ? code : (code | (faces << FSHIFT));
                    const int iface = (code & OPAQUE) != 0 || faces != 0;
                    const uint32_t word = 18 + (x >> 1) + 4 * y + 32 * z;
                    rec[word] |= (x & 1) ? (result << 16) : result;
                    if (alive && result != 0 && iface) {
                        const int c = (x >> 2) | ((y >> 2) << 1) | ((z >> 2) << 2);
                        const int m = (x & 3) | ((y & 3) << 2) | ((z & 3) << 4);
                        occ[2 * c + (m >> 5)] |= 1u << (m & 31);
                        if (x < mn[0]) mn[0] = x;
                        if (x > mx[0]) mx[0] = x;
                        if (y < mn[1]) mn[1] = y;
                        if (y > mx[1]) mx[1] = y;
                        if (z < mn[2]) mn[2] = z;
                        if (z > mx[2]) mx[2] = z;
                    }
                }
        uint32_t coarse = 0;
        for (int c = 0; c < 8; ++c)
            if (occ[2 * c] | occ[2 * c + 1]) coarse |= 1u << c;
        const uint32_t pos = ((uint32_t)bx & gmask) | (((uint32_t)by & gmask) << gshift) |
                             (((uint32_t)bz & gmask) << (2 * gshift));
        rec[0] = (pos & 0xFFFFu) | (coarse << 16);
        uint32_t bounds = 0;
        if (mx[0] >= 0)
            bounds = (uint32_t)mn[0] | ((uint32_t)mn[1] << 3) | ((uint32_t)mn[2] << 6) | ((uint32_t)mx[0] << 9) |
                     ((uint32_t)mx[1] << 12) | ((uint32_t)mx[2] << 15);
        rec[1] = bounds;
        memcpy(rec + 2, occ, sizeof(occ));
    }
}

static uint32_t morton10(uint32_t x, uint32_t y, uint32_t z) { return oc_morton(x, y, z); }

typedef struct light_brick {
    uint32_t key; /* group << 12 | Morton of the group-local brick position (group_shift <= 4) */
    uint32_t brick;
} light_brick;

static int cmp_light(const void* a, const void* b)
{
    const light_brick* x = (const light_brick*)a;
    const light_brick* y = (const light_brick*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->brick < y->brick ? -1 : (x->brick > y->brick);
}

/* The record of one light brick: header + face entries. Returns the entry count. */
static uint32_t light_record(const oc_scene_desc* d, const oc_scene* s, uint32_t b, uint32_t pos, oc_record* h,
                             uint32_t* entries)
{
    const int32_t bx = d->keys[3 * b], by = d->keys[3 * b + 1], bz = d->keys[3 * b + 2];
    const uint16_t* vox = d->voxels + 512ull * b;
    static const int dx[6] = {1, -1, 0, 0, 0, 0}, dy[6] = {0, 0, 1, -1, 0, 0}, dz[6] = {0, 0, 0, 0, 1, -1};
    const float P = d->power[b];
    const uint32_t OPAQUE = opaque_mask(d->encoding);
    uint32_t open[512];
    uint32_t counts[6] = {0};
    for (uint32_t vi = 0; vi < 512; ++vi) {
        const int x = vi & 7, y = (vi >> 3) & 7, z = vi >> 6;
        open[vi] = 0;
        if (!is_light_code(s, vox[vi])) continue;
        for (int f = 0; f < 6; ++f) {
            const uint32_t nv = voxel_at(d, s, bx, by, bz, x + dx[f], y + dy[f], z + dz[f]);
            if (!(nv & OPAQUE)) open[vi] |= 1u << f;
        }
        for (int f = 0; f < 6; ++f) counts[f] += (open[vi] >> f) & 1u;
    }
    uint32_t base[6], written = 0;
    for (int f = 0; f < 6; ++f) {
        base[f] = written;
        written += counts[f];
    }
    uint32_t cursor[6] = {0};
    float lane_sums[32][6];
    memset(lane_sums, 0, sizeof(lane_sums));
    uint32_t lo[3] = {8, 8, 8}, hi[3] = {0, 0, 0};
    for (uint32_t vi = 0; vi < 512; ++vi) {
        if (!open[vi]) continue;
        const uint32_t lane = vi >> 4;
        /* LtLuminance of the voxel's emission times the brick's power (each channel times P). */
        const float* e = d->emission + 3ull * oc_material_code(vox[vi], d->encoding);
        const float weight = (e[0] * P) * 0.2126f + (e[1] * P) * 0.7152f + (e[2] * P) * 0.0722f;
        for (int f = 0; f < 6; ++f) {
            if (!((open[vi] >> f) & 1u)) continue;
            entries[base[f] + cursor[f]] = vi | ((uint32_t)vox[vi] << 16);
            ++cursor[f];
            lane_sums[lane][f] += weight;
        }
        const uint32_t p[3] = {vi & 7, (vi >> 3) & 7, vi >> 6};
        for (int k = 0; k < 3; ++k) {
            if (p[k] < lo[k]) lo[k] = p[k];
            if (p[k] + 1 > hi[k]) hi[k] = p[k] + 1;
        }
    }
    for (int off = 16; off >= 1; off >>= 1)
        for (int l = 0; l < off; ++l)
            for (int f = 0; f < 6; ++f) lane_sums[l][f] += lane_sums[l + off][f];
    for (int f = 0; f < 6; ++f) h->face[f] = lane_sums[0][f];
    const uint32_t gshift = d->group_shift;
    const uint32_t gmask = (1u << gshift) - 1u;
    const uint32_t org[3] = {((uint32_t)bx & gmask) * 8, ((uint32_t)by & gmask) * 8, ((uint32_t)bz & gmask) * 8};
    if (written == 0) {
        lo[0] = lo[1] = lo[2] = 0;
        hi[0] = hi[1] = hi[2] = 0;
    }
    h->box_lo = (org[0] + lo[0]) | ((org[1] + lo[1]) << 10) | ((org[2] + lo[2]) << 20);
    h->box_hi = (org[0] + hi[0]) | ((org[1] + hi[1]) << 10) | ((org[2] + hi[2]) << 20);
    h->pos = pos;
    h->entry_count = written;
    h->counts_lo = counts[0] | (counts[1] << 10) | (counts[2] << 20);
    h->counts_hi = counts[3] | (counts[4] << 10) | (counts[5] << 20);
    return written;
}

static void build_lights(const oc_scene_desc* d, oc_scene* s)
{
    const uint32_t n = d->brick_count;
    const uint32_t gshift = d->group_shift;
    const uint32_t gmask = (1u << gshift) - 1u;
    for (int k = 0; k < 3; ++k) s->groups[k] = (d->grid[k] + gmask) >> gshift;
    s->group_count = s->groups[0] * s->groups[1] * s->groups[2];
    light_brick* lb = (light_brick*)malloc(sizeof(light_brick) * (n ? n : 1));
    uint32_t m = 0;
    for (uint32_t b = 0; b < n && d->lights; ++b) {
        if (!(d->power[b] > 0.0f)) continue;
        int any = 0;
        for (uint32_t vi = 0; vi < 512 && !any; ++vi) any = is_light_code(s, d->voxels[512ull * b + vi]);
        if (!any) continue;
        const uint32_t bx = (uint32_t)(d->keys[3 * b] - d->origin[0]), by = (uint32_t)(d->keys[3 * b + 1] - d->origin[1]),
                       bz = (uint32_t)(d->keys[3 * b + 2] - d->origin[2]);
        const uint32_t g = (bx >> gshift) + s->groups[0] * ((by >> gshift) + s->groups[1] * (bz >> gshift));
        lb[m].key = (g << (3 * gshift)) | morton10(bx & gmask, by & gmask, bz & gmask);
        lb[m].brick = b;
        ++m;
    }
    qsort(lb, m, sizeof(light_brick), cmp_light);
    s->light_count = m;
    s->light_headers = (oc_record*)calloc(m ? m : 1, sizeof(oc_record));
    s->light_group = (uint32_t*)calloc(m ? m : 1, 4);
    s->light_entry = (uint32_t*)calloc(m ? m : 1, 4);
    s->light_brick = (uint32_t*)calloc(m ? m : 1, 4);
    s->group_rows = (uint32_t*)calloc((size_t)s->group_count * 8, 4);
    s->group_frames = (oc_frame*)calloc(s->group_count ? s->group_count : 1, sizeof(oc_frame));
    for (uint32_t g = 0; g < s->group_count; ++g) {
        const uint32_t gx = g % s->groups[0], gy = (g / s->groups[0]) % s->groups[1],
                       gz = g / (s->groups[0] * s->groups[1]);
        oc_frame* f = &s->group_frames[g];
        f->origin[0] = (float)(8ll * ((int64_t)d->origin[0] + ((int64_t)gx << gshift)));
        f->origin[1] = (float)(8ll * ((int64_t)d->origin[1] + ((int64_t)gy << gshift)));
        f->origin[2] = (float)(8ll * ((int64_t)d->origin[2] + ((int64_t)gz << gshift)));
        f->rot[0] = f->rot[4] = f->rot[8] = 1.0f;
    }
    /* Heap: one block per group with light bricks, in group order. */
    size_t cap_words = 64;
    uint32_t* heap = (uint32_t*)calloc(cap_words, 4);
    size_t used_units = 1; /* unit 0 stays unused: block_units 0 means no block */
    uint32_t* entries = (uint32_t*)malloc(4 * 3072);
    uint32_t i = 0;
    while (i < m) {
        const uint32_t g = lb[i].key >> (3 * gshift);
        uint32_t j = i;
        while (j < m && (lb[j].key >> (3 * gshift)) == g) ++j;
        const uint32_t count = j - i;
        /* Size: header unit, index entries, records. */
        oc_record* hdrs = s->light_headers + i;
        uint32_t* ents = (uint32_t*)malloc(4ull * 3072 * count);
        uint32_t* ecount = (uint32_t*)malloc(4ull * count);
        size_t units = 1 + count;
        for (uint32_t k = 0; k < count; ++k) {
            const uint32_t b = lb[i + k].brick;
            const uint32_t pos = s->records[(size_t)b * OC_RECORD_WORDS] & 0xFFFFu;
            ecount[k] = light_record(d, s, b, pos, &hdrs[k], ents + 3072ull * k);
            units += (48 + 4ull * ecount[k] + 15) / 16;
            s->light_group[i + k] = g;
            s->light_entry[i + k] = k;
            s->light_brick[i + k] = b;
        }
        while ((used_units + units) * 4 > cap_words) {
            const size_t old = cap_words;
            cap_words *= 2;
            heap = (uint32_t*)realloc(heap, cap_words * 4);
            memset(heap + old, 0, (cap_words - old) * 4);
        }
        const size_t block = used_units;
        uint32_t* bw = heap + 4 * block;
        bw[0] = count;
        size_t rec_unit = 1 + count;
        uint32_t faces = 0;
        for (uint32_t k = 0; k < count; ++k) {
            uint32_t* ie = bw + 4 * (1 + k);
            ie[0] = hdrs[k].pos;
            ie[1] = lb[i + k].brick;
            ie[2] = (uint32_t)rec_unit;
            ie[3] = i + k; /* tree 0, leaf = gather order */
            uint32_t* rw = bw + 4 * rec_unit;
            memcpy(rw, &hdrs[k], 48);
            memcpy(rw + 12, ents + 3072ull * k, 4ull * ecount[k]);
            rec_unit += (48 + 4ull * ecount[k] + 15) / 16;
            faces += ecount[k];
        }
        uint32_t* row = s->group_rows + 8ull * g;
        row[0] = (uint32_t)block;
        row[1] = (uint32_t)units;
        row[2] = 0;
        row[5] = count;
        row[6] = faces;
        used_units += units;
        free(ents);
        free(ecount);
        i = j;
    }
    free(entries);
    free(lb);
    s->heap = heap;
    s->heap_words = (uint32_t)(used_units * 4);
}

int oc_scene_build(const oc_scene_desc* d, oc_scene* s)
{
    memset(s, 0, sizeof(*s));
    for (int k = 0; k < 3; ++k) {
        s->grid[k] = d->grid[k];
        s->origin[k] = d->origin[k];
    }
    s->group_shift = d->group_shift;
    s->brick_count = d->brick_count;
    s->encoding = d->encoding;
    s->emission = d->emission;
    s->light_codes = (uint32_t*)malloc(4 * (OC_MATERIAL_CODES / 32));
    oc_light_codes(d->emission, d->encoding, d->min_emission, s->light_codes);
    s->keys = (int32_t*)malloc(12ull * (d->brick_count ? d->brick_count : 1));
    memcpy(s->keys, d->keys, 12ull * d->brick_count);
    build_hash(d, s);
    build_records(d, s);
    /* Brick occupancy bitmap by linear brick index of the box (origin, grid). */
    const uint64_t cells = (uint64_t)d->grid[0] * d->grid[1] * d->grid[2];
    s->bitmap_words = (uint32_t)((cells + 31) / 32);
    s->bitmap = (uint32_t*)calloc(s->bitmap_words ? s->bitmap_words : 1, 4);
    for (uint32_t b = 0; b < d->brick_count; ++b) {
        const uint64_t c = (uint64_t)(uint32_t)(d->keys[3 * b] - d->origin[0]) +
                           d->grid[0] * ((uint64_t)(uint32_t)(d->keys[3 * b + 1] - d->origin[1]) +
                                         (uint64_t)d->grid[1] * (uint32_t)(d->keys[3 * b + 2] - d->origin[2]));
        s->bitmap[c >> 5] |= 1u << (c & 31);
    }
    build_lights(d, s);
    return 0;
}

void oc_scene_free(oc_scene* s)
{
    free(s->light_codes);
    free(s->keys);
    free(s->records);
    free(s->hash_slots);
    free(s->bitmap);
    free(s->light_headers);
    free(s->light_group);
    free(s->light_entry);
    free(s->light_brick);
    free(s->heap);
    free(s->group_rows);
    free(s->group_frames);
    memset(s, 0, sizeof(*s));
}
