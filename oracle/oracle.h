/* CPU oracle of the scene-flush and trace hot path of the Caelix voxel renderer.
 *
 * TEST INFRASTRUCTURE ONLY. This is a scalar C restatement of the reference's HLSL kernels, used
 * as the checker by the parity tests, by the smoke check and as the timed CPU baseline of the
 * benchmark. The product library never links, loads or calls it.
 *
 * Layouts restate lib/src/light/light_tree_layout.h of the reference byte for byte (the structs
 * below carry the same offsets; tests/test_layout.py compares them with the reference header
 * compiled by oracle/ref_layout.mk). Arithmetic is IEEE fp32 without contraction (built with
 * -ffp-contract=off), in the operation order of the HLSL source.
 */
#ifndef CAELIX_ORACLE_H
#define CAELIX_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OC_NONE 0xFFFFFFFFu
#define OC_CHILD_LEAF_BIT 0x80000000u

/* LightSummary (light_tree_layout.h:89-102): 48 bytes. */
typedef struct oc_summary {
    float face[6];
    float lo[3];
    float hi[3];
} oc_summary;

/* BrickLightRecordHeader (light_tree_layout.h:298-323): 48 bytes. */
typedef struct oc_record {
    float face[6];
    uint32_t box_lo; /* packed group-local voxel x | y << 10 | z << 20, inclusive */
    uint32_t box_hi; /* exclusive */
    uint32_t pos;
    uint32_t entry_count;
    uint32_t counts_lo;
    uint32_t counts_hi;
} oc_record;

/* LightBvhLeaf (light_tree_layout.h:338-354): 64 bytes. */
typedef struct oc_leaf {
    oc_summary s;
    uint32_t group;
    uint32_t entry;
    uint32_t pad;
    uint32_t parent; /* node << 2 | slot */
} oc_leaf;

/* LightBvhNode (light_tree_layout.h:359-389): 224 bytes. */
typedef struct oc_node {
    float child_face[4][6];
    float child_lo[4][3];
    float child_hi[4][3];
    uint32_t child[4];
    uint32_t parent;
    uint32_t parent_slot;
    uint32_t pad[2];
} oc_node;

/* LightTreeHeader (light_tree_layout.h:105-121): 64 bytes. */
typedef struct oc_header {
    oc_summary s;
    uint32_t root;
    uint32_t leaf_count;
    uint32_t node_count;
    uint32_t pad;
} oc_header;

/* The frame a record's group-local box is moved to world space with (the group's voxel origin
 * and its entity's object-to-world rows, caelix_light_tree_layout.hlsl:409-433). */
typedef struct oc_frame {
    float origin[3];
    float rot[9]; /* row-major rows */
    float trans[3];
} oc_frame;

/* Every array the build writes, each of leaf_capacity elements unless stated. The build
 * scratch arrays of light_tree_layout.h:392-423. */
typedef struct oc_build_out {
    oc_leaf* leaves;         /* [leaf_capacity] */
    oc_node* nodes;          /* [node_capacity] */
    oc_header* header;       /* [1] */
    uint32_t* keys;          /* sorted Morton codes */
    uint32_t* values;        /* sorted leaf indices */
    uint32_t* left;          /* binary node children (OC_CHILD_LEAF_BIT: sorted leaf position) */
    uint32_t* right;
    uint32_t* parent;        /* binary node parent, OC_NONE = root */
    uint32_t* leaf_parent;   /* binary parent of the leaf at each sorted position */
    uint32_t* depth;         /* binary node depth */
    uint32_t* wide;          /* 4-wide node index of an even-depth binary node (the scan) */
    oc_summary* aggregates;  /* binary node summaries */
    float* bounds;           /* [6] centre bounds lo[3], hi[3] */
    uint32_t* node_overflow; /* [1] */
} oc_build_out;

/* 30-bit Morton code of a cell (caelix_light_tree_layout.hlsl:247-261). */
uint32_t oc_morton(uint32_t x, uint32_t y, uint32_t z);

/* Stable LSD radix sort of (key, value) pairs by the 32-bit key, 8-bit digits, 4 passes. */
void oc_radix_sort_pairs(uint32_t* keys, uint32_t* values, uint32_t n);

/* The light BVH build of one tree over `n` brick light records (leaf i = record i):
 * gather emit, centre bounds, Morton codes, radix sort, Karras, aggregation, depth, wide
 * collapse, finish. rec_group / rec_entry give each leaf's (group, entry) words and
 * group_frames the frame of every group (rec_group NULL: group 0, entry i, identity frame at
 * origin 0). Returns 0, or -1 when a depth guard was exceeded. */
int oc_lt_build(const oc_record* records, uint32_t n, const uint32_t* rec_group,
                const uint32_t* rec_entry, const oc_frame* group_frames, uint32_t leaf_capacity,
                uint32_t node_capacity, const oc_build_out* out);

/* The importance of a summary for a point receiver x with unit normal n (0: no surface),
 * caelix_light_tree.hlsl:114-160. */
float oc_importance(const float x[3], const float n[3], const float lo[3], const float hi[3],
                    const float face[6]);

/* ---- scene (oracle/scene.c) ---- */

#define OC_RECORD_WORDS 274
#define OC_MATERIAL_CODES 65536

/* Block encodings (include/caelix/caelix.h:243-249): packed (0) is opaque on 0xC000, transparent
 * id = value & 0xFF, face bits at 8; block-ID (1) is opaque on 0x8000, id = value & 0x1FF, face
 * bits at 9. */
#define OC_ENCODING_PACKED 0u
#define OC_ENCODING_BLOCK_ID 1u
/* The material table index of a raw value: opaque values as they are, transparent ones without
 * their face bits (caelix_record.hlsl:205-212 BlockMaterialCode). */
uint32_t oc_material_code(uint32_t value, uint32_t encoding);

/* A voxel world of bricks: keys[i] = brick coordinate (x, y, z) of brick i, every coordinate in
 * [origin, origin + grid), in increasing linear index of that box; voxels[512 i + x + 8 y + 64 z]
 * = raw block value; power[i] = the brick's emitter power (a factor of its voxels' emission).
 * emission: the material table's emission, [65536][3] by code (a transparent code with face bits
 * is looked up without them); a light voxel's code has an emission luminance of at least
 * min_emission (the light code set, oc_light_codes). lights = 0: no light records. */
typedef struct oc_scene_desc {
    uint32_t grid[3];
    uint32_t group_shift;
    uint32_t brick_count;
    uint32_t encoding;
    int32_t origin[3];    /* brick key of grid cell 0, a multiple of the group edge */
    uint32_t lights;
    float min_emission;
    uint32_t pad;
    const int32_t* keys;
    const uint16_t* voxels;
    const float* power;
    const float* emission;
} oc_scene_desc;

/* The light code set (lib/src/light/light_tree.cpp:186-200 RebuildCodes): bit c of out[c / 32]
 * for every code whose canonical entry's emission luminance 0.2126 r + 0.7152 g + 0.0722 b is at
 * least min_emission. out: 2048 words. */
void oc_light_codes(const float* emission, uint32_t encoding, float min_emission, uint32_t* out);

struct oc_entity;
struct oc_light_tree;

typedef struct oc_scene {
    uint32_t grid[3];
    uint32_t group_shift;
    int32_t origin[3];
    uint32_t encoding;
    const float* emission;    /* the material table's emission [65536][3] (the desc's) */
    uint32_t* light_codes;    /* [2048] */
    int32_t* keys;            /* [brick_count][3] (a copy of the desc's) */
    uint32_t brick_count;
    uint32_t hash_capacity;   /* home slots (load factor 0.5) */
    uint32_t hash_slot_count; /* slots including the tail */
    uint32_t hash_max_probe;
    uint32_t bitmap_words;
    uint32_t light_count;
    uint32_t heap_words;
    uint32_t group_count;
    uint32_t groups[3];
    uint32_t pad;
    uint32_t* records;     /* [brick_count][274] */
    uint32_t* hash_slots;  /* [hash_slot_count][4]: key_lo, key_hi, record, 0 */
    uint32_t* bitmap;      /* brick occupancy by linear brick index */
    oc_record* light_headers; /* [light_count] in leaf (gather) order */
    uint32_t* light_group;
    uint32_t* light_entry;
    uint32_t* light_brick; /* scene record of every light brick */
    uint32_t* heap;        /* group light blocks (16-byte units) */
    uint32_t* group_rows;  /* [group_count][8] GroupLightRow */
    oc_frame* group_frames;
    /* Entities beside this scene's bricks (the static world, entity 0): rays also traverse each
     * entity's own scene under its transform; their lights are the light set `dyn`. */
    const struct oc_entity* entities;
    uint32_t entity_count;
    uint32_t pad2;
    /* The dynamic entities' lights (NULL: none): their light blocks, group rows, frames and power
     * merged into one light set (entity e's groups from its group_base, its bricks' power after
     * the others', every index entry's leaf word 0x80000000 | leaf of the dynamic tree) and the
     * dynamic light tree (tree 1) built over them. Static entities' lights are merged the same
     * way after the world's own into this scene's light set (heap, group rows, frames; leaf words
     * without the mark), with tree 0 built over both (the caller passes that tree and power). */
    const struct oc_scene* dyn;
    const struct oc_light_tree* dyn_tree;
    const float* dyn_power;
} oc_scene;

/* An entity: its bricks (a scene of their own, entity-local block coordinates from 0, with its
 * bricks' power and light records) and its object-to-world transform, world = rot * local + pos
 * (rot row-major). */
typedef struct oc_entity {
    const oc_scene* scene;
    float rot[9];
    float pos[3];
    uint32_t group_base; /* its first group in the light set of its tree */
    uint32_t id;         /* its entity id (the voxel id's entity word) */
    uint32_t tree;       /* the tree holding its lights: 0 (a static entity: the scene's own light set,
                          * which then holds the world's lights first and the static entities' after
                          * them), 1 (a dynamic entity: `dyn`), OC_NONE (none) */
    const float* power;  /* its bricks' emitter power */
} oc_entity;

/* An entity hit (oc_hit.attrib bit 15; the hit's group is then entity << 24 | the group in the
 * entity, its normal the rotated face normal and object_hit the entity-local point; cell is
 * bits 6..14, the block bits 16..31, so bit 15 is free). */
#define OC_ENTITY_HIT 0x8000u

/* Rotation rows of a quaternion (x, y, z, w; normalised first), computed in double and rounded:
 * the same arithmetic as the library's caelix_scene_set_entity_transform. */
void oc_entity_rows(const float q[4], float rot[9]);

int oc_scene_build(const oc_scene_desc* d, oc_scene* s);
void oc_scene_free(oc_scene* s);
void oc_hash_fingerprint(int32_t x, int32_t y, int32_t z, uint32_t* key_lo, uint32_t* key_hi);
uint32_t oc_hash_home(uint32_t key_lo, uint32_t capacity);
uint32_t oc_hash_lookup(const oc_scene* s, int32_t x, int32_t y, int32_t z);

/* ---- trace (oracle/trace.c) ---- */

typedef struct oc_camera {
    float position[3];
    float right[3];
    float up[3];
    float forward[3];
    float tan_half_fov_y;
    float aspect;
} oc_camera;

typedef struct oc_render_desc {
    uint32_t width;
    uint32_t height;
    uint32_t spp;
    uint32_t bounce_count;
    uint32_t frame_seed;
    uint32_t light_nee; /* 1: light-tree NEE with MIS */
    uint32_t x0, y0, x1, y1; /* pixel window rendered (the rest is left untouched) */
    uint32_t* voxel_id;  /* optional: [height][width][2], the voxel id of the camera ray's first hit */
    float voxel_id_tmax; /* hits farther than this are voxel id misses (0: no limit) */
    uint32_t pad;
} oc_render_desc;

/* A built light tree (the build's output) for the trace. */
typedef struct oc_light_tree {
    const oc_leaf* leaves;
    const oc_node* nodes;
    const oc_header* header;
} oc_light_tree;

typedef struct oc_hit {
    uint32_t hit;
    float t;
    uint32_t attrib;
    uint32_t record;
    uint32_t group;
    float normal[3];
    float object_hit[3];
} oc_hit;

/* Closest hit of a ray (unit direction) over the bricks, t in [tmin, tmax): the scene's own
 * bricks, then every entity in order (a ray in the entity's frame, local = rot^T (x - pos); an
 * entity hit replaces the current one only when strictly nearer). */
oc_hit oc_trace_ray(const oc_scene* s, const float origin[3], const float dir[3], float tmin, float tmax);

/* Renders the pixel window; radiance[3 * (y * width + x)] (fp32 RGB, averaged over spp);
 * rays[3]: primary, bounce, shadow rays traced. albedo: the material table's albedo [65536][3] by
 * code; power: per brick. Threads > 1 splits rows across threads. */
void oc_render(const oc_scene* s, const oc_light_tree* t, const float* albedo, const float* power,
               const oc_camera* cam, const oc_render_desc* r, float* radiance, uint64_t* rays, int threads);

/* The voxel id of a hit (shaders/render/caelix_scene_trace.hlsl:171-200): two hashes of (entity
 * id, entity-local voxel); the world is entity 0, an entity hit takes its oc_entity::id. */
void oc_voxel_id(const oc_scene* s, const oc_hit* h, uint32_t out[2]);

/* The adjoint reference (double precision): the estimator with the sampling quantities of the
 * fp32 render at (albedo, power) held fixed, evaluated at (A, P) (double; NULL = the fp32
 * parameters). image (may be NULL): the double image. d_radiance (may be NULL): dL/d(pixel);
 * then d_albedo [65536][3] (by material code) and d_power [brick_count] receive dL/dA and dL/dP
 * at (A, P). */
void oc_adjoint(const oc_scene* s, const oc_light_tree* t, const float* albedo, const float* power,
                const oc_camera* cam, const oc_render_desc* r, const double* A, const double* P,
                const float* d_radiance, double* image, double* d_albedo, double* d_power, int threads);

/* Light tree draw for a point receiver (caelix_light_tree.hlsl:749-767): returns 1 and fills
 * out[0..2] position, out[3..5] normal, out[6] pdf, words[0..5] block, voxel, face, group, entry,
 * tree (0: the world's light set, 1: the entities', s->dyn). */
int oc_light_sample(const oc_scene* s, const oc_light_tree* t, const float x[3], const float n[3], uint32_t rng,
                    float out[7], uint32_t words[6]);
/* count draws of oc_light_sample at one receiver (the reference probe's draw mode,
 * tests/light_tree_test.cpp:961 CheckHistogram): per draw out[4 i ..] = group, voxel in group
 * (x | y << 10 | z << 20), face, 1 | tree << 1 (all zero for a failed draw; tree 1: a group of
 * s->dyn). The draws' generator states come from an xorshift sequence started at seed. */
void oc_light_draws(const oc_scene* s, const oc_light_tree* t, const float x[3], const float n[3], uint32_t seed,
                    uint32_t count, uint32_t* out);
/* The balance-heuristic MIS weight of one side (caelix_light_nee.hlsl:20-34): p_area is the
 * light tree's area density of the lamp point, d its distance, cos_l the lamp-side cosine, n_r the
 * receiver normal, w the unit direction to the lamp; nee_side selects the light-sampling side. */
float oc_mis_weight(float p_area, const float n_r[3], const float w[3], float d, float cos_l, int nee_side);
/* The light tree pdf of a light face point (caelix_light_tree.hlsl:936-949). */
float oc_light_point_pdf(const oc_scene* s, const oc_light_tree* t, const float x[3], const float n[3],
                         uint32_t group, const uint32_t voxel_in_group[3], uint32_t face, uint32_t block);
/* The same for a light face of either light set (tree 1: group of s->dyn). */
float oc_light_point_pdf_tree(const oc_scene* s, const oc_light_tree* t, const float x[3], const float n[3],
                              uint32_t tree, uint32_t group, const uint32_t voxel_in_group[3], uint32_t face,
                              uint32_t block);

#ifdef __cplusplus
}
#endif
#endif
