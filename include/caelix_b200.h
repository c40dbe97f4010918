/* caelix_b200.h — C ABI of the B200-native scene-flush (light-tree build) and trace path of the
 * Caelix voxel renderer.
 *
 * C99-clean. Every entry point mirrors an entry point or an internal interface of the reference
 * library (betairylia/Caelix-Renderer); each declaration names the reference interface it replaces
 * by file:line (paths inside the reference project). Conventions kept from the reference
 * (include/caelix/caelix.h:1-140):
 *   - opaque handles owned by the library; destroy(NULL) is ignored;
 *   - every fallible call returns CaelixResult; exceptions never cross the ABI, failures are
 *     logged through the host callback;
 *   - input arrays are borrowed for the duration of the call;
 *   - calls on one object are externally synchronized by the host.
 * The Vulkan handles of the reference become CUDA ones: a device is a CUDA device ordinal, a
 * command buffer is a cudaStream_t carried as uint64_t (0 = the legacy default stream), buffer
 * device addresses are CUDA device pointers carried as uint64_t or typed pointers.
 */
#ifndef CAELIX_B200_H
#define CAELIX_B200_H

#include <stdint.h>

#if defined(_WIN32)
#define CAELIX_API __declspec(dllexport)
#else
#define CAELIX_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces include/caelix/caelix.h:99 (the ABI version of this library's structs). */
#define CAELIX_ABI_VERSION 2u

typedef struct CaelixVersion
{
    uint32_t major;
    uint32_t minor;
    uint32_t patch;
    uint32_t abi;
} CaelixVersion;

/* Replaces include/caelix/caelix.h:108-111. */
CAELIX_API void caelix_get_version(CaelixVersion* out);
CAELIX_API const char* caelix_version_string(void);

/* Replaces include/caelix/caelix.h:114-122. CAELIX_ERROR_CUDA takes the value of the reference's
   CAELIX_ERROR_VULKAN (a device API call failed). CAELIX_ERROR_DEVICE_STATUS is new: a kernel
   reported a failure in its status word (a bounded wait gave up, a guard or a capacity was
   exceeded) instead of trapping; the log names the bits. */
typedef enum CaelixResult
{
    CAELIX_OK = 0,
    CAELIX_ERROR_INVALID_ARGUMENT = 1,
    CAELIX_ERROR_UNSUPPORTED = 2,
    CAELIX_ERROR_CUDA = 3,
    CAELIX_ERROR_OUT_OF_MEMORY = 4,
    CAELIX_ERROR_DEVICE_STATUS = 5
} CaelixResult;

typedef enum CaelixLogLevel
{
    CAELIX_LOG_DEBUG = 0,
    CAELIX_LOG_INFO = 1,
    CAELIX_LOG_WARNING = 2,
    CAELIX_LOG_ERROR = 3
} CaelixLogLevel;

typedef void (*CaelixLogCallback)(CaelixLogLevel level, const char* message, void* user_data);
/* Replaces include/caelix/caelix.h:137-139. */
CAELIX_API void caelix_set_log_callback(CaelixLogCallback callback, void* user_data);

/* ---------------------------------------------------------------------------
 * Device
 * ------------------------------------------------------------------------- */

typedef struct CaelixDevice CaelixDevice;

typedef struct CaelixDeviceDesc
{
    int32_t cuda_device; /* CUDA device ordinal */
    uint32_t reserved;   /* must be 0 */
} CaelixDeviceDesc;

/* Replaces caelix_device_adopt (include/caelix/caelix.h:233): the library uses the host's CUDA
   device instead of adopting a VkDevice. Checks that the device is sm_100 (B200 class); another
   architecture returns CAELIX_ERROR_UNSUPPORTED. */
CAELIX_API CaelixResult caelix_device_create(const CaelixDeviceDesc* desc, CaelixDevice** out_device);
/* Replaces caelix_device_destroy (include/caelix/caelix.h:236). NULL is ignored. */
CAELIX_API void caelix_device_destroy(CaelixDevice* device);

/* Waits for the device to finish its work and reads (then clears) the status word that the
   asynchronous entry points without an object of their own (caelix_radix_sort_pairs) OR their
   device-side failures into. Replaces the host's wait on a safe frame followed by a readback
   (lib/src/light/light_tree_record.cpp:371-435). CAELIX_ERROR_DEVICE_STATUS when it was not 0;
   *out_status (may be NULL) receives the bits. */
CAELIX_API CaelixResult caelix_device_check(CaelixDevice* device, uint32_t* out_status);

/* ---------------------------------------------------------------------------
 * Light BVH: the build of one light tree over brick light records
 * ------------------------------------------------------------------------- */

/* A brick light record's header (lib/src/light/light_tree_layout.h:298-323), 48 bytes, 16-byte
   aligned in device memory. Face entries are not read by the build. */
typedef struct CaelixBrickLightRecord
{
    float face[6];        /* face sums +X, -X, +Y, -Y, +Z, -Z */
    uint32_t box_lo;      /* group-local voxel x | y << 10 | z << 20, inclusive */
    uint32_t box_hi;      /* exclusive */
    uint32_t pos;         /* group-local brick position */
    uint32_t entry_count;
    uint32_t counts_lo;
    uint32_t counts_hi;
} CaelixBrickLightRecord;

/* The frame of a render group (caelix_light_tree_layout.hlsl:409-433): the group's entity-local
   voxel origin and its entity's object-to-world rotation rows and translation. */
typedef struct CaelixGroupFrame
{
    float origin[3];
    float rotation[9]; /* row-major */
    float translation[3];
} CaelixGroupFrame;

/* One build's input (device pointers). Leaf i is record i (the reference's gather order,
   caelix_light_gather_emit.hlsl:66-85). record_group / record_entry: the (group, entry) words
   of each leaf; group_frames: group_count frames, one per group (a record whose group is not
   below group_count is emitted with the identity frame at origin 0 and sets a device status
   bit). All three NULL: group 0, entry i, identity frame at origin 0. */
typedef struct CaelixLightBvhInput
{
    const CaelixBrickLightRecord* records;
    uint32_t count;
    uint32_t group_count; /* frames in group_frames; 0 when it is NULL */
    const uint32_t* record_group;
    const uint32_t* record_entry;
    const CaelixGroupFrame* group_frames;
} CaelixLightBvhInput;

/* Device pointers of a built tree and of its build scratch (the kLtScratch* arrays of
   lib/src/light/light_tree_layout.h:392-423), for the trace kernels, tests and hosts. Valid
   until the next build or destroy of the object. */
typedef struct CaelixLightBvhView
{
    uint64_t leaves;      /* LightBvhLeaf[leaf_capacity], 64 bytes each */
    uint64_t nodes;       /* LightBvhNode[node_capacity], 224 bytes each */
    uint64_t header;      /* LightTreeHeader, 64 bytes, then LightTreeState, 64 bytes */
    uint64_t keys;        /* u32 sorted Morton codes */
    uint64_t values;      /* u32 sorted leaf indices */
    uint64_t left;        /* u32 binary node children */
    uint64_t right;
    uint64_t parent;      /* u32 binary node parents */
    uint64_t leaf_parent; /* u32 binary parent of each sorted leaf */
    uint64_t depth;       /* u32 binary node depths */
    uint64_t wide;        /* u32 4-wide index of each even-depth binary node */
    uint64_t aggregates;  /* LightSummary per binary node, in 64-byte slots (16 bytes of padding) */
    uint32_t leaf_capacity;
    uint32_t node_capacity;
} CaelixLightBvhView;

typedef struct CaelixLightBvh CaelixLightBvh;

/* Replaces the BVH part of LightTree (lib/src/light/light_tree.h:43-88; capacities and scratch,
   light_tree_layout.h:434-439): device buffers for up to leaf_capacity leaves. */
CAELIX_API CaelixResult caelix_light_bvh_create(CaelixDevice* device, uint32_t leaf_capacity,
                                                CaelixLightBvh** out_bvh);
CAELIX_API void caelix_light_bvh_destroy(CaelixLightBvh* bvh);

/* Replaces LightTree::RecordTree (lib/src/light/light_tree_record.cpp:230-309): records the
   gather emit and the build of one tree into `stream` (a cudaStream_t; asynchronous, nothing is
   read back). A count above the leaf capacity keeps the first leaf_capacity records and counts
   the rest as dropped, as the reference does. */
CAELIX_API CaelixResult caelix_light_bvh_build(CaelixLightBvh* bvh, const CaelixLightBvhInput* input,
                                               uint64_t stream);
CAELIX_API CaelixResult caelix_light_bvh_get_view(const CaelixLightBvh* bvh, CaelixLightBvhView* out);

/* The newest build's outcome, read back after synchronizing its stream (replaces the readback of
   LightTree::Recycle, lib/src/light/light_tree_record.cpp:371-435). */
typedef struct CaelixLightBvhStats
{
    uint32_t leaves;         /* header leaf_count */
    uint32_t nodes;          /* header node_count */
    uint32_t root;           /* 0, or 0xFFFFFFFF for an empty tree */
    uint32_t builds;
    uint32_t leaves_found;
    uint32_t leaves_dropped;
    uint32_t node_overflow;
    uint32_t status;         /* device status bits of the build (0 = none) */
    float bounds[6];         /* leaf centre bounds lo[3], hi[3] */
    float gpu_ms;            /* device time of the newest build (events around it) */
    uint32_t kernel_launches; /* kernels the newest build launched */
    float stage_ms[7];       /* with profiling on (caelix_light_bvh_set_profiling): device time of the
                                stages emit+bounds, morton+histograms, radix sort (4 passes and the
                                gather), karras, depth+scan, aggregation with the 4-wide nodes inside
                                tiles + aggregation of the nodes that cross tiles, 4-wide nodes over
                                those + finish; 0 otherwise */
    uint32_t pad;
} CaelixLightBvhStats;

/* Turns per-stage device timing of the following builds on (1) or off (0, the default): events
   between the stages, reported in CaelixLightBvhStats::stage_ms. Replaces the per-pass GpuTimer
   queries of the reference (lib/src/rhi/gpu_timer.h:9-82). */
CAELIX_API CaelixResult caelix_light_bvh_set_profiling(CaelixLightBvh* bvh, uint32_t enabled);

/* Synchronizes the stream of the newest build and fills *out. Returns CAELIX_ERROR_DEVICE_STATUS
   when the build's status word is not 0 (a bounded look-back gave up, a depth guard was hit, or the
   node capacity overflowed; *out is still filled). */
CAELIX_API CaelixResult caelix_light_bvh_get_stats(CaelixLightBvh* bvh, CaelixLightBvhStats* out);

/* ---------------------------------------------------------------------------
 * Radix sort
 * ------------------------------------------------------------------------- */

/* Replaces the radix sort kernels caelix_light_bvh_sort_histogram / caelix_light_bvh_scan /
   caelix_light_bvh_sort_scatter (shaders/light/bvh/caelix_light_bvh_sort.hlsl:13-36, bound by
   tests/light_tree_test.cpp:1460-1515): a stable sort of `count` (key, value) pairs by the 32-bit
   key, in place in `keys` / `values` (device pointers). `values` NULL is not allowed; with
   identity_values = 1 the input values are taken as 0 .. count-1 and not read. The device keeps
   one scratch buffer for the call, grown on demand. Asynchronous on `stream`; a device-side
   failure (a look-back that gave up) is reported by caelix_device_check. */
CAELIX_API CaelixResult caelix_radix_sort_pairs(CaelixDevice* device, uint32_t* keys, uint32_t* values,
                                                uint32_t count, uint32_t identity_values, uint64_t stream);

/* No counterpart in the reference: a failure-injection hook for tests of the bounded device waits
   (the reference's look-back has no bound; this library's waits give up and report instead of
   hanging). Runs the multi-tile sort of caelix_radix_sort_pairs (count > 4096) with tile
   `silent_tile` (1 .. tiles - 1, tiles of 4096 pairs) of the first pass never publishing its
   look-back status, and every look-back wait limited to `spin_limit` polls (1 .. 2^22): the tile
   after it gives up, sets the look-back timeout bit in the device status word and finishes with a
   wrong prefix (the output is not a valid sort). caelix_device_check then returns
   CAELIX_ERROR_DEVICE_STATUS with that bit; nothing traps or hangs, and the device stays usable. */
CAELIX_API CaelixResult caelix_radix_sort_pairs_wait_test(CaelixDevice* device, uint32_t* keys, uint32_t* values,
                                                          uint32_t count, uint32_t silent_tile, uint32_t spin_limit,
                                                          uint64_t stream);

/* No counterpart in the reference. The same sort for callers that cannot allocate device memory
   while they record work (an engine render thread that records a frame and must not stall it on
   an allocation, a host whose device memory budget is fixed up front): it allocates nothing. Its scratch is an array
   compiled into the library, about 2.4 MB reserved on every GPU that loads it until the process
   exits, so one call sorts at most 262144 pairs (more returns CAELIX_ERROR_INVALID_ARGUMENT).
   Runs on the current CUDA device. The first call on a device looks up the array's device address
   (cudaGetSymbolAddress); make that first call before any stream capture. Every call shares the
   array and clears what must start at zero; calls whose work overlaps on the GPU (other streams,
   other host threads) race on it and must be serialized by the caller. `status` (a device word,
   may be NULL) receives device-side failures OR-ed in (a look-back that gave up); with NULL such a
   failure is not reported anywhere. Asynchronous on `stream`. */
CAELIX_API CaelixResult caelix_radix_sort_pairs_static(uint32_t* keys, uint32_t* values, uint32_t count,
                                                       uint32_t identity_values, uint32_t* status, uint64_t stream);

/* ---------------------------------------------------------------------------
 * Scene: voxel bricks on the device
 *
 * Bricks are 8x8x8 blocks of 16-bit values, voxel index x + 8y + 64z, in one of the reference's
 * two block encodings (include/caelix/caelix.h:240-249):
 *   0 packed scene colour (the default): opaque when (value & 0xC000) != 0; transparent id =
 *     value & 0xFF, face bits at bits 8..13;
 *   1 block-ID: opaque when (value & 0x8000) != 0; transparent id = value & 0x1FF, face bits at
 *     bits 9..14.
 * A brick key is the brick coordinate, each axis in [-2^20, 2^20) as in the reference
 * (include/caelix/caelix.h:334). The device tables span the box of the keys (rounded to whole
 * render groups): a flush whose box holds more than 2^32 brick cells returns
 * CAELIX_ERROR_UNSUPPORTED (the occupancy bitmap is dense over the box).
 * Entity 0 is the scene's static world with the identity transform; caelix_scene_add_entity adds
 * entities 1, 2, ... with their own bricks (entity-local keys, the same range) under a rigid
 * transform. caelix_scene_flush builds, on the device: the brick records (the finalize rules of
 * the reference), the brick hash table, the brick occupancy bitmap, the brick light records and
 * the light tree of the world, and the same tables of every entity.
 * ------------------------------------------------------------------------- */

typedef struct CaelixScene CaelixScene;

/* Replaces CaelixSceneDesc (include/caelix/caelix.h:274-294): the same 32-byte layout. */
typedef struct CaelixSceneDesc
{
    uint64_t staging_bytes;    /* stored (bricks are staged in device memory, grown on demand);
                                  0 or >= 4 MiB */
    uint32_t records_per_page; /* 0 or a power of two; stored (records are dense per flush) */
    uint32_t group_shift;      /* render group edge in bricks = 1 << group_shift; 0 = 4; 1..4
                                  (5..8: CAELIX_ERROR_UNSUPPORTED) */
    uint32_t block_bytes;      /* 0 or 2 (4: CAELIX_ERROR_UNSUPPORTED) */
    uint32_t encoding;         /* 0 = packed scene colour (the default), 1 = block-ID; other values
                                  return CAELIX_ERROR_INVALID_ARGUMENT */
    uint64_t scratch_bytes;    /* stored (no acceleration structures: the build sizes its scratch) */
} CaelixSceneDesc;

/* Replaces caelix_scene_create / caelix_scene_destroy (include/caelix/caelix.h:296-300). */
CAELIX_API CaelixResult caelix_scene_create(CaelixDevice* device, const CaelixSceneDesc* desc,
                                            CaelixScene** out_scene);
CAELIX_API void caelix_scene_destroy(CaelixScene* scene);

/* Replaces the reference's entities (include/caelix/caelix.h:302-332). Entity ids are small
   indices; the id of a removed entity is reused by a later add. Entity 0 is the world: it is
   neither added, moved nor removed. */
typedef uint32_t CaelixEntityId;
#define CAELIX_INVALID_ENTITY 0xFFFFFFFFu

typedef struct CaelixEntityDesc
{
    uint8_t guid[16];  /* stored for the host; the library does not interpret it */
    float position[3]; /* world position of the entity origin */
    float rotation[4]; /* unit quaternion x, y, z, w (normalised by the library) */
} CaelixEntityDesc;

/* Adds an entity with no bricks: world = R(rotation) * local + position, local = the
   entity-local block coordinate. Its bricks are traced (closest hit over the world and every
   entity, ties to the world and then to the lower id) and shaded with the scene's materials. Its
   light voxels (the scene's light codes, in bricks with power above 0) are lights of one of the two
   light trees, as in the reference (docs/LIGHT_TREE.md:136-176): a static entity's (the default
   motion) join the world's in tree 0, a dynamic entity's the second tree, each tree's records
   merged in id order under the entities' transforms and rebuilt at a flush after any change of
   its lights or a move; NEE picks between the two trees by importance. Takes effect at the next
   flush. */
CAELIX_API CaelixResult caelix_scene_add_entity(CaelixScene* scene, const CaelixEntityDesc* desc,
                                                CaelixEntityId* out_id);
/* Removes the entity and all its bricks at once (waiting for the device first). */
CAELIX_API CaelixResult caelix_scene_remove_entity(CaelixScene* scene, CaelixEntityId entity);
/* Moves an entity; takes effect at the next flush. The rotation rows are computed in double from
   the normalised quaternion and rounded to float. */
CAELIX_API CaelixResult caelix_scene_set_entity_transform(CaelixScene* scene, CaelixEntityId entity,
                                                          const float position[3], const float rotation[4]);
/* Entity motion (include/caelix/caelix.h:322-332): it picks the light tree of the entity's lights,
   tree 0 for CAELIX_ENTITY_STATIC (a new entity's), the dynamic tree for CAELIX_ENTITY_DYNAMIC;
   takes effect at the next flush. Other values return CAELIX_ERROR_INVALID_ARGUMENT. */
#define CAELIX_ENTITY_STATIC 0u
#define CAELIX_ENTITY_DYNAMIC 1u
CAELIX_API CaelixResult caelix_scene_set_entity_motion(CaelixScene* scene, CaelixEntityId entity, uint32_t motion);

typedef struct CaelixBrickKey
{
    int32_t x, y, z;
} CaelixBrickKey;

/* Replaces caelix_scene_upload_bricks (include/caelix/caelix.h:340-352): count raw bricks of 512
   uint16_t values each (host memory, borrowed for the call); a brick with the same key is
   replaced. entity: 0 (the world) or an added entity. Every key is checked first: one out of range returns
   CAELIX_ERROR_INVALID_ARGUMENT and accepts nothing. *consumed (may be NULL) = count. */
CAELIX_API CaelixResult caelix_scene_upload_bricks(CaelixScene* scene, uint32_t entity, uint32_t count,
                                                   const CaelixBrickKey* keys, const void* blocks,
                                                   uint32_t* consumed);

/* Replaces caelix_scene_remove_bricks (include/caelix/caelix.h:353-356): removes the bricks of the
   given keys (host memory, borrowed for the call); keys the scene does not have, including keys
   outside the range an upload accepts, are ignored, and a key repeated in the call is removed
   once. entity: 0 (the world) or an added entity. The next flush rebuilds that entity's tables from the remaining bricks
   (their groups, and a group's light block, go with their last brick). A removed brick's power
   goes with it: a later upload of the same key starts with power 0 unless the host sets it. */
CAELIX_API CaelixResult caelix_scene_remove_bricks(CaelixScene* scene, uint32_t entity, uint32_t count,
                                                   const CaelixBrickKey* keys);

/* New (no reference counterpart): the emitter power of bricks (host arrays), a factor of the
   emission of every voxel of the brick: a voxel emits its material's emission times its brick's
   power, and a light voxel (its code in the light code set, see caelix_scene_set_light_options)
   of a brick with power 0 is no light. Every brick's power is 1 until set, so a host that never
   calls this gets the reference's emission (include/caelix/caelix.h:600-630). The benchmark
   scenes give each emissive brick its own power. Keys without an uploaded brick are kept and
   apply when it arrives; a removed brick's power goes with it. power >= 0 and finite. entity: 0
   (the world's lights) or an added entity (the entities' light tree). */
CAELIX_API CaelixResult caelix_scene_set_brick_power(CaelixScene* scene, uint32_t entity, uint32_t count,
                                                     const CaelixBrickKey* keys, const float* power);

/* Replaces CaelixMaterial (include/caelix/caelix.h:529-556): the same 112-byte entry. Every scene
   has a table of 65536 entries, one per 16-bit block code; a transparent code is looked up without
   its face bits (include/caelix/caelix.h:478-515). This version shades every hit voxel with a
   Lambertian lobe of `albedo` and its `emission` (times its brick's power, fp32 on the device);
   the other fields are validated and stored. Built-in content, as in the reference:
     packed: an opaque code with bit 15 is albedo rgb5 / 31 (r = bits 14..10, g = 9..5, b = 4..0);
       an emissive code (bits 15..14 = 01) is albedo rgb4 / 15 (r = bits 13..10, g = 9..6,
       b = 5..2) and emission albedo * 2^(3 * (code & 3)); a transparent code is albedo 1, no
       emission (the glass palette's tints are not carried: glass is not traced here);
     block-ID: an opaque code is a pastel hash colour of code & 0x7FFF, a transparent id 1..511 a
       pastel hash colour of the id, air albedo 1; no emission.
   Transparent voxels with face bits are hit like opaque ones (no refraction). */
typedef struct CaelixMaterial
{
    float albedo[3];
    float smoothness;
    float emission[3];
    float metallic;
    float ior;
    float extinction;
    uint32_t sss_model;
    float sss_probability;
    float sss_albedo[3];
    float sss_anisotropy;
    uint32_t sss_steps;
    float sss_params[8];
    uint32_t texture_set;
    uint32_t connect_group;
    uint32_t reserved;
} CaelixMaterial;

/* Replaces caelix_scene_set_materials (include/caelix/caelix.h:558-568): entries [0, count) become
   the table entries of codes [0, count), codes [count, 65536) get the built-in default of the
   scene's encoding. count <= 65536 (0 restores the default table). The reference's value checks:
   every float finite with a magnitude <= 65504, ior > 0, extinction >= 0, sss_model <= 255,
   sss_probability and every sss_albedo in [0, 1], sss_anisotropy in [-1, 1], sss_steps <= 255,
   texture_set and connect_group <= 0xFFFF; an invalid entry returns CAELIX_ERROR_INVALID_ARGUMENT
   and changes nothing. Takes effect at the next flush (a change of the light code set rebuilds the
   scene's records there). */
CAELIX_API CaelixResult caelix_scene_set_materials(CaelixScene* scene, const CaelixMaterial* entries,
                                                   uint32_t count);

/* Replaces CaelixMaterialEntry (include/caelix/caelix.h:576-581): 116 bytes. */
typedef struct CaelixMaterialEntry
{
    uint32_t code; /* 0 .. 0xFFFF */
    CaelixMaterial material;
} CaelixMaterialEntry;

/* Replaces caelix_scene_set_material_entries (include/caelix/caelix.h:583-592): writes
   entries[i].material at code entries[i].code over the current table; one bad code or entry
   returns CAELIX_ERROR_INVALID_ARGUMENT and changes nothing; count 0 is a no-op. */
CAELIX_API CaelixResult caelix_scene_set_material_entries(CaelixScene* scene, const CaelixMaterialEntry* entries,
                                                          uint32_t count);

/* Replaces caelix_scene_get_material (include/caelix/caelix.h:593-597): the current entry of a raw
   block code (face bits of a transparent code removed first), the host copy. */
CAELIX_API CaelixResult caelix_scene_get_material(const CaelixScene* scene, uint32_t code, CaelixMaterial* out);

/* Replaces CaelixLightOptions / caelix_scene_set_light_options (include/caelix/caelix.h:632-646).
   A light voxel is a voxel whose material emission luminance, 0.2126 r + 0.7152 g + 0.0722 b, is at
   least min_emission, in a brick with power above 0 (caelix_scene_set_brick_power). Invalid values
   (enabled not 0 or 1, min_emission negative or not finite, heap_bytes above 2^32 x 16) return
   CAELIX_ERROR_INVALID_ARGUMENT and change nothing. Takes effect at the next flush: enabling or
   disabling the tree, or a change of the light code set, rebuilds the scene's tables; any other
   change rebuilds the light tree alone. With the tree disabled the voxels still emit (their
   emission is seen by the paths that hit them); there is no light-tree NEE. */
typedef struct CaelixLightOptions
{
    uint32_t enabled;    /* 0 = no light tree (the default), 1 = build it */
    float min_emission;  /* light voxel threshold (luminance of the material emission); 0 = 20 */
    uint64_t heap_bytes; /* stored; the heap is sized exactly at every flush */
} CaelixLightOptions;
CAELIX_API CaelixResult caelix_scene_set_light_options(CaelixScene* scene, const CaelixLightOptions* options);

/* Replaces CaelixFrameDesc (include/caelix/caelix.h:358-364): command_buffer is a cudaStream_t. */
typedef struct CaelixFrameDesc
{
    uint64_t command_buffer;
    uint64_t frame_number;      /* strictly increasing across flushes, > safe_frame_number */
    uint64_t safe_frame_number;
} CaelixFrameDesc;

/* Replaces caelix_scene_flush (include/caelix/caelix.h:379; lib/src/scene/scene_flush.cpp:567):
   builds the device scene from everything uploaded so far when it changed (records, hash table,
   bitmap, light records, light tree) on the frame's stream and waits for it (the build reads
   back its sizes). The frame contract is checked as in the reference. */
CAELIX_API CaelixResult caelix_scene_flush(CaelixScene* scene, const CaelixFrameDesc* desc);

/* Replaces CaelixLightStats (include/caelix/caelix.h:650-677, 104 bytes); tree index 1 (dynamic
   entities) stays 0 in this version. */
typedef struct CaelixLightStats
{
    uint32_t enabled;
    uint32_t light_groups;
    uint64_t light_bricks;
    uint64_t light_faces;
    uint64_t bricks_dropped;
    uint64_t heap_bytes_used;
    uint64_t heap_bytes_capacity;
    uint32_t passes;
    uint32_t failed_passes;
    uint32_t records_recomputed;
    uint32_t records_copied;
    float gpu_ms;
    uint32_t pad;
    uint32_t tree_leaves[2];
    uint32_t tree_nodes[2];
    uint32_t tree_builds[2];
    uint32_t tree_leaves_dropped[2];
} CaelixLightStats;
/* Replaces caelix_scene_get_light_stats (include/caelix/caelix.h:681). NULL arguments are ignored. */
CAELIX_API void caelix_scene_get_light_stats(const CaelixScene* scene, CaelixLightStats* out);

/* Device pointers and sizes of the built scene, for tests and hosts (replaces the descriptor of
   caelix_scene_get_light_tree, include/caelix/caelix.h:688, and the scene tables the reference's
   tests read back). Valid until the next flush that rebuilds or the scene's destruction. */
typedef struct CaelixSceneView
{
    uint32_t grid[3];       /* brick cells of the box per axis from `origin` */
    uint32_t group_shift;
    uint32_t groups[3];
    uint32_t brick_count;
    uint32_t hash_capacity;
    uint32_t hash_slot_count;
    uint32_t hash_max_probe;
    uint32_t light_count;
    uint32_t heap_words;
    uint32_t group_count;
    uint64_t keys;          /* int32 [brick_count][3], increasing linear brick index */
    uint64_t records;       /* u32 [brick_count][274] */
    uint64_t hash_slots;    /* u32 [hash_slot_count][4]: key_lo, key_hi, record, 0 */
    uint64_t bitmap;        /* u32 brick occupancy by linear brick index */
    uint64_t heap;          /* u32 group light blocks */
    uint64_t group_rows;    /* u32 [group_count][8]: GroupLightRow (block offset, block units,
                               generation = life << 16 | version, 0, 0, light bricks, light faces, 0) */
    uint64_t light_headers; /* CaelixBrickLightRecord [light_count], leaf order */
    uint64_t light_group;   /* u32 [light_count] */
    uint64_t light_entry;   /* u32 [light_count] */
    uint64_t light_brick;   /* u32 [light_count] */
    uint64_t tree_header;   /* LightTreeHeader + LightTreeState */
    uint64_t tree_nodes;
    uint64_t tree_leaves;
    int32_t origin[3];      /* brick key of cell 0 of the box (a multiple of the group edge) */
    uint32_t encoding;
} CaelixSceneView;
CAELIX_API CaelixResult caelix_scene_get_view(const CaelixScene* scene, CaelixSceneView* out);

/* Replaces caelix_scene_get_light_tree (include/caelix/caelix.h:688): the device address of the
   light tree header (LightTreeHeader, then LightTreeState); 0 without a tree. */
CAELIX_API uint64_t caelix_scene_get_light_tree(const CaelixScene* scene);

/* ---------------------------------------------------------------------------
 * Renderer: path-traces a scene into a headless device radiance buffer
 * ------------------------------------------------------------------------- */

typedef struct CaelixRenderer CaelixRenderer;

/* Replaces caelix_renderer_create / destroy (include/caelix/caelix.h:800-805). */
CAELIX_API CaelixResult caelix_renderer_create(CaelixDevice* device, CaelixScene* scene,
                                               CaelixRenderer** out_renderer);
CAELIX_API void caelix_renderer_destroy(CaelixRenderer* renderer);

/* Replaces CaelixCamera (include/caelix/caelix.h:814-844), the same layout and pinhole mapping
   (common/caelix_frame.hlsl:164-171); jitter must be 0 in this version, projection is unused. */
typedef struct CaelixCamera
{
    float position[3];
    float pad0;
    float right[3];
    float pad1;
    float up[3];
    float pad2;
    float forward[3];
    float pad3;
    float tan_half_fov_y;
    float aspect;
    float near_z, far_z;
    float projection[16];
    float jitter[2];
} CaelixCamera;

/* Replaces CaelixRenderTargets (include/caelix/caelix.h:1130-1200): one headless target, the fp32
   RGB radiance of every pixel (row 0 = the top row), deterministic + albedo * stochastic as the
   reference's composite forms it (shaders/render/caelix_composite.hlsl:7). */
typedef struct CaelixRenderTargets
{
    uint64_t radiance; /* device float[height][width][3] */
    uint32_t width;
    uint32_t height;
    /* Optional (0 = none; the reference's voxel id target, include/caelix/caelix.h:1176-1190,
       R32G32_UINT): device uint32[height][width][2], two independent hashes of (entity id,
       entity-local integer voxel position) of the camera ray's first hit
       (shaders/render/caelix_scene_trace.hlsl:171-200): every pixel of one voxel shares the key; a
       miss, and a hit farther than CaelixRenderOptions::voxel_id_tmax, are 0xFFFFFFFF in both
       words. Written once per render call, from the camera ray of the first sample. */
    uint64_t voxel_id;
} CaelixRenderTargets;

/* Replaces CaelixRenderOptions (include/caelix/caelix.h:1043-1126): the fields of the path-traced
   mode that this version implements, under the reference's names. */
typedef struct CaelixRenderOptions
{
    uint32_t mode;         /* 1 = CAELIX_MODE_PATH_TRACE (the only mode of this version) */
    uint32_t bounce_count; /* stochastic bounces after the primary hit, 0 .. 14 */
    uint32_t frame_seed;   /* per-pixel random streams depend on the pixel and this value only */
    uint32_t spp;          /* new: samples per pixel (frame seeds frame_seed .. + spp - 1, averaged); 0 = 1 */
    float voxel_id_tmax;   /* the voxel id target: hits farther than this along the camera ray are
                              misses; 0 = no limit. Finite and >= 0. */
    uint32_t reserved[3];  /* must be 0 */
} CaelixRenderOptions;

/* Replaces caelix_renderer_render (include/caelix/caelix.h:1257): records the trace of one frame
   into the frame's stream (asynchronous). */
CAELIX_API CaelixResult caelix_renderer_render(CaelixRenderer* renderer, const CaelixFrameDesc* frame,
                                               const CaelixRenderTargets* targets, const CaelixCamera* camera,
                                               const CaelixRenderOptions* options);

/* New (no reference counterpart; the reference traces with ray queries inside one compute
   shader): the kernel organisation of caelix_renderer_render. Both give the same radiance, bit
   for bit.
     CAELIX_TRACE_WAVEFRONT (default): path state in device memory, one kernel per stage (trace,
       shade) over compacted ray and path queues, every bounce; wave_capacity bounds the paths in
       flight (0 = one per pixel; else at least 32), the rest of the pixels follow in later waves.
     CAELIX_TRACE_MEGAKERNEL: one thread per pixel runs its whole path in one kernel. */
#define CAELIX_TRACE_WAVEFRONT 0u
#define CAELIX_TRACE_MEGAKERNEL 1u
CAELIX_API CaelixResult caelix_renderer_set_trace_mode(CaelixRenderer* renderer, uint32_t mode,
                                                       uint32_t wave_capacity);

/* Replaces CaelixLightNeeOptions / caelix_renderer_set_light_nee_options
   (include/caelix/caelix.h:1283-1297). flags must be 0 (MIS on, no visibility hint). */
typedef struct CaelixLightNeeOptions
{
    uint32_t enabled;
    uint32_t flags;
    uint32_t hint_patch;
    uint32_t reserved;
} CaelixLightNeeOptions;
CAELIX_API CaelixResult caelix_renderer_set_light_nee_options(CaelixRenderer* renderer,
                                                              const CaelixLightNeeOptions* options);

/* Replaces CaelixGpuTimings / caelix_renderer_get_gpu_timings (include/caelix/caelix.h:1324-1339):
   events around the newest render and flush, read after waiting for them. */
typedef struct CaelixGpuTimings
{
    float trace_ms;
    float flush_ms;
    uint64_t frame_number;
    float composite_ms;
    float denoise_ms;
    float upscale_ms;
    float pad;
} CaelixGpuTimings;
CAELIX_API void caelix_renderer_get_gpu_timings(const CaelixRenderer* renderer, CaelixGpuTimings* out);

/* New: rays traced by the newest render call, by kind (read after waiting for it). */
typedef struct CaelixRenderStats
{
    uint64_t primary_rays;
    uint64_t bounce_rays;
    uint64_t shadow_rays;
    uint32_t kernel_launches;
    uint32_t pad;
} CaelixRenderStats;
CAELIX_API CaelixResult caelix_renderer_get_stats(CaelixRenderer* renderer, CaelixRenderStats* out);

/* New (no reference counterpart): the adjoint of caelix_renderer_render for an image loss L.
   d_radiance: device float[height][width][3], dL/d(radiance) of the frame the same renderer,
   target size, camera and options render. Writes (after zeroing them) the gradients of L with
   respect to the albedo of every material table entry, d_albedo: device float[65536][3] (row =
   the material code), and to the emitter power of every brick, d_power: device float[brick_count] in
   the scene's brick order (the keys of caelix_scene_get_view: increasing linear brick index).
   A scene's entities are traced and shaded as in the render (their voxels' albedo gradients go to
   the shared material table); the power of their bricks is not differentiated. Sampling quantities (pdfs, MIS weights, Russian-roulette probabilities, discrete decisions) are
   held fixed. The frame is traced twice (path replay): once recording each sample's radiance (one
   image per sample index, in device memory the renderer keeps), once more gathering the
   gradients; nothing of the paths is stored. When
   targets->radiance is not 0 it also receives the forward radiance (bit-identical to
   caelix_renderer_render). Asynchronous on frame->command_buffer; rays and timings through
   caelix_renderer_get_stats / caelix_renderer_get_gpu_timings. */
CAELIX_API CaelixResult caelix_renderer_backward(CaelixRenderer* renderer, const CaelixFrameDesc* frame,
                                                 const CaelixRenderTargets* targets, const CaelixCamera* camera,
                                                 const CaelixRenderOptions* options, const float* d_radiance,
                                                 float* d_albedo, float* d_power);

/* ---------------------------------------------------------------------------
 * Batch: many scenes and viewports in one CUDA graph launch
 *
 * No counterpart in the reference (it renders one scene per renderer call). A batch holds up to
 * 256 views (a renderer, hence its scene and NEE options, plus a camera, a target and render
 * options each). One run is one CUDA graph launch: the light tree of every distinct scene is
 * rebuilt (as caelix_scene_flush does after caelix_scene_set_light_options), the builds of
 * different scenes running as parallel branches, then every view is traced, either by one
 * persistent kernel whose resident threads take pixels of all views from one work counter, or by
 * the wavefront kernels over the paths of all views at once (CaelixBatchTuning::kernel; a batch
 * with a scene that has entities always runs the wavefront kernels, which trace them, and its runs
 * also rebuild the entities' light tree). Each view's radiance is bit-identical to
 * caelix_renderer_render of the same renderer, target, camera and options.
 *
 * The scenes must be flushed before the batch is created. A full re-flush of a scene (bricks,
 * powers or materials changed) moves its device tables: the next run notices it and captures
 * the graph again. Calls on a batch and on its scenes and renderers are externally synchronized.
 * ------------------------------------------------------------------------- */

typedef struct CaelixBatch CaelixBatch;

typedef struct CaelixBatchView
{
    CaelixRenderer* renderer;
    CaelixCamera camera;
    CaelixRenderTargets target;
    CaelixRenderOptions options;
} CaelixBatchView;

typedef struct CaelixBatchDesc
{
    uint32_t view_count; /* 1 .. 256 */
    uint32_t rebuild_light_trees; /* 1: every run rebuilds the light trees first; 0: trace only */
    const CaelixBatchView* views; /* copied */
    uint32_t reserved[4]; /* must be 0 */
} CaelixBatchDesc;

/* The launch parameters of a run, chosen by caelix_batch_autotune or set by hand. */
typedef struct CaelixBatchTuning
{
    uint32_t min_blocks;           /* persistent kernel: its register cap, 4, 6 or 8 CTAs of 128
                                      threads resident per SM (128, 80 or 64 registers) */
    uint32_t wavefront;            /* paths in flight. Persistent kernel: its threads, rounded down
                                      to whole CTAs, 0 = every resident thread. Wavefront kernels:
                                      the slots of one sub-wave (at least 32), 0 = 4M */
    uint32_t block_width;          /* pixel block of 32 consecutive work items: 8 (8x4), 16 (16x2)
                                      or 32 (32x1) */
    uint32_t refill_min;           /* persistent kernel: a warp takes new pixels once this many of its
                                      lanes are idle, 1..32 */
    uint32_t sort_keys_per_thread; /* the light-tree radix sort's tile: 256 x 4, 8 or 16 keys */
    uint32_t order;                /* 0 = views in the given order, 1 = the most pixel samples first */
    uint32_t kernel;               /* CAELIX_BATCH_PERSISTENT: one persistent launch traces every
                                      view; CAELIX_BATCH_WAVEFRONT: the wavefront kernels of
                                      caelix_renderer_set_trace_mode over the paths of every view */
    uint32_t reserved;             /* must be 0 */
} CaelixBatchTuning;
#define CAELIX_BATCH_PERSISTENT 0u
#define CAELIX_BATCH_WAVEFRONT 1u

/* Creates a batch (device buffers, no GPU work). Fails with INVALID_ARGUMENT on a bad view (NULL
   renderer, scene not flushed, target not a device buffer of the right size, options as
   caelix_renderer_render rejects them). */
CAELIX_API CaelixResult caelix_batch_create(CaelixDevice* device, const CaelixBatchDesc* desc,
                                            CaelixBatch** out_batch);
CAELIX_API void caelix_batch_destroy(CaelixBatch* batch);

/* Launches one run on frame->command_buffer (asynchronous). The first run, and the first after a
   change of tuning or a scene re-flush, captures the graph first (waiting for the previous run).
   Runs of one batch share its device buffers: two runs must not overlap (same stream, or the
   host waits in between). */
CAELIX_API CaelixResult caelix_batch_run(CaelixBatch* batch, const CaelixFrameDesc* frame);

CAELIX_API CaelixResult caelix_batch_set_tuning(CaelixBatch* batch, const CaelixBatchTuning* tuning);
CAELIX_API CaelixResult caelix_batch_get_tuning(const CaelixBatch* batch, CaelixBatchTuning* out);

/* Picks the tuning of this batch on this GPU. With a cache file (JSON, NULL = none) whose entry
   for this GPU and workload exists, takes it without running anything; else times candidate
   tunings on frame->command_buffer (coordinate descent: the sort tile on the light-tree builds
   alone, then the trace parameters on the trace alone, each candidate timed by CUDA events over
   `repeats` runs after one warm-up run; 0 = 2), applies the best and, with a cache file, stores
   it there. The kernel organisation is a coordinate too (each with its own parameters).
   Synchronous. */
CAELIX_API CaelixResult caelix_batch_autotune(CaelixBatch* batch, const CaelixFrameDesc* frame,
                                              const char* cache_path, uint32_t repeats,
                                              CaelixBatchTuning* out);

/* Rays and GPU time of the newest run (read after waiting for it); the status words of the run's
   builds and trace are checked (CAELIX_ERROR_DEVICE_STATUS on a device-side failure). */
typedef struct CaelixBatchStats
{
    uint64_t primary_rays;
    uint64_t bounce_rays;
    uint64_t shadow_rays;
    float gpu_ms;             /* the whole graph launch */
    uint32_t kernel_launches; /* kernel nodes of the graph */
    uint32_t light_tree_builds;
    uint32_t wavefront;       /* persistent threads of the trace */
    uint32_t graph_captures;  /* captures so far */
    uint32_t pad;
} CaelixBatchStats;
CAELIX_API CaelixResult caelix_batch_get_stats(CaelixBatch* batch, CaelixBatchStats* out);
/* Rays of one view in the newest run (kernel_launches = 1: the shared persistent launch). */
CAELIX_API CaelixResult caelix_batch_get_view_stats(CaelixBatch* batch, uint32_t view, CaelixRenderStats* out);

/* ---------------------------------------------------------------------------
   World files (.cxw, format version 8 and older). Replaces the reference's reader crate
   (host-rs/caelix-cxw/src/lib.rs: CxwFile::open :207-229, decode :243-248, decode_all :250-259,
   the read rules of parse_index :339-452, region :455-493 and decode_payload :544-630) and the
   world loader of its host (host-rs/caelix-app/src/world.rs, WorldLoader::open :93-170 and
   upload :206-262), for the static world entity of this library's scenes.

   Errors: a file that breaks a read rule returns CAELIX_ERROR_INVALID_ARGUMENT (a newer format
   version: CAELIX_ERROR_UNSUPPORTED) and logs the reason in the words of the reference's error
   (bad magic, truncated data at an offset, region size, duplicate sector, brick map counters,
   inflate failure, payload structure). */
typedef struct CaelixWorldFile CaelixWorldFile;

typedef struct CaelixWorldInfo
{
    uint16_t version;
    uint16_t has_player_pose; /* version 7+ world record with the pose flag */
    uint32_t entity_count;
    uint64_t sector_count;    /* all entities */
    float player_position[3];
    float player_rotation[4]; /* quaternion x, y, z, w */
} CaelixWorldInfo;

/* One entity record after the reader's version migrations (flags bit 0 HasBody, bit 1 Static;
   before version 6 from the legacy body state; velocity zero before version 4). */
typedef struct CaelixWorldEntity
{
    uint8_t guid[16];
    float position[3];
    float rotation[4];
    float velocity[6]; /* linear xyz, angular xyz */
    uint16_t require_update_flags;
    uint8_t flags;
    uint8_t is_protected;
    uint32_t sector_count;
} CaelixWorldEntity;

typedef struct CaelixWorldSector
{
    uint32_t entity;
    int32_t coord[3];
    uint64_t region_offset;
    uint32_t region_size;
    uint32_t pad;
} CaelixWorldSector;

/* Reads the header, the world record, the entity table and every sector index, and checks every
   region (CxwFile::open). The file is read into host memory; *out is owned by the caller. */
CAELIX_API CaelixResult caelix_world_open(const char* path, CaelixWorldFile** out);
CAELIX_API void caelix_world_close(CaelixWorldFile* file);
CAELIX_API CaelixResult caelix_world_get_info(const CaelixWorldFile* file, CaelixWorldInfo* out);
CAELIX_API CaelixResult caelix_world_get_entity(const CaelixWorldFile* file, uint32_t index,
                                                CaelixWorldEntity* out);
/* Sectors in entity order, then sector index order. */
CAELIX_API CaelixResult caelix_world_get_sector(const CaelixWorldFile* file, uint64_t index,
                                                CaelixWorldSector* out);
/* Inflates and decodes one sector: its non-air bricks in ascending brick index (a brick whose 512
   values are all 0 is dropped), entity-local keys (sector coord * 16 + brick in sector), the raw
   values (voxel x + 8y + 64z), the preview word of each kept brick, and the count of non-zero
   values. With keys == NULL only *brick_count (and *voxels) are written; otherwise the arrays
   hold `capacity` bricks (fewer: CAELIX_ERROR_INVALID_ARGUMENT). */
CAELIX_API CaelixResult caelix_world_decode_sector(const CaelixWorldFile* file, uint64_t index, uint32_t capacity,
                                                   CaelixBrickKey* keys, uint16_t* blocks, uint32_t* summaries,
                                                   uint32_t* brick_count, uint64_t* voxels);
/* Decodes every sector of one entity on `threads` host threads (0 = all) and uploads its bricks
   to the scene (caelix_scene_upload_bricks) with the file's keys unchanged, as the reference's
   loader passes the decoder's keys through (host-rs/caelix-app/src/world.rs:212-247); `origin`
   (may be NULL) receives the move applied to the keys, which is 0. A key outside [-2^20, 2^20):
   the upload's CAELIX_ERROR_INVALID_ARGUMENT. *bricks (may be NULL) = bricks uploaded. */
CAELIX_API CaelixResult caelix_world_upload_entity(const CaelixWorldFile* file, uint32_t entity, CaelixScene* scene,
                                                   uint32_t threads, int32_t origin[3], uint64_t* bricks);
/* Loads every entity of the file, as the reference's WorldLoader::open + upload
   (host-rs/caelix-app/src/world.rs:93-262): file entity 0 into the scene's world (as
   caelix_world_upload_entity), every other entity as a scene entity (caelix_scene_add_entity,
   motion from its Static flag) with its transform expressed in the world's frame:
   x_scene = R0^T (x_file - p0), so the added entity has rotation conj(q0) qi and position
   R0^T (pi - p0) (computed in double, rounded to float).
   ids (may be NULL) receives the scene entity of every file entity (0 for the world). A failure
   removes the entities added (the world's bricks uploaded before it stay). *bricks (may be NULL)
   = bricks uploaded. */
CAELIX_API CaelixResult caelix_world_load(const CaelixWorldFile* file, CaelixScene* scene, uint32_t threads,
                                          uint32_t* ids, uint64_t* bricks);

#ifdef __cplusplus
}
#endif
#endif /* CAELIX_B200_H */
