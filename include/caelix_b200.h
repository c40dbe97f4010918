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
                                stages emit+bounds, morton+histograms, radix sort (4 passes), karras,
                                aggregate, depth+scan, wide+finish; 0 otherwise */
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

#ifdef __cplusplus
}
#endif
#endif /* CAELIX_B200_H */
