// Device data layouts of the light tree and the brick records, shared by the host code and the
// CUDA kernels of libcaelix_b200.
//
// The byte layouts are the reference's, so that a host which reads the light tree (its tests, the
// Unity bridge, a debugger) sees the same bytes: the structs restate
// lib/src/light/light_tree_layout.h (LightSummary :89-102, LightTreeHeader :105-121,
// BrickLightRecordHeader :298-323, LightBvhLeaf :338-354, LightBvhNode :359-389) and the brick
// record of shaders/common/caelix_record.hlsl:14-28. The static_asserts pin every offset.
#pragma once
#include <cstddef>
#include <cstdint>

// Returns the first failing CUDA call's error from a host function returning cudaError_t.
#define CX_TRY(x)                         \
    do {                                  \
        const cudaError_t e_ = (x);       \
        if (e_ != cudaSuccess) return e_; \
    } while (0)

namespace cx {

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr uint32_t kChildLeafBit = 0x80000000u;
constexpr uint32_t kParentSlotBits = 2;
constexpr uint32_t kParentSlotMask = 3u;
constexpr uint32_t kNodeSlots = 4;

// Face sums (+X, -X, +Y, -Y, +Z, -Z) and a box.
struct alignas(16) LightSummary
{
    float face[6];
    float lo[3];
    float hi[3];
};
static_assert(offsetof(LightSummary, lo) == 24 && offsetof(LightSummary, hi) == 36);
static_assert(sizeof(LightSummary) == 48);

struct alignas(16) LightTreeHeader
{
    LightSummary summary;
    uint32_t root;  // kNone = empty tree
    uint32_t leaf_count;
    uint32_t node_count;
    uint32_t pad;
};
static_assert(offsetof(LightTreeHeader, root) == 48 && offsetof(LightTreeHeader, node_count) == 56);
static_assert(sizeof(LightTreeHeader) == 64);

// The header of a brick light record; uint32_t face entries follow (face family 0 .. 5, each
// sorted by voxel index; entry = voxel index | raw block value << 16).
struct alignas(16) BrickLightRecord
{
    float face[6];
    uint32_t box_lo;  // packed group-local voxel x | y << 10 | z << 20, inclusive
    uint32_t box_hi;  // exclusive
    uint32_t pos;     // group-local brick position
    uint32_t entry_count;
    uint32_t counts_lo;  // family counts of +X, -X, +Y (10 bits each)
    uint32_t counts_hi;  // family counts of -Y, +Z, -Z
};
static_assert(offsetof(BrickLightRecord, box_lo) == 24 && offsetof(BrickLightRecord, pos) == 32);
static_assert(offsetof(BrickLightRecord, counts_hi) == 44 && sizeof(BrickLightRecord) == 48);
constexpr uint32_t kVoxelBits = 10;
constexpr uint32_t kVoxelMask = 0x3FFu;
constexpr uint32_t kFamilyCountBits = 10;
constexpr uint32_t kFamilyCountMask = 0x3FFu;
constexpr uint32_t kFaceEntryVoxelMask = 0x1FFu;
constexpr uint32_t kFaceEntryBlockShift = 16;

struct alignas(16) LightBvhLeaf
{
    LightSummary summary;  // world face sums and world AABB
    uint32_t group;
    uint32_t entry;
    uint32_t pad;
    uint32_t parent;  // node << kParentSlotBits | slot
};
static_assert(offsetof(LightBvhLeaf, group) == 48 && offsetof(LightBvhLeaf, parent) == 60);
static_assert(sizeof(LightBvhLeaf) == 64);

// 4-wide node, child summaries inline, slots filled from 0.
struct alignas(16) LightBvhNode
{
    float child_face[4][6];
    float child_lo[4][3];
    float child_hi[4][3];
    uint32_t child[4];  // kChildLeafBit | leaf index, else node index; kNone = empty slot
    uint32_t parent;    // kNone = root
    uint32_t parent_slot;
    uint32_t pad[2];
};
static_assert(offsetof(LightBvhNode, child_lo) == 96 && offsetof(LightBvhNode, child_hi) == 144);
static_assert(offsetof(LightBvhNode, child) == 192 && offsetof(LightBvhNode, parent) == 208);
static_assert(offsetof(LightBvhNode, parent_slot) == 212 && sizeof(LightBvhNode) == 224);

// The frame that moves a record's group-local box to world space: the group's voxel origin and
// its entity's object-to-world rotation rows and translation.
struct GroupFrame
{
    float origin[3];
    float rot[9];
    float trans[3];
};
static_assert(sizeof(GroupFrame) == 60);

// Brick record (16-bit blocks): 274 words, caelix_record.hlsl:14-28.
//   word 0      bits 0..15 group-local brick position, bits 16..23 coarse occupancy (2x2x2)
//   word 1      tight bounds minX | minY<<3 | minZ<<6 | maxX<<9 | maxY<<12 | maxZ<<15 (inclusive)
//   words 2..17 micro occupancy: coarse cell c owns words 2+2c, 3+2c; bit (micro & 31) with
//               micro = (x&3) | (y&3)<<2 | (z&3)<<4 in word 2 + 2c + (micro >> 5)
//   words 18..  payload, block (x, y, z) in word 18 + (x>>1) + 4y + 32z, even x in the low half
constexpr uint32_t kRecordWords = 274;
constexpr uint32_t kRecordBytes = kRecordWords * 4;
constexpr uint32_t kRecordPayloadWord = 18;
constexpr uint32_t kBrickEdge = 8;
constexpr uint32_t kBrickVoxels = 512;

// Block encodings (CaelixSceneDesc::encoding).
constexpr uint32_t kEncodingPacked = 0;
constexpr uint32_t kEncodingBlockId = 1;

// The status word bits that device code sets instead of trapping; the host turns them into
// CAELIX_ERROR_DEVICE_STATUS.
constexpr uint32_t kStatusLookbackTimeout = 1u << 0;  // a decoupled look-back gave up waiting
constexpr uint32_t kStatusDepthGuard = 1u << 1;       // a walk exceeded its iteration guard
constexpr uint32_t kStatusNodeOverflow = 1u << 2;     // more 4-wide nodes than the capacity
constexpr uint32_t kStatusHashProbeLimit = 1u << 3;   // a hash probe ran past the table
constexpr uint32_t kStatusRecordOverflow = 1u << 4;   // a light record did not fit its capacity
constexpr uint32_t kStatusBadGroup = 1u << 5;         // a record named a group without a frame
constexpr uint32_t kStatusCopyTimeout = 1u << 6;      // a bulk copy into shared memory did not arrive in time

}  // namespace cx
