// Kernels and host sequence of the light BVH build (lt_build.cuh describes the pipeline).
#include <cuda/atomic>

#include "cx_device.cuh"
#include "lookback.cuh"
#include "lt_build.cuh"
#include "radix_sort.cuh"

namespace cx {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ float power6(const float f[6])
{
    return f[0] + f[1] + f[2] + f[3] + f[4] + f[5];
}

__device__ __forceinline__ float hmin(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float hmax(float a, float b) { return b > a ? b : a; }

__device__ __forceinline__ LightSummary load_summary(const LightSummary* p)
{
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    const float4 b = __ldg(reinterpret_cast<const float4*>(p) + 1);
    const float4 c = __ldg(reinterpret_cast<const float4*>(p) + 2);
    LightSummary s;
    s.face[0] = a.x; s.face[1] = a.y; s.face[2] = a.z; s.face[3] = a.w;
    s.face[4] = b.x; s.face[5] = b.y; s.lo[0] = b.z; s.lo[1] = b.w;
    s.lo[2] = c.x; s.hi[0] = c.y; s.hi[1] = c.z; s.hi[2] = c.w;
    return s;
}

// A summary written by another thread of the same kernel: read through L2 (not the
// non-coherent read-only path).
__device__ __forceinline__ LightSummary load_summary_cg(const LightSummary* p)
{
    const float4 a = __ldcg(reinterpret_cast<const float4*>(p));
    const float4 b = __ldcg(reinterpret_cast<const float4*>(p) + 1);
    const float4 c = __ldcg(reinterpret_cast<const float4*>(p) + 2);
    LightSummary s;
    s.face[0] = a.x; s.face[1] = a.y; s.face[2] = a.z; s.face[3] = a.w;
    s.face[4] = b.x; s.face[5] = b.y; s.lo[0] = b.z; s.lo[1] = b.w;
    s.lo[2] = c.x; s.hi[0] = c.y; s.hi[1] = c.z; s.hi[2] = c.w;
    return s;
}

__device__ __forceinline__ void store_summary(LightSummary* p, const LightSummary& s)
{
    float4* q = reinterpret_cast<float4*>(p);
    q[0] = make_float4(s.face[0], s.face[1], s.face[2], s.face[3]);
    q[1] = make_float4(s.face[4], s.face[5], s.lo[0], s.lo[1]);
    q[2] = make_float4(s.lo[2], s.hi[0], s.hi[1], s.hi[2]);
}

// LtUnion (caelix_light_tree_layout.hlsl:315-334): a summary of power 0 is skipped.
__device__ __forceinline__ LightSummary lt_union(const LightSummary& a, const LightSummary& b)
{
    if (power6(a.face) <= 0.0f) return b;
    if (power6(b.face) <= 0.0f) return a;
    LightSummary s;
#pragma unroll
    for (int f = 0; f < 6; ++f) s.face[f] = a.face[f] + b.face[f];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        s.lo[k] = hmin(a.lo[k], b.lo[k]);
        s.hi[k] = hmax(a.hi[k], b.hi[k]);
    }
    return s;
}

__device__ __forceinline__ uint32_t part1by2(uint32_t v)
{
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ uint32_t morton30(uint32_t x, uint32_t y, uint32_t z)
{
    return part1by2(x) | (part1by2(y) << 1) | (part1by2(z) << 2);
}

// ---------------------------------------------------------------------------------------------
// Gather emit + centre bounds: a thread per record (grid-stride), its 48-byte record, group, entry
// and group frame loaded up front, its 64-byte leaf written as four 16-byte stores (a warp's four
// store instructions fill whole lines between them); the centre codes max-reduced per warp at the
// end, one atomic per warp and code.
static_assert(sizeof(BrickLightRecord) == 48 && sizeof(LightBvhLeaf) == 64, "record and leaf sizes");

// One record's leaf (into q: a staging slot) and centre (the loads done by the caller).
__device__ __forceinline__ void emit_record(uint32_t i, uint4 w0, uint4 w1, uint32_t g, uint32_t e,
                                            const GroupFrame* __restrict__ frames, uint32_t frame_count,
                                            uint4* q, float4* __restrict__ centres,
                                            BuildControl* __restrict__ control, uint32_t lo_code[3],
                                            uint32_t hi_code[3])
{
    LightSummary local;
    local.face[0] = __uint_as_float(w0.x);
    local.face[1] = __uint_as_float(w0.y);
    local.face[2] = __uint_as_float(w0.z);
    local.face[3] = __uint_as_float(w0.w);
    local.face[4] = __uint_as_float(w1.x);
    local.face[5] = __uint_as_float(w1.y);
    const uint32_t box_lo = w1.z;
    const uint32_t box_hi = w1.w;
    float origin[3] = {0.0f, 0.0f, 0.0f};
    float r[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    float t[3] = {0.0f, 0.0f, 0.0f};
    if (frames && g >= frame_count) atomicOr(&control->status, kStatusBadGroup);
    if (frames && g < frame_count) {
        const GroupFrame* f = frames + g;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            origin[k] = __ldg(&f->origin[k]);
            t[k] = __ldg(&f->trans[k]);
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) r[k] = __ldg(&f->rot[k]);
    }
    local.lo[0] = origin[0] + (float)(box_lo & kVoxelMask);
    local.lo[1] = origin[1] + (float)((box_lo >> kVoxelBits) & kVoxelMask);
    local.lo[2] = origin[2] + (float)((box_lo >> (2 * kVoxelBits)) & kVoxelMask);
    local.hi[0] = origin[0] + (float)(box_hi & kVoxelMask);
    local.hi[1] = origin[1] + (float)((box_hi >> kVoxelBits) & kVoxelMask);
    local.hi[2] = origin[2] + (float)((box_hi >> (2 * kVoxelBits)) & kVoxelMask);

    // LtWorldSummary (caelix_light_gather_emit.hlsl:11-34).
    float centre[3], half[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        centre[k] = 0.5f * (local.lo[k] + local.hi[k]);
        half[k] = 0.5f * (local.hi[k] - local.lo[k]);
    }
    LightSummary w;
#pragma unroll
    for (int row = 0; row < 3; ++row) {
        const float wc = r[3 * row] * centre[0] + r[3 * row + 1] * centre[1] + r[3 * row + 2] * centre[2] +
                         t[row];
        const float wh = fabsf(r[3 * row]) * half[0] + fabsf(r[3 * row + 1]) * half[1] +
                         fabsf(r[3 * row + 2]) * half[2];
        w.lo[row] = wc - wh;
        w.hi[row] = wc + wh;
    }
#pragma unroll
    for (int f = 0; f < 6; ++f) w.face[f] = 0.0f;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const int axis = f >> 1;
        const float sign = (f & 1) ? -1.0f : 1.0f;
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const float d = sign * r[3 * b + axis];
            w.face[2 * b] += local.face[f] * hmax(0.0f, d);
            w.face[2 * b + 1] += local.face[f] * hmax(0.0f, -d);
        }
    }
    q[0] = make_uint4(__float_as_uint(w.face[0]), __float_as_uint(w.face[1]), __float_as_uint(w.face[2]),
                      __float_as_uint(w.face[3]));
    q[1] = make_uint4(__float_as_uint(w.face[4]), __float_as_uint(w.face[5]), __float_as_uint(w.lo[0]),
                      __float_as_uint(w.lo[1]));
    q[2] = make_uint4(__float_as_uint(w.lo[2]), __float_as_uint(w.hi[0]), __float_as_uint(w.hi[1]),
                      __float_as_uint(w.hi[2]));
    q[3] = make_uint4(g, e, 0u, kNone);
    float c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        c[k] = 0.5f * (w.lo[k] + w.hi[k]);
        const uint32_t code = float_order(c[k]);
        lo_code[k] = max(lo_code[k], ~code);
        hi_code[k] = max(hi_code[k], code);
    }
    centres[i] = make_float4(c[0], c[1], c[2], 0.0f);  // for the Morton codes (16 bytes, not the leaf)
}

__global__ void __launch_bounds__(kThreads)
    lt_emit_kernel(const BrickLightRecord* __restrict__ records, uint32_t n,
                   const uint32_t* __restrict__ record_group, const uint32_t* __restrict__ record_entry,
                   const GroupFrame* __restrict__ frames, uint32_t frame_count, LightBvhLeaf* __restrict__ leaves,
                   float4* __restrict__ centres, BuildControl* __restrict__ control)
{
    // A warp's 2 x 32 leaves are staged in shared memory and stored as whole 512-byte rows.
    __shared__ __align__(16) uint4 s_leaf[kThreads / 32][2][32 * 4];
    uint32_t lo_code[3] = {0, 0, 0};  // ~order(centre), max-reduced
    uint32_t hi_code[3] = {0, 0, 0};  // order(centre), max-reduced
    const uint4* rsrc = reinterpret_cast<const uint4*>(records);
    uint4* ldst = reinterpret_cast<uint4*>(leaves);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint4* stage0 = s_leaf[warp][0];
    uint4* stage1 = s_leaf[warp][1];
    // Two runs of 32 records per warp and step (base and base + stride), both loaded before either
    // is written (more loads in flight).
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + warp * 32u; base < n; base += 2 * stride) {
        const uint32_t i = base + lane;
        const uint32_t base2 = base + stride;
        const uint32_t i2 = base2 + lane;
        const bool one = i < n, two = i2 < n;
        uint4 a0 = make_uint4(0u, 0u, 0u, 0u), a1 = a0, b0 = a0, b1 = a0;
        uint32_t ag = 0, ae = 0, bg = 0, be = 0;
        if (one) {
            a0 = __ldg(rsrc + 3ull * i);
            a1 = __ldg(rsrc + 3ull * i + 1);
            ag = record_group ? __ldg(record_group + i) : 0u;
            ae = record_entry ? __ldg(record_entry + i) : i;
        }
        if (two) {
            b0 = __ldg(rsrc + 3ull * i2);
            b1 = __ldg(rsrc + 3ull * i2 + 1);
            bg = record_group ? __ldg(record_group + i2) : 0u;
            be = record_entry ? __ldg(record_entry + i2) : i2;
        }
        if (one) emit_record(i, a0, a1, ag, ae, frames, frame_count, stage0 + 4 * lane, centres, control, lo_code, hi_code);
        if (two) emit_record(i2, b0, b1, bg, be, frames, frame_count, stage1 + 4 * lane, centres, control, lo_code, hi_code);
        __syncwarp();
        // 16-byte unit u of the run is leaf u / 4's word u % 4.
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t u = 32u * q + lane;
            if (base + u / 4 < n) ldst[4ull * base + u] = stage0[u];
            if (base2 + u / 4 < n) ldst[4ull * base2 + u] = stage1[u];
        }
        __syncwarp();
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lo_code[k] = __reduce_max_sync(0xFFFFFFFFu, lo_code[k]);
        hi_code[k] = __reduce_max_sync(0xFFFFFFFFu, hi_code[k]);
    }
    if ((threadIdx.x & 31u) == 0) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            if (lo_code[k]) atomicMax(&control->bounds_code[k], lo_code[k]);
            if (hi_code[k]) atomicMax(&control->bounds_code[3 + k], hi_code[k]);
        }
    }
}

// The centre bounds of the build from the reduced codes (3e38 / -3e38 without leaves, as the
// reference's one-workgroup reduction starts).
__device__ __forceinline__ void decode_bounds(const BuildControl* control, float lo[3], float hi[3])
{
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const uint32_t l = control->bounds_code[k];
        const uint32_t h = control->bounds_code[3 + k];
        lo[k] = l ? float_unorder(~l) : 3.0e38f;
        hi[k] = h ? float_unorder(h) : -3.0e38f;
    }
}

// ---------------------------------------------------------------------------------------------
// Morton codes (value = leaf index) from the box centres the emit wrote + the four digit histograms
// + clearing the arrival counters and the range-count differences.
__global__ void __launch_bounds__(kThreads)
    lt_morton_kernel(const float4* __restrict__ centres, uint32_t n, const BuildControl* __restrict__ control,
                     uint32_t* __restrict__ keys, uint32_t* __restrict__ counter, uint32_t* __restrict__ cover,
                     uint32_t* __restrict__ hist)
{
    __shared__ uint32_t s_hist[4][kRadix];
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) (&s_hist[0][0])[i] = 0;
    float lo[3], hi[3];
    decode_bounds(control, lo, hi);
    float extent[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) extent[k] = hmax(hi[k] - lo[k], 1e-6f);
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 ctr = __ldg(centres + i);  // the world box centre (emit: 0.5 (lo + hi))
        const float centre[3] = {ctr.x, ctr.y, ctr.z};
        uint32_t cell[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const float q = hmin(hmax((centre[k] - lo[k]) / extent[k] * 1024.0f, 0.0f), 1023.0f);
            cell[k] = (uint32_t)q;
        }
        const uint32_t key = morton30(cell[0], cell[1], cell[2]);
        keys[i] = key;
        counter[i] = 0;
        cover[i] = 0;
#pragma unroll
        for (int p = 0; p < 4; ++p) atomicAdd(&s_hist[p][(key >> (8 * p)) & 255u], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) {
        const uint32_t v = (&s_hist[0][0])[i];
        if (v) atomicAdd(&hist[i], v);
    }
}

// ---------------------------------------------------------------------------------------------
// Karras 2012 binary radix tree over the sorted keys; ties broken by sorted position. Also the
// range-count differences: node i covers the leaf boundaries [a, b) of its range [a, b], so
// cover[a] += 1, cover[b] -= 1 (their prefix sum counts the nodes over every boundary).
__device__ __forceinline__ int lt_delta(const uint32_t* __restrict__ keys, int i, int j, int n, uint32_t key_i)
{
    if (j < 0 || j >= n) return -1;
    const uint32_t key_j = __ldg(keys + j);
    if (key_i == key_j) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clz(key_i ^ key_j);
}

__global__ void __launch_bounds__(kThreads)
    lt_karras_kernel(const uint32_t* __restrict__ keys, int n, uint32_t* __restrict__ left,
                     uint32_t* __restrict__ right, uint32_t* __restrict__ parent, uint32_t* __restrict__ leaf_parent,
                     uint32_t* __restrict__ cover, uint32_t* __restrict__ range_end)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    if (i == 0) parent[0] = kNone;
    const uint32_t key_i = __ldg(keys + i);
    const int d = lt_delta(keys, i, i + 1, n, key_i) - lt_delta(keys, i, i - 1, n, key_i) >= 0 ? 1 : -1;
    const int delta_min = lt_delta(keys, i, i - d, n, key_i);
    // The searches with shifts for the divisions by powers of two (lengths are positive, so the
    // quotients and the ceilings are those of the divisions).
    int length_max = 2;
    while (lt_delta(keys, i, i + (d > 0 ? length_max : -length_max), n, key_i) > delta_min) length_max <<= 1;
    int length = 0;
    for (int step = length_max >> 1; step >= 1; step >>= 1)
        if (lt_delta(keys, i, i + (d > 0 ? length + step : -(length + step)), n, key_i) > delta_min) length += step;
    const int j = i + (d > 0 ? length : -length);
    const int delta_node = lt_delta(keys, i, j, n, key_i);
    int split = 0;
    uint32_t shift = 1;  // the divisor 2^shift
    int step2 = (int)(((uint32_t)length + 1u) >> 1);
    for (;;) {
        if (lt_delta(keys, i, i + (d > 0 ? split + step2 : -(split + step2)), n, key_i) > delta_node) split += step2;
        if (step2 == 1) break;
        ++shift;
        step2 = (int)(((uint32_t)length + ((1u << shift) - 1u)) >> shift);
    }
    const int gamma = i + split * d + min(d, 0);
    const int a = min(i, j);
    const int b = max(i, j);
    const uint32_t l = a == gamma ? (kChildLeafBit | (uint32_t)gamma) : (uint32_t)gamma;
    const uint32_t r = b == gamma + 1 ? (kChildLeafBit | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
    left[i] = l;
    right[i] = r;
    if (l & kChildLeafBit) leaf_parent[l & ~kChildLeafBit] = (uint32_t)i;
    else parent[l] = (uint32_t)i;
    if (r & kChildLeafBit) leaf_parent[r & ~kChildLeafBit] = (uint32_t)i;
    else parent[r] = (uint32_t)i;
    range_end[i] = (uint32_t)j;
    atomicAdd(cover + a, 1u);
    atomicAdd(cover + b, 0xFFFFFFFFu);
}

// ---------------------------------------------------------------------------------------------
// Bottom-up aggregation and the 4-wide collapse, by tiles. A CTA owns a tile of kAggTile
// consecutive sorted leaves and the binary nodes with the same indices (a node is an end of its
// leaf range, so every node whose range lies inside the tile has its index there). The tile's leaf
// summaries (each sorted leaf read through the permutation), node links, 4-wide indices, leaf
// indices, arrival counters and node summaries live in shared memory; then
//   0. the summaries of the leaves under a node that crosses the tile (a parent or grandparent
//      outside it) are written in sorted order (`sorted`) for the two upper kernels;
//   1. one walk per leaf: the second thread to arrive at an in-tile node computes its summary from
//      both children and goes on (block-scope arrivals, nothing but shared memory touched). A walk
//      stops at the first node whose range crosses the tile and lists the child it comes from
//      (`upper`: an in-tile node, or a leaf with the leaf bit) for lt_aggregate_upper_kernel;
//   2. the in-tile summaries go to their 64-byte global slots (coalesced full-sector writes);
//   3. every in-tile node at even depth becomes its 224-byte 4-wide node: four threads per node
//      (thread c: child slot c) write its row into a staging buffer of kRowChunk rows, which the
//      CTA then stores as 16-byte units; the parent words of its leaf slots go into the leaves.
//      Even-depth nodes that cross the tile are listed (`crossing`) for lt_wide_upper_kernel.
// The depths and 4-wide indices come from the scans, which run before this kernel.
constexpr uint32_t kAggTile = 256;
constexpr uint32_t kNodeQuads = sizeof(LightBvhNode) / 16;  // 14
constexpr uint32_t kRowChunk = kAggTile / 4;                 // 4-wide rows staged at a time (4 threads each)

__device__ __forceinline__ void store_slot(AggregateSlot* p, const LightSummary& s)
{
    float4* q = reinterpret_cast<float4*>(p);
    q[0] = make_float4(s.face[0], s.face[1], s.face[2], s.face[3]);
    q[1] = make_float4(s.face[4], s.face[5], s.lo[0], s.lo[1]);
    q[2] = make_float4(s.lo[2], s.hi[0], s.hi[1], s.hi[2]);
    q[3] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// The child slots of the 4-wide node over a binary node with children l and r (a child's own
// children from `link_of`): ll, then lr or (l a leaf) rl, then rl or rr, then rr or nothing; a leaf
// child stands for itself, an empty slot is kNone.
template <typename LinkOf>
__device__ __forceinline__ void wide_slots(uint32_t l, uint32_t r, LinkOf link_of, uint32_t slots[4])
{
    const bool l_leaf = (l & kChildLeafBit) != 0;
    const bool r_leaf = (r & kChildLeafBit) != 0;
    uint32_t ll = l, lr = kNone, rl = r, rr = kNone;
    if (!l_leaf) {
        const uint2 c = link_of(l);
        ll = c.x;
        lr = c.y;
    }
    if (!r_leaf) {
        const uint2 c = link_of(r);
        rl = c.x;
        rr = c.y;
    }
    slots[0] = ll;
    slots[1] = l_leaf ? rl : lr;
    slots[2] = l_leaf ? rr : rl;
    slots[3] = l_leaf ? kNone : rr;
}

// Summary word `idx` (faces 0..5, lo 6..8, hi 9..11) of row word wd (0..47) of a 4-wide node: the
// child slot and the word within its summary.
__device__ __forceinline__ void row_word(uint32_t wd, uint32_t& c, uint32_t& idx)
{
    if (wd < 24) {
        c = wd / 6;
        idx = wd % 6;
    } else if (wd < 36) {
        c = (wd - 24) / 3;
        idx = 6 + (wd - 24) % 3;
    } else {
        c = (wd - 36) / 3;
        idx = 9 + (wd - 36) % 3;
    }
}

__global__ void __launch_bounds__(kAggTile)
    lt_tile_kernel(uint32_t n, uint32_t node_capacity, LightSummary* __restrict__ sorted,
                   const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                   const uint32_t* __restrict__ parent, const uint32_t* __restrict__ leaf_parent,
                   const uint32_t* __restrict__ range_end, const uint32_t* __restrict__ depth,
                   const uint32_t* __restrict__ wide, const uint32_t* __restrict__ values,
                   AggregateSlot* __restrict__ aggregates, uint32_t* __restrict__ upper,
                   uint32_t* __restrict__ crossing, LightBvhLeaf* __restrict__ leaves,
                   LightBvhNode* __restrict__ nodes, BuildControl* control)
{
    // The arrival counters and the tile's lists are dead once the rows are built: they share
    // their memory with the row staging.
    union Scratch
    {
        struct
        {
            uint32_t count[kAggTile];
            uint32_t upper[kAggTile];  // the tile's upper walks and crossing even-depth nodes,
            uint32_t cross[kAggTile];  // copied to the global lists with one atomic each
        } walk;
        uint4 row[kRowChunk * kNodeQuads];  // rows being built
    };
    __shared__ __align__(16) Scratch s_x;
    uint32_t* const s_count = s_x.walk.count;
    uint32_t* const s_upper = s_x.walk.upper;
    uint32_t* const s_cross = s_x.walk.cross;
    uint4* const s_row = s_x.row;
    __shared__ LightSummary s_leaf[kAggTile];
    __shared__ LightSummary s_sum[kAggTile];
    __shared__ uint4 s_link[kAggTile];  // left, right, parent, range end of the nodes lo .. lo + kAggTile - 1
    __shared__ uint32_t s_wide[kAggTile];
    __shared__ uint32_t s_value[kAggTile];
    __shared__ uint32_t s_even[kAggTile];  // the tile's in-tile even-depth nodes (offsets from lo), in order
    __shared__ uint32_t s_scan[kAggTile / 32];
    __shared__ uint32_t s_row_w[kRowChunk];
    __shared__ uint32_t s_upper_count, s_cross_count, s_upper_base, s_cross_base;
    const uint32_t lo = blockIdx.x * kAggTile;
    const uint32_t hi = min(lo + kAggTile, n) - 1;  // last leaf of the tile
    const uint32_t k = threadIdx.x;
    const uint32_t j = lo + k;  // this thread's leaf, and the node of the same index
    const uint32_t count = min(control->node_count, node_capacity);
    if (k == 0) {
        s_upper_count = 0;
        s_cross_count = 0;
    }
    s_count[k] = 0;
    uint32_t node = kNone;
    bool mine = false;  // node j lies inside the tile
    bool even = false;
    if (j < n) {
        // The sorted leaf's summary, read through the permutation (the leaves' parent words,
        // written below by other tiles, are other bytes of the rows).
        const uint32_t v = __ldg(values + j);
        s_value[k] = v;
        s_leaf[k] = load_summary(&leaves[v].summary);
        node = __ldg(leaf_parent + j);
    }
    if (j + 1 < n) {
        const uint4 link = make_uint4(__ldg(left + j), __ldg(right + j), __ldg(parent + j), __ldg(range_end + j));
        s_link[k] = link;
        s_wide[k] = __ldg(wide + j);
        mine = min(j, link.w) >= lo && max(j, link.w) <= hi;
        even = (__ldg(depth + j) & 1u) == 0;
    }
    // The in-tile even-depth nodes in node order (their 4-wide indices rise with it); the block
    // scan's barriers also publish the loads above.
    uint32_t evens;
    {
        const uint32_t at = block_exclusive_sum<kAggTile>(even && mine ? 1u : 0u, s_scan, evens);
        if (even && mine) s_even[at] = k;
    }
    if (even && !mine) s_cross[atomicAdd(&s_cross_count, 1u)] = j;
    // The summaries of the leaves under a node that crosses the tile (a parent or a grandparent
    // outside it), in sorted order for the upper kernels.
    if (j < n && node != kNone) {
        const auto inside_node = [&](uint32_t x) {
            return x - lo < kAggTile && x + 1 < n && min(x, s_link[x - lo].w) >= lo && max(x, s_link[x - lo].w) <= hi;
        };
        bool needed = !inside_node(node);
        if (!needed) {
            const uint32_t g = s_link[node - lo].z;
            needed = g != kNone && !inside_node(g);
        }
        if (needed) store_summary(sorted + j, s_leaf[k]);
    }
    // 1. The walks.
    if (j < n) {
        LightSummary cur = s_leaf[k];
        uint32_t from = kChildLeafBit | j;
        uint32_t steps = 0;
        for (; steps < 128 && node != kNone; ++steps) {
            uint4 link = make_uint4(0u, 0u, 0u, 0u);
            bool inside = node - lo < kAggTile && node + 1 < n;
            if (inside) {
                link = s_link[node - lo];
                inside = min(node, link.w) >= lo && max(node, link.w) <= hi;
            }
            if (!inside) {
                s_upper[atomicAdd(&s_upper_count, 1u)] = from;  // the upper walks go on from here
                break;
            }
            cuda::atomic_ref<uint32_t, cuda::thread_scope_block> arrival(s_count[node - lo]);
            if (arrival.fetch_add(1u, cuda::memory_order_acq_rel) == 0) break;
            const uint32_t l = link.x;
            const uint32_t sibling = l == from ? link.y : l;
            const uint32_t sib_at = (sibling & ~kChildLeafBit) - lo;
            if (sib_at >= kAggTile) {  // a child outside its parent's range: a broken tree
                atomicOr(&control->status, kStatusDepthGuard);
                break;
            }
            const LightSummary& sib = (sibling & kChildLeafBit) ? s_leaf[sib_at] : s_sum[sib_at];
            cur = l == from ? lt_union(cur, sib) : lt_union(sib, cur);
            s_sum[node - lo] = cur;
            from = node;
            node = link.z;
        }
        if (steps == 128) atomicOr(&control->status, kStatusDepthGuard);
    }
    __syncthreads();
    if (k == 0) {
        s_upper_base = s_upper_count ? atomicAdd(&control->upper_count, s_upper_count) : 0u;
        s_cross_base = s_cross_count ? atomicAdd(&control->crossing_count, s_cross_count) : 0u;
    }
    // 2. The in-tile summaries.
    if (mine) store_slot(aggregates + j, s_sum[k]);
    __syncthreads();
    if (k < s_upper_count) upper[s_upper_base + k] = s_upper[k];
    if (k < s_cross_count) crossing[s_cross_base + k] = s_cross[k];
    // 3. The in-tile 4-wide nodes, kRowChunk at a time: four threads per node (thread c: child
    // slot c; the children of an in-tile node are in the tile) write its row into shared memory,
    // then the CTA stores the rows as 16-byte units (consecutive rows are consecutive 4-wide nodes,
    // except where a node that crosses the tile takes its place).
    __syncthreads();  // the lists are copied out: their memory takes the rows
    const uint32_t r = k >> 2;
    const uint32_t c = k & 3u;
    for (uint32_t first = 0; first < evens; first += kRowChunk) {
        const uint32_t rows = min(kRowChunk, evens - first);
        if (r < rows) {
            const uint32_t i = lo + s_even[first + r];
            const uint4 link = s_link[i - lo];
            const uint32_t w = s_wide[i - lo];
            uint32_t slots[4];
            wide_slots(link.x, link.y, [&](uint32_t x) { const uint4 cl = s_link[x - lo]; return make_uint2(cl.x, cl.y); },
                       slots);
            const uint32_t slot = c == 0 ? slots[0] : c == 1 ? slots[1] : c == 2 ? slots[2] : slots[3];
            float* row = reinterpret_cast<float*>(s_row + r * kNodeQuads);
            float4 a = make_float4(0.0f, 0.0f, 0.0f, 0.0f), b4 = a, c4 = a;
            uint32_t word = kNone;
            if (slot != kNone) {
                const uint32_t at = (slot & ~kChildLeafBit) - lo;
                const float4* sm = reinterpret_cast<const float4*>((slot & kChildLeafBit) ? &s_leaf[at] : &s_sum[at]);
                a = sm[0];
                b4 = sm[1];
                c4 = sm[2];
                word = (slot & kChildLeafBit) ? (kChildLeafBit | s_value[at]) : s_wide[at];
                if ((slot & kChildLeafBit) && w < count)
                    leaves[s_value[at]].parent = (w << kParentSlotBits) | c;  // the leaf's parent word
            }
            // faces 6c .. 6c + 5, lo 24 + 3c .., hi 36 + 3c .. (a summary: faces, lo, hi), child c
            float2* face = reinterpret_cast<float2*>(row + 6 * c);
            face[0] = make_float2(a.x, a.y);
            face[1] = make_float2(a.z, a.w);
            face[2] = make_float2(b4.x, b4.y);
            row[24 + 3 * c] = b4.z;
            row[25 + 3 * c] = b4.w;
            row[26 + 3 * c] = c4.x;
            row[36 + 3 * c] = c4.y;
            row[37 + 3 * c] = c4.z;
            row[38 + 3 * c] = c4.w;
            reinterpret_cast<uint32_t*>(row)[48 + c] = word;
            if (c == 0) {
                s_row_w[r] = w < count ? w : kNone;  // past the node capacity: the header reports the overflow
                // The node's own parent link: the 4-wide parent is the binary grandparent (the
                // guard keeps a broken tree from reading outside the arrays).
                uint32_t up_node = kNone, up_slot = 0;
                if (i != 0) {
                    const auto link_of = [&](uint32_t x) {
                        return x - lo < kAggTile ? s_link[x - lo]
                                                 : make_uint4(__ldg(left + x), __ldg(right + x), __ldg(parent + x), 0u);
                    };
                    const uint32_t p = link.z;
                    const uint4 lp = p + 1 < n ? link_of(p) : make_uint4(kNone, kNone, kNone, 0u);
                    const uint32_t g = lp.z;
                    if (g + 1 < n) {
                        const uint32_t gl = link_of(g).x;
                        const uint32_t b0 = p == gl ? 0u : ((gl & kChildLeafBit) ? 1u : 2u);
                        up_slot = b0 + (lp.y == i ? 1u : 0u);
                        up_node = g - lo < kAggTile ? s_wide[g - lo] : __ldg(wide + g);
                    }
                }
                s_row[r * kNodeQuads + 13] = make_uint4(up_node, up_slot, 0u, 0u);
            }
        }
        __syncthreads();
        for (uint32_t t = k; t < rows * kNodeQuads; t += kAggTile) {
            const uint32_t rr = t / kNodeQuads;
            const uint32_t w = s_row_w[rr];
            if (w != kNone) reinterpret_cast<uint4*>(nodes + w)[t - rr * kNodeQuads] = s_row[t];
        }
        __syncthreads();
    }
}

// The walks up through the nodes whose range crosses a tile, from the children the tiles listed
// (an in-tile node, its summary in its slot, or a leaf): the second thread to arrive at a node
// computes it and goes on. The walks were run inside the tile kernel at first: chains of
// dependent device-scope atomics and L2 loads that kept each tile's CTA resident for them. Up to
// kUpperOneCtaItems walks (one per thread: builds of up to about 16 k leaves) run in one CTA
// (kOneCta), whose arrivals are block-scope and whose siblings' summaries come through L1; more
// run on a persistent grid with device-scope arrivals (the list's length is known on the device
// only: each variant checks it). With six walks per thread (97 k leaves) the one CTA was slower
// than the grid (the light-tree flush of the 2 M-brick world 0.22 against 0.18 ms).
constexpr uint32_t kUpperOneCtaItems = 1024;
constexpr uint32_t kUpperOneCtaThreads = 1024;

// A summary written earlier by this kernel's CTA (after an acquire: weak loads through L1).
__device__ __forceinline__ LightSummary load_summary_weak(const LightSummary* p)
{
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = q[0], b = q[1], c = q[2];
    LightSummary s;
    s.face[0] = a.x; s.face[1] = a.y; s.face[2] = a.z; s.face[3] = a.w;
    s.face[4] = b.x; s.face[5] = b.y; s.lo[0] = b.z; s.lo[1] = b.w;
    s.lo[2] = c.x; s.hi[0] = c.y; s.hi[1] = c.z; s.hi[2] = c.w;
    return s;
}

template <bool kOneCta>
__global__ void __launch_bounds__(kOneCta ? kUpperOneCtaThreads : kThreads)
    lt_aggregate_upper_kernel(const LightSummary* __restrict__ sorted, const uint32_t* __restrict__ left,
                              const uint32_t* __restrict__ right, const uint32_t* __restrict__ parent,
                              const uint32_t* __restrict__ leaf_parent, uint32_t* counter,
                              AggregateSlot* aggregates, const uint32_t* __restrict__ upper, BuildControl* control)
{
    constexpr cuda::thread_scope kScope = kOneCta ? cuda::thread_scope_block : cuda::thread_scope_device;
    const uint32_t count = control->upper_count;
    if (kOneCta ? count > kUpperOneCtaItems : count <= kUpperOneCtaItems) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        uint32_t from = upper[i];
        const bool leaf = (from & kChildLeafBit) != 0;
        LightSummary cur = leaf ? load_summary_cg(sorted + (from & ~kChildLeafBit)) : load_summary_cg(&aggregates[from].summary);
        uint32_t node = leaf ? __ldg(leaf_parent + (from & ~kChildLeafBit)) : __ldg(parent + from);
        uint32_t depth = 0;
        for (; depth < 128 && node != kNone; ++depth) {
            const uint32_t l = __ldg(left + node);
            const uint32_t r = __ldg(right + node);
            const uint32_t up = __ldg(parent + node);
            const uint32_t sibling = l == from ? r : l;
            cuda::atomic_ref<uint32_t, kScope> arrival(counter[node]);
            if (arrival.fetch_add(1u, cuda::memory_order_acq_rel) == 0) break;
            LightSummary sib;
            if (sibling & kChildLeafBit) sib = load_summary_cg(sorted + (sibling & ~kChildLeafBit));
            else if (kOneCta) sib = load_summary_weak(&aggregates[sibling].summary);
            else sib = load_summary_cg(&aggregates[sibling].summary);
            cur = l == from ? lt_union(cur, sib) : lt_union(sib, cur);
            store_slot(aggregates + node, cur);
            from = node;
            node = up;
        }
        if (depth == 128) atomicOr(&control->status, kStatusDepthGuard);
    }
}

// The 4-wide nodes over the even-depth binary nodes that cross a tile (listed by the tile kernel):
// one thread per node, children and summaries read from the global arrays and slots, the row
// written by the thread; the parent words of its leaf slots written into the leaves.
__global__ void __launch_bounds__(kThreads)
    lt_wide_upper_kernel(uint32_t n, uint32_t node_capacity, const uint32_t* __restrict__ values,
                         const uint32_t* __restrict__ left, const uint32_t* __restrict__ right,
                         const uint32_t* __restrict__ parent, const uint32_t* __restrict__ crossing,
                         const uint32_t* __restrict__ wide, const LightSummary* __restrict__ sorted,
                         const AggregateSlot* __restrict__ aggregates, LightBvhLeaf* __restrict__ leaves,
                         LightBvhNode* __restrict__ nodes, const BuildControl* __restrict__ control)
{
    const uint32_t count = min(control->node_count, node_capacity);
    const uint32_t listed = control->crossing_count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < listed; t += gridDim.x * blockDim.x) {
        const uint32_t i = crossing[t];
        const uint32_t w = __ldg(wide + i);
        if (w >= count) continue;
        uint32_t slots[4];
        wide_slots(__ldg(left + i), __ldg(right + i),
                   [&](uint32_t x) { return make_uint2(__ldg(left + x), __ldg(right + x)); }, slots);
        uint4* row = reinterpret_cast<uint4*>(nodes + w);
        LightSummary sm[4];
        uint32_t word[4];
#pragma unroll
        for (uint32_t c = 0; c < 4; ++c) {
#pragma unroll
            for (int f = 0; f < 6; ++f) sm[c].face[f] = 0.0f;
#pragma unroll
            for (int k = 0; k < 3; ++k) sm[c].lo[k] = sm[c].hi[k] = 0.0f;
            word[c] = kNone;
            const uint32_t slot = slots[c];
            if (slot == kNone) continue;
            if (slot & kChildLeafBit) {
                const uint32_t p = slot & ~kChildLeafBit;
                sm[c] = load_summary_cg(sorted + p);
                const uint32_t leaf = __ldg(values + p);
                word[c] = kChildLeafBit | leaf;
                leaves[leaf].parent = (w << kParentSlotBits) | c;  // the leaf's parent word, in place
            } else {
                sm[c] = load_summary_cg(&aggregates[slot].summary);
                word[c] = __ldg(wide + slot);
            }
        }
        float f[48];
#pragma unroll
        for (uint32_t wd = 0; wd < 48; ++wd) {
            uint32_t c, idx;
            row_word(wd, c, idx);
            f[wd] = reinterpret_cast<const float*>(&sm[c])[idx];
        }
#pragma unroll
        for (int u = 0; u < 12; ++u) row[u] = make_uint4(__float_as_uint(f[4 * u]), __float_as_uint(f[4 * u + 1]),
                                                         __float_as_uint(f[4 * u + 2]), __float_as_uint(f[4 * u + 3]));
        row[12] = make_uint4(word[0], word[1], word[2], word[3]);
        // The node's own parent link.
        uint32_t up_node = kNone, up_slot = 0;
        if (i != 0) {
            const uint32_t p = __ldg(parent + i);
            const uint32_t g = p + 1 < n ? __ldg(parent + p) : kNone;
            if (g + 1 < n) {
                const uint32_t gl = __ldg(left + g);
                const uint32_t b0 = p == gl ? 0u : ((gl & kChildLeafBit) ? 1u : 2u);
                up_slot = b0 + (__ldg(right + p) == i ? 1u : 0u);
                up_node = __ldg(wide + g);
            }
        }
        row[13] = make_uint4(up_node, up_slot, 0u, 0u);
    }
}

// ---------------------------------------------------------------------------------------------
// Single-pass exclusive scans over tiles of kScanItems per thread (decoupled look-back by one warp,
// warp_lookback).
constexpr int kScanItems = 32;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

// A thread's kScanItems consecutive words from base (a multiple of kScanItems): 16-byte loads
// when all lie below count, else word by word (zero past count).
__device__ __forceinline__ void load_run(const uint32_t* p, uint32_t base, uint32_t count, uint32_t (&v)[kScanItems])
{
    if (base + kScanItems <= count) {
        const uint4* q = reinterpret_cast<const uint4*>(p + base);
#pragma unroll
        for (int k = 0; k < kScanItems / 4; ++k) {
            const uint4 x = q[k];
            v[4 * k] = x.x;
            v[4 * k + 1] = x.y;
            v[4 * k + 2] = x.z;
            v[4 * k + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = base + k < count ? p[base + k] : 0u;
    }
}

__device__ __forceinline__ void store_run(uint32_t* p, uint32_t base, uint32_t count, const uint32_t (&v)[kScanItems])
{
    if (base + kScanItems <= count) {
        uint4* q = reinterpret_cast<uint4*>(p + base);
#pragma unroll
        for (int k = 0; k < kScanItems / 4; ++k) q[k] = make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k)
            if (base + k < count) p[base + k] = v[k];
    }
}

// cover[g] for g < count becomes the number of binary nodes over leaf boundary g (inclusive prefix
// sum of the differences). The u32 differences wrap; the prefix is exact.
__global__ void __launch_bounds__(kScanThreads)
    lt_cover_scan_kernel(uint32_t count, uint32_t* cover, uint32_t* states, uint32_t* tile_counter,
                         BuildControl* control)
{
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_scan[kScanThreads / 32];
    __shared__ uint32_t s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    load_run(cover, base, count, v);
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) sum += v[k];
    uint32_t total;
    const uint32_t local = block_exclusive_sum<kScanThreads>(sum, s_scan, total);
    // The look-back values are 30-bit: the range counts (at most the tree depth) never need more,
    // but a tile's sum of differences can be "negative"; carry it as its low 30 bits.
    if (threadIdx.x < 32) {
        const uint32_t p = warp_lookback<false>(states, tile, total & kTileValueMask, &control->status);
        if (threadIdx.x == 0) s_prefix = p;
    }
    __syncthreads();
    uint32_t run = s_prefix + local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        run += v[k];
        v[k] = run & kTileValueMask;
    }
    store_run(cover, base, count, v);
}

// The depth of binary node i is the number of nodes over its split boundary minus one (the nodes
// over boundary gamma are node i and its ancestors); even depths are flagged and scanned into the
// 4-wide node index (wide[i]). The last tile writes the node count.
__global__ void __launch_bounds__(kScanThreads)
    lt_flags_scan_kernel(uint32_t nodes, const uint32_t* __restrict__ left, const uint32_t* __restrict__ cover,
                         uint32_t* __restrict__ depth_out, uint32_t* __restrict__ wide, uint32_t* states,
                         uint32_t* tile_counter, BuildControl* control)
{
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_scan[kScanThreads / 32];
    __shared__ uint32_t s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t flag[kScanItems];
    uint32_t v[kScanItems];
    load_run(left, base, nodes, v);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) v[k] = base + k < nodes ? __ldg(cover + (v[k] & ~kChildLeafBit)) - 1u : 0u;
    store_run(depth_out, base, nodes, v);
    uint32_t sum = 0;
    bool deep = false;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        deep = deep || (base + k < nodes && v[k] >= 128u);
        flag[k] = base + k < nodes && (v[k] & 1u) == 0 ? 1u : 0u;
        sum += flag[k];
    }
    if (deep) atomicOr(&control->status, kStatusDepthGuard);
    uint32_t total;
    const uint32_t local = block_exclusive_sum<kScanThreads>(sum, s_scan, total);
    if (threadIdx.x < 32) {
        const uint32_t p = warp_lookback<false>(states, tile, total, &control->status);
        if (threadIdx.x == 0) {
            s_prefix = p;
            if (tile == gridDim.x - 1) control->node_count = p + total;
        }
    }
    __syncthreads();
    uint32_t run = s_prefix + local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = run;
        run += flag[k];
    }
    store_run(wide, base, nodes, v);
}

// ---------------------------------------------------------------------------------------------
// The header (one thread): root summary, counts, overflow; the one-leaf tree's single node.
__global__ void lt_finish_kernel(uint32_t n, uint32_t found, uint32_t node_capacity, LightBvhLeaf* leaves,
                                 LightBvhNode* nodes, const AggregateSlot* aggregates, LightTreeHeader* header,
                                 LightTreeState* state, const BuildControl* control)
{
    LightSummary root;
#pragma unroll
    for (int f = 0; f < 6; ++f) root.face[f] = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) root.lo[k] = root.hi[k] = 0.0f;
    uint32_t root_index = kNone, node_count = 0, overflow = 0;
    if (n == 1) {
        root = load_summary_cg(&leaves[0].summary);
        LightBvhNode* node = nodes;
        float4* q = reinterpret_cast<float4*>(node);
        for (int v = 0; v < 12; ++v) q[v] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        for (int f = 0; f < 6; ++f) node->child_face[0][f] = root.face[f];
        for (int k = 0; k < 3; ++k) {
            node->child_lo[0][k] = root.lo[k];
            node->child_hi[0][k] = root.hi[k];
        }
        *reinterpret_cast<uint4*>(node->child) = make_uint4(kChildLeafBit, kNone, kNone, kNone);
        *reinterpret_cast<uint4*>(&node->parent) = make_uint4(kNone, 0u, 0u, 0u);
        leaves[0].parent = 0;
        root_index = 0;
        node_count = 1;
    } else if (n >= 2) {
        node_count = control->node_count;
        if (node_count > node_capacity) {
            overflow = 1;
        } else {
            root = load_summary_cg(&aggregates[0].summary);
            root_index = 0;
        }
    }
    store_summary(&header->summary, root);
    *reinterpret_cast<uint4*>(&header->root) = make_uint4(root_index, overflow ? 0u : n, node_count, 0u);
    float lo[3], hi[3];
    decode_bounds(control, lo, hi);
    state->building = 0;
    state->leaves_found = found;
    state->leaves_dropped = found - n;
    state->builds += 1;
    state->node_overflow = overflow;
    state->status = control->status | (overflow ? kStatusNodeOverflow : 0u);
    for (int k = 0; k < 3; ++k) {
        state->bounds[k] = lo[k];
        state->bounds[3 + k] = hi[k];
    }
}

uint32_t grid_for(uint32_t n, uint32_t per_block, uint32_t cap)
{
    uint32_t g = (n + per_block - 1) / per_block;
    if (g == 0) g = 1;
    return g < cap ? g : cap;
}

uint64_t align256(uint64_t x) { return (x + 255u) & ~uint64_t{255}; }

// Resident CTAs of `kernel` per SM at `threads` threads (at least 1).
template <typename Kernel>
uint32_t ctas_per_sm(Kernel kernel, int threads)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1)
        return 1;
    return (uint32_t)per_sm;
}

uint64_t zero_words(uint32_t n, uint32_t kpt)
{
    // control words, the sort scratch of tiles of 256 * kpt keys, then two scan states and their
    // tile counters
    return sizeof(BuildControl) / 4 + sort_scratch_words(n, kpt) + 2ull * ((n + kScanTile - 1) / kScanTile) + 2;
}

}  // namespace

uint64_t lt_buffer_bytes(uint32_t cap)
{
    const uint64_t c = cap < 2 ? 2 : cap;
    uint64_t b = 0;
    b += align256(c * sizeof(LightBvhLeaf));
    b += align256(c * sizeof(LightBvhNode));  // node capacity = leaf capacity (>= n - 1 nodes)
    b += align256(128);                       // header + state
    b += 12 * align256(c * 4);                // u32 arrays
    b += align256(c * sizeof(AggregateSlot));
    b += align256(c * sizeof(LightSummary));
    b += align256(zero_words((uint32_t)c, kSortMinKeysPerThread) * 4);
    return b;
}

LightBvhBuffers lt_carve(void* base, uint32_t cap)
{
    const uint64_t c = cap < 2 ? 2 : cap;
    LightBvhBuffers b;
    b.leaf_capacity = cap;
    b.node_capacity = (uint32_t)c;
    char* p = static_cast<char*>(base);
    auto take = [&](uint64_t bytes) {
        char* q = p;
        p += align256(bytes);
        return q;
    };
    auto u32 = [&]() { return reinterpret_cast<uint32_t*>(take(c * 4)); };
    b.leaves = reinterpret_cast<LightBvhLeaf*>(take(c * sizeof(LightBvhLeaf)));
    b.nodes = reinterpret_cast<LightBvhNode*>(take(c * sizeof(LightBvhNode)));
    char* hs = take(128);
    b.header = reinterpret_cast<LightTreeHeader*>(hs);
    b.state = reinterpret_cast<LightTreeState*>(hs + 64);
    b.keys = u32();
    b.values = u32();
    b.keys_alt = u32();
    b.values_alt = u32();
    b.left = u32();
    b.right = u32();
    b.parent = u32();
    b.leaf_parent = u32();
    b.counter = u32();
    b.depth = u32();
    b.wide = u32();
    b.cover = u32();
    b.aggregates = reinterpret_cast<AggregateSlot*>(take(c * sizeof(AggregateSlot)));
    b.sorted = reinterpret_cast<LightSummary*>(take(c * sizeof(LightSummary)));
    char* z = take(zero_words((uint32_t)c, kSortMinKeysPerThread) * 4);
    b.control = reinterpret_cast<BuildControl*>(z);
    b.sort_scratch = reinterpret_cast<uint32_t*>(z + sizeof(BuildControl));
    return b;
}

cudaError_t lt_build(const LightBvhBuffers& b, const LightBvhInput& in, cudaStream_t stream, cudaEvent_t* stage)
{
    const uint32_t found = in.count;
    const uint32_t n = found < b.leaf_capacity ? found : b.leaf_capacity;
    auto mark = [&](int k) {
        if (stage) cudaEventRecord(stage[k], stream);
    };
    mark(0);
    // Zeroed words of this build: control, the sort scratch sized for n, two scan state arrays and
    // their tile counters.
    const uint32_t kpt = sort_keys_per_thread_ok(in.sort_keys_per_thread) ? in.sort_keys_per_thread
                                                                             : sort_keys_per_thread_for(n);
    const uint32_t scan_tiles_n = (n + kScanTile - 1) / kScanTile;
    uint32_t* cover_states = b.sort_scratch + sort_scratch_words(n, kpt);
    uint32_t* flag_states = cover_states + scan_tiles_n;
    uint32_t* scan_counters = flag_states + scan_tiles_n;
    cudaError_t e = cudaMemsetAsync(b.control, 0, zero_words(n, kpt) * 4, stream);
    if (e != cudaSuccess) return e;
    const uint32_t sms = current_sm_count();
    if (n > 0) {
        // The grid-stride kernels run one full wave of resident CTAs.
        static const uint32_t emit_per_sm = ctas_per_sm(lt_emit_kernel, kThreads);
        static const uint32_t morton_per_sm = ctas_per_sm(lt_morton_kernel, kThreads);
        lt_emit_kernel<<<grid_for(n, 2 * kThreads, sms * emit_per_sm), kThreads, 0, stream>>>(
            in.records, n, in.record_group, in.record_entry, in.group_frames, in.group_count, b.leaves,
            reinterpret_cast<float4*>(b.aggregates), b.control);  // the slots hold the centres until aggregation
        mark(1);
        lt_morton_kernel<<<grid_for(n, kThreads * 4, sms * morton_per_sm), kThreads, 0, stream>>>(
            reinterpret_cast<const float4*>(b.aggregates), n, b.control, b.keys, b.counter, b.cover, b.sort_scratch);
        mark(2);
        // The sort (one small-sort CTA up to kSmallSortKeys pairs); later kernels read a sorted
        // leaf's summary through the permutation.
        onesweep_sort(b.keys, b.values, b.keys_alt, b.values_alt, n, true, b.sort_scratch, &b.control->status,
                      stream, nullptr, kpt);
        mark(3);
    } else {
        mark(1);
        mark(2);
        mark(3);
    }
    if (n >= 2) {
        const uint32_t nodes = n - 1;
        // values_alt (free after the sort) holds each node's range end.
        lt_karras_kernel<<<grid_for(nodes, kThreads, 1u << 30), kThreads, 0, stream>>>(
            b.keys, (int)n, b.left, b.right, b.parent, b.leaf_parent, b.cover, b.values_alt);
        mark(4);
        const uint32_t tiles = (nodes + kScanTile - 1) / kScanTile;
        lt_cover_scan_kernel<<<tiles, kScanThreads, 0, stream>>>(nodes, b.cover, cover_states, scan_counters,
                                                                  b.control);
        lt_flags_scan_kernel<<<tiles, kScanThreads, 0, stream>>>(nodes, b.left, b.cover, b.depth, b.wide, flag_states,
                                                                  scan_counters + 1, b.control);
        mark(5);
        // cover (free after the flags scan) lists the upper walks, keys_alt (free after the sort) the
        // even-depth nodes that cross a tile.
        lt_tile_kernel<<<(n + kAggTile - 1) / kAggTile, kAggTile, 0, stream>>>(
            n, b.node_capacity, b.sorted, b.left, b.right, b.parent, b.leaf_parent, b.values_alt, b.depth, b.wide,
            b.values, b.aggregates, b.cover, b.keys_alt, b.leaves, b.nodes, b.control);
        lt_aggregate_upper_kernel<true><<<1, kUpperOneCtaThreads, 0, stream>>>(
            b.sorted, b.left, b.right, b.parent, b.leaf_parent, b.counter, b.aggregates, b.cover, b.control);
        lt_aggregate_upper_kernel<false><<<grid_for(nodes, kThreads, sms * 8), kThreads, 0, stream>>>(
            b.sorted, b.left, b.right, b.parent, b.leaf_parent, b.counter, b.aggregates, b.cover, b.control);
        mark(6);
        lt_wide_upper_kernel<<<grid_for(nodes, kThreads, sms * 8), kThreads, 0, stream>>>(
            n, b.node_capacity, b.values, b.left, b.right, b.parent, b.keys_alt, b.wide, b.sorted, b.aggregates,
            b.leaves, b.nodes, b.control);
    } else {
        mark(4);
        mark(5);
        mark(6);
    }
    lt_finish_kernel<<<1, 1, 0, stream>>>(n, found, b.node_capacity, b.leaves, b.nodes, b.aggregates, b.header,
                                          b.state, b.control);
    mark(7);
    return cudaGetLastError();
}

uint32_t lt_kernel_launches(uint32_t n)
{
    // emit, Morton, the sort (one small-sort CTA, or four passes), the seven tree kernels from two
    // leaves (the upper aggregation's two variants both launch; one of them returns at once),
    // finish.
    if (n == 0) return 1;
    const uint32_t sort = n <= kSmallSortKeys ? 1u : 4u;
    return 2 + sort + (n >= 2 ? 7u : 0u) + 1;
}

}  // namespace cx
