// The scene build (scene.cuh): brick records (finalize), the canonical brick hash table, the
// brick occupancy bitmap, the light records in group light blocks, and the light tree.
#include <algorithm>
#include <cstring>
#include <vector>

#include "cx_device.cuh"
#include "lookback.cuh"
#include "radix_sort.cuh"
#include "scene.cuh"
#include "scene_device.cuh"

namespace cx {

namespace {

constexpr int kThreads = 256;
constexpr int kScanItems = 16;
constexpr uint32_t kScanTile = kThreads * kScanItems;

__host__ __device__ __forceinline__ uint32_t part1by2(uint32_t v)
{
    v &= 0x3FFu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}
__host__ __device__ __forceinline__ uint32_t morton30(uint32_t x, uint32_t y, uint32_t z)
{
    return part1by2(x) | (part1by2(y) << 1) | (part1by2(z) << 2);
}

// ---------------------------------------------------------------------------------------------
// Single-pass scan with a decoupled look-back over tiles of kScanTile u32 values (30-bit
// results). kMax: inclusive running maximum; else exclusive sum (the last tile writes the total).
template <bool kMax>
__global__ void __launch_bounds__(kThreads)
    lookback_scan_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t count,
                         uint32_t* states, uint32_t* tile_counter, uint32_t* total, uint32_t* status)
{
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_warp[kThreads / 32];
    __shared__ uint32_t s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t base = tile * kScanTile + threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t agg = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < count ? in[base + k] : 0u;
        agg = kMax ? max(agg, v[k]) : agg + v[k];
    }
    // Block-level exclusive scan of the per-thread aggregates.
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t inc = agg;
#pragma unroll
    for (uint32_t d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xFFFFFFFFu, inc, d);
        if (lane >= d) inc = kMax ? max(inc, o) : inc + o;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    uint32_t before = 0, tile_agg = 0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
        const uint32_t s = s_warp[w];
        if ((uint32_t)w < warp) before = kMax ? max(before, s) : before + s;
        tile_agg = kMax ? max(tile_agg, s) : tile_agg + s;
    }
    uint32_t excl_in_warp = __shfl_up_sync(0xFFFFFFFFu, inc, 1);
    if (lane == 0) excl_in_warp = 0;
    const uint32_t local = kMax ? max(before, excl_in_warp) : before + excl_in_warp;
    if (threadIdx.x < 32) {
        const uint32_t prefix = warp_lookback<kMax>(states, tile, tile_agg, status);
        if (threadIdx.x == 0) {
            s_prefix = prefix;
            if (!kMax && tile == gridDim.x - 1 && total) *total = prefix + tile_agg;
        }
    }
    __syncthreads();
    uint32_t run = kMax ? max(s_prefix, local) : s_prefix + local;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (kMax) {
            run = max(run, v[k]);
            if (base + k < count) out[base + k] = run;
        } else {
            if (base + k < count) out[base + k] = run;
            run += v[k];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Hash table.

__global__ void hash_home_kernel(const int32_t* __restrict__ keys, uint32_t n, uint32_t capacity,
                                 uint32_t* __restrict__ lo, uint32_t* __restrict__ hi, uint32_t* __restrict__ home)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t l, h;
    hash_fingerprint(keys[3 * i], keys[3 * i + 1], keys[3 * i + 2], l, h);
    lo[i] = l;
    hi[i] = h;
    home[i] = hash_home(l, capacity);
}

// v_k = home_k - k + n over the homes in sorted order (the input of the running maximum).
__global__ void hash_shift_kernel(const uint32_t* __restrict__ home_sorted, uint32_t n, uint32_t* __restrict__ v)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) v[k] = home_sorted[k] + n - k;
}

// pos_k = k + max_{j <= k} v_j - n: the first free slot at or after the home in (home, brick) order.
__global__ void hash_place_kernel(const uint32_t* __restrict__ running_max, const uint32_t* __restrict__ home_sorted,
                                  const uint32_t* __restrict__ order, const uint32_t* __restrict__ lo,
                                  const uint32_t* __restrict__ hi, uint32_t n, uint4* __restrict__ slots,
                                  uint32_t* max_probe)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const uint32_t pos = k + running_max[k] - n;
    const uint32_t b = order[k];
    slots[pos] = make_uint4(lo[b], hi[b], b, 0u);
    atomicMax(max_probe, pos - home_sorted[k]);
}

__global__ void bitmap_kernel(const int32_t* __restrict__ keys, uint32_t n, int32_t ox, int32_t oy, int32_t oz,
                              uint32_t gx, uint32_t gy, uint32_t* __restrict__ bitmap)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t c = (uint64_t)(uint32_t)(keys[3 * i] - ox) +
                       gx * ((uint64_t)(uint32_t)(keys[3 * i + 1] - oy) + (uint64_t)gy * (uint32_t)(keys[3 * i + 2] - oz));
    atomicOr(bitmap + (c >> 5), 1u << (c & 31));
}

// ---------------------------------------------------------------------------------------------
// Finalize (caelix_finalize.hlsl:110-340): one warp per brick, grid-stride. Lane l owns the 16
// voxels vi = l + 32k (x = l & 7, y = (l >> 3) + 4 (k & 1), z = k >> 1), so that every in-brick
// neighbour read (vi +- 1, 8, 64) is a conflict-free shared-memory read of consecutive values.
// The brick and its six neighbour faces are staged in shared memory (coalesced 16-byte loads
// where the face is contiguous); the record (274 words) is staged too and stored in 8-byte
// units, every word of it written (no clear of the record array is needed). Bricks whose values
// are all air or opaque take a bit-mask path (see the kernel).

struct FinalizeArgs
{
    const int32_t* keys;
    const uint16_t* voxels;
    uint32_t n;
    uint32_t group_shift;
    const uint4* slots;
    uint32_t capacity;
    uint32_t max_probe;
    uint32_t* records;
    const uint32_t* list;        // nullptr: every brick; else the bricks list[0 .. *list_count)
    const uint32_t* list_count;
};

constexpr uint32_t kFinalizeWarps = 8;
constexpr uint32_t kFinalizeStageWords = 256 + 6 * 32;  // the brick + six faces of 64 values
constexpr uint32_t kFinalizeRecordWords = 276;           // kRecordWords rounded up to 16 bytes
static_assert(kRecordWords <= kFinalizeRecordWords && kRecordWords % 2 == 0, "record staging");

// The 16 bits of a coarse cell's 4 x 4 voxels (x = 4 cx .. 4 cx + 3, 4 rows) in one ballot of
// lanes x + 8 (y & 3): bit (x & 3) + 4 (y & 3).
__device__ __forceinline__ uint32_t coarse_rows(uint32_t ballot, uint32_t cx)
{
    const uint32_t b = ballot >> (4 * cx);
    return (b & 0xFu) | ((b >> 4) & 0xF0u) | ((b >> 8) & 0xF00u) | ((b >> 12) & 0xF000u);
}

// Bit 15 of each 16-bit half of a pair of values (one u32): the value is opaque (kEnc: the block
// encoding; packed values are opaque on bit 14 or 15, block-ID values on bit 15).
template <uint32_t kEnc>
__device__ __forceinline__ uint32_t opaque_top(uint32_t w)
{
    return kEnc == kEncodingPacked ? (w | (w << 1)) : w;
}

// Whether a pair of values (one u32) / a value holds a non-opaque value other than air.
template <uint32_t kEnc>
__device__ __forceinline__ bool impure(uint32_t w)
{
    const uint32_t clear = ~opaque_top<kEnc>(w) & 0x80008000u;
    const uint32_t nonzero = ((w & 0x7FFF7FFFu) + 0x7FFF7FFFu) & 0x80008000u;
    return (clear & nonzero) != 0;
}
template <uint32_t kEnc>
__device__ __forceinline__ bool impure(const uint4& v)
{
    return impure<kEnc>(v.x) || impure<kEnc>(v.y) || impure<kEnc>(v.z) || impure<kEnc>(v.w);
}
template <uint32_t kEnc>
__device__ __forceinline__ bool impure16(uint32_t v)
{
    return !(v & encoding_of(kEnc).opaque_mask) && v != 0;
}

// The opaque bits of 8 values (bit j = value j).
template <uint32_t kEnc>
__device__ __forceinline__ uint32_t opaque_byte(const uint4& v)
{
    const uint32_t w[4] = {opaque_top<kEnc>(v.x), opaque_top<kEnc>(v.y), opaque_top<kEnc>(v.z), opaque_top<kEnc>(v.w)};
    uint32_t b = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) b |= (((w[i] >> 15) & 1u) | ((w[i] >> 30) & 2u)) << (2 * i);
    return b;
}

// The light bits of 8 values (bit j = value j's material code is in the light code set).
template <uint32_t kEnc>
__device__ __forceinline__ uint32_t light_byte(const uint4& v, const uint32_t* __restrict__ codes)
{
    constexpr Encoding E = encoding_of(kEnc);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    uint32_t b = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t c = material_code((w[i >> 1] >> (16 * (i & 1))) & 0xFFFFu, E);
        b |= ((__ldg(codes + (c >> 5)) >> (c & 31)) & 1u) << i;
    }
    return b;
}

// Bits 0 .. 3 of n to bits 0, 8, 16, 24 (one per row of a mask word).
__device__ __forceinline__ uint32_t spread_rows(uint32_t n)
{
    return (n & 1u) | ((n & 2u) << 7) | ((n & 4u) << 14) | ((n & 8u) << 21);
}

// A brick and its six neighbour faces in registers (one warp): lane l holds values 8l .. 8l + 7
// (v0) and 256 + 8l .. (v1); the y and z faces one row of 8 values each (fv: row lane & 7 of face
// 2 + (lane >> 3): rows (x, 0 / 7, z) of the +-y neighbours, rows (x, y, 0 / 7) of the +-z ones);
// the x faces two values each (xf: (0, y, z) of the +x neighbour at y + 8 z = lane and lane + 32,
// then (7, y, z) of the -x one). Absent neighbours read as air.
struct BrickFaces
{
    uint4 v0, v1, fv;
    uint32_t xf[4];  // +x lane, -x lane, +x lane + 32, -x lane + 32
};

__device__ __forceinline__ BrickFaces load_brick_faces(const int32_t* __restrict__ keys,
                                                       const uint16_t* __restrict__ voxels, const uint4* slots,
                                                       uint32_t capacity, uint32_t max_probe, uint32_t b, uint32_t lane)
{
    BrickFaces f;
    const int32_t bx = __ldg(keys + 3ull * b), by = __ldg(keys + 3ull * b + 1), bz = __ldg(keys + 3ull * b + 2);
    const uint4* own = reinterpret_cast<const uint4*>(voxels + 512ull * b);
    f.v0 = __ldg(own + lane);
    f.v1 = __ldg(own + 32 + lane);
    uint32_t my_nbr = 0xFFFFFFFFu;
    if (lane < 6) {
        const int dx = lane == 0 ? 1 : (lane == 1 ? -1 : 0);
        const int dy = lane == 2 ? 1 : (lane == 3 ? -1 : 0);
        const int dz = lane == 4 ? 1 : (lane == 5 ? -1 : 0);
        my_nbr = hash_lookup(slots, capacity, max_probe, bx + dx, by + dy, bz + dz);
    }
    const uint32_t fj = lane & 7u, fg = lane >> 3;
    const uint32_t nx_pos = __shfl_sync(0xFFFFFFFFu, my_nbr, 0);
    const uint32_t nx_neg = __shfl_sync(0xFFFFFFFFu, my_nbr, 1);
    const uint32_t nf = __shfl_sync(0xFFFFFFFFu, my_nbr, 2 + fg);
    const uint32_t fq = fg == 0 ? 8 * fj : (fg == 1 ? 8 * fj + 7 : (fg == 2 ? fj : 56 + fj));
    f.fv = nf == 0xFFFFFFFFu ? make_uint4(0, 0, 0, 0) : __ldg(reinterpret_cast<const uint4*>(voxels + 512ull * nf) + fq);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const uint32_t i = lane + 32 * h;
        f.xf[2 * h] = nx_pos == 0xFFFFFFFFu ? 0u : (uint32_t)voxels[512ull * nx_pos + 8 * i];
        f.xf[2 * h + 1] = nx_neg == 0xFFFFFFFFu ? 0u : (uint32_t)voxels[512ull * nx_neg + 7 + 8 * i];
    }
    return f;
}

// Opaque masks of a brick and of its six neighbours of every voxel: lane k < 16 gets word k (bit
// x + 8 (y & 3) for the rows y = 4 (k & 1) + 0 .. 3 at z = k >> 1) of the brick's opaque voxels
// (o) and of the voxels whose neighbour in direction d is opaque (n[d]: +x, -x, +y, -y, +z, -z).
struct OpaqueMasks
{
    uint32_t o, n[6];
};

// The mask words of per-lane bytes (b0: values 8 lane .. 8 lane + 7, b1: 256 + 8 lane ..): lane
// k < 16 gets word k (bit j = value 32 k + j), the lanes above get the bytes of lanes k - 16 (no use).
__device__ __forceinline__ uint32_t mask_word(uint32_t b0, uint32_t b1, uint32_t lane)
{
    uint32_t o = 0;
#pragma unroll
    for (uint32_t i = 0; i < 4; ++i) {
        const uint32_t src = (4 * lane + i) & 31u;
        const uint32_t t0 = __shfl_sync(0xFFFFFFFFu, b0, src), t1 = __shfl_sync(0xFFFFFFFFu, b1, src);
        o |= (lane < 8 ? t0 : t1) << (8 * i);
    }
    return o;
}

template <uint32_t kEnc>
__device__ __forceinline__ OpaqueMasks opaque_masks(const BrickFaces& f, uint32_t lane)
{
    constexpr uint32_t kOpaque = encoding_of(kEnc).opaque_mask;
    const uint32_t kz = (lane >> 1) & 7u, kyh = lane & 1u;
    const uint32_t o = mask_word(opaque_byte<kEnc>(f.v0), opaque_byte<kEnc>(f.v1), lane);
    const uint32_t fxp0 = __ballot_sync(0xFFFFFFFFu, f.xf[0] & kOpaque);
    const uint32_t fxn0 = __ballot_sync(0xFFFFFFFFu, f.xf[1] & kOpaque);
    const uint32_t fxp1 = __ballot_sync(0xFFFFFFFFu, f.xf[2] & kOpaque);
    const uint32_t fxn1 = __ballot_sync(0xFFFFFFFFu, f.xf[3] & kOpaque);
    const uint32_t fb = opaque_byte<kEnc>(f.fv);
    const uint32_t fyp = __shfl_sync(0xFFFFFFFFu, fb, kz), fyn = __shfl_sync(0xFFFFFFFFu, fb, 8 + kz);
    uint32_t fzp = 0, fzn = 0;
#pragma unroll
    for (uint32_t i = 0; i < 4; ++i) {
        fzp |= __shfl_sync(0xFFFFFFFFu, fb, 16 + 4 * kyh + i) << (8 * i);
        fzn |= __shfl_sync(0xFFFFFFFFu, fb, 24 + 4 * kyh + i) << (8 * i);
    }
    const uint32_t o_next = __shfl_down_sync(0xFFFFFFFFu, o, 1), o_prev = __shfl_up_sync(0xFFFFFFFFu, o, 1);
    const uint32_t o_up = __shfl_down_sync(0xFFFFFFFFu, o, 2), o_down = __shfl_up_sync(0xFFFFFFFFu, o, 2);
    const uint32_t xs = (4 * lane) & 31u;
    const uint32_t nib_p = ((lane < 8 ? fxp0 : fxp1) >> xs) & 0xFu;
    const uint32_t nib_n = ((lane < 8 ? fxn0 : fxn1) >> xs) & 0xFu;
    OpaqueMasks m;
    m.o = lane < 16 ? o : 0u;
    m.n[0] = ((o >> 1) & 0x7F7F7F7Fu) | (spread_rows(nib_p) << 7);
    m.n[1] = ((o << 1) & 0xFEFEFEFEu) | spread_rows(nib_n);
    m.n[2] = (o >> 8) | ((kyh == 0 ? (o_next & 0xFFu) : fyp) << 24);
    m.n[3] = (o << 8) | (kyh == 1 ? (o_prev >> 24) : fyn);
    m.n[4] = kz < 7 ? o_up : fzp;
    m.n[5] = kz > 0 ? o_down : fzn;
    return m;
}

template <uint32_t kEnc>
__global__ void __launch_bounds__(kFinalizeWarps * 32, 6) finalize_kernel(const FinalizeArgs a)
{
    constexpr Encoding E = encoding_of(kEnc);
    __shared__ __align__(16) uint32_t s_stage[kFinalizeWarps][kFinalizeStageWords];
    __shared__ __align__(16) uint32_t s_record[kFinalizeWarps][kFinalizeRecordWords];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint16_t* vox = reinterpret_cast<uint16_t*>(s_stage[warp]);  // [512] then faces [6][64]
    uint16_t* rec16 = reinterpret_cast<uint16_t*>(s_record[warp]);
    const uint32_t x = lane & 7u, ylo = lane >> 3;
    const uint32_t fj = lane & 7u, fg = lane >> 3;  // face loads: row fj of face 2 + fg
    const uint32_t items = a.list ? *a.list_count : a.n;
    for (uint32_t item = blockIdx.x * kFinalizeWarps + warp; item < items; item += gridDim.x * kFinalizeWarps) {
        const uint32_t b = a.list ? __ldg(a.list + item) : item;
        const int32_t bx = __ldg(a.keys + 3ull * b), by = __ldg(a.keys + 3ull * b + 1), bz = __ldg(a.keys + 3ull * b + 2);
        const BrickFaces bf = load_brick_faces(a.keys, a.voxels, a.slots, a.capacity, a.max_probe, b, lane);
        const uint4 v0 = bf.v0, v1 = bf.v1, fv = bf.fv;
        const uint32_t* xf = bf.xf;
        __syncwarp();  // the previous brick's reads of the staging are done
        reinterpret_cast<uint4*>(vox)[lane] = v0;
        reinterpret_cast<uint4*>(vox)[32 + lane] = v1;
        reinterpret_cast<uint4*>(vox + 512 + 64 * (2 + fg))[fj] = fv;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            vox[512 + lane + 32 * h] = (uint16_t)xf[2 * h];
            vox[512 + 64 + lane + 32 * h] = (uint16_t)xf[2 * h + 1];
        }
        __syncwarp();
        // A clean brick (every value of it and of its six neighbour faces air or opaque) keeps
        // its raw values as the payload, and a voxel of it is occupied iff it is opaque and not
        // all six of its neighbours are: shifted masks of the opaque voxels. Other bricks take
        // the per-voxel rules.
        const bool dirty =
            __any_sync(0xFFFFFFFFu, impure<kEnc>(v0) || impure<kEnc>(v1) || impure<kEnc>(fv) || impure16<kEnc>(xf[0]) ||
                                        impure16<kEnc>(xf[1]) || impure16<kEnc>(xf[2]) || impure16<kEnc>(xf[3]));
        // Lane k < 16 ends with word k of the occupied voxels: bit x + 8 (y & 3) for the rows
        // y = 4 (k & 1) + (0 .. 3) at z = k >> 1.
        uint32_t my_occ = 0;
        const uint32_t kz = (lane >> 1) & 7u, kyh = lane & 1u;
        if (!dirty) {
            const OpaqueMasks m = opaque_masks<kEnc>(bf, lane);
            my_occ = m.o & ~(m.n[0] & m.n[1] & m.n[2] & m.n[3] & m.n[4] & m.n[5]);
        } else {
#pragma unroll 2
            for (uint32_t k = 0; k < 16; ++k) {
                const uint32_t y = ylo + 4 * (k & 1), z = k >> 1;
                const uint32_t vi = lane + 32 * k;
                const uint32_t raw = vox[vi];
                const uint32_t v = material_code(raw, E);
                uint32_t nb[6];
                nb[0] = vox[x < 7 ? vi + 1 : 512 + 0 * 64 + y + 8 * z];
                nb[1] = vox[x > 0 ? vi - 1 : 512 + 1 * 64 + y + 8 * z];
                nb[2] = vox[y < 7 ? vi + 8 : 512 + 2 * 64 + x + 8 * z];
                nb[3] = vox[y > 0 ? vi - 8 : 512 + 3 * 64 + x + 8 * z];
                nb[4] = vox[z < 7 ? vi + 64 : 512 + 4 * 64 + x + 8 * y];
                nb[5] = vox[z > 0 ? vi - 64 : 512 + 5 * 64 + x + 8 * y];
                uint32_t opaque_count = 0, faces = 0;
#pragma unroll
                for (int d = 0; d < 6; ++d) {
                    const bool nop = (nb[d] & E.opaque_mask) != 0;
                    opaque_count += nop ? 1u : 0u;
                    if (!nop && (nb[d] & E.id_mask) != v) faces |= 1u << d;
                }
                const uint32_t result = (v & E.opaque_mask) ? v : (v | (faces << E.face_shift));
                const bool iface = (v & E.opaque_mask) != 0 || faces != 0;
                rec16[2 * kRecordPayloadWord + vi] = (uint16_t)result;
                const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, opaque_count < 6 && result != 0 && iface);
                if (lane == k) my_occ = ballot;
            }
        }
        // Occupancy word w = 2 cell + half of coarse cell c = (x >> 2) + 2 (y >> 2) + 4 (z >> 2),
        // bit (x & 3) + 4 (y & 3) + 16 (z & 3) - 32 half: the lanes of even z join the next z.
        const uint32_t c0 = coarse_rows(my_occ, 0), c1 = coarse_rows(my_occ, 1);
        const uint32_t c0_next = __shfl_down_sync(0xFFFFFFFFu, c0, 2), c1_next = __shfl_down_sync(0xFFFFFFFFu, c1, 2);
        const uint32_t cell_yz = 2 * kyh + 4 * (kz >> 2), half = (kz & 3) >> 1;
        if (lane < 16 && (kz & 1) == 0) {
            s_record[warp][2 + 2 * cell_yz + half] = c0 | (c0_next << 16);
            s_record[warp][2 + 2 * (cell_yz + 1) + half] = c1 | (c1_next << 16);
        }
        const uint32_t row_any = ((my_occ & 0xFFu) ? 1u : 0u) | ((my_occ & 0xFF00u) ? 2u : 0u) |
                                 ((my_occ & 0xFF0000u) ? 4u : 0u) | ((my_occ & 0xFF000000u) ? 8u : 0u);
        const uint32_t xmask = __reduce_or_sync(0xFFFFFFFFu, (my_occ | (my_occ >> 8) | (my_occ >> 16) | (my_occ >> 24)) & 0xFFu);
        const uint32_t ymask = __reduce_or_sync(0xFFFFFFFFu, row_any << (4 * kyh));
        const uint32_t zmask = __reduce_or_sync(0xFFFFFFFFu, (my_occ ? 1u : 0u) << kz);
        const uint32_t coarse = __reduce_or_sync(0xFFFFFFFFu, ((c0 ? 1u : 0u) << cell_yz) | ((c1 ? 1u : 0u) << (cell_yz + 1)));
        if (lane == 0) {
            uint32_t bounds = 0;
            if (xmask) {
                const uint32_t x0 = __ffs(xmask) - 1, y0 = __ffs(ymask) - 1, z0 = __ffs(zmask) - 1;
                const uint32_t x1 = 31 - __clz(xmask), y1 = 31 - __clz(ymask), z1 = 31 - __clz(zmask);
                bounds = x0 | (y0 << 3) | (z0 << 6) | (x1 << 9) | (y1 << 12) | (z1 << 15);
            }
            const uint32_t gm = (1u << a.group_shift) - 1u;
            const uint32_t pos = ((uint32_t)bx & gm) | (((uint32_t)by & gm) << a.group_shift) |
                                 (((uint32_t)bz & gm) << (2 * a.group_shift));
            s_record[warp][0] = (pos & 0xFFFFu) | (coarse << 16);
            s_record[warp][1] = bounds;
        }
        __syncwarp();
        // The record: header words (0 .. 17) from the staging; the payload from the staging, or
        // the raw values of a clean brick.
        uint2* dst = reinterpret_cast<uint2*>(a.records + (uint64_t)b * kRecordWords);
        const uint2* src = reinterpret_cast<const uint2*>(s_record[warp]);
        if (lane < kRecordPayloadWord / 2) dst[lane] = src[lane];
        if (!dirty) {
            dst[kRecordPayloadWord / 2 + 2 * lane] = make_uint2(v0.x, v0.y);
            dst[kRecordPayloadWord / 2 + 2 * lane + 1] = make_uint2(v0.z, v0.w);
            dst[kRecordPayloadWord / 2 + 64 + 2 * lane] = make_uint2(v1.x, v1.y);
            dst[kRecordPayloadWord / 2 + 64 + 2 * lane + 1] = make_uint2(v1.z, v1.w);
        } else {
#pragma unroll
            for (uint32_t i = 0; i < 4; ++i)
                dst[kRecordPayloadWord / 2 + lane + 32 * i] = src[kRecordPayloadWord / 2 + lane + 32 * i];
        }
    }
}

// ---------------------------------------------------------------------------------------------
// Light records (caelix_light_tree_build.hlsl:93-285): a light voxel is a voxel whose material code
// is in the light code set (LtOpenFaces) in a brick with emitter power above 0; its open faces
// (the neighbour across is not opaque, an absent brick being air) are the entries; a face's
// weight is the luminance of its voxel's emission times the brick's power.

struct LightArgs
{
    const int32_t* keys;
    const uint16_t* voxels;
    const float* power;
    uint32_t n;
    uint32_t group_shift;
    uint32_t groups[3];
    int32_t origin[3];
    const uint4* slots;
    uint32_t capacity;
    uint32_t max_probe;
    const float4* materials;
    const uint32_t* light_codes;
};

// A brick with power above 0 and a voxel whose code is a light code is a light brick. A warp takes
// 32 consecutive bricks: each lane reads one brick's power, then the warp reads the values of each
// brick with power (two 16-byte words per lane) and appends the light bricks with one atomic.
template <uint32_t kEnc>
__global__ void light_collect_kernel(const LightArgs a, uint32_t* counter, uint32_t* lkeys, uint32_t* lbricks)
{
    const uint32_t first = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32u;
    const uint32_t lane = threadIdx.x & 31u;
    if (first >= a.n) return;
    const uint32_t i = first + lane;
    uint32_t todo = __ballot_sync(0xFFFFFFFFu, i < a.n && a.power[i] > 0.0f);
    uint32_t found = 0;
    while (todo) {
        const uint32_t l = (uint32_t)(__ffs(todo) - 1);
        todo &= todo - 1u;
        const uint4* vox = reinterpret_cast<const uint4*>(a.voxels + 512ull * (first + l));
        const uint32_t bits = light_byte<kEnc>(__ldg(vox + lane), a.light_codes) |
                              light_byte<kEnc>(__ldg(vox + 32 + lane), a.light_codes);
        if (__any_sync(0xFFFFFFFFu, bits != 0u)) found |= 1u << l;
    }
    if (!found) return;
    uint32_t base = 0;
    if (lane == 0) base = atomicAdd(counter, (uint32_t)__popc(found));
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (!((found >> lane) & 1u)) return;
    const uint32_t gs = a.group_shift, gm = (1u << gs) - 1u;
    const int32_t kx = a.keys[3 * i], ky = a.keys[3 * i + 1], kz = a.keys[3 * i + 2];
    const uint32_t bx = (uint32_t)(kx - a.origin[0]), by = (uint32_t)(ky - a.origin[1]), bz = (uint32_t)(kz - a.origin[2]);
    const uint32_t g = (bx >> gs) + a.groups[0] * ((by >> gs) + a.groups[1] * (bz >> gs));
    const uint32_t slot = base + (uint32_t)__popc(found & lanemask_lt());
    lkeys[slot] = (g << (3 * gs)) | morton30(bx & gm, by & gm, bz & gm);
    lbricks[slot] = i;
}

// The open faces of the light voxels of light brick b (a face is open when the neighbour across it
// is not opaque, an absent brick being air), per family f (+x, -x, +y, -y, +z, -z) in the word
// layout of opaque_masks: lane k < 16 gets word k of each family.
template <uint32_t kEnc>
__device__ __forceinline__ void light_open_masks(const BrickFaces& f, const uint32_t* __restrict__ codes, uint32_t lane,
                                                 uint32_t open[6])
{
    const OpaqueMasks m = opaque_masks<kEnc>(f, lane);
    const uint32_t word = mask_word(light_byte<kEnc>(f.v0, codes), light_byte<kEnc>(f.v1, codes), lane);
    const uint32_t light = lane < 16 ? word : 0u;
#pragma unroll
    for (int d = 0; d < 6; ++d) open[d] = light & ~m.n[d];
}

// The weight of a light face of value v in a brick of power P: LtLuminance of its material emission
// times P (each channel times P first).
template <uint32_t kEnc>
__device__ __forceinline__ float light_weight(const float4* __restrict__ materials, uint32_t v, float P)
{
    const float4 e = __ldg(materials + 2ull * material_code(v, encoding_of(kEnc)) + 1);
    return (e.x * P) * 0.2126f + (e.y * P) * 0.7152f + (e.z * P) * 0.0722f;
}

constexpr uint32_t kLightWarps = 4;

// The previous build's light records, for a rebuild over the same bricks: a light brick that is
// not marked with `epoch` (its values, its neighbours' and its power unchanged) keeps its record,
// copied from the previous heap (prev_unit[b]: its first 16-byte unit there, kNone: none).
struct LightReuse
{
    const uint32_t* prev_unit;  // nullptr: every record is recomputed
    const uint32_t* prev_heap;
    const uint32_t* marks;
    uint32_t epoch;
};

__device__ __forceinline__ uint32_t reused_unit(const LightReuse& r, uint32_t b)
{
    if (!r.prev_unit) return kNone;
    const uint32_t u = __ldg(r.prev_unit + b);
    return (u != kNone && __ldg(r.marks + b) != r.epoch) ? u : kNone;
}

// Warp per light brick (sorted order): the family counts and the record's units (of a reused
// record, from its header).
template <uint32_t kEnc>
__global__ void __launch_bounds__(kLightWarps * 32) light_measure_kernel(const LightArgs a,
                                                                        const uint32_t* __restrict__ lbricks,
                                                                        uint32_t m, uint32_t* __restrict__ counts6,
                                                                        uint32_t* __restrict__ units,
                                                                        const LightReuse reuse)
{
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    if (k >= m) return;
    const uint32_t pu = reused_unit(reuse, lbricks[k]);
    if (pu != kNone) {
        if (lane < 6) {
            const uint32_t* hdr = reuse.prev_heap + 4ull * pu;
            const uint32_t word = lane < 3 ? hdr[10] : hdr[11];
            counts6[6 * k + lane] = (word >> (kFamilyCountBits * (lane % 3))) & kFamilyCountMask;
            if (lane == 0) units[k] = 3 + (4 * hdr[9] + 15) / 16;
        }
        return;
    }
    const BrickFaces bf = load_brick_faces(a.keys, a.voxels, a.slots, a.capacity, a.max_probe, lbricks[k], lane);
    uint32_t open[6];
    light_open_masks<kEnc>(bf, a.light_codes, lane, open);
    uint32_t total = 0;
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, __popc(open[f]));
        if (lane == 0) counts6[6 * k + f] = c;
        total += c;
    }
    if (lane == 0) units[k] = 3 + (4 * total + 15) / 16;
}

// Per light: its block's extra units (header + index entries) when it starts its group.
__global__ void light_group_kernel(const uint32_t* __restrict__ lkeys, uint32_t m, uint32_t gshift,
                                   const uint32_t* __restrict__ units, uint32_t* __restrict__ total_units,
                                   uint32_t* __restrict__ group_start, uint32_t* __restrict__ group_end)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m) return;
    const uint32_t g = lkeys[k] >> (3 * gshift);
    // The group's first light (binary search for the first key of group g).
    uint32_t lo = 0, hi = k;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if ((lkeys[mid] >> (3 * gshift)) < g) lo = mid + 1;
        else hi = mid;
    }
    const uint32_t start = lo;
    group_start[k] = start;
    uint32_t extra = 0;
    if (k == start) {
        uint32_t a = k, b = m;
        while (a < b) {
            const uint32_t mid = (a + b) >> 1;
            if ((lkeys[mid] >> (3 * gshift)) <= g) a = mid + 1;
            else b = mid;
        }
        extra = 1 + (a - k);
        group_end[k] = a;  // the end of the group's lights, for the group's first light
    }
    total_units[k] = units[k] + extra;
}

struct LightWriteArgs
{
    LightArgs a;
    const uint32_t* lkeys;
    const uint32_t* lbricks;
    uint32_t m;
    const uint32_t* counts6;
    const uint32_t* units;
    const uint32_t* offsets;  // exclusive scan of the total units
    const uint32_t* group_start;
    const uint32_t* group_end;  // at a group's first light: the end of its lights
    uint32_t total;  // all units
    uint32_t* heap;
    uint32_t* group_rows;
    BrickLightRecord* headers;
    uint32_t* light_group;
    uint32_t* light_entry;
    uint32_t* light_brick;
    LightReuse reuse;
    uint32_t* unit_of_brick;  // out: the first unit of every light brick's record
};

template <uint32_t kEnc>
__global__ void __launch_bounds__(kLightWarps * 32) light_write_kernel(const LightWriteArgs w)
{
    __shared__ __align__(16) uint4 s_vox[kLightWarps][64];
    const uint32_t k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (k >= w.m) return;
    const LightArgs& a = w.a;
    const uint32_t b = w.lbricks[k];
    const uint32_t gs = a.group_shift;
    const uint32_t g = w.lkeys[k] >> (3 * gs);
    const uint32_t s = w.group_start[k];
    // The group's light count: the next group's start, or the end.
    const uint32_t block = 1 + w.offsets[s];
    const uint32_t count = w.group_end[s] - s;
    const uint32_t rec_unit = 1 + w.offsets[k] + (k == s ? 1 + count : 0);
    uint32_t* rec = w.heap + 4ull * rec_unit;
    BrickLightRecord h;
    const uint32_t pu = reused_unit(w.reuse, b);
    if (pu != kNone) {
        // The previous build's record, copied whole (header, entries, padding of its last unit).
        const uint4* src = reinterpret_cast<const uint4*>(w.reuse.prev_heap) + pu;
        uint4* dst = reinterpret_cast<uint4*>(rec);
        for (uint32_t i = lane; i < w.units[k]; i += 32) dst[i] = src[i];
        if (lane == 0) {
            uint4* hp = reinterpret_cast<uint4*>(&h);
            hp[0] = src[0];
            hp[1] = src[1];
            hp[2] = src[2];
        }
    } else {
        const BrickFaces bf = load_brick_faces(a.keys, a.voxels, a.slots, a.capacity, a.max_probe, b, lane);
        s_vox[warp][lane] = bf.v0;
        s_vox[warp][32 + lane] = bf.v1;
        __syncwarp();
        const uint16_t* vox = reinterpret_cast<const uint16_t*>(s_vox[warp]);
        uint32_t open[6];
        light_open_masks<kEnc>(bf, a.light_codes, lane, open);
        const float P = a.power[b];
        // Entries per family in voxel order: lane k writes the voxels of word k (32k + bit) after the
        // family's entries of the lanes before it.
        uint32_t fam_count[6];
        uint32_t written = 0;
        float sums[6];
#pragma unroll
        for (int f = 0; f < 6; ++f) {
            const uint32_t c = __popc(open[f]);
            const uint32_t inc = warp_inclusive_sum(c);
            fam_count[f] = __shfl_sync(0xFFFFFFFFu, inc, 31);
            uint32_t* out = rec + 12 + written + (inc - c);
            uint32_t bits = open[f];
            while (bits) {
                const uint32_t bit = __ffs(bits) - 1;
                bits &= bits - 1;
                const uint32_t vi = 32 * lane + bit;
                *out++ = vi | ((uint32_t)vox[vi] << 16);
            }
            written += fam_count[f];
            // The face sum as sixteen-voxel partial sums (voxels 16l .. 16l + 15 in lane l, each open
            // face's weight added in voxel order), then a tree over the lanes.
            const uint32_t word = __shfl_sync(0xFFFFFFFFu, open[f], lane >> 1);
            uint32_t half = (word >> (16 * (lane & 1))) & 0xFFFFu;
            float part = 0.0f;
            while (half) {
                const uint32_t bit = __ffs(half) - 1;
                half &= half - 1;
                part += light_weight<kEnc>(a.materials, vox[16 * lane + bit], P);
            }
            sums[f] = part;
        }
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1)
#pragma unroll
            for (int f = 0; f < 6; ++f) sums[f] += __shfl_down_sync(0xFFFFFFFFu, sums[f], off);
        // The tight box of the voxels with an open face.
        const uint32_t any = open[0] | open[1] | open[2] | open[3] | open[4] | open[5];
        const uint32_t kz = (lane >> 1) & 7u, kyh = lane & 1u;
        const uint32_t rows = ((any & 0xFFu) ? 1u : 0u) | ((any & 0xFF00u) ? 2u : 0u) | ((any & 0xFF0000u) ? 4u : 0u) |
                              ((any & 0xFF000000u) ? 8u : 0u);
        const uint32_t xm = __reduce_or_sync(0xFFFFFFFFu, (any | (any >> 8) | (any >> 16) | (any >> 24)) & 0xFFu);
        const uint32_t ym = __reduce_or_sync(0xFFFFFFFFu, rows << (4 * kyh));
        const uint32_t zm = __reduce_or_sync(0xFFFFFFFFu, (any ? 1u : 0u) << kz);
        uint32_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        if (xm) {
            lo[0] = __ffs(xm) - 1;
            lo[1] = __ffs(ym) - 1;
            lo[2] = __ffs(zm) - 1;
            hi[0] = 32 - __clz(xm);
            hi[1] = 32 - __clz(ym);
            hi[2] = 32 - __clz(zm);
        }
        // Zero padding of the record's last unit.
        const uint32_t padded = (w.units[k] - 3) * 4;
        for (uint32_t e = written + lane; e < padded; e += 32) rec[12 + e] = 0u;
        if (lane == 0) {
            // Group-local positions: the grid origin is a multiple of the group edge, so the low
            // bits of a key (two's complement for a negative key) are its position in its group.
            const uint32_t gm = (1u << gs) - 1u;
            const int32_t bx = a.keys[3 * b], by = a.keys[3 * b + 1], bz = a.keys[3 * b + 2];
            const uint32_t org[3] = {((uint32_t)bx & gm) * 8, ((uint32_t)by & gm) * 8, ((uint32_t)bz & gm) * 8};
            const uint32_t pos = ((uint32_t)bx & gm) | (((uint32_t)by & gm) << gs) | (((uint32_t)bz & gm) << (2 * gs));
            for (int f = 0; f < 6; ++f) h.face[f] = sums[f];
            h.box_lo = (org[0] + lo[0]) | ((org[1] + lo[1]) << 10) | ((org[2] + lo[2]) << 20);
            h.box_hi = (org[0] + hi[0]) | ((org[1] + hi[1]) << 10) | ((org[2] + hi[2]) << 20);
            h.pos = pos;
            h.entry_count = written;
            h.counts_lo = fam_count[0] | (fam_count[1] << 10) | (fam_count[2] << 20);
            h.counts_hi = fam_count[3] | (fam_count[4] << 10) | (fam_count[5] << 20);
            const uint4* hp = reinterpret_cast<const uint4*>(&h);
            uint4* r4 = reinterpret_cast<uint4*>(rec);
            r4[0] = hp[0];
            r4[1] = hp[1];
            r4[2] = hp[2];
        }
    }
    if (lane == 0) {
        w.headers[k] = h;
        w.unit_of_brick[b] = rec_unit;
        const uint32_t entry = k - s;
        uint32_t* ie = w.heap + 4ull * (block + 1 + entry);
        ie[0] = h.pos;
        ie[1] = b;
        ie[2] = rec_unit - block;
        ie[3] = k;
        w.light_group[k] = g;
        w.light_entry[k] = entry;
        w.light_brick[k] = b;
        atomicAdd(w.group_rows + 8ull * g + 6, h.entry_count);  // the group's light faces
        if (k == s) {
            uint32_t* bh = w.heap + 4ull * block;
            bh[0] = count;
            bh[1] = bh[2] = bh[3] = 0;
            const uint32_t end = count + s < w.m ? w.offsets[s + count] : w.total;
            uint32_t* row = w.group_rows + 8ull * g;
            row[0] = block;
            row[1] = end - w.offsets[s];
            row[2] = 0;
            row[3] = 0;
            row[4] = 0;
            row[5] = count;
            row[7] = 0;
        }
    }
}

// ---- group generations ----
// GroupLightRow::generation (lib/src/light/light_tree_layout.h:217-254, LtNextLife / LtNextVersion
// in shaders/common/caelix_light_tree_layout.hlsl:126-135): the group's life in the high 16 bits
// (the next life when the group is released: it had bricks and has none), the version of its
// light block in the low 16 (the next version when the block is rebuilt). A full build rebuilds
// every block that has or had light bricks; an edit flush the blocks of the groups holding a
// refinalized brick that is or was a light brick (the reference's kLtGpuLightChanged: a finalized
// brick whose old or new light face count is not 0). A new grid (origin, group grid or group edge
// changed: every group index names another place) starts every group at a life above all earlier
// ones, version 0. A light brick reference (group, entry, generation) stays valid while the row's
// generation is unchanged.
constexpr uint32_t kGroupLitBefore = 1u;       // the previous build's block had light bricks
constexpr uint32_t kGroupOccupied = 2u;        // this build: the group has bricks
constexpr uint32_t kGroupOccupiedBefore = 4u;  // the previous full build: the group had bricks
constexpr uint32_t kGroupTouched = 8u;         // this edit flush: a refinalized brick is or was a light brick

__device__ __forceinline__ uint32_t brick_group(const int32_t* keys, uint32_t i, const int32_t origin[3],
                                                const uint32_t groups[3], uint32_t gs)
{
    const uint32_t bx = (uint32_t)(keys[3 * i] - origin[0]), by = (uint32_t)(keys[3 * i + 1] - origin[1]),
                   bz = (uint32_t)(keys[3 * i + 2] - origin[2]);
    return (bx >> gs) + groups[0] * ((by >> gs) + groups[1] * (bz >> gs));
}

struct GroupGrid
{
    int32_t origin[3];
    uint32_t groups[3];
    uint32_t shift;
};

__global__ void group_occupancy_kernel(const int32_t* __restrict__ keys, uint32_t n, const GroupGrid gg,
                                       uint32_t* __restrict__ flags)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t g = brick_group(keys, i, gg.origin, gg.groups, gg.shift);
    if (!(flags[g] & kGroupOccupied)) atomicOr(&flags[g], kGroupOccupied);
}

__global__ void group_touch_kernel(const int32_t* __restrict__ keys, uint32_t n, const uint32_t* __restrict__ marks,
                                   uint32_t epoch, const uint32_t* __restrict__ unit_now,
                                   const uint32_t* __restrict__ unit_before, const GroupGrid gg, uint32_t* __restrict__ flags)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || marks[i] != epoch) return;
    if (unit_now[i] == kNone && (!unit_before || unit_before[i] == kNone)) return;
    atomicOr(&flags[brick_group(keys, i, gg.origin, gg.groups, gg.shift)], kGroupTouched);
}

// full: a full build (else an edit flush); fresh: a new grid, every group starting at fresh_gen.
__global__ void group_generation_kernel(uint32_t count, uint32_t* __restrict__ rows, uint32_t* __restrict__ gens,
                                        uint32_t* __restrict__ flags, uint32_t full, uint32_t fresh, uint32_t fresh_gen)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= count) return;
    const uint32_t f = fresh ? 0u : flags[g];
    uint32_t gen = fresh ? fresh_gen : gens[g];
    const bool lit = rows[8ull * g + 5] != 0;  // the block's light bricks
    uint32_t next;
    if (full) {
        const bool occupied = (flags[g] & kGroupOccupied) != 0;
        if ((f & kGroupOccupiedBefore) && !occupied)
            gen = ((gen >> 16) + 1u) << 16;  // released: the next life
        else if (lit || (f & kGroupLitBefore))
            gen = (gen & 0xFFFF0000u) | ((gen + 1u) & 0xFFFFu);  // rebuilt: the next version
        next = (lit ? kGroupLitBefore : 0u) | (occupied ? kGroupOccupiedBefore : 0u);
    } else {
        if (f & kGroupTouched) gen = (gen & 0xFFFF0000u) | ((gen + 1u) & 0xFFFFu);
        next = (lit ? kGroupLitBefore : 0u) | (f & kGroupOccupiedBefore);
    }
    gens[g] = gen;
    rows[8ull * g + 2] = gen;
    flags[g] = next;
}

uint32_t blocks_for(uint64_t n, uint32_t per) { return (uint32_t)std::max<uint64_t>(1, (n + per - 1) / per); }

// Resident CTAs of finalize_kernel on every SM of the current device, at most one warp per brick.
uint32_t finalize_grid(uint32_t n)
{
    static int per_sm = 0, sms = 0;
    if (per_sm == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, finalize_kernel<kEncodingBlockId>, kFinalizeWarps * 32, 0);
        per_sm = std::max(per_sm, 1);
        sms = std::max(sms, 1);
    }
    return std::min<uint32_t>(blocks_for(n, kFinalizeWarps), (uint32_t)(per_sm * sms));
}

template <typename T>
cudaError_t alloc(T*& p, uint64_t& capacity, uint64_t count)
{
    count = std::max<uint64_t>(count, 1);
    if (p && count <= capacity) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    capacity = 0;
    // An eighth of headroom: a scene that grows by a few bricks keeps its buffers.
    const uint64_t grown = count + count / 8;
    CX_TRY(cudaMalloc(&p, grown * sizeof(T)));
    capacity = grown;
    return cudaSuccess;
}

cudaError_t run_scan(bool max_op, const uint32_t* in, uint32_t* out, uint32_t count, uint32_t* scratch,
                     uint32_t* total, uint32_t* status, cudaStream_t stream)
{
    if (count == 0) return cudaSuccess;
    const uint32_t tiles = blocks_for(count, kScanTile);
    uint32_t* counter = scratch;
    uint32_t* states = scratch + 1;
    CX_TRY(cudaMemsetAsync(scratch, 0, (1 + (uint64_t)tiles) * 4, stream));
    if (max_op)
        lookback_scan_kernel<true><<<tiles, kThreads, 0, stream>>>(in, out, count, states, counter, total, status);
    else
        lookback_scan_kernel<false><<<tiles, kThreads, 0, stream>>>(in, out, count, states, counter, total, status);
    return cudaGetLastError();
}

}  // namespace

bool scene_grid(const int32_t key_min[3], const int32_t key_max[3], uint32_t group_shift, int32_t origin[3],
                uint32_t grid[3])
{
    const int64_t edge = 1ll << group_shift;
    uint64_t cells = 1;
    for (int k = 0; k < 3; ++k) {
        const int64_t lo = key_min[k] >= 0 ? (key_min[k] / edge) * edge : -((-(int64_t)key_min[k] + edge - 1) / edge) * edge;
        const int64_t extent = (int64_t)key_max[k] - lo + 1;
        if (extent < 1 || extent > (1ll << 32)) return false;
        origin[k] = (int32_t)lo;
        grid[k] = (uint32_t)extent;
        cells *= (uint64_t)((extent + edge - 1) / edge) * (uint64_t)edge;
        if (cells > (1ull << 32)) return false;
    }
    return true;
}

SceneView scene_view(const DeviceScene& s)
{
    SceneView v;
    for (int k = 0; k < 3; ++k) {
        v.grid[k] = s.grid[k];
        v.groups[k] = s.groups[k];
        v.origin[k] = s.origin[k];
    }
    v.enc = encoding_of(s.encoding);
    v.group_shift = s.group_shift;
    v.brick_count = s.brick_count;
    v.records = s.records;
    v.hash_slots = s.hash_slots;
    v.hash_capacity = s.hash_capacity;
    v.hash_max_probe = s.hash_max_probe;
    v.bitmap = s.bitmap;
    v.power = s.power;
    v.materials = s.materials;
    v.light_codes = s.light_codes;
    v.keys = s.keys;
    v.heap = s.heap;
    v.group_rows = s.group_rows;
    v.frames = s.frames;
    v.leaves = s.tree.leaves;
    v.nodes = s.tree.nodes;
    v.header = s.tree.header;
    v.light_count = s.light_count;
    v.group_count = s.group_count;
    v.entities = nullptr;
    v.entity_count = 0;
    v.entity_nodes = nullptr;
    v.dyn = nullptr;
    return v;
}

namespace {

// One thread per group of the entity (its row, its light block, its frame), then one per light
// record (its group).
__global__ void dyn_patch_kernel(uint32_t* __restrict__ heap, uint32_t* __restrict__ rows, GroupFrame* __restrict__ frames,
                                 uint32_t group_count, uint32_t* __restrict__ light_group, uint32_t light_count,
                                 const DynPart part)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < group_count) {
        uint32_t* row = rows + 8ull * (part.group_base + i);
        if (row[1] != 0u) {
            row[0] += part.unit_base;
            uint32_t* block = heap + 4ull * row[0];
            const uint32_t count = block[0];
            for (uint32_t e = 0; e < count; ++e) {
                uint32_t* ie = block + 4 + 4ull * e;
                ie[1] += part.record_base;
                if (ie[3] != kNone) ie[3] = part.leaf_flag | (part.light_base + (ie[3] & 0x7FFFFFFFu));
            }
        }
        GroupFrame& f = frames[part.group_base + i];
        for (int k = 0; k < 9; ++k) f.rot[k] = part.rot[k];
        for (int k = 0; k < 3; ++k) f.trans[k] = part.pos[k];
    }
    if (i < light_count) light_group[part.light_base + i] += part.group_base;
}

}  // namespace

cudaError_t dyn_append(const DeviceScene& e, const DynPart& part, uint32_t* dst_heap, uint32_t* dst_rows,
                       GroupFrame* dst_frames, float* dst_power, BrickLightRecord* dst_headers, uint32_t* dst_group,
                       uint32_t* dst_entry, cudaStream_t stream)
{
    const cudaMemcpyKind d2d = cudaMemcpyDeviceToDevice;
    if (e.heap_words) CX_TRY(cudaMemcpyAsync(dst_heap + 4ull * part.unit_base, e.heap, 4ull * e.heap_words, d2d, stream));
    CX_TRY(cudaMemcpyAsync(dst_rows + 8ull * part.group_base, e.group_rows, 32ull * e.group_count, d2d, stream));
    CX_TRY(cudaMemcpyAsync(dst_frames + part.group_base, e.frames, sizeof(GroupFrame) * e.group_count, d2d, stream));
    if (e.brick_count)
        CX_TRY(cudaMemcpyAsync(dst_power + part.record_base, e.power, 4ull * e.brick_count, d2d, stream));
    if (e.light_count) {
        CX_TRY(cudaMemcpyAsync(dst_headers + part.light_base, e.light_headers, sizeof(BrickLightRecord) * e.light_count,
                               d2d, stream));
        CX_TRY(cudaMemcpyAsync(dst_group + part.light_base, e.light_group, 4ull * e.light_count, d2d, stream));
        CX_TRY(cudaMemcpyAsync(dst_entry + part.light_base, e.light_entry, 4ull * e.light_count, d2d, stream));
    }
    const uint32_t n = std::max(e.group_count, e.light_count);
    if (n) dyn_patch_kernel<<<(n + 127) / 128, 128, 0, stream>>>(dst_heap, dst_rows, dst_frames, e.group_count, dst_group,
                                                             e.light_count, part);
    return cudaGetLastError();
}

// The build scratch of a scene of s.brick_count bricks (sized by scene_build_device): 8 arrays of
// n words, 6 n words of family counts, the sort scratch, scan states.
struct BuildScratch
{
    uint32_t *lo, *hi, *home, *order, *home_alt, *order_alt, *tmp, *tmp2, *counts6, *sortw, *small;
};

static uint64_t build_scratch_words(uint32_t n)
{
    return 14ull * std::max(n, 1u) + sort_scratch_words(std::max(n, 1u), kSortMinKeysPerThread) + 2 +
           blocks_for(std::max(n, 1u), kScanTile) + 64;
}

static BuildScratch build_scratch(const DeviceScene& s)
{
    const uint64_t n = s.brick_count;
    uint32_t* w = s.scratch;
    BuildScratch b;
    b.lo = w;
    b.hi = w + n;
    b.home = w + 2 * n;
    b.order = w + 3 * n;
    b.home_alt = w + 4 * n;
    b.order_alt = w + 5 * n;
    b.tmp = w + 6 * n;
    b.tmp2 = w + 7 * n;
    b.counts6 = w + 8 * n;
    b.sortw = w + 14 * n;
    b.small = b.sortw + sort_scratch_words(std::max(s.brick_count, 1u), kSortMinKeysPerThread);
    return b;
}

void scene_release(DeviceScene& s)
{
    void* ptrs[] = {s.keys,          s.voxels,       s.power,        s.records,       s.hash_slots,
                    s.bitmap,        s.heap,         s.group_rows,    s.frames,
                    s.light_headers, s.light_group,  s.light_entry,  s.light_brick,   s.scratch,
                    s.tree_memory,   s.status,       s.heap_prev,    s.unit_of_brick, s.unit_of_brick_prev,
                    s.group_gen,     s.group_flag};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (s.pinned) cudaFreeHost(s.pinned);
    s = DeviceScene();
}

cudaError_t scene_alloc_inputs(DeviceScene& s, uint32_t n, cudaStream_t stream)
{
    if (!s.status) CX_TRY(cudaMalloc(&s.status, 64));
    if (!s.pinned) CX_TRY(cudaHostAlloc(reinterpret_cast<void**>(&s.pinned), 32, cudaHostAllocDefault));
    CX_TRY(cudaMemsetAsync(s.status, 0, 64, stream));
    CX_TRY(alloc(s.keys, s.capacity.keys, 3ull * n));
    CX_TRY(alloc(s.voxels, s.capacity.voxels, 512ull * n));
    CX_TRY(alloc(s.power, s.capacity.power, n));
    return cudaSuccess;
}

namespace {

void launch_finalize(const FinalizeArgs& fa, uint32_t encoding, uint32_t items, cudaStream_t stream)
{
    if (encoding == kEncodingPacked)
        finalize_kernel<kEncodingPacked><<<finalize_grid(items), kFinalizeWarps * 32, 0, stream>>>(fa);
    else
        finalize_kernel<kEncodingBlockId><<<finalize_grid(items), kFinalizeWarps * 32, 0, stream>>>(fa);
}

}  // namespace

cudaError_t scene_build_device(DeviceScene& s, const int32_t origin[3], const uint32_t grid[3], uint32_t group_shift,
                               uint32_t n, cudaStream_t stream, uint32_t* device_status_out)
{
    if (!s.materials || !s.light_codes) return cudaErrorInvalidValue;
    for (int k = 0; k < 3; ++k) s.grid[k] = grid[k];
    for (int k = 0; k < 3; ++k) s.origin[k] = origin[k];
    s.group_shift = group_shift;
    const uint32_t gm = (1u << group_shift) - 1u;
    for (int k = 0; k < 3; ++k) s.groups[k] = (grid[k] + gm) >> group_shift;
    s.group_count = s.groups[0] * s.groups[1] * s.groups[2];
    s.brick_count = n;

    const uint32_t hash_kpt = sort_keys_per_thread_for(n);
    const uint64_t sort_words = sort_scratch_words(std::max(n, 1u), hash_kpt);
    const uint64_t need = build_scratch_words(n);
    if (need > s.scratch_words) {
        CX_TRY(alloc(s.scratch, s.capacity.scratch, need));
        s.scratch_words = need;
    }
    const BuildScratch bs = build_scratch(s);
    uint32_t* lo = bs.lo;
    uint32_t* hi = bs.hi;
    uint32_t* home = bs.home;
    uint32_t* order = bs.order;
    uint32_t* home_alt = bs.home_alt;
    uint32_t* order_alt = bs.order_alt;
    uint32_t* tmp = bs.tmp;
    uint32_t* tmp2 = bs.tmp2;
    uint32_t* sortw = bs.sortw;
    uint32_t* small = bs.small;

    // Hash table.
    s.hash_capacity = std::max(2u * n, 2u);
    s.hash_slot_count = s.hash_capacity + n + 1;
    CX_TRY(alloc(s.hash_slots, s.capacity.hash_slots, s.hash_slot_count));
    CX_TRY(cudaMemsetAsync(s.hash_slots, 0, 16ull * s.hash_slot_count, stream));
    uint32_t* d_max_probe = s.status + 4;
    if (n > 0) {
        hash_home_kernel<<<blocks_for(n, kThreads), kThreads, 0, stream>>>(s.keys, n, s.hash_capacity, lo, hi, home);
        CX_TRY(cudaMemsetAsync(sortw, 0, sort_words * 4, stream));
        radix_histogram(home, n, sortw, std::min<uint32_t>(blocks_for(n, 2048), current_sm_count() * 4), stream);
        onesweep_sort(home, order, home_alt, order_alt, n, true, sortw, s.status, stream, nullptr, hash_kpt, nullptr,
                      bits_below(s.hash_capacity));
        hash_shift_kernel<<<blocks_for(n, kThreads), kThreads, 0, stream>>>(home, n, tmp);
        CX_TRY(run_scan(true, tmp, tmp2, n, small, nullptr, s.status, stream));
        hash_place_kernel<<<blocks_for(n, kThreads), kThreads, 0, stream>>>(tmp2, home, order, lo, hi, n, s.hash_slots,
                                                                            d_max_probe);
    }
    // Bitmap.
    const uint64_t cells = (uint64_t)grid[0] * grid[1] * grid[2];
    CX_TRY(alloc(s.bitmap, s.capacity.bitmap, (cells + 31) / 32));
    CX_TRY(cudaMemsetAsync(s.bitmap, 0, 4 * ((cells + 31) / 32), stream));
    if (n > 0)
        bitmap_kernel<<<blocks_for(n, kThreads), kThreads, 0, stream>>>(s.keys, n, origin[0], origin[1], origin[2],
                                                                         grid[0], grid[1], s.bitmap);
    CX_TRY(cudaMemcpyAsync(&s.hash_max_probe, d_max_probe, 4, cudaMemcpyDeviceToHost, stream));
    CX_TRY(cudaStreamSynchronize(stream));

    // Records.
    CX_TRY(alloc(s.records, s.capacity.records, (uint64_t)kRecordWords * n));
    if (n > 0) {
        FinalizeArgs fa{s.keys,  s.voxels,          n,         group_shift, s.hash_slots, s.hash_capacity,
                        s.hash_max_probe, s.records, nullptr, nullptr};
        launch_finalize(fa, s.encoding, n, stream);
    }
    return scene_build_lights(s, stream, device_status_out);
}

cudaError_t scene_refinalize(DeviceScene& s, const uint32_t* list, const uint32_t* list_count, uint32_t max_count,
                             cudaStream_t stream)
{
    if (max_count == 0) return cudaSuccess;
    FinalizeArgs fa{s.keys,  s.voxels,          s.brick_count, s.group_shift, s.hash_slots, s.hash_capacity,
                    s.hash_max_probe, s.records, list,       list_count};
    launch_finalize(fa, s.encoding, max_count, stream);
    return cudaGetLastError();
}

// The generation word of every group row (group_generation_kernel), after the rows are written.
cudaError_t update_generations(DeviceScene& s, const uint32_t* marks, uint32_t epoch, cudaStream_t stream)
{
    const uint32_t count = s.group_count;
    if (count == 0) return cudaSuccess;
    const bool same = s.group_gen && s.gen_count == count && s.gen_shift == s.group_shift &&
                      std::memcmp(s.gen_origin, s.origin, sizeof(s.gen_origin)) == 0 &&
                      std::memcmp(s.gen_groups, s.groups, sizeof(s.gen_groups)) == 0;
    uint32_t fresh_gen = 0;
    if (!same) {
        // A new grid: every group starts at a life above every earlier one.
        if (s.group_gen && s.gen_count) {
            std::vector<uint32_t> old(s.gen_count);
            CX_TRY(cudaMemcpyAsync(old.data(), s.group_gen, 4ull * s.gen_count, cudaMemcpyDeviceToHost, stream));
            CX_TRY(cudaStreamSynchronize(stream));
            uint32_t life = 0;
            for (uint32_t g : old) life = std::max(life, g >> 16);
            fresh_gen = ((life + 1u) & 0xFFFFu) << 16;
        }
        CX_TRY(alloc(s.group_gen, s.capacity.group_gen, count));
        CX_TRY(alloc(s.group_flag, s.capacity.group_flag, count));
        CX_TRY(cudaMemsetAsync(s.group_flag, 0, 4ull * count, stream));
        s.gen_count = count;
        s.gen_shift = s.group_shift;
        std::memcpy(s.gen_origin, s.origin, sizeof(s.gen_origin));
        std::memcpy(s.gen_groups, s.groups, sizeof(s.gen_groups));
    }
    GroupGrid gg;
    for (int k = 0; k < 3; ++k) {
        gg.origin[k] = s.origin[k];
        gg.groups[k] = s.groups[k];
    }
    gg.shift = s.group_shift;
    const uint32_t n = s.brick_count;
    if (n > 0) {
        if (!marks)
            group_occupancy_kernel<<<blocks_for(n, kThreads), kThreads, 0, stream>>>(s.keys, n, gg, s.group_flag);
        else
            group_touch_kernel<<<blocks_for(n, kThreads), kThreads, 0, stream>>>(
                s.keys, n, marks, epoch, s.unit_of_brick, s.unit_of_brick_prev, gg, s.group_flag);
    }
    group_generation_kernel<<<blocks_for(count, kThreads), kThreads, 0, stream>>>(
        count, s.group_rows, s.group_gen, s.group_flag, marks ? 0u : 1u, same ? 0u : 1u, fresh_gen);
    return cudaGetLastError();
}

cudaError_t scene_build_lights(DeviceScene& s, cudaStream_t stream, uint32_t* device_status_out,
                               const uint32_t* marks, uint32_t epoch)
{
    const uint32_t n = s.brick_count;
    LightReuse reuse{nullptr, nullptr, nullptr, 0};
    if (marks && s.unit_of_brick) {
        // The previous build's heap and map become the source; the new ones take the other buffers.
        std::swap(s.heap, s.heap_prev);
        std::swap(s.capacity.heap, s.capacity.heap_prev);
        std::swap(s.unit_of_brick, s.unit_of_brick_prev);
        std::swap(s.capacity.unit_of_brick, s.capacity.unit_of_brick_prev);
        reuse = LightReuse{s.unit_of_brick_prev, s.heap_prev, marks, epoch};
    }
    CX_TRY(alloc(s.unit_of_brick, s.capacity.unit_of_brick, std::max(n, 1u)));
    CX_TRY(cudaMemsetAsync(s.unit_of_brick, 0xFF, 4ull * std::max(n, 1u), stream));
    const uint32_t group_shift = s.group_shift;
    const BuildScratch bs = build_scratch(s);
    uint32_t* home = bs.home;
    uint32_t* order = bs.order;
    uint32_t* tmp = bs.tmp;
    uint32_t* tmp2 = bs.tmp2;
    uint32_t* counts6 = bs.counts6;
    uint32_t* sortw = bs.sortw;
    uint32_t* small = bs.small;

    // Light records.
    if (!s.materials || !s.light_codes) return cudaErrorInvalidValue;
    const bool packed = s.encoding == kEncodingPacked;
    LightArgs la{s.keys,
                 s.voxels,
                 s.power,
                 n,
                 group_shift,
                 {s.groups[0], s.groups[1], s.groups[2]},
                 {s.origin[0], s.origin[1], s.origin[2]},
                 s.hash_slots,
                 s.hash_capacity,
                 s.hash_max_probe,
                 s.materials,
                 s.light_codes};
    uint32_t* d_light_count = s.status + 5;
    uint32_t* lkeys = bs.lo;  // reuse the hash scratch
    uint32_t* lbricks = bs.hi;
    uint32_t* lkeys_alt = bs.home_alt;
    uint32_t* lbricks_alt = bs.order_alt;
    if (n > 0 && s.lights) {
        if (packed)
            light_collect_kernel<kEncodingPacked>
                <<<blocks_for(n, kThreads), kThreads, 0, stream>>>(la, d_light_count, lkeys, lbricks);
        else
            light_collect_kernel<kEncodingBlockId>
                <<<blocks_for(n, kThreads), kThreads, 0, stream>>>(la, d_light_count, lkeys, lbricks);
    }
    CX_TRY(cudaMemcpyAsync(s.pinned, d_light_count, 4, cudaMemcpyDeviceToHost, stream));
    CX_TRY(cudaStreamSynchronize(stream));
    const uint32_t m = s.pinned[0];
    s.light_count = m;
    CX_TRY(alloc(s.group_rows, s.capacity.group_rows, 8ull * s.group_count));
    CX_TRY(cudaMemsetAsync(s.group_rows, 0, 32ull * s.group_count, stream));
    CX_TRY(alloc(s.light_headers, s.capacity.light_headers, m));
    CX_TRY(alloc(s.light_group, s.capacity.light_group, m));
    CX_TRY(alloc(s.light_entry, s.capacity.light_entry, m));
    CX_TRY(alloc(s.light_brick, s.capacity.light_brick, m));
    // The group frames (their origins follow from the grid origin and the group grid; identity
    // rotations): uploaded when the grid changed or their buffer moved.
    GroupFrame* const old_frames = s.frames;
    CX_TRY(alloc(s.frames, s.capacity.frames, s.group_count));
    const bool same_frames = s.frames == old_frames && s.frames_shift == group_shift &&
                             std::memcmp(s.frames_origin, s.origin, sizeof(s.frames_origin)) == 0 &&
                             std::memcmp(s.frames_groups, s.groups, sizeof(s.frames_groups)) == 0;
    if (!same_frames) {
        std::vector<GroupFrame> frames(s.group_count);
        for (uint32_t g = 0; g < s.group_count; ++g) {
            const uint32_t gx = g % s.groups[0], gy = (g / s.groups[0]) % s.groups[1],
                           gz = g / (s.groups[0] * s.groups[1]);
            GroupFrame f;
            std::memset(&f, 0, sizeof(f));
            // The group's voxel origin in the scene: (grid origin + group cell * group edge) * 8.
            const uint32_t cell[3] = {gx, gy, gz};
            for (int k = 0; k < 3; ++k)
                f.origin[k] = (float)(8ll * ((int64_t)s.origin[k] + ((int64_t)cell[k] << group_shift)));
            f.rot[0] = f.rot[4] = f.rot[8] = 1.0f;
            frames[g] = f;
        }
        CX_TRY(cudaMemcpyAsync(s.frames, frames.data(), sizeof(GroupFrame) * s.group_count, cudaMemcpyHostToDevice,
                               stream));
        std::memcpy(s.frames_origin, s.origin, sizeof(s.frames_origin));
        std::memcpy(s.frames_groups, s.groups, sizeof(s.frames_groups));
        s.frames_shift = group_shift;
    }
    uint32_t total_units = 0;
    if (m > 0) {
        const uint32_t light_kpt = sort_keys_per_thread_for(m);
        CX_TRY(cudaMemsetAsync(sortw, 0, sort_scratch_words(m, light_kpt) * 4, stream));
        radix_histogram(lkeys, m, sortw, std::min<uint32_t>(blocks_for(m, 2048), current_sm_count() * 4), stream);
        // Keys: the group index above 3 * group_shift bits of position in the group.
        onesweep_sort(lkeys, lbricks, lkeys_alt, lbricks_alt, m, false, sortw, s.status, stream, nullptr, light_kpt,
                      nullptr, 3 * group_shift + bits_below(s.group_count));
        uint32_t* units = home;    // m words
        uint32_t* totals = order;  // m words
        uint32_t* group_start = tmp;
        uint32_t* offsets = tmp2;
        if (packed)
            light_measure_kernel<kEncodingPacked><<<blocks_for(32ull * m, kLightWarps * 32), kLightWarps * 32, 0, stream>>>(
                la, lbricks, m, counts6, units, reuse);
        else
            light_measure_kernel<kEncodingBlockId><<<blocks_for(32ull * m, kLightWarps * 32), kLightWarps * 32, 0, stream>>>(
                la, lbricks, m, counts6, units, reuse);
        uint32_t* group_end = lkeys_alt;  // free once the light sort is done
        light_group_kernel<<<blocks_for(m, kThreads), kThreads, 0, stream>>>(lkeys, m, group_shift, units, totals,
                                                                             group_start, group_end);
        uint32_t* d_total = s.status + 6;
        CX_TRY(run_scan(false, totals, offsets, m, small, d_total, s.status, stream));
        CX_TRY(cudaMemcpyAsync(s.pinned + 1, d_total, 4, cudaMemcpyDeviceToHost, stream));
        CX_TRY(cudaStreamSynchronize(stream));
        total_units = s.pinned[1];
        s.heap_words = 4 * (1 + total_units);
        CX_TRY(alloc(s.heap, s.capacity.heap, s.heap_words));
        // Unit 0 is reserved (zero); light_write_kernel writes every other unit (block headers,
        // index entries, records with their padding).
        CX_TRY(cudaMemsetAsync(s.heap, 0, 16, stream));
        LightWriteArgs wa{la,           lkeys,         lbricks,         m,           counts6,
                          units,        offsets,       group_start,     group_end,   total_units, s.heap,
                          s.group_rows, s.light_headers, s.light_group, s.light_entry, s.light_brick,
                          reuse,        s.unit_of_brick};
        if (packed)
            light_write_kernel<kEncodingPacked><<<blocks_for(32ull * m, kLightWarps * 32), kLightWarps * 32, 0, stream>>>(wa);
        else
            light_write_kernel<kEncodingBlockId><<<blocks_for(32ull * m, kLightWarps * 32), kLightWarps * 32, 0, stream>>>(wa);
    } else {
        s.heap_words = 4;
        CX_TRY(alloc(s.heap, s.capacity.heap, 4));
        CX_TRY(cudaMemsetAsync(s.heap, 0, 16, stream));
    }
    CX_TRY(update_generations(s, marks, epoch, stream));
    if (!marks) {
        // The buffers the next rebuild over the same bricks swaps in, sized now (a full build
        // allocates anyway; the edit flushes that follow then allocate nothing while the heap
        // keeps its size).
        CX_TRY(alloc(s.heap_prev, s.capacity.heap_prev, s.heap_words));
        CX_TRY(alloc(s.unit_of_brick_prev, s.capacity.unit_of_brick_prev, std::max(n, 1u)));
    }

    // The light tree over the light records (leaf = gather order).
    const uint32_t cap = std::max(m, 1u);
    if (cap > s.tree_capacity) {
        if (s.tree_memory) cudaFree(s.tree_memory);
        s.tree_memory = nullptr;
        const uint32_t grown = cap + cap / 8;
        CX_TRY(cudaMalloc(&s.tree_memory, lt_buffer_bytes(grown)));
        s.tree = lt_carve(s.tree_memory, grown);
        s.tree_capacity = grown;
        CX_TRY(cudaMemsetAsync(s.tree.header, 0, 128, stream));
    }
    CX_TRY(scene_build_light_tree(s, stream));
    return scene_read_status(s, stream, device_status_out);
}

cudaError_t scene_build_light_tree(const DeviceScene& s, cudaStream_t stream, uint32_t sort_keys_per_thread)
{
    if (s.tree_capacity < std::max(s.light_count, 1u)) return cudaErrorInvalidValue;
    LightBvhInput in;
    in.records = s.light_headers;
    in.count = s.light_count;
    in.record_group = s.light_group;
    in.record_entry = s.light_entry;
    in.group_frames = s.frames;
    in.group_count = s.group_count;
    in.sort_keys_per_thread = sort_keys_per_thread;
    return lt_build(s.tree, in, stream, nullptr);
}

cudaError_t scene_read_status(const DeviceScene& s, cudaStream_t stream, uint32_t* device_status_out)
{
    if (!s.status || !s.pinned) return cudaErrorInvalidValue;  // never built
    CX_TRY(cudaMemcpyAsync(s.pinned + 2, s.status, 4, cudaMemcpyDeviceToHost, stream));
    CX_TRY(cudaMemcpyAsync(s.pinned + 3, &s.tree.state->status, 4, cudaMemcpyDeviceToHost, stream));
    CX_TRY(cudaStreamSynchronize(stream));
    if (device_status_out) *device_status_out = s.pinned[2] | s.pinned[3];
    return cudaGetLastError();
}

}  // namespace cx
