// World files (.cxw, format version 8 and older) behind the C ABI (include/caelix_b200.h):
// the header, the world record, the entity table with its version migrations, the sector
// indices with their region checks, the raw-deflate sector payloads and their brick tables, and
// a loader of one entity into a scene. The read rules are the reference reader's
// (host-rs/caelix-cxw/src/lib.rs: parse_index :339-452, region :455-493, Scratch::inflate
// :513-542, decode_payload :544-630); the loader replaces its host's streaming loader
// (host-rs/caelix-app/src/world.rs :93-262) for this library's static world entity.
#include <zlib.h>

#include <algorithm>
#include <atomic>
#include <cinttypes>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <set>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "abi_internal.h"

namespace {

constexpr uint32_t kFileMagic = 0x534C5843u;    // "CXLS"
constexpr uint32_t kLegacyMagic = 0x534C5856u;  // "VXLS", accepted on read
constexpr uint16_t kNewestVersion = 8;
constexpr uint16_t kFlagDeflate = 1;
constexpr uint32_t kPayloadMagic = 0x32535856u;  // "VXS2"
constexpr int32_t kBricksPerAxis = 16;
constexpr uint32_t kBricksInSector = 4096;
constexpr uint32_t kBlocksInBrick = 512;
constexpr uint64_t kHeaderBytes = 64;
constexpr uint64_t kPreviewBytes = kBricksInSector * 4ull;
constexpr uint64_t kRegionOverhead = kPreviewBytes + 4;  // preview + payload size
constexpr uint64_t kIndexEntryBytes = 24;
constexpr uint64_t kMinEntityRecordBytes = 16 + 28 + 2 + 8 + 4;
constexpr uint32_t kMaxSlots = 16;
constexpr uint8_t kSlotBlock = 0;
constexpr uint16_t kBlockStride = 2;
constexpr uint64_t kMaxPayloadBytes = 1ull << 30;
constexpr uint8_t kEntityHasBody = 1, kEntityStatic = 2;
constexpr uint8_t kWorldHasPlayerPose = 1;
// Version gates of the entity record and the world record.
constexpr uint16_t kVersionEntityFlags = 3, kVersionVelocity = 4, kVersionProtected = 5, kVersionFlagsV6 = 6,
                   kVersionWorldRecord = 7;

struct ReadError
{
    CaelixResult code;
    std::string message;
};

[[noreturn]] void fail(CaelixResult code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
[[noreturn]] void fail(CaelixResult code, const char* fmt, ...)
{
    char buf[512];
    va_list args;
    va_start(args, fmt);
    vsnprintf(buf, sizeof(buf), fmt, args);
    va_end(args);
    throw ReadError{code, buf};
}

// Bounds-checked little-endian reads over a byte range.
struct Cursor
{
    const uint8_t* data;
    uint64_t size;
    uint64_t pos;

    const uint8_t* take(uint64_t n, const char* what)
    {
        if (n > size || pos > size - n)
            fail(CAELIX_ERROR_INVALID_ARGUMENT, "truncated data reading %s at offset %" PRIu64, what, pos);
        const uint8_t* p = data + pos;
        pos += n;
        return p;
    }
    template <typename T>
    T get(const char* what)
    {
        T v;
        std::memcpy(&v, take(sizeof(T), what), sizeof(T));
        return v;
    }
    void floats(float* out, int n, const char* what) { std::memcpy(out, take(4ull * n, what), 4ull * n); }
};

// The entity flags of a legacy (version 3 .. 5) body-state byte.
uint8_t flags_from_body_state(uint8_t body_state)
{
    if (body_state == 1) return kEntityHasBody | kEntityStatic;
    if (body_state == 2) return kEntityHasBody;
    return kEntityStatic;
}

struct Region
{
    const uint8_t* preview;
    const uint8_t* payload;
    uint32_t payload_size;
};

// One sector region: the preview, the payload size and the payload, with the size rule
// region_size == 16388 + payload size.
Region region(const std::vector<uint8_t>& data, const int32_t coord[3], uint64_t offset, uint32_t size)
{
    const uint64_t len = data.size();
    if (offset > len || len - offset < kRegionOverhead)
        fail(CAELIX_ERROR_INVALID_ARGUMENT, "truncated data reading sector region at offset %" PRIu64, offset);
    Region r;
    r.preview = data.data() + offset;
    std::memcpy(&r.payload_size, data.data() + offset + kPreviewBytes, 4);
    const uint64_t expected = kRegionOverhead + r.payload_size;
    if (expected != size)
        fail(CAELIX_ERROR_INVALID_ARGUMENT,
             "sector (%d, %d, %d): region size is %u, expected %" PRIu64 " (16388 + payload size)", coord[0],
             coord[1], coord[2], size, expected);
    const uint64_t start = offset + kRegionOverhead;
    if (start + r.payload_size > len)
        fail(CAELIX_ERROR_INVALID_ARGUMENT, "truncated data reading sector payload at offset %" PRIu64, start);
    r.payload = data.data() + start;
    return r;
}

// Inflates a raw deflate stream (no zlib header) into out.
void inflate_raw(const uint8_t* in, uint32_t in_size, const int32_t coord[3], std::vector<uint8_t>& out)
{
    z_stream z;
    std::memset(&z, 0, sizeof(z));
    if (inflateInit2(&z, -15) != Z_OK)
        fail(CAELIX_ERROR_OUT_OF_MEMORY, "inflate failed: sector (%d, %d, %d): inflateInit2", coord[0], coord[1],
             coord[2]);
    out.clear();
    out.resize(std::min<uint64_t>(std::max<uint64_t>(4ull * in_size, 64 * 1024), kMaxPayloadBytes));
    z.next_in = const_cast<Bytef*>(in);
    z.avail_in = in_size;
    uint64_t produced = 0;
    for (;;) {
        if (produced == out.size()) {
            if (out.size() >= kMaxPayloadBytes) {
                inflateEnd(&z);
                fail(CAELIX_ERROR_INVALID_ARGUMENT,
                     "inflate failed: sector (%d, %d, %d): payload inflates to more than 1 GiB", coord[0], coord[1],
                     coord[2]);
            }
            out.resize(std::min<uint64_t>(2 * out.size(), kMaxPayloadBytes));
        }
        z.next_out = out.data() + produced;
        z.avail_out = (uInt)std::min<uint64_t>(out.size() - produced, 1u << 30);
        const uInt before_out = z.avail_out, before_in = z.avail_in;
        const int rc = inflate(&z, Z_NO_FLUSH);
        produced += before_out - z.avail_out;
        if (rc == Z_STREAM_END) break;
        if (rc != Z_OK && rc != Z_BUF_ERROR) {
            const std::string msg = z.msg ? z.msg : "corrupt deflate stream";
            inflateEnd(&z);
            fail(CAELIX_ERROR_INVALID_ARGUMENT, "inflate failed: sector (%d, %d, %d): %s", coord[0], coord[1],
                 coord[2], msg.c_str());
        }
        const bool stalled = z.avail_out == before_out && z.avail_in == before_in;
        if (stalled && produced < out.size()) {
            inflateEnd(&z);
            fail(CAELIX_ERROR_INVALID_ARGUMENT,
                 "inflate failed: sector (%d, %d, %d): deflate stream ends before its final block", coord[0],
                 coord[1], coord[2]);
        }
    }
    inflateEnd(&z);
    out.resize(produced);
}

struct Decoded
{
    std::vector<CaelixBrickKey> keys;
    std::vector<uint16_t> blocks;
    std::vector<uint32_t> summaries;
    uint64_t voxels = 0;
};

// The non-air bricks of one inflated sector payload.
void decode_payload(const std::vector<uint8_t>& raw, const uint8_t* preview, const int32_t coord[3], Decoded& d)
{
    Cursor c{raw.data(), raw.size(), 0};
    const uint32_t magic = c.get<uint32_t>("payload header");
    if (magic != kPayloadMagic)
        fail(CAELIX_ERROR_INVALID_ARGUMENT, "bad sector payload magic 0x%08X (expected VXS2)", magic);
    const uint32_t capacity = c.get<uint32_t>("payload header");
    const uint32_t count = c.get<uint32_t>("payload header");
    const uint32_t free_count = c.get<uint32_t>("payload header");
    if (capacity > kBricksInSector || count > capacity || free_count > capacity ||
        (uint64_t)count + free_count != capacity)
        fail(CAELIX_ERROR_INVALID_ARGUMENT, "invalid brick map counters: capacity %u, count %u, free %u", capacity,
             count, free_count);
    const uint8_t* indices = c.take(kBricksInSector * 2ull, "payload brick indices");
    c.take(2ull * free_count, "payload free list");
    c.take(2 + kBricksInSector * 2ull, "payload require-update flags");
    const uint32_t slot_count = c.get<uint32_t>("payload slot record count");
    auto bad = [&](const char* reason) {
        fail(CAELIX_ERROR_INVALID_ARGUMENT, "sector (%d, %d, %d): invalid payload: %s", coord[0], coord[1], coord[2],
             reason);
    };
    if (slot_count > kMaxSlots) bad("more than 16 slot records");
    uint32_t seen = 0;
    const uint8_t* block_data = nullptr;
    for (uint32_t i = 0; i < slot_count; ++i) {
        const uint8_t id = c.get<uint8_t>("payload slot record header");
        const uint16_t stride = c.get<uint16_t>("payload slot record header");
        if (id >= kMaxSlots || (seen >> id) & 1u) bad("invalid or duplicate slot id");
        seen |= 1u << id;
        if (stride == 0) bad("slot stride is 0");
        const uint8_t* data = c.take((uint64_t)capacity * kBlocksInBrick * stride, "payload slot data");
        if (id == kSlotBlock) {
            if (stride != kBlockStride) bad("Block slot stride is not 2");
            block_data = data;
        }
    }
    // Trailing bytes are tolerated.
    const int32_t base[3] = {(int32_t)((uint32_t)coord[0] * (uint32_t)kBricksPerAxis),
                             (int32_t)((uint32_t)coord[1] * (uint32_t)kBricksPerAxis),
                             (int32_t)((uint32_t)coord[2] * (uint32_t)kBricksPerAxis)};
    for (uint32_t bi = 0; bi < kBricksInSector; ++bi) {
        int16_t id;
        std::memcpy(&id, indices + 2ull * bi, 2);
        if (id == -1) continue;
        if (id < -1 || (uint32_t)id >= capacity) bad("brick index table entry outside -1..capacity-1");
        if (!block_data) bad("allocated bricks but no Block slot");
        const size_t start = d.blocks.size();
        d.blocks.resize(start + kBlocksInBrick);
        std::memcpy(d.blocks.data() + start, block_data + (uint64_t)id * kBlocksInBrick * 2, kBlocksInBrick * 2);
        uint64_t non_zero = 0;
        for (uint32_t v = 0; v < kBlocksInBrick; ++v) non_zero += d.blocks[start + v] != 0;
        if (non_zero == 0) {
            d.blocks.resize(start);
            continue;
        }
        d.voxels += non_zero;
        const int32_t b = (int32_t)bi;
        d.keys.push_back(CaelixBrickKey{(int32_t)((uint32_t)base[0] + (uint32_t)(b & 15)),
                                        (int32_t)((uint32_t)base[1] + (uint32_t)((b >> 4) & 15)),
                                        (int32_t)((uint32_t)base[2] + (uint32_t)(b >> 8))});
        uint32_t word;
        std::memcpy(&word, preview + 4ull * bi, 4);
        d.summaries.push_back(word);
    }
}

}  // namespace

struct CaelixWorldFile
{
    std::vector<uint8_t> data;
    CaelixWorldInfo info{};
    std::vector<CaelixWorldEntity> entities;
    std::vector<CaelixWorldSector> sectors;
};

namespace {

void parse_index(CaelixWorldFile& f)
{
    const std::vector<uint8_t>& data = f.data;
    const uint64_t len = data.size();
    if (len < kHeaderBytes) fail(CAELIX_ERROR_INVALID_ARGUMENT, "truncated data reading header at offset 0");
    Cursor h{data.data(), len, 0};
    const uint32_t magic = h.get<uint32_t>("header");
    if (magic != kFileMagic && magic != kLegacyMagic)
        fail(CAELIX_ERROR_INVALID_ARGUMENT, "bad file magic 0x%08X (expected CXLS or VXLS)", magic);
    const uint16_t version = h.get<uint16_t>("header");
    if (version > kNewestVersion)
        fail(CAELIX_ERROR_UNSUPPORTED, "format version %u is not supported (newest supported: %u)", version,
             kNewestVersion);
    const uint16_t flags = h.get<uint16_t>("header");
    if (flags != kFlagDeflate)
        fail(CAELIX_ERROR_INVALID_ARGUMENT, "unsupported save flags 0x%04X (must be 1 = Deflate)", flags);
    const uint64_t table = h.get<uint64_t>("header");
    if (table < kHeaderBytes || table > len)
        fail(CAELIX_ERROR_INVALID_ARGUMENT, "truncated data reading entity table at offset %" PRIu64, table);
    f.info.version = version;
    Cursor c{data.data(), len, table};
    if (version >= kVersionWorldRecord) {
        const uint8_t world_flags = c.get<uint8_t>("world record");
        float pos[3], rot[4];
        c.floats(pos, 3, "world record");
        c.floats(rot, 4, "world record");
        if (world_flags & kWorldHasPlayerPose) {
            f.info.has_player_pose = 1;
            std::memcpy(f.info.player_position, pos, sizeof(pos));
            std::memcpy(f.info.player_rotation, rot, sizeof(rot));
        }
    }
    const uint32_t count = c.get<uint32_t>("entity count");
    f.entities.reserve(std::min<uint64_t>(count, (len - c.pos) / kMinEntityRecordBytes));
    std::vector<uint64_t> index_offsets;
    for (uint32_t i = 0; i < count; ++i) {
        const char* what = "entity record";
        CaelixWorldEntity e{};
        std::memcpy(e.guid, c.take(16, what), 16);
        c.floats(e.position, 3, what);
        c.floats(e.rotation, 4, what);
        e.require_update_flags = c.get<uint16_t>(what);
        if (version >= kVersionFlagsV6) e.flags = c.get<uint8_t>(what) & (kEntityHasBody | kEntityStatic);
        else if (version >= kVersionEntityFlags) e.flags = flags_from_body_state(c.get<uint8_t>(what));
        else e.flags = kEntityStatic;
        if (version >= kVersionVelocity) c.floats(e.velocity, 6, what);
        e.is_protected = version >= kVersionProtected && c.get<uint8_t>(what) != 0;
        index_offsets.push_back(c.get<uint64_t>(what));
        e.sector_count = c.get<uint32_t>(what);
        f.entities.push_back(e);
    }
    for (uint32_t ei = 0; ei < f.entities.size(); ++ei) {
        const uint64_t start = index_offsets[ei];
        const uint64_t bytes = (uint64_t)f.entities[ei].sector_count * kIndexEntryBytes;
        if (start < kHeaderBytes || start > len || bytes > len - start)
            fail(CAELIX_ERROR_INVALID_ARGUMENT, "truncated data reading sector index at offset %" PRIu64, start);
        Cursor s{data.data(), len, start};
        std::set<std::tuple<int32_t, int32_t, int32_t>> seen;
        for (uint32_t k = 0; k < f.entities[ei].sector_count; ++k) {
            CaelixWorldSector sec{};
            sec.entity = ei;
            for (int a = 0; a < 3; ++a) sec.coord[a] = s.get<int32_t>("sector index");
            sec.region_offset = s.get<uint64_t>("sector index");
            sec.region_size = s.get<uint32_t>("sector index");
            region(data, sec.coord, sec.region_offset, sec.region_size);
            if (!seen.insert({sec.coord[0], sec.coord[1], sec.coord[2]}).second)
                fail(CAELIX_ERROR_INVALID_ARGUMENT, "sector (%d, %d, %d) appears twice in one entity's sector index",
                     sec.coord[0], sec.coord[1], sec.coord[2]);
            f.sectors.push_back(sec);
        }
    }
    f.info.entity_count = (uint32_t)f.entities.size();
    f.info.sector_count = f.sectors.size();
}

void decode_sector(const CaelixWorldFile& f, const CaelixWorldSector& s, std::vector<uint8_t>& scratch, Decoded& d)
{
    const Region r = region(f.data, s.coord, s.region_offset, s.region_size);
    inflate_raw(r.payload, r.payload_size, s.coord, scratch);
    decode_payload(scratch, r.preview, s.coord, d);
}

CaelixResult report(const ReadError& e)
{
    cx::log(CAELIX_LOG_ERROR, "%s", e.message.c_str());
    return e.code;
}

}  // namespace

extern "C" {

CAELIX_API CaelixResult caelix_world_open(const char* path, CaelixWorldFile** out)
{
    CAELIX_GUARD_BEGIN
    if (!path || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out = nullptr;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) {
        cx::log(CAELIX_LOG_ERROR, "I/O error: cannot open %s", path);
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    CaelixWorldFile* f = new CaelixWorldFile();
    std::fseek(fp, 0, SEEK_END);
    const long size = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    f->data.resize(size > 0 ? (size_t)size : 0);
    const size_t got = f->data.empty() ? 0 : std::fread(f->data.data(), 1, f->data.size(), fp);
    std::fclose(fp);
    if (size < 0 || got != f->data.size()) {
        delete f;
        cx::log(CAELIX_LOG_ERROR, "I/O error: cannot read %s", path);
        return CAELIX_ERROR_INVALID_ARGUMENT;
    }
    try {
        parse_index(*f);
    } catch (const ReadError& e) {
        delete f;
        return report(e);
    }
    *out = f;
    return CAELIX_OK;
    CAELIX_GUARD_END
}

CAELIX_API void caelix_world_close(CaelixWorldFile* file) { delete file; }

CAELIX_API CaelixResult caelix_world_get_info(const CaelixWorldFile* file, CaelixWorldInfo* out)
{
    if (!file || !out) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out = file->info;
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_world_get_entity(const CaelixWorldFile* file, uint32_t index, CaelixWorldEntity* out)
{
    if (!file || !out || index >= file->entities.size()) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out = file->entities[index];
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_world_get_sector(const CaelixWorldFile* file, uint64_t index, CaelixWorldSector* out)
{
    if (!file || !out || index >= file->sectors.size()) return CAELIX_ERROR_INVALID_ARGUMENT;
    *out = file->sectors[index];
    return CAELIX_OK;
}

CAELIX_API CaelixResult caelix_world_decode_sector(const CaelixWorldFile* file, uint64_t index, uint32_t capacity,
                                                   CaelixBrickKey* keys, uint16_t* blocks, uint32_t* summaries,
                                                   uint32_t* brick_count, uint64_t* voxels)
{
    CAELIX_GUARD_BEGIN
    if (!file || index >= file->sectors.size() || (keys && (!blocks || !summaries))) return CAELIX_ERROR_INVALID_ARGUMENT;
    Decoded d;
    std::vector<uint8_t> scratch;
    try {
        decode_sector(*file, file->sectors[index], scratch, d);
    } catch (const ReadError& e) {
        return report(e);
    }
    const uint32_t n = (uint32_t)d.keys.size();
    if (brick_count) *brick_count = n;
    if (voxels) *voxels = d.voxels;
    if (!keys) return CAELIX_OK;
    if (capacity < n) return CAELIX_ERROR_INVALID_ARGUMENT;
    std::memcpy(keys, d.keys.data(), sizeof(CaelixBrickKey) * n);
    std::memcpy(blocks, d.blocks.data(), 2ull * kBlocksInBrick * n);
    std::memcpy(summaries, d.summaries.data(), 4ull * n);
    return CAELIX_OK;
    CAELIX_GUARD_END
}

}  // extern "C"

namespace {

// Every sector of one file entity decoded on the host threads (each with its own inflate buffer);
// org (the move applied to its keys) is 0.
CaelixResult decode_entity(const CaelixWorldFile* file, uint32_t entity, uint32_t threads, const char* what,
                           std::vector<Decoded>& decoded, int32_t org[3])
{
    std::vector<const CaelixWorldSector*> mine;
    for (const CaelixWorldSector& s : file->sectors)
        if (s.entity == entity) mine.push_back(&s);
    decoded.assign(mine.size(), Decoded());
    std::atomic<size_t> next{0};
    std::atomic<bool> failed{false};
    const uint32_t nt = std::max(1u, std::min<uint32_t>(threads ? threads : std::thread::hardware_concurrency(),
                                                        (uint32_t)std::max<size_t>(mine.size(), 1)));
    std::vector<ReadError> first(nt);
    std::vector<char> has_error(nt, 0);
    auto work = [&](uint32_t t) {
        std::vector<uint8_t> scratch;
        for (size_t i = next++; i < mine.size() && !failed; i = next++) {
            try {
                decode_sector(*file, *mine[i], scratch, decoded[i]);
            } catch (const ReadError& e) {
                first[t] = e;
                has_error[t] = 1;
                failed = true;
            }
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (std::thread& th : pool) th.join();
    for (uint32_t t = 0; t < nt; ++t)
        if (has_error[t]) return report(first[t]);
    // The keys go to the scene as the file holds them (the reference's loader passes the decoder's
    // keys through): the scene takes [-2^20, 2^20) per axis and its flush checks the box.
    (void)what;
    for (int a = 0; a < 3; ++a) org[a] = 0;
    return CAELIX_OK;
}

// Uploads decoded bricks to entity `target` of the scene in sector order, the keys moved to `org`.
CaelixResult upload_decoded(const std::vector<Decoded>& decoded, const int32_t org[3], CaelixScene* scene,
                            uint32_t target, uint64_t* bricks)
{
    std::vector<CaelixBrickKey> keys;
    for (const Decoded& d : decoded) {
        if (d.keys.empty()) continue;
        keys.resize(d.keys.size());
        for (size_t i = 0; i < d.keys.size(); ++i)
            keys[i] = CaelixBrickKey{d.keys[i].x - org[0], d.keys[i].y - org[1], d.keys[i].z - org[2]};
        uint32_t consumed = 0;
        const CaelixResult r = caelix_scene_upload_bricks(scene, target, (uint32_t)keys.size(), keys.data(),
                                                          d.blocks.data(), &consumed);
        if (r != CAELIX_OK) return r;
        if (bricks) *bricks += consumed;
    }
    return CAELIX_OK;
}

// Rotation rows of a quaternion (x, y, z, w), normalised, in double.
void quat_rows(const float q[4], double r[9])
{
    const double n = std::sqrt((double)q[0] * q[0] + (double)q[1] * q[1] + (double)q[2] * q[2] + (double)q[3] * q[3]);
    const double x = q[0] / n, y = q[1] / n, z = q[2] / n, w = q[3] / n;
    const double m[9] = {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * w), 2.0 * (x * z + y * w),
                         2.0 * (x * y + z * w), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * w),
                         2.0 * (x * z - y * w), 2.0 * (y * z + x * w), 1.0 - 2.0 * (x * x + y * y)};
    for (int i = 0; i < 9; ++i) r[i] = m[i];
}

}  // namespace

extern "C" {

CAELIX_API CaelixResult caelix_world_upload_entity(const CaelixWorldFile* file, uint32_t entity, CaelixScene* scene,
                                                   uint32_t threads, int32_t origin[3], uint64_t* bricks)
{
    CAELIX_GUARD_BEGIN
    if (bricks) *bricks = 0;
    if (!file || !scene || entity >= file->entities.size()) return CAELIX_ERROR_INVALID_ARGUMENT;
    std::vector<Decoded> decoded;
    int32_t org[3];
    CaelixResult r = decode_entity(file, entity, threads, "caelix_world_upload_entity", decoded, org);
    if (r != CAELIX_OK) return r;
    if (origin) std::memcpy(origin, org, sizeof(org));
    return upload_decoded(decoded, org, scene, 0, bricks);
    CAELIX_GUARD_END
}

CAELIX_API CaelixResult caelix_world_load(const CaelixWorldFile* file, CaelixScene* scene, uint32_t threads,
                                          CaelixEntityId* ids, uint64_t* bricks)
{
    CAELIX_GUARD_BEGIN
    if (bricks) *bricks = 0;
    if (!file || !scene || file->entities.empty()) return CAELIX_ERROR_INVALID_ARGUMENT;
    const uint32_t count = (uint32_t)file->entities.size();
    if (ids)
        for (uint32_t i = 0; i < count; ++i) ids[i] = CAELIX_INVALID_ENTITY;
    // File entity 0 is the world: the scene's frame is its frame, moved by its origin,
    // x_scene = R0^T (x_file - p0) - 8 org0.
    std::vector<Decoded> decoded;
    int32_t org0[3];
    CaelixResult r = decode_entity(file, 0, threads, "caelix_world_load", decoded, org0);
    if (r != CAELIX_OK) return r;
    const CaelixWorldEntity& w = file->entities[0];
    double r0[9];
    quat_rows(w.rotation, r0);
    // Every other entity first decoded and added (a failure removes the ones added), then the
    // bricks uploaded.
    std::vector<CaelixEntityId> added;
    auto undo = [&](CaelixResult res) {
        for (CaelixEntityId id : added) caelix_scene_remove_entity(scene, id);
        if (ids)
            for (uint32_t i = 0; i < count; ++i) ids[i] = CAELIX_INVALID_ENTITY;
        return res;
    };
    r = upload_decoded(decoded, org0, scene, 0, bricks);
    if (r != CAELIX_OK) return r;
    if (ids) ids[0] = 0;
    for (uint32_t i = 1; i < count; ++i) {
        std::vector<Decoded> dec;
        int32_t org[3];
        r = decode_entity(file, i, threads, "caelix_world_load", dec, org);
        if (r != CAELIX_OK) return undo(r);
        const CaelixWorldEntity& e = file->entities[i];
        double ri[9];
        quat_rows(e.rotation, ri);
        // Its keys start at its origin: x_file = Ri (local + 8 org) + pi.
        double v[3];
        for (int k = 0; k < 3; ++k)
            v[k] = (ri[3 * k] * (8.0 * org[0]) + ri[3 * k + 1] * (8.0 * org[1]) + ri[3 * k + 2] * (8.0 * org[2])) +
                   ((double)e.position[k] - (double)w.position[k]);
        CaelixEntityDesc desc;
        std::memcpy(desc.guid, e.guid, sizeof(desc.guid));
        for (int k = 0; k < 3; ++k)
            desc.position[k] = (float)((r0[k] * v[0] + r0[3 + k] * v[1] + r0[6 + k] * v[2]) - 8.0 * org0[k]);
        // The rotation R0^T Ri as a quaternion: conj(q0) * qi.
        const double n0 = std::sqrt((double)w.rotation[0] * w.rotation[0] + (double)w.rotation[1] * w.rotation[1] +
                                    (double)w.rotation[2] * w.rotation[2] + (double)w.rotation[3] * w.rotation[3]);
        const double ax = -w.rotation[0] / n0, ay = -w.rotation[1] / n0, az = -w.rotation[2] / n0,
                     aw = w.rotation[3] / n0;
        const double bx = e.rotation[0], by = e.rotation[1], bz = e.rotation[2], bw = e.rotation[3];
        desc.rotation[0] = (float)(aw * bx + ax * bw + ay * bz - az * by);
        desc.rotation[1] = (float)(aw * by - ax * bz + ay * bw + az * bx);
        desc.rotation[2] = (float)(aw * bz + ax * by - ay * bx + az * bw);
        desc.rotation[3] = (float)(aw * bw - ax * bx - ay * by - az * bz);
        CaelixEntityId id = CAELIX_INVALID_ENTITY;
        r = caelix_scene_add_entity(scene, &desc, &id);
        if (r != CAELIX_OK) return undo(r);
        added.push_back(id);
        caelix_scene_set_entity_motion(scene, id, (e.flags & 2u) ? CAELIX_ENTITY_STATIC : CAELIX_ENTITY_DYNAMIC);
        r = upload_decoded(dec, org, scene, id, bricks);
        if (r != CAELIX_OK) return undo(r);
        if (ids) ids[i] = id;
    }
    return CAELIX_OK;
    CAELIX_GUARD_END
}

}  // extern "C"
