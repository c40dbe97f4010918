"""Writer of synthetic .cxw world files for the reader tests (test infrastructure).

The layout follows the format's read rules (little-endian throughout):
  header (64 bytes): magic u32 ("CXLS", legacy "VXLS"), version u16, flags u16 (1 = Deflate),
      entity table offset u64, zero padding;
  entity table: [version >= 7: world flags u8, player position 3 x f32, rotation 4 x f32],
      entity count u32, then per entity: guid 16 bytes, position 3 x f32, rotation 4 x f32,
      require-update flags u16, [v >= 3: flags / legacy body state u8], [v >= 4: velocity 6 x f32],
      [v >= 5: protected u8], sector index offset u64, sector count u32;
  sector index (per entity): coord 3 x i32, region offset u64, region size u32;
  region: preview 4096 x u32, payload size u32, raw-deflate payload; region size = 16388 + size;
  payload: magic "VXS2", capacity, count, free count (u32 each), brick index table 4096 x i16
      (-1 = no brick, else a brick id), free list (free count x i16), require-update flags
      (2 + 4096 x 2 bytes), slot record count u32, slot records: id u8, stride u16, then
      capacity x 512 x stride bytes (slot 0 = the block values, stride 2).
This writer puts the entity table first and the regions last, so a reader that follows the
offsets (and not the order of the reference's writer) is what the tests check.
"""
from __future__ import annotations

import struct
import zlib
from dataclasses import dataclass, field

FILE_MAGIC = 0x534C5843
LEGACY_FILE_MAGIC = 0x534C5856
PAYLOAD_MAGIC = 0x32535856


def deflate_raw(raw: bytes) -> bytes:
    c = zlib.compressobj(1, zlib.DEFLATED, -15)
    return c.compress(raw) + c.flush()


def preview_word(bi: int) -> int:
    """A recognisable preview word per brick index."""
    return 0xA5A00000 | (bi << 8) | 0x0F


@dataclass
class Sector:
    coord: tuple
    bricks: list  # (brick index in the sector 0..4095, 512 uint16 values)
    free: int = 0  # free brick ids, below the used ones (so the used ids are remapped)
    physics_slot_first: bool = False  # a stride-1 slot record before the block slot
    payload_magic: int = PAYLOAD_MAGIC
    compressed: bytes | None = None  # replaces the deflated payload
    counts: tuple | None = None  # (capacity, count, free) written instead of the true ones
    block_stride: int = 2
    truncate_payload: int = 0  # bytes cut from the end of the raw payload


@dataclass
class Entity:
    sectors: list
    guid: bytes = bytes(range(1, 17))
    position: tuple = (1.0, 2.0, 3.0)
    rotation: tuple = (0.0, 0.0, 0.0, 1.0)
    require: int = 0
    flags_byte: int = 2
    velocity: tuple = (0.0,) * 6
    protected: int = 0


@dataclass
class World:
    version: int
    entities: list
    magic: int = FILE_MAGIC
    flags: int = 1
    world_flags: int = 0
    player_position: tuple = (0.0, 0.0, 0.0)
    player_rotation: tuple = (0.0, 0.0, 0.0, 1.0)


def payload(s: Sector) -> bytes:
    n = len(s.bricks)
    capacity = n + s.free
    indices = [-1] * 4096
    for i, (bi, _) in enumerate(s.bricks):
        indices[bi] = capacity - 1 - i  # used ids from the top down
    cap, cnt, fr = s.counts if s.counts else (capacity, n, s.free)
    out = bytearray(struct.pack("<4I", s.payload_magic, cap, cnt, fr))
    out += struct.pack("<4096h", *indices)
    out += struct.pack(f"<{s.free}h", *range(s.free))
    out += struct.pack("<H", 1) + bytes(4096 * 2)
    out += struct.pack("<I", 2 if s.physics_slot_first else 1)
    if s.physics_slot_first:
        out += struct.pack("<BH", 1, 1) + bytes([0x7E]) * (capacity * 512)
    out += struct.pack("<BH", 0, s.block_stride)
    block = [0xFFFF] * (capacity * 512)  # free ids hold values that must never be read
    for i, (_, values) in enumerate(s.bricks):
        bid = capacity - 1 - i
        block[bid * 512:(bid + 1) * 512] = [int(v) for v in values]
    if s.block_stride == 2:
        out += struct.pack(f"<{capacity * 512}H", *block)
    else:
        out += bytes(capacity * 512 * s.block_stride)
    if s.truncate_payload:
        out = out[:-s.truncate_payload]
    return bytes(out)


def record_bytes(version: int) -> int:
    return 16 + 28 + 2 + (version >= 3) + (24 if version >= 4 else 0) + (version >= 5) + 12


def build(w: World) -> bytes:
    """The file bytes: header | world record + entity table | per entity: sector index, regions."""
    table_offset = 64
    table_len = (29 if w.version >= 7 else 0) + 4 + len(w.entities) * record_bytes(w.version)
    body = bytearray()
    index_offsets = []
    for e in w.entities:
        index_offset = table_offset + table_len + len(body)
        index_offsets.append(index_offset)
        regions_start = index_offset + 24 * len(e.sectors)
        index = bytearray()
        regions = bytearray()
        for s in e.sectors:
            compressed = s.compressed if s.compressed is not None else deflate_raw(payload(s))
            region_offset = regions_start + len(regions)
            preview = [0] * 4096
            for bi, _ in s.bricks:
                preview[bi] = preview_word(bi)
            regions += struct.pack("<4096I", *preview)
            regions += struct.pack("<I", len(compressed)) + compressed
            index += struct.pack("<3iQI", *s.coord, region_offset, 16388 + len(compressed))
        body += index + regions
    out = bytearray(struct.pack("<IHHQ", w.magic, w.version, w.flags, table_offset))
    out += bytes(64 - len(out))
    if w.version >= 7:
        out += struct.pack("<B3f4f", w.world_flags, *w.player_position, *w.player_rotation)
    out += struct.pack("<I", len(w.entities))
    for e, io in zip(w.entities, index_offsets):
        out += e.guid + struct.pack("<3f4fH", *e.position, *e.rotation, e.require)
        if w.version >= 3:
            out += struct.pack("<B", e.flags_byte)
        if w.version >= 4:
            out += struct.pack("<6f", *e.velocity)
        if w.version >= 5:
            out += struct.pack("<B", e.protected)
        out += struct.pack("<QI", io, len(e.sectors))
    assert len(out) == table_offset + table_len
    return bytes(out + body)


def brick(seed: int, non_zero: int) -> list:
    """512 values: the first `non_zero` opaque (0x8000 | ...), the rest air."""
    return [((seed + i) & 0xFFFF) | 0x8000 if i < non_zero else 0 for i in range(512)]


def expected_sector(s: Sector):
    """The decode the reader must give: (keys, blocks, summaries, non-zero count) of the
    non-air bricks in ascending brick index."""
    keys, blocks, summaries, voxels = [], [], [], 0
    for bi, values in sorted(s.bricks, key=lambda t: t[0]):
        nz = sum(1 for v in values if v)
        if nz == 0:
            continue
        voxels += nz
        keys.append((s.coord[0] * 16 + (bi & 15), s.coord[1] * 16 + ((bi >> 4) & 15), s.coord[2] * 16 + (bi >> 8)))
        blocks.append(list(values))
        summaries.append(preview_word(bi))
    return keys, blocks, summaries, voxels
