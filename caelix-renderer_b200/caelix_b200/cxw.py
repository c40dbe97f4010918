"""Writer of .cxw world files (format version 8 and older): synthetic worlds for the reader's tests
and generated scenes saved as world files (`from_voxel_scene`).

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
from dataclasses import dataclass

import numpy as np

FILE_MAGIC = 0x534C5843
LEGACY_FILE_MAGIC = 0x534C5856
PAYLOAD_MAGIC = 0x32535856


def deflate_raw(raw: bytes) -> bytes:
    c = zlib.compressobj(1, zlib.DEFLATED, -15)
    return c.compress(raw) + c.flush()


def preview_word(bi):
    """A recognisable preview word per brick index (an int or an array of them)."""
    return 0xA5A00000 | (bi << 8) | 0x0F


@dataclass
class Sector:
    coord: tuple
    bricks: object  # [(brick index 0..4095, 512 uint16 values)], or (indices [n], values [n, 512])
    free: int = 0  # free brick ids, below the used ones (so the used ids are remapped)
    physics_slot_first: bool = False  # a stride-1 slot record before the block slot
    payload_magic: int = PAYLOAD_MAGIC
    compressed: bytes | None = None  # replaces the deflated payload
    counts: tuple | None = None  # (capacity, count, free) written instead of the true ones
    block_stride: int = 2
    truncate_payload: int = 0  # bytes cut from the end of the raw payload

    def arrays(self):
        """(brick indices int64 [n], values uint16 [n, 512]) of the bricks, in list order."""
        if isinstance(self.bricks, tuple):
            return self.bricks
        bi = np.array([b for b, _ in self.bricks], np.int64)
        values = np.array([v for _, v in self.bricks], np.uint16).reshape(len(self.bricks), 512)
        return bi, values


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
    bis, values = s.arrays()
    n = len(bis)
    capacity = n + s.free
    indices = np.full(4096, -1, np.int16)
    indices[bis] = capacity - 1 - np.arange(n)  # used ids from the top down
    cap, cnt, fr = s.counts if s.counts else (capacity, n, s.free)
    out = bytearray(struct.pack("<4I", s.payload_magic, cap, cnt, fr))
    out += indices.astype("<i2").tobytes()
    out += np.arange(s.free, dtype="<i2").tobytes()
    out += struct.pack("<H", 1) + bytes(4096 * 2)
    out += struct.pack("<I", 2 if s.physics_slot_first else 1)
    if s.physics_slot_first:
        out += struct.pack("<BH", 1, 1) + bytes([0x7E]) * (capacity * 512)
    out += struct.pack("<BH", 0, s.block_stride)
    if s.block_stride == 2:
        block = np.full((capacity, 512), 0xFFFF, "<u2")  # free ids hold values that must never be read
        block[capacity - 1 - np.arange(n)] = values
        out += block.tobytes()
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
            preview = np.zeros(4096, "<u4")
            bis = s.arrays()[0]
            preview[bis] = preview_word(bis.astype(np.uint32))
            regions += preview.tobytes()
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


def sectors_of(keys, voxels) -> list:
    """The sectors (16^3 bricks) holding bricks of the given keys and values, in coordinate order."""
    keys = np.asarray(keys, np.int64)
    coords = keys // 16
    local = keys - coords * 16
    bi = local[:, 0] + 16 * (local[:, 1] + 16 * local[:, 2])
    order = np.lexsort((bi, coords[:, 0], coords[:, 1], coords[:, 2]))
    c = coords[order]
    starts = np.flatnonzero(np.r_[True, (c[1:] != c[:-1]).any(axis=1)])
    ends = np.r_[starts[1:], len(order)]
    voxels = np.asarray(voxels, np.uint16)
    return [Sector(tuple(int(v) for v in c[a]), (bi[order[a:b]], voxels[order[a:b]])) for a, b in zip(starts, ends)]


def from_voxel_scene(vs, shift=(0, 0, 0), version: int = 8) -> bytes:
    """A .cxw file holding the bricks of a workloads.VoxelScene as one static entity, the brick
    keys moved by `shift` bricks (sectors of 16^3 bricks; all-air bricks are written too, the
    reader drops them)."""
    keys = np.asarray(vs.keys, np.int64) + np.asarray(shift, np.int64)
    return build(World(version, [Entity(sectors_of(keys, vs.voxels), flags_byte=2)]))
