"""The .cxw world-file reader (caelix_world_*) on synthetic files: version gates and migrations
(versions 2 to 8), payload details (free lists and remapped brick ids, all-air bricks, extra slot
records, negative sector coordinates), and every read rule's error. The cases follow the
reference reader's tests (host-rs/caelix-cxw/tests/synthetic.rs); the files come from
caelix_b200/cxw.py."""
import struct

import numpy as np
import pytest

from caelix_b200 import cxw as W


def open_world(tmp_path, data: bytes, name="w.cxw"):
    import caelix_b200

    path = tmp_path / name
    path.write_bytes(data)
    return caelix_b200.WorldFile(str(path))


def open_error(tmp_path, data: bytes):
    import caelix_b200

    with pytest.raises(caelix_b200.CaelixError) as e:
        open_world(tmp_path, data)
    return e.value


def assert_decodes(f, index, sector):
    keys, blocks, summaries, voxels = f.decode(index)
    ek, eb, es, ev = W.expected_sector(sector)
    assert keys.tolist() == [list(k) for k in ek]
    assert blocks.tolist() == eb
    assert summaries.tolist() == es
    assert voxels == ev


def simple_sector(coord):
    return W.Sector(coord, [(0, W.brick(1, 512)), (4095, W.brick(7, 3))])


def test_v8_world_record_and_payload_details(tmp_path):
    s0 = W.Sector((0, 0, 0), [(5, W.brick(10, 512)), (17, W.brick(20, 100)), (300, [0] * 512),
                              (4095, W.brick(30, 1))], free=3, physics_slot_first=True)
    s1 = W.Sector((-1, 2, -3), [(1, W.brick(40, 200)), (2048, W.brick(50, 512))])
    e0 = W.Entity([s0, s1], require=0x0102, flags_byte=0x07, velocity=(1, 2, 3, 4, 5, 6), protected=1)
    e1 = W.Entity([simple_sector((4, 0, 0))], guid=bytes(range(100, 116)), flags_byte=1)
    w = W.World(8, [e0, e1], world_flags=1, player_position=(10.0, 20.0, 30.0), player_rotation=(0.1, 0.2, 0.3, 0.9))
    f = open_world(tmp_path, W.build(w))
    info = f.info()
    assert (info.version, info.has_player_pose, info.entity_count, info.sector_count) == (8, 1, 2, 3)
    assert list(info.player_position) == [10.0, 20.0, 30.0]
    assert np.allclose(list(info.player_rotation), [0.1, 0.2, 0.3, 0.9])
    ents = f.entities()
    assert bytes(ents[0].guid) == bytes(range(1, 17)) and bytes(ents[1].guid) == bytes(range(100, 116))
    assert ents[0].flags == 0x03  # the v6+ byte masked to HasBody | Static
    assert ents[0].is_protected == 1 and ents[0].require_update_flags == 0x0102
    assert list(ents[0].velocity) == [1, 2, 3, 4, 5, 6]
    assert list(ents[0].position) == [1.0, 2.0, 3.0] and list(ents[0].rotation) == [0.0, 0.0, 0.0, 1.0]
    assert (ents[0].sector_count, ents[1].sector_count) == (2, 1)
    secs = f.sectors()
    assert [(s.entity, tuple(s.coord)) for s in secs] == [(0, (0, 0, 0)), (0, (-1, 2, -3)), (1, (4, 0, 0))]
    assert_decodes(f, 0, s0)  # remapped ids, the all-air brick dropped, the physics slot skipped
    assert_decodes(f, 1, s1)  # negative coordinates
    keys, _, _, _ = f.decode(1)
    assert keys[0].tolist() == [-16 + 1, 32, -48]
    f.close()


def test_v7_without_pose(tmp_path):
    w = W.World(7, [W.Entity([simple_sector((0, 0, 0))])], world_flags=0, player_position=(5.0, 5.0, 5.0))
    f = open_world(tmp_path, W.build(w))
    assert f.info().has_player_pose == 0
    assert list(f.info().player_position) == [0.0, 0.0, 0.0]


@pytest.mark.parametrize("version", [3, 4, 5])
def test_legacy_flag_migration(tmp_path, version):
    # Legacy body state: 1 = static body, 2 = dynamic body, anything else = static, no body.
    ents = [W.Entity([], flags_byte=b, velocity=(9, 9, 9, 9, 9, 9), protected=1) for b in (0, 1, 2, 7)]
    f = open_world(tmp_path, W.build(W.World(version, ents)))
    got = f.entities()
    assert [e.flags for e in got] == [2, 3, 1, 2]
    for e in got:
        assert list(e.velocity) == ([9.0] * 6 if version >= 4 else [0.0] * 6)
        assert e.is_protected == (1 if version >= 5 else 0)


def test_v2_has_no_flags_byte(tmp_path):
    f = open_world(tmp_path, W.build(W.World(2, [W.Entity([simple_sector((1, 1, 1))])])))
    assert f.entities()[0].flags == 2  # static
    assert_decodes(f, 0, simple_sector((1, 1, 1)))


def test_legacy_magic_accepted(tmp_path):
    w = W.World(6, [W.Entity([simple_sector((0, 0, 0))])], magic=W.LEGACY_FILE_MAGIC)
    assert open_world(tmp_path, W.build(w)).info().version == 6


def base():
    return W.World(8, [W.Entity([simple_sector((0, 0, 0)), simple_sector((1, 0, 0))])])


def test_bad_magic(tmp_path):
    data = bytearray(W.build(base()))
    data[0:4] = struct.pack("<I", 0x12345678)
    e = open_error(tmp_path, bytes(data))
    assert e.code == 1 and "bad file magic 0x12345678" in e.log[-1]


def test_bad_flags(tmp_path):
    w = base()
    w.flags = 3
    e = open_error(tmp_path, W.build(w))
    assert e.code == 1 and "unsupported save flags 0x0003" in e.log[-1]


def test_unsupported_version(tmp_path):
    data = bytearray(W.build(base()))
    data[4:6] = struct.pack("<H", 9)
    e = open_error(tmp_path, bytes(data))
    assert e.code == 2 and "format version 9 is not supported" in e.log[-1]


def test_file_shorter_than_header(tmp_path):
    e = open_error(tmp_path, W.build(base())[:40])
    assert e.code == 1 and "truncated data reading header at offset 0" in e.log[-1]


def test_truncated_region_payload(tmp_path):
    data = W.build(base())
    e = open_error(tmp_path, data[:-10])
    assert e.code == 1 and "truncated data reading sector payload" in e.log[-1]


def test_truncated_region_preview(tmp_path):
    w = W.World(8, [W.Entity([simple_sector((0, 0, 0))])])
    data = W.build(w)
    secs_at = 64 + 29 + 4 + W.record_bytes(8)
    region_offset = struct.unpack_from("<Q", data, secs_at + 12)[0]
    e = open_error(tmp_path, data[:region_offset + 100])
    assert e.code == 1 and f"truncated data reading sector region at offset {region_offset}" in e.log[-1]


def test_truncated_entity_table(tmp_path):
    data = W.build(base())
    e = open_error(tmp_path, data[:64 + 29 + 4 + 20])
    assert e.code == 1 and "truncated data reading entity record" in e.log[-1]


def test_bad_region_size(tmp_path):
    data = bytearray(W.build(base()))
    at = 64 + 29 + 4 + W.record_bytes(8) + 20  # the first index entry's region size
    size = struct.unpack_from("<I", data, at)[0]
    struct.pack_into("<I", data, at, size + 1)
    e = open_error(tmp_path, bytes(data))
    assert e.code == 1 and f"region size is {size + 1}, expected {size}" in e.log[-1]


def test_duplicate_sector(tmp_path):
    w = W.World(8, [W.Entity([simple_sector((2, 3, 4)), simple_sector((2, 3, 4))])])
    e = open_error(tmp_path, W.build(w))
    assert e.code == 1 and "sector (2, 3, 4) appears twice" in e.log[-1]
    # The same coordinate in two entities is fine.
    w = W.World(8, [W.Entity([simple_sector((2, 3, 4))]), W.Entity([simple_sector((2, 3, 4))])])
    assert open_world(tmp_path, W.build(w), "ok.cxw").info().sector_count == 2


def test_bad_sector_magic_and_upload_error(tmp_path):
    import caelix_b200

    s = simple_sector((0, 0, 0))
    s.payload_magic = 0xDEADBEEF
    f = open_world(tmp_path, W.build(W.World(8, [W.Entity([s])])))  # opens: payloads are read on decode
    with pytest.raises(caelix_b200.CaelixError) as e:
        f.decode(0)
    assert e.value.code == 1 and "bad sector payload magic 0xDEADBEEF" in e.value.log[-1]


@pytest.mark.parametrize("counts", [(5000, 1, 4999), (4, 5, 0), (4, 2, 1)])
def test_bad_counts(tmp_path, counts):
    import caelix_b200

    s = simple_sector((0, 0, 0))
    s.counts = counts
    f = open_world(tmp_path, W.build(W.World(8, [W.Entity([s])])))
    with pytest.raises(caelix_b200.CaelixError) as e:
        f.decode(0)
    assert "invalid brick map counters" in e.value.log[-1]


def test_corrupt_deflate(tmp_path):
    import caelix_b200

    good = simple_sector((0, 0, 0))
    bad = simple_sector((1, 0, 0))
    bad.compressed = bytes([0xFF]) * 64  # an invalid block type
    cut = simple_sector((2, 0, 0))
    cut.compressed = W.deflate_raw(W.payload(cut))[:100]  # ends before its final block
    f = open_world(tmp_path, W.build(W.World(8, [W.Entity([good, bad, cut])])))
    assert_decodes(f, 0, good)
    for i in (1, 2):
        with pytest.raises(caelix_b200.CaelixError) as e:
            f.decode(i)
        assert e.value.code == 1 and "inflate failed" in e.value.log[-1]
    assert "deflate stream ends before its final block" in e.value.log[-1]


def test_payload_structure_errors(tmp_path):
    import caelix_b200

    short = simple_sector((0, 0, 0))
    short.truncate_payload = 1000
    stride = simple_sector((1, 0, 0))
    stride.block_stride = 3
    f = open_world(tmp_path, W.build(W.World(8, [W.Entity([short, stride])])))
    with pytest.raises(caelix_b200.CaelixError) as e:
        f.decode(0)
    assert "truncated data reading payload slot data" in e.value.log[-1]
    with pytest.raises(caelix_b200.CaelixError) as e:
        f.decode(1)
    assert "Block slot stride is not 2" in e.value.log[-1]


def test_large_payload_grows_inflate_buffer(tmp_path):
    rng = np.random.default_rng(3)
    bricks = [(bi, [int(v) for v in rng.integers(0, 1 << 16, 512, dtype=np.uint16)]) for bi in range(0, 4096, 2)]
    s = W.Sector((3, -2, 1), bricks)
    f = open_world(tmp_path, W.build(W.World(8, [W.Entity([s])])))
    assert_decodes(f, 0, s)


def test_scene_round_trip(tmp_path):
    """A generated scene written as a world file (caelix_b200.cxw.from_voxel_scene, keys moved to
    negative sectors) decodes back to its non-air bricks, sector by sector."""
    from caelix_b200 import workloads

    vs = workloads.noise_world(grid_bricks=(20, 12, 18), brick_occupancy=0.4, emissive_fraction=0.05, seed=21)
    vox = vs.voxels.copy()
    vox[::7] = 0  # all-air bricks are written and dropped by the reader
    vs = workloads.VoxelScene(vs.grid, vs.keys, vox, vs.power, vs.albedo, vs.camera, vs.group_shift)
    shift = (-37, 5, -16)
    f = open_world(tmp_path, W.from_voxel_scene(vs, shift))
    got = {}
    for i in range(f.info().sector_count):
        keys, blocks, summaries, _ = f.decode(i)
        for k, b in zip(keys, blocks):
            got[tuple(int(v) for v in k)] = b
    keep = (vs.voxels != 0).any(axis=1)
    want = {tuple(int(v) + s for v, s in zip(k, shift)): b for k, b, kp in zip(vs.keys, vs.voxels, keep) if kp}
    assert got.keys() == want.keys()
    assert all(np.array_equal(got[k], want[k]) for k in want)
