"""The scenes, cameras and CPU expectations of two of the reference's own known-answer tests of the
trace path, restated (test infrastructure):

* the voxel id test (tests/trace_test.cpp:3596-3730 FloorVoxel / CheckVoxelIds and :3735-3945): a
  grey floor of 8 x 8 bricks at brick y = -1 (voxels x, z in [0, 64), top layer y = -1) in the packed
  encoding, a camera 12 above the floor's -X edge looking straight down with a 60 degree vertical
  field of view, 256 x 256 pixels. The CPU expectation of every pixel is the floor voxel under the
  unjittered centre ray, computed in double: floor(wx), -1, floor(wz), or a miss for wx < 0 (with
  entity B, the same bricks turned 180 degrees about Y at (0, 0, 64), wx in [-64, 0) is B's voxel
  (floor(-wx), -1, floor(64 - wz))); pixels within 1e-3 of a voxel border are ambiguous;
* the one-bounce energy test (tests/trace_test.cpp:1116-1288 UploadRoom, LookDown,
  CeilingHitProbability): the same floor under an emissive ceiling of 8 x 8 bricks at brick y = 3
  (packed code 0x4000 | rgb4 15/15/15, strength 0: emission 1), a camera at (32, 12, 32) looking down
  with a 30 degree field of view, black sky, one bounce. The mean of the centre pixels is the floor
  albedo times the probability that a cosine-distributed direction from a uniform point of the
  floor square under them reaches the ceiling, a CPU Monte Carlo estimate.
The floor's albedo is the packed code's rgb5 15/31 in fp32 here (the reference compares after its
composite quantizes the albedo target to 8 bits)."""
import math

import numpy as np

from caelix_b200 import workloads

SIZE = 256
GREY_FLOOR = 0x8000 | (15 << 10) | (15 << 5) | 15  # rgb5 15/31
WHITE_EMITTER = 0x4000 | (15 << 10) | (15 << 6) | (15 << 2)  # rgb4 1, strength 0: emission 1
CEILING_Y = 24.0
ROOM_SIZE = 64.0
CAMERA_HEIGHT = 12.0
FLOOR_ALBEDO = np.float32(15.0) / np.float32(31.0)


def _bricks(y, value):
    keys = np.array([[x, y, z] for z in range(8) for x in range(8)], np.int32)
    return keys, np.full((len(keys), 512), value, np.uint16)


def _sorted_scene(keys, voxels, camera, power=None, min_emission=20.0, lights=False):
    """A packed-encoding VoxelScene of the bricks in increasing linear index of their box."""
    origin, grid = workloads.scene_grid(keys, 4)
    k = keys.astype(np.int64) - np.array(origin)
    lin = k[:, 0] + grid[0] * (k[:, 1] + grid[1] * k[:, 2])
    o = np.argsort(lin, kind="stable")
    power = np.ones(len(keys), np.float32) if power is None else power
    return workloads.VoxelScene(grid, keys[o], voxels[o], power[o], None, camera, 4,
                                encoding=workloads.ENCODING_PACKED, min_emission=min_emission, lights=lights)


def look_down(x, height, z, fov_deg):
    """LookDown / LookDownFrom: right +X, up +Z, forward -Y, aspect 1."""
    return {
        "position": np.array([x, height, z], np.float32),
        "right": np.array([1.0, 0.0, 0.0], np.float32),
        "up": np.array([0.0, 0.0, 1.0], np.float32),
        "forward": np.array([0.0, -1.0, 0.0], np.float32),
        "tan_half_fov_y": np.float32(math.tan(np.float32(fov_deg / 2.0) * np.float32(3.14159265) / np.float32(180.0))),
        "aspect": np.float32(1.0),
    }


def floor_scene():
    """UploadFloor with the voxel id test's camera LookDown60(0, 12, 32)."""
    keys, voxels = _bricks(-1, GREY_FLOOR)
    return _sorted_scene(keys, voxels, look_down(0.0, 12.0, 32.0, 60.0))


def room_scene(lights=False, min_emission=0.5):
    """UploadRoom with the energy test's camera LookDown()."""
    fk, fv = _bricks(-1, GREY_FLOOR)
    ck, cv = _bricks(3, WHITE_EMITTER)
    return _sorted_scene(np.concatenate([fk, ck]), np.concatenate([fv, cv]),
                         look_down(32.0, CAMERA_HEIGHT, 32.0, 30.0), min_emission=min_emission, lights=lights)


# Entity B of the voxel id test: 180 degrees about Y, origin at (0, 0, 64).
ENTITY_B_POSITION = (0.0, 0.0, 64.0)
ENTITY_B_ROTATION = (0.0, 1.0, 0.0, 0.0)


def floor_voxel(camera, px, py, entity_b=False):
    """FloorVoxel: ("ambiguous",), ("miss",) or ("hit", entity, x, y, z) (entity-local voxel)."""
    ndc_x = (px + 0.5) / SIZE * 2.0 - 1.0
    ndc_y = 1.0 - (py + 0.5) / SIZE * 2.0
    height = float(camera["position"][1])
    tan = float(camera["tan_half_fov_y"])
    wx = float(camera["position"][0]) + ndc_x * tan * float(camera["aspect"]) * height
    wz = float(camera["position"][2]) + ndc_y * tan * height

    def near_integer(v):
        return abs(v - round(v)) < 1e-3

    if near_integer(wx) or near_integer(wz):
        return ("ambiguous",)
    assert 0.0 < wz < 64.0 and wx < 64.0
    if wx >= 0.0:
        return ("hit", 0, int(math.floor(wx)), -1, int(math.floor(wz)))
    if not entity_b or wx < -64.0:
        return ("miss",)
    return ("hit", 1, int(math.floor(-wx)), -1, int(math.floor(64.0 - wz)))


def _avalanche(v):
    v ^= v >> 16
    v = (v * 0x7FEB352D) & 0xFFFFFFFF
    v ^= v >> 15
    v = (v * 0x846CA68B) & 0xFFFFFFFF
    v ^= v >> 16
    return v


def voxel_key(entity, x, y, z):
    """The voxel id of (entity, voxel): VoxelIdWord with the two seeds (two words)."""
    words = []
    for seed in (0x9E3779B9, 0x85EBCA6B):
        h = _avalanche(seed ^ entity)
        for c in (x, y, z):
            h = _avalanche(h ^ (c & 0xFFFFFFFF))
        words.append(0xFFFFFFFE if h == 0xFFFFFFFF else h)
    return tuple(words)


def check_voxel_ids(ids, camera, entity_b=False):
    """CheckVoxelIds: one key per CPU voxel and one voxel per key, the miss value exactly on the
    misses; here also every key equal to the hash of its CPU voxel. Returns the number of keys."""
    keys_of_voxel, voxels_of_key = {}, {}
    bad_misses = wrong_key = 0
    for y in range(SIZE):
        for x in range(SIZE):
            v = floor_voxel(camera, x, y, entity_b)
            key = (int(ids[y, x, 0]), int(ids[y, x, 1]))
            if v[0] == "ambiguous":
                continue
            if v[0] == "miss":
                bad_misses += key != (0xFFFFFFFF, 0xFFFFFFFF)
                continue
            if 0xFFFFFFFF in key:
                bad_misses += 1
                continue
            keys_of_voxel.setdefault(v[1:], set()).add(key)
            voxels_of_key.setdefault(key, set()).add(v[1:])
            wrong_key += key != voxel_key(*v[1:])
    assert bad_misses == 0, bad_misses
    assert all(len(k) == 1 for k in keys_of_voxel.values())
    assert all(len(v) == 1 for v in voxels_of_key.values())
    assert len(keys_of_voxel) == len(voxels_of_key)
    assert wrong_key == 0, wrong_key
    return len(voxels_of_key)


def ceiling_hit_probability(half_extent, samples=2_000_000, seed=42):
    """CeilingHitProbability: the fraction of cosine-distributed directions from uniform points of
    the floor square [32 - h, 32 + h]^2 (y = 0) that reach the ceiling's bottom face (y = 24, x and z
    in [0, 64)); numpy's generator instead of the reference's mt19937_64."""
    rng = np.random.default_rng(seed)
    px = 32.0 + (rng.random(samples) * 2.0 - 1.0) * half_extent
    pz = 32.0 + (rng.random(samples) * 2.0 - 1.0) * half_extent
    r1 = rng.random(samples)
    phi = 2.0 * math.pi * rng.random(samples)
    s = np.sqrt(r1)
    dx, dz = s * np.cos(phi), s * np.sin(phi)
    dy = np.sqrt(np.maximum(0.0, 1.0 - r1))
    ok = dy > 0.0
    t = CEILING_Y / np.where(ok, dy, 1.0)
    x, z = px + dx * t, pz + dz * t
    hit = ok & (x >= 0.0) & (x < ROOM_SIZE) & (z >= 0.0) & (z < ROOM_SIZE)
    return float(hit.mean())


def half_extent(size, camera):
    """The floor half extent under the centre `size` pixels of the 256-pixel image."""
    return size / SIZE * float(camera["tan_half_fov_y"]) * CAMERA_HEIGHT


def centre_window(size):
    lo = (SIZE - size) // 2
    return (lo, lo, lo + size, lo + size)
