"""A world file into a scene: caelix_world_upload_entity decodes a .cxw world written from a
generated scene (sectors of 16^3 bricks, moved to negative sector coordinates, or spread wider than
1024 bricks) and uploads its keys unchanged, as the reference's loader does; the flushed scene
equals the oracle's build of the same bricks."""
import numpy as np
import pytest

from caelix_b200 import cxw as W
import oracle_lib
from caelix_b200 import workloads
from test_trace_gpu import assert_scene_equal

pytestmark = pytest.mark.gpu


def test_world_file_into_scene(cuda_device, oracle, tmp_path):
    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(20, 12, 18), brick_occupancy=0.4, emissive_fraction=0.05, seed=21)
    shift = (-37, 5, -16)
    path = tmp_path / "world.cxw"
    path.write_bytes(W.from_voxel_scene(vs, shift))
    f = caelix_b200.WorldFile(str(path))
    scene = caelix_b200.Scene.for_voxel_scene(cuda_device, vs)
    origin, bricks = f.upload_entity(0, scene, threads=4)
    keep = (vs.voxels != 0).any(axis=1)  # the reader drops all-air bricks
    keys = vs.keys[keep]
    assert bricks == int(keep.sum())
    assert origin == (0, 0, 0)  # the keys go in as the file holds them
    exp = in_box_order(vs, keys + np.array(shift, np.int32), vs.voxels[keep], vs.power[keep])
    scene.set_brick_power(exp.keys, exp.power)
    scene.flush()
    assert_scene_equal(scene, oracle_lib.OracleScene(oracle, exp), exp)
    scene.close()
    f.close()


def in_box_order(src, keys, voxels, power):
    """A VoxelScene of the bricks in increasing linear index of the box of their keys (the order of
    the flushed scene's tables)."""
    keys = keys.astype(np.int32)
    origin, grid = workloads.scene_grid(keys, src.group_shift)
    k = keys.astype(np.int64) - np.array(origin, np.int64)
    lin = k[:, 0] + grid[0] * (k[:, 1] + grid[1] * k[:, 2])
    o = np.argsort(lin, kind="stable")
    return workloads.VoxelScene(tuple(int(v) for v in grid), keys[o], voxels[o], power[o], src.albedo, src.camera,
                                src.group_shift)


def test_world_wider_than_1024_bricks(cuda_device, oracle, tmp_path):
    """A world of two clusters 1,200 bricks apart, one at negative keys: loaded unchanged and
    flushed, its tables equal the oracle's."""
    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(6, 5, 6), brick_occupancy=0.5, emissive_fraction=0.1, seed=29)
    half = vs.brick_count // 2
    keys = vs.keys.copy()
    keys[:half] += np.array([-600, -3, 2], np.int32)
    keys[half:] += np.array([600, 1, -40], np.int32)
    path = tmp_path / "wide.cxw"
    path.write_bytes(W.build(W.World(8, [W.Entity(W.sectors_of(keys, vs.voxels))])))
    f = caelix_b200.WorldFile(str(path))
    scene = caelix_b200.Scene.for_voxel_scene(cuda_device, vs)
    origin, bricks = f.upload_entity(0, scene, threads=2)
    keep = (vs.voxels != 0).any(axis=1)
    assert origin == (0, 0, 0) and bricks == int(keep.sum())
    exp = in_box_order(vs, keys[keep], vs.voxels[keep], vs.power[keep])
    assert exp.keys[:, 0].max() - exp.keys[:, 0].min() > 1024
    scene.set_brick_power(exp.keys, exp.power)
    scene.flush()
    assert_scene_equal(scene, oracle_lib.OracleScene(oracle, exp), exp)
    scene.close()
    f.close()


def rows64(q):
    """Rotation rows of a quaternion in double, as the library computes them."""
    import math

    q = [float(np.float32(v)) for v in q]
    n = math.sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3])
    x, y, z, w = q[0] / n, q[1] / n, q[2] / n, q[3] / n
    return [1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - z * w), 2.0 * (x * z + y * w),
            2.0 * (x * y + z * w), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - x * w),
            2.0 * (x * z - y * w), 2.0 * (y * z + x * w), 1.0 - 2.0 * (x * x + y * y)]


def test_world_load_with_entities(cuda_device, oracle, tmp_path):
    """caelix_world_load: file entity 0 (rotated and moved) becomes the scene's world, entity 1 a
    scene entity whose transform is expressed in the world's frame; the render equals the oracle's
    with the same bricks and the transform computed here the library's way (double, then float)."""
    import math

    import caelix_b200
    from test_entities_oracle import entity_bricks
    from test_trace_gpu import assert_radiance_close

    vs = workloads.noise_world(grid_bricks=(10, 8, 9), brick_occupancy=0.4, emissive_fraction=0.06, seed=23)
    ent = entity_bricks(grid=(2, 2, 2), seed=7)
    shift0, shift1 = np.array([-37, 5, -16]), np.array([3, -5, 20])
    q0, p0 = (0.05, -0.1, 0.02, 0.99), (4.0, -2.5, 1.0)
    q1, p1 = (0.2, 0.3, -0.1, 0.92), (60.0, 40.0, -30.0)
    world_file = W.World(8, [W.Entity(W.sectors_of(vs.keys + shift0, vs.voxels), position=p0, rotation=q0, flags_byte=2),
                             W.Entity(W.sectors_of(ent.keys + shift1, ent.voxels), guid=bytes(range(16, 32)),
                                      position=p1, rotation=q1, flags_byte=0)])
    path = tmp_path / "entities.cxw"
    path.write_bytes(W.build(world_file))
    f = caelix_b200.WorldFile(str(path))
    scene = caelix_b200.Scene.for_voxel_scene(cuda_device, vs)
    ids, bricks = f.load(scene, threads=4)
    assert ids == [0, 1]
    keep0 = (vs.voxels != 0).any(axis=1)
    keep1 = (ent.voxels != 0).any(axis=1)
    assert bricks == int(keep0.sum() + keep1.sum())
    # The keys go in unchanged (no origin move).
    world = in_box_order(vs, vs.keys[keep0] + shift0, vs.voxels[keep0], vs.power[keep0])
    # The loader sets no power: the entity's bricks keep the default power 1 (they emit).
    body = in_box_order(ent, ent.keys[keep1] + shift1, ent.voxels[keep1], np.ones(int(keep1.sum()), np.float32))
    scene.set_brick_power(world.keys, world.power)
    scene.flush()
    assert_scene_equal(scene, oracle_lib.OracleScene(oracle, world), world)

    # The entity's transform in the world's frame, the library's arithmetic.
    r0 = rows64(q0)
    v = [(float(np.float32(p1[k])) - float(np.float32(p0[k]))) for k in range(3)]
    pos = tuple(np.float32(r0[k] * v[0] + r0[3 + k] * v[1] + r0[6 + k] * v[2]) for k in range(3))
    a = [float(np.float32(c)) for c in q0]
    n0 = math.sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2] + a[3] * a[3])
    ax, ay, az, aw = -a[0] / n0, -a[1] / n0, -a[2] / n0, a[3] / n0
    bx, by, bz, bw = (float(np.float32(c)) for c in q1)
    rot = (np.float32(aw * bx + ax * bw + ay * bz - az * by), np.float32(aw * by - ax * bz + ay * bw + az * bx),
           np.float32(aw * bz + ax * by - ay * bx + az * bw), np.float32(aw * bw - ax * bx - ay * by - az * bz))

    cam = workloads.look_at(np.array(pos, np.float64) + np.array([-30.0, 20.0, -30.0]), np.array(pos, np.float64))
    osc = oracle_lib.OracleScene(oracle, world)
    osc.set_entities([(oracle_lib.OracleScene(oracle, body), rot, pos)], motions=[1])  # its Static flag is clear
    r = caelix_b200.Renderer(cuda_device, scene)
    import torch

    out = torch.zeros(48 * 64 * 3, dtype=torch.float32, device="cuda")
    r.render(out, 64, 48, cam, bounces=3, seed=4, spp=2)
    st = r.stats()
    gpu = out.cpu().numpy().reshape(48, 64, 3)
    ref, rays = osc.render(64, 48, spp=2, bounces=3, seed=4, threads=8, camera=cam)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)
    hits = 0
    for py in range(0, 48, 4):
        for px in range(0, 64, 4):
            d = np.array(cam["right"]) * ((px + 0.5) / 64 * 2 - 1) * cam["tan_half_fov_y"] * cam["aspect"] + \
                np.array(cam["up"]) * (1 - (py + 0.5) / 48 * 2) * cam["tan_half_fov_y"] + np.array(cam["forward"])
            h = osc.trace(np.array(cam["position"], np.float32), (d / np.linalg.norm(d)).astype(np.float32))
            hits += bool(h.hit and (h.attrib & 0x8000))
    assert hits > 0  # the entity is in view
    r.close()
    scene.close()
    f.close()
