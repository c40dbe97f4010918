"""The CUDA path (through the C ABI) on two of the reference's own known answers of the trace path
(tests/trace_test.cpp; the scenes and CPU expectations are restated in reference_scenes.py), and on
the drop-in semantics they need:

* the voxel id target: every pixel's key is the CPU floor voxel's (one key per voxel, the miss value
  on the misses), bit-identical to the oracle's image, also with entity B (180 degrees about Y) and
  with voxel_id_tmax; the floor is at brick y = -1 in the packed encoding;
* the one-bounce energy test: a scene lit only by its materials' emission (the packed emitter code,
  no brick power set), without and with the light tree; the centre mean within 3 % of the CPU Monte
  Carlo estimate, the raw 1 spp frame only 0 or the albedo, and the frame equal to the oracle's;
* brick keys across the whole range: a world at negative and far keys equals the oracle bit for
  bit (tables, light tree, radiance)."""
import numpy as np
import pytest

import oracle_lib
import reference_scenes as R
from caelix_b200 import workloads
from test_trace_gpu import assert_radiance_close, assert_scene_equal

pytestmark = pytest.mark.gpu


def render_ids(cuda_device, scene, camera, tmax=0.0):
    import torch

    import caelix_b200

    r = caelix_b200.Renderer(cuda_device, scene)
    out = torch.zeros(R.SIZE * R.SIZE * 3, dtype=torch.float32, device="cuda")
    ids = torch.full((R.SIZE * R.SIZE * 2,), 7, dtype=torch.int32, device="cuda")
    r.render(out, R.SIZE, R.SIZE, camera, bounces=0, seed=1, spp=1, voxel_id=ids, voxel_id_tmax=tmax)
    res = ids.cpu().numpy().view(np.uint32).reshape(R.SIZE, R.SIZE, 2)
    r.close()
    return res


def test_voxel_id_floor(cuda_device, oracle):
    import caelix_b200

    vs = R.floor_scene()
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    osc = oracle_lib.OracleScene(oracle, vs)
    assert_scene_equal(scene, osc, vs)
    ids = render_ids(cuda_device, scene, vs.camera)
    assert R.check_voxel_ids(ids, vs.camera) > 50
    _, _, ref = osc.render(R.SIZE, R.SIZE, bounces=0, light_nee=False, threads=8, voxel_ids=True)
    assert np.array_equal(ids, ref)
    assert (render_ids(cuda_device, scene, vs.camera, 6.0) == 0xFFFFFFFF).all()
    assert np.array_equal(render_ids(cuda_device, scene, vs.camera, 1000.0), ids)

    # Entity B: the same bricks turned 180 degrees about Y at (0, 0, 64).
    e = scene.add_entity(R.ENTITY_B_POSITION, R.ENTITY_B_ROTATION)
    scene.upload_bricks(vs.keys, vs.voxels, entity=e)
    scene.flush()
    ids = render_ids(cuda_device, scene, vs.camera)
    R.check_voxel_ids(ids, vs.camera, entity_b=True)
    b = oracle_lib.OracleScene(oracle, vs)
    osc.set_entities([(b, R.ENTITY_B_ROTATION, R.ENTITY_B_POSITION)], ids=[e])
    _, _, ref = osc.render(R.SIZE, R.SIZE, bounces=0, light_nee=False, threads=8, voxel_ids=True)
    assert np.array_equal(ids, ref)
    osc.set_entities([])
    b.close()
    osc.close()
    scene.close()


@pytest.mark.parametrize("lights", [False, True])
def test_one_bounce_under_the_emissive_ceiling(cuda_device, oracle, lights):
    import torch

    import caelix_b200

    vs = R.room_scene(lights=lights)
    scene = caelix_b200.Scene(cuda_device, 4, workloads.ENCODING_PACKED)
    # The reference's defaults: no brick power set (every brick 1), the built-in packed table.
    scene.upload_bricks(vs.keys, vs.voxels)
    if lights:
        scene.set_light_options(True, 0.5)
    scene.flush()
    assert (scene.light_stats().light_bricks > 0) == lights
    osc = oracle_lib.OracleScene(oracle, vs)
    assert_scene_equal(scene, osc, vs)
    r = caelix_b200.Renderer(cuda_device, scene)
    out = torch.zeros(R.SIZE * R.SIZE * 3, dtype=torch.float32, device="cuda")
    r.render(out, R.SIZE, R.SIZE, vs.camera, bounces=1, seed=1000, spp=2048)
    img = out.cpu().numpy().reshape(R.SIZE, R.SIZE, 3)
    x0, y0, x1, y1 = R.centre_window(32)
    cpu = float(R.FLOOR_ALBEDO) * R.ceiling_hit_probability(R.half_extent(32, vs.camera))
    assert abs(img[y0:y1, x0:x1, 0].astype(np.float64).mean() / cpu - 1.0) < 0.03
    # The oracle on a few pixels of the same frame.
    win = (120, 120, 128, 124)
    ref, _ = osc.render(R.SIZE, R.SIZE, spp=2048, bounces=1, seed=1000, light_nee=lights, window=win, threads=8)
    assert_radiance_close(img[120:124, 120:128], ref[120:124, 120:128])
    if not lights:
        r.render(out, R.SIZE, R.SIZE, vs.camera, bounces=1, seed=77, spp=1)
        raw = out.cpu().numpy().reshape(R.SIZE, R.SIZE, 3)[64:192, 64:192, 0]
        assert np.isin(raw, [0.0, R.FLOOR_ALBEDO]).all()
        cpu128 = float(R.FLOOR_ALBEDO) * R.ceiling_hit_probability(R.half_extent(128, vs.camera))
        assert abs(raw.astype(np.float64).mean() / cpu128 - 1.0) < 0.05
    r.close()
    osc.close()
    scene.close()


def test_keys_across_the_range(cuda_device, oracle):
    """The plain scene's generator moved to negative keys, and a second cluster of bricks far away
    (the box still within the bitmap limit): tables, light tree and radiance equal the oracle's."""
    import caelix_b200
    from test_trace_gpu import render_both

    base = workloads.noise_world(grid_bricks=(10, 8, 12), brick_occupancy=0.45, emissive_fraction=0.08, seed=31)
    far = workloads.noise_world(grid_bricks=(4, 4, 4), brick_occupancy=0.6, emissive_fraction=0.2, seed=32)
    keys = np.concatenate([base.keys + np.array([-1000, -37, 500], np.int32),
                           far.keys + np.array([-1000 + 300, -37 + 40, 500 + 200], np.int32)])
    voxels = np.concatenate([base.voxels, far.voxels])
    power = np.concatenate([base.power, far.power])
    origin, grid = workloads.scene_grid(keys, 4)
    k = keys.astype(np.int64) - np.array(origin)
    o = np.argsort(k[:, 0] + grid[0] * (k[:, 1] + grid[1] * k[:, 2]), kind="stable")
    cam = workloads.look_at(np.array([-8030.0, -140.0, 3960.0]), np.array([-7950.0, -270.0, 4080.0]))
    vs = base.like(grid=grid, keys=keys[o], voxels=voxels[o], power=power[o], camera=cam)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    osc = oracle_lib.OracleScene(oracle, vs)
    assert osc.origin[0] < 0 and osc.origin[1] < 0
    assert_scene_equal(scene, osc, vs)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, vs, 96, 64, spp=2, bounces=4, seed=5)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)
    assert float(gpu.max()) > 0.0
    # Keys beyond the range are refused before anything is accepted.
    with pytest.raises(caelix_b200.CaelixError) as err:
        scene.upload_bricks(np.array([[0, 0, 0], [1 << 20, 0, 0]], np.int32), np.zeros((2, 512), np.uint16))
    assert err.value.code == caelix_b200.CAELIX_ERROR_INVALID_ARGUMENT
    scene.close()
    osc.close()


def test_box_beyond_the_bitmap_limit_is_refused(cuda_device):
    import caelix_b200

    scene = caelix_b200.Scene(cuda_device, 4, workloads.ENCODING_BLOCK_ID)
    keys = np.array([[-(1 << 20), -(1 << 20), -(1 << 20)], [(1 << 20) - 1, (1 << 20) - 1, (1 << 20) - 1]], np.int32)
    scene.upload_bricks(keys, np.full((2, 512), 0x8001, np.uint16))
    with pytest.raises(caelix_b200.CaelixError) as err:
        scene.flush()
    assert err.value.code == caelix_b200.CAELIX_ERROR_UNSUPPORTED
    scene.close()


def test_materials_api(cuda_device):
    """caelix_scene_set_materials / set_material_entries / get_material: the built-in packed codes,
    replacement, the value checks."""
    import caelix_b200

    scene = caelix_b200.Scene(cuda_device, 4, workloads.ENCODING_PACKED)
    m = scene.material(R.WHITE_EMITTER)
    assert tuple(m.emission) == (1.0, 1.0, 1.0) and tuple(m.albedo) == (1.0, 1.0, 1.0)
    m = scene.material(R.GREY_FLOOR)
    assert abs(m.albedo[0] - 15.0 / 31.0) < 1e-7 and tuple(m.emission) == (0.0, 0.0, 0.0)
    m = scene.material(0x4000 | (15 << 10) | 3)  # rgb4 red 15/15, strength 2^9
    assert tuple(m.albedo) == (1.0, 0.0, 0.0) and tuple(m.emission) == (512.0, 0.0, 0.0)
    scene.set_material_entries([(0x8123, (0.25, 0.5, 0.75), (2.0, 0.0, 0.0))])
    m = scene.material(0x8123)
    assert tuple(m.albedo) == (0.25, 0.5, 0.75) and tuple(m.emission) == (2.0, 0.0, 0.0)
    # A transparent code is looked up without its face bits.
    scene.set_material_entries([(0x0005, (0.1, 0.2, 0.3), (0.0, 0.0, 0.0))])
    assert tuple(scene.material(0x0005 | (0x3F << 8)).albedo) == tuple(np.float32([0.1, 0.2, 0.3]))
    with pytest.raises(caelix_b200.CaelixError):
        scene.set_material_entries([(0x8000, (1e6, 0.0, 0.0), (0.0, 0.0, 0.0))])  # above the half range
    with pytest.raises(caelix_b200.CaelixError):
        scene.set_material_entries([(0x10000, (0.5, 0.5, 0.5), (0.0, 0.0, 0.0))])
    scene.set_materials([])  # the built-in table again
    assert tuple(scene.material(0x8123).emission) == (0.0, 0.0, 0.0)
    scene.close()
