"""The oracle against two of the reference's own known answers of the trace path (CPU; the scenes
and expectations are restated in reference_scenes.py):

* the voxel id test (tests/trace_test.cpp:3735-3945): every pixel's camera-ray hit is the floor
  voxel the CPU computes in double (one key per voxel, one voxel per key, the miss value on the
  misses), also with entity B turned 180 degrees about Y; voxel_id_tmax cuts hits. This pins the
  world DDA, the brick DDA, negative brick keys, the packed encoding and entity transforms to an
  answer the reference holds, not to the oracle itself;
* the one-bounce energy test (tests/trace_test.cpp:1227-1288): the centre mean of the floor under an
  emissive ceiling is the albedo times the CPU Monte Carlo hit probability, within 3 % (path
  tracing, and light-tree NEE with MIS over the ceiling's light voxels), and a 1 spp frame of pure
  path tracing holds only 0 and the albedo, its centre mean within 5 % of the CPU estimate."""
import numpy as np
import pytest

import oracle_lib
import reference_scenes as R


@pytest.fixture(scope="module")
def floor(oracle):
    vs = R.floor_scene()
    osc = oracle_lib.OracleScene(oracle, vs)
    yield vs, osc
    osc.close()


def test_floor_is_negative_keys_in_packed_encoding(floor):
    vs, osc = floor
    assert vs.keys[:, 1].min() == -1 and vs.encoding == 0
    assert osc.origin == (0, -16, 0) and osc.grid == (8, 16, 8)


def test_voxel_ids_match_the_cpu_floor(floor):
    vs, osc = floor
    _, _, ids = osc.render(R.SIZE, R.SIZE, spp=1, bounces=0, seed=1, light_nee=False, threads=8, voxel_ids=True)
    assert R.check_voxel_ids(ids, vs.camera) > 50  # the reference's 7 x 14 voxels


def test_voxel_id_tmax(floor):
    vs, osc = floor
    _, _, near = osc.render(R.SIZE, R.SIZE, bounces=0, light_nee=False, threads=8, voxel_ids=True, voxel_id_tmax=6.0)
    assert (near == 0xFFFFFFFF).all()  # the floor is 12 away
    _, _, far = osc.render(R.SIZE, R.SIZE, bounces=0, light_nee=False, threads=8, voxel_ids=True, voxel_id_tmax=1000.0)
    _, _, free = osc.render(R.SIZE, R.SIZE, bounces=0, light_nee=False, threads=8, voxel_ids=True)
    assert np.array_equal(far, free)


def test_voxel_ids_with_entity_b(oracle, floor):
    vs, osc = floor
    b = oracle_lib.OracleScene(oracle, R.floor_scene())
    osc.set_entities([(b, R.ENTITY_B_ROTATION, R.ENTITY_B_POSITION)], ids=[1])
    _, _, ids = osc.render(R.SIZE, R.SIZE, bounces=0, light_nee=False, threads=8, voxel_ids=True)
    R.check_voxel_ids(ids, vs.camera, entity_b=True)
    keys_of, local_of = [set(), set()], [set(), set()]
    for y in range(R.SIZE):
        for x in range(R.SIZE):
            v = R.floor_voxel(vs.camera, x, y, True)
            if v[0] == "hit":
                keys_of[v[1]].add(tuple(ids[y, x]))
                local_of[v[1]].add(v[2:])
    assert len(local_of[0] & local_of[1]) > 50
    assert not keys_of[0] & keys_of[1]
    osc.set_entities([])
    b.close()


@pytest.mark.parametrize("lights", [False, True])
def test_one_bounce_under_the_emissive_ceiling(oracle, lights):
    vs = R.room_scene(lights=lights)
    osc = oracle_lib.OracleScene(oracle, vs)
    assert (osc.light_count > 0) == lights
    img, _ = osc.render(R.SIZE, R.SIZE, spp=2048, bounces=1, seed=1000, light_nee=lights, window=R.centre_window(32),
                        threads=8)
    x0, y0, x1, y1 = R.centre_window(32)
    gpu_like = img[y0:y1, x0:x1].astype(np.float64)
    cpu = float(R.FLOOR_ALBEDO) * R.ceiling_hit_probability(R.half_extent(32, vs.camera))
    ratio = gpu_like[..., 0].mean() / cpu
    assert abs(ratio - 1.0) < 0.03, ratio
    assert np.abs(gpu_like[..., 1] - gpu_like[..., 0]).max() < 1e-6
    assert np.abs(gpu_like[..., 2] - gpu_like[..., 0]).max() < 1e-6
    osc.close()


def test_one_bounce_raw_frame(oracle):
    vs = R.room_scene(lights=False)
    osc = oracle_lib.OracleScene(oracle, vs)
    window = R.centre_window(128)
    img, _ = osc.render(R.SIZE, R.SIZE, spp=1, bounces=1, seed=77, light_nee=False, window=window, threads=8)
    x0, y0, x1, y1 = window
    c = img[y0:y1, x0:x1, 0]
    assert np.isin(c, [0.0, R.FLOOR_ALBEDO]).all()  # one bounce, emission 1: exactly 0 or the albedo
    cpu = float(R.FLOOR_ALBEDO) * R.ceiling_hit_probability(R.half_extent(128, vs.camera))
    assert abs(c.astype(np.float64).mean() / cpu - 1.0) < 0.05
    osc.close()
