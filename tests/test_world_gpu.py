"""A world file into a scene: caelix_world_upload_entity decodes a .cxw world written from a
generated scene (sectors of 16^3 bricks, moved to negative sector coordinates) and uploads it; the
flushed scene equals the oracle's build of the same bricks moved to the returned origin."""
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
    scene = caelix_b200.Scene(cuda_device, vs.group_shift)
    origin, bricks = f.upload_entity(0, scene, threads=4)
    keep = (vs.voxels != 0).any(axis=1)  # the reader drops all-air bricks
    keys = vs.keys[keep]
    assert bricks == int(keep.sum())
    assert origin == tuple(int(keys[:, a].min()) + shift[a] for a in range(3))
    moved = keys + np.array(shift, np.int32) - np.array(origin, np.int32)
    grid = tuple(int(v) for v in moved.max(axis=0) + 1)
    lin = moved[:, 0] + grid[0] * (moved[:, 1] + grid[1] * moved[:, 2].astype(np.int64))
    o = np.argsort(lin, kind="stable")
    exp = workloads.VoxelScene(grid, moved[o], vs.voxels[keep][o], vs.power[keep][o], vs.albedo, vs.camera,
                               vs.group_shift)
    emissive = exp.power > 0
    scene.set_brick_power(exp.keys[emissive], exp.power[emissive])
    scene.set_albedo(exp.albedo)
    scene.flush()
    assert_scene_equal(scene, oracle_lib.OracleScene(oracle, exp), exp)
    scene.close()
    f.close()
