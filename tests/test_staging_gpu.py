"""Device-resident brick staging: bricks uploaded in pieces, in any order, with overwrites and
repeated keys inside one upload, give the same scene as one upload of the final bricks (bit-exact
against the oracle), and a flush after edits rebuilds the edited scene."""
import numpy as np
import pytest

import oracle_lib
from caelix_b200 import workloads
from test_trace_gpu import assert_scene_equal, assert_radiance_close, render_both

pytestmark = pytest.mark.gpu


def incremental_scene(cuda_device, vs, rng, pieces=5):
    """The bricks of `vs` uploaded shuffled in `pieces` calls; a third of them first with other
    voxels, some repeated inside a call (the last copy right); half the power set before the
    upload of its brick, half after."""
    import caelix_b200

    s = caelix_b200.Scene.for_voxel_scene(cuda_device, vs)
    n = vs.brick_count
    emissive = np.nonzero(vs.power > 0)[0]
    dark = np.nonzero(vs.power <= 0)[0]
    early = np.concatenate([emissive[: len(emissive) // 2], dark[: len(dark) // 2]])
    if len(early):
        s.set_brick_power(vs.keys[early], vs.power[early])
    junk = rng.choice(n, size=n // 3, replace=False)
    s.upload_bricks(vs.keys[junk], rng.integers(0, 1 << 16, size=(len(junk), 512), dtype=np.uint16))
    order = rng.permutation(n)
    for part in np.array_split(order, pieces):
        if len(part) == 0:
            continue
        rep = part[rng.random(len(part)) < 0.1]
        keys = np.concatenate([vs.keys[rep], vs.keys[part]])
        vox = np.concatenate([np.full((len(rep), 512), 0x8003, np.uint16), vs.voxels[part]])
        s.upload_bricks(keys, vox)
    late = np.concatenate([emissive[len(emissive) // 2:], dark[len(dark) // 2:]])
    if len(late):
        s.set_brick_power(vs.keys[late], vs.power[late])
    s.flush()
    return s


@pytest.mark.parametrize("seed", [2, 8])
def test_incremental_uploads_equal_one_upload(cuda_device, oracle, seed):
    vs = workloads.noise_world(grid_bricks=(8, 6, 10), brick_occupancy=0.45, emissive_fraction=0.08, seed=seed)
    scene = incremental_scene(cuda_device, vs, np.random.default_rng(seed))
    osc = oracle_lib.OracleScene(oracle, vs)
    assert_scene_equal(scene, osc, vs)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, vs, 96, 64, spp=2, bounces=4, seed=seed)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)
    scene.close()


def test_config2_incremental_then_edit(cuda_device, oracle):
    """The 4,096-brick scene uploaded in pieces, flushed, then a tenth of its bricks rewritten,
    new bricks added (the grid grows) and a flush: both states equal the oracle's."""
    vs = workloads.noise_world()
    rng = np.random.default_rng(11)
    scene = incremental_scene(cuda_device, vs, rng, pieces=7)
    assert_scene_equal(scene, oracle_lib.OracleScene(oracle, vs), vs)

    edit = rng.choice(vs.brick_count, size=vs.brick_count // 10, replace=False)
    voxels = vs.voxels.copy()
    voxels[edit] = np.where(rng.random((len(edit), 512)) < 0.5, 0x8002, 0).astype(np.uint16)
    gx, gy, gz = vs.grid
    extra = np.array([[gx, 0, 0], [gx + 1, gy, 2], [0, 0, gz + 3]], np.int32)
    extra_vox = np.full((3, 512), 0x8001, np.uint16)
    keys = np.concatenate([vs.keys, extra])
    allvox = np.concatenate([voxels, extra_vox])
    lin = keys[:, 0] + (gx + 2) * (keys[:, 1] + (gy + 1) * keys[:, 2].astype(np.int64))
    o = np.argsort(lin, kind="stable")
    power = np.concatenate([vs.power, np.ones(3, np.float32)])  # a new brick's power is 1 until set
    edited = workloads.VoxelScene((gx + 2, gy + 1, gz + 4), keys[o], allvox[o], power[o], vs.albedo, vs.camera,
                                  vs.group_shift)
    scene.upload_bricks(np.concatenate([vs.keys[edit], extra]), np.concatenate([voxels[edit], extra_vox]))
    scene.flush()
    assert_scene_equal(scene, oracle_lib.OracleScene(oracle, edited), edited)
    scene.close()


def test_empty_and_power_only_flushes(cuda_device, oracle):
    """A scene flushed with no bricks; then bricks; then only a power change (the edited bricks'
    records again, the light records and the light tree rebuilt)."""
    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(6, 6, 6), brick_occupancy=0.5, emissive_fraction=0.1, seed=4)
    s = caelix_b200.Scene.for_voxel_scene(cuda_device, vs)
    s.flush()
    assert s.view().brick_count == 0
    s.upload_bricks(vs.keys, vs.voxels)
    s.flush()
    # Every brick's power is 1 until set: every brick emits.
    lit = vs.like(power=np.ones_like(vs.power))
    assert_scene_equal(s, oracle_lib.OracleScene(oracle, lit), lit)
    s.set_brick_power(vs.keys, vs.power)
    s.flush()
    assert_scene_equal(s, oracle_lib.OracleScene(oracle, vs), vs)
    s.close()


def test_edits_without_new_bricks(cuda_device, oracle):
    """Edits that add no brick (rewritten values, bricks emptied, powers changed, a new albedo
    table) take the incremental flush; each state equals the oracle's build of the edited scene,
    and so does the render."""
    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(10, 8, 12), brick_occupancy=0.45, emissive_fraction=0.08, seed=12)
    rng = np.random.default_rng(12)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    voxels, power, albedo = vs.voxels.copy(), vs.power.copy(), vs.albedo.copy()
    for step in range(3):
        n = vs.brick_count
        edit = rng.choice(n, size=n // 10, replace=False)
        fresh = np.where(rng.random((len(edit), 512)) < 0.5,
                         0x8000 | rng.integers(1, 65, size=(len(edit), 512)), 0).astype(np.uint16)
        fresh[: len(edit) // 8] = 0  # emptied bricks stay in the scene
        voxels[edit] = fresh
        scene.upload_bricks(vs.keys[edit], fresh)
        relit = rng.choice(n, size=max(1, n // 20), replace=False)
        power[relit] = np.where(rng.random(len(relit)) < 0.5, 0.0, rng.lognormal(0.0, 1.0, len(relit))).astype(np.float32)
        scene.set_brick_power(vs.keys[relit], power[relit])
        if step == 1:
            albedo = rng.uniform(0.1, 0.9, size=albedo.shape).astype(np.float32)
            scene.set_albedo(albedo)
        scene.flush()
        cur = workloads.VoxelScene(vs.grid, vs.keys, voxels, power, albedo, vs.camera, vs.group_shift)
        osc = oracle_lib.OracleScene(oracle, cur)
        assert_scene_equal(scene, osc, cur)
        gpu, ref, st, rays = render_both(cuda_device, scene, osc, cur, 64, 48, spp=2, bounces=3, seed=step + 1)
        assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
        assert_radiance_close(gpu, ref)
    # An albedo change alone: no rebuild, the render follows the new table.
    albedo = rng.uniform(0.1, 0.9, size=albedo.shape).astype(np.float32)
    scene.set_albedo(albedo)
    scene.flush()
    cur = workloads.VoxelScene(vs.grid, vs.keys, voxels, power, albedo, vs.camera, vs.group_shift)
    osc = oracle_lib.OracleScene(oracle, cur)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, cur, 64, 48, spp=2, bounces=3, seed=9)
    assert_radiance_close(gpu, ref)
    scene.close()


def scene_of(keys, voxels, power, vs):
    """A VoxelScene of the given bricks in increasing linear brick index of the grid their keys
    span (the grid always holds brick 0, as the scene's)."""
    grid = tuple(int(g) for g in np.maximum(keys.max(axis=0), 0) + 1) if len(keys) else (1, 1, 1)
    lin = keys[:, 0] + grid[0] * (keys[:, 1] + grid[1] * keys[:, 2].astype(np.int64))
    o = np.argsort(lin, kind="stable")
    return workloads.VoxelScene(grid, keys[o], voxels[o], power[o], vs.albedo, vs.camera, vs.group_shift)


def test_remove_bricks(cuda_device, oracle):
    """caelix_scene_remove_bricks: a quarter of the bricks removed (every brick of the highest x
    plane among them, so the grid shrinks; emissive bricks; repeated, absent and out-of-range keys
    that are ignored), then some of them uploaded again (one emissive brick without its power: it
    comes back with the default power 1), then every brick removed. Each flushed state equals the oracle's build of the
    remaining bricks, and so does the render. A brick uploaded again has power 1 until set."""
    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(9, 7, 8), brick_occupancy=0.5, emissive_fraction=0.08, seed=5)
    rng = np.random.default_rng(5)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    n = vs.brick_count
    top = np.nonzero(vs.keys[:, 0] == vs.keys[:, 0].max())[0]
    gone = np.unique(np.concatenate([rng.choice(n, size=n // 4, replace=False), top,
                                     np.nonzero(vs.power > 0)[0][:3]]))
    extra = np.array([[vs.grid[0] + 5, 0, 0], [-1, 2, 2], [0, -3, 1], [1 << 21, 0, 0]], np.int32)  # absent, out of range
    scene.remove_bricks(np.concatenate([vs.keys[gone], vs.keys[gone[:10]], extra]))
    scene.flush()
    keep = np.setdiff1d(np.arange(n), gone)
    cur = scene_of(vs.keys[keep], vs.voxels[keep], vs.power[keep], vs)
    assert cur.grid[0] < vs.grid[0]
    osc = oracle_lib.OracleScene(oracle, cur)
    assert_scene_equal(scene, osc, cur)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, cur, 64, 48, spp=2, bounces=3, seed=3)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)

    back = gone[rng.random(len(gone)) < 0.5]
    lit_back = back[vs.power[back] > 0]
    scene.upload_bricks(vs.keys[back], vs.voxels[back])
    unset = lit_back[:1]
    set_back = np.setdiff1d(back, unset)
    if len(set_back):
        scene.set_brick_power(vs.keys[set_back], vs.power[set_back])
    scene.flush()
    power = vs.power.copy()
    power[unset] = 1.0
    now = np.union1d(keep, back)
    cur = scene_of(vs.keys[now], vs.voxels[now], power[now], vs)
    osc = oracle_lib.OracleScene(oracle, cur)
    assert_scene_equal(scene, osc, cur)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, cur, 64, 48, spp=2, bounces=3, seed=4)
    assert_radiance_close(gpu, ref)

    scene.remove_bricks(vs.keys)
    scene.flush()
    assert scene.view().brick_count == 0
    scene.close()


def generation_state(scene):
    """The group generations (row word 2), the brick keys, the keys of the light bricks and the
    grid (origin, group grid, group edge shift) of a flushed scene."""
    import gpu_util

    v = scene.view()
    g, n, m = int(v.group_count), int(v.brick_count), int(v.light_count)
    rows = gpu_util.from_device(v.group_rows, np.uint32, 8 * g).reshape(-1, 8)
    keys = gpu_util.from_device(v.keys, np.int32, 3 * n).reshape(-1, 3) if n else np.zeros((0, 3), np.int32)
    lb = gpu_util.from_device(v.light_brick, np.uint32, m) if m else np.zeros(0, np.uint32)
    grid = (tuple(int(x) for x in v.origin), tuple(int(x) for x in v.groups), int(v.group_shift))
    return rows[:, 2].copy(), keys, {tuple(k) for k in keys[lb].tolist()}, grid


def groups_of(keys, grid):
    origin, groups, gs = grid
    c = (np.asarray(keys, np.int64).reshape(-1, 3) - np.array(origin, np.int64)) >> gs
    return set((c[:, 0] + groups[0] * (c[:, 1] + groups[1] * c[:, 2])).tolist())


def next_version(gen):
    return (gen & 0xFFFF0000) | ((gen + 1) & 0xFFFF)


def test_group_generations(cuda_device):
    """GroupLightRow::generation (life << 16 | version) over a flush history: the first build gives
    every group with light bricks version 1; an edit flush bumps the version of exactly the groups
    holding a refinalized brick (an edited brick or one of its six neighbours) that is or was a
    light brick; a full rebuild bumps every group that has or had light bricks; a group that loses
    all its bricks takes the next life (version 0); a new grid starts every group at a life above
    all earlier ones."""
    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(12, 10, 12), brick_occupancy=0.5, emissive_fraction=0.06, seed=21)
    vs = vs.like(group_shift=2)
    rng = np.random.default_rng(21)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    gen0, keys0, lit0, grid0 = generation_state(scene)
    lit_groups = groups_of(list(lit0), grid0)
    assert 1 < len(lit_groups) < len(gen0)
    assert np.array_equal(gen0, np.array([1 if g in lit_groups else 0 for g in range(len(gen0))], np.uint32))

    # An edit flush: two light bricks emptied, three dark bricks rewritten, one power change.
    key_set = {tuple(k) for k in keys0.tolist()}
    lit_list = sorted(lit0)
    dark = [k for k in map(tuple, keys0.tolist()) if k not in lit0]
    pick_lit = [lit_list[i] for i in rng.choice(len(lit_list), size=2, replace=False)]
    pick_dark = [dark[i] for i in rng.choice(len(dark), size=3, replace=False)]
    edit = np.array(pick_lit + pick_dark, np.int32)
    vox = np.where(rng.random((len(edit), 512)) < 0.5, 0x8001, 0).astype(np.uint16)
    vox[:2] = 0
    scene.upload_bricks(edit, vox)
    relit = np.array([dark[int(rng.integers(len(dark)))]], np.int32)
    scene.set_brick_power(relit, np.array([0.0], np.float32))
    scene.flush()
    gen1, keys1, lit1, grid1 = generation_state(scene)
    assert grid1 == grid0 and np.array_equal(keys1, keys0)
    refin = set()
    for k in np.concatenate([edit, relit]).tolist():
        for d in ((0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            b = (k[0] + d[0], k[1] + d[1], k[2] + d[2])
            if b in key_set:
                refin.add(b)
    touched = groups_of([b for b in refin if b in lit0 or b in lit1], grid0) if refin else set()
    expect = gen0.copy()
    for g in touched:
        expect[g] = next_version(int(expect[g]))
    assert touched and len(touched) < len(gen0)
    assert np.array_equal(gen1, expect)

    # A full rebuild over the same grid: a brick added in an empty cell.
    cell = next((x, y, z) for z in range(vs.grid[2]) for y in range(vs.grid[1]) for x in range(vs.grid[0])
                if (x, y, z) not in key_set)
    scene.upload_bricks(np.array([cell], np.int32), np.full((1, 512), 0x8002, np.uint16))
    scene.set_brick_power(np.array([cell], np.int32), np.array([0.0], np.float32))
    scene.flush()
    gen2, keys2, lit2, grid2 = generation_state(scene)
    assert grid2 == grid0
    rebuilt = groups_of(list(lit1 | lit2), grid0)
    expect = gen1.copy()
    for g in rebuilt:
        expect[g] = next_version(int(expect[g]))
    assert np.array_equal(gen2, expect)

    # Every brick of one inner group removed (the grid stays): that group takes the next life.
    origin, groups, gs = grid0
    inner = [g for g in groups_of(keys2, grid0)
             if 0 < g % groups[0] < groups[0] - 1 and 0 < (g // groups[0]) % groups[1] < groups[1] - 1
             and 0 < g // (groups[0] * groups[1]) < groups[2] - 1]
    assert inner
    gone = inner[0]
    members = np.array([k for k in keys2.tolist() if groups_of([k], grid0) == {gone}], np.int32)
    scene.remove_bricks(members)
    scene.flush()
    gen3, keys3, lit3, grid3 = generation_state(scene)
    assert grid3 == grid0
    expect = gen2.copy()
    for g in groups_of(list(lit2 | lit3), grid0):
        expect[g] = next_version(int(expect[g]))
    expect[gone] = ((int(gen2[gone]) >> 16) + 1) << 16
    assert np.array_equal(gen3, expect)

    # A brick beyond the grid: a new grid, every group at a new life.
    far = np.array([[int(keys3[:, 0].max()) + (1 << gs) + 1, 0, 0]], np.int32)
    scene.upload_bricks(far, np.full((1, 512), 0x8002, np.uint16))
    scene.flush()
    gen4, keys4, lit4, grid4 = generation_state(scene)
    assert grid4 != grid0
    life = (int(gen3.max() >> 16) if len(gen3) else 0) + 1
    lit_groups = groups_of(list(lit4), grid4)
    assert np.array_equal(gen4, np.array([(life << 16) | (1 if g in lit_groups else 0) for g in range(len(gen4))],
                                         np.uint32))
    scene.close()
