"""Entities through the C ABI against the oracle: a world with two entities (one rotated, one
translated), rendered with the wavefront and the per-frame kernels; then an entity moved, an
entity's bricks edited, an entity removed and a new one added in its id, then entity lights (a
dynamic entity's in the second light tree, a static entity's in tree 0 beside the world's), a lit
entity moved and a static entity made dynamic. Every state's radiance and ray counts equal the
oracle's with the same entities (bit-exact expected; the 1e-5 relative bound of the trace parity
tests)."""
import numpy as np
import pytest

import oracle_lib
from caelix_b200 import workloads
from test_entities_oracle import entity_bricks
from test_trace_gpu import assert_radiance_close

pytestmark = pytest.mark.gpu

Q1 = (0.12, -0.31, 0.2, 0.92)
Q1_MOVED = (-0.4, 0.1, 0.3, 0.86)
IDENTITY = (0.0, 0.0, 0.0, 1.0)


def render_pair(cuda_device, scene, osc, vs, mode=None, spp=2):
    import torch

    import caelix_b200

    r = caelix_b200.Renderer(cuda_device, scene)
    if mode is not None:
        r.set_trace_mode(mode, 0)
    out = torch.zeros(56 * 72 * 3, dtype=torch.float32, device="cuda")
    r.render(out, 72, 56, vs.camera, bounces=4, seed=5, spp=spp)
    st = r.stats()
    gpu = out.cpu().numpy().reshape(56, 72, 3)
    ref, rays = osc.render(72, 56, spp=spp, bounces=4, seed=5, threads=8)
    r.close()
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)
    return gpu


def test_entities_parity(cuda_device, oracle):
    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(8, 6, 10), brick_occupancy=0.45, emissive_fraction=0.08, seed=3)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    cam = vs.camera
    ahead = np.asarray(cam["position"], np.float64) + 14.0 * np.asarray(cam["forward"], np.float64)
    p1 = tuple((ahead - 8.0).astype(np.float32))
    p2 = tuple((ahead + np.array([10.0, -6.0, 12.0])).astype(np.float32))
    b1 = entity_bricks(grid=(2, 2, 2), seed=7)
    b2 = entity_bricks(grid=(1, 2, 1), seed=8, fill=0.8)
    e1 = scene.add_entity(p1, Q1)
    e2 = scene.add_entity(p2, IDENTITY)
    assert (e1, e2) == (1, 2)
    scene.upload_bricks(b1.keys, b1.voxels, entity=e1)
    scene.upload_bricks(b2.keys, b2.voxels, entity=e2)
    # Entity bricks emit with power 1 until set: these start dark.
    scene.set_brick_power(b1.keys, b1.power, entity=e1)
    scene.set_brick_power(b2.keys, b2.power, entity=e2)
    scene.set_entity_motion(e2, 1)
    scene.flush()

    osc = oracle_lib.OracleScene(oracle, vs)
    o1 = oracle_lib.OracleScene(oracle, b1)
    o2 = oracle_lib.OracleScene(oracle, b2)
    osc.set_entities([(o1, Q1, p1), (o2, IDENTITY, p2)], motions=[0, 1])
    img = render_pair(cuda_device, scene, osc, vs)
    render_pair(cuda_device, scene, osc, vs, mode=caelix_b200.Renderer.TRACE_MEGAKERNEL, spp=1)
    plain = oracle_lib.OracleScene(oracle, vs).render(72, 56, spp=2, bounces=4, seed=5, threads=8)[0]
    assert not np.array_equal(img, plain)  # the entities are in view

    # Moved; the next flush applies it.
    scene.set_entity_transform(e1, p1, Q1_MOVED)
    scene.flush()
    osc.set_entities([(o1, Q1_MOVED, p1), (o2, IDENTITY, p2)], motions=[0, 1])
    render_pair(cuda_device, scene, osc, vs)

    # Edited bricks of an entity (no new key: that entity's incremental flush).
    rng = np.random.default_rng(3)
    vox2 = b2.voxels.copy()
    vox2[0] = np.where(rng.random(512) < 0.5, 0x8000 | 17, 0).astype(np.uint16)
    scene.upload_bricks(b2.keys[:1], vox2[:1], entity=e2)
    scene.flush()
    b2e = workloads.VoxelScene(b2.grid, b2.keys, vox2, b2.power, b2.albedo, b2.camera, b2.group_shift)
    o2 = oracle_lib.OracleScene(oracle, b2e)
    osc.set_entities([(o1, Q1_MOVED, p1), (o2, IDENTITY, p2)], motions=[0, 1])
    render_pair(cuda_device, scene, osc, vs)

    # Removed: the remaining entity keeps its order; a new entity takes the free id.
    scene.remove_entity(e1)
    osc.set_entities([(o2, IDENTITY, p2)], motions=[1])
    render_pair(cuda_device, scene, osc, vs)  # the removal applies at once
    e3 = scene.add_entity(p1, IDENTITY)
    assert e3 == e1
    scene.upload_bricks(b1.keys, b1.voxels, entity=e3)
    scene.set_brick_power(b1.keys, b1.power, entity=e3)
    scene.flush()
    osc.set_entities([(o1, IDENTITY, p1), (o2, IDENTITY, p2)], motions=[0, 1])
    render_pair(cuda_device, scene, osc, vs)

    # Entity lights: some bricks of both entities emit (the second light tree), then one moves.
    rng = np.random.default_rng(4)
    p_1 = np.where(rng.random(b1.brick_count) < 0.5, rng.lognormal(0.0, 1.0, b1.brick_count), 0.0).astype(np.float32)
    p_2 = np.where(rng.random(b2.brick_count) < 0.5, rng.lognormal(0.0, 1.0, b2.brick_count), 0.0).astype(np.float32)
    p_2[0] = 2.0  # both trees hold entity lights
    scene.set_brick_power(b1.keys, p_1, entity=e3)
    scene.set_brick_power(b2.keys, p_2, entity=e2)
    scene.flush()
    l1 = oracle_lib.OracleScene(oracle, workloads.VoxelScene(b1.grid, b1.keys, b1.voxels, p_1, b1.albedo, b1.camera,
                                                             b1.group_shift))
    l2 = oracle_lib.OracleScene(oracle, workloads.VoxelScene(b2.grid, b2.keys, vox2, p_2, b2.albedo, b2.camera,
                                                             b2.group_shift))
    osc.set_entities([(l1, IDENTITY, p1), (l2, IDENTITY, p2)], motions=[0, 1])
    assert osc.s.dyn and osc._merged0 is not None  # e3's lights in tree 0, e2's in tree 1
    lit = render_pair(cuda_device, scene, osc, vs)
    render_pair(cuda_device, scene, osc, vs, mode=caelix_b200.Renderer.TRACE_MEGAKERNEL, spp=1)
    scene.set_entity_transform(e3, p1, Q1)
    scene.flush()
    osc.set_entities([(l1, Q1, p1), (l2, IDENTITY, p2)], motions=[0, 1])
    moved = render_pair(cuda_device, scene, osc, vs)
    assert not np.array_equal(lit, moved)

    # A batch takes the scene with its entities (the wavefront kernels, both light trees rebuilt):
    # each view equals the plain render, whatever kernel the tuning names.
    import torch

    r = caelix_b200.Renderer(cuda_device, scene)
    out = torch.zeros(40 * 32 * 3, dtype=torch.float32, device="cuda")
    ref = torch.zeros_like(out)
    r.render(ref, 40, 32, vs.camera, bounces=3, seed=2, spp=2)
    for kernel in (0, 1):
        batch = caelix_b200.Batch(cuda_device, [(r, out, 40, 32, vs.camera, 3, 2, 2)], rebuild_light_trees=True)
        batch.set_tuning(min_blocks=6, block_width=8, refill_min=4, order=1, sort_keys_per_thread=16, kernel=kernel,
                         wavefront=0)
        out.fill_(-1.0)
        batch.run()
        st = batch.stats()
        assert st.light_tree_builds >= 1
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        # An entity moved: the next run captures again and follows it.
        scene.set_entity_transform(e3, p1, Q1_MOVED if kernel == 0 else Q1)
        scene.flush()
        r.render(ref, 40, 32, vs.camera, bounces=3, seed=2, spp=2)
        batch.run()
        batch.stats()
        torch.cuda.synchronize()
        assert torch.equal(out, ref)
        batch.close()
    r.close()

    # A static entity made dynamic: its lights leave tree 0 for the dynamic tree at the next flush.
    scene.set_entity_motion(e3, 1)
    scene.flush()
    osc.set_entities([(l1, Q1, p1), (l2, IDENTITY, p2)], motions=[1, 1])
    assert osc._merged0 is None
    render_pair(cuda_device, scene, osc, vs)

    # Entity 0 cannot be moved or removed; motion takes two values.
    with pytest.raises(caelix_b200.CaelixError):
        scene.remove_entity(0)
    with pytest.raises(caelix_b200.CaelixError):
        scene.set_entity_motion(e3, 2)
    with pytest.raises(caelix_b200.CaelixError):
        scene.upload_bricks(b1.keys, b1.voxels, entity=7)
    scene.close()


def test_backward_with_entities(cuda_device, oracle):
    """caelix_renderer_backward of a scene with a lit, rotated entity: the forward image is the
    render, and the gradients of the world's bricks' power and of the material table's albedo
    (entity voxels included) match the double-precision oracle adjoint within 1e-3 relative; the
    entity's emission and its lamps enter the radiance as fixed terms."""
    import torch

    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(8, 6, 10), brick_occupancy=0.45, emissive_fraction=0.1, seed=13)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    cam = vs.camera
    ahead = np.asarray(cam["position"], np.float64) + 14.0 * np.asarray(cam["forward"], np.float64)
    p1 = tuple((ahead - 8.0).astype(np.float32))
    b1 = entity_bricks(grid=(2, 2, 2), seed=7)
    rng = np.random.default_rng(9)
    p_1 = np.where(rng.random(b1.brick_count) < 0.5, rng.lognormal(0.0, 1.0, b1.brick_count), 0.0).astype(np.float32)
    e1 = scene.add_entity(p1, Q1)
    scene.upload_bricks(b1.keys, b1.voxels, entity=e1)
    scene.set_brick_power(b1.keys, p_1, entity=e1)
    scene.flush()
    osc = oracle_lib.OracleScene(oracle, vs)
    o1 = oracle_lib.OracleScene(oracle, b1.like(power=p_1))
    osc.set_entities([(o1, Q1, p1)])
    w, h, spp, bounces = 64, 48, 2, 3
    r = caelix_b200.Renderer(cuda_device, scene)
    img = torch.zeros(h * w * 3, device="cuda")
    r.render(img, w, h, cam, bounces=bounces, seed=3, spp=spp)
    target = torch.from_numpy(0.9 * img.cpu().numpy()).cuda()
    d_rad = 2.0 * (img - target)
    d_alb = torch.zeros(65536 * 3, device="cuda")
    d_pow = torch.zeros(vs.brick_count, device="cuda")
    fwd = torch.zeros_like(img)
    r.backward(d_rad, w, h, cam, d_alb, d_pow, bounces=bounces, seed=3, spp=spp, image=fwd)
    torch.cuda.synchronize()
    assert torch.equal(fwd, img)
    _, rA, rP = osc.adjoint(w, h, spp=spp, bounces=bounces, seed=3, d_radiance=d_rad.cpu().numpy(), threads=8)
    gA = d_alb.cpu().numpy().reshape(65536, 3).astype(np.float64)
    gP = d_pow.cpu().numpy().astype(np.float64)
    for gpu, ref in ((gA, rA), (gP, rP)):
        scale = np.abs(ref).max()
        assert scale > 0
        big = np.abs(ref) >= 1e-3 * scale
        assert np.max(np.abs(gpu[big] - ref[big]) / np.abs(ref[big])) <= 1e-3
        assert np.abs(gpu - ref).max() <= 1e-3 * scale
    r.close()
    osc.set_entities([])
    scene.close()


def test_many_entities_parity(cuda_device, oracle):
    """64 entities (the scene's entity BVH): 40 scattered round the view with random rotations, some
    lit, and 24 in a row along the camera's axis (more boxes on one ray than the candidate list
    holds: those rays take every entity in order). The radiance and ray counts equal the oracle's,
    which loops over every entity, for both kernels; then 40 removed (the BVH rebuilt)."""
    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(8, 6, 10), brick_occupancy=0.3, emissive_fraction=0.08, seed=21)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    cam = vs.camera
    pos = np.asarray(cam["position"], np.float64)
    fwd = np.asarray(cam["forward"], np.float64)
    rng = np.random.default_rng(17)
    shapes = [entity_bricks(grid=(1, 1, 1), seed=30 + i, fill=0.7) for i in range(4)]
    placed = []
    for i in range(64):
        if i < 40:
            p = pos + rng.uniform(6.0, 40.0) * fwd + rng.uniform(-14.0, 14.0, 3)
            q = rng.normal(size=4)
            q = tuple(float(x) for x in q / np.linalg.norm(q))
        else:
            p = pos + (6.0 + 3.0 * (i - 40)) * fwd - 4.0
            q = IDENTITY
        shape = shapes[i % 4]
        power = np.where(rng.random(shape.brick_count) < 0.3, 2.0, 0.0).astype(np.float32)
        e = scene.add_entity(tuple(p.astype(np.float32)), q)
        assert e == i + 1
        scene.upload_bricks(shape.keys, shape.voxels, entity=e)
        scene.set_brick_power(shape.keys, power, entity=e)
        placed.append((shape.like(power=power), q, tuple(p.astype(np.float32))))
    scene.flush()
    oscs = {}

    def oracle_entities(items):
        out = []
        for vsub, q, p in items:
            key = (id(vsub.voxels), float(vsub.power.sum()), tuple(vsub.power))
            if key not in oscs:
                oscs[key] = oracle_lib.OracleScene(oracle, vsub)
            out.append((oscs[key], q, p))
        return out

    osc = oracle_lib.OracleScene(oracle, vs)
    osc.set_entities(oracle_entities(placed))
    img = render_pair(cuda_device, scene, osc, vs)
    render_pair(cuda_device, scene, osc, vs, mode=caelix_b200.Renderer.TRACE_MEGAKERNEL, spp=1)
    plain = oracle_lib.OracleScene(oracle, vs).render(72, 56, spp=2, bounces=4, seed=5, threads=8)[0]
    assert not np.array_equal(img, plain)

    for e in range(1, 41):
        scene.remove_entity(e)
    osc.set_entities(oracle_entities(placed[40:]))
    render_pair(cuda_device, scene, osc, vs)
    scene.flush()
    render_pair(cuda_device, scene, osc, vs, mode=caelix_b200.Renderer.TRACE_MEGAKERNEL, spp=1)
    osc.set_entities([])
    scene.close()
