"""Entities in the oracle: bricks of their own traversed under a rigid transform after the world's
bricks (the reference's TLAS instances, shaders/render/caelix_scene_trace.hlsl:104-131: the ray in
the instance's object space, the committed object-to-world normal). Checked against independent
restatements: an entity at a translation equals the same bricks merged into the world; a rotated
solid brick is hit where an exact slab test in double precision says; an entity no ray reaches
leaves the render bit-identical."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib
from caelix_b200 import workloads


def entity_bricks(grid=(2, 2, 2), seed=7, fill=0.55):
    """A small brick set of its own (power 0: entity bricks do not emit)."""
    vs = workloads.noise_world(grid_bricks=grid, brick_occupancy=1.0, voxel_fill=fill, emissive_fraction=0.0, seed=seed)
    return workloads.VoxelScene(vs.grid, vs.keys, vs.voxels, np.zeros_like(vs.power), vs.albedo, vs.camera,
                                vs.group_shift)


@pytest.fixture(scope="module")
def world():
    return workloads.noise_world(grid_bricks=(6, 6, 6), brick_occupancy=0.4, emissive_fraction=0.08, seed=3)


def hit_voxel(h, o, d):
    n = np.array(h.normal[:], np.float64)
    p = np.asarray(o, np.float64) + np.asarray(d, np.float64) * h.t
    return np.floor(p - 0.25 * n).astype(np.int64)


def test_translated_entity_equals_merged_world(oracle, world):
    ent = entity_bricks()
    shift = np.array([9, 1, 2], np.int32)  # four bricks of air between the world and the entity
    keys = np.concatenate([world.keys, ent.keys + shift])
    grid = tuple(int(v) for v in keys.max(axis=0) + 1)
    lin = keys[:, 0] + grid[0] * (keys[:, 1] + grid[1] * keys[:, 2].astype(np.int64))
    o = np.argsort(lin, kind="stable")
    merged = workloads.VoxelScene(grid, keys[o], np.concatenate([world.voxels, ent.voxels])[o],
                                  np.concatenate([world.power, ent.power])[o], world.albedo, world.camera,
                                  world.group_shift)
    w = oracle_lib.OracleScene(oracle, world)
    e = oracle_lib.OracleScene(oracle, ent)
    w.set_entities([(e, (0.0, 0.0, 0.0, 1.0), tuple(8.0 * shift))])
    m = oracle_lib.OracleScene(oracle, merged)
    rng = np.random.default_rng(5)
    span = np.array(grid, np.float64) * 8
    hits = entity_hits = same = 0
    for _ in range(4000):
        org = (rng.uniform(-0.1, 1.1, 3) * span).astype(np.float32)
        d = rng.normal(size=3)
        d = (d / np.linalg.norm(d)).astype(np.float32)
        a = w.trace(org, d)
        b = m.trace(org, d)
        assert bool(a.hit) == bool(b.hit)
        if not a.hit:
            continue
        hits += 1
        entity_hits += bool(a.attrib & 0x8000)
        assert abs(a.t - b.t) <= 1e-3 * max(1.0, b.t)
        same += (a.attrib & ~0x8000) == b.attrib and np.array_equal(hit_voxel(a, org, d), hit_voxel(b, org, d))
    assert entity_hits > 50
    assert same >= hits - hits // 200, (same, hits)


def test_rotated_solid_brick(oracle, world):
    solid = np.full((1, 512), 0x8005, np.uint16)
    ent = workloads.VoxelScene((1, 1, 1), np.zeros((1, 3), np.int32), solid, np.zeros(1, np.float32), world.albedo,
                               world.camera, world.group_shift)
    e = oracle_lib.OracleScene(oracle, ent)
    empty = workloads.VoxelScene((1, 1, 1), np.zeros((0, 3), np.int32), np.zeros((0, 512), np.uint16),
                                 np.zeros(0, np.float32), world.albedo, world.camera, world.group_shift)
    w = oracle_lib.OracleScene(oracle, empty)
    rng = np.random.default_rng(11)
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    pos = np.array([30.0, -12.0, 7.5], np.float32)
    w.set_entities([(e, tuple(q), tuple(pos))])
    rot = np.zeros(9, np.float32)
    oracle.oc_entity_rows(np.ascontiguousarray(q, np.float32).ctypes.data, rot.ctypes.data)
    R = rot.reshape(3, 3).astype(np.float64)
    centre = R @ np.full(3, 4.0) + pos
    for _ in range(300):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        org = (centre - 40.0 * d).astype(np.float32)
        dd = d.astype(np.float32)
        h = w.trace(org, dd)
        assert h.hit and (h.attrib & 0x8000) and h.group == 0
        # Exact slab test in the entity frame (double).
        ol = R.T @ (org.astype(np.float64) - pos)
        dl = R.T @ dd.astype(np.float64)
        t0 = (0.0 - ol) / dl
        t1 = (8.0 - ol) / dl
        near = np.minimum(t0, t1)
        axis = int(np.argmax(near))
        assert abs(h.t - near[axis]) < 2e-3
        n_local = np.zeros(3)
        n_local[axis] = -np.sign(dl[axis])
        assert np.allclose(np.array(h.normal[:]), R @ n_local, atol=1e-5)


def test_unreached_entity_leaves_the_render(oracle, world):
    w = oracle_lib.OracleScene(oracle, world)
    ref, rays = w.render(40, 32, spp=1, bounces=3, seed=2, threads=4)
    e = oracle_lib.OracleScene(oracle, entity_bricks())
    cam = world.camera
    behind = np.asarray(cam["position"], np.float64) - 1e6 * np.asarray(cam["forward"], np.float64)
    w.set_entities([(e, (0.0, 0.0, 0.0, 1.0), tuple(behind.astype(np.float32)))])
    img, rays2 = w.render(40, 32, spp=1, bounces=3, seed=2, threads=4)
    assert np.array_equal(img, ref) and np.array_equal(rays, rays2)


def test_entity_in_view_changes_the_render(oracle, world):
    """An entity in front of the camera is hit first: the render changes, stays finite and
    deterministic, and entity bricks add no emission (an all-entity view with NEE off is black)."""
    w = oracle_lib.OracleScene(oracle, world)
    ref, _ = w.render(40, 32, spp=1, bounces=3, seed=2, threads=4)
    e = oracle_lib.OracleScene(oracle, entity_bricks(fill=1.0))
    cam = world.camera
    front = np.asarray(cam["position"], np.float64) + 6.0 * np.asarray(cam["forward"], np.float64) - 8.0
    w.set_entities([(e, (0.1, 0.2, 0.05, 0.97), tuple(front.astype(np.float32)))])
    img, _ = w.render(40, 32, spp=1, bounces=3, seed=2, threads=4)
    img2, _ = w.render(40, 32, spp=1, bounces=3, seed=2, threads=1)
    assert np.array_equal(img, img2)
    assert np.all(np.isfinite(img)) and not np.array_equal(img, ref)
    dark, _ = w.render(40, 32, spp=1, bounces=0, seed=2, light_nee=False, threads=4)
    centre = dark[12:20, 16:24]
    assert np.all(centre == 0.0)
