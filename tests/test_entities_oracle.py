"""Entities in the oracle: bricks of their own traversed under a rigid transform after the world's
bricks (the reference's TLAS instances, shaders/render/caelix_scene_trace.hlsl:104-131: the ray in
the instance's object space, the committed object-to-world normal). Checked against independent
restatements: an entity at a translation equals the same bricks merged into the world; a rotated
solid brick is hit where an exact slab test in double precision says; an entity no ray reaches
leaves the render bit-identical. Entity lights (the reference's dynamic light tree,
docs/LIGHT_TREE.md:136-176): the pdf over both trees is normalised, draws from the second tree
match their pdf, and NEE over both trees with entity lamps converges to path tracing."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib
from caelix_b200 import workloads


def entity_bricks(grid=(2, 2, 2), seed=7, fill=0.55):
    """A small brick set of its own, without emitters."""
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


def light_faces(heap, rows, group_shift):
    """(group, voxel in group, face, block) of every face entry of a light set's blocks."""
    faces = []
    gm = (1 << group_shift) - 1
    for g, row in enumerate(rows):
        if row[1] == 0:
            continue
        block = int(row[0]) * 4
        for e in range(int(heap[block])):
            ie = block + 4 + 4 * e
            rec = block + 4 * int(heap[ie + 2])
            pos = int(heap[rec + 8])
            clo, chi = int(heap[rec + 10]), int(heap[rec + 11])
            counts = [(clo >> (10 * f)) & 0x3FF for f in range(3)] + [(chi >> (10 * f)) & 0x3FF for f in range(3)]
            bo = np.array([pos & gm, (pos >> group_shift) & gm, (pos >> (2 * group_shift)) & gm]) * 8
            first = 0
            for f in range(6):
                for q in range(counts[f]):
                    ent = int(heap[rec + 12 + first + q])
                    vi = ent & 0x1FF
                    v = bo + np.array([vi & 7, (vi >> 3) & 7, vi >> 6])
                    faces.append((g, v.astype(np.uint32), f, ent >> 16))
                first += counts[f]
    return faces


def lit_entity(grid, seed, fill=0.6, lit=0.5):
    vs = entity_bricks(grid=grid, seed=seed, fill=fill)
    rng = np.random.default_rng(seed)
    power = np.where(rng.random(vs.brick_count) < lit, rng.lognormal(0.0, 1.0, vs.brick_count), 0.0).astype(np.float32)
    return workloads.VoxelScene(vs.grid, vs.keys, vs.voxels, power, vs.albedo, vs.camera, vs.group_shift)


@pytest.fixture(scope="module")
def lit_scene(oracle, world):
    w = oracle_lib.OracleScene(oracle, world)
    e1 = oracle_lib.OracleScene(oracle, lit_entity((2, 2, 2), 31))
    e2 = oracle_lib.OracleScene(oracle, lit_entity((2, 1, 2), 32))
    # e1 static (its lights join the world's in tree 0), e2 dynamic (tree 1).
    w.set_entities([(e1, (0.2, -0.1, 0.3, 0.93), (60.0, 10.0, 5.0)), (e2, (0.0, 0.0, 0.0, 1.0), (-30.0, 20.0, 12.0))],
                   motions=[0, 1])
    assert w.s.dyn and w.dyn_tree["header"][0]["root"] != 0xFFFFFFFF
    assert w._merged0 is not None and w.tree["header"][0]["leaf_count"] == w.light_count + e1.light_count
    return w


def test_pdf_normalised_over_both_trees(lit_scene, world):
    """The light-tree pdf summed over every light face of the world and of the entities (each face
    of area 1 in its frame) is 1 (1e-4) for every receiver: the tree choice and both trees' walks
    are consistent (the reference's CheckNormalisation over its two trees; tree 0 holds the world's
    and the static entity's lights)."""
    w = lit_scene
    faces0 = light_faces(w.heap0, w.rows0, w.s.group_shift)
    assert len(faces0) > len(light_faces(w.heap, w.group_rows, w.s.group_shift))
    faces1 = light_faces(w.dyn_heap, w.dyn_rows, w.s.group_shift)
    assert faces0 and faces1
    rng = np.random.default_rng(8)
    span = np.array(world.grid, np.float64) * 8
    for _ in range(8):
        x = (rng.uniform(-0.5, 1.5, 3) * span).astype(np.float32)
        n = rng.normal(size=3)
        n = (n / np.linalg.norm(n)).astype(np.float32)
        total = 0.0
        for tree, faces in ((0, faces0), (1, faces1)):
            for g, v, f, blk in faces:
                total += w.lib.oc_light_point_pdf_tree(C.byref(w.s), C.byref(w.lt), x.ctypes.data, n.ctypes.data, tree,
                                                       g, np.ascontiguousarray(v).ctypes.data, f, blk)
        assert abs(total - 1.0) <= 1e-4, total


def test_entity_light_draws_match_their_pdf(lit_scene, world):
    """Draws from both trees: a drawn point's pdf equals the pdf evaluated at its face (1e-4), its
    position lies on the face under the entity's transform, and tree 1 is drawn."""
    w = lit_scene
    rng = np.random.default_rng(9)
    span = np.array(world.grid, np.float64) * 8
    drawn = [0, 0]
    for i in range(400):
        x = (rng.uniform(-0.5, 1.5, 3) * span).astype(np.float32)
        n = np.zeros(3, np.float32)
        out = np.zeros(7, np.float32)
        words = np.zeros(6, np.uint32)
        if not w.lib.oc_light_sample(C.byref(w.s), C.byref(w.lt), x.ctypes.data, n.ctypes.data, 77 + i,
                                     out.ctypes.data, words.ctypes.data):
            continue
        block, vi, face, group, entry, tree = (int(v) for v in words)
        drawn[tree] += 1
        frames = w.dyn_frames if tree else w.frames0
        fr = frames[group]
        R = fr["rotation"].reshape(3, 3).astype(np.float64)
        local = R.T @ (out[:3].astype(np.float64) - fr["translation"]) - fr["origin"]
        nl = R.T @ out[3:6].astype(np.float64)
        v = np.floor(local - 0.25 * nl + 1e-9).astype(np.int64)
        pdf = w.lib.oc_light_point_pdf_tree(C.byref(w.s), C.byref(w.lt), x.ctypes.data, n.ctypes.data, tree, group,
                                            np.ascontiguousarray(v.astype(np.uint32)).ctypes.data, face, block)
        assert abs(pdf - out[6]) <= 1e-4 * max(pdf, out[6]), (tree, pdf, out[6])
    assert drawn[0] > 20 and drawn[1] > 20, drawn


def test_entity_lamps_unbiased(oracle):
    """NEE with MIS over both trees converges to the plain path tracer when the lamps are entity
    bricks (rotated lamp panels in a closed room): the emission of entity hits, the second tree's
    draws and its pdf on BSDF hits agree (mean ratio in [0.97, 1.03], block PSNR above 30 dB)."""
    import os

    from test_light_nee_oracle import compare_light, lamp_box

    room = lamp_box()
    walls = room.power == 0
    world = workloads.VoxelScene(room.grid, room.keys[walls], room.voxels[walls], room.power[walls], room.albedo,
                                 room.camera, room.group_shift)
    panel = np.zeros((1, 512), np.uint16)
    v = np.arange(512)
    vx, vy, vz = v % 8, (v // 8) % 8, v // 64
    panel[0] = np.where((vy == 0) & (vx < 6) & (vz < 6), 0x8009, 0)
    lamp = workloads.VoxelScene((1, 1, 1), np.zeros((1, 3), np.int32), panel, np.full(1, 16.0, np.float32),
                                room.albedo, room.camera, room.group_shift)
    w = oracle_lib.OracleScene(oracle, world)
    lamps = [oracle_lib.OracleScene(oracle, lamp) for _ in range(3)]
    w.set_entities([(lamps[0], (0.1, 0.0, 0.05, 0.99), (10.0, 37.0, 12.0)),
                    (lamps[1], (0.0, 0.3, 0.0, 0.95), (28.0, 38.0, 26.0)),
                    (lamps[2], (-0.08, 0.0, 0.1, 0.99), (14.0, 36.0, 30.0))])
    threads = max(1, min(8, os.cpu_count() or 1))
    pt = w.render(32, 32, spp=2048, bounces=4, seed=100000, light_nee=False, threads=threads)[0]
    nee, rays = w.render(32, 32, spp=512, bounces=4, seed=200000, light_nee=True, threads=threads)
    assert rays[2] > 0
    ref_mean, test_mean, psnr = compare_light(pt, nee, direct=8.0)
    assert ref_mean > 0.01
    assert 0.97 < test_mean / ref_mean < 1.03, (ref_mean, test_mean)
    assert psnr > 30.0, psnr


def test_draw_histogram_over_both_trees(lit_scene, world):
    """2^21 draws at one receiver land on the light faces of both trees in proportion to their pdf
    (5 sigma for faces with at least 50 expected draws; no draw on a face of pdf 0), the
    reference's CheckHistogram over its two trees."""
    w = lit_scene
    faces = [(0, f) for f in light_faces(w.heap0, w.rows0, w.s.group_shift)] + \
            [(1, f) for f in light_faces(w.dyn_heap, w.dyn_rows, w.s.group_shift)]
    key = {}
    for i, (tree, (g, v, f, blk)) in enumerate(faces):
        key[(tree, g, int(v[0]) | (int(v[1]) << 10) | (int(v[2]) << 20), f)] = i
    x = (np.array(world.grid, np.float32) * 8 * np.float32(0.5)).astype(np.float32)
    n = np.zeros(3, np.float32)
    pdfs = np.array([w.lib.oc_light_point_pdf_tree(C.byref(w.s), C.byref(w.lt), x.ctypes.data, n.ctypes.data, tree, g,
                                                   np.ascontiguousarray(v).ctypes.data, f, blk)
                     for tree, (g, v, f, blk) in faces], np.float64)
    draws = 1 << 21
    out = np.zeros((draws, 4), np.uint32)
    w.lib.oc_light_draws(C.byref(w.s), C.byref(w.lt), x.ctypes.data, n.ctypes.data, 555, draws, out.ctypes.data)
    assert np.all(out[:, 3] & 1)
    rows, per = np.unique(np.column_stack([out[:, 3] >> 1, out[:, :3]]), axis=0, return_counts=True)
    counts = np.zeros(len(faces), np.int64)
    for r, c in zip(rows, per):
        i = key.get((int(r[0]), int(r[1]), int(r[2]), int(r[3])))
        assert i is not None, r
        counts[i] += c
    expected = pdfs * draws
    assert np.all(counts[pdfs == 0.0] == 0)
    big = expected >= 50.0
    in_dyn = np.array([t == 1 for t, _ in faces])
    assert big[in_dyn].sum() > 0 and big[~in_dyn].sum() > 0
    assert np.all(np.abs(counts[big] - expected[big]) <= 5.0 * np.sqrt(expected[big]))
