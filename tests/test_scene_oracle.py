"""The oracle's scene and light-tree device API against the reference's known answers
(tests/light_tree_test.cpp: CheckNormalisation :888, sample/pdf consistency, the light-face CPU
model; tests/hash_table_test.cpp: the fingerprint) and against independent numpy restatements:
finalize occupancy, the canonical hash layout, brick light records."""
import numpy as np
import pytest

import oracle_lib
from caelix_b200 import workloads


@pytest.fixture(scope="module")
def small_scene():
    return workloads.noise_world(grid_bricks=(8, 8, 8), brick_occupancy=0.4, emissive_fraction=0.05, seed=9)


@pytest.fixture(scope="module")
def osc(oracle, small_scene):
    return oracle_lib.OracleScene(oracle, small_scene)


def splitmix64(x):
    x = (x + 0x9E3779B97F4A7C15) & (2**64 - 1)
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
    return x ^ (x >> 31)


def fingerprint(x, y, z):
    h = splitmix64(0 ^ ((y & 0xFFFFFFFF) << 32 | (x & 0xFFFFFFFF)))
    h = splitmix64(h ^ (z & 0xFFFFFFFF))
    lo, hi = h & 0xFFFFFFFF, h >> 32
    return max(lo, 1), hi if hi else 1


def test_splitmix64_known_answer():
    # splitmix64 reference outputs for seed 0 (Vigna's generator: state += golden; mix).
    assert splitmix64(0) == 0xE220A8397B1DCDAF


def test_hash_table_canonical_layout(osc, small_scene):
    s = small_scene
    n = s.brick_count
    cap = 2 * n
    slots = osc.hash_slots
    assert slots.shape[0] == cap + n + 1
    # Every key is found, at its home or after a run of occupied slots.
    for i, (x, y, z) in enumerate(s.keys):
        assert osc.lookup(int(x), int(y), int(z)) == i
    # History independence: placing keys in (home, brick) order gives the oracle's table.
    fp = [fingerprint(*map(int, k)) for k in s.keys]
    homes = np.array([(lo * cap) >> 32 for lo, hi in fp], np.int64)
    order = np.lexsort((np.arange(n), homes))
    expect = np.zeros_like(slots)
    prev = -1
    for b in order:
        pos = max(homes[b], prev + 1)
        prev = pos
        expect[pos] = (fp[b][0], fp[b][1], b, 0)
    assert np.array_equal(expect, slots)
    # Absent keys miss.
    assert osc.lookup(500, 500, 500) == 0xFFFFFFFF
    assert osc.lookup(-1, 0, 0) == 0xFFFFFFFF


def test_finalize_occupancy_matches_numpy(osc, small_scene):
    s = small_scene
    gx, gy, gz = s.grid
    dense = np.zeros((gz * 8 + 2, gy * 8 + 2, gx * 8 + 2), np.uint16)  # padded z, y, x
    for (x, y, z), vox in zip(s.keys, s.voxels):
        dense[1 + z * 8:1 + z * 8 + 8, 1 + y * 8:1 + y * 8 + 8, 1 + x * 8:1 + x * 8 + 8] = vox.reshape(8, 8, 8)
    opaque = (dense & 0x8000) != 0
    nb = (opaque[2:, 1:-1, 1:-1].astype(int) + opaque[:-2, 1:-1, 1:-1] + opaque[1:-1, 2:, 1:-1] +
          opaque[1:-1, :-2, 1:-1] + opaque[1:-1, 1:-1, 2:] + opaque[1:-1, 1:-1, :-2])
    occupied = opaque[1:-1, 1:-1, 1:-1] & (nb < 6)
    for i, (x, y, z) in enumerate(s.keys):
        occ = occupied[z * 8:z * 8 + 8, y * 8:y * 8 + 8, x * 8:x * 8 + 8]
        rec = osc.records[i]
        bits = np.zeros((8, 8, 8), bool)
        for vz in range(8):
            for vy in range(8):
                for vx in range(8):
                    c = (vx >> 2) | ((vy >> 2) << 1) | ((vz >> 2) << 2)
                    m = (vx & 3) | ((vy & 3) << 2) | ((vz & 3) << 4)
                    w = rec[2 + 2 * c + (m >> 5)]
                    bits[vz, vy, vx] = (w >> (m & 31)) & 1
        assert np.array_equal(bits, occ), i
        # Tight bounds and the coarse byte.
        if occ.any():
            zz, yy, xx = np.nonzero(occ)
            tb = int(rec[1])
            assert (tb & 7, (tb >> 3) & 7, (tb >> 6) & 7) == (xx.min(), yy.min(), zz.min())
            assert ((tb >> 9) & 7, (tb >> 12) & 7, (tb >> 15) & 7) == (xx.max(), yy.max(), zz.max())
        # The payload keeps the uploaded values.
        pay = rec[18:274]
        vals = np.stack([pay & 0xFFFF, pay >> 16], -1).reshape(-1).astype(np.uint16)
        assert np.array_equal(vals, s.voxels[i])


def test_light_records_count_open_faces(osc, small_scene):
    s = small_scene
    emissive = np.nonzero(s.power > 0)[0]
    assert osc.light_count == len(emissive)
    assert set(osc.light_brick.tolist()) == set(emissive.tolist())
    for k in range(osc.light_count):
        h = osc.light_headers[k]
        counts = [(h["counts_lo"] >> (10 * f)) & 0x3FF for f in range(3)] + \
                 [(h["counts_hi"] >> (10 * f)) & 0x3FF for f in range(3)]
        assert sum(counts) == h["entry_count"]
        P = np.float32(s.power[osc.light_brick[k]])
        for f in range(6):
            # All entries of a brick carry the same weight: the sum is close to count * weight.
            assert abs(float(h["face"][f]) - counts[f] * float(P)) <= 1e-5 * max(1.0, counts[f] * float(P))


def receivers(small_scene, count, seed):
    rng = np.random.default_rng(seed)
    world = np.array(small_scene.grid, np.float64) * 8
    x = rng.uniform(-0.2, 1.2, size=(count, 3)) * world
    n = rng.normal(size=(count, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    return x.astype(np.float32), n.astype(np.float32)


def all_light_faces(osc):
    """(group, voxel_in_group, face, block) of every face entry of every light record."""
    import ctypes as C

    faces = []
    heap = osc.heap
    for g, row in enumerate(osc.group_rows):
        if row[1] == 0:
            continue
        block = int(row[0]) * 4
        count = heap[block]
        for e in range(count):
            ie = block + 4 + 4 * e
            rec = block + 4 * int(heap[ie + 2])
            pos = int(heap[rec + 8])
            clo, chi = int(heap[rec + 10]), int(heap[rec + 11])
            counts = [(clo >> (10 * f)) & 0x3FF for f in range(3)] + [(chi >> (10 * f)) & 0x3FF for f in range(3)]
            first = 0
            gs = osc.s.group_shift
            gm = (1 << gs) - 1
            bo = np.array([pos & gm, (pos >> gs) & gm, (pos >> (2 * gs)) & gm]) * 8
            for f in range(6):
                for q in range(counts[f]):
                    ent = int(heap[rec + 12 + first + q])
                    vi = ent & 0x1FF
                    v = bo + np.array([vi & 7, (vi >> 3) & 7, vi >> 6])
                    faces.append((g, v.astype(np.uint32), f, ent >> 16))
                first += counts[f]
    return faces


def test_light_pdf_normalisation(osc, small_scene):
    """Sum of the pdfs of all light faces (each of area 1) is 1 for every receiver
    (the reference's CheckNormalisation, tests/light_tree_test.cpp:888, tolerance 1e-4)."""
    import ctypes as C

    faces = all_light_faces(osc)
    assert faces
    xs, ns = receivers(small_scene, 12, 4)
    for x, n in zip(xs, ns):
        total = 0.0
        for g, v, f, blk in faces:
            total += osc.lib.oc_light_point_pdf(C.byref(osc.s), C.byref(osc.lt), x.ctypes.data, n.ctypes.data, g,
                                                np.ascontiguousarray(v).ctypes.data, f, blk)
        assert abs(total - 1.0) <= 1e-4, total


def test_light_sample_pdf_consistency(osc, small_scene):
    """A drawn point's pdf equals the pdf evaluated at its face (1e-4 relative)."""
    import ctypes as C

    xs, ns = receivers(small_scene, 64, 5)
    checked = 0
    for i, (x, n) in enumerate(zip(xs, ns)):
        out = np.zeros(7, np.float32)
        words = np.zeros(6, np.uint32)
        ok = osc.lib.oc_light_sample(C.byref(osc.s), C.byref(osc.lt), x.ctypes.data, n.ctypes.data, 1000 + i,
                                     out.ctypes.data, words.ctypes.data)
        if not ok:
            continue
        block, vi, face, group, entry, tree = (int(w) for w in words)
        assert tree == 0
        fr = osc.group_frames[group]
        v = np.floor(out[:3] - 0.25 * out[3:6] - fr["origin"]).astype(np.int64)
        pdf = osc.lib.oc_light_point_pdf(C.byref(osc.s), C.byref(osc.lt), x.ctypes.data, n.ctypes.data, group,
                                         np.ascontiguousarray(v.astype(np.uint32)).ctypes.data, face, block)
        assert abs(pdf - out[6]) <= 1e-4 * max(pdf, out[6]), (pdf, out[6])
        checked += 1
    assert checked > 10


def test_sincos_accuracy(oracle):
    import ctypes as C

    oracle_lib._bind_scene(oracle)
    s, c = C.c_float(), C.c_float()
    for a in np.linspace(0.0, 2 * np.pi, 4001, dtype=np.float32):
        oracle.oc_sincos(float(a), C.byref(s), C.byref(c))
        assert abs(s.value - np.sin(np.float64(a))) < 2e-6
        assert abs(c.value - np.cos(np.float64(a))) < 2e-6


def test_oracle_render_properties(osc):
    img, rays = osc.render(48, 48, spp=1, bounces=4, seed=3)
    assert np.all(np.isfinite(img)) and np.all(img >= 0)
    assert rays[0] == 48 * 48
    img2, rays2 = osc.render(48, 48, spp=1, bounces=4, seed=3, threads=4)
    assert np.array_equal(img, img2) and np.array_equal(rays, rays2)


def face_table(osc):
    """The light faces keyed like the reference's RefFace index: (group, packed voxel in group, face)."""
    faces = all_light_faces(osc)
    keys = {}
    for i, (g, v, f, blk) in enumerate(faces):
        keys[(g, int(v[0]) | (int(v[1]) << 10) | (int(v[2]) << 20), f)] = i
    assert len(keys) == len(faces)
    return faces, keys


def face_pdfs(osc, faces, x, n):
    import ctypes as C

    return np.array([osc.lib.oc_light_point_pdf(C.byref(osc.s), C.byref(osc.lt), x.ctypes.data, n.ctypes.data, g,
                                                np.ascontiguousarray(v).ctypes.data, f, blk)
                     for g, v, f, blk in faces], np.float32)


@pytest.mark.parametrize("with_normal", [False, True])
def test_light_sample_histogram(osc, small_scene, with_normal):
    """2^21 draws at one receiver land on each light face in proportion to its pdf: every face with
    at least 50 expected draws is within 5 sigma of pdf * draws, and a face of pdf 0 is never drawn
    (the reference's CheckHistogram, tests/light_tree_test.cpp:961-993)."""
    import ctypes as C

    faces, keys = face_table(osc)
    world = np.array(small_scene.grid, np.float32) * 8
    x = np.ascontiguousarray(world * np.float32(0.45))
    n = np.zeros(3, np.float32)
    if with_normal:
        n = np.array([0.3, 0.8, -0.52], np.float32)
        n /= np.float32(np.linalg.norm(n))
    pdfs = face_pdfs(osc, faces, x, n)
    draws = 1 << 21
    out = np.zeros((draws, 4), np.uint32)
    osc.lib.oc_light_draws(C.byref(osc.s), C.byref(osc.lt), x.ctypes.data, n.ctypes.data, 777, draws,
                           out.ctypes.data)
    assert np.all(out[:, 3] == 1)
    packed, inverse = np.unique(out[:, :3], axis=0, return_inverse=True)
    counts = np.zeros(len(faces), np.int64)
    per_key = np.bincount(inverse.reshape(-1), minlength=len(packed))
    for row, c in zip(packed, per_key):
        index = keys.get((int(row[0]), int(row[1]), int(row[2])))
        assert index is not None, row
        counts[index] += c
    expected = pdfs.astype(np.float64) * draws
    assert np.all(counts[pdfs == 0.0] == 0)
    big = expected >= 50.0
    assert big.sum() > 0
    assert np.all(np.abs(counts[big] - expected[big]) <= 5.0 * np.sqrt(expected[big])), \
        np.max(np.abs(counts[big] - expected[big]) / np.sqrt(expected[big]))


def test_light_pdf_bound(osc):
    """A receiver that sees a light face's centre with both cosines above 0.05 gets a positive pdf
    for that face: the tree's importance bounds never cull a contributing light (the reference's
    CheckBound, tests/light_tree_test.cpp:995-1064; receivers within 4 or 60 voxels of the centre,
    every second one without a normal)."""
    import ctypes as C

    faces = all_light_faces(osc)
    dirs = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], np.float32)
    rng = np.random.default_rng(1234)
    checked = 0
    for k in range(4096):
        g, v, f, blk = faces[int(rng.integers(len(faces)))]
        fr = osc.group_frames[g]
        rot = fr["rotation"].reshape(3, 3)
        centre = rot @ (fr["origin"] + v.astype(np.float32) + 0.5 + 0.5 * dirs[f]) + fr["translation"]
        normal = rot @ dirs[f]
        rng_range = 4.0 if k % 3 == 0 else 60.0
        x = (centre + rng.uniform(-1.0, 1.0, 3) * rng_range).astype(np.float32)
        m = rng.uniform(-1.0, 1.0, 3)
        has_normal = k % 2 == 0
        n = (m / np.linalg.norm(m)).astype(np.float32) if has_normal else np.zeros(3, np.float32)
        d = x - centre
        dist = float(np.linalg.norm(d))
        if dist < 0.5:
            continue
        emitter = float(normal @ d) / dist
        receiving = float(-(n @ d)) / dist if has_normal else 1.0
        if emitter < 0.05 or receiving < 0.05:
            continue
        pdf = osc.lib.oc_light_point_pdf(C.byref(osc.s), C.byref(osc.lt), x.ctypes.data, n.ctypes.data, g,
                                         np.ascontiguousarray(v).ctypes.data, f, blk)
        assert pdf > 0.0, (k, g, v, f)
        checked += 1
    assert checked > 100
