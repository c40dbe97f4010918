"""The oracle's NEE/MIS pieces against the reference's light NEE tests
(tests/light_nee_test.cpp:552-675): the MIS weight at degenerate and regular inputs, and both MIS
sides of a drawn lamp point (the light draw and the BSDF ray that reaches the same light face) seeing
the same pdf, with weights that sum to 1. The CUDA integrator's mis_weight has the same branches
and is checked through whole renders against the oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib
from caelix_b200 import workloads

INV_SQRT2 = np.float32(1.0 / np.sqrt(2.0))
INF = np.float32(np.inf)
NAN = np.float32(np.nan)

# (name, p_area, d, cos_l, w, expected nee weight, expected bsdf weight); None: both positive.
# The receiver normal is +Y in every case.
MIS_CASES = [
    ("regular", 0.01, 10.0, 0.5, (0.0, INV_SQRT2, INV_SQRT2), None, None),
    ("regular, grazing receiver", 0.2, 30.0, 0.9, (0.0, 1e-4, 1.0), None, None),
    ("lamp facing away", 0.01, 10.0, -0.5, (0.0, 1.0, 0.0), 1.0, 0.0),
    ("lamp edge-on", 0.01, 10.0, 0.0, (0.0, 1.0, 0.0), 1.0, 0.0),
    ("infinite density", INF, 10.0, 0.5, (0.0, 1.0, 0.0), 1.0, 0.0),
    ("NaN density", NAN, 10.0, 0.5, (0.0, 1.0, 0.0), 1.0, 0.0),
    ("overflowing solid-angle density", 1e30, 1e10, 1e-10, (0.0, 1.0, 0.0), 1.0, 0.0),
    ("zero density, receiver facing away", 0.0, 10.0, 0.5, (0.0, -1.0, 0.0), 0.0, 1.0),
    ("zero density", 0.0, 10.0, 0.5, (0.0, 1.0, 0.0), 0.0, 1.0),
    ("receiver facing away", 0.01, 10.0, 0.5, (0.0, -1.0, 0.0), 1.0, 0.0),
]


@pytest.fixture(scope="module")
def lamp_scene(oracle):
    vs = workloads.noise_world(grid_bricks=(8, 8, 8), brick_occupancy=0.35, emissive_fraction=0.08, seed=21)
    return vs, oracle_lib.OracleScene(oracle, vs)


def mis(lib, p_area, n, w, d, cos_l, nee_side):
    n = np.ascontiguousarray(n, np.float32)
    w = np.ascontiguousarray(w, np.float32)
    return lib.oc_mis_weight(float(p_area), n.ctypes.data, w.ctypes.data, float(d), float(cos_l), 1 if nee_side else 0)


@pytest.mark.parametrize("case", MIS_CASES, ids=[c[0] for c in MIS_CASES])
def test_mis_weight_degenerate_inputs(oracle, case):
    oracle_lib._bind_scene(oracle)
    name, p_area, d, cos_l, w, nee, bsdf = case
    n = (0.0, 1.0, 0.0)
    w_nee = mis(oracle, p_area, n, w, d, cos_l, True)
    w_bsdf = mis(oracle, p_area, n, w, d, cos_l, False)
    assert np.isfinite(w_nee) and np.isfinite(w_bsdf)
    assert abs(float(w_nee) + float(w_bsdf) - 1.0) < 1e-6
    if nee is None:
        assert w_nee > 0.0 and w_bsdf > 0.0
    else:
        assert w_nee == nee and w_bsdf == bsdf


def surface_receivers(vs, osc, count, seed):
    """Surface points with their normals: the first hits of random rays from inside the world."""
    rng = np.random.default_rng(seed)
    world = np.array(vs.grid, np.float64) * 8
    out = []
    while len(out) < count:
        o = rng.uniform(0.05, 0.95, 3) * world
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        h = osc.trace(o, d)
        if not h.hit:
            continue
        normal = np.array(h.normal[:], np.float32)
        x = (o.astype(np.float32) + d.astype(np.float32) * np.float32(h.t)) + np.float32(0.002) * normal
        out.append((x.astype(np.float32), normal))
    return out


def test_mis_sides_see_the_same_pdf(lamp_scene):
    """A lamp point drawn by the light tree, reached again by a ray toward it (the BSDF side), has the
    same pdf on both sides (1e-4 relative: the draw multiplies its choices top-down, the evaluation
    walks bottom-up) and the two MIS weights sum to 1 (1e-4)."""
    vs, osc = lamp_scene
    lib = osc.lib
    draws_per_receiver = 8
    ok = total = 0
    for i, (x, n) in enumerate(surface_receivers(vs, osc, 150, 23)):
        for k in range(draws_per_receiver):
            total += 1
            out = np.zeros(7, np.float32)
            words = np.zeros(6, np.uint32)
            if not lib.oc_light_sample(C.byref(osc.s), C.byref(osc.lt), x.ctypes.data, n.ctypes.data,
                                       99 + 977 * i + k, out.ctypes.data, words.ctypes.data):
                continue
            p_nee = float(out[6])
            d = out[:3] - x
            dist = np.float32(np.sqrt(np.float32(d @ d)))
            if not dist > 0:
                continue
            w = (d / dist).astype(np.float32)
            cos_l = float(-(out[3:6] @ w))
            if not (cos_l > 0.0 and float(n @ w) > 0.0):
                continue
            h = osc.trace(x, w, 0.0, float(dist) + 1.0)
            if not h.hit:
                continue
            hit_normal = np.array(h.normal[:], np.float32)
            voxel = np.floor(np.array(h.object_hit[:], np.float32) - np.float32(0.25) * hit_normal).astype(np.int64)
            face = (h.attrib & 0x3F).bit_length() - 1
            block = (h.attrib >> 16) & 0xFFFF
            fr = osc.group_frames[h.group]
            vig = (voxel - fr["origin"].astype(np.int64)).astype(np.uint32)
            same = (h.group == words[3] and face == words[2] and block == words[0] and
                    np.array_equal(vig, np.floor(out[:3] - 0.25 * out[3:6] - fr["origin"]).astype(np.uint32)))
            if not same:
                continue  # occluded: the BSDF ray ends on another surface
            p_bsdf = lib.oc_light_point_pdf(C.byref(osc.s), C.byref(osc.lt), x.ctypes.data, n.ctypes.data, h.group,
                                            np.ascontiguousarray(vig).ctypes.data, face, block)
            assert p_bsdf > 0.0
            assert abs(p_bsdf / p_nee - 1.0) < 1e-4, (p_nee, p_bsdf)
            w_nee = mis(lib, p_nee, n, w, dist, cos_l, True)
            w_bsdf = mis(lib, p_bsdf, n, w, float(h.t), float(-(hit_normal @ w)), False)
            assert abs(float(w_nee) + float(w_bsdf) - 1.0) < 1e-4, (w_nee, w_bsdf)
            ok += 1
    assert ok >= 50, (ok, total)  # 125 of 1200 draws reach their lamp unoccluded in this cave world


def lamp_box(n=6, power=16.0):
    """A closed room of n^3 bricks (walls one voxel thick, eight albedo materials) lit only by four
    4 x 1 x 4-voxel lamp panels below the ceiling, each in a brick of its own with emitter power
    `power`; the camera looks across the room from near one wall."""
    v = np.arange(512)
    vx, vy, vz = v % 8, (v // 8) % 8, v // 64
    size = n * 8
    keys, voxels, power_of = [], [], []
    for bz in range(n):
        for by in range(n):
            for bx in range(n):
                gx, gy, gz = bx * 8 + vx, by * 8 + vy, bz * 8 + vz
                wall = (gx == 0) | (gx == size - 1) | (gy == 0) | (gy == size - 1) | (gz == 0) | (gz == size - 1)
                panel = (by == n - 2) and bx in (1, n - 2) and bz in (1, n - 2)
                lamp = panel & (vy == 4) & (vx >= 2) & (vx < 6) & (vz >= 2) & (vz < 6)
                material = (1 + (gx * 7 + gy * 3 + gz * 5) % 8).astype(np.uint16)
                if wall.any():
                    keys.append((bx, by, bz))
                    voxels.append(np.where(wall, np.uint16(0x8000) | material, np.uint16(0)))
                    power_of.append(0.0)
                elif lamp.any():
                    keys.append((bx, by, bz))
                    voxels.append(np.where(lamp, np.uint16(0x8000 | 9), np.uint16(0)))
                    power_of.append(power)
    albedo = np.full((128, 3), 0.6, np.float32)
    albedo[1:9] = np.linspace(0.3, 0.8, 24, dtype=np.float32).reshape(8, 3)
    camera = workloads.look_at((size * 0.5, size * 0.35, size * 0.08), (size * 0.5, size * 0.45, size * 0.9))
    return workloads.VoxelScene((n, n, n), np.array(keys, np.int32), np.array(voxels, np.uint16),
                                np.array(power_of, np.float32), albedo, camera, 4)


def compare_light(ref, test, direct, block=8):
    """The reference's CompareLight (tests/trace_test.cpp:3034-3087): pixels that see a lamp
    directly (a channel above `direct` in the reference image) are left out; returns the mean
    ratio test / reference and the PSNR of the block means clamped to [0, 1]."""
    h, w, _ = ref.shape
    squared = values = 0.0
    blocks = 0
    ref_sum = test_sum = 0.0
    for by in range(0, h, block):
        for bx in range(0, w, block):
            r = ref[by:by + block, bx:bx + block].reshape(-1, 3).astype(np.float64)
            t = test[by:by + block, bx:bx + block].reshape(-1, 3).astype(np.float64)
            keep = ~(r > direct).any(axis=1)
            used = int(keep.sum())
            if used == 0:
                continue
            rb, tb = r[keep].sum(0), t[keep].sum(0)
            ref_sum += rb.sum()
            test_sum += tb.sum()
            squared += float(((np.clip(tb / used, 0, 1) - np.clip(rb / used, 0, 1)) ** 2).sum())
            values += 3 * used
            blocks += 1
    mse = squared / (3 * blocks)
    return ref_sum / values, test_sum / values, 10 * np.log10(1 / mse) if mse > 0 else 99.0


def test_light_nee_unbiased_against_path_tracing(oracle):
    """Light-tree NEE with MIS converges to the plain path tracer (lamps found only by bounce rays):
    mean ratio in [0.97, 1.03] and 8 x 8-block PSNR above 30 dB over the pixels that do not see a
    lamp directly (the reference's unbiasedness test, tests/trace_test.cpp:3100-3173; here 2048
    path-traced and 512 NEE samples per pixel of a 32 x 32 view of a lamp-lit room)."""
    import os

    vs = lamp_box()
    osc = oracle_lib.OracleScene(oracle, vs)
    threads = max(1, min(8, os.cpu_count() or 1))
    pt = osc.render(32, 32, spp=2048, bounces=4, seed=100000, light_nee=False, threads=threads)[0]
    nee, rays = osc.render(32, 32, spp=512, bounces=4, seed=200000, light_nee=True, threads=threads)
    assert rays[2] > 0  # shadow rays: NEE ran
    ref_mean, test_mean, psnr = compare_light(pt, nee, direct=8.0)
    assert ref_mean > 0.01
    assert 0.97 < test_mean / ref_mean < 1.03, (ref_mean, test_mean)
    assert psnr > 30.0, psnr
