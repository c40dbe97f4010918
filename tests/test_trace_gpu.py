"""Parity of the CUDA scene build and trace (through the C ABI) with the oracle: bit-exact brick
records, hash table contents, light records and blocks, light tree; per-pixel radiance of the
path tracer with the same random streams (bit-exact expected; the tolerance written below is the
1e-5 relative bound), and equal ray counts (so every DDA hit and NEE decision matched)."""
import numpy as np
import pytest

import gpu_util
import oracle_lib
from caelix_b200 import workloads

pytestmark = pytest.mark.gpu

AGG_TOL = 1e-5  # per-pixel relative tolerance of the radiance (fp32)


def build_both(cuda_device, oracle, vs):
    import caelix_b200

    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    osc = oracle_lib.OracleScene(oracle, vs)
    return scene, osc


def fetch(v, dtype, ptr_name, count):
    return gpu_util.from_device(getattr(v, ptr_name), dtype, count)


def assert_scene_equal(scene, osc, vs):
    v = scene.view()
    n = vs.brick_count
    assert v.brick_count == n
    assert tuple(v.grid) == tuple(osc.grid) and tuple(v.origin) == tuple(osc.origin)
    assert v.encoding == vs.encoding
    assert fetch(v, np.int32, "keys", 3 * n).reshape(n, 3).tobytes() == vs.keys.tobytes()
    words = int(osc.s.bitmap_words)
    bitmap = np.ctypeslib.as_array(oracle_lib.C.cast(osc.s.bitmap, oracle_lib.C.POINTER(oracle_lib.C.c_uint32)),
                                   (max(words, 1),))[:words]
    assert np.array_equal(fetch(v, np.uint32, "bitmap", words), bitmap)
    rec = fetch(v, np.uint32, "records", 274 * n).reshape(n, 274)
    assert np.array_equal(rec, osc.records)
    assert v.hash_slot_count == osc.hash_slots.shape[0]
    assert v.hash_max_probe == osc.s.hash_max_probe
    slots = fetch(v, np.uint32, "hash_slots", 4 * v.hash_slot_count).reshape(-1, 4)
    assert np.array_equal(slots, osc.hash_slots)
    assert v.light_count == osc.light_count
    m = v.light_count
    if m:
        hdr = fetch(v, workloads.RECORD_DTYPE, "light_headers", m)
        assert hdr.tobytes() == osc.light_headers.tobytes()
        assert np.array_equal(fetch(v, np.uint32, "light_group", m), osc.light_group)
        assert np.array_equal(fetch(v, np.uint32, "light_entry", m), osc.light_entry)
        assert np.array_equal(fetch(v, np.uint32, "light_brick", m), osc.light_brick)
    assert v.heap_words == len(osc.heap)
    assert np.array_equal(fetch(v, np.uint32, "heap", v.heap_words), osc.heap)
    rows = fetch(v, np.uint32, "group_rows", 8 * v.group_count).reshape(-1, 8)
    # Word 2 is the group's generation, which follows the scene's flush history (the oracle builds
    # from scratch): tests/test_staging_gpu.py::test_group_generations checks it.
    words = [0, 1, 3, 4, 5, 6, 7]
    assert np.array_equal(rows[:, words], osc.group_rows[:, words])
    # The light tree.
    hdr = fetch(v, oracle_lib.HEADER_DTYPE, "tree_header", 1)
    assert hdr.tobytes() == osc.tree["header"].tobytes()
    if m:
        leaves = fetch(v, oracle_lib.LEAF_DTYPE, "tree_leaves", m)
        assert leaves.tobytes() == osc.tree["leaves"][:m].tobytes()
        nc = int(hdr[0]["node_count"])
        nodes = fetch(v, oracle_lib.NODE_DTYPE, "tree_nodes", nc)
        a = nodes.view(np.uint8).reshape(nc, 224)[:, :216]
        b = osc.tree["nodes"][:nc].view(np.uint8).reshape(nc, 224)[:, :216]
        assert np.array_equal(a, b)


def render_both(cuda_device, scene, osc, vs, width, height, spp=1, bounces=4, seed=1, window=None):
    import torch

    import caelix_b200

    r = caelix_b200.Renderer(cuda_device, scene)
    out = torch.zeros(height * width * 3, dtype=torch.float32, device="cuda")
    r.render(out, width, height, vs.camera, bounces=bounces, seed=seed, spp=spp)
    st = r.stats()
    gpu = out.cpu().numpy().reshape(height, width, 3)
    ref, rays = osc.render(width, height, spp=spp, bounces=bounces, seed=seed, window=window, threads=8)
    r.close()
    return gpu, ref, st, rays


def assert_radiance_close(gpu, ref, tol=AGG_TOL):
    diff = np.abs(gpu.astype(np.float64) - ref)
    bound = tol * np.maximum(np.abs(ref), 1e-30) + 1e-30
    bad = diff > bound
    assert not bad.any(), (int(bad.sum()), float(diff.max()))


def test_scene_and_trace_config2(cuda_device, oracle):
    vs = workloads.noise_world()
    scene, osc = build_both(cuda_device, oracle, vs)
    assert_scene_equal(scene, osc, vs)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, vs, 512, 512)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)
    scene.close()


@pytest.mark.parametrize("seed", [3, 9])
def test_scene_and_trace_small_scenes(cuda_device, oracle, seed):
    vs = workloads.noise_world(grid_bricks=(8, 6, 10), brick_occupancy=0.45, emissive_fraction=0.08, seed=seed)
    scene, osc = build_both(cuda_device, oracle, vs)
    assert_scene_equal(scene, osc, vs)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, vs, 96, 64, spp=2, bounces=6, seed=seed)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)
    scene.close()


def test_single_brick_and_edges(cuda_device, oracle):
    # One fully solid emissive brick next to a half-solid one: shared faces are closed, the rest open.
    keys = np.array([[0, 0, 0], [1, 0, 0]], np.int32)
    vox = np.full((2, 512), 0x8001, np.uint16)
    vox[1, 256:] = 0
    power = np.array([2.0, 0.0], np.float32)
    albedo = np.full((128, 3), 0.5, np.float32)
    cam = workloads.look_at([-10.0, 20.0, -15.0], [8.0, 4.0, 4.0])
    vs = workloads.VoxelScene((2, 1, 1), keys, vox, power, albedo, cam)
    scene, osc = build_both(cuda_device, oracle, vs)
    assert_scene_equal(scene, osc, vs)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, vs, 64, 64, spp=4, bounces=3)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)
    scene.close()


def test_scene_with_non_opaque_values(cuda_device, oracle):
    """Bricks holding non-opaque values other than air (finalize's per-voxel rules: face bits of
    differing neighbours) next to bricks of air and opaque values only (its mask path)."""
    vs = workloads.noise_world(grid_bricks=(8, 6, 10), brick_occupancy=0.45, emissive_fraction=0.08, seed=6)
    rng = np.random.default_rng(6)
    vox = vs.voxels.copy()
    mixed = rng.random(vs.brick_count) < 0.3
    cells = rng.random((vs.brick_count, 512)) < 0.2
    values = rng.integers(1, 0x8000, size=(vs.brick_count, 512)).astype(np.uint16)
    pick = mixed[:, None] & cells & (vox == 0)
    vox[pick] = values[pick]
    vs = workloads.VoxelScene(vs.grid, vs.keys, vox, vs.power, vs.albedo, vs.camera, vs.group_shift)
    scene, osc = build_both(cuda_device, oracle, vs)
    assert_scene_equal(scene, osc, vs)
    gpu, ref, st, rays = render_both(cuda_device, scene, osc, vs, 96, 64, spp=2, bounces=4, seed=6)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(gpu, ref)
    scene.close()


def test_render_is_deterministic(cuda_device, oracle):
    import torch

    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(8, 8, 8), seed=5)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    r = caelix_b200.Renderer(cuda_device, scene)
    a = torch.zeros(128 * 128 * 3, device="cuda")
    b = torch.zeros(128 * 128 * 3, device="cuda")
    r.render(a, 128, 128, vs.camera, seed=7)
    r.render(b, 128, 128, vs.camera, seed=7)
    assert torch.equal(a, b)
    r.close()
    scene.close()


@pytest.mark.parametrize("capacity", [0, 4096, 777])
def test_wavefront_equals_megakernel(cuda_device, capacity):
    """The two kernel organisations give the same radiance bit for bit and the same ray counts,
    whatever the wave capacity (small capacities split a sample into many sub-waves)."""
    import torch

    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(10, 8, 12), brick_occupancy=0.4, emissive_fraction=0.06, seed=13)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    r = caelix_b200.Renderer(cuda_device, scene)
    w, h = 100, 70
    outs, rays = [], []
    for mode in (caelix_b200.Renderer.TRACE_MEGAKERNEL, caelix_b200.Renderer.TRACE_WAVEFRONT):
        r.set_trace_mode(mode, capacity if mode == caelix_b200.Renderer.TRACE_WAVEFRONT else 0)
        out = torch.full((w * h * 3,), -1.0, device="cuda")
        r.render(out, w, h, vs.camera, bounces=5, seed=4, spp=3)
        st = r.stats()
        outs.append(out.cpu().numpy())
        rays.append((st.primary_rays, st.bounce_rays, st.shadow_rays))
    assert outs[0].view(np.uint32).tobytes() == outs[1].view(np.uint32).tobytes()
    assert rays[0] == rays[1]
    r.close()
    scene.close()
