"""The batched path (caelix_batch_*): per-scene light-tree rebuilds and one persistent trace launch
in a CUDA graph. Each view's radiance must be bit-identical to a plain render of the same
renderer, target, camera and options (itself checked against the oracle), with the same ray
counts, for every register-cap variant, pixel block shape, refill threshold and view order; the
rebuilt light trees must equal the flush-built ones byte for byte; a light-tree-only flush must
leave the tree unchanged; the autotuner must store and reuse its cache entry."""
import json

import numpy as np
import pytest

import gpu_util
import oracle_lib
from caelix_b200 import workloads

pytestmark = pytest.mark.gpu


def tree_bytes(scene):
    v = scene.view()
    hdr = gpu_util.from_device(v.tree_header, oracle_lib.HEADER_DTYPE, 1)
    m = int(hdr[0]["leaf_count"])
    nc = int(hdr[0]["node_count"])
    leaves = gpu_util.from_device(v.tree_leaves, oracle_lib.LEAF_DTYPE, max(m, 1))[:m]
    nodes = gpu_util.from_device(v.tree_nodes, oracle_lib.NODE_DTYPE, max(nc, 1))[:nc]
    return hdr.tobytes() + leaves.tobytes() + nodes.view(np.uint8).reshape(-1, 224)[:, :216].tobytes()


@pytest.fixture(scope="module")
def small_batch(cuda_device):
    """Three scenes, six views of uneven sizes (ragged pixel blocks included), and their plain
    renders."""
    import torch

    import caelix_b200

    worlds = [
        workloads.noise_world(grid_bricks=(8, 8, 8), brick_occupancy=0.45, emissive_fraction=0.08, seed=3),
        workloads.noise_world(grid_bricks=(12, 10, 9), emissive_fraction=0.05, seed=7),
        workloads.batch_scene(3000, seed=11),
    ]
    scenes = [caelix_b200.Scene.from_voxel_scene(cuda_device, vs) for vs in worlds]
    renderers = [caelix_b200.Renderer(cuda_device, s) for s in scenes]
    # (scene, width, height, bounces, seed, spp)
    shapes = [(0, 64, 48, 4, 1, 2), (1, 40, 40, 3, 5, 1), (2, 128, 64, 4, 2, 2), (0, 33, 17, 6, 9, 3),
              (2, 96, 96, 2, 4, 1), (1, 70, 31, 4, 8, 2)]
    views, plain = [], []
    for si, w, h, bounces, seed, spp in shapes:
        vs = worlds[si]
        cam = dict(vs.camera)
        cam["aspect"] = np.float32(w / h)
        out = torch.zeros(h * w * 3, dtype=torch.float32, device="cuda")
        renderers[si].render(out, w, h, cam, bounces=bounces, seed=seed, spp=spp)
        st = renderers[si].stats()
        plain.append((out.cpu().numpy().reshape(h, w, 3).copy(),
                      (st.primary_rays, st.bounce_rays, st.shadow_rays)))
        target = torch.full((h * w * 3,), -1.0, dtype=torch.float32, device="cuda")
        views.append((renderers[si], target, w, h, cam, bounces, seed, spp))
    trees = [tree_bytes(s) for s in scenes]
    yield dict(worlds=worlds, scenes=scenes, renderers=renderers, views=views, plain=plain, trees=trees,
               shapes=shapes)
    for r in renderers:
        r.close()
    for s in scenes:
        s.close()


def check_views(batch, small_batch):
    for i, ((_, target, w, h, *_), (ref, rays)) in enumerate(zip(small_batch["views"], small_batch["plain"])):
        got = target.cpu().numpy().reshape(h, w, 3)
        assert got.view(np.uint32).tobytes() == ref.view(np.uint32).tobytes(), f"view {i}"
        st = batch.view_stats(i)
        assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == rays, f"view {i}"


@pytest.mark.parametrize("min_blocks", [4, 6, 8, "wave"])
def test_batch_matches_plain_renders(cuda_device, small_batch, min_blocks):
    import caelix_b200

    batch = caelix_b200.Batch(cuda_device, small_batch["views"], rebuild_light_trees=True)
    wave = min_blocks == "wave"
    for block_width, refill_min, order in [(16, 4, 1), (8, 1, 0), (32, 16, 1)]:
        for v in small_batch["views"]:
            v[1].fill_(-1.0)
        batch.set_tuning(min_blocks=6 if wave else min_blocks, block_width=block_width, refill_min=refill_min,
                         order=order, sort_keys_per_thread=4 if order else 16, kernel=1 if wave else 0,
                         wavefront=(4096 if order else 0) if wave else 0)
        batch.run()
        st = batch.stats()
        check_views(batch, small_batch)
        assert st.primary_rays == sum(r[1][0] for r in small_batch["plain"])
        assert st.light_tree_builds == 3 and st.kernel_launches > 3
    # The rebuilt light trees are the flush-built ones.
    for s, t in zip(small_batch["scenes"], small_batch["trees"]):
        assert tree_bytes(s) == t
    batch.close()


def test_batch_small_wavefront_and_trace_only(cuda_device, small_batch):
    import caelix_b200

    batch = caelix_b200.Batch(cuda_device, small_batch["views"], rebuild_light_trees=False)
    batch.set_tuning(min_blocks=6, wavefront=128 * 3, refill_min=2)  # 3 CTAs: long-lived lanes
    batch.run()
    st = batch.stats()
    assert st.wavefront == 128 * 3 and st.light_tree_builds == 0
    check_views(batch, small_batch)
    batch.close()


def test_batch_view_vs_oracle(cuda_device, oracle, small_batch):
    """One batched view against the oracle directly (1e-5 relative, equal ray counts)."""
    import caelix_b200
    from test_trace_gpu import assert_radiance_close

    vs = small_batch["worlds"][1]
    batch = caelix_b200.Batch(cuda_device, [small_batch["views"][1]])
    batch.run()
    _, target, w, h, cam, bounces, seed, spp = small_batch["views"][1]
    ref_vs = workloads.VoxelScene(vs.grid, vs.keys, vs.voxels, vs.power, vs.albedo, cam)
    ref, rays = oracle_lib.OracleScene(oracle, ref_vs).render(w, h, spp=spp, bounces=bounces, seed=seed, threads=8)
    st = batch.view_stats(0)
    assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == tuple(int(x) for x in rays)
    assert_radiance_close(target.cpu().numpy().reshape(h, w, 3), ref)
    batch.close()


def test_light_tree_only_flush(cuda_device, small_batch):
    scene = small_batch["scenes"][1]
    scene.set_light_options(True)
    scene.flush()
    assert tree_bytes(scene) == small_batch["trees"][1]
    assert scene.light_stats().tree_builds[0] >= 2


def test_autotune_cache(cuda_device, small_batch, tmp_path):
    import caelix_b200

    cache = tmp_path / "tuning.json"
    batch = caelix_b200.Batch(cuda_device, small_batch["views"][:3])
    t = batch.autotune(str(cache), repeats=1)
    doc = json.loads(cache.read_text())
    assert doc["format"] == "caelix-batch-tuning/1" and len(doc["entries"]) == 1
    e = doc["entries"][0]
    assert {k: e[k] for k in t.as_dict()} == t.as_dict()
    # A new batch of the same workload takes the entry.
    batch2 = caelix_b200.Batch(cuda_device, small_batch["views"][:3])
    t2 = batch2.autotune(str(cache), repeats=1)
    assert t2.as_dict() == t.as_dict()
    for v in small_batch["views"][:3]:
        v[1].fill_(-1.0)
    batch2.run()
    batch2.stats()
    for i, ((_, target, w, h, *_), (ref, _)) in enumerate(zip(small_batch["views"][:3], small_batch["plain"][:3])):
        assert target.cpu().numpy().reshape(h, w, 3).tobytes() == ref.tobytes(), f"view {i}"
    batch.close()
    batch2.close()


def test_scene_reflush_recaptures(cuda_device):
    """A full re-flush moves the scene's tables: the next run captures the graph again and traces
    the new scene."""
    import torch

    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(8, 8, 8), seed=21)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    r = caelix_b200.Renderer(cuda_device, scene)
    out = torch.zeros(48 * 48 * 3, device="cuda")
    batch = caelix_b200.Batch(cuda_device, [(r, out, 48, 48, vs.camera, 3, 1, 1)])
    batch.run()
    assert batch.stats().graph_captures == 1
    vs2 = workloads.noise_world(grid_bricks=(8, 8, 8), seed=22)
    scene.upload_bricks(vs2.keys, vs2.voxels)
    scene.flush()
    batch.run()
    assert batch.stats().graph_captures == 2
    ref = torch.zeros_like(out)
    r.render(ref, 48, 48, vs.camera, bounces=3, seed=1, spp=1)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    batch.close()
    r.close()
    scene.close()


def test_batch_after_entity_removed(cuda_device):
    """A scene whose only entity was added, flushed and removed again has no entity the trace sees:
    it is batched, and its view equals the plain render."""
    import torch

    import caelix_b200

    vs = workloads.noise_world(grid_bricks=(8, 8, 8), seed=23)
    scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
    ent = workloads.noise_world(grid_bricks=(2, 2, 2), brick_occupancy=1.0, voxel_fill=0.5, seed=24)
    e = scene.add_entity((20.0, 20.0, 20.0))
    scene.upload_bricks(ent.keys, ent.voxels, entity=e)
    scene.flush()
    scene.remove_entity(e)
    scene.flush()
    r = caelix_b200.Renderer(cuda_device, scene)
    out = torch.zeros(40 * 40 * 3, device="cuda")
    batch = caelix_b200.Batch(cuda_device, [(r, out, 40, 40, vs.camera, 3, 1, 1)])
    batch.run()
    batch.stats()
    ref = torch.zeros_like(out)
    r.render(ref, 40, 40, vs.camera, bounces=3, seed=1, spp=1)
    torch.cuda.synchronize()
    assert torch.equal(out, ref)
    batch.close()
    r.close()
    scene.close()


def test_full_batch_plan_views_match_the_oracle(cuda_device, oracle):
    """The real 64-scene plan of the batched workload (brick counts log-uniform in [1k, 500k],
    viewports among 256/512/1024, 2 spp, 4 bounces) in one batch run: a pixel window of six views
    (the three smallest scenes: the oracle's own build; the three largest: the oracle's trace over
    their flushed tables) equals the oracle within 1e-5 relative; every view's ray counts equal
    its plain render's."""
    import torch

    import caelix_b200
    from test_trace_gpu import assert_radiance_close

    plan = workloads.batch_plan(64)
    order = sorted(range(len(plan)), key=lambda i: plan[i][0])
    checked = order[:3] + order[-3:]
    scenes, renderers, views, worlds = [], [], [], {}
    for i, (count, side) in enumerate(plan):
        vs = workloads.batch_scene(count, seed=100 + i)
        scene = caelix_b200.Scene.from_voxel_scene(cuda_device, vs)
        renderer = caelix_b200.Renderer(cuda_device, scene)
        out = torch.zeros(side * side * 3, dtype=torch.float32, device="cuda")
        views.append((renderer, out, side, side, vs.camera, 4, 1 + i, 2))
        scenes.append(scene)
        renderers.append(renderer)
        if i in checked:
            worlds[i] = vs
        del vs
    batch = caelix_b200.Batch(cuda_device, views, rebuild_light_trees=True)
    batch.set_tuning(min_blocks=8, block_width=8, refill_min=4, order=1, sort_keys_per_thread=16, kernel=1,
                     wavefront=1 << 22)
    batch.run()
    batch.stats()
    for i in checked:
        renderer, out, w, h, cam, bounces, seed, spp = views[i]
        got = out.cpu().numpy().reshape(h, w, 3)
        vs = worlds[i]
        small = i in order[:3]
        osc = oracle_lib.OracleScene(oracle, vs) if small else oracle_lib.TablesScene(oracle, vs, scenes[i].view())
        x0, y0 = w // 2 - 16, h // 2 - 16
        ref, _ = osc.render(w, h, spp=spp, bounces=bounces, seed=seed, window=(x0, y0, x0 + 32, y0 + 32), threads=16)
        assert_radiance_close(got[y0:y0 + 32, x0:x0 + 32], ref[y0:y0 + 32, x0:x0 + 32])
        assert float(ref[y0:y0 + 32, x0:x0 + 32].max()) > 0.0, i
        st = batch.view_stats(i)
        plain = torch.zeros_like(out)
        renderer.render(plain, w, h, cam, bounces=bounces, seed=seed, spp=spp)
        ps = renderer.stats()
        assert (st.primary_rays, st.bounce_rays, st.shadow_rays) == (ps.primary_rays, ps.bounce_rays, ps.shadow_rays)
        assert torch.equal(plain, out)
        osc.close()
    batch.close()
    for r in renderers:
        r.close()
    for s in scenes:
        s.close()
