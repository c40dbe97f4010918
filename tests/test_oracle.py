"""The oracle (the checker) against the reference's own known answers: the radix sort golden
vectors of tests/light_tree_test.cpp:1460-1515 (std::mt19937(3), std::sort), the reference's
BVH invariants (CheckBvh), and the Morton code definition (caelix_light_tree_layout.hlsl:247-261)."""
import hashlib
import os

import numpy as np
import pytest

import bvh_checks
import oracle_lib
from caelix_b200 import workloads

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = np.load(os.path.join(REPO, "tests", "golden", "sort_mt19937_3.npz"))


@pytest.mark.parametrize("n", [1, 2, 1000, 100000])
def test_oracle_sort_matches_reference_golden(oracle, n):
    keys = GOLDEN[f"n{n}_keys"].copy()
    values = np.arange(n, dtype=np.uint32)
    oracle.oc_radix_sort_pairs(keys.ctypes.data, values.ctypes.data, n)
    digest = hashlib.sha256(keys.tobytes() + values.tobytes()).digest()
    assert digest == GOLDEN[f"n{n}_sha256"].tobytes()
    if n <= 1000:
        assert np.array_equal(keys, GOLDEN[f"n{n}_sorted_keys"])
        assert np.array_equal(values, GOLDEN[f"n{n}_sorted_values"])


def morton_numpy(x, y, z):
    out = np.zeros_like(x, dtype=np.uint64)
    for b in range(10):
        out |= ((x.astype(np.uint64) >> b) & 1) << (3 * b)
        out |= ((y.astype(np.uint64) >> b) & 1) << (3 * b + 1)
        out |= ((z.astype(np.uint64) >> b) & 1) << (3 * b + 2)
    return out.astype(np.uint32)


def test_oracle_morton_is_bit_interleave(oracle):
    rng = np.random.default_rng(5)
    c = rng.integers(0, 1024, size=(2000, 3))
    ours = np.array([oracle.oc_morton(int(a), int(b), int(d)) for a, b, d in c], np.uint32)
    assert np.array_equal(ours, morton_numpy(c[:, 0], c[:, 1], c[:, 2]))
    assert oracle.oc_morton(1023, 1023, 1023) == 0x3FFFFFFF


def test_oracle_build_config1_structure(oracle):
    rec, _, _ = workloads.brick_light_records(4096)
    o = oracle_lib.lt_build(oracle, rec)
    assert o["status"] == 0
    h = o["header"][0]
    assert h["leaf_count"] == 4096
    assert o["node_overflow"][0] == 0
    bvh_checks.check_bvh(h, o["leaves"][:4096], o["nodes"][: h["node_count"]])
    # The sort is a stable sort by Morton key of the identity values.
    order = np.argsort(o["keys"][:4096], kind="stable")
    assert np.array_equal(order, np.arange(4096))
    # Total power equals the record sum within float rounding.
    total = float(rec["face"].astype(np.float64).sum())
    assert abs(float(h["face"].astype(np.float64).sum()) - total) <= 1e-4 * total


@pytest.mark.parametrize("n", [0, 1, 2, 3, 5, 17, 64, 1000])
def test_oracle_build_small_structure(oracle, n):
    rec, _, _ = workloads.brick_light_records(n, seed=7, stream=n + 1) if n else (np.zeros(0, workloads.RECORD_DTYPE), 0, 0)
    o = oracle_lib.lt_build(oracle, rec, leaf_capacity=max(n, 1))
    h = o["header"][0]
    assert h["leaf_count"] == n
    bvh_checks.check_bvh(h, o["leaves"][:n], o["nodes"][: h["node_count"]])


def test_oracle_build_duplicate_keys(oracle):
    # Every record in the same brick: all Morton codes equal, ties by sorted position.
    rec, _, _ = workloads.brick_light_records(300, grid_bricks=1)
    o = oracle_lib.lt_build(oracle, rec)
    assert len(set(o["keys"][:300].tolist())) == 1
    h = o["header"][0]
    bvh_checks.check_bvh(h, o["leaves"][:300], o["nodes"][: h["node_count"]])


def test_oracle_build_grouped_frames(oracle):
    rec, group, frames = workloads.brick_light_records(20000, grid_bricks=256, group_shift=4)
    o = oracle_lib.lt_build(oracle, rec, record_group=group, group_frames=frames)
    h = o["header"][0]
    bvh_checks.check_bvh(h, o["leaves"][:20000], o["nodes"][: h["node_count"]])
    # Leaves are the world-space brick boxes.
    lo = o["leaves"]["lo"][:20000]
    assert np.all(lo >= 0) and np.all(o["leaves"]["hi"][:20000] <= 256 * 8)


def test_batch_plan_distribution():
    """The batched workload's plan: brick counts within [1k, 500k], log-uniform (the median near
    the geometric mean), square viewports among 256, 512, 1024, deterministic."""
    import numpy as np

    from caelix_b200 import workloads

    plan = workloads.batch_plan()
    assert len(plan) == 64 and plan == workloads.batch_plan()
    bricks = np.array([b for b, _ in plan], np.float64)
    assert bricks.min() >= 1000 and bricks.max() <= 500_000
    assert 0.25 < np.median(bricks) / np.sqrt(1000 * 500_000) < 4
    assert {s for _, s in plan} <= set(workloads.BATCH_VIEWPORTS)
    assert len({s for _, s in plan}) == 3


def test_solid_brick_scene_and_target():
    """The differentiation world: the first draw of a repeated coordinate kept, bricks in
    increasing linear index, every brick solid and emissive; the target perturbs albedo and power
    by at most 10 %."""
    import numpy as np

    from caelix_b200 import workloads

    vs = workloads.solid_brick_scene(n=600, grid_bricks=16, seed=3)
    lin = vs.keys[:, 0] + 16 * (vs.keys[:, 1] + 16 * vs.keys[:, 2])
    assert np.all(np.diff(lin) > 0)
    rng = workloads.Pcg32(3, 1)
    coords = (rng.next_u32(3 * 600).reshape(600, 3) >> np.uint32(28)).astype(np.int64)
    power = rng.lognormal(600)
    first = {}
    for i, c in enumerate(map(tuple, coords)):
        first.setdefault(c, i)
    assert len(first) == vs.brick_count
    for k, p in zip(map(tuple, vs.keys), vs.power):
        assert np.float32(power[first[k]]) == p
    assert np.all(vs.voxels & 0x8000) and np.all(vs.power > 0)
    t = workloads.perturbed(vs)
    ra = t.albedo[1:65] / vs.albedo[1:65]
    rp = t.power / vs.power
    assert np.all(np.abs(ra - 1) <= 0.1 + 1e-6) and np.all(np.abs(rp - 1) <= 0.1 + 1e-6)
    assert np.array_equal(t.keys, vs.keys) and np.array_equal(t.voxels, vs.voxels)
