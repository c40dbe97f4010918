"""Parity of the CUDA light BVH build (through the C ABI) with the oracle: bit-exact Morton codes,
sorted permutation, Karras topology, aggregates, depths, 4-wide nodes, leaves and header; the
radix sort against the reference's golden vectors; determinism; capacity and edge cases."""
import hashlib
import os

import numpy as np
import pytest

import bvh_checks
import gpu_util
import oracle_lib
from caelix_b200 import workloads

pytestmark = pytest.mark.gpu

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = np.load(os.path.join(REPO, "tests", "golden", "sort_mt19937_3.npz"))
AGG_SLOT_DTYPE = np.dtype([("s", oracle_lib.SUMMARY_DTYPE), ("pad", "<u4", (4,))])


def gpu_build(dev, rec, group=None, frames=None, capacity=None):
    import caelix_b200

    n = len(rec)
    bvh = caelix_b200.LightBvh(dev, capacity or max(n, 1))
    d_rec = gpu_util.to_device(rec)
    d_group = gpu_util.to_device(group) if group is not None else None
    d_frames = gpu_util.to_device(frames) if frames is not None else None
    bvh.build(d_rec, n, record_group=d_group, group_frames=d_frames,
              group_count=len(frames) if frames is not None else None)
    stats = bvh.stats()
    v = bvh.view()
    m = min(n, v.leaf_capacity)
    out = {
        "stats": stats,
        "header": gpu_util.from_device(v.header, oracle_lib.HEADER_DTYPE, 1),
        "leaves": gpu_util.from_device(v.leaves, oracle_lib.LEAF_DTYPE, m),
        "keys": gpu_util.from_device(v.keys, np.uint32, m),
        "values": gpu_util.from_device(v.values, np.uint32, m),
        "left": gpu_util.from_device(v.left, np.uint32, max(m - 1, 0)),
        "right": gpu_util.from_device(v.right, np.uint32, max(m - 1, 0)),
        "parent": gpu_util.from_device(v.parent, np.uint32, max(m - 1, 0)),
        "leaf_parent": gpu_util.from_device(v.leaf_parent, np.uint32, m if m >= 2 else 0),
        "depth": gpu_util.from_device(v.depth, np.uint32, max(m - 1, 0)),
        "wide": gpu_util.from_device(v.wide, np.uint32, max(m - 1, 0)),
        "aggregates": gpu_util.from_device(v.aggregates, AGG_SLOT_DTYPE, max(m - 1, 0))["s"].copy(),
    }
    nc = int(out["header"][0]["node_count"])
    out["nodes"] = gpu_util.from_device(v.nodes, oracle_lib.NODE_DTYPE, nc)
    bvh.close()
    return out


def node_bytes(nodes):
    # Every field but the two pad words.
    return nodes.view(np.uint8).reshape(len(nodes), 224)[:, :216].tobytes()


def assert_same_build(g, o, n):
    m = min(n, len(g["leaves"]))
    assert g["header"].tobytes() == o["header"].tobytes()
    assert g["keys"].tobytes() == o["keys"][:m].tobytes()
    assert g["values"].tobytes() == o["values"][:m].tobytes()
    assert g["leaves"].tobytes() == o["leaves"][:m].tobytes()
    if m >= 2:
        for k in ("left", "right", "parent", "depth"):
            assert g[k].tobytes() == o[k][: m - 1].tobytes(), k
        assert g["leaf_parent"].tobytes() == o["leaf_parent"][:m].tobytes()
        even = (o["depth"][: m - 1] & 1) == 0
        assert np.array_equal(g["wide"][even], o["wide"][: m - 1][even])
        assert g["aggregates"].tobytes() == o["aggregates"][: m - 1].tobytes()
    nc = int(o["header"][0]["node_count"])
    assert node_bytes(g["nodes"]) == node_bytes(o["nodes"][:nc])


@pytest.mark.parametrize("n", [1, 2, 1000, 100000])
def test_radix_sort_matches_reference_golden(cuda_device, n):
    import torch

    keys = torch.from_numpy(GOLDEN[f"n{n}_keys"].astype(np.int32)).cuda()
    values = torch.zeros(n, dtype=torch.int32, device="cuda")
    cuda_device.radix_sort_pairs(keys, values, n, identity_values=True)
    assert cuda_device.check_status() == 0
    k = keys.cpu().numpy().view(np.uint32)
    v = values.cpu().numpy().view(np.uint32)
    assert hashlib.sha256(k.tobytes() + v.tobytes()).digest() == GOLDEN[f"n{n}_sha256"].tobytes()


@pytest.mark.parametrize("n", [3, 511, 512, 513, 4095, 4096, 4097, 200000, 1 << 22])
def test_radix_sort_random_is_stable_sort(cuda_device, n):
    import torch

    rng = np.random.default_rng(n)
    keys_np = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    keys_np[::7] = keys_np[0]  # duplicates
    vals_np = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    keys = torch.from_numpy(keys_np.view(np.int32)).cuda()
    values = torch.from_numpy(vals_np.view(np.int32)).cuda()
    cuda_device.radix_sort_pairs(keys, values, n)
    assert cuda_device.check_status() == 0
    order = np.argsort(keys_np, kind="stable")
    assert np.array_equal(keys.cpu().numpy().view(np.uint32), keys_np[order])
    assert np.array_equal(values.cpu().numpy().view(np.uint32), vals_np[order])


def test_build_config1_bit_exact(cuda_device, oracle):
    rec, _, _ = workloads.brick_light_records(4096)
    g = gpu_build(cuda_device, rec)
    o = oracle_lib.lt_build(oracle, rec)
    assert g["stats"].status == 0
    assert_same_build(g, o, 4096)
    bvh_checks.check_bvh(g["header"][0], g["leaves"], g["nodes"])


@pytest.mark.parametrize("n", [0, 1, 2, 3, 5, 17, 64, 1000, 4097, 100003])
def test_build_sizes_bit_exact(cuda_device, oracle, n):
    if n:
        rec, _, _ = workloads.brick_light_records(n, seed=11, stream=n)
    else:
        rec = np.zeros(0, workloads.RECORD_DTYPE)
    g = gpu_build(cuda_device, rec)
    o = oracle_lib.lt_build(oracle, rec, leaf_capacity=max(n, 1))
    assert_same_build(g, o, n)


def test_build_duplicate_keys_bit_exact(cuda_device, oracle):
    rec, _, _ = workloads.brick_light_records(5000, grid_bricks=2)
    g = gpu_build(cuda_device, rec)
    o = oracle_lib.lt_build(oracle, rec)
    assert_same_build(g, o, 5000)


def test_build_rotated_frames_bit_exact(cuda_device, oracle):
    rec, group, frames = workloads.brick_light_records(30000, grid_bricks=128, group_shift=3)
    rng = np.random.default_rng(3)
    for i in range(len(frames)):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        x, y, z, w = q
        rot = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]], np.float32)
        frames[i]["rotation"] = rot.reshape(9)
        frames[i]["translation"] = rng.uniform(-100, 100, 3).astype(np.float32)
    g = gpu_build(cuda_device, rec, group, frames)
    o = oracle_lib.lt_build(oracle, rec, record_group=group, group_frames=frames)
    assert_same_build(g, o, len(rec))


def test_build_large_grouped_bit_exact(cuda_device, oracle):
    n = 1 << 21
    rec, group, frames = workloads.brick_light_records(n, grid_bricks=1024, group_shift=4)
    g = gpu_build(cuda_device, rec, group, frames)
    o = oracle_lib.lt_build(oracle, rec, record_group=group, group_frames=frames)
    assert g["stats"].status == 0
    assert_same_build(g, o, n)


def test_build_capacity_drops_rest(cuda_device, oracle):
    rec, _, _ = workloads.brick_light_records(3000, seed=4, stream=2)
    g = gpu_build(cuda_device, rec, capacity=2048)
    assert g["stats"].leaves_found == 3000
    assert g["stats"].leaves_dropped == 952
    o = oracle_lib.lt_build(oracle, rec, leaf_capacity=2048)
    assert_same_build(g, o, 2048)


def test_build_is_deterministic(cuda_device):
    rec, group, frames = workloads.brick_light_records(200000, grid_bricks=512, group_shift=4)
    a = gpu_build(cuda_device, rec, group, frames)
    b = gpu_build(cuda_device, rec, group, frames)
    for k in ("keys", "values", "left", "right", "aggregates", "leaves"):
        assert a[k].tobytes() == b[k].tobytes(), k
    assert node_bytes(a["nodes"]) == node_bytes(b["nodes"])
