"""Structural checks of a built light BVH, restating the reference's CheckBvh
(tests/light_tree_test.cpp:505-639): every leaf reached exactly once from the root, parent links
of leaves and nodes, leaf slot summaries byte-equal to the leaves, node slot face sums within
1e-5 relative / 1e-4 absolute of the child's slot sums, boxes that contain the children's, the
header summary."""
import numpy as np

NONE = 0xFFFFFFFF
LEAF_BIT = 0x80000000


def near(a, b, rel=1e-5, abs_=1e-4):
    return abs(a - b) <= max(abs_, rel * max(abs(a), abs(b)))


def check_bvh(header, leaves, nodes):
    leaf_count = int(header["leaf_count"])
    if leaf_count == 0:
        assert int(header["root"]) == NONE
        return
    assert int(header["root"]) == 0
    node_count = int(header["node_count"])
    assert node_count >= 1
    assert int(nodes[0]["parent"]) == NONE
    leaf_seen = np.zeros(leaf_count, np.int32)
    node_seen = np.zeros(node_count, np.int32)

    def node_sum(n):
        face = np.zeros(6, np.float64)
        lo = np.full(3, np.inf, np.float32)
        hi = np.full(3, -np.inf, np.float32)
        for s in range(4):
            if int(nodes[n]["child"][s]) == NONE:
                continue
            f = nodes[n]["child_face"][s].astype(np.float64)
            face += f
            if f.sum() > 0:
                lo = np.minimum(lo, nodes[n]["child_lo"][s])
                hi = np.maximum(hi, nodes[n]["child_hi"][s])
        return face, lo, hi

    stack = [0]
    while stack:
        n = stack.pop()
        assert n < node_count
        assert node_seen[n] == 0
        node_seen[n] = 1
        used = 0
        for s in range(4):
            child = int(nodes[n]["child"][s])
            if child == NONE:
                continue
            used += 1
            if child & LEAF_BIT:
                leaf = child & ~LEAF_BIT
                assert leaf < leaf_count
                assert leaf_seen[leaf] == 0
                leaf_seen[leaf] = 1
                assert int(leaves[leaf]["parent"]) == (n << 2) | s
                assert nodes[n]["child_face"][s].tobytes() == leaves[leaf]["face"].tobytes()
                assert nodes[n]["child_lo"][s].tobytes() == leaves[leaf]["lo"].tobytes()
                assert nodes[n]["child_hi"][s].tobytes() == leaves[leaf]["hi"].tobytes()
            else:
                assert child < node_count
                assert int(nodes[child]["parent"]) == n
                assert int(nodes[child]["parent_slot"]) == s
                face, lo, hi = node_sum(child)
                for f in range(6):
                    assert near(float(nodes[n]["child_face"][s][f]), face[f])
                if face.sum() > 0:
                    assert np.all(nodes[n]["child_lo"][s] <= lo)
                    assert np.all(nodes[n]["child_hi"][s] >= hi)
                stack.append(child)
        assert used >= (1 if leaf_count == 1 else 2)
    assert np.all(leaf_seen == 1)
    assert np.all(node_seen == 1)
    face, lo, hi = node_sum(0)
    for f in range(6):
        assert near(float(header["face"][f]), face[f])
    assert np.all(header["lo"] <= lo)
    assert np.all(header["hi"] >= hi)
