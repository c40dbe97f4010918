"""The byte layouts of the light tree structs: the product header (caelix-renderer_b200/csrc/
cx_layout.h), the oracle (tests/oracle_lib.py dtypes) and the C ABI mirror all equal the reference's
lib/src/light/light_tree_layout.h, pinned by tests/golden/ref_layout.json (written by
oracle/ref_layout.mk from the reference header itself)."""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle_lib

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = json.load(open(os.path.join(REPO, "tests", "golden", "ref_layout.json")))

PROBE = r"""
#include <cstddef>
#include <cstdio>
#include "cx_layout.h"
#define F(R, S, m) std::printf("\"%s.%s\": %zu,\n", #R, #m, offsetof(cx::S, m))
#define Z(R, S) std::printf("\"%s.sizeof\": %zu,\n", #R, sizeof(cx::S))
int main() {
  std::printf("{\n");
  F(LightSummary, LightSummary, face); F(LightSummary, LightSummary, lo); F(LightSummary, LightSummary, hi);
  Z(LightSummary, LightSummary);
  F(LightTreeHeader, LightTreeHeader, summary); F(LightTreeHeader, LightTreeHeader, root);
  F(LightTreeHeader, LightTreeHeader, leaf_count); F(LightTreeHeader, LightTreeHeader, node_count);
  Z(LightTreeHeader, LightTreeHeader);
  F(BrickLightRecordHeader, BrickLightRecord, face); F(BrickLightRecordHeader, BrickLightRecord, box_lo);
  F(BrickLightRecordHeader, BrickLightRecord, box_hi); F(BrickLightRecordHeader, BrickLightRecord, pos);
  F(BrickLightRecordHeader, BrickLightRecord, entry_count); F(BrickLightRecordHeader, BrickLightRecord, counts_lo);
  F(BrickLightRecordHeader, BrickLightRecord, counts_hi); Z(BrickLightRecordHeader, BrickLightRecord);
  F(LightBvhLeaf, LightBvhLeaf, summary); F(LightBvhLeaf, LightBvhLeaf, group); F(LightBvhLeaf, LightBvhLeaf, entry);
  F(LightBvhLeaf, LightBvhLeaf, parent); Z(LightBvhLeaf, LightBvhLeaf);
  F(LightBvhNode, LightBvhNode, child_face); F(LightBvhNode, LightBvhNode, child_lo);
  F(LightBvhNode, LightBvhNode, child_hi); F(LightBvhNode, LightBvhNode, child); F(LightBvhNode, LightBvhNode, parent);
  F(LightBvhNode, LightBvhNode, parent_slot); Z(LightBvhNode, LightBvhNode);
  std::printf("\"kLtChildLeafBit\": %u,\n\"kLtNone\": %u,\n\"kLtParentSlotBits\": %u,\n\"kLtVoxelBits\": %u,\n"
              "\"kLtFamilyCountBits\": %u\n}\n", cx::kChildLeafBit, cx::kNone, cx::kParentSlotBits, cx::kVoxelBits,
              cx::kFamilyCountBits);
}
"""


@pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")
def test_product_layout_matches_reference(tmp_path):
    src = tmp_path / "probe.cpp"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(REPO, "caelix-renderer_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)
    ours = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    for key, value in ours.items():
        assert GOLDEN[key] == value, key
    # Every reference entry except LightTreeState (the product keeps its own state struct) is covered.
    missing = [k for k in GOLDEN if k not in ours and not k.startswith("LightTreeState")]
    assert not missing


def test_oracle_layout_matches_reference():
    leaf = oracle_lib.LEAF_DTYPE
    node = oracle_lib.NODE_DTYPE
    hdr = oracle_lib.HEADER_DTYPE
    assert leaf.fields["group"][1] == GOLDEN["LightBvhLeaf.group"]
    assert leaf.fields["entry"][1] == GOLDEN["LightBvhLeaf.entry"]
    assert leaf.fields["parent"][1] == GOLDEN["LightBvhLeaf.parent"]
    assert leaf.itemsize == GOLDEN["LightBvhLeaf.sizeof"]
    for f in ("child_face", "child_lo", "child_hi", "child", "parent", "parent_slot"):
        assert node.fields[f][1] == GOLDEN[f"LightBvhNode.{f}"], f
    assert node.itemsize == GOLDEN["LightBvhNode.sizeof"]
    assert hdr.fields["root"][1] == GOLDEN["LightTreeHeader.root"]
    assert hdr.fields["node_count"][1] == GOLDEN["LightTreeHeader.node_count"]
    assert hdr.itemsize == GOLDEN["LightTreeHeader.sizeof"]


def test_workload_record_dtype_matches_reference():
    from caelix_b200 import workloads

    d = workloads.RECORD_DTYPE
    for f in ("face", "box_lo", "box_hi", "pos", "entry_count", "counts_lo", "counts_hi"):
        assert d.fields[f][1] == GOLDEN[f"BrickLightRecordHeader.{f}"], f
    assert d.itemsize == GOLDEN["BrickLightRecordHeader.sizeof"]
