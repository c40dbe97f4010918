// Prints the byte layout of the reference's light tree structs (lib/src/light/light_tree_layout.h,
// compiled from the reference source tree by oracle/ref_layout.mk) as JSON: the pin of the
// layouts that libcaelix_b200 and the oracle restate.
#include <cstddef>
#include <cstdio>

#include "light/light_tree_layout.h"

#define F(S, m) std::printf("  \"%s.%s\": %zu,\n", #S, #m, offsetof(caelix::S, m))
#define Z(S) std::printf("  \"%s.sizeof\": %zu,\n", #S, sizeof(caelix::S))

int main()
{
    std::printf("{\n");
    F(LightSummary, face); F(LightSummary, lo); F(LightSummary, hi); Z(LightSummary);
    F(LightTreeHeader, summary); F(LightTreeHeader, root); F(LightTreeHeader, leaf_count);
    F(LightTreeHeader, node_count); Z(LightTreeHeader);
    F(LightTreeState, building); F(LightTreeState, leaves_found); F(LightTreeState, leaves_dropped);
    F(LightTreeState, builds); F(LightTreeState, node_overflow); F(LightTreeState, bounds); Z(LightTreeState);
    F(BrickLightRecordHeader, face); F(BrickLightRecordHeader, box_lo); F(BrickLightRecordHeader, box_hi);
    F(BrickLightRecordHeader, pos); F(BrickLightRecordHeader, entry_count); F(BrickLightRecordHeader, counts_lo);
    F(BrickLightRecordHeader, counts_hi); Z(BrickLightRecordHeader);
    F(LightBvhLeaf, summary); F(LightBvhLeaf, group); F(LightBvhLeaf, entry); F(LightBvhLeaf, parent);
    Z(LightBvhLeaf);
    F(LightBvhNode, child_face); F(LightBvhNode, child_lo); F(LightBvhNode, child_hi); F(LightBvhNode, child);
    F(LightBvhNode, parent); F(LightBvhNode, parent_slot); Z(LightBvhNode);
    std::printf("  \"kLtChildLeafBit\": %u,\n", caelix::kLtChildLeafBit);
    std::printf("  \"kLtNone\": %u,\n", caelix::kLtNone);
    std::printf("  \"kLtParentSlotBits\": %u,\n", caelix::kLtParentSlotBits);
    std::printf("  \"kLtVoxelBits\": %u,\n", caelix::kLtVoxelBits);
    std::printf("  \"kLtFamilyCountBits\": %u\n", caelix::kLtFamilyCountBits);
    std::printf("}\n");
    return 0;
}
