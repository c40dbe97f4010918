// The material table of a scene on the host: the built-in entries of the two block encodings, the
// value checks of the setters, the device form and the light code set. Replaces the reference's
// MaterialTable (lib/src/scene/material_table.cpp:71-225) and LightTree::RebuildCodes
// (lib/src/light/light_tree.cpp:186-200) for the fields the path uses.
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/caelix_b200.h"

namespace cx {

// The table index of a raw block code (face bits of a transparent code removed).
uint32_t canonical_code(uint32_t code, uint32_t encoding);

// The built-in entry of a code in an encoding (include/caelix/caelix.h:501-515).
CaelixMaterial builtin_material(uint32_t code, uint32_t encoding);

// The setters' value checks (include/caelix/caelix.h:558-568); false with a reason.
bool material_valid(const CaelixMaterial& m, const char** reason);

// The device table: for every code, two float4 (albedo rgb, 0; emission rgb, 0) of its canonical
// entry; out holds 8 * 65536 floats.
void pack_materials(const std::vector<CaelixMaterial>& table, uint32_t encoding, std::vector<float>& out);

// The light code set: bit c (word c / 32) for every code whose canonical entry's emission
// luminance, 0.2126 r + 0.7152 g + 0.0722 b, is at least min_emission.
void light_code_set(const std::vector<CaelixMaterial>& table, uint32_t encoding, float min_emission,
                    std::vector<uint32_t>& out);

}  // namespace cx
