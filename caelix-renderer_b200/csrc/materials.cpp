// The host side of a scene's material table (materials.h).
#include "materials.h"

#include <cmath>
#include <cstring>

namespace cx {

namespace {

constexpr uint32_t kCodes = 65536;
constexpr float kHalfMax = 65504.0f;  // the reference stores halves on the GPU and checks this range

// An integer hash (Chris Wellons' "lowbias32" constants), the pastel colours of block-ID codes.
uint32_t hash32(uint32_t v)
{
    v ^= v >> 16;
    v *= 0x7FEB352Du;
    v ^= v >> 15;
    v *= 0x846CA68Bu;
    v ^= v >> 16;
    return v;
}

void pastel(uint32_t h, float rgb[3])
{
    for (int c = 0; c < 3; ++c) rgb[c] = 0.35f + 0.6f * ((float)((h >> (8 * c)) & 0xFFu) / 255.0f);
}

CaelixMaterial opaque(float r, float g, float b)
{
    CaelixMaterial m;
    std::memset(&m, 0, sizeof(m));
    m.albedo[0] = r;
    m.albedo[1] = g;
    m.albedo[2] = b;
    m.ior = 1.5f;
    return m;
}

bool finite_within(const float* v, int n)
{
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(v[i]) || std::fabs(v[i]) > kHalfMax) return false;
    return true;
}

bool in_range(const float* v, int n, float lo, float hi)
{
    for (int i = 0; i < n; ++i)
        if (!(v[i] >= lo && v[i] <= hi)) return false;
    return true;
}

}  // namespace

uint32_t canonical_code(uint32_t code, uint32_t encoding)
{
    code &= 0xFFFFu;
    const uint32_t opaque_mask = encoding == 0 ? 0xC000u : 0x8000u;
    const uint32_t id_mask = encoding == 0 ? 0xFFu : 0x1FFu;
    return (code & opaque_mask) ? code : (code & id_mask);
}

CaelixMaterial builtin_material(uint32_t code, uint32_t encoding)
{
    code &= 0xFFFFu;
    if (encoding == 0) {
        if ((code & 0xC000u) == 0) {
            // Transparent: the palette's air entry (albedo 1, smoothness 1, ior 1); glass tints are
            // not carried.
            CaelixMaterial m;
            std::memset(&m, 0, sizeof(m));
            m.albedo[0] = m.albedo[1] = m.albedo[2] = 1.0f;
            m.smoothness = 1.0f;
            m.ior = 1.0f;
            return m;
        }
        if (code & 0x8000u)
            return opaque((float)((code >> 10) & 31u) / 31.0f, (float)((code >> 5) & 31u) / 31.0f,
                          (float)(code & 31u) / 31.0f);
        CaelixMaterial m = opaque((float)((code >> 10) & 15u) / 15.0f, (float)((code >> 6) & 15u) / 15.0f,
                                  (float)((code >> 2) & 15u) / 15.0f);
        const float strength = std::exp2(3.0f * (float)(code & 3u));
        for (int c = 0; c < 3; ++c) m.emission[c] = m.albedo[c] * strength;
        return m;
    }
    float rgb[3];
    if (code & 0x8000u) {
        pastel(hash32(code & 0x7FFFu), rgb);
        return opaque(rgb[0], rgb[1], rgb[2]);
    }
    const uint32_t id = code & 0x1FFu;
    if (id == 0) return builtin_material(0, 0);  // air: the vacuum entry
    pastel(hash32(id | 0x10000u), rgb);
    return opaque(rgb[0], rgb[1], rgb[2]);
}

bool material_valid(const CaelixMaterial& m, const char** reason)
{
    if (!finite_within(m.albedo, 3) || !finite_within(&m.smoothness, 1) || !finite_within(m.emission, 3) ||
        !finite_within(&m.metallic, 1) || !finite_within(&m.ior, 1) || !finite_within(&m.extinction, 1) ||
        !finite_within(&m.sss_probability, 1) || !finite_within(m.sss_albedo, 3) ||
        !finite_within(&m.sss_anisotropy, 1) || !finite_within(m.sss_params, 8)) {
        *reason = "a value is not finite or its magnitude is above 65504";
        return false;
    }
    if (!(m.ior > 0.0f)) {
        *reason = "ior must be > 0";
        return false;
    }
    if (!(m.extinction >= 0.0f)) {
        *reason = "extinction must be >= 0";
        return false;
    }
    if (m.sss_model > 255u || m.sss_steps > 255u) {
        *reason = "sss_model and sss_steps must be <= 255";
        return false;
    }
    if (!in_range(&m.sss_probability, 1, 0.0f, 1.0f) || !in_range(m.sss_albedo, 3, 0.0f, 1.0f)) {
        *reason = "sss_probability and sss_albedo must be in [0, 1]";
        return false;
    }
    if (!in_range(&m.sss_anisotropy, 1, -1.0f, 1.0f)) {
        *reason = "sss_anisotropy must be in [-1, 1]";
        return false;
    }
    if (m.texture_set > 0xFFFFu || m.connect_group > 0xFFFFu) {
        *reason = "texture_set and connect_group must be <= 0xFFFF";
        return false;
    }
    return true;
}

void pack_materials(const std::vector<CaelixMaterial>& table, uint32_t encoding, std::vector<float>& out)
{
    out.assign(8ull * kCodes, 0.0f);
    for (uint32_t c = 0; c < kCodes; ++c) {
        const CaelixMaterial& m = table[canonical_code(c, encoding)];
        float* o = out.data() + 8ull * c;
        for (int k = 0; k < 3; ++k) {
            o[k] = m.albedo[k];
            o[4 + k] = m.emission[k];
        }
    }
}

void light_code_set(const std::vector<CaelixMaterial>& table, uint32_t encoding, float min_emission,
                    std::vector<uint32_t>& out)
{
    out.assign(kCodes / 32, 0u);
    for (uint32_t c = 0; c < kCodes; ++c) {
        const float* e = table[canonical_code(c, encoding)].emission;
        const float lum = 0.2126f * e[0] + 0.7152f * e[1] + 0.0722f * e[2];
        if (lum >= min_emission) out[c >> 5] |= 1u << (c & 31);
    }
}

}  // namespace cx
