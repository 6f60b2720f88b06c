// Stand-in for the reference's missing `ks/geometry.h`: the MeshData buffers
// that the reference's tessellation sources fill (flat float positions,
// texture coordinates and vertex normals, uint32 indices), written from
// scratch so that displaced_tessellation.cpp compiles unmodified for the
// oracle build (oracle/Makefile).
#pragma once
#include "maths.h"

#include <cstdint>
#include <vector>

namespace ks
{

struct MeshData
{
    std::vector<float> vertices;       // xyz per vertex (+1 padding float once finalized)
    std::vector<float> texcoords;      // uv per vertex (+2)
    std::vector<float> vertex_normals; // xyz per vertex (+1)
    std::vector<uint32_t> indices;     // 3 per triangle

    int tri_count() const { return (int)(indices.size() / 3); }
    vec3 get_pos(uint32_t k) const { return vec3(vertices[3 * k], vertices[3 * k + 1], vertices[3 * k + 2]); }
};

} // namespace ks
