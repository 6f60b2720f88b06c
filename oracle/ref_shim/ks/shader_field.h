// Stand-in for the reference's missing `ks/shader_field.h`: the declarations
// emission_tile.cpp's emission_from_field needs to compile. The oracle build
// never calls that function (it builds emission tiles from texel grids).
#pragma once
#include "maths.h"

namespace ks
{
using mat2 = Eigen::Matrix<float, 2, 2>;

template <typename T>
struct ShaderField
{
    virtual ~ShaderField() = default;
    virtual T operator()(const vec2 &uv, const mat2 &duvdxy) const = 0;
};

inline float luminance(const color3 &c) { return (0.2126f * c[0] + 0.7152f * c[1]) + 0.0722f * c[2]; }
} // namespace ks
