// Geometry types of the public C++ API (same conventions as the reference's
// cpp/include/pdmk/types.hpp:1-40): Mat3 m[j][i] = component i of lattice vector j.
#pragma once
#include <array>

namespace pdmk {

using Vec3 = std::array<double, 3>;
using Mat3 = std::array<std::array<double, 3>, 3>;

template <int DIM>
struct dim_types;
template <>
struct dim_types<3> {
    using Vec = Vec3;
    using Mat = Mat3;
};
template <int DIM>
using VecND = typename dim_types<DIM>::Vec;
template <int DIM>
using MatND = typename dim_types<DIM>::Mat;

}  // namespace pdmk
