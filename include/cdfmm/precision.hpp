// Scalar precision of a plan (upstream include/cdfmm/precision.hpp:10-13).
#pragma once

namespace cdfmm {

enum class StaticPrecision { Float32, Float64 };

} // namespace cdfmm
