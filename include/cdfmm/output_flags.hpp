// Output selection and per-target result records.
//
// Values and layout follow the upstream API (include/cdfmm/output_flags.hpp:
// 12-39 in dip-fmm): Potential = 1, Field = 2, Both = 3; FloatPotentialField is
// {phi, H.x, H.y, H.z} in that order (16 bytes), which the device path writes
// directly when the caller asks for interleaved results.
#pragma once

#include "cdfmm/vec3.hpp"

namespace cdfmm {

enum class OutputFlags : unsigned { None = 0u, Potential = 1u, Field = 2u, Both = 3u };

inline OutputFlags operator|(OutputFlags a, OutputFlags b) {
  return static_cast<OutputFlags>(static_cast<unsigned>(a) | static_cast<unsigned>(b));
}

inline bool has_flag(OutputFlags flags, OutputFlags test) {
  return (static_cast<unsigned>(flags) & static_cast<unsigned>(test)) != 0u;
}

/// FP64 potential and field of one target.
struct PotentialField {
  double phi{0.0};
  Vec3 H{};
};

/// FP32 potential and field of one target.
struct FloatPotentialField {
  float phi{0.0F};
  FloatVec3 H{};
};

} // namespace cdfmm
