// Cartesian three-vectors used by the public cdfmm API.
//
// Same member names and value semantics as the upstream public type
// (include/cdfmm/vec3.hpp:7-58 in dip-fmm) so user code that fills positions
// and moments compiles unchanged against this library.
#pragma once

namespace cdfmm {

/// FP64 three-vector (positions, moments and widened results).
struct Vec3 {
  double x{0.0};
  double y{0.0};
  double z{0.0};

  Vec3() = default;
  Vec3(double x_, double y_, double z_) : x(x_), y(y_), z(z_) {}

  double &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  Vec3 operator+(const Vec3 &o) const { return {x + o.x, y + o.y, z + o.z}; }
  Vec3 operator-(const Vec3 &o) const { return {x - o.x, y - o.y, z - o.z}; }
  Vec3 operator*(double s) const { return {x * s, y * s, z * s}; }
  Vec3 &operator+=(const Vec3 &o) {
    x += o.x;
    y += o.y;
    z += o.z;
    return *this;
  }
};

/// FP32 three-vector (results of an FP32 plan).
struct FloatVec3 {
  float x{0.0F};
  float y{0.0F};
  float z{0.0F};

  FloatVec3() = default;
  FloatVec3(float x_, float y_, float z_) : x(x_), y(y_), z(z_) {}

  float &operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  FloatVec3 &operator+=(const FloatVec3 &o) {
    x += o.x;
    y += o.y;
    z += o.z;
    return *this;
  }
};

inline Vec3 operator*(double s, const Vec3 &v) { return v * s; }
inline double dot(const Vec3 &a, const Vec3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

} // namespace cdfmm
