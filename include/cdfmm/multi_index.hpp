// Cartesian multi-indices and the total-degree expansion basis.
//
// The basis order is part of the data contract with upstream dip-fmm
// (include/cdfmm/multi_index.hpp:57-71): degrees ascending; within one degree
// alpha_x ascending, then alpha_y ascending, alpha_z = degree - alpha_x -
// alpha_y.  Coefficient vectors returned by multipole()/local() use it, so it
// must not change.  index() uses the closed-form rank of that order instead
// of a search.
#pragma once

#include <cmath>
#include <stdexcept>
#include <vector>

#include "cdfmm/vec3.hpp"

namespace cdfmm {

struct MultiIndex {
  int ax{0};
  int ay{0};
  int az{0};

  int degree() const { return ax + ay + az; }
  int operator[](int i) const { return i == 0 ? ax : (i == 1 ? ay : az); }
};

inline bool leq(const MultiIndex &a, const MultiIndex &b) {
  return a.ax <= b.ax && a.ay <= b.ay && a.az <= b.az;
}
inline MultiIndex add(const MultiIndex &a, const MultiIndex &b) {
  return {a.ax + b.ax, a.ay + b.ay, a.az + b.az};
}
inline MultiIndex sub(const MultiIndex &a, const MultiIndex &b) {
  return {a.ax - b.ax, a.ay - b.ay, a.az - b.az};
}

/// Number of multi-indices of total degree <= p in three dimensions.
inline int basis_size(int p) { return p < 0 ? 0 : (p + 1) * (p + 2) * (p + 3) / 6; }

/// Position of a multi-index in the total-degree basis (independent of p).
inline int basis_rank(const MultiIndex &a) {
  const int d = a.degree();
  return d * (d + 1) * (d + 2) / 6 + a.ax * (d + 1) - a.ax * (a.ax - 1) / 2 + a.ay;
}

class MultiIndexSet {
public:
  explicit MultiIndexSet(int p) : p_(p) {
    if (p < 0) {
      return;
    }
    indices_.reserve(static_cast<std::size_t>(basis_size(p)));
    for (int d = 0; d <= p; ++d) {
      for (int ax = 0; ax <= d; ++ax) {
        for (int ay = 0; ay + ax <= d; ++ay) {
          indices_.push_back({ax, ay, d - ax - ay});
        }
      }
    }
  }

  int order() const { return p_; }
  int size() const { return static_cast<int>(indices_.size()); }
  const MultiIndex &operator[](int i) const { return indices_.at(static_cast<std::size_t>(i)); }

  int index(const MultiIndex &a) const {
    if (a.ax < 0 || a.ay < 0 || a.az < 0 || a.degree() > p_) {
      throw std::out_of_range("multi-index not found");
    }
    return basis_rank(a);
  }

  static double factorial(int n) {
    double v = 1.0;
    for (int i = 2; i <= n; ++i) {
      v *= i;
    }
    return v;
  }
  static double multi_factorial(const MultiIndex &a) {
    return factorial(a.ax) * factorial(a.ay) * factorial(a.az);
  }
  /// r^alpha / alpha!
  static double monomial_over_factorial(const Vec3 &r, const MultiIndex &a) {
    return std::pow(r.x, a.ax) * std::pow(r.y, a.ay) * std::pow(r.z, a.az) / multi_factorial(a);
  }

private:
  int p_;
  std::vector<MultiIndex> indices_;
};

} // namespace cdfmm
