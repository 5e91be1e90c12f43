// One box of the complete uniform octree.
//
// Member names, meanings and the half-open [begin, end) range convention follow
// upstream dip-fmm (include/cdfmm/tree_node.hpp:29-71); the tree parity tests
// compare these fields with the reference element by element.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "cdfmm/vec3.hpp"

namespace cdfmm {

struct TreeNode {
  int index{-1};
  int level{0};
  int parent{-1};
  std::array<int, 8> children{{-1, -1, -1, -1, -1, -1, -1, -1}};
  int ix{0};
  int iy{0};
  int iz{0};
  std::uint64_t morton_index{0};
  Vec3 centre{};
  double half_width{0.0};
  std::size_t source_begin{0};
  std::size_t source_end{0};
  std::size_t target_begin{0};
  std::size_t target_end{0};
  /// Same-level boxes touching this one (3x3x3 clipped), itself included,
  /// ascending flat index.
  std::vector<int> list1{};
  /// Children of the parent's list1 that are not in list1, ascending.
  std::vector<int> list2{};

  bool is_leaf() const {
    for (int c : children) {
      if (c >= 0) {
        return false;
      }
    }
    return true;
  }
  std::size_t source_count() const { return source_end - source_begin; }
  std::size_t target_count() const { return target_end - target_begin; }
};

} // namespace cdfmm
