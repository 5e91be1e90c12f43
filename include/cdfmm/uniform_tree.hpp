// Complete uniform octree with level-wise Morton ordering.
//
// Construction semantics are those of upstream dip-fmm's UniformTree
// (src/uniform_tree.cpp:129-523): a cubic root around the combined source and
// target bounding box (or the caller's centre / half-width), leaves assigned
// by floor((x - lo) / w) clamped to [0, n-1] with a 1e-12 boundary tolerance,
// sources and targets stably sorted (independently) by leaf Morton key, flat
// node index = (8^level - 1)/7 + morton(ix, iy, iz), half-open ranges per node
// and list1/list2 in ascending flat index.  The permutations, ranges and lists
// are bit-exact with the reference; the stable sort is a counting sort over
// leaf keys, which yields the same order as std::stable_sort on the key.
#pragma once

#include <array>
#include <cstdint>
#include <optional>
#include <span>
#include <vector>

#include "cdfmm/timings.hpp"
#include "cdfmm/tree_node.hpp"

namespace cdfmm {

struct UniformTreeOptions {
  int max_level{1};
  bool include_empty_nodes{true};
  bool cubic_root_box{true};
  std::optional<Vec3> root_centre{};
  std::optional<double> root_half_width{};
};

/// Interleave the low 21 bits of each coordinate: bit 3b+0 <- x, 3b+1 <- y, 3b+2 <- z.
std::uint64_t morton_encode(int ix, int iy, int iz);
std::array<int, 3> morton_decode(std::uint64_t morton);
/// (8^level - 1) / 7: flat index of the first node of a level.
int level_offset(int level);
int node_index(int level, int ix, int iy, int iz);

class UniformTree {
public:
  UniformTree(const std::vector<Vec3> &source_positions, const UniformTreeOptions &options);
  UniformTree(const std::vector<Vec3> &source_positions,
              const std::vector<Vec3> &target_positions, const UniformTreeOptions &options);

  int max_level() const { return max_level_; }
  int n_levels() const { return max_level_ + 1; }
  int leaf_level() const { return max_level_; }
  const Vec3 &root_centre() const { return root_centre_; }
  double root_half_width() const { return root_half_width_; }
  std::span<const TreeNode> nodes() const { return nodes_; }
  std::span<const Vec3> sorted_source_positions() const { return sources_sorted_; }
  std::span<const Vec3> sorted_target_positions() const { return targets_sorted_; }
  std::span<const int> source_permutation() const { return source_perm_; }
  std::span<const int> source_inverse_permutation() const { return source_inv_; }
  std::span<const int> target_permutation() const { return target_perm_; }
  std::span<const int> target_inverse_permutation() const { return target_inv_; }
  std::span<const int> leaf_indices() const { return leaf_indices_; }
  std::span<const int> occupied_source_leaves() const { return occupied_source_leaves_; }
  std::span<const int> occupied_target_leaves() const { return occupied_target_leaves_; }
  const TreeBuildTimings &build_timings() const { return timings_; }
  int leaf_index_for_source(std::size_t sorted_source_index) const {
    return source_leaf_.at(sorted_source_index);
  }
  int leaf_index_for_target(std::size_t sorted_target_index) const {
    return target_leaf_.at(sorted_target_index);
  }

  /// Exclusive prefix of source counts over leaves in Morton order
  /// (8^max_level + 1 entries): leaf m owns sorted sources [o[m], o[m+1]).
  std::vector<int> leaf_source_offsets() const;
  std::vector<int> leaf_target_offsets() const;

private:
  void build(const std::vector<Vec3> &sources, const std::vector<Vec3> &targets,
             const UniformTreeOptions &options);

  std::vector<TreeNode> nodes_{};
  std::vector<Vec3> sources_sorted_{};
  std::vector<int> source_perm_{};
  std::vector<int> source_inv_{};
  std::vector<int> source_leaf_{};
  std::vector<Vec3> targets_sorted_{};
  std::vector<int> target_perm_{};
  std::vector<int> target_inv_{};
  std::vector<int> target_leaf_{};
  std::vector<int> leaf_indices_{};
  std::vector<int> occupied_source_leaves_{};
  std::vector<int> occupied_target_leaves_{};
  TreeBuildTimings timings_{};
  Vec3 root_centre_{};
  double root_half_width_{0.0};
  int max_level_{0};
};

} // namespace cdfmm
