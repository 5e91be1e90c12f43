// Complete uniform octree (host, FP64 geometry).
//
// Follows upstream src/uniform_tree.cpp:129-523 operation for operation where
// the result must be bit-exact: the root cube (:141-196), leaf assignment
// (:198-223), node centres (:227-261), Morton keys (:71-85), stable ordering
// of each population by leaf key (:290-357), half-open ranges with the
// population-size sentinel for empty boxes (:359-438) and list1/list2 in
// ascending flat index (:455-516).  The stable sort is a counting sort on the
// leaf Morton key (same permutation as a stable comparison sort, O(N)).
#include "cdfmm/uniform_tree.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <limits>
#include <numeric>
#include <stdexcept>

namespace cdfmm {

namespace {

using Clock = std::chrono::steady_clock;
constexpr double kBoundaryTolerance = 1.0e-12;

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

std::size_t complete_node_count(int max_level) {
  std::size_t total = 0;
  std::size_t per_level = 1;
  for (int l = 0; l <= max_level; ++l) {
    total += per_level;
    per_level *= 8;
  }
  return total;
}

// Spread the low 21 bits of v so that bit b lands on bit 3b.
std::uint64_t spread3(std::uint64_t v) {
  v &= 0x1fffffULL;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}

int compact3(std::uint64_t v) {
  v &= 0x1249249249249249ULL;
  v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ULL;
  v = (v ^ (v >> 4)) & 0x100f00f00f00f00fULL;
  v = (v ^ (v >> 8)) & 0x1f0000ff0000ffULL;
  v = (v ^ (v >> 16)) & 0x1f00000000ffffULL;
  v = (v ^ (v >> 32)) & 0x1fffffULL;
  return static_cast<int>(v);
}

} // namespace

std::uint64_t morton_encode(int ix, int iy, int iz) {
  return spread3(static_cast<std::uint64_t>(ix)) |
         (spread3(static_cast<std::uint64_t>(iy)) << 1) |
         (spread3(static_cast<std::uint64_t>(iz)) << 2);
}

std::array<int, 3> morton_decode(std::uint64_t m) {
  return {compact3(m), compact3(m >> 1), compact3(m >> 2)};
}

int level_offset(int level) {
  std::size_t p = 1;
  for (int i = 0; i < level; ++i) {
    p *= 8;
  }
  return static_cast<int>((p - 1) / 7);
}

int node_index(int level, int ix, int iy, int iz) {
  return level_offset(level) + static_cast<int>(morton_encode(ix, iy, iz));
}

UniformTree::UniformTree(const std::vector<Vec3> &source_positions,
                         const UniformTreeOptions &options) {
  build(source_positions, {}, options);
}

UniformTree::UniformTree(const std::vector<Vec3> &source_positions,
                         const std::vector<Vec3> &target_positions,
                         const UniformTreeOptions &options) {
  build(source_positions, target_positions, options);
}

void UniformTree::build(const std::vector<Vec3> &sources, const std::vector<Vec3> &targets,
                        const UniformTreeOptions &options) {
  const auto t_total = Clock::now();
  if (options.max_level < 0) {
    throw std::invalid_argument("UniformTreeOptions.max_level must be >= 0");
  }
  if (options.root_half_width.has_value() && options.root_half_width.value() <= 0.0) {
    throw std::invalid_argument("UniformTreeOptions.root_half_width must be positive");
  }
  if (options.max_level > 20) {
    throw std::invalid_argument("UniformTreeOptions.max_level must be <= 20");
  }
  max_level_ = options.max_level;

  // --- root cube ---------------------------------------------------------
  auto t0 = Clock::now();
  const double inf = std::numeric_limits<double>::infinity();
  Vec3 lo{inf, inf, inf};
  Vec3 hi{-inf, -inf, -inf};
  bool any = false;
  for (const auto *population : {&sources, &targets}) {
    for (const Vec3 &p : *population) {
      any = true;
      lo.x = std::min(lo.x, p.x);
      lo.y = std::min(lo.y, p.y);
      lo.z = std::min(lo.z, p.z);
      hi.x = std::max(hi.x, p.x);
      hi.y = std::max(hi.y, p.y);
      hi.z = std::max(hi.z, p.z);
    }
  }
  if (!any) {
    lo = {0.0, 0.0, 0.0};
    hi = {0.0, 0.0, 0.0};
  }
  root_centre_ = options.root_centre.has_value() ? options.root_centre.value() : (lo + hi) * 0.5;
  if (options.root_half_width.has_value()) {
    root_half_width_ = options.root_half_width.value();
  } else if (!any) {
    root_half_width_ = 1.0;
  } else {
    const Vec3 up = hi - root_centre_;
    const Vec3 down = root_centre_ - lo;
    root_half_width_ = std::max({up.x, up.y, up.z, down.x, down.y, down.z});
  }
  const Vec3 box_lo = root_centre_ - Vec3{root_half_width_, root_half_width_, root_half_width_};
  const Vec3 box_hi = root_centre_ + Vec3{root_half_width_, root_half_width_, root_half_width_};
  timings_.root_bounds.add(seconds_since(t0));

  const int n_leaf_side = 1 << max_level_;
  const double cell_width = (2.0 * root_half_width_) / static_cast<double>(n_leaf_side);
  auto leaf_coordinate = [&](double v, double lo_v) {
    int i = static_cast<int>(std::floor((v - lo_v) / cell_width));
    if (i < 0) {
      i = 0;
    }
    if (i >= n_leaf_side) {
      i = n_leaf_side - 1;
    }
    return i;
  };
  auto inside = [&](double v, double a, double b) {
    return v >= a - kBoundaryTolerance && v <= b + kBoundaryTolerance;
  };
  // Leaf Morton key of one point (throws for points outside the root cube).
  auto leaf_key = [&](const Vec3 &p) -> std::uint64_t {
    if (!inside(p.x, box_lo.x, box_hi.x) || !inside(p.y, box_lo.y, box_hi.y) ||
        !inside(p.z, box_lo.z, box_hi.z)) {
      throw std::invalid_argument("Point lies outside the requested root box");
    }
    if (max_level_ == 0) {
      return 0;
    }
    return morton_encode(leaf_coordinate(p.x, box_lo.x), leaf_coordinate(p.y, box_lo.y),
                         leaf_coordinate(p.z, box_lo.z));
  };

  // --- nodes ---------------------------------------------------------------
  t0 = Clock::now();
  nodes_.assign(complete_node_count(max_level_), TreeNode{});
  for (int level = 0; level <= max_level_; ++level) {
    const int n = 1 << level;
    const int base = level_offset(level);
    const std::int64_t count = static_cast<std::int64_t>(n) * n * n;
#pragma omp parallel for schedule(static) if (count >= 4096)
    for (std::int64_t m = 0; m < count; ++m) {
      const auto c = morton_decode(static_cast<std::uint64_t>(m));
      TreeNode &node = nodes_[static_cast<std::size_t>(base + m)];
      node.index = static_cast<int>(base + m);
      node.level = level;
      node.ix = c[0];
      node.iy = c[1];
      node.iz = c[2];
      node.morton_index = static_cast<std::uint64_t>(m);
      node.parent = level == 0 ? -1 : level_offset(level - 1) + static_cast<int>(m >> 3);
      node.half_width = root_half_width_ / static_cast<double>(1 << level);
      const double dn = static_cast<double>(n);
      const Vec3 offset{((static_cast<double>(c[0]) + 0.5) / dn - 0.5) * 2.0 * root_half_width_,
                        ((static_cast<double>(c[1]) + 0.5) / dn - 0.5) * 2.0 * root_half_width_,
                        ((static_cast<double>(c[2]) + 0.5) / dn - 0.5) * 2.0 * root_half_width_};
      node.centre = root_centre_ + offset;
      if (level < max_level_) {
        // Child slot bits are (dx, dy, dz) = Morton bits, so the 8 children of
        // Morton m are Morton 8m .. 8m+7 at the next level.
        const int child_base = level_offset(level + 1) + static_cast<int>(m << 3);
        for (int k = 0; k < 8; ++k) {
          node.children[static_cast<std::size_t>(k)] = child_base + k;
        }
      }
    }
  }
  timings_.node_construction.add(seconds_since(t0));

  // --- stable leaf-key ordering of each population -------------------------
  const int leaf_base = level_offset(max_level_);
  const std::size_t n_leaves = static_cast<std::size_t>(1) << (3 * max_level_);
  auto order_population = [&](const std::vector<Vec3> &pts, std::vector<Vec3> &sorted,
                              std::vector<int> &perm, std::vector<int> &inv,
                              std::vector<int> &leaf_of, PhaseTiming &t_key, PhaseTiming &t_sort) {
    const auto tk = Clock::now();
    const std::size_t n = pts.size();
    std::vector<std::uint64_t> keys(n);
    // Keys are computed serially so the first out-of-box point raises.
    for (std::size_t i = 0; i < n; ++i) {
      keys[i] = leaf_key(pts[i]);
    }
    t_key.add(seconds_since(tk));
    const auto ts = Clock::now();
    perm.resize(n);
    if (n_leaves <= (static_cast<std::size_t>(1) << 24)) {
      std::vector<int> start(n_leaves + 1, 0);
      for (std::size_t i = 0; i < n; ++i) {
        ++start[keys[i] + 1];
      }
      std::partial_sum(start.begin(), start.end(), start.begin());
      for (std::size_t i = 0; i < n; ++i) {
        perm[static_cast<std::size_t>(start[keys[i]]++)] = static_cast<int>(i);
      }
    } else {
      std::iota(perm.begin(), perm.end(), 0);
      std::stable_sort(perm.begin(), perm.end(),
                       [&](int a, int b) { return keys[static_cast<std::size_t>(a)] <
                                                  keys[static_cast<std::size_t>(b)]; });
    }
    sorted.resize(n);
    inv.resize(n);
    leaf_of.resize(n);
    for (std::size_t s = 0; s < n; ++s) {
      const int original = perm[s];
      sorted[s] = pts[static_cast<std::size_t>(original)];
      inv[static_cast<std::size_t>(original)] = static_cast<int>(s);
      leaf_of[s] = leaf_base + static_cast<int>(keys[static_cast<std::size_t>(original)]);
    }
    t_sort.add(seconds_since(ts));
  };
  order_population(sources, sources_sorted_, source_perm_, source_inv_, source_leaf_,
                   timings_.source_morton, timings_.source_sorting);
  order_population(targets, targets_sorted_, target_perm_, target_inv_, target_leaf_,
                   timings_.target_morton, timings_.target_sorting);

  // --- ranges ----------------------------------------------------------------
  t0 = Clock::now();
  const std::size_t ns = sources_sorted_.size();
  const std::size_t nt = targets_sorted_.size();
  for (TreeNode &node : nodes_) {
    node.source_begin = node.source_end = ns;
    node.target_begin = node.target_end = nt;
  }
  auto leaf_ranges = [&](const std::vector<int> &leaf_of, bool is_source) {
    std::size_t cursor = 0;
    while (cursor < leaf_of.size()) {
      std::size_t next = cursor + 1;
      while (next < leaf_of.size() && leaf_of[next] == leaf_of[cursor]) {
        ++next;
      }
      TreeNode &leaf = nodes_[static_cast<std::size_t>(leaf_of[cursor])];
      (is_source ? leaf.source_begin : leaf.target_begin) = cursor;
      (is_source ? leaf.source_end : leaf.target_end) = next;
      cursor = next;
    }
    const std::size_t population = is_source ? ns : nt;
    for (int level = max_level_ - 1; level >= 0; --level) {
      const int b = level_offset(level);
      const int e = level_offset(level + 1);
      for (int idx = b; idx < e; ++idx) {
        TreeNode &node = nodes_[static_cast<std::size_t>(idx)];
        std::size_t first = population;
        std::size_t last = 0;
        bool occupied = false;
        for (int child : node.children) {
          const TreeNode &c = nodes_[static_cast<std::size_t>(child)];
          const std::size_t cb = is_source ? c.source_begin : c.target_begin;
          const std::size_t ce = is_source ? c.source_end : c.target_end;
          if (cb == ce) {
            continue;
          }
          occupied = true;
          first = std::min(first, cb);
          last = std::max(last, ce);
        }
        if (!occupied) {
          last = first;
        }
        (is_source ? node.source_begin : node.target_begin) = first;
        (is_source ? node.source_end : node.target_end) = last;
      }
    }
  };
  leaf_ranges(source_leaf_, true);
  leaf_ranges(target_leaf_, false);
  timings_.ranges.add(seconds_since(t0));

  leaf_indices_.resize(n_leaves);
  occupied_source_leaves_.clear();
  occupied_target_leaves_.clear();
  for (std::size_t m = 0; m < n_leaves; ++m) {
    const int idx = leaf_base + static_cast<int>(m);
    leaf_indices_[m] = idx;
    if (nodes_[static_cast<std::size_t>(idx)].source_count() > 0) {
      occupied_source_leaves_.push_back(idx);
    }
    if (nodes_[static_cast<std::size_t>(idx)].target_count() > 0) {
      occupied_target_leaves_.push_back(idx);
    }
  }

  // --- interaction lists -------------------------------------------------------
  t0 = Clock::now();
  for (int level = 0; level <= max_level_; ++level) {
    const int n = 1 << level;
    const int b = level_offset(level);
    const int e = level_offset(level + 1);
#pragma omp parallel for schedule(static) if (e - b >= 512)
    for (int idx = b; idx < e; ++idx) {
      TreeNode &node = nodes_[static_cast<std::size_t>(idx)];
      node.list1.clear();
      node.list1.reserve(27);
      for (int dz = -1; dz <= 1; ++dz) {
        for (int dy = -1; dy <= 1; ++dy) {
          for (int dx = -1; dx <= 1; ++dx) {
            const int x = node.ix + dx;
            const int y = node.iy + dy;
            const int z = node.iz + dz;
            if (x >= 0 && x < n && y >= 0 && y < n && z >= 0 && z < n) {
              node.list1.push_back(node_index(level, x, y, z));
            }
          }
        }
      }
      std::sort(node.list1.begin(), node.list1.end());
      node.list2.clear();
      if (level == 0) {
        continue;
      }
      // Parent neighbours' children that do not touch this box: per axis the
      // child coordinate lies in [2(p-1), 2(p+1)+1] and |child - self| >= 2
      // on at least one axis.
      const int px = node.ix >> 1;
      const int py = node.iy >> 1;
      const int pz = node.iz >> 1;
      node.list2.reserve(189);
      for (int z = 2 * pz - 2; z <= 2 * pz + 3; ++z) {
        for (int y = 2 * py - 2; y <= 2 * py + 3; ++y) {
          for (int x = 2 * px - 2; x <= 2 * px + 3; ++x) {
            if (x < 0 || x >= n || y < 0 || y >= n || z < 0 || z >= n) {
              continue;
            }
            if (std::abs(x - node.ix) <= 1 && std::abs(y - node.iy) <= 1 &&
                std::abs(z - node.iz) <= 1) {
              continue;
            }
            node.list2.push_back(node_index(level, x, y, z));
          }
        }
      }
      std::sort(node.list2.begin(), node.list2.end());
    }
  }
  timings_.interaction_lists.add(seconds_since(t0));
  timings_.total.add(seconds_since(t_total));
}

std::vector<int> UniformTree::leaf_source_offsets() const {
  const int base = level_offset(max_level_);
  const std::size_t n_leaves = leaf_indices_.size();
  std::vector<int> off(n_leaves + 1, 0);
  for (std::size_t m = 0; m < n_leaves; ++m) {
    off[m + 1] = off[m] + static_cast<int>(nodes_[base + m].source_count());
  }
  return off;
}

std::vector<int> UniformTree::leaf_target_offsets() const {
  const int base = level_offset(max_level_);
  const std::size_t n_leaves = leaf_indices_.size();
  std::vector<int> off(n_leaves + 1, 0);
  for (std::size_t m = 0; m < n_leaves; ++m) {
    off[m + 1] = off[m] + static_cast<int>(nodes_[base + m].target_count());
  }
  return off;
}

} // namespace cdfmm
