// Plan geometry on the device: the uniform octree of user-order positions
// (root cube, leaf Morton keys, stable ordering, leaf ranges) and the
// per-point arrays the evaluator reads (leaf-relative FP32 positions,
// inverse permutations, the identity self map).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

namespace cdfmm_b200 {

// Root cube request: each part explicit or derived from the bounding box.
struct RootRequest {
  bool has_centre = false;
  double centre[3] = {0.0, 0.0, 0.0};
  bool has_half_width = false;
  double half_width = 0.0;
};

// One population ordered by leaf: device arrays the builder allocates (the
// caller owns and frees them) and the host copy of the leaf ranges.
struct SortedPopulation {
  double *positions = nullptr; // [n][3] FP64, leaf order
  int *permutation = nullptr;  // [n] sorted index -> user index
  int *offsets = nullptr;      // [8^depth + 1] leaf m holds [o[m], o[m+1])
  std::vector<int> host_offsets;
};

// Builds the tree of `ns` sources and `nt` targets (device FP64 [n][3] user
// order; targets == nullptr: the targets are the sources) at `depth` on
// stream `s` and returns "" or the message of an invalid input (a point
// outside the root box, a non-finite coordinate).  The root cube, each leaf
// key and the stable ordering are bit-identical to cdfmm::UniformTree's.
// Output arrays are allocated with cudaMalloc; on error none is left.
std::string build_device_tree(const double *sources, int ns, const double *targets, int nt, int depth,
                              const RootRequest &root, double centre_out[3], double &half_width_out,
                              SortedPopulation &src, SortedPopulation &tgt, cudaStream_t s);

// Leaf-relative normalised FP32 positions (x - leaf centre) / (2 hw), .w = 0,
// of Morton-sorted FP64 positions; the FP64 operations of the host
// normalisation, in the same order and without contraction.
void launch_relative_positions(const double *pos, const int *offsets, int n_leaves, int n, int depth,
                               const double centre[3], double half_width, double inv_scale, float4 *out,
                               cudaStream_t s);
// Root-normalised FP64 positions (x - centre) * inv_scale, [n][3].
void launch_normalised_positions(const double *pos, int n, const double centre[3], double inv_scale, double *out,
                                 cudaStream_t s);
// inv[perm[j]] = j; `inv` must hold -1 everywhere on entry.  Sets bit 1 of
// *flag for an entry out of [0, n), bit 2 for a repeated entry.
void launch_inverse_permutation(const int *perm, int n, int *inv, int *flag, cudaStream_t s);
// The self map of targets that are the sources (one stable ordering for
// both): sorted target j is sorted source j; per leaf the self-source range
// is the leaf's own range.
void launch_identity_self(int n, const int *offsets, int n_leaves, int *self_idx, int2 *leaf_self, cudaStream_t s);

} // namespace cdfmm_b200
