// Plan geometry on the device (see geometry.hpp).
//
// The tree follows the host tree (upstream src/uniform_tree.cpp) where the
// result must be bit-exact:
//   root cube  (:141-196): bounding box of both populations, centre
//              (lo + hi) * 0.5, half width the largest of hi - c and c - lo;
//   leaf keys  (:198-223): floor((x - box_lo) / cell_width) clamped to the
//              grid, inside-the-box test with the 1e-12 tolerance, Morton
//              interleave x | y << 1 | z << 2;
//   ordering   (:290-357): each population stably ordered by leaf key.
// Every FP64 operation is the IEEE-rounded intrinsic of the same operation
// (no contraction), so the keys equal the host's.  The ordering is CUB's LSD
// radix sort of (key, user index) pairs, which is stable: points of one leaf
// keep their user order, as in the reference's stable sort.
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <new>
#include <stdexcept>

#include "geometry.hpp"
#include "kernels.cuh"

namespace cdfmm_b200 {

namespace {

constexpr double kBoundaryTolerance = 1.0e-12;
constexpr int kThreads = 256;

// Monotone map of finite doubles to unsigned integers (both zeros map to
// the key of +0), so min / max are integer atomics.
__host__ __device__ inline unsigned long long order_key(double v) {
  if (v == 0.0) v = 0.0;
  unsigned long long u;
  std::memcpy(&u, &v, sizeof u);
  return (u >> 63) != 0ULL ? ~u : (u | (1ULL << 63));
}

inline double from_order_key(unsigned long long k) {
  const unsigned long long u = (k >> 63) != 0ULL ? (k & ~(1ULL << 63)) : ~k;
  double v;
  std::memcpy(&v, &u, sizeof v);
  return v;
}

struct Bounds {
  unsigned long long lo[3];
  unsigned long long hi[3];
  int first_zero[3]; // first point (sources, then targets) whose coordinate is +-0
  int bad;           // first point with a non-finite coordinate
};

__device__ inline unsigned long long warp_min(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ inline unsigned long long warp_max(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ inline int warp_min_int(int v) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Bounding box of sources [0, ns) and targets [ns, ns + nt).
__global__ void __launch_bounds__(kThreads) bounds_kernel(const double *src, int ns, const double *tgt, int nt,
                                                          Bounds *out) {
  unsigned long long lo[3] = {~0ULL, ~0ULL, ~0ULL}, hi[3] = {0ULL, 0ULL, 0ULL};
  int zero[3] = {INT_MAX, INT_MAX, INT_MAX};
  int bad = INT_MAX;
  const int n = ns + nt;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double *p = i < ns ? src + 3 * static_cast<size_t>(i) : tgt + 3 * static_cast<size_t>(i - ns);
    const double v[3] = {p[0], p[1], p[2]};
    if (!isfinite(v[0]) || !isfinite(v[1]) || !isfinite(v[2])) {
      bad = min(bad, i);
      continue;
    }
    for (int a = 0; a < 3; ++a) {
      const unsigned long long k = order_key(v[a]);
      lo[a] = min(lo[a], k);
      hi[a] = max(hi[a], k);
      if (v[a] == 0.0) zero[a] = min(zero[a], i);
    }
  }
  for (int a = 0; a < 3; ++a) {
    lo[a] = warp_min(lo[a]);
    hi[a] = warp_max(hi[a]);
    zero[a] = warp_min_int(zero[a]);
  }
  bad = warp_min_int(bad);
  if ((threadIdx.x & 31) == 0) {
    for (int a = 0; a < 3; ++a) {
      if (lo[a] != ~0ULL) atomicMin(&out->lo[a], lo[a]);
      if (hi[a] != 0ULL) atomicMax(&out->hi[a], hi[a]);
      if (zero[a] != INT_MAX) atomicMin(&out->first_zero[a], zero[a]);
    }
    if (bad != INT_MAX) atomicMin(&out->bad, bad);
  }
}

struct KeyParams {
  double box_lo[3];
  double in_lo[3]; // box_lo - tolerance
  double in_hi[3]; // box_hi + tolerance
  double cell_width;
  int side;
  int depth;
};

__device__ inline int leaf_coordinate(double v, double lo, double width, int side) {
  int i = static_cast<int>(floor(__ddiv_rn(__dsub_rn(v, lo), width)));
  if (i < 0) i = 0;
  if (i >= side) i = side - 1;
  return i;
}

// Leaf key and user index of every point; *outside = the first point
// outside the (tolerance-widened) root box.
__global__ void __launch_bounds__(kThreads) leaf_key_kernel(const double *pos, int n, KeyParams kp, uint32_t *keys,
                                                            int *index, int *outside) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v[3] = {pos[3 * static_cast<size_t>(i)], pos[3 * static_cast<size_t>(i) + 1],
                       pos[3 * static_cast<size_t>(i) + 2]};
  bool inside = true;
  for (int a = 0; a < 3; ++a) inside = inside && v[a] >= kp.in_lo[a] && v[a] <= kp.in_hi[a];
  uint32_t key = 0;
  if (!inside) {
    atomicMin(outside, i);
  } else if (kp.depth > 0) {
    key = morton3(static_cast<uint32_t>(leaf_coordinate(v[0], kp.box_lo[0], kp.cell_width, kp.side)),
                  static_cast<uint32_t>(leaf_coordinate(v[1], kp.box_lo[1], kp.cell_width, kp.side)),
                  static_cast<uint32_t>(leaf_coordinate(v[2], kp.box_lo[2], kp.cell_width, kp.side)));
  }
  keys[i] = key;
  index[i] = i;
}

// offsets[m] = first sorted point whose key is >= m, m in [0, n_leaves].
__global__ void __launch_bounds__(kThreads) leaf_offsets_kernel(const uint32_t *keys, int n, int n_leaves,
                                                                int *offsets) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > n_leaves) return;
  int a = 0, b = n;
  while (a < b) {
    const int mid = (a + b) >> 1;
    if (keys[mid] < static_cast<uint32_t>(m)) a = mid + 1;
    else b = mid;
  }
  offsets[m] = a;
}

__global__ void __launch_bounds__(kThreads) gather_positions_kernel(const double *pos, const int *perm, int n,
                                                                    double *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const size_t j = static_cast<size_t>(perm[i]);
  for (int a = 0; a < 3; ++a) out[3 * static_cast<size_t>(i) + a] = pos[3 * j + a];
}

__device__ inline int leaf_of(const int *offsets, int n_leaves, int j) {
  // last m with offsets[m] <= j (that leaf is non-empty and holds j)
  int a = 0, b = n_leaves;
  while (a < b) {
    const int mid = (a + b + 1) >> 1;
    if (offsets[mid] <= j) a = mid;
    else b = mid - 1;
  }
  return a;
}

__global__ void __launch_bounds__(kThreads) relative_positions_kernel(const double *pos, const int *offsets,
                                                                      int n_leaves, int n, int side, double cx,
                                                                      double cy, double cz, double hw, double inv,
                                                                      float4 *out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int m = leaf_of(offsets, n_leaves, j);
  int c3[3];
  demorton3(static_cast<uint32_t>(m), c3[0], c3[1], c3[2]);
  const double centre[3] = {cx, cy, cz};
  float r[3];
  for (int a = 0; a < 3; ++a) {
    // ((c + 0.5) / side - 0.5) * 2 * hw, then (leaf centre - centre) * inv
    const double offset =
        __dmul_rn(__dmul_rn(__dsub_rn(__ddiv_rn(__dadd_rn(static_cast<double>(c3[a]), 0.5), static_cast<double>(side)),
                                      0.5),
                            2.0),
                  hw);
    const double nc = __dmul_rn(__dsub_rn(__dadd_rn(centre[a], offset), centre[a]), inv);
    const double np = __dmul_rn(__dsub_rn(pos[3 * static_cast<size_t>(j) + a], centre[a]), inv);
    r[a] = __double2float_rn(__dsub_rn(np, nc));
  }
  out[j] = make_float4(r[0], r[1], r[2], 0.0F);
}

__global__ void __launch_bounds__(kThreads) normalised_positions_kernel(const double *pos, int n, double cx, double cy,
                                                                        double cz, double inv, double *out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double centre[3] = {cx, cy, cz};
  for (int a = 0; a < 3; ++a)
    out[3 * static_cast<size_t>(j) + a] = __dmul_rn(__dsub_rn(pos[3 * static_cast<size_t>(j) + a], centre[a]), inv);
}

__global__ void __launch_bounds__(kThreads) inverse_permutation_kernel(const int *perm, int n, int *inv, int *flag) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int v = perm[j];
  if (v < 0 || v >= n) {
    atomicOr(flag, 1);
  } else if (atomicExch(&inv[v], j) != -1) {
    atomicOr(flag, 2);
  }
}

__global__ void __launch_bounds__(kThreads) identity_self_kernel(int n, const int *offsets, int n_leaves,
                                                                 int *self_idx, int2 *leaf_self) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) self_idx[i] = i;
  if (i < n_leaves) {
    const int a = offsets[i], b = offsets[i + 1];
    leaf_self[i] = a < b ? make_int2(a, b - 1) : make_int2(INT_MAX, -1);
  }
}

int blocks_for(long long n) { return static_cast<int>((n + kThreads - 1) / kThreads); }

struct DeviceBuffers {
  std::vector<void *> ptrs;
  ~DeviceBuffers() {
    for (void *p : ptrs)
      if (p != nullptr) cudaFree(p);
  }
  template <typename T> T *alloc(size_t count) {
    void *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      throw std::bad_alloc();
    }
    ptrs.push_back(p);
    return static_cast<T *>(p);
  }
  // Hands the allocation over to the caller (not freed here).
  void release(const void *p) {
    for (void *&q : ptrs)
      if (q == p) q = nullptr;
  }
};

void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Keys, stable order, ranges and sorted positions of one population.
void order_population(const double *pos, int n, int depth, const KeyParams &kp, SortedPopulation &out,
                      DeviceBuffers &owned, DeviceBuffers &tmp, int *outside, cudaStream_t s) {
  const int n_leaves = 1 << (3 * depth);
  out.positions = owned.alloc<double>(3 * static_cast<size_t>(n));
  out.permutation = owned.alloc<int>(static_cast<size_t>(n));
  out.offsets = owned.alloc<int>(static_cast<size_t>(n_leaves) + 1);
  out.host_offsets.assign(static_cast<size_t>(n_leaves) + 1, 0);
  if (n == 0) {
    check_cuda(cudaMemsetAsync(out.offsets, 0, sizeof(int) * (static_cast<size_t>(n_leaves) + 1), s), "memset");
    return;
  }
  uint32_t *keys = tmp.alloc<uint32_t>(static_cast<size_t>(n));
  uint32_t *keys_sorted = tmp.alloc<uint32_t>(static_cast<size_t>(n));
  int *index = tmp.alloc<int>(static_cast<size_t>(n));
  leaf_key_kernel<<<blocks_for(n), kThreads, 0, s>>>(pos, n, kp, keys, index, outside);
  check_cuda(cudaGetLastError(), "leaf keys");
  // bits [0, 3 depth) hold the key (one bit at depth 0: all keys are 0)
  const int end_bit = depth > 0 ? 3 * depth : 1;
  size_t temp_bytes = 0;
  check_cuda(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys, keys_sorted, index, out.permutation, n, 0,
                                             end_bit, s),
             "radix sort (size)");
  void *temp = tmp.alloc<unsigned char>(temp_bytes);
  check_cuda(cub::DeviceRadixSort::SortPairs(temp, temp_bytes, keys, keys_sorted, index, out.permutation, n, 0,
                                             end_bit, s),
             "radix sort");
  leaf_offsets_kernel<<<blocks_for(static_cast<long long>(n_leaves) + 1), kThreads, 0, s>>>(keys_sorted, n, n_leaves,
                                                                                           out.offsets);
  gather_positions_kernel<<<blocks_for(n), kThreads, 0, s>>>(pos, out.permutation, n, out.positions);
  check_cuda(cudaGetLastError(), "leaf ranges");
}

} // namespace

std::string build_device_tree(const double *sources, int ns, const double *targets, int nt, int depth,
                              const RootRequest &root, double centre_out[3], double &half_width_out,
                              SortedPopulation &src, SortedPopulation &tgt, cudaStream_t s) {
  DeviceBuffers owned, tmp;
  // Unless the build succeeds, `owned` frees the arrays: the outputs must
  // not keep pointers to them.
  struct ClearUnlessDone {
    SortedPopulation &a, &b;
    bool done = false;
    ~ClearUnlessDone() {
      if (!done) {
        a = SortedPopulation();
        b = SortedPopulation();
      }
    }
  } guard{src, tgt};
  const bool same = targets == nullptr;
  if (same) nt = ns;
  // --- root cube (bounding box over both populations) ---
  Bounds init;
  for (int a = 0; a < 3; ++a) {
    init.lo[a] = ~0ULL;
    init.hi[a] = 0ULL;
    init.first_zero[a] = INT_MAX;
  }
  init.bad = INT_MAX;
  Bounds *d_bounds = tmp.alloc<Bounds>(1);
  int *d_outside = tmp.alloc<int>(2);
  check_cuda(cudaMemcpyAsync(d_bounds, &init, sizeof init, cudaMemcpyHostToDevice, s), "bounds init");
  const int big = INT_MAX;
  check_cuda(cudaMemcpyAsync(d_outside, &big, sizeof big, cudaMemcpyHostToDevice, s), "flag init");
  check_cuda(cudaMemcpyAsync(d_outside + 1, &big, sizeof big, cudaMemcpyHostToDevice, s), "flag init");
  const int n_all = ns + (same ? 0 : nt);
  if (n_all > 0) {
    bounds_kernel<<<std::min(blocks_for(n_all), 4 * 148), kThreads, 0, s>>>(sources, ns, targets, same ? 0 : nt,
                                                                           d_bounds);
    check_cuda(cudaGetLastError(), "bounds");
  }
  Bounds b;
  check_cuda(cudaMemcpyAsync(&b, d_bounds, sizeof b, cudaMemcpyDeviceToHost, s), "bounds D2H");
  check_cuda(cudaStreamSynchronize(s), "bounds");
  if (b.bad != INT_MAX) return "Point lies outside the requested root box";
  const bool any = n_all > 0;
  double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {0.0, 0.0, 0.0};
  if (any) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = from_order_key(b.lo[a]);
      hi[a] = from_order_key(b.hi[a]);
      // the host tree keeps the first of equal extremes: for +-0 that
      // point's zero decides the sign
      if ((lo[a] == 0.0 || hi[a] == 0.0) && b.first_zero[a] != INT_MAX) {
        const int i = b.first_zero[a];
        const double *p = i < ns ? sources + 3 * static_cast<size_t>(i) : targets + 3 * static_cast<size_t>(i - ns);
        double z = 0.0;
        check_cuda(cudaMemcpy(&z, p + a, sizeof z, cudaMemcpyDeviceToHost), "zero sign");
        if (lo[a] == 0.0) lo[a] = z;
        if (hi[a] == 0.0) hi[a] = z;
      }
    }
  }
  double c[3];
  for (int a = 0; a < 3; ++a) c[a] = root.has_centre ? root.centre[a] : (lo[a] + hi[a]) * 0.5;
  double hw;
  if (root.has_half_width) {
    hw = root.half_width;
  } else if (!any) {
    hw = 1.0;
  } else {
    hw = -std::numeric_limits<double>::infinity();
    for (int a = 0; a < 3; ++a) hw = std::max(hw, hi[a] - c[a]);
    for (int a = 0; a < 3; ++a) hw = std::max(hw, c[a] - lo[a]);
  }
  KeyParams kp{};
  for (int a = 0; a < 3; ++a) {
    kp.box_lo[a] = c[a] - hw;
    kp.in_lo[a] = kp.box_lo[a] - kBoundaryTolerance;
    kp.in_hi[a] = (c[a] + hw) + kBoundaryTolerance;
  }
  kp.side = 1 << depth;
  kp.depth = depth;
  kp.cell_width = (2.0 * hw) / static_cast<double>(kp.side);
  // --- keys, stable ordering, leaf ranges ---
  order_population(sources, ns, depth, kp, src, owned, tmp, d_outside, s);
  if (same) {
    const int n_leaves = 1 << (3 * depth);
    tgt.positions = owned.alloc<double>(3 * static_cast<size_t>(nt));
    tgt.permutation = owned.alloc<int>(static_cast<size_t>(nt));
    tgt.offsets = owned.alloc<int>(static_cast<size_t>(n_leaves) + 1);
    if (nt > 0) {
      check_cuda(cudaMemcpyAsync(tgt.positions, src.positions, 24 * static_cast<size_t>(nt), cudaMemcpyDeviceToDevice, s),
                 "copy");
      check_cuda(cudaMemcpyAsync(tgt.permutation, src.permutation, 4 * static_cast<size_t>(nt),
                                 cudaMemcpyDeviceToDevice, s),
                 "copy");
    }
    check_cuda(cudaMemcpyAsync(tgt.offsets, src.offsets, 4 * (static_cast<size_t>(n_leaves) + 1),
                               cudaMemcpyDeviceToDevice, s),
               "copy");
  } else {
    order_population(targets, nt, depth, kp, tgt, owned, tmp, d_outside + 1, s);
  }
  int outside[2] = {INT_MAX, INT_MAX};
  check_cuda(cudaMemcpyAsync(outside, d_outside, sizeof outside, cudaMemcpyDeviceToHost, s), "flag D2H");
  src.host_offsets.resize((static_cast<size_t>(1) << (3 * depth)) + 1);
  check_cuda(cudaMemcpyAsync(src.host_offsets.data(), src.offsets, sizeof(int) * src.host_offsets.size(),
                             cudaMemcpyDeviceToHost, s),
             "offsets D2H");
  check_cuda(cudaStreamSynchronize(s), "tree");
  if (outside[0] != INT_MAX || outside[1] != INT_MAX) return "Point lies outside the requested root box";
  tgt.host_offsets = src.host_offsets;
  if (!same) {
    check_cuda(cudaMemcpy(tgt.host_offsets.data(), tgt.offsets, sizeof(int) * tgt.host_offsets.size(),
                          cudaMemcpyDeviceToHost),
               "offsets D2H");
  }
  for (const void *p : {static_cast<const void *>(src.positions), static_cast<const void *>(src.permutation),
                        static_cast<const void *>(src.offsets), static_cast<const void *>(tgt.positions),
                        static_cast<const void *>(tgt.permutation), static_cast<const void *>(tgt.offsets)})
    owned.release(p);
  for (int a = 0; a < 3; ++a) centre_out[a] = c[a];
  half_width_out = hw;
  guard.done = true;
  return std::string();
}

void launch_relative_positions(const double *pos, const int *offsets, int n_leaves, int n, int depth,
                               const double centre[3], double half_width, double inv_scale, float4 *out,
                               cudaStream_t s) {
  if (n == 0) return;
  relative_positions_kernel<<<blocks_for(n), kThreads, 0, s>>>(pos, offsets, n_leaves, n, 1 << depth, centre[0],
                                                               centre[1], centre[2], half_width, inv_scale, out);
}

void launch_normalised_positions(const double *pos, int n, const double centre[3], double inv_scale, double *out,
                                 cudaStream_t s) {
  if (n == 0) return;
  normalised_positions_kernel<<<blocks_for(n), kThreads, 0, s>>>(pos, n, centre[0], centre[1], centre[2], inv_scale,
                                                                 out);
}

void launch_inverse_permutation(const int *perm, int n, int *inv, int *flag, cudaStream_t s) {
  if (n == 0) return;
  inverse_permutation_kernel<<<blocks_for(n), kThreads, 0, s>>>(perm, n, inv, flag);
}

void launch_identity_self(int n, const int *offsets, int n_leaves, int *self_idx, int2 *leaf_self, cudaStream_t s) {
  const long long m = std::max<long long>(n, n_leaves);
  if (m == 0) return;
  identity_self_kernel<<<blocks_for(m), kThreads, 0, s>>>(n, offsets, n_leaves, self_idx, leaf_self);
}

} // namespace cdfmm_b200
