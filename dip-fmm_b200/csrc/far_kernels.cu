// Far-field stages of the evaluator, FP32 SIMT: moment gather, P2M, M2M, L2L,
// L2P (fused with the near/far combine and the unsort to user order).
//
// Layouts (K = states of the call):
//   mom [ns][K]            float4 (mx, my, mz, 0), Morton-sorted, scaled by 1/scale^3
//   M, L [node][coef][K]   node = (8^level - 1)/7 + morton(ix, iy, iz)
//   near [nt][K]           float4 (phi, Hx, Hy, Hz), Morton-sorted
// Each expansion coefficient is written by exactly one thread (no atomics),
// so results are deterministic run to run.
#include <cuda_runtime.h>

#include "far_kernels.hpp"
#include "kernels.cuh"

namespace cdfmm_b200 {

namespace {

// ---------------------------------------------------------------------------
// moments: user order [K][ns][3] (f32 / f64) -> sorted [ns][K] float4 / scale^3
// (upstream src/far_field.cpp:248-275, src/cuda_fmm.cu:56-64).
template <typename T>
__global__ void gather_moments_kernel(const T *__restrict__ user, const int *__restrict__ perm,
                                      int ns, int K, double inv_scale, float inv_scale3_f,
                                      float4 *__restrict__ mom) {
  const long long total = static_cast<long long>(ns) * K;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < total;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int j = static_cast<int>(q / K);
    const int k = static_cast<int>(q - static_cast<long long>(j) * K);
    const T *m = user + (static_cast<long long>(k) * ns + perm[j]) * 3;
    float4 v;
    if constexpr (sizeof(T) == 8) {
      // Same arithmetic as the reference FP32 boundary: m / s / s / s in FP64.
      v.x = static_cast<float>(static_cast<double>(m[0]) * inv_scale * inv_scale * inv_scale);
      v.y = static_cast<float>(static_cast<double>(m[1]) * inv_scale * inv_scale * inv_scale);
      v.z = static_cast<float>(static_cast<double>(m[2]) * inv_scale * inv_scale * inv_scale);
    } else {
      v.x = static_cast<float>(m[0]) * inv_scale3_f;
      v.y = static_cast<float>(m[1]) * inv_scale3_f;
      v.z = static_cast<float>(m[2]) * inv_scale3_f;
    }
    v.w = 0.0F;
    mom[q] = v;
  }
}

// Monomials d^mu / mu! for every |mu| <= q, written into out[rank(mu)].
__device__ inline void monomials(float dx, float dy, float dz, int q, float *out) {
  float xa = 1.0F;
  for (int a = 0; a <= q; ++a) {
    float xb = xa;
    for (int b = 0; a + b <= q; ++b) {
      float xc = xb;
      for (int c = 0; a + b + c <= q; ++c) {
        out[rank3(a, b, c)] = xc;
        xc = xc * dz * kInvInt[c + 1];
      }
      xb = xb * dy * kInvInt[b + 1];
    }
    xa = xa * dx * kInvInt[a + 1];
  }
}

// ---------------------------------------------------------------------------
// P2M (upstream docs/math.md P2M; src/static_operators.cpp:186-220):
//   M_alpha = (-1)^|alpha| sum_j sum_{k: alpha_k > 0} m_jk d_j^(alpha-e_k)/(alpha-e_k)!
// One CTA per leaf.  Accumulators for the leaf (n*K) live in shared memory,
// each owned by one thread; sources are staged in chunks with their
// monomials of degree <= p-1 precomputed once per source.
__global__ void p2m_kernel(const float4 *__restrict__ src_rel, const float4 *__restrict__ mom,
                           const int *__restrict__ src_off, const int8_t *__restrict__ basis,
                           float *__restrict__ M, int n, int p, int K, int leaf_node_base, int chunk) {
  extern __shared__ float smem[];
  const int nm1 = basis_size_d(p - 1);
  float *acc = smem;                                  // [n*K], padded to 16 bytes
  float *mono = acc + ((n * K + 3) & ~3);             // [chunk][nm1]
  float4 *smom = reinterpret_cast<float4 *>(mono + ((chunk * nm1 + 3) & ~3)); // [chunk][K]
  const int leaf = blockIdx.x;
  const int s0 = src_off[leaf];
  const int s1 = src_off[leaf + 1];
  const int items = n * K;
  for (int q = threadIdx.x; q < items; q += blockDim.x) acc[q] = 0.0F;
  for (int c0 = s0; c0 < s1; c0 += chunk) {
    const int cn = min(chunk, s1 - c0);
    __syncthreads();
    for (int j = threadIdx.x; j < cn; j += blockDim.x) {
      const float4 d = src_rel[c0 + j];
      if (nm1 > 0) monomials(d.x, d.y, d.z, p - 1, mono + j * nm1);
    }
    for (int q = threadIdx.x; q < cn * K; q += blockDim.x) smom[q] = mom[static_cast<long long>(c0) * K + q];
    __syncthreads();
    for (int q = threadIdx.x; q < items; q += blockDim.x) {
      const int a = q / K;
      const int k = q - a * K;
      const int ax = basis[4 * a], ay = basis[4 * a + 1], az = basis[4 * a + 2];
      if (ax + ay + az == 0) continue;
      const int ix = ax > 0 ? rank3(ax - 1, ay, az) : -1;
      const int iy = ay > 0 ? rank3(ax, ay - 1, az) : -1;
      const int iz = az > 0 ? rank3(ax, ay, az - 1) : -1;
      float v = 0.0F;
      for (int j = 0; j < cn; ++j) {
        const float4 m = smom[j * K + k];
        const float *mj = mono + j * nm1;
        if (ix >= 0) v = fmaf(m.x, mj[ix], v);
        if (iy >= 0) v = fmaf(m.y, mj[iy], v);
        if (iz >= 0) v = fmaf(m.z, mj[iz], v);
      }
      acc[q] += ((ax + ay + az) & 1) ? -v : v;
    }
  }
  __syncthreads();
  float *out = M + static_cast<long long>(leaf_node_base + leaf) * items;
  for (int q = threadIdx.x; q < items; q += blockDim.x) out[q] = acc[q];
}

// ---------------------------------------------------------------------------
// M2M for one parent level (upstream src/far_field.cpp:303-331):
//   M_parent[alpha] = sum_children sum_{g <= alpha} A_class[g] M_child[alpha - g]
// Stages the pair list (offsets + packed pairs) and the 8 class coefficient
// rows of one level in shared memory.
__device__ inline void stage_pairs(const int *pair_off, const int *pairs, const float *cf, int n, int n_pairs,
                                   int *soff, int *spair, float *scoef) {
  for (int q = threadIdx.x; q <= n; q += blockDim.x) soff[q] = pair_off[q];
  for (int q = threadIdx.x; q < n_pairs; q += blockDim.x) spair[q] = pairs[q];
  for (int q = threadIdx.x; q < 8 * n; q += blockDim.x) scoef[q] = cf[q];
  __syncthreads();
}

// One thread per parent output coefficient (parent, alpha, state); the loads
// of the 8 children are independent of each other, so they overlap.
__global__ void __launch_bounds__(256) m2m_kernel(float *__restrict__ M, const int *__restrict__ pair_off,
                                                  const int *__restrict__ pairs, const float *__restrict__ coef,
                                                  int n, int K, int parent_level, int n_pairs) {
  extern __shared__ int shp[];
  int *soff = shp;
  int *spair = soff + n + 1;
  float *scoef = reinterpret_cast<float *>(spair + n_pairs);
  stage_pairs(pair_off, pairs, coef + static_cast<long long>(parent_level + 1) * 8 * n, n, n_pairs, soff, spair,
              scoef);
  const int parent_base = level_offset_d(parent_level);
  const int child_base = level_offset_d(parent_level + 1);
  const long long per = static_cast<long long>(n) * K;
  const long long total = (static_cast<long long>(1) << (3 * parent_level)) * per;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q >= total) return;
  const long long parent = q / per;
  const int rem = static_cast<int>(q - parent * per);
  const int a = rem / K;
  const int k = rem - a * K;
  const int e0 = soff[a], e1 = soff[a + 1];
  const float *child0 = M + (child_base + parent * 8) * per + k;
  float v = 0.0F;
#pragma unroll 2
  for (int c = 0; c < 8; ++c) {
    const float *child = child0 + c * per;
    const float *cc = scoef + c * n;
    for (int e = e0; e < e1; ++e) {
      const int pr = spair[e];
      v = fmaf(cc[pr & 0xffff], __ldg(child + static_cast<long long>(pr >> 16) * K), v);
    }
  }
  M[(parent_base + parent) * per + rem] = v;
}

// ---------------------------------------------------------------------------
// L2L for one child level (upstream src/far_field.cpp:533-581):
//   L_child[beta] += sum_{|beta + g| <= p} B_class[g] L_parent[beta + g]
__global__ void __launch_bounds__(256) l2l_kernel(float *__restrict__ L, const int *__restrict__ pair_off,
                                                  const int *__restrict__ pairs, const float *__restrict__ coef,
                                                  int n, int K, int child_level, int n_pairs) {
  extern __shared__ int shl[];
  int *soff = shl;
  int *spair = soff + n + 1;
  float *scoef = reinterpret_cast<float *>(spair + n_pairs);
  stage_pairs(pair_off, pairs, coef + static_cast<long long>(child_level) * 8 * n, n, n_pairs, soff, spair, scoef);
  const int child_base = level_offset_d(child_level);
  const int parent_base = level_offset_d(child_level - 1);
  const long long per = static_cast<long long>(n) * K;
  const long long total = (static_cast<long long>(1) << (3 * child_level)) * per;
  const long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x;
  if (q >= total) return;
  const long long child = q / per;
  const int rem = static_cast<int>(q - child * per);
  const int b = rem / K;
  const int k = rem - b * K;
  const int cls = static_cast<int>(child & 7);
  const float *parent = L + (parent_base + (child >> 3)) * per + k;
  const float *cc = scoef + cls * n;
  float v = 0.0F;
  for (int e = soff[b]; e < soff[b + 1]; ++e) {
    const int pr = spair[e];
    v = fmaf(cc[pr & 0xffff], __ldg(parent + static_cast<long long>(pr >> 16) * K), v);
  }
  L[(child_base + child) * per + rem] += v;
}

// ---------------------------------------------------------------------------
// L2P + combine + unsort (upstream docs/math.md L2P; src/cuda_fmm.cu:503-516):
//   phi = sum_b L_b dx^b/b!,  H_k = -sum_{b_k > 0} L_b dx^(b-e_k)/(b-e_k)!
// then result = far + near (near from the P2P kernel), phi times the root
// width, written at the target's user index.  One CTA per leaf; the leaf's
// local expansion (n*K) is staged in shared memory; a thread owns
// (target, group of up to 4 states).
__global__ void l2p_kernel(const float *__restrict__ L, const float4 *__restrict__ tgt_rel,
                           const int *__restrict__ tgt_off, const int *__restrict__ tgt_perm,
                           const float4 *__restrict__ near, int n, int p, int K, int nt,
                           int leaf_node_base, unsigned output, int layout, float phi_scale,
                           float *__restrict__ field, float *__restrict__ potential) {
  extern __shared__ float sL[]; // [n][K]
  const int leaf = blockIdx.x;
  const int t0 = tgt_off[leaf];
  const int t1 = tgt_off[leaf + 1];
  if (t0 == t1) return;
  const float *src = L + static_cast<long long>(leaf_node_base + leaf) * n * K;
  for (int q = threadIdx.x; q < n * K; q += blockDim.x) sL[q] = src[q];
  __syncthreads();
  const bool want_phi = (output & 1u) != 0u;
  const bool want_h = (output & 2u) != 0u;
  const int groups = (K + 3) / 4;
  const int items = (t1 - t0) * groups;
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    const int g = it / (t1 - t0);
    const int i = t0 + (it - g * (t1 - t0));
    const int kb = g * 4;
    const int kn = min(4, K - kb);
    const float4 d = tgt_rel[i];
    float phi[4] = {0, 0, 0, 0}, hx[4] = {0, 0, 0, 0}, hy[4] = {0, 0, 0, 0}, hz[4] = {0, 0, 0, 0};
    float xa = 1.0F;
    for (int a = 0; a <= p; ++a) {
      float xb = xa;
      for (int b = 0; a + b <= p; ++b) {
        float xc = xb;
        for (int c = 0; a + b + c <= p; ++c) {
          const int deg = a + b + c;
          const float *l0 = sL + rank3(a, b, c) * K + kb;
          const float *lx = deg < p ? sL + rank3(a + 1, b, c) * K + kb : nullptr;
          const float *ly = deg < p ? sL + rank3(a, b + 1, c) * K + kb : nullptr;
          const float *lz = deg < p ? sL + rank3(a, b, c + 1) * K + kb : nullptr;
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            if (s < kn) {
              if (want_phi) phi[s] = fmaf(l0[s], xc, phi[s]);
              if (want_h && deg < p) {
                hx[s] = fmaf(lx[s], xc, hx[s]);
                hy[s] = fmaf(ly[s], xc, hy[s]);
                hz[s] = fmaf(lz[s], xc, hz[s]);
              }
            }
          }
          xc = xc * d.z * kInvInt[c + 1];
        }
        xb = xb * d.y * kInvInt[b + 1];
      }
      xa = xa * d.x * kInvInt[a + 1];
    }
    const int u = tgt_perm[i];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      if (s >= kn) break;
      const int k = kb + s;
      const float4 nr = near[static_cast<long long>(i) * K + k];
      const float rphi = want_phi ? (phi[s] + nr.x) * phi_scale : 0.0F;
      const float rx = want_h ? nr.y - hx[s] : 0.0F;
      const float ry = want_h ? nr.z - hy[s] : 0.0F;
      const float rz = want_h ? nr.w - hz[s] : 0.0F;
      const long long o = static_cast<long long>(k) * nt + u;
      if (layout == 1) {
        reinterpret_cast<float4 *>(field)[o] = make_float4(rphi, rx, ry, rz);
      } else {
        if (want_h) {
          field[3 * o] = rx;
          field[3 * o + 1] = ry;
          field[3 * o + 2] = rz;
        }
        if (want_phi && potential != nullptr) potential[o] = rphi;
      }
    }
  }
}

} // namespace

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

void launch_gather_moments(const void *user, int dtype, const int *perm, int ns, int K,
                           double scale, float4 *mom, cudaStream_t s) {
  if (ns == 0) return;
  const long long total = static_cast<long long>(ns) * K;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 16));
  const double inv = 1.0 / scale;
  const float inv3f = static_cast<float>(inv * inv * inv);
  if (dtype == 1)
    gather_moments_kernel<double><<<blocks, 256, 0, s>>>(static_cast<const double *>(user), perm, ns, K, inv, inv3f, mom);
  else
    gather_moments_kernel<float><<<blocks, 256, 0, s>>>(static_cast<const float *>(user), perm, ns, K, inv, inv3f, mom);
}

size_t p2m_smem_bytes(int n, int p, int K, int chunk) {
  const int nm1 = basis_size_d(p - 1);
  return sizeof(float) * (((static_cast<size_t>(n) * K + 3) & ~static_cast<size_t>(3)) + ((chunk * nm1 + 3) & ~3)) +
         sizeof(float4) * static_cast<size_t>(chunk) * K;
}

void launch_p2m(const float4 *src_rel, const float4 *mom, const int *src_off, const int8_t *basis,
                float *M, int n, int p, int K, int depth, int chunk, cudaStream_t s) {
  const int leaves = 1 << (3 * depth);
  const size_t smem = p2m_smem_bytes(n, p, K, chunk);
  p2m_kernel<<<leaves, 128, smem, s>>>(src_rel, mom, src_off, basis, M, n, p, K,
                                       level_offset_d(depth), chunk);
}

static size_t pair_smem(int n, int n_pairs) {
  return sizeof(int) * (static_cast<size_t>(n) + 1 + n_pairs) + sizeof(float) * 8 * static_cast<size_t>(n);
}

void launch_m2m(float *M, const int *pair_off, const int *pairs, const float *coef, int n, int K,
                int parent_level, int n_pairs, cudaStream_t s) {
  const long long total = (static_cast<long long>(1) << (3 * parent_level)) * n * K;
  const long long blocks = (total + 255) / 256;
  m2m_kernel<<<static_cast<unsigned>(blocks), 256, pair_smem(n, n_pairs), s>>>(M, pair_off, pairs, coef, n, K,
                                                                              parent_level, n_pairs);
}

void launch_l2l(float *L, const int *pair_off, const int *pairs, const float *coef, int n, int K,
                int child_level, int n_pairs, cudaStream_t s) {
  const long long total = (static_cast<long long>(1) << (3 * child_level)) * n * K;
  const long long blocks = (total + 255) / 256;
  l2l_kernel<<<static_cast<unsigned>(blocks), 256, pair_smem(n, n_pairs), s>>>(L, pair_off, pairs, coef, n, K,
                                                                              child_level, n_pairs);
}

void launch_l2p(const float *L, const float4 *tgt_rel, const int *tgt_off, const int *tgt_perm,
                const float4 *near, int n, int p, int K, int nt, int depth, unsigned output,
                int layout, float phi_scale, float *field, float *potential, cudaStream_t s) {
  const int leaves = 1 << (3 * depth);
  const size_t smem = sizeof(float) * static_cast<size_t>(n) * K;
  l2p_kernel<<<leaves, 128, smem, s>>>(L, tgt_rel, tgt_off, tgt_perm, near, n, p, K, nt,
                                       level_offset_d(depth), output, layout, phi_scale, field,
                                       potential);
}

void configure_far_kernels(size_t max_smem) {
  allow_dynamic_smem(p2m_kernel, max_smem);
  allow_dynamic_smem(l2p_kernel, max_smem);
  allow_dynamic_smem(m2m_kernel, max_smem);
  allow_dynamic_smem(l2l_kernel, max_smem);
}

} // namespace cdfmm_b200
