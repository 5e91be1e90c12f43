// List-1 P2P near field (FP32) and the FP64 direct-sum reference kernel.
//
// Pair formula (upstream docs/math.md "Kernel, dipole potential, and field";
// src/operators.cpp:178-199), r = x_target - x_source:
//   phi += (m.r) / (4 pi |r|^3)
//   H   += [3 r (m.r) / |r|^5 - m / |r|^3] / (4 pi)
// The pair tensor is recomputed from positions in every evaluation instead of
// being stored per pair as the reference does (src/static_operators.cpp:405-470;
// 851.8M pairs at N = 1M would need ~30 GB FP32).  Positions are kept relative
// to their leaf centre, and the neighbour-leaf offset (an exact multiple of the
// leaf width) is added once per staged source, so |r| keeps FP32 precision
// relative to the leaf size rather than to the root box.
// Self exclusion is by sorted source index (never by coordinate equality); a
// coincident non-self pair produces NaN exactly as the reference's NaN tensor
// block does (src/static_operators.cpp:435-446).
#include <cuda_runtime.h>

#include <cmath>

#include "far_kernels.hpp"
#include "kernels.cuh"

namespace cdfmm_b200 {

namespace {

struct Neighbours {
  int count;
  int begin[27];
  int prefix[28];
  float sx[27], sy[27], sz[27];
};

// Builds the clipped 3x3x3 leaf neighbourhood of `leaf` (list1, upstream
// src/uniform_tree.cpp:455-480) with each neighbour's source range and the
// offset (neighbour centre - this centre) in normalised units.
__device__ void build_neighbours(Neighbours &nb, int leaf, int depth, const int *src_off) {
  int ix, iy, iz;
  demorton3(static_cast<uint32_t>(leaf), ix, iy, iz);
  const int side = 1 << depth;
  const float w = 1.0F / static_cast<float>(side);
  int c = 0;
  nb.prefix[0] = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        const int x = ix + dx, y = iy + dy, z = iz + dz;
        if (x < 0 || y < 0 || z < 0 || x >= side || y >= side || z >= side) continue;
        const uint32_t m = morton3(x, y, z);
        const int b = src_off[m];
        const int e = src_off[m + 1];
        if (e <= b) continue;
        nb.begin[c] = b;
        nb.sx[c] = static_cast<float>(dx) * w;
        nb.sy[c] = static_cast<float>(dy) * w;
        nb.sz[c] = static_cast<float>(dz) * w;
        nb.prefix[c + 1] = nb.prefix[c] + (e - b);
        ++c;
      }
  nb.count = c;
}

// Stages sources [g0, g0 + cnt) of the flattened neighbourhood: position
// relative to the target leaf centre and the sorted source index in .w.
__device__ inline void stage_source(const Neighbours &nb, int g, const float4 *src_rel,
                                    float4 &pos, int &j) {
  int b = 0;
  while (b + 1 < nb.count && nb.prefix[b + 1] <= g) ++b;
  j = nb.begin[b] + (g - nb.prefix[b]);
  const float4 d = src_rel[j];
  pos = make_float4(d.x + nb.sx[b], d.y + nb.sy[b], d.z + nb.sz[b], __int_as_float(j));
}

template <bool PHI>
__device__ __forceinline__ void pair_k1(const float4 &ti, int self, const float4 &s, const float4 &m,
                                        float &phi, float &hx, float &hy, float &hz) {
  const float dx = ti.x - s.x;
  const float dy = ti.y - s.y;
  const float dz = ti.z - s.z;
  float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  r2 = (__float_as_int(s.w) == self) ? __int_as_float(0x7f800000) : r2;
  const float rinv = rsqrtf(r2);
  const float rinv2 = rinv * rinv;
  const float rinv3 = rinv2 * rinv;
  const float mr = fmaf(m.x, dx, fmaf(m.y, dy, m.z * dz));
  if (PHI) phi = fmaf(mr, rinv3, phi);
  const float a = 3.0F * mr * rinv2;
  hx = fmaf(rinv3, fmaf(a, dx, -m.x), hx);
  hy = fmaf(rinv3, fmaf(a, dy, -m.y), hy);
  hz = fmaf(rinv3, fmaf(a, dz, -m.z), hz);
}

constexpr int kK1Chunk = 1024;
constexpr int kK1TargetChunk = 128;

// K = 1: one CTA per target leaf, all neighbour sources staged in shared
// memory; each warp owns 4 targets at a time, lanes stride over the staged
// sources and the partial sums are combined with warp shuffles.
template <bool PHI>
__global__ void __launch_bounds__(128) p2p_k1_kernel(const float4 *__restrict__ src_rel,
                                                     const float4 *__restrict__ mom,
                                                     const int *__restrict__ src_off,
                                                     const float4 *__restrict__ tgt_rel,
                                                     const int *__restrict__ tgt_off,
                                                     const int *__restrict__ self_idx, int depth,
                                                     float4 *__restrict__ near) {
  __shared__ float4 sPos[kK1Chunk];
  __shared__ float4 sMom[kK1Chunk];
  __shared__ float4 sAcc[kK1TargetChunk];
  __shared__ Neighbours nb;
  const int leaf = blockIdx.x;
  const int t0 = tgt_off[leaf];
  const int t1 = tgt_off[leaf + 1];
  if (t0 == t1) return;
  if (threadIdx.x == 0) build_neighbours(nb, leaf, depth, src_off);
  __syncthreads();
  const int total = nb.prefix[nb.count];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int tc = t0; tc < t1; tc += kK1TargetChunk) {
    const int tn = min(kK1TargetChunk, t1 - tc);
    for (int q = threadIdx.x; q < tn; q += blockDim.x) sAcc[q] = make_float4(0, 0, 0, 0);
    for (int sc = 0; sc < total; sc += kK1Chunk) {
      const int sn = min(kK1Chunk, total - sc);
      __syncthreads();
      for (int q = threadIdx.x; q < sn; q += blockDim.x) {
        float4 pos;
        int j;
        stage_source(nb, sc + q, src_rel, pos, j);
        sPos[q] = pos;
        sMom[q] = mom[j];
      }
      __syncthreads();
      for (int tb = warp * 4; tb < tn; tb += 16) {
        float4 ti[4];
        int self[4];
        float acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = tc + min(tb + u, tn - 1);
          ti[u] = tgt_rel[i];
          self[u] = self_idx != nullptr ? self_idx[i] : -1;
          acc[u][0] = acc[u][1] = acc[u][2] = acc[u][3] = 0.0F;
        }
        for (int q = lane; q < sn; q += 32) {
          const float4 s = sPos[q];
          const float4 m = sMom[q];
#pragma unroll
          for (int u = 0; u < 4; ++u) pair_k1<PHI>(ti[u], self[u], s, m, acc[u][0], acc[u][1], acc[u][2], acc[u][3]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int c = 0; c < 4; ++c)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[u][c] += __shfl_xor_sync(0xffffffffu, acc[u][c], o);
        if (lane == 0) {
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (tb + u < tn) {
              float4 a = sAcc[tb + u];
              a.x += acc[u][0];
              a.y += acc[u][1];
              a.z += acc[u][2];
              a.w += acc[u][3];
              sAcc[tb + u] = a;
            }
          }
        }
      }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < tn; q += blockDim.x) {
      const float4 a = sAcc[q];
      near[tc + q] = make_float4(a.x * kInvFourPiF, a.y * kInvFourPiF, a.z * kInvFourPiF, a.w * kInvFourPiF);
    }
    __syncthreads();
  }
}

// K > 1: a thread owns (target, group of KG states); per staged source the
// geometry is computed once and applied to the KG states.  Lanes of a warp
// share the state group, so moment reads are shared-memory broadcasts.
template <int KG, bool PHI>
__global__ void __launch_bounds__(256) p2p_kn_kernel(const float4 *__restrict__ src_rel,
                                                     const float4 *__restrict__ mom,
                                                     const int *__restrict__ src_off,
                                                     const float4 *__restrict__ tgt_rel,
                                                     const int *__restrict__ tgt_off,
                                                     const int *__restrict__ self_idx, int depth,
                                                     int K, int chunk, float4 *__restrict__ near) {
  extern __shared__ float4 dyn[];
  float4 *sPos = dyn;          // [chunk]
  float4 *sMom = dyn + chunk;  // [chunk][K]
  __shared__ Neighbours nb;
  const int leaf = blockIdx.x;
  const int t0 = tgt_off[leaf];
  const int t1 = tgt_off[leaf + 1];
  if (t0 == t1) return;
  if (threadIdx.x == 0) build_neighbours(nb, leaf, depth, src_off);
  __syncthreads();
  const int total = nb.prefix[nb.count];
  const int nt_leaf = t1 - t0;
  const int groups = (K + KG - 1) / KG;
  const int items = nt_leaf * groups;
  for (int base = 0; base < items; base += blockDim.x) {
    const int item = base + threadIdx.x;
    const bool active = item < items;
    const int g = active ? item / nt_leaf : 0;
    const int i = t0 + (active ? item - g * nt_leaf : 0);
    const int kb = g * KG;
    const float4 ti = tgt_rel[i];
    const int self = self_idx != nullptr ? self_idx[i] : -1;
    float acc[KG][4];
#pragma unroll
    for (int s = 0; s < KG; ++s) acc[s][0] = acc[s][1] = acc[s][2] = acc[s][3] = 0.0F;
    for (int sc = 0; sc < total; sc += chunk) {
      const int sn = min(chunk, total - sc);
      __syncthreads();
      for (int q = threadIdx.x; q < sn; q += blockDim.x) {
        float4 pos;
        int j;
        stage_source(nb, sc + q, src_rel, pos, j);
        sPos[q] = pos;
      }
      __syncthreads();
      for (int q = threadIdx.x; q < sn * K; q += blockDim.x) {
        const int qs = q / K;
        const int k = q - qs * K;
        sMom[q] = mom[static_cast<long long>(__float_as_int(sPos[qs].w)) * K + k];
      }
      __syncthreads();
      if (active) {
        for (int q = 0; q < sn; ++q) {
          const float4 s = sPos[q];
          const float dx = ti.x - s.x;
          const float dy = ti.y - s.y;
          const float dz = ti.z - s.z;
          float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
          r2 = (__float_as_int(s.w) == self) ? __int_as_float(0x7f800000) : r2;
          const float rinv = rsqrtf(r2);
          const float rinv2 = rinv * rinv;
          const float rinv3 = rinv2 * rinv;
          const float a3 = 3.0F * rinv2;
          const float4 *mq = sMom + q * K + kb;
#pragma unroll
          for (int s2 = 0; s2 < KG; ++s2) {
            if (kb + s2 < K) {
              const float4 m = mq[s2];
              const float mr = fmaf(m.x, dx, fmaf(m.y, dy, m.z * dz));
              if (PHI) acc[s2][0] = fmaf(mr, rinv3, acc[s2][0]);
              const float a = a3 * mr;
              acc[s2][1] = fmaf(rinv3, fmaf(a, dx, -m.x), acc[s2][1]);
              acc[s2][2] = fmaf(rinv3, fmaf(a, dy, -m.y), acc[s2][2]);
              acc[s2][3] = fmaf(rinv3, fmaf(a, dz, -m.z), acc[s2][3]);
            }
          }
        }
      }
    }
    if (active) {
#pragma unroll
      for (int s2 = 0; s2 < KG; ++s2) {
        if (kb + s2 < K) {
          near[static_cast<long long>(i) * K + kb + s2] =
              make_float4(acc[s2][0] * kInvFourPiF, acc[s2][1] * kInvFourPiF,
                          acc[s2][2] * kInvFourPiF, acc[s2][3] * kInvFourPiF);
        }
      }
    }
    __syncthreads();
  }
}

// FP64 O(N*M) direct sum, one thread per target, sources tiled through
// shared memory (upstream validation.cpp:71-111; cuda_fmm.cu:518-569).
__global__ void __launch_bounds__(256) direct_fp64_kernel(const double *__restrict__ src,
                                                          const double *__restrict__ mom, int ns,
                                                          const double *__restrict__ tgt, int nt,
                                                          const int *__restrict__ self,
                                                          double *__restrict__ phi,
                                                          double *__restrict__ field) {
  __shared__ double sp[256][3];
  __shared__ double sm[256][3];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < nt;
  double x = 0, y = 0, z = 0;
  int me = -1;
  if (active) {
    x = tgt[3 * i];
    y = tgt[3 * i + 1];
    z = tgt[3 * i + 2];
    me = self != nullptr ? self[i] : -1;
  }
  double p = 0, hx = 0, hy = 0, hz = 0;
  for (int s0 = 0; s0 < ns; s0 += 256) {
    const int cnt = min(256, ns - s0);
    __syncthreads();
    for (int q = threadIdx.x; q < cnt; q += blockDim.x) {
      for (int c = 0; c < 3; ++c) {
        sp[q][c] = src[3 * (s0 + q) + c];
        sm[q][c] = mom[3 * (s0 + q) + c];
      }
    }
    __syncthreads();
    if (active) {
      for (int q = 0; q < cnt; ++q) {
        if (s0 + q == me) continue;
        const double rx = x - sp[q][0], ry = y - sp[q][1], rz = z - sp[q][2];
        const double r2 = rx * rx + ry * ry + rz * rz;
        const double rinv = 1.0 / sqrt(r2);
        const double rinv3 = rinv * rinv * rinv;
        const double mr = sm[q][0] * rx + sm[q][1] * ry + sm[q][2] * rz;
        p += mr * rinv3;
        const double f = 3.0 * mr * rinv3 * rinv * rinv;
        hx += rx * f - sm[q][0] * rinv3;
        hy += ry * f - sm[q][1] * rinv3;
        hz += rz * f - sm[q][2] * rinv3;
      }
    }
  }
  if (active) {
    const double c = 1.0 / (4.0 * 3.14159265358979323846);
    if (phi != nullptr) phi[i] = p * c;
    if (field != nullptr) {
      field[3 * i] = hx * c;
      field[3 * i + 1] = hy * c;
      field[3 * i + 2] = hz * c;
    }
  }
}

template <int KG>
void launch_kn(const float4 *src_rel, const float4 *mom, const int *src_off, const float4 *tgt_rel,
               const int *tgt_off, const int *self_idx, int depth, int K, bool want_phi,
               float4 *near, cudaStream_t s) {
  const int leaves = 1 << (3 * depth);
  int chunk = static_cast<int>((96 * 1024) / (16 + 16 * static_cast<size_t>(K)));
  chunk = std::max(8, std::min(256, chunk));
  const size_t smem = sizeof(float4) * (static_cast<size_t>(chunk) + static_cast<size_t>(chunk) * K);
  if (want_phi)
    p2p_kn_kernel<KG, true><<<leaves, 256, smem, s>>>(src_rel, mom, src_off, tgt_rel, tgt_off, self_idx, depth, K, chunk, near);
  else
    p2p_kn_kernel<KG, false><<<leaves, 256, smem, s>>>(src_rel, mom, src_off, tgt_rel, tgt_off, self_idx, depth, K, chunk, near);
}

} // namespace

void launch_p2p(const float4 *src_rel, const float4 *mom, const int *src_off,
                const float4 *tgt_rel, const int *tgt_off, const int *self_idx, int depth, int K,
                bool want_phi, float4 *near, cudaStream_t s) {
  const int leaves = 1 << (3 * depth);
  if (K == 1) {
    if (want_phi)
      p2p_k1_kernel<true><<<leaves, 128, 0, s>>>(src_rel, mom, src_off, tgt_rel, tgt_off, self_idx, depth, near);
    else
      p2p_k1_kernel<false><<<leaves, 128, 0, s>>>(src_rel, mom, src_off, tgt_rel, tgt_off, self_idx, depth, near);
  } else if (K >= 8) {
    launch_kn<8>(src_rel, mom, src_off, tgt_rel, tgt_off, self_idx, depth, K, want_phi, near, s);
  } else {
    launch_kn<4>(src_rel, mom, src_off, tgt_rel, tgt_off, self_idx, depth, K, want_phi, near, s);
  }
}

void configure_p2p(size_t max_smem) {
  allow_dynamic_smem(p2p_kn_kernel<8, true>, max_smem);
  allow_dynamic_smem(p2p_kn_kernel<8, false>, max_smem);
  allow_dynamic_smem(p2p_kn_kernel<4, true>, max_smem);
  allow_dynamic_smem(p2p_kn_kernel<4, false>, max_smem);
}

void launch_direct_fp64(const double *src, const double *mom, int ns, const double *tgt, int nt,
                        const int *self, double *phi, double *field, cudaStream_t s) {
  if (nt == 0) return;
  direct_fp64_kernel<<<(nt + 255) / 256, 256, 0, s>>>(src, mom, ns, tgt, nt, self, phi, field);
}

} // namespace cdfmm_b200
