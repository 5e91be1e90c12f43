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
// (upstream src/far_field.cpp:248-275, src/cuda_fmm.cu:56-64).  A CTA takes
// 32 consecutive user indices and 32 states at a time through a shared tile:
// the reads are contiguous runs of each state's user array, the writes
// contiguous runs of each sorted row (inv = user -> sorted index).
template <typename T>
__global__ void __launch_bounds__(256) gather_moments_kernel(const T *__restrict__ user, const int *__restrict__ inv,
                                                             int ns, int K, double inv_scale, float inv_scale3_f,
                                                             bool paired, float4 *__restrict__ mom, int k0,
                                                             int krow) {
  __shared__ float tile[32][32 * 3 + 1]; // [user][state * 3 + component]
  const int u0 = blockIdx.x * 32;
  const int nu = min(32, ns - u0);
  for (int kc = 0; kc < K; kc += 32) {
    const int kn = min(32, K - kc);
    for (int e = threadIdx.x; e < kn * nu * 3; e += blockDim.x) {
      const int k = e / (nu * 3);
      const int r = e - k * nu * 3;
      const int t = r / 3;
      const T v = user[(static_cast<long long>(kc + k) * ns + u0) * 3 + r];
      float f;
      if constexpr (sizeof(T) == 8)
        f = static_cast<float>(static_cast<double>(v) * inv_scale * inv_scale * inv_scale); // m / s / s / s in FP64
      else
        f = static_cast<float>(v) * inv_scale3_f;
      tile[t][3 * k + (r - 3 * t)] = f;
    }
    __syncthreads();
    if (paired) {
      // state pairs (k, k+1) as (x_k, x_k1, y_k, y_k1), (z_k, z_k1, 0, 0); a
      // missing partner (K odd) is zero
      const int kp = (kn + 1) >> 1;
      const int row = krow;
      for (int e = threadIdx.x; e < nu * kp; e += blockDim.x) {
        const int t = e / kp;
        const int k = 2 * (e - t * kp);
        const bool b = k + 1 < kn;
        float4 *dst = mom + static_cast<long long>(inv[u0 + t]) * row + k0 + kc + k;
        dst[0] = make_float4(tile[t][3 * k], b ? tile[t][3 * k + 3] : 0.0F, tile[t][3 * k + 1],
                             b ? tile[t][3 * k + 4] : 0.0F);
        dst[1] = make_float4(tile[t][3 * k + 2], b ? tile[t][3 * k + 5] : 0.0F, 0.0F, 0.0F);
      }
    } else {
      for (int e = threadIdx.x; e < nu * kn; e += blockDim.x) {
        const int t = e / kn;
        const int k = e - t * kn;
        mom[static_cast<long long>(inv[u0 + t]) * krow + k0 + kc + k] =
            make_float4(tile[t][3 * k], tile[t][3 * k + 1], tile[t][3 * k + 2], 0.0F);
      }
    }
    __syncthreads();
  }
}

// Cuboid sources (upstream docs/math.md "Finite cuboid geometry";
// src/static_operators.cpp:222-255): the point monomial d^mu/mu! is replaced
// by its average over the source cuboid (side lengths h centred at d),
// J_mu(d, h) = prod over axes of j(mu_axis), where per axis
//   j(a) = sum_{g even <= a} d^(a-g)/(a-g)! * (h/2)^g/(g+1)!
// (the average of (d+u)^a/a! over u in [-h/2, h/2]).  q <= 9.
__device__ inline void cuboid_axis(float d, float h, int q, float (&j)[10]) {
  float pw[10], c[10];
  pw[0] = 1.0F;
  c[0] = 1.0F;
  c[1] = 0.0F;
  const float hh = 0.25F * h * h;
#pragma unroll
  for (int i = 1; i < 10; ++i) pw[i] = i <= q ? pw[i - 1] * d * kInvInt[i] : 0.0F;
#pragma unroll
  for (int g = 2; g < 10; ++g) c[g] = (g & 1) ? 0.0F : c[g - 2] * hh * kInvInt[g] * kInvInt[g + 1];
#pragma unroll
  for (int a = 0; a < 10; ++a) {
    float v = 0.0F;
#pragma unroll
    for (int g = 0; g <= a; g += 2) v = fmaf(pw[a - g], c[g], v);
    j[a] = v;
  }
}

// The cuboid-averaged monomials of x-degree a in part r of 4 (the split of
// monomials_part), or all of them for r < 0.
__device__ inline void cuboid_monomials_part(float dx, float dy, float dz, float4 h, int q, float *out, int r) {
  float jx[10], jy[10], jz[10];
  cuboid_axis(dx, h.x, q, jx);
  cuboid_axis(dy, h.y, q, jy);
  cuboid_axis(dz, h.z, q, jz);
  for (int a = 0; a <= q; ++a) {
    if (r >= 0) {
      const int m8 = a & 7;
      if (m8 != r && m8 != 7 - r) continue;
    }
    float xa = 0.0F;
#pragma unroll
    for (int i = 0; i < 10; ++i) xa = i == a ? jx[i] : xa;
    for (int b = 0; a + b <= q; ++b) {
      float yb = 0.0F;
#pragma unroll
      for (int i = 0; i < 10; ++i) yb = i == b ? jy[i] : yb;
      const float xy = xa * yb;
#pragma unroll
      for (int c = 0; c < 10; ++c)
        if (a + b + c <= q) out[rank3(a, b, c)] = xy * jz[c];
    }
  }
}

// ---------------------------------------------------------------------------
// P2M (upstream docs/math.md P2M; src/static_operators.cpp:186-220):
//   M_alpha = (-1)^|alpha| sum_j sum_{k: alpha_k > 0} m_jk d_j^(alpha-e_k)/(alpha-e_k)!
// computed per leaf as three small GEMMs
//   P_c[mu][s] = sum_j m_jcs d_j^mu / mu!        (|mu| <= p-1, s = state)
//   M_alpha[s] = (-1)^|alpha| sum_{c: alpha_c > 0} P_c[alpha - e_c][s].
// One CTA per leaf.  Sources are staged in chunks (monomials [j][mu] and
// moments [j][s]); a thread owns a register tile of 4 consecutive mu x 4
// states (s = kb, kb + Kq, ...; consecutive lanes take consecutive kb, so the
// float4 moment loads are conflict-free and the monomial quad a broadcast)
// and adds it into P in shared memory after each chunk.  States are handled
// in blocks of Kb so P fits in shared memory for any K.
constexpr int kP2mThreads = 256;
constexpr int kP2mChunk = 32;

// Few states (K < 4): one thread per (alpha, state) accumulator, sources
// staged in chunks with their monomials (the register tiles below would
// leave most lanes idle).
__global__ void __launch_bounds__(128) p2m_small_kernel(const float4 *__restrict__ src_rel,
                                                        const float4 *__restrict__ mom,
                                                        const int *__restrict__ src_off,
                                                        const int8_t *__restrict__ basis, float *__restrict__ M,
                                                        int n, int p, int K, int leaf_node_base,
                                                        const float4 *__restrict__ size, int size_step) {
  __shared__ float mono[kP2mChunk * 220];
  __shared__ float4 smom[kP2mChunk * 3];
  const int nm1 = basis_size_d(p - 1);
  const int leaf = blockIdx.x;
  const int s0 = src_off[leaf];
  const int s1 = src_off[leaf + 1];
  const int items = n * K;
  float *out = M + static_cast<long long>(leaf_node_base + leaf) * items;
  for (int base = 0; base < items; base += blockDim.x) {
    const int q = base + threadIdx.x;
    const bool valid = q < items;
    const int a = valid ? q / K : 0;
    const int k = valid ? q - a * K : 0;
    const int ax = basis[4 * a], ay = basis[4 * a + 1], az = basis[4 * a + 2];
    const int ix = ax > 0 ? rank3(ax - 1, ay, az) : -1;
    const int iy = ay > 0 ? rank3(ax, ay - 1, az) : -1;
    const int iz = az > 0 ? rank3(ax, ay, az - 1) : -1;
    float v = 0.0F;
    for (int c0 = s0; c0 < s1; c0 += kP2mChunk) {
      const int cn = min(kP2mChunk, s1 - c0);
      __syncthreads();
      for (int j = threadIdx.x; j < cn; j += blockDim.x) {
        const float4 d = src_rel[c0 + j];
        if (nm1 > 0) {
          if (size != nullptr)
            cuboid_monomials_part(d.x, d.y, d.z, size[(c0 + j) * size_step], p - 1, mono + j * nm1, -1);
          else
            monomials(d.x, d.y, d.z, p - 1, mono + j * nm1);
        }
      }
      for (int e = threadIdx.x; e < cn * K; e += blockDim.x) smom[e] = mom[static_cast<long long>(c0) * K + e];
      __syncthreads();
      if (valid) {
        for (int j = 0; j < cn; ++j) {
          const float4 m = smom[j * K + k];
          const float *mj = mono + j * nm1;
          if (ix >= 0) v = fmaf(m.x, mj[ix], v);
          if (iy >= 0) v = fmaf(m.y, mj[iy], v);
          if (iz >= 0) v = fmaf(m.z, mj[iz], v);
        }
      }
    }
    if (valid) out[q] = ((ax + ay + az) & 1) ? -v : v;
  }
}

__global__ void __launch_bounds__(kP2mThreads) p2m_kernel(const float4 *__restrict__ src_rel,
                                                          const float4 *__restrict__ mom,
                                                          const int *__restrict__ src_off,
                                                          const int8_t *__restrict__ basis, float *__restrict__ M,
                                                          int n, int p, int K, int leaf_node_base, int Kb,
                                                          const float4 *__restrict__ size, int size_step) {
  extern __shared__ float4 p2m_smem[];
  const int nm1 = basis_size_d(p - 1);
  const int nm1p = (nm1 + 3) & ~3;
  float4 *smom = p2m_smem;                                              // [chunk][Kc]
  float *P = reinterpret_cast<float *>(smom + kP2mChunk * Kb);          // [3][nm1p][Kc + 2]
  float *mono = P + 3 * nm1p * (Kb + 2);                                // [chunk][nm1p]
  short *sidx = reinterpret_cast<short *>(mono + kP2mChunk * nm1p);     // [n][4] P rows of alpha - e_c (-1: none), sign
  const int tid = threadIdx.x;
  const int leaf = blockIdx.x;
  const int s0 = src_off[leaf];
  const int s1 = src_off[leaf + 1];
  float *out = M + static_cast<long long>(leaf_node_base + leaf) * n * K;
  // the P rows each output coefficient combines (once per CTA)
  for (int a = tid; a < n; a += blockDim.x) {
    const int ax = basis[4 * a], ay = basis[4 * a + 1], az = basis[4 * a + 2];
    sidx[4 * a] = static_cast<short>(ax > 0 ? rank3(ax - 1, ay, az) : -1);
    sidx[4 * a + 1] = static_cast<short>(ay > 0 ? nm1p + rank3(ax, ay - 1, az) : -1);
    sidx[4 * a + 2] = static_cast<short>(az > 0 ? 2 * nm1p + rank3(ax, ay, az - 1) : -1);
    sidx[4 * a + 3] = static_cast<short>(((ax + ay + az) & 1) ? -1 : 1);
  }
  for (int kblk = blockIdx.y * Kb; kblk < K; kblk += Kb * gridDim.y) {
    const int Kc = min(Kb, K - kblk);
    const int Kq = (Kc + 3) >> 2;
    // P row stride Kc + 2: the 4 monomial quads of a warp's tile updates
    // fall in different banks
    const int Ps = Kc + 2;
    const int tiles = (nm1p >> 2) * Kq;
    for (int q = tid; q < 3 * nm1p * Ps; q += blockDim.x) P[q] = 0.0F;
    for (int c0 = s0; c0 < s1; c0 += kP2mChunk) {
      const int cn = min(kP2mChunk, s1 - c0);
      __syncthreads();
      // four threads per source (consecutive lanes: consecutive sources, one part)
      for (int w = tid; w < 4 * cn; w += blockDim.x) {
        const int r = w / cn;
        const int j = w - r * cn;
        const float4 d = src_rel[c0 + j];
        if (nm1 > 0) {
          if (size != nullptr)
            cuboid_monomials_part(d.x, d.y, d.z, size[(c0 + j) * size_step], p - 1, mono + j * nm1p, r);
          else
            monomials_part(d.x, d.y, d.z, p - 1, mono + j * nm1p, 1, r, false);
        }
        if (r == 0)
          for (int q = nm1; q < nm1p; ++q) mono[j * nm1p + q] = 0.0F;
      }
      {
        // paired layout (K >= 4): states (2i, 2i+1) share two float4
        // (x, x', y, y'), (z, z', 0, 0).  A thread loads whole pairs (each
        // pair read once) in batches of 4 pairs whose loads are all issued
        // before the shared-memory stores that consume them.
        const int pp0 = kblk >> 1;
        const int npair = ((kblk + Kc - 1) >> 1) - pp0 + 1;
        const int np = cn * npair;
        const long long row_len = (K + 1) & ~1;
        for (int q0 = tid; q0 < np; q0 += 4 * blockDim.x) {
          float4 A[4], B[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int q = q0 + u * blockDim.x;
            if (q < np) {
              const int j = q / npair;
              const float4 *pr = mom + (c0 + j) * row_len + 2 * (pp0 + q - j * npair);
              A[u] = pr[0];
              B[u] = pr[1];
            }
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int q = q0 + u * blockDim.x;
            if (q < np) {
              const int j = q / npair;
              const int s0 = 2 * (pp0 + q - j * npair) - kblk; // state of the pair's first half, block-relative
              if (s0 >= 0) smom[j * Kc + s0] = make_float4(A[u].x, A[u].z, B[u].x, 0.0F);
              if (s0 + 1 < Kc) smom[j * Kc + s0 + 1] = make_float4(A[u].y, A[u].w, B[u].y, 0.0F);
            }
          }
        }
      }
      __syncthreads();
      for (int t = tid; t < tiles; t += blockDim.x) {
        const int mb = t / Kq;
        const int kb = t - mb * Kq;
        const int mu0 = mb * 4;
        // acc[c][u pair][kk]: packed FP32x2 FMAs over pairs of monomials
        float2 acc[3][2][4];
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
          for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) acc[c][u][kk] = make_float2(0.0F, 0.0F);
        for (int j = 0; j < cn; ++j) {
          const float4 mo = *reinterpret_cast<const float4 *>(mono + j * nm1p + mu0);
          const float2 m01 = make_float2(mo.x, mo.y), m23 = make_float2(mo.z, mo.w);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const int k = kb + kk * Kq;
            const float4 m = k < Kc ? smom[j * Kc + k] : make_float4(0, 0, 0, 0);
            const float2 X = make_float2(m.x, m.x), Y = make_float2(m.y, m.y), Z = make_float2(m.z, m.z);
            acc[0][0][kk] = __ffma2_rn(m01, X, acc[0][0][kk]);
            acc[0][1][kk] = __ffma2_rn(m23, X, acc[0][1][kk]);
            acc[1][0][kk] = __ffma2_rn(m01, Y, acc[1][0][kk]);
            acc[1][1][kk] = __ffma2_rn(m23, Y, acc[1][1][kk]);
            acc[2][0][kk] = __ffma2_rn(m01, Z, acc[2][0][kk]);
            acc[2][1][kk] = __ffma2_rn(m23, Z, acc[2][1][kk]);
          }
        }
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const int k = kb + kk * Kq;
          if (k < Kc) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
              for (int u = 0; u < 4; ++u)
                P[(c * nm1p + mu0 + u) * Ps + k] += (u & 1) ? acc[c][u >> 1][kk].y : acc[c][u >> 1][kk].x;
          }
        }
      }
    }
    __syncthreads();
    for (int q = tid; q < n * Kc; q += blockDim.x) {
      const int a = q / Kc;
      const int k = q - a * Kc;
      const short *ix = sidx + 4 * a;
      float v = 0.0F;
      if (ix[0] >= 0) v += P[ix[0] * Ps + k];
      if (ix[1] >= 0) v += P[ix[1] * Ps + k];
      if (ix[2] >= 0) v += P[ix[2] * Ps + k];
      out[static_cast<long long>(a) * K + kblk + k] = ix[3] < 0 ? -v : v;
    }
    __syncthreads();
  }
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

// M2M, one CTA per (parent, block of Ks states): the 8 children's
// multipoles of the block are staged in shared memory ([child][coef][state],
// rows of Ks), then a thread forms one parent coefficient for 4
// consecutive states: per (child, pair) one class coefficient, one pair entry
// and one float4 of staged multipoles feed 4 FMAs.  Lanes of a warp take
// consecutive state quads of the same coefficient (conflict-free float4
// loads, broadcast pair/coefficient loads).
constexpr int kShiftThreads = 256;

__device__ __forceinline__ void store_quad(float *dst, const float4 &v, int valid, bool add) {
  const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
  for (int j = 0; j < 4; ++j)
    if (j < valid) dst[j] = add ? dst[j] + e[j] : e[j];
}

__global__ void __launch_bounds__(kShiftThreads) m2m_kernel(float *__restrict__ M, const int *__restrict__ pair_off,
                                                            const int *__restrict__ pairs,
                                                            const float *__restrict__ coef, int n, int K,
                                                            int parent_level, int n_pairs, int Ks) {
  extern __shared__ float4 shp4[];
  float *sM = reinterpret_cast<float *>(shp4);                  // [8 children][n][Ks]
  float *scoef = sM + 8 * n * Ks;                     // [8][n]
  int *soff = reinterpret_cast<int *>(scoef + 8 * n);
  int *spair = soff + n + 1;
  stage_pairs(pair_off, pairs, coef + static_cast<long long>(parent_level + 1) * 8 * n, n, n_pairs, soff, spair,
              scoef);
  const long long parent = blockIdx.x;
  const int kb = blockIdx.y * Ks;
  const int kc = min(Ks, K - kb);
  const int nq = (kc + 3) >> 2;
  const long long per = static_cast<long long>(n) * K;
  const float *child0 = M + (level_offset_d(parent_level + 1) + parent * 8) * per + kb;
  const int qpr = Ks >> 2; // float4 quads per staged row
  if ((K & 3) == 0) {
    // rows of 4-aligned states: one asynchronous 16-byte copy per quad (all
    // of a thread's copies in flight at once), one division per quad
    for (int q = threadIdx.x; q < 8 * n * qpr; q += kShiftThreads) {
      const int cr = q / qpr; // child * n + coefficient
      const int kq = q - cr * qpr;
      const int c = cr / n;
      if (4 * kq < kc)
        cp_async16(reinterpret_cast<float4 *>(sM) + q, child0 + c * per + static_cast<long long>(cr - c * n) * K + 4 * kq);
      else
        reinterpret_cast<float4 *>(sM)[q] = make_float4(0, 0, 0, 0);
    }
    cp_async_commit();
    cp_async_wait<0>();
  } else {
    for (int q = threadIdx.x; q < 8 * n * Ks; q += kShiftThreads) {
      const int cr = q / Ks;
      const int k = q - cr * Ks;
      sM[q] = k < kc ? child0[(cr / n) * per + static_cast<long long>(cr % n) * K + k] : 0.0F;
    }
  }
  __syncthreads();
  float *out = M + (level_offset_d(parent_level) + parent) * per + kb;
  for (int q = threadIdx.x; q < n * nq; q += kShiftThreads) {
    const int a = q / nq;
    const int kq = q - a * nq;
    const int e0 = soff[a], e1 = soff[a + 1];
    float4 v = make_float4(0, 0, 0, 0);
    for (int c = 0; c < 8; ++c) {
      const float *cc = scoef + c * n;
      const float *mc = sM + c * n * Ks + 4 * kq;
      for (int e = e0; e < e1; ++e) {
        const int pr = spair[e];
        const float w = cc[pr & 0xffff];
        const float4 m = *reinterpret_cast<const float4 *>(mc + (pr >> 16) * Ks);
        v.x = fmaf(w, m.x, v.x);
        v.y = fmaf(w, m.y, v.y);
        v.z = fmaf(w, m.z, v.z);
        v.w = fmaf(w, m.w, v.w);
      }
    }
    store_quad(out + static_cast<long long>(a) * K + 4 * kq, v, kc - 4 * kq, false);
  }
}

// ---------------------------------------------------------------------------
// L2L for one child level (upstream src/far_field.cpp:533-581):
//   L_child[beta] += sum_{|beta + g| <= p} B_class[g] L_parent[beta + g]
// One CTA per (parent, block of states): the parent's locals are staged once
// and shifted to its 8 children; a thread adds one child coefficient for 4
// consecutive states.
__global__ void __launch_bounds__(kShiftThreads) l2l_kernel(float *__restrict__ L, const int *__restrict__ pair_off,
                                                            const int *__restrict__ pairs,
                                                            const float *__restrict__ coef, int n, int K,
                                                            int child_level, int n_pairs, int Ks) {
  extern __shared__ float4 shl4[];
  float *sL = reinterpret_cast<float *>(shl4);                  // [n][Ks]
  float *scoef = sL + n * Ks;                         // [8][n]
  int *soff = reinterpret_cast<int *>(scoef + 8 * n);
  int *spair = soff + n + 1;
  stage_pairs(pair_off, pairs, coef + static_cast<long long>(child_level) * 8 * n, n, n_pairs, soff, spair, scoef);
  const long long parent = blockIdx.x;
  const int kb = blockIdx.y * Ks;
  const int kc = min(Ks, K - kb);
  const int nq = (kc + 3) >> 2;
  const long long per = static_cast<long long>(n) * K;
  const float *src = L + (level_offset_d(child_level - 1) + parent) * per + kb;
  const int qpr = Ks >> 2;
  if ((K & 3) == 0) {
    for (int q = threadIdx.x; q < n * qpr; q += kShiftThreads) {
      const int b = q / qpr;
      const int kq = q - b * qpr;
      if (4 * kq < kc)
        cp_async16(reinterpret_cast<float4 *>(sL) + q, src + static_cast<long long>(b) * K + 4 * kq);
      else
        reinterpret_cast<float4 *>(sL)[q] = make_float4(0, 0, 0, 0);
    }
    cp_async_commit();
    cp_async_wait<0>();
  } else {
    for (int q = threadIdx.x; q < n * Ks; q += kShiftThreads) {
      const int b = q / Ks;
      const int k = q - b * Ks;
      sL[q] = k < kc ? src[static_cast<long long>(b) * K + k] : 0.0F;
    }
  }
  __syncthreads();
  float *child0 = L + (level_offset_d(child_level) + parent * 8) * per + kb;
  for (int q = threadIdx.x; q < 8 * n * nq; q += kShiftThreads) {
    const int cr = q / nq; // child * n + coefficient
    const int kq = q - cr * nq;
    const int c = cr / n;
    const int b = cr - c * n;
    const float *cc = scoef + c * n;
    float4 v = make_float4(0, 0, 0, 0);
    for (int e = soff[b]; e < soff[b + 1]; ++e) {
      const int pr = spair[e];
      const float w = cc[pr & 0xffff];
      const float4 l = *reinterpret_cast<const float4 *>(sL + (pr >> 16) * Ks + 4 * kq);
      v.x = fmaf(w, l.x, v.x);
      v.y = fmaf(w, l.y, v.y);
      v.z = fmaf(w, l.z, v.z);
      v.w = fmaf(w, l.w, v.w);
    }
    store_quad(child0 + c * per + static_cast<long long>(b) * K + 4 * kq, v, kc - 4 * kq, true);
  }
}

// ---------------------------------------------------------------------------
// L2P + combine (upstream docs/math.md L2P; src/cuda_fmm.cu:503-516):
//   phi = sum_b L_b dx^b/b!,  H_c = -sum_{|mu| <= p-1} L_{mu+e_c} dx^mu/mu!
// then result = far + near (near from the P2P kernel), phi times the root
// width, written back over near[target][state] (sorted order); the unsort
// kernel below moves it to user order with contiguous writes.  (Writing user
// order here would scatter 4-byte stores over the whole output.)  One CTA
// per leaf; the leaf's
// local expansion (n x Kc states, a state block) and the monomials of up to
// 32 targets ([b][t]) are staged in shared memory; a thread owns a register
// tile of 4 targets x 4 consecutive states, reading float4 quads of both
// (consecutive lanes take consecutive state quads of the same target quad:
// conflict-free L loads, broadcast monomial loads).
constexpr int kL2pThreads = 128;
constexpr int kL2pTargets = 32;
static_assert(kL2pThreads == 4 * kL2pTargets, "L2P monomials: four threads per target");

// One pass of L2P register tiles over a staged target chunk: tile =
// (TU consecutive targets, 4 consecutive states).
template <int TU>
__device__ __forceinline__ void l2p_tiles(int tid, int tn, int Kq, int Kcp, int Kc, int n, int nm1,
                                          const float *mono, const float *sL, const short *sidx, bool want_phi,
                                          bool want_h, float4 *__restrict__ near, int tc, int kblk, int K,
                                          float phi_scale, int k_near_end) {
  const int tiles = ((tn + TU - 1) / TU) * Kq;
  for (int tile = tid; tile < tiles; tile += kL2pThreads) {
    const int tq = tile / Kq;
    const int kq = tile - tq * Kq;
    float ph[TU][4], hx[TU][4], hy[TU][4], hz[TU][4];
#pragma unroll
    for (int u = 0; u < TU; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) ph[u][v] = hx[u][v] = hy[u][v] = hz[u][v] = 0.0F;
    const float *mq = mono + TU * tq;
    const float *lq = sL + 4 * kq;
    auto load_mono = [&](int b, float (&mv)[TU]) {
      if constexpr (TU == 4) {
        const float4 mo = *reinterpret_cast<const float4 *>(mq + b * kL2pTargets);
        mv[0] = mo.x;
        mv[1] = mo.y;
        mv[2] = mo.z;
        mv[3] = mo.w;
      } else if constexpr (TU == 2) {
        const float2 mo = *reinterpret_cast<const float2 *>(mq + b * kL2pTargets);
        mv[0] = mo.x;
        mv[1] = mo.y;
      } else {
        mv[0] = mq[b * kL2pTargets];
      }
    };
    if (want_phi) {
      for (int b = 0; b < n; ++b) {
        float mv[TU];
        load_mono(b, mv);
        const float4 l = *reinterpret_cast<const float4 *>(lq + b * Kcp);
        const float lv[4] = {l.x, l.y, l.z, l.w};
#pragma unroll
        for (int u = 0; u < TU; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) ph[u][v] = fmaf(mv[u], lv[v], ph[u][v]);
      }
    }
    if (want_h) {
      for (int mu = 0; mu < nm1; ++mu) {
        float mv[TU];
        load_mono(mu, mv);
        const float4 lx = *reinterpret_cast<const float4 *>(lq + sidx[3 * mu] * Kcp);
        const float4 ly = *reinterpret_cast<const float4 *>(lq + sidx[3 * mu + 1] * Kcp);
        const float4 lz = *reinterpret_cast<const float4 *>(lq + sidx[3 * mu + 2] * Kcp);
        const float xv[4] = {lx.x, lx.y, lx.z, lx.w};
        const float yv[4] = {ly.x, ly.y, ly.z, ly.w};
        const float zv[4] = {lz.x, lz.y, lz.z, lz.w};
#pragma unroll
        for (int u = 0; u < TU; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            hx[u][v] = fmaf(mv[u], xv[v], hx[u][v]);
            hy[u][v] = fmaf(mv[u], yv[v], hy[u][v]);
            hz[u][v] = fmaf(mv[u], zv[v], hz[u][v]);
          }
      }
    }
    // Combine with the near field: each target's 4 near values are loaded
    // together (one batch of independent loads per target, not one
    // load-store round trip per value), then written back.
#pragma unroll
    for (int u = 0; u < TU; ++u) {
      const int t = TU * tq + u;
      const int i = tc + t;
      float4 nv[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int kl = 4 * kq + v;
        // states from k_near_end on have no near field yet (it is added later)
        nv[v] = (t < tn && kl < Kc && kblk + kl < k_near_end) ? near[static_cast<long long>(i) * K + kblk + kl]
                                                              : make_float4(0, 0, 0, 0);
      }
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int kl = 4 * kq + v;
        if (t < tn && kl < Kc)
          near[static_cast<long long>(i) * K + kblk + kl] =
              make_float4(want_phi ? (ph[u][v] + nv[v].x) * phi_scale : 0.0F, want_h ? nv[v].y - hx[u][v] : 0.0F,
                          want_h ? nv[v].z - hy[u][v] : 0.0F, want_h ? nv[v].w - hz[u][v] : 0.0F);
      }
    }
  }
}

__global__ void __launch_bounds__(kL2pThreads) l2p_kernel(const float *__restrict__ L, const float4 *__restrict__ tgt_rel,
                                                          const int *__restrict__ tgt_off, float4 *__restrict__ near,
                                                          const int8_t *__restrict__ basis, int n, int p, int K,
                                                          int leaf_node_base, unsigned output, float phi_scale,
                                                          int Kb, int k_begin, int k_end, int k_near_end) {
  extern __shared__ float4 l2p_smem[];
  const int Kbp = (Kb + 3) & ~3;
  float *sL = reinterpret_cast<float *>(l2p_smem);                 // [n][Kcp]
  float *mono = sL + n * Kbp;                                      // [n][kL2pTargets]
  short *sidx = reinterpret_cast<short *>(mono + n * kL2pTargets); // [nm1][3] rank of mu + e_c
  const int tid = threadIdx.x;
  const int leaf = blockIdx.x;
  const int t0 = tgt_off[leaf];
  const int t1 = tgt_off[leaf + 1];
  if (t0 == t1) return;
  const int nm1 = basis_size_d(p - 1);
  for (int q = tid; q < nm1; q += kL2pThreads) {
    const int a = basis[4 * q], b = basis[4 * q + 1], c = basis[4 * q + 2];
    sidx[3 * q] = static_cast<short>(rank3(a + 1, b, c));
    sidx[3 * q + 1] = static_cast<short>(rank3(a, b + 1, c));
    sidx[3 * q + 2] = static_cast<short>(rank3(a, b, c + 1));
  }
  const bool want_phi = (output & 1u) != 0u;
  const bool want_h = (output & 2u) != 0u;
  const float *src = L + static_cast<long long>(leaf_node_base + leaf) * n * K;
  for (int kblk = k_begin + blockIdx.y * Kb; kblk < k_end; kblk += Kb * gridDim.y) {
    const int Kc = min(Kb, k_end - kblk);
    const int Kcp = (Kc + 3) & ~3;
    const int Kq = Kcp >> 2;
    __syncthreads();
    if ((K & 3) == 0 && (kblk & 3) == 0 && (Kc & 3) == 0) {
      // 4-aligned rows: asynchronous 16-byte copies, all in flight at once
      const int nq = Kcp >> 2;
      for (int q = tid; q < n * nq; q += kL2pThreads) {
        const int b = q / nq;
        cp_async16(reinterpret_cast<float4 *>(sL) + q, src + static_cast<long long>(b) * K + kblk + 4 * (q - b * nq));
      }
      cp_async_commit();
      cp_async_wait<0>();
    } else {
      for (int q = tid; q < n * Kcp; q += kL2pThreads) {
        const int b = q / Kcp;
        const int k = q - b * Kcp;
        sL[q] = k < Kc ? src[static_cast<long long>(b) * K + kblk + k] : 0.0F;
      }
    }
    for (int tc = t0; tc < t1; tc += kL2pTargets) {
      const int tn = min(kL2pTargets, t1 - tc);
      __syncthreads();
      {
        // four threads per target: warp r computes part r of every target's monomials
        const int t = tid & (kL2pTargets - 1);
        const float4 d = t < tn ? tgt_rel[tc + t] : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
        monomials_part(d.x, d.y, d.z, p, mono + t, kL2pTargets, tid / kL2pTargets, t >= tn);
      }
      __syncthreads();
      // register tiles of TU targets x 4 states: TU = 4 for wide state
      // blocks, fewer targets per thread for narrow ones so that the 128
      // threads stay busy
      if (Kq >= 16)
        l2p_tiles<4>(tid, tn, Kq, Kcp, Kc, n, nm1, mono, sL, sidx, want_phi, want_h, near, tc, kblk, K, phi_scale,
                     k_near_end);
      else if (Kq >= 8)
        l2p_tiles<2>(tid, tn, Kq, Kcp, Kc, n, nm1, mono, sL, sidx, want_phi, want_h, near, tc, kblk, K, phi_scale,
                     k_near_end);
      else
        l2p_tiles<1>(tid, tn, Kq, Kcp, Kc, n, nm1, mono, sL, sidx, want_phi, want_h, near, tc, kblk, K, phi_scale,
                     k_near_end);
    }
  }
}

// Few states (K < 4): one thread per (target, state), writing user order
// directly.
__global__ void __launch_bounds__(128) l2p_small_kernel(const float *__restrict__ L, const float4 *__restrict__ tgt_rel,
                                                        const int *__restrict__ tgt_off, const int *__restrict__ tgt_perm,
                                                        const float4 *__restrict__ near, int n, int p, int K, int nt,
                                                        int leaf_node_base, unsigned output, int layout,
                                                        float phi_scale, float *__restrict__ field,
                                                        float *__restrict__ potential) {
  __shared__ float sL[286 * 3];
  const int leaf = blockIdx.x;
  const int t0 = tgt_off[leaf];
  const int t1 = tgt_off[leaf + 1];
  if (t0 == t1) return;
  const float *src = L + static_cast<long long>(leaf_node_base + leaf) * n * K;
  for (int q = threadIdx.x; q < n * K; q += blockDim.x) sL[q] = src[q];
  __syncthreads();
  const bool want_phi = (output & 1u) != 0u;
  const bool want_h = (output & 2u) != 0u;
  for (int it = threadIdx.x; it < (t1 - t0) * K; it += blockDim.x) {
    const int k = it / (t1 - t0);
    const int i = t0 + (it - k * (t1 - t0));
    const float4 d = tgt_rel[i];
    float phi = 0.0F, hx = 0.0F, hy = 0.0F, hz = 0.0F;
    float xa = 1.0F;
    for (int a = 0; a <= p; ++a) {
      float xb = xa;
      for (int b = 0; a + b <= p; ++b) {
        float xc = xb;
        for (int c = 0; a + b + c <= p; ++c) {
          const int deg = a + b + c;
          if (want_phi) phi = fmaf(sL[rank3(a, b, c) * K + k], xc, phi);
          if (want_h && deg < p) {
            hx = fmaf(sL[rank3(a + 1, b, c) * K + k], xc, hx);
            hy = fmaf(sL[rank3(a, b + 1, c) * K + k], xc, hy);
            hz = fmaf(sL[rank3(a, b, c + 1) * K + k], xc, hz);
          }
          xc = xc * d.z * kInvInt[c + 1];
        }
        xb = xb * d.y * kInvInt[b + 1];
      }
      xa = xa * d.x * kInvInt[a + 1];
    }
    const float4 nr = near[static_cast<long long>(i) * K + k];
    const float rphi = want_phi ? (phi + nr.x) * phi_scale : 0.0F;
    const float rx = want_h ? nr.y - hx : 0.0F;
    const float ry = want_h ? nr.z - hy : 0.0F;
    const float rz = want_h ? nr.w - hz : 0.0F;
    const long long o = static_cast<long long>(k) * nt + tgt_perm[i];
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

// Sorted results res[nt][K] (phi, Hx, Hy, Hz) -> user order: field[K][nt][3]
// and potential[K][nt] (layout 0) or field[K][nt][4] (layout 1).  A CTA takes
// 32 consecutive user indices and 32 states through a shared tile: the reads
// are contiguous runs of each sorted row (inv = user -> sorted), the writes
// contiguous runs of each state's user array.
__global__ void __launch_bounds__(256) unsort_results_kernel(const float4 *__restrict__ res, const int *__restrict__ inv,
                                                             int nt, int K, unsigned output, int layout,
                                                             float *__restrict__ field, float *__restrict__ potential,
                                                             int k_begin, int k_end) {
  __shared__ float4 tile[32][33];
  const int u0 = blockIdx.x * 32;
  const int nu = min(32, nt - u0);
  const bool want_phi = (output & 1u) != 0u;
  const bool want_h = (output & 2u) != 0u;
  for (int kc = k_begin; kc < k_end; kc += 32) {
    const int kn = min(32, k_end - kc);
    for (int e = threadIdx.x; e < nu * kn; e += blockDim.x) {
      const int t = e / kn;
      const int k = e - t * kn;
      tile[t][k] = res[static_cast<long long>(inv[u0 + t]) * K + kc + k];
    }
    __syncthreads();
    if (layout == 1) {
      for (int e = threadIdx.x; e < kn * nu; e += blockDim.x) {
        const int k = e / nu;
        const int t = e - k * nu;
        reinterpret_cast<float4 *>(field)[static_cast<long long>(kc + k) * nt + u0 + t] = tile[t][k];
      }
    } else {
      if (want_h) {
        for (int e = threadIdx.x; e < kn * nu * 3; e += blockDim.x) {
          const int k = e / (nu * 3);
          const int r = e - k * nu * 3;
          const int t = r / 3;
          const int c = r - 3 * t;
          const float4 v = tile[t][k];
          field[(static_cast<long long>(kc + k) * nt + u0) * 3 + r] = c == 0 ? v.y : (c == 1 ? v.z : v.w);
        }
      }
      if (want_phi && potential != nullptr) {
        for (int e = threadIdx.x; e < kn * nu; e += blockDim.x) {
          const int k = e / nu;
          const int t = e - k * nu;
          potential[static_cast<long long>(kc + k) * nt + u0 + t] = tile[t][k].x;
        }
      }
    }
    __syncthreads();
  }
}

// Position gradient of L = sum_k w_k . H_k (reverse mode; no counterpart in
// the reference), far part.  H_k = -grad phi_k, so dL/dx_j = -sum_k sum_c
// w_kc d_c d_j phi_k, and from phi = sum_b L_b dx^b/b! (the exact derivative
// of the evaluated polynomial) the Hessian at the target is
//   S_cj[k] = sum_{|mu| <= p-2} x^mu/mu! L_{mu + e_c + e_j}[k]   (6 unique c <= j),
// so g_j -= sum_k sum_c w_kc S_cj[k].  Per leaf
// the leaf's locals (a state block) and the monomials of 32 targets are
// staged in shared memory; a thread owns a register tile of 2 targets x 4
// states x 6 Hessian components (a small GEMM over the monomials), contracts
// it with the weights and adds its 2 targets' partial gradients into shared
// memory; then the list-1 part (gpart, one partial per state group) is added
// and the result written in user order.
constexpr int kL2pGradThreads = 128;

__global__ void __launch_bounds__(kL2pGradThreads) l2p_grad_kernel(
    const float *__restrict__ L, const float4 *__restrict__ tgt_rel, const int *__restrict__ tgt_off,
    const int *__restrict__ tgt_perm, const float4 *__restrict__ W, const float4 *__restrict__ gpart, int G, int n,
    int p, int K, int leaf_node_base, float inv_scale, float *__restrict__ out, int Kb) {
  extern __shared__ float4 l2pg_smem[];
  const int Kbp = (Kb + 3) & ~3;
  const int q = max(p - 2, 0);
  const int nm2 = p >= 2 ? basis_size_d(p - 2) : 0;
  float *sL = reinterpret_cast<float *>(l2pg_smem);               // [n][Kcp]
  float *mono = sL + n * Kbp;                                      // [nm2][kL2pTargets]
  float *gsum = mono + nm2 * kL2pTargets;                          // [kL2pTargets][3]
  short *sidx = reinterpret_cast<short *>(gsum + 3 * kL2pTargets); // [nm2][6] ranks of mu + e_c + e_j
  const int tid = threadIdx.x;
  const int leaf = blockIdx.x;
  const int t0 = tgt_off[leaf];
  const int t1 = tgt_off[leaf + 1];
  if (t0 == t1) return;
  for (int m = tid; m < nm2; m += kL2pGradThreads) {
    int a = 0, b = 0, c = 0;
    for (int aa = 0; aa <= q; ++aa)
      for (int bb = 0; aa + bb <= q; ++bb)
        for (int cc = 0; aa + bb + cc <= q; ++cc)
          if (rank3(aa, bb, cc) == m) {
            a = aa;
            b = bb;
            c = cc;
          }
    sidx[6 * m + 0] = static_cast<short>(rank3(a + 2, b, c));         // xx
    sidx[6 * m + 1] = static_cast<short>(rank3(a + 1, b + 1, c));     // xy
    sidx[6 * m + 2] = static_cast<short>(rank3(a + 1, b, c + 1));     // xz
    sidx[6 * m + 3] = static_cast<short>(rank3(a, b + 2, c));         // yy
    sidx[6 * m + 4] = static_cast<short>(rank3(a, b + 1, c + 1));     // yz
    sidx[6 * m + 5] = static_cast<short>(rank3(a, b, c + 2));         // zz
  }
  const float *src = L + static_cast<long long>(leaf_node_base + leaf) * n * K;
  for (int tc = t0; tc < t1; tc += kL2pTargets) {
    const int tn = min(kL2pTargets, t1 - tc);
    __syncthreads(); // previous chunk's gsum and mono reads are done
    if (tid < 3 * kL2pTargets) gsum[tid] = 0.0F;
    if (nm2 > 0) {
      const int t = tid & (kL2pTargets - 1);
      const float4 d = t < tn ? tgt_rel[tc + t] : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
      monomials_part(d.x, d.y, d.z, q, mono + t, kL2pTargets, tid / kL2pTargets, t >= tn);
    }
    for (int kblk = 0; kblk < K; kblk += Kb) {
      const int Kc = min(Kb, K - kblk);
      const int Kcp = (Kc + 3) & ~3;
      const int Kq = Kcp >> 2;
      __syncthreads(); // previous block's sL reads are done
      if ((K & 3) == 0 && (kblk & 3) == 0 && (Kc & 3) == 0) {
        const int nq = Kcp >> 2;
        for (int e = tid; e < n * nq; e += kL2pGradThreads) {
          const int b = e / nq;
          cp_async16(reinterpret_cast<float4 *>(sL) + e, src + static_cast<long long>(b) * K + kblk + 4 * (e - b * nq));
        }
        cp_async_commit();
        cp_async_wait<0>();
      } else {
        for (int e = tid; e < n * Kcp; e += kL2pGradThreads) {
          const int b = e / Kcp;
          const int k = e - b * Kcp;
          sL[e] = k < Kc ? src[static_cast<long long>(b) * K + kblk + k] : 0.0F;
        }
      }
      __syncthreads();
      if (nm2 == 0) continue;
      const int tiles = ((tn + 1) >> 1) * Kq;
      for (int tile = tid; tile < tiles; tile += kL2pGradThreads) {
        const int tp = tile / Kq;
        const int kq = tile - tp * Kq;
        float hs[2][4][6];
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int v = 0; v < 4; ++v)
#pragma unroll
            for (int h = 0; h < 6; ++h) hs[u][v][h] = 0.0F;
        const float *mq = mono + 2 * tp;
        const float *lq = sL + 4 * kq;
        for (int m = 0; m < nm2; ++m) {
          const float2 mo = *reinterpret_cast<const float2 *>(mq + m * kL2pTargets);
#pragma unroll
          for (int h = 0; h < 6; ++h) {
            const float4 l = *reinterpret_cast<const float4 *>(lq + sidx[6 * m + h] * Kcp);
            hs[0][0][h] = fmaf(mo.x, l.x, hs[0][0][h]);
            hs[0][1][h] = fmaf(mo.x, l.y, hs[0][1][h]);
            hs[0][2][h] = fmaf(mo.x, l.z, hs[0][2][h]);
            hs[0][3][h] = fmaf(mo.x, l.w, hs[0][3][h]);
            hs[1][0][h] = fmaf(mo.y, l.x, hs[1][0][h]);
            hs[1][1][h] = fmaf(mo.y, l.y, hs[1][1][h]);
            hs[1][2][h] = fmaf(mo.y, l.z, hs[1][2][h]);
            hs[1][3][h] = fmaf(mo.y, l.w, hs[1][3][h]);
          }
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int t = 2 * tp + u;
          float g0 = 0.0F, g1 = 0.0F, g2 = 0.0F;
#pragma unroll
          for (int v = 0; v < 4; ++v) {
            const int kl = 4 * kq + v;
            const float4 w = (t < tn && kl < Kc) ? W[static_cast<long long>(tc + t) * K + kblk + kl]
                                                 : make_float4(0.0F, 0.0F, 0.0F, 0.0F);
            g0 = fmaf(w.x, hs[u][v][0], fmaf(w.y, hs[u][v][1], fmaf(w.z, hs[u][v][2], g0)));
            g1 = fmaf(w.x, hs[u][v][1], fmaf(w.y, hs[u][v][3], fmaf(w.z, hs[u][v][4], g1)));
            g2 = fmaf(w.x, hs[u][v][2], fmaf(w.y, hs[u][v][4], fmaf(w.z, hs[u][v][5], g2)));
          }
          if (t < tn) {
            atomicAdd(&gsum[3 * t], -g0);
            atomicAdd(&gsum[3 * t + 1], -g1);
            atomicAdd(&gsum[3 * t + 2], -g2);
          }
        }
      }
    }
    __syncthreads();
    for (int t = tid; t < tn; t += kL2pGradThreads) {
      const int i = tc + t;
      float g0 = gsum[3 * t], g1 = gsum[3 * t + 1], g2 = gsum[3 * t + 2];
      for (int gi = 0; gi < G; ++gi) {
        const float4 v = gpart[static_cast<long long>(i) * G + gi];
        g0 += v.x;
        g1 += v.y;
        g2 += v.z;
      }
      const int u = tgt_perm[i];
      out[3 * static_cast<long long>(u)] = g0 * inv_scale;
      out[3 * static_cast<long long>(u) + 1] = g1 * inv_scale;
      out[3 * static_cast<long long>(u) + 2] = g2 * inv_scale;
    }
  }
}

} // namespace

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------

void launch_gather_moments(const void *user, int dtype, const int *inv, int ns, int K,
                           double scale, float4 *mom, cudaStream_t s, bool paired, int k0, int k_total) {
  if (ns == 0) return;
  if (k_total < 0) k_total = K;
  const int krow = paired ? (k_total + 1) & ~1 : k_total;
  const int blocks = (ns + 31) / 32;
  const double invs = 1.0 / scale;
  const float inv3f = static_cast<float>(invs * invs * invs);
  if (dtype == 1)
    gather_moments_kernel<double><<<blocks, 256, 0, s>>>(static_cast<const double *>(user), inv, ns, K, invs, inv3f,
                                                         paired, mom, k0, krow);
  else
    gather_moments_kernel<float><<<blocks, 256, 0, s>>>(static_cast<const float *>(user), inv, ns, K, invs, inv3f,
                                                        paired, mom, k0, krow);
}

// State block of the P2M kernel for K states: the largest of 64, 32, ...
// (<= K) whose shared memory stays within 100 KB (two CTAs per SM).
#ifndef CDFMM_P2M_KB
#define CDFMM_P2M_KB 32
#endif
#ifndef CDFMM_P2M_SPLIT
#define CDFMM_P2M_SPLIT 0
#endif
#ifndef CDFMM_L2P_KB
#define CDFMM_L2P_KB 64
#endif
#ifndef CDFMM_L2P_SPLIT
#define CDFMM_L2P_SPLIT 0
#endif
#ifndef CDFMM_P2M_SMEM_CAP
#define CDFMM_P2M_SMEM_CAP (64 * 1024)
#endif
static int p2m_state_block(int p, int K) {
  int Kb = std::min(K, CDFMM_P2M_KB);
  while (Kb > 4 && p2m_smem_bytes(0, p, Kb, 0) > CDFMM_P2M_SMEM_CAP) Kb = (Kb + 1) / 2;
  return Kb;
}

size_t p2m_smem_bytes(int n, int p, int K, int chunk) {
  (void)n;
  (void)chunk;
  const int nm1p = (basis_size_d(p - 1) + 3) & ~3;
  const size_t Kb = static_cast<size_t>(std::min(K, CDFMM_P2M_KB));
  return sizeof(float4) * kP2mChunk * Kb + sizeof(float) * (3 * nm1p * (Kb + 2) + static_cast<size_t>(kP2mChunk) * nm1p) +
         sizeof(short) * 4 * static_cast<size_t>(basis_size_d(p));
}

void launch_p2m(const float4 *src_rel, const float4 *mom, const int *src_off, const int8_t *basis,
                float *M, int n, int p, int K, int depth, int chunk, cudaStream_t s, const float4 *size,
                int size_step) {
  (void)chunk;
  const int leaves = 1 << (3 * depth);
  if (K < 4) {
    p2m_small_kernel<<<leaves, 128, 0, s>>>(src_rel, mom, src_off, basis, M, n, p, K, level_offset_d(depth), size,
                                            size_step);
    return;
  }
  // State blocks of <= 32 keep a CTA within 64 KB (several CTAs per SM hide
  // the staging latency); 128 threads cover the 4 x 4 tiles of p <= 6.
  const int Kb = p2m_state_block(p, K);
  const size_t smem = p2m_smem_bytes(n, p, Kb, 0);
  const int nm1p = (basis_size_d(p - 1) + 3) & ~3;
  const int threads = (nm1p / 4) * ((Kb + 3) / 4) <= 128 ? 128 : kP2mThreads;
  const dim3 grid(leaves, CDFMM_P2M_SPLIT ? (K + Kb - 1) / Kb : 1);
  p2m_kernel<<<grid, threads, smem, s>>>(src_rel, mom, src_off, basis, M, n, p, K, level_offset_d(depth), Kb, size,
                                         size_step);
}

static size_t pair_smem(int n, int n_pairs) {
  return sizeof(int) * (static_cast<size_t>(n) + 1 + n_pairs) + sizeof(float) * 8 * static_cast<size_t>(n);
}

// State block of the shift kernels: the largest of 32, 16, 8, 4 whose staged
// block (children for M2M) fits 48 KB of shared memory, so that several CTAs
// per SM overlap one CTA's staging with another's arithmetic.
static int shift_state_block(int n, int n_pairs, int K, int rows) {
  int Ks = 32;
  while (Ks > 4 && pair_smem(n, n_pairs) + sizeof(float) * rows * static_cast<size_t>(n) * Ks + 16 > 48 * 1024) Ks /= 2;
  return std::min(Ks, (K + 3) & ~3);
}

void launch_m2m(float *M, const int *pair_off, const int *pairs, const float *coef, int n, int K,
                int parent_level, int n_pairs, cudaStream_t s) {
  const int Ks = shift_state_block(n, n_pairs, K, 8);
  const dim3 grid(1u << (3 * parent_level), static_cast<unsigned>((K + Ks - 1) / Ks));
  const size_t smem = pair_smem(n, n_pairs) + sizeof(float) * 8 * static_cast<size_t>(n) * Ks + 16;
  m2m_kernel<<<grid, kShiftThreads, smem, s>>>(M, pair_off, pairs, coef, n, K, parent_level, n_pairs, Ks);
}

void launch_l2l(float *L, const int *pair_off, const int *pairs, const float *coef, int n, int K,
                int child_level, int n_pairs, cudaStream_t s) {
  const int Ks = shift_state_block(n, n_pairs, K, 1);
  const dim3 grid(1u << (3 * (child_level - 1)), static_cast<unsigned>((K + Ks - 1) / Ks));
  const size_t smem = pair_smem(n, n_pairs) + sizeof(float) * static_cast<size_t>(n) * Ks + 16;
  l2l_kernel<<<grid, kShiftThreads, smem, s>>>(L, pair_off, pairs, coef, n, K, child_level, n_pairs, Ks);
}

size_t l2p_smem_bytes(int n, int p, int Kb) {
  const int Kbp = (Kb + 3) & ~3;
  return sizeof(float) * (static_cast<size_t>(n) * Kbp + static_cast<size_t>(n) * kL2pTargets) +
         sizeof(short) * 3 * static_cast<size_t>(basis_size_d(p - 1)) + 16;
}

void launch_l2p(const float *L, const float4 *tgt_rel, const int *tgt_off, const int *tgt_perm, const int *tgt_inv,
                float4 *near, const int8_t *basis, int n, int p, int K, int nt, int depth, unsigned output,
                int layout, float phi_scale, float *field, float *potential, cudaStream_t s, int k_begin,
                int k_end, int k_near_end, bool unsort) {
  if (nt == 0) return;
  if (k_end < 0) k_end = K;
  if (k_near_end < 0) k_near_end = K;
  const int leaves = 1 << (3 * depth);
  if (K < 4) {
    l2p_small_kernel<<<leaves, 128, 0, s>>>(L, tgt_rel, tgt_off, tgt_perm, near, n, p, K, nt, level_offset_d(depth),
                                            output, layout, phi_scale, field, potential);
    return;
  }
  int Kb = std::min(K, CDFMM_L2P_KB);
  while (Kb > 4 && l2p_smem_bytes(n, p, Kb) > 60 * 1024) Kb = (Kb + 1) / 2;
  const size_t smem = l2p_smem_bytes(n, p, Kb);
  const dim3 grid(leaves, CDFMM_L2P_SPLIT ? (k_end - k_begin + Kb - 1) / Kb : 1);
  if (k_end > k_begin)
    l2p_kernel<<<grid, kL2pThreads, smem, s>>>(L, tgt_rel, tgt_off, near, basis, n, p, K, level_offset_d(depth), output,
                                               phi_scale, Kb, k_begin, k_end, k_near_end);
  if (unsort) launch_unsort(near, tgt_inv, nt, K, output, layout, field, potential, s, k_begin, k_end);
}

void launch_unsort(const float4 *res, const int *tgt_inv, int nt, int K, unsigned output, int layout, float *field,
                   float *potential, cudaStream_t s, int k_begin, int k_end) {
  if (nt == 0 || k_end <= k_begin) return;
  unsort_results_kernel<<<(nt + 31) / 32, 256, 0, s>>>(res, tgt_inv, nt, K, output, layout, field, potential, k_begin,
                                                       k_end);
}

void launch_l2p_grad(const float *L, const float4 *tgt_rel, const int *tgt_off, const int *tgt_perm,
                     const float4 *W, const float4 *gpart, int G, int n, int p, int K, int nt, int depth,
                     float inv_scale, float *out, cudaStream_t s) {
  if (nt == 0) return;
  const int leaves = 1 << (3 * depth);
  const int nm2 = p >= 2 ? basis_size_d(p - 2) : 0;
  auto smem_of = [&](int Kb) {
    return sizeof(float) * (static_cast<size_t>(n) * ((Kb + 3) & ~3) + static_cast<size_t>(nm2) * kL2pTargets +
                            3 * kL2pTargets) +
           sizeof(short) * 6 * static_cast<size_t>(nm2) + 16;
  };
  int Kb = std::min(K, 64);
  while (Kb > 4 && smem_of(Kb) > 48 * 1024) Kb = (Kb + 1) / 2;
  l2p_grad_kernel<<<leaves, kL2pGradThreads, smem_of(Kb), s>>>(L, tgt_rel, tgt_off, tgt_perm, W, gpart, G, n, p, K,
                                                              level_offset_d(depth), inv_scale, out, Kb);
}

void configure_far_kernels(size_t max_smem) {
  allow_dynamic_smem(l2p_grad_kernel, max_smem);
  allow_dynamic_smem(p2m_kernel, max_smem);
  allow_dynamic_smem(l2p_kernel, max_smem);
  allow_dynamic_smem(m2m_kernel, max_smem);
  allow_dynamic_smem(l2l_kernel, max_smem);
  prefer_max_shared_carveout(l2l_kernel); // runs beside the co-resident near field
}

} // namespace cdfmm_b200
