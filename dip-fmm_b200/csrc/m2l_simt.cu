// M2L, FP32 SIMT (the plain per-state path).
//
//   L_beta(t) = D_L[l][beta] sum_{s in list2(t)} sum_alpha T^(t-s)[beta][alpha] D_M[l][alpha] M_alpha(s)
// (upstream docs/math.md "M2L normalisation and cross-level reuse";
// src/static_operators.cpp:16-102; src/cuda_fmm.cu:119-189).
//
// list2 is implicit: a target t = 2p + c (parent p, child parity class c)
// interacts exactly with the sources s = t - o for the 189 offsets o with
// o_axis in [c_axis - 3, c_axis + 2] and not all |o_axis| <= 1, clipped to the
// grid (children of the parent's clipped 3x3x3 neighbourhood minus the
// target's own 3x3x3, src/uniform_tree.cpp:482-516).  Empty source boxes have
// M = 0 and contribute nothing, as the reference's skip of empty boxes does.
//
// The operator is applied in its traceless-reduced form (M2lTraceless, the
// same reduction as the tensor-core M2L): the (p+1)^2 - 1 folded moments
// M'_alpha (alpha_z <= 1) times the sub-block of T on the (p+1)^2 locals with
// beta_z <= 1; the other locals follow from L_beta = -L_(beta-2z+2x) -
// L_(beta-2z+2y).  Exact in exact arithmetic, a third of the FMA work at
// p = 6.
//
// Work decomposition: one CTA per (level, class, 4x4x4 block of parents) and
// state; for each offset the CTA stages that offset's reduced matrix (alpha
// chunk by alpha chunk) and the 64 source boxes' folded moments in shared
// memory and accumulates a 64-target x n_out tile in registers (8 targets x J
// betas per thread); the epilogue expands each target's locals to all n
// coefficients in shared memory.
#include <cuda_runtime.h>

#include <algorithm>

#include "far_kernels.hpp"
#include "kernels.cuh"

namespace cdfmm_b200 {

namespace {

constexpr int kAlphaChunk = 32;
constexpr int kTileTargets = 64;

struct SimtReduction {
  const int *fold_off; // [n_in + 1]
  const int *fold;     // full rank | (coefficient + 64) << 16, the input's own rank first
  const int *expand;   // [n_out] full ranks of the reduced locals, then d | s1 << 10 | s2 << 20
  int n_in, n_out, n_derived;
};

template <int J>
__global__ void __launch_bounds__(128) m2l_simt_kernel(const float *__restrict__ Mf, float *__restrict__ L,
                                                       const float *__restrict__ T,
                                                       const float *__restrict__ scale_m,
                                                       const float *__restrict__ scale_l,
                                                       const int4 *__restrict__ tiles, int n,
                                                       int ld, int K, int node_base, const SimtReduction r) {
  constexpr int BW = 16 * J; // reduced betas covered by the CTA (>= n_out)
  extern __shared__ float smem[];
  float *sT = smem;                                  // [kAlphaChunk][BW]
  float *sM = sT + kAlphaChunk * BW;                 // [64][kAlphaChunk + 1]
  float *sE = smem;                                  // epilogue: [64][n + 1] full-basis locals
  __shared__ int sSrc[kTileTargets];
  __shared__ int sTgt[kTileTargets];

  const int4 tile = tiles[blockIdx.x];
  const int level = tile.x;
  const int cls = tile.y;
  const int k = blockIdx.y;
  const int side = 1 << level;
  const int pside = side >> 1;
  const int px0 = tile.z & 1023, py0 = (tile.z >> 10) & 1023, pz0 = (tile.z >> 20) & 1023;
  const int cx = cls & 1, cy = (cls >> 1) & 1, cz = (cls >> 2) & 1;
  const int lvl_off = level_offset_d(level);
  const long long node_stride = static_cast<long long>(n) * K;

  const int tt = threadIdx.x >> 4;
  const int bb = threadIdx.x & 15;

  // Target boxes of this tile (node index or -1 outside the grid).
  if (threadIdx.x < kTileTargets) {
    const int u = threadIdx.x;
    const int px = px0 + (u & 3), py = py0 + ((u >> 2) & 3), pz = pz0 + (u >> 4);
    sTgt[u] = (px < pside && py < pside && pz < pside)
                  ? lvl_off + static_cast<int>(morton3(2 * px + cx, 2 * py + cy, 2 * pz + cz))
                  : -1;
  }

  float acc[8][J];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < J; ++j) acc[i][j] = 0.0F;

  for (int oz = cz - 3; oz <= cz + 2; ++oz)
    for (int oy = cy - 3; oy <= cy + 2; ++oy)
      for (int ox = cx - 3; ox <= cx + 2; ++ox) {
        if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1 && oz >= -1 && oz <= 1) continue;
        const float *Ts = T + static_cast<long long>((ox + 3) * 49 + (oy + 3) * 7 + (oz + 3)) * r.n_in * ld;
        __syncthreads();
        if (threadIdx.x < kTileTargets) {
          const int u = threadIdx.x;
          const int px = px0 + (u & 3), py = py0 + ((u >> 2) & 3), pz = pz0 + (u >> 4);
          const int sx = 2 * px + cx - ox, sy = 2 * py + cy - oy, sz = 2 * pz + cz - oz;
          const bool ok = sTgt[u] >= 0 && sx >= 0 && sy >= 0 && sz >= 0 && sx < side && sy < side && sz < side;
          sSrc[u] = ok ? lvl_off + static_cast<int>(morton3(sx, sy, sz)) : -1;
        }
        for (int a0 = 0; a0 < r.n_in; a0 += kAlphaChunk) {
          const int an = min(kAlphaChunk, r.n_in - a0);
          __syncthreads();
          // matrix rows a0 .. a0+an-1, betas 0 .. BW-1 (ld >= BW, 16-byte rows)
          for (int q = threadIdx.x; q < an * (BW / 4); q += blockDim.x) {
            const int row = q / (BW / 4);
            const int c4 = q - row * (BW / 4);
            reinterpret_cast<float4 *>(sT + row * BW)[c4] =
                reinterpret_cast<const float4 *>(Ts + static_cast<long long>(a0 + row) * ld)[c4];
          }
          for (int q = threadIdx.x; q < kTileTargets * kAlphaChunk; q += blockDim.x) {
            const int u = q / kAlphaChunk;
            const int a = q - u * kAlphaChunk;
            const int src = sSrc[u];
            float v = 0.0F;
            if (src >= 0 && a < an)
              v = Mf[(static_cast<long long>(src - node_base) * r.n_in + a0 + a) * K + k]; // folded, scaled
            sM[u * (kAlphaChunk + 1) + a] = v;
          }
          __syncthreads();
          for (int a = 0; a < an; ++a) {
            float tv[J];
#pragma unroll
            for (int j = 0; j < J; ++j) tv[j] = sT[a * BW + bb + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              const float mv = sM[(tt * 8 + i) * (kAlphaChunk + 1) + a];
#pragma unroll
              for (int j = 0; j < J; ++j) acc[i][j] = fmaf(tv[j], mv, acc[i][j]);
            }
          }
        }
      }

  // Epilogue: the reduced locals at their full ranks (row per target), the
  // rest from the trace relations, all n scaled and stored.
  const int es = n + 1;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < J; ++j) {
      const int b = bb + 16 * j;
      if (b < r.n_out) sE[(tt * 8 + i) * es + __ldg(r.expand + b)] = acc[i][j];
    }
  __syncthreads();
  if (threadIdx.x < kTileTargets) {
    const int u = threadIdx.x;
    const int node = sTgt[u];
    if (node >= 0) {
      float *e = sE + u * es;
      for (int q = 0; q < r.n_derived; ++q) {
        const int d = __ldg(r.expand + r.n_out + q);
        e[d & 1023] = -(e[(d >> 10) & 1023] + e[d >> 20]);
      }
      for (int b = 0; b < n; ++b) L[node * node_stride + static_cast<long long>(b) * K + k] = e[b] * scale_l[level * n + b];
    }
  }
}

// Folded, scaled moments of every box of levels 2..depth, once per call:
// Mf[box][j][k] = 2^(l|alpha_j|) sum_f c_f M_(a_f)[k] over the fold entries
// of input j (one degree, its own rank first, fixed order).
__global__ void __launch_bounds__(128) fold_moments_kernel(const float *__restrict__ M,
                                                           const float *__restrict__ scale_m,
                                                           const int *__restrict__ fold_off,
                                                           const int *__restrict__ fold, int n, int n_in, int K,
                                                           int depth, int node_base, float *__restrict__ Mf) {
  const int box = blockIdx.x;
  const int node = node_base + box;
  int level = 0;
  while (level < depth && level_offset_d(level + 1) <= node) ++level;
  const float *src = M + static_cast<long long>(node) * n * K;
  float *dst = Mf + static_cast<long long>(box) * n_in * K;
  for (int e = threadIdx.x; e < n_in * K; e += blockDim.x) {
    const int j = e / K;
    const int k = e - j * K;
    const int f0 = __ldg(fold_off + j), f1 = __ldg(fold_off + j + 1);
    float v = 0.0F;
    for (int f = f0; f < f1; ++f) {
      const int c = __ldg(fold + f);
      v = fmaf(static_cast<float>((c >> 16) - 64), src[static_cast<long long>(c & 0xffff) * K + k], v);
    }
    dst[e] = v * scale_m[level * n + (__ldg(fold + f0) & 0xffff)];
  }
}

template <int J>
void launch_j(const float *Mf, float *L, const float *T, const float *sm, const float *sl,
              const int4 *tiles, int n_tiles, int n, int ld, int K, const SimtReduction &r, cudaStream_t s) {
  const size_t smem = sizeof(float) * std::max<size_t>(kAlphaChunk * 16 * J + kTileTargets * (kAlphaChunk + 1),
                                                       static_cast<size_t>(kTileTargets) * (n + 1));
  dim3 grid(n_tiles, K);
  m2l_simt_kernel<J><<<grid, 128, smem, s>>>(Mf, L, T, sm, sl, tiles, n, ld, K, level_offset_d(2), r);
}

} // namespace

int m2l_simt_beta_per_thread(int n) {
  const int j = (n + 15) / 16;
  if (j <= 1) return 1;
  if (j <= 2) return 2;
  if (j <= 3) return 3;
  if (j <= 4) return 4;
  if (j <= 6) return 6;
  if (j <= 8) return 8;
  if (j <= 11) return 11;
  if (j <= 14) return 14;
  return 18;
}

void launch_m2l_simt(const float *M, float *Mf, float *L, const float *T, const float *scale_m,
                     const float *scale_l, const int4 *tiles, int n_tiles, int n, int ld, int K, int depth,
                     const int *fold_off, const int *fold, const int *expand, int n_in, int n_out, int n_derived,
                     cudaStream_t s) {
  if (n_tiles == 0) return;
  const int node_base = level_offset_d(2);
  fold_moments_kernel<<<level_offset_d(depth + 1) - node_base, 128, 0, s>>>(M, scale_m, fold_off, fold, n, n_in, K,
                                                                           depth, node_base, Mf);
  // the main kernel reads the folded moments
  const SimtReduction r{fold_off, fold, expand, n_in, n_out, n_derived};
  switch (m2l_simt_beta_per_thread(n_out)) {
  case 1: launch_j<1>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  case 2: launch_j<2>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  case 3: launch_j<3>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  case 4: launch_j<4>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  case 6: launch_j<6>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  case 8: launch_j<8>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  case 11: launch_j<11>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  case 14: launch_j<14>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  default: launch_j<18>(Mf, L, T, scale_m, scale_l, tiles, n_tiles, n, ld, K, r, s); break;
  }
}

void configure_m2l_simt(size_t max_smem) {
  allow_dynamic_smem(m2l_simt_kernel<1>, max_smem);
  allow_dynamic_smem(m2l_simt_kernel<2>, max_smem);
  allow_dynamic_smem(m2l_simt_kernel<3>, max_smem);
  allow_dynamic_smem(m2l_simt_kernel<4>, max_smem);
  allow_dynamic_smem(m2l_simt_kernel<6>, max_smem);
  allow_dynamic_smem(m2l_simt_kernel<8>, max_smem);
  allow_dynamic_smem(m2l_simt_kernel<11>, max_smem);
  allow_dynamic_smem(m2l_simt_kernel<14>, max_smem);
  allow_dynamic_smem(m2l_simt_kernel<18>, max_smem);
}

} // namespace cdfmm_b200
