// Position gradient of L = sum_k w_k . H_k over the list-1 near field, K >= 8
// states, on the 5th-generation tensor cores.
//
// For a pair (target t, source s) the FP32 kernel sums, over the states,
// a = m.r, b = w.r, C = w.m, P = a b and V = b m + a w (r = x_t - x_s) and
// adds f5 V + (f5 C - f7 P) r (f5 = 3/|r|^5, f7 = 15/|r|^7; no counterpart in
// the reference).  All of them are linear in the 3 x 3 matrix
//
//   X_ts[c][d] = sum_k w_tk[c] m_sk[d]:   C = tr X,  P = r.X r,
//                                        V = X r + X^T r,
//
// so the states' work per pair is one matrix product per work unit: rows
// (c, t) (3 components x 32 targets, padded to 128) times columns (s, d)
// (16 sources x 3 components) with the states as the reduction, the weights
// W as the A operand (fixed per unit, written once into tensor memory) and
// the moments as B (pre-split per block of 16 sources into TF32 hi / lo,
// K-major core matrices [hi, lo][K/4][48 rows][4 states]).  kind::tf32 MMAs,
// three products (A_hi B_hi + A_hi B_lo + A_lo B_hi), FP32 accumulation over
// the K states of one chunk (24 MMAs into a fresh accumulator).
//
// Four epilogue warps read each chunk's X (warp c: row c of every pair of
// its lane's target) and add the row's share of the pair's gradient,
//   g_j += f5 (r_c X[c][j] + [j = c] X[c].r) + (f5 X[c][c] - f7 r_c X[c].r) r_j,
// in FP32 registers; the three rows' shares are summed at the end.  r is
// formed exactly as the FP32 kernels form it (target - (source + neighbour
// offset)), so the close-pair correction applies unchanged; the self source
// gets 1/|r| = 0, empty block slots lie 3e18 away.  Bounded waits as in the
// forward tensor-core near field.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "kernels.cuh"
#include "m2l_tc.hpp"
#include "near_grad_tc.hpp"
#include "tcgen05.cuh"

namespace cdfmm_b200 {

namespace {

using namespace tc;

constexpr int kNgThreads = 192;       // warps 0-3 weights + epilogue, 4 copies, 5 MMA
constexpr uint32_t kNgTmemCols = 256; // two CTAs per SM
constexpr int kNgRows = 3 * kNearGradSources; // 48 accumulator columns per chunk
constexpr int kNgBSlots = 3;
constexpr int kNgPosCap = 96;         // neighbourhood blocks whose positions are staged
constexpr uint32_t kNgMiscBytes = 640;
// sources of the epilogue's loop unrolled at a time (code size vs ILP)
#ifndef CDFMM_NGT_UNROLL
#define CDFMM_NGT_UNROLL 16
#endif
constexpr int kNgUnroll = CDFMM_NGT_UNROLL;
// epilogue rows: one run-time copy (1) or a template per row (0)
#ifndef CDFMM_NGT_RUNTIME_ROW
#define CDFMM_NGT_RUNTIME_ROW 1
#endif
constexpr bool kNgRuntimeRow = CDFMM_NGT_RUNTIME_ROW != 0;

__host__ __device__ inline int ng_kpad(int K) { return (K + 7) / 8 * 8; }

struct NgSmem {
  uint32_t slot_bytes; // one block: [hi, lo][Kpad/4][48][4] floats
  uint32_t pos_off;    // [kNgPosCap + 1][16] float4, then [4 warps][16] scratch
  uint32_t red_off;    // [3 components][32 targets][4] floats
  uint32_t bar_off;
  uint32_t misc_off;
  uint32_t total;
};
__host__ __device__ inline NgSmem ng_smem(int Kpad) {
  NgSmem m;
  m.slot_bytes = 2u * static_cast<uint32_t>(Kpad) / 4u * kNgRows * 16u;
  m.pos_off = kNgBSlots * m.slot_bytes;
  m.red_off = m.pos_off + (kNgPosCap + 1) * kNearGradSources * 16u + 4u * kNearGradSources * 16u;
  m.bar_off = m.red_off + 3u * 32u * 4u * 4u;
  m.misc_off = m.bar_off + (2u * kNgBSlots + 2u + 2u + 3u) * 8u;
  m.total = m.misc_off + kNgMiscBytes;
  return m;
}

struct NgArgs {
  const float4 *blk_pos; // [(n_blocks + 1) * 16]
  const int *blk_off;    // [leaves + 1]
  const uint8_t *b_ops;  // [(n_blocks + 1)] blocks of slot_bytes
  const int4 *work;
  const float4 *tgt_rel;
  const int *self_idx;
  const float4 *W;       // [nt][K] weights (x, y, z, 0)
  float4 *gpart;         // [nt][G]
  int *error_flag;
  int depth, K, Kpad, G, zero_block;
  uint32_t wait_limit;
};

__device__ __forceinline__ bool ng_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  // a suspended poll lasts up to ~1 us: the iteration budget is scaled so
  // the bound stays near the polled one (limit 0 still expires at once)
  return mbar_wait_suspend(bar, parity, limit > 32u ? limit >> 5 : limit, 1000u);
}
__device__ __forceinline__ void ng_abort(int *abort_flag, int *error_flag, int code) {
  *abort_flag = 1;
  atomicExch(error_flag, code);
}
__device__ __forceinline__ bool ng_aborted(const int *abort_flag) {
  return *reinterpret_cast<const volatile int *>(abort_flag) != 0;
}
__device__ __forceinline__ float4 ng_far_slot() {
  return make_float4(3.0e18F, 3.0e18F, 3.0e18F, __int_as_float(-1));
}
__device__ __forceinline__ void ng_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Row c's share of the gradient of one pair (see the file comment); rc is
// the c-th component of r, xc the row X[c][0..2].
template <int C>
__device__ __forceinline__ void pair_row_grad(float rx, float ry, float rz, float f5, float f7, float x0, float x1,
                                              float x2, float (&g)[3]) {
  const float rc = C == 0 ? rx : (C == 1 ? ry : rz);
  const float xr = fmaf(x0, rx, fmaf(x1, ry, x2 * rz));
  const float xcc = C == 0 ? x0 : (C == 1 ? x1 : x2);
  const float coef = fmaf(f5, xcc, -f7 * rc * xr);
  const float v0 = fmaf(rc, x0, C == 0 ? xr : 0.0F);
  const float v1 = fmaf(rc, x1, C == 1 ? xr : 0.0F);
  const float v2 = fmaf(rc, x2, C == 2 ? xr : 0.0F);
  g[0] = fmaf(f5, v0, fmaf(coef, rx, g[0]));
  g[1] = fmaf(f5, v1, fmaf(coef, ry, g[1]));
  g[2] = fmaf(f5, v2, fmaf(coef, rz, g[2]));
}

// The same with the row c chosen at run time (one copy of the unrolled loop
// instead of three: a third of the code the epilogue streams through the
// instruction cache).
__device__ __forceinline__ void chunk_grad_any(int c, const float4 *p16, float tx, float ty, float tz, int self,
                                               const float (&x)[kNgRows], float (&g)[3]) {
  const float e0 = c == 0 ? 1.0F : 0.0F, e1 = c == 1 ? 1.0F : 0.0F, e2 = c == 2 ? 1.0F : 0.0F;
#pragma unroll
  for (int q = 0; q < kNearGradSources; ++q) {
    const float4 p = p16[q];
    const float rx = tx - p.x, ry = ty - p.y, rz = tz - p.z;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
    const float rinv = __float_as_int(p.w) == self ? 0.0F : rsqrtf(r2);
    const float r2inv = rinv * rinv;
    const float f5 = 3.0F * r2inv * r2inv * rinv;
    const float f7 = 5.0F * f5 * r2inv;
    const float x0 = x[3 * q], x1 = x[3 * q + 1], x2 = x[3 * q + 2];
    const float rc = fmaf(e0, rx, fmaf(e1, ry, e2 * rz));
    const float xcc = fmaf(e0, x0, fmaf(e1, x1, e2 * x2));
    const float xr = fmaf(x0, rx, fmaf(x1, ry, x2 * rz));
    const float coef = fmaf(f5, xcc, -f7 * rc * xr);
    g[0] = fmaf(f5, fmaf(rc, x0, e0 * xr), fmaf(coef, rx, g[0]));
    g[1] = fmaf(f5, fmaf(rc, x1, e1 * xr), fmaf(coef, ry, g[1]));
    g[2] = fmaf(f5, fmaf(rc, x2, e2 * xr), fmaf(coef, rz, g[2]));
  }
}

template <int C>
__device__ __forceinline__ void chunk_grad(const float4 *p16, float tx, float ty, float tz, int self,
                                           const float (&x)[kNgRows], float (&g)[3]) {
#pragma unroll kNgUnroll
  for (int q = 0; q < kNearGradSources; ++q) {
    const float4 p = p16[q];
    const float rx = tx - p.x, ry = ty - p.y, rz = tz - p.z;
    const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
    const float rinv = __float_as_int(p.w) == self ? 0.0F : rsqrtf(r2);
    const float r2inv = rinv * rinv;
    const float f5 = 3.0F * r2inv * r2inv * rinv;
    const float f7 = 5.0F * f5 * r2inv;
    pair_row_grad<C>(rx, ry, rz, f5, f7, x[3 * q], x[3 * q + 1], x[3 * q + 2], g);
  }
}

__global__ void __launch_bounds__(kNgThreads, 2) near_grad_tc_kernel(const NgArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int Kpad = a.Kpad;
  constexpr int SB = kNgBSlots;
  const NgSmem lay = ng_smem(Kpad);
  float4 *spos = reinterpret_cast<float4 *>(smem + lay.pos_off);
  float *red = reinterpret_cast<float *>(smem + lay.red_off);
  uint64_t *bfull = reinterpret_cast<uint64_t *>(smem + lay.bar_off);
  uint64_t *bempty = bfull + SB;
  uint64_t *dfull = bempty + SB; // [2]
  uint64_t *dempty = dfull + 2;  // [2]
  uint64_t *aready = dempty + 2;
  uint64_t *pfull = aready + 1;
  uint64_t *done = pfull + 1;
  int *misc = reinterpret_cast<int *>(smem + lay.misc_off);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(misc);
  int *abort_flag = misc + 1;
  int *nb_count = misc + 2;
  int *last_chunk = misc + 4;     // [SB]
  int *nb_first = misc + 8;       // [27]
  int *nb_prefix = nb_first + 27; // [28]
  float *nb_off = reinterpret_cast<float *>(nb_prefix + 28); // [27][3]

  const int4 unit = a.work[blockIdx.x];
  const int leaf = unit.x;
  const int t0 = unit.y;
  const int nt = unit.z;
  const uint32_t blk_bytes = lay.slot_bytes;

  if (tid == 0) {
    for (int s = 0; s < SB; ++s) {
      mbar_init(&bfull[s], 1);
      mbar_init(&bempty[s], 1);
    }
    for (int d = 0; d < 2; ++d) {
      mbar_init(&dfull[d], 1);
      mbar_init(&dempty[d], 4);
    }
    mbar_init(aready, 4);
    mbar_init(pfull, 1);
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < SB) last_chunk[tid] = -1;
  if (warp == 4) {
    // the clipped 3x3x3 neighbourhood (z outermost, x fastest), leaves with
    // sources compacted in that order with their block counts
    int ix, iy, iz;
    demorton3(static_cast<uint32_t>(leaf), ix, iy, iz);
    const int side = 1 << a.depth;
    const float w = 1.0F / static_cast<float>(side);
    const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
    const int x = ix + dx, y = iy + dy, z = iz + dz;
    int b = 0, e = 0;
    if (lane < 27 && x >= 0 && y >= 0 && z >= 0 && x < side && y < side && z < side) {
      const uint32_t m = morton3(x, y, z);
      b = a.blk_off[m];
      e = a.blk_off[m + 1];
    }
    const bool use = e > b;
    const unsigned mask = __ballot_sync(0xffffffffu, use);
    const int slot = __popc(mask & ((1u << lane) - 1u));
    int incl = use ? e - b : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (use) {
      nb_first[slot] = b;
      nb_prefix[slot + 1] = incl;
      nb_off[3 * slot] = static_cast<float>(dx) * w;
      nb_off[3 * slot + 1] = static_cast<float>(dy) * w;
      nb_off[3 * slot + 2] = static_cast<float>(dz) * w;
    }
    if (lane == 0) {
      nb_prefix[0] = 0;
      *nb_count = __popc(mask);
    }
  }
  if (warp == 5) tmem_alloc(tmem_slot, kNgTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int n_nb = *nb_count;
  const int chunks = nb_prefix[n_nb]; // one block of 16 sources per chunk
  const bool staged = chunks <= kNgPosCap;
  const uint32_t dcol0 = 2u * static_cast<uint32_t>(Kpad); // accumulators after A_hi, A_lo

  if (warp == 4) {
    if (staged) {
      if (lane == 0) mbar_expect_tx(pfull, static_cast<uint32_t>(chunks) * kNearGradSources * 16u);
      __syncwarp();
      if (lane < n_nb) {
        const int cnt = nb_prefix[lane + 1] - nb_prefix[lane];
        bulk_g2s(spos + kNearGradSources * nb_prefix[lane], a.blk_pos + static_cast<long long>(kNearGradSources) * nb_first[lane],
                 static_cast<uint32_t>(cnt) * kNearGradSources * 16u, pfull);
      }
    }
    int nbi = 0;
    for (int i = 0; i < chunks; ++i) {
      const int s = i % SB;
      int ok = 1;
      if (lane == 0) {
        if (i >= SB && !ng_wait(&bempty[s], static_cast<uint32_t>((i / SB) - 1) & 1u, a.wait_limit))
          ng_abort(abort_flag, a.error_flag, 8);
        ok = !ng_aborted(abort_flag);
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      while (nbi + 1 < n_nb && nb_prefix[nbi + 1] <= i) ++nbi;
      const size_t blk = static_cast<size_t>(nb_first[nbi] + (i - nb_prefix[nbi]));
      if (lane == 0) {
        mbar_expect_tx(&bfull[s], blk_bytes);
        bulk_g2s(smem + static_cast<uint32_t>(s) * lay.slot_bytes, a.b_ops + blk * blk_bytes, blk_bytes, &bfull[s]);
        last_chunk[s] = i;
      }
      __syncwarp();
    }
  } else if (warp == 5) {
    // MMA issuer: chunk i -> accumulator i % 2 once the epilogue read its
    // chunk i - 2; per k-step of 8 states three MMAs (A_hi B_hi, A_hi B_lo,
    // A_lo B_hi), N = 48.  B: core matrices 8 rows x 4 states, row groups
    // 128 bytes apart (SBO), state groups 768 bytes (LBO), lo after hi.
    if (lane == 0) {
      const uint32_t idesc = instr_desc_tf32(kNgRows);
      const uint64_t desc0 = smem_desc(smem_u32(smem), kNgRows * 16u, 128u);
      const uint32_t lo_off = (static_cast<uint32_t>(Kpad) / 4u * kNgRows * 16u) >> 4;
      bool ok = chunks == 0 || ng_wait(aready, 0, a.wait_limit);
      if (!ok) ng_abort(abort_flag, a.error_flag, 9);
      for (int i = 0; ok && i < chunks; ++i) {
        const int s = i % SB;
        const int db = i & 1;
        if ((i >= 2 && !ng_wait(&dempty[db], static_cast<uint32_t>((i / 2) - 1) & 1u, a.wait_limit)) ||
            !ng_wait(&bfull[s], static_cast<uint32_t>(i / SB) & 1u, a.wait_limit)) {
          ng_abort(abort_flag, a.error_flag, 9);
          break;
        }
        tc_fence_after();
        const uint32_t dcol = tmem + dcol0 + static_cast<uint32_t>(db * kNgRows);
        const uint64_t bd = desc0 + ((static_cast<uint32_t>(s) * lay.slot_bytes) >> 4);
        for (int j = 0; j < Kpad / 8; ++j) {
          const uint64_t bh = bd + ((2u * static_cast<uint32_t>(j) * kNgRows * 16u) >> 4);
          const uint32_t ah = tmem + 8u * static_cast<uint32_t>(j);
          const uint32_t al = ah + static_cast<uint32_t>(Kpad);
          mma_tf32_ts(dcol, ah, bh, idesc, j == 0 ? 0u : 1u);
          mma_tf32_ts(dcol, ah, bh + lo_off, idesc, 1);
          mma_tf32_ts(dcol, al, bh, idesc, 1);
        }
        mma_commit(&bempty[s]);
        mma_commit(&dfull[db]);
      }
      mma_commit(done);
    }
    __syncwarp();
  } else {
    // Warps 0-3: the unit's weights into tensor memory (warp c: row block c,
    // lane t: target t; warp 3 the zero rows), the positions' leaf offsets,
    // then the epilogue of every chunk.
    const int c = warp;
    const uint32_t lane_base = static_cast<uint32_t>(32 * c) << 16;
    const bool tv = lane < nt;
    const int it = t0 + (tv ? lane : 0);
    {
      const float4 *wrow = a.W + static_cast<long long>(it) * a.K;
      for (int k0 = 0; k0 < Kpad; k0 += 8) {
        float hv[8], lv[8];
#pragma unroll
        for (int kk = 0; kk < 8; ++kk) {
          float v = 0.0F;
          if (c < 3 && tv && k0 + kk < a.K) {
            const float4 w4 = wrow[k0 + kk];
            v = c == 0 ? w4.x : (c == 1 ? w4.y : w4.z);
          }
          hv[kk] = tf32_hi(v);
          lv[kk] = tf32_hi(v - hv[kk]);
        }
        tmem_st8(tmem + lane_base + static_cast<uint32_t>(k0), hv);
        tmem_st8(tmem + lane_base + static_cast<uint32_t>(Kpad + k0), lv);
      }
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(aready);
    }
    const float4 tp = a.tgt_rel[it];
    const int self = (a.self_idx != nullptr && tv) ? a.self_idx[it] : -2;
    bool ok = true;
    if (staged && chunks > 0) ok = ng_wait(pfull, 0, a.wait_limit);
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && lane == 0) ng_abort(abort_flag, a.error_flag, 10);
    if (staged) {
      if (ok)
        for (int e = tid; e < kNearGradSources * chunks; e += 128) {
          const int g = e / kNearGradSources;
          int n = 0;
          while (n + 1 < n_nb && nb_prefix[n + 1] <= g) ++n;
          const float4 q = spos[e];
          spos[e] = make_float4(q.x + nb_off[3 * n], q.y + nb_off[3 * n + 1], q.z + nb_off[3 * n + 2], q.w);
        }
      ng_bar();
    }
    float4 *scratch = spos + kNearGradSources * (kNgPosCap + 1) + kNearGradSources * warp;
    float g[3] = {0.0F, 0.0F, 0.0F};
    for (int i = 0; ok && i < chunks; ++i) {
      const int db = i & 1;
      bool got = ng_wait(&dfull[db], static_cast<uint32_t>(i / 2) & 1u, a.wait_limit);
      got = __all_sync(0xffffffffu, got);
      int go = got ? 1 : 0;
      if (lane == 0) {
        if (!got) ng_abort(abort_flag, a.error_flag, 10);
        go = go && !ng_aborted(abort_flag);
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
      tc_fence_after();
      float x[kNgRows];
      if (c < 3) {
        const uint32_t tcol = tmem + lane_base + dcol0 + static_cast<uint32_t>(db * kNgRows);
        float v[16];
        tmem_ld16(tcol, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) x[q] = v[q];
        tmem_ld16(tcol + 16u, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) x[16 + q] = v[q];
        tmem_ld16(tcol + 32u, v);
#pragma unroll
        for (int q = 0; q < 16; ++q) x[32 + q] = v[q];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&dempty[db]);
      if (c == 3) continue;
      const float4 *p16 = spos + kNearGradSources * i;
      if (!staged) {
        if (lane < kNearGradSources) {
          int n = 0;
          while (n + 1 < n_nb && nb_prefix[n + 1] <= i) ++n;
          float4 q = a.blk_pos[static_cast<long long>(kNearGradSources) * (nb_first[n] + (i - nb_prefix[n])) + lane];
          scratch[lane] = make_float4(q.x + nb_off[3 * n], q.y + nb_off[3 * n + 1], q.z + nb_off[3 * n + 2], q.w);
        }
        __syncwarp();
        p16 = scratch;
      }
      if (kNgRuntimeRow)
        chunk_grad_any(c, p16, tp.x, tp.y, tp.z, self, x, g);
      else if (c == 0)
        chunk_grad<0>(p16, tp.x, tp.y, tp.z, self, x, g);
      else if (c == 1)
        chunk_grad<1>(p16, tp.x, tp.y, tp.z, self, x, g);
      else
        chunk_grad<2>(p16, tp.x, tp.y, tp.z, self, x, g);
      if (!staged) __syncwarp(); // scratch reads done before the next chunk overwrites it
    }
    // the three rows' shares of each target's gradient; NaN after an expired wait
    bool quiet = mbar_wait(done, 0, kTcWaitLimit);
    quiet = __all_sync(0xffffffffu, quiet);
    int poison = quiet ? 0 : 1;
    if (lane == 0) {
      if (!quiet) ng_abort(abort_flag, a.error_flag, 11);
      poison = poison || ng_aborted(abort_flag);
    }
    poison = __shfl_sync(0xffffffffu, poison, 0);
    if (c < 3) {
      red[(c * 32 + lane) * 4] = g[0];
      red[(c * 32 + lane) * 4 + 1] = g[1];
      red[(c * 32 + lane) * 4 + 2] = g[2];
    }
    ng_bar();
    if (c == 0 && tv) {
      float s3[3];
#pragma unroll
      for (int j = 0; j < 3; ++j)
        s3[j] = (red[lane * 4 + j] + red[(32 + lane) * 4 + j] + red[(64 + lane) * 4 + j]) * kInvFourPiF;
      if (poison) s3[0] = s3[1] = s3[2] = __int_as_float(0x7fc00000);
      float4 *out = a.gpart + static_cast<long long>(t0 + lane) * a.G;
      out[0] = make_float4(s3[0], s3[1], s3[2], 0.0F);
      for (int q = 1; q < a.G; ++q) out[q] = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (ng_aborted(abort_flag) && tid < 32) {
    // copies issued and never consumed may still be in flight
    if (tid < SB) {
      const int u = last_chunk[tid];
      if (u >= 0) mbar_wait(&bfull[tid], static_cast<uint32_t>(u / SB) & 1u, kTcWaitLimit);
    }
    if (tid == SB && staged && chunks > 0) mbar_wait(pfull, 0, kTcWaitLimit);
  }
  __syncthreads();
  if (warp == 5) {
    tc_fence_after();
    tmem_dealloc(tmem, kNgTmemCols);
  }
}

// Moments -> TF32 hi / lo blocks of 16 sources: per block [hi, lo][Kpad/4]
// [48 rows = (source, component)][4 states]; states k >= K and empty slots
// zero.  Thread per (block, state group, row).
template <bool PAIRED>
__global__ void __launch_bounds__(256) near_grad_pack_kernel(const float4 *__restrict__ mom,
                                                             const int *__restrict__ blk_src, long long total, int K,
                                                             int Kpad, float4 *__restrict__ ops) {
  const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const int row = static_cast<int>(e % kNgRows);
  const long long bg = e / kNgRows;
  const int groups = Kpad / 4;
  const int g = static_cast<int>(bg % groups);
  const long long b = bg / groups;
  const int q = row / 3, d = row - 3 * (row / 3);
  const int j = blk_src[b * kNearGradSources + q];
  float h[4], l[4];
#pragma unroll
  for (int kk = 0; kk < 4; ++kk) {
    const int k = 4 * g + kk;
    float m = 0.0F;
    if (j >= 0 && k < K) {
      if constexpr (PAIRED) {
        const float4 *rowp = mom + static_cast<long long>(j) * ((K + 1) & ~1) + (k & ~1);
        if (d < 2) {
          const float4 r0 = rowp[0];
          m = d == 0 ? ((k & 1) ? r0.y : r0.x) : ((k & 1) ? r0.w : r0.z);
        } else {
          const float4 r1 = rowp[1];
          m = (k & 1) ? r1.y : r1.x;
        }
      } else {
        const float4 r = mom[static_cast<long long>(j) * K + k];
        m = d == 0 ? r.x : (d == 1 ? r.y : r.z);
      }
    }
    h[kk] = tf32_hi(m);
    l[kk] = tf32_hi(m - h[kk]);
  }
  const long long per_half = static_cast<long long>(groups) * kNgRows; // float4 entries of one half
  const long long base = b * 2 * per_half + static_cast<long long>(g) * kNgRows + row;
  ops[base] = make_float4(h[0], h[1], h[2], h[3]);
  ops[base + per_half] = make_float4(l[0], l[1], l[2], l[3]);
}

__global__ void __launch_bounds__(256) near_grad_positions_kernel(const float4 *__restrict__ src_rel,
                                                                  const int *__restrict__ blk_src, int slots,
                                                                  float4 *__restrict__ blk_pos) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= slots) return;
  const int j = blk_src[e];
  // an empty slot lies far from every target: its pair terms underflow to 0
  blk_pos[e] = j >= 0 ? make_float4(src_rel[j].x, src_rel[j].y, src_rel[j].z, __int_as_float(j)) : ng_far_slot();
}

} // namespace

NearGradLayout near_grad_layout(const int *src_off, int depth) {
  NearGradLayout lay;
  const int leaves = 1 << (3 * depth);
  lay.blk_off.assign(static_cast<size_t>(leaves) + 1, 0);
  for (int l = 0; l < leaves; ++l) {
    const int cnt = src_off[l + 1] - src_off[l];
    lay.blk_off[static_cast<size_t>(l) + 1] =
        lay.blk_off[static_cast<size_t>(l)] + (cnt + kNearGradSources - 1) / kNearGradSources;
  }
  lay.n_blocks = lay.blk_off[static_cast<size_t>(leaves)];
  lay.blk_src.assign(static_cast<size_t>(lay.n_blocks + 1) * kNearGradSources, -1);
  for (int l = 0; l < leaves; ++l)
    for (int j = src_off[l]; j < src_off[l + 1]; ++j)
      lay.blk_src[static_cast<size_t>(lay.blk_off[static_cast<size_t>(l)]) * kNearGradSources +
                  static_cast<size_t>(j - src_off[l])] = j;
  return lay;
}

size_t near_grad_operand_bytes(int n_blocks, int K) {
  return static_cast<size_t>(n_blocks + 1) * ng_smem(ng_kpad(std::max(K, 1))).slot_bytes;
}

void launch_near_grad_positions(const float4 *src_rel, const int *blk_src, int n_blocks, float4 *blk_pos,
                                cudaStream_t s) {
  const int slots = (n_blocks + 1) * kNearGradSources;
  near_grad_positions_kernel<<<(slots + 255) / 256, 256, 0, s>>>(src_rel, blk_src, slots, blk_pos);
}

void launch_near_grad_tc(const NearGradLaunch &a, const float4 *mom, const float4 *tgt_rel, const int *self_idx,
                         int depth, int K, const float4 *W, float4 *gpart, int G, cudaStream_t s) {
  if (a.n_work == 0 || K < kNearTcMinStates || K > kNearTcMaxStates) return;
  const int Kpad = ng_kpad(K);
  const long long total = static_cast<long long>(a.n_blocks + 1) * (Kpad / 4) * kNgRows;
  near_grad_pack_kernel<true><<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
      mom, a.blk_src, total, K, Kpad, static_cast<float4 *>(a.b_ops));
  NgArgs args{};
  args.blk_pos = a.blk_pos;
  args.blk_off = a.blk_off;
  args.b_ops = static_cast<const uint8_t *>(a.b_ops);
  args.work = a.work;
  args.tgt_rel = tgt_rel;
  args.self_idx = self_idx;
  args.W = W;
  args.gpart = gpart;
  args.error_flag = a.error_flag;
  args.depth = depth;
  args.K = K;
  args.Kpad = Kpad;
  args.G = G;
  args.zero_block = a.n_blocks;
  args.wait_limit = a.wait_limit;
  // at least a third of the SM's shared memory: no third CTA waits on the
  // tensor memory the two resident ones hold
  const size_t smem = std::max<size_t>(ng_smem(Kpad).total, 80 * 1024);
  near_grad_tc_kernel<<<a.n_work, kNgThreads, smem, s>>>(args);
}

bool configure_near_grad_tc(size_t max_smem) {
  prefer_max_shared_carveout(near_grad_tc_kernel);
  return allow_dynamic_smem(near_grad_tc_kernel, max_smem);
}

} // namespace cdfmm_b200
