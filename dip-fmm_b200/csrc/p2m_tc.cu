// Leaf multipoles (P2M) of K >= 8 states on the 5th-generation tensor cores.
//
// For one leaf the multipoles of every state are one matrix product
//
//   M[alpha, k] = sum_(s, d) A[alpha, (s, d)] * m_s[d][k],
//   A[alpha, (s, d)] = (-1)^|alpha| (x_s - c)^(alpha - e_d) / (alpha - e_d)!
//
// (zero where alpha_d = 0), the dipole P2M of upstream src/far_field.cpp
// (P2M of a point dipole: the moments of m . grad of the monomials), with
// rows alpha (n <= 128 coefficients: orders p <= 7), N = K states (rounded
// up to 16) and 3 x the leaf's sources of reduction.  B is the moment
// operand the tensor-core near field already packs for the same evaluation:
// per block of 4 sources [3 components][hi, lo][N states][4 sources], TF32
// hi / lo in K-major core matrices, so this kernel adds no pass over the
// moments.  A is formed per sub-chunk of 8 sources: warp 0 writes each
// source's monomials of degree <= p - 1 into shared memory (the recurrences
// of monomials_part(), bit-identical to the FP32 P2M's), then thread alpha
// gathers its 24 entries, splits them x = hi + lo (hi = x rounded to TF32,
// lo = the rest rounded to TF32) and stores both into tensor memory, where
// the MMAs read A; per k-step of 8 three products A_hi B_hi + A_hi B_lo +
// A_lo B_hi accumulate in FP32 tensor memory (a leaf's ~45 MMAs in one
// accumulator: FP32-level accuracy).  The epilogue reads row alpha back
// (tcgen05.ld) and stores M[leaf][alpha][k].
//
// Every wait is bounded: on expiry the kernel records an error code, stops
// issuing, waits (full limit) for what it issued, writes NaN for the leaf's
// multipoles, frees its tensor memory and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "kernels.cuh"
#include "m2l_tc.hpp"
#include "p2m_tc.hpp"
#include "tcgen05.cuh"

namespace cdfmm_b200 {

namespace {

using namespace tc;

constexpr int kPtThreads = 128;      // thread = row alpha = tensor-memory lane
constexpr uint32_t kPtTmemCols = 128; // D: N <= 64 columns; A: 24 hi + 24 lo columns from column 64
constexpr uint32_t kPtACol = 64;
constexpr int kPtSub = 8;            // sources per sub-chunk (2 blocks, 3 k-steps)
constexpr int kPtMaxMono = 120;      // monomials of degree <= 6 (p <= 7)
constexpr uint32_t kPtMiscBytes = 128; // barriers and flags ahead of the ring
constexpr int kPtPosCap = 64;          // leaves of <= 64 blocks: positions staged by one bulk copy

struct PtArgs {
  const float4 *blk_pos; // [(n_blocks + 1) * 4] leaf-relative positions, .w: sorted index (-1: empty)
  const int *blk_off;    // [leaves + 1] first block of each leaf
  const uint8_t *b_ops;  // packed moment blocks, 96 N bytes each
  const int8_t *basis;   // [n][4] exponents
  float *M;              // [node][n][K]
  int *error_flag;
  int n, p, K, N, leaf_node_base, zero_block;
  uint32_t wait_limit;
};

// Bounded, polled wait (the phases a CTA waits for complete within a few
// microseconds).
__device__ __forceinline__ bool pt_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  return mbar_wait(bar, parity, limit);
}

__global__ void __launch_bounds__(kPtThreads, 4) p2m_tc_kernel(const PtArgs a) {
  extern __shared__ __align__(128) uint8_t smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int N = a.N;
  const uint32_t blk_bytes = 96u * static_cast<uint32_t>(N);
  const uint32_t slot_bytes = 2u * blk_bytes;
  // [barriers, flags: 128 B][ring: 2 slots x 2 blocks][monomials]; the
  // epilogue's rows reuse the ring and monomial area
  uint64_t *bfull = reinterpret_cast<uint64_t *>(smem);
  uint64_t *mdone = bfull + 2;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(mdone + 2);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
  int *last_copy = abort_flag + 1; // [2] last sub-chunk whose copies went into each slot
  uint64_t *pfull = reinterpret_cast<uint64_t *>(smem + 48);
  uint8_t *ring = smem + kPtMiscBytes;
  float *mono = reinterpret_cast<float *>(ring + 2 * slot_bytes); // [8][kPtMaxMono]
  float4 *spos = reinterpret_cast<float4 *>(mono + kPtSub * kPtMaxMono); // [kPtPosCap * 4] the leaf's positions

  const int leaf = blockIdx.x;
  const int b0 = a.blk_off[leaf];
  const int nb = a.blk_off[leaf + 1] - b0;
  const int subs = (nb + 1) / 2;
  const int q1 = a.p - 1; // monomial degree
  const bool staged = nb > 0 && nb <= kPtPosCap;

  // row alpha = tid: the monomial ranks it reads per component and its sign
  int ix[3] = {-1, -1, -1};
  float sign = 1.0F;
  if (tid < a.n) {
    const int ax = a.basis[4 * tid], ay = a.basis[4 * tid + 1], az = a.basis[4 * tid + 2];
    if (ax > 0) ix[0] = rank3(ax - 1, ay, az);
    if (ay > 0) ix[1] = rank3(ax, ay - 1, az);
    if (az > 0) ix[2] = rank3(ax, ay, az - 1);
    sign = ((ax + ay + az) & 1) ? -1.0F : 1.0F;
  }

  auto issue_copies = [&](int i) { // thread 0: sub-chunk i's two blocks into slot i & 1
    const int s = i & 1;
    uint8_t *dst = ring + static_cast<uint32_t>(s) * slot_bytes;
    mbar_expect_tx(&bfull[s], slot_bytes);
    for (int h = 0; h < 2; ++h) {
      const int g = 2 * i + h;
      const int blk = g < nb ? b0 + g : a.zero_block;
      bulk_g2s(dst + static_cast<uint32_t>(h) * blk_bytes, a.b_ops + static_cast<size_t>(blk) * blk_bytes, blk_bytes,
               &bfull[s]);
    }
    last_copy[s] = i;
  };

  if (tid == 0) {
    for (int s = 0; s < 2; ++s) {
      mbar_init(&bfull[s], 1);
      mbar_init(&mdone[s], 1);
    }
    mbar_init(pfull, 1);
    *abort_flag = 0;
    last_copy[0] = last_copy[1] = -1;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (staged) {
      // the leaf's block positions (contiguous, 64 bytes per block)
      mbar_expect_tx(pfull, static_cast<uint32_t>(nb) * 64u);
      bulk_g2s(spos, a.blk_pos + 4LL * b0, static_cast<uint32_t>(nb) * 64u, pfull);
    }
    if (subs > 0) issue_copies(0);
  }
  if (warp == 0) tmem_alloc(tmem_slot, kPtTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t lane_base = static_cast<uint32_t>(32 * warp) << 16;
  const uint32_t ta = tmem + lane_base + kPtACol;
  const uint32_t idesc = instr_desc_tf32(N);
  int issued = 0;

  for (int i = 0; i < subs; ++i) {
    const int s = i & 1;
    if (warp == 0) {
      // sub-chunk i's monomials while the MMAs of i - 1 run (their A was
      // formed from the previous monomials before they were issued): source
      // q = lane / 4 of the sub-chunk, part lane % 4 of its monomials
      const int q = lane >> 2;
      const int g = 2 * i + (q >> 2);
      float4 x = make_float4(0.0F, 0.0F, 0.0F, __int_as_float(-1));
      bool ok = true;
      if (i == 0 && staged) ok = pt_wait(pfull, 0, a.wait_limit);
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) {
          *abort_flag = 1;
          atomicExch(a.error_flag, 8);
        }
      } else if (g < nb) {
        x = staged ? spos[4 * g + (q & 3)] : a.blk_pos[4LL * (b0 + g) + (q & 3)];
      }
      monomials_part(x.x, x.y, x.z, q1, mono + q * kPtMaxMono, 1, lane & 3, __float_as_int(x.w) < 0);
    }
    if (tid == 0) {
      // the MMAs of sub-chunk i - 1 have completed: the A columns and slot
      // (i + 1) & 1 are free
      if (i >= 1 && *abort_flag == 0 &&
          !pt_wait(&mdone[(i - 1) & 1], static_cast<uint32_t>((i - 1) >> 1) & 1u, a.wait_limit)) {
        *abort_flag = 1;
        atomicExch(a.error_flag, 8);
      }
      if (*abort_flag == 0 && i + 1 < subs) issue_copies(i + 1);
    }
    __syncthreads();
    if (*reinterpret_cast<volatile int *>(abort_flag) != 0) break;
    tc_fence_after();
    float hv[24], lv[24];
#pragma unroll
    for (int q = 0; q < kPtSub; ++q)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        const float v = ix[d] >= 0 ? sign * mono[q * kPtMaxMono + ix[d]] : 0.0F;
        const int col = 12 * (q >> 2) + 4 * d + (q & 3);
        hv[col] = tf32_hi(v);
        lv[col] = tf32_hi(v - hv[col]);
      }
    tmem_st16(ta, hv);
    tmem_st8(ta + 16u, hv + 16);
    tmem_st16(ta + 24u, lv);
    tmem_st8(ta + 40u, lv + 16);
    tmem_wait_st();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      if (!pt_wait(&bfull[s], static_cast<uint32_t>(i >> 1) & 1u, a.wait_limit)) {
        *abort_flag = 1;
        atomicExch(a.error_flag, 8);
      } else {
        tc_fence_after();
        // B: core matrices 8 states x 4 sources, 8-state groups 128 bytes
        // apart (SBO), K-adjacent core matrices (next component, or the next
        // block's first) 32 N bytes apart (LBO); B_lo 16 N bytes after B_hi
        const uint64_t bd =
            smem_desc(smem_u32(ring) + static_cast<uint32_t>(s) * slot_bytes, 32u * static_cast<uint32_t>(N), 128u);
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const uint64_t bj = bd + ((2u * static_cast<uint32_t>(j) * 32u * static_cast<uint32_t>(N)) >> 4);
          const uint32_t ah = tmem + kPtACol + 8u * static_cast<uint32_t>(j);
          const uint32_t al = ah + 24u;
          mma_tf32_ts(tmem, ah, bj, idesc, (i > 0 || j > 0) ? 1u : 0u);
          mma_tf32_ts(tmem, ah, bj + ((16u * static_cast<uint32_t>(N)) >> 4), idesc, 1u);
          mma_tf32_ts(tmem, al, bj, idesc, 1u);
        }
        mma_commit(&mdone[s]);
        issued = i + 1;
      }
    }
  }
  if (tid == 0) {
    // every MMA issued has completed (full limit: the accumulator must be
    // quiet before it is read or freed); after an abort, the copies issued
    // and never consumed as well
    if (issued > 0 && !mbar_wait(&mdone[(issued - 1) & 1], static_cast<uint32_t>((issued - 1) >> 1) & 1u, kTcWaitLimit)) {
      *abort_flag = 1;
      atomicExch(a.error_flag, 8);
    }
    if (staged) mbar_wait(pfull, 0, kTcWaitLimit); // the position copy has landed (at once unless aborted)
    if (*abort_flag != 0)
      for (int s = 0; s < 2; ++s)
        if (last_copy[s] >= issued) mbar_wait(&bfull[s], static_cast<uint32_t>(last_copy[s] >> 1) & 1u, kTcWaitLimit);
  }
  __syncthreads();
  tc_fence_after();
  const bool poison = *reinterpret_cast<volatile int *>(abort_flag) != 0;
  // Rows through shared memory (the idle ring; row stride N + 1), then
  // stored along the leaf's [alpha][k] block so that consecutive threads
  // write consecutive words.
  float *stage = reinterpret_cast<float *>(ring);
  const int ss = N + 1;
  for (int c0 = 0; c0 < N; c0 += 16) {
    float v[16];
    tmem_ld16(tmem + lane_base + static_cast<uint32_t>(c0), v);
    if (tid < a.n) {
#pragma unroll
      for (int kk = 0; kk < 16; ++kk) stage[tid * ss + c0 + kk] = v[kk];
    }
  }
  __syncthreads();
  float *out = a.M + (static_cast<long long>(a.leaf_node_base) + leaf) * a.n * a.K;
  for (int e = tid; e < a.n * a.K; e += kPtThreads) {
    const int r = e / a.K;
    const int k = e - r * a.K;
    out[e] = poison ? __int_as_float(0x7fc00000) : (subs > 0 ? stage[r * ss + k] : 0.0F);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tmem, kPtTmemCols);
  }
}

size_t p2m_tc_smem(int N) {
  const size_t pipe = 2u * 2u * 96u * static_cast<size_t>(N) + sizeof(float) * kPtSub * kPtMaxMono +
                      sizeof(float4) * 4u * kPtPosCap;
  const size_t rows = sizeof(float) * static_cast<size_t>(kPtThreads) * static_cast<size_t>(N + 1);
  return kPtMiscBytes + std::max(pipe, rows);
}

} // namespace

bool p2m_tc_supported(int n, int K) { return n <= kPtThreads && K >= kNearTcMinStates && K <= kNearTcMaxStates; }

void launch_p2m_tc(const NearTcLaunch &ntc, const int8_t *basis, float *M, int n, int p, int K, int depth,
                   cudaStream_t s) {
  PtArgs args{};
  args.blk_pos = ntc.blk_pos;
  args.blk_off = ntc.blk_off;
  args.b_ops = static_cast<const uint8_t *>(ntc.b_ops);
  args.basis = basis;
  args.M = M;
  args.error_flag = ntc.error_flag;
  args.n = n;
  args.p = p;
  args.K = K;
  args.N = (K + 15) / 16 * 16;
  args.leaf_node_base = level_offset_d(depth);
  args.zero_block = ntc.n_blocks;
  args.wait_limit = ntc.wait_limit;
  // at most four CTAs per SM: their tensor memory (128 columns each) fills
  // the SM's 512, so a fifth would only wait in its allocation
  const size_t smem = std::max<size_t>(p2m_tc_smem(args.N), 52 * 1024);
  p2m_tc_kernel<<<1 << (3 * depth), kPtThreads, smem, s>>>(args);
}

bool configure_p2m_tc(size_t max_smem) {
  prefer_max_shared_carveout(p2m_tc_kernel);
  return allow_dynamic_smem(p2m_tc_kernel, max_smem);
}

} // namespace cdfmm_b200
