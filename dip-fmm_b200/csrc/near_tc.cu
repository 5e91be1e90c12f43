// List-1 near field of K >= 8 states on the 5th-generation tensor cores.
//
// For a work unit of up to 32 targets of one leaf and the sources of its
// 3x3x3 leaf neighbourhood (upstream list1, src/uniform_tree.cpp:455-480),
// the near field of every state is one matrix product
//
//   D[(c, t), k] = sum_(s, d) A[(c, t), (s, d)] * m_s[d][k]
//
// with rows (c, t) = (component, target), c = 0 the potential and c = 1..3
// the field components, and the pair tensors (r = x_t - x_s, upstream
// src/operators.cpp:178-199 without the 1/(4 pi))
//
//   A[(0, t), (s, d)] = r_d / |r|^3
//   A[(c, t), (s, d)] = 3 r_c r_d / |r|^5 - delta_(c, d) / |r|^3,
//
// so that phi = D[0] / (4 pi) and H_c = D[c] / (4 pi): 128 rows (an MMA M
// tile), N = K states (rounded up to 16), and 3 x sources of reduction.  It
// runs as kind::tf32 MMAs on split operands x = hi + lo (hi = x rounded to
// TF32, lo = x - hi, read by the tensor core as TF32) with the three
// products A_hi B_hi + A_hi B_lo + A_lo B_hi: the dropped A_lo B_lo and the
// truncation of lo are ~2^-21 of each product, FP32-level accuracy, with FP32
// accumulation in tensor memory.
//
// A is computed from positions in every evaluation (the reference stores its
// pair tensors per pair, src/static_operators.cpp:405-470) and never leaves
// the SM: four warps form the pair tensors of a chunk of 8 sources -- warp c
// the row block of component c, lane t target t -- and write them straight
// into tensor memory (tcgen05.st), where the MMA reads its A operand.  B is
// the moment operand: sources are grouped per leaf into blocks of 4, and
// each block's moments are pre-split (pack kernel) into TF32 hi / lo in the
// canonical K-major core-matrix layout ([3 components][N states][4 sources]),
// so a chunk's operand is four bulk copies (cp.async.bulk) of 48 N bytes plus
// the blocks' positions, issued by a producer warp into a ring of slots.
// One thread issues the MMAs (3 k-steps of 8 x 3 products per chunk) and
// commits each chunk to the slot's "empty" mbarrier; after the last chunk the
// four warps read D back (tcgen05.ld), scale it by 1/(4 pi) and store
// near[t][k] = (phi, Hx, Hy, Hz) through a shared-memory transpose.
//
// The pair vector r is formed exactly as the FP32 near-field kernels and the
// close-pair search form it (target - (source + neighbour offset)), so the
// close-pair correction applies unchanged.  The self pair and empty block
// slots get 1/|r| = 0; a coincident non-self pair gives NaN, as in the
// reference.  Every wait is bounded: on expiry the kernel records an error
// code, stops issuing, drains what it issued, writes NaN for its targets,
// frees its tensor memory and returns.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

#include "kernels.cuh"
#include "m2l_tc.hpp"
#include "near_tc.hpp"
#include "tcgen05.cuh"

namespace cdfmm_b200 {

namespace {

using namespace tc;

// Warp roles: 0-3 pair tensors (warp c: component c); 4 copies; 5 MMA issue
// and tensor-memory allocation; 6-9 accumulator drains and the epilogue.
// Pair-tensor warpgroups (chunks are dealt round robin): one with two
// CTAs per SM (256 tensor-memory columns each), or several with one CTA per
// SM (all 512 columns: more A slots).
#ifndef CDFMM_NTC_WG
#define CDFMM_NTC_WG 1
#endif
constexpr int kNtWg = CDFMM_NTC_WG;
constexpr int kNtCtasPerSm = kNtWg == 1 ? 2 : 1;
constexpr int kNtCopyWarp = 4 * kNtWg;
constexpr int kNtMmaWarp = kNtCopyWarp + 1;
constexpr int kNtDrainWarp = kNtCopyWarp + 2; // four drain warps
constexpr int kNtThreads = 32 * (kNtDrainWarp + 4);
constexpr uint32_t kNtTmemCols = kNtCtasPerSm == 2 ? 256 : 512;
constexpr int kNtStageStride = 33;    // epilogue transpose row (32 targets + 1)
constexpr int kNtPosCap = 384;        // neighbourhood blocks whose positions are staged in shared memory
// Blocks of 4 sources per pipeline chunk (even), and whether a k-step's
// hi x hi and hi x lo products run as one MMA of width 2 K (A_hi x
// [B_hi | B_lo]; twice the accumulator columns) or as two.
#ifndef CDFMM_NTC_CB
#define CDFMM_NTC_CB 4
#endif
#ifndef CDFMM_NTC_FUSE
#define CDFMM_NTC_FUSE 0
#endif
constexpr int kNtCB = CDFMM_NTC_CB;
constexpr bool kNtFuse = CDFMM_NTC_FUSE != 0;
constexpr int kNtAW = 24 * kNtCB;                                     // A-slot columns (hi, then lo)
constexpr int kNtBSlots = (kNtCtasPerSm == 2 ? 8 : 16) / kNtCB;        // moment operand ring
constexpr uint32_t kNtMiscBytes = 640;

// Chunks (8 sources, 9 MMAs) accumulated in one tensor-memory buffer before
// the drain warps add it into their FP32 registers: the tensor core's
// accumulation is not round-to-nearest, so its error grows with the number
// of MMAs summed into one accumulator at its magnitude.
#ifndef CDFMM_NTC_GROUP
#define CDFMM_NTC_GROUP 2
#endif

// Accumulator buffers: 2 (the MMAs of the next group run while a group is
// drained) or 1 (more A slots; the MMAs wait for each drain).
#ifndef CDFMM_NTC_DBUF
#define CDFMM_NTC_DBUF 1
#endif
constexpr int kNtDBuf = CDFMM_NTC_DBUF;

__host__ __device__ inline int nt_N(int K) { return (K + 15) / 16 * 16; }
// A-operand slots in tensor memory after the accumulators (2 N columns
// each: hi x [B_hi | B_lo] side by side), 48 columns each (24 hi + 24 lo).
__host__ __device__ inline int nt_acc_cols(int N) { return kNtFuse ? 2 * N : N; }
__host__ __device__ inline int nt_slots(int N) {
  const int s = (static_cast<int>(kNtTmemCols) - kNtDBuf * nt_acc_cols(N)) / kNtAW;
  return s < 8 ? s : 8;
}

struct NtSmem {
  uint32_t slot_bytes; // 2 blocks of [3 components][hi, lo][N states][4 sources]
  uint32_t pos_off;    // staged neighbourhood positions [kNtPosCap + 1][4] float4, then [4 kNtWg][8] scratch
  uint32_t stage_off;  // epilogue transpose [4 components][16 states][33]
  uint32_t bar_off;
  uint32_t misc_off;
  uint32_t total;
};
__host__ __device__ inline NtSmem nt_smem(int N, int SA) {
  NtSmem m;
  m.slot_bytes = 96u * kNtCB * static_cast<uint32_t>(N);
  m.pos_off = kNtBSlots * m.slot_bytes;
  m.stage_off = m.pos_off + (kNtPosCap + kNtCB) * 64u + 4u * kNtWg * 128u;
  m.bar_off = m.stage_off + 4u * 16u * kNtStageStride * 4u;
  m.misc_off = m.bar_off + (2u * kNtBSlots + 2u * static_cast<uint32_t>(SA) + 6u) * 8u;
  m.total = m.misc_off + kNtMiscBytes;
  return m;
}

struct NtArgs {
  const float4 *blk_pos;
  const int *blk_off;
  const uint8_t *b_ops;
  const int4 *work;
  const float4 *tgt_rel;
  const int *self_idx;
  float4 *near;
  int *error_flag;
  int depth, K, N, slots, want_phi, zero_block;
  uint32_t wait_limit;
};

// Veltkamp split of two values: hi keeps 11 significant bits (exactly a
// TF32 value), lo = x - hi exactly; FP32x2 arithmetic on the FMA pipe.
__device__ __forceinline__ void split_tf32x2(float2 x, float2 &hi, float2 &lo) {
  const float2 gamma = __fmul2_rn(x, make_float2(8193.0F, 8193.0F)); // 2^13 + 1
  const float2 delta = __ffma2_rn(gamma, make_float2(-1.0F, -1.0F), x);
  hi = __fadd2_rn(gamma, delta);
  lo = __ffma2_rn(hi, make_float2(-1.0F, -1.0F), x);
}

// Pair tensors of component C (0: potential, 1..3: field x, y, z) for one
// target and the 8 sources of a chunk (positions relative to this leaf's
// centre: source + neighbour offset), as TF32 hi / lo columns
// 12 b + 4 d + q (b: block, d: moment component, q: source in the block).
// With d = source - target (= -r, formed as -(target - source) is, bit for
// bit):
//   C = 0:  A_d = -d_d / |d|^3
//   C > 0:  A_d = 3 d_C d_d / |d|^5 - delta_(C, d) / |d|^3.
// The self source gets 1/|d| = 0; an empty slot lies 3e18 away (every
// entry underflows to zero).  Four independent FP32x2 source pairs.
template <int C>
__device__ __forceinline__ void chunk_tensors(const float4 *p8, float ntx, float nty, float ntz, int self, float *hv,
                                              float *lv) {
#pragma unroll
  for (int pr = 0; pr < 4; ++pr) {
    const float4 p0 = p8[2 * pr], p1 = p8[2 * pr + 1];
    const float2 dx = __fadd2_rn(make_float2(p0.x, p1.x), make_float2(ntx, ntx));
    const float2 dy = __fadd2_rn(make_float2(p0.y, p1.y), make_float2(nty, nty));
    const float2 dz = __fadd2_rn(make_float2(p0.z, p1.z), make_float2(ntz, ntz));
    const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    rinv.x = __float_as_int(p0.w) == self ? 0.0F : rinv.x;
    rinv.y = __float_as_int(p1.w) == self ? 0.0F : rinv.y;
    const float2 rinv2 = __fmul2_rn(rinv, rinv);
    const float2 v = __fmul2_rn(rinv2, rinv);
    const float2 nv = __fmul2_rn(v, make_float2(-1.0F, -1.0F));
    float2 e[3];
    if constexpr (C == 0) {
      e[0] = __fmul2_rn(dx, nv);
      e[1] = __fmul2_rn(dy, nv);
      e[2] = __fmul2_rn(dz, nv);
    } else {
      const float2 f = __fmul2_rn(__fmul2_rn(v, rinv2), make_float2(3.0F, 3.0F));
      const float2 g = __fmul2_rn(f, C == 1 ? dx : (C == 2 ? dy : dz));
      e[0] = C == 1 ? __ffma2_rn(g, dx, nv) : __fmul2_rn(g, dx);
      e[1] = C == 2 ? __ffma2_rn(g, dy, nv) : __fmul2_rn(g, dy);
      e[2] = C == 3 ? __ffma2_rn(g, dz, nv) : __fmul2_rn(g, dz);
    }
    const int col = 12 * (pr >> 1) + 2 * (pr & 1);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float2 hi, lo;
      split_tf32x2(e[d], hi, lo);
      hv[col + 4 * d] = hi.x;
      hv[col + 4 * d + 1] = hi.y;
      lv[col + 4 * d] = lo.x;
      lv[col + 4 * d + 1] = lo.y;
    }
  }
}

__device__ __forceinline__ float4 far_slot() {
  return make_float4(3.0e18F, 3.0e18F, 3.0e18F, __int_as_float(-1));
}

__device__ __forceinline__ void agen_bar() { asm volatile("bar.sync 2, %0;" ::"r"(128 * kNtWg) : "memory"); }

// Waits of the pipeline: hardware-suspended (1) or polled with short
// sleeps (0).
#ifndef CDFMM_NTC_SUSPEND
#define CDFMM_NTC_SUSPEND 1
#endif
__device__ __forceinline__ bool nt_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  // a suspended poll lasts up to ~1 us: the iteration budget is scaled so
  // the bound stays near the polled one (limit 0 still expires at once)
  if (CDFMM_NTC_SUSPEND) return mbar_wait_suspend(bar, parity, limit > 32u ? limit >> 5 : limit, 1000u);
  return mbar_wait_sleepy(bar, parity, limit, 32);
}

__device__ __forceinline__ void drain_bar() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Records an expired wait (code) and raises the CTA's abort flag.
__device__ __forceinline__ void nt_abort(int *abort_flag, int *error_flag, int code) {
  *abort_flag = 1;
  atomicExch(error_flag, code);
}
__device__ __forceinline__ bool nt_aborted(const int *abort_flag) {
  return *reinterpret_cast<const volatile int *>(abort_flag) != 0;
}

__global__ void __launch_bounds__(kNtThreads, kNtCtasPerSm) near_tc_kernel(const NtArgs a) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int N = a.N;
  const int SA = a.slots;
  constexpr int SB = kNtBSlots;
  constexpr int G = CDFMM_NTC_GROUP;
  const NtSmem lay = nt_smem(N, SA);
  float4 *spos = reinterpret_cast<float4 *>(smem + lay.pos_off);
  float *stage = reinterpret_cast<float *>(smem + lay.stage_off);
  uint64_t *bfull = reinterpret_cast<uint64_t *>(smem + lay.bar_off);
  uint64_t *bempty = bfull + SB;
  uint64_t *aready = bempty + SB;
  uint64_t *aempty = aready + SA;
  uint64_t *dready = aempty + SA; // [2]
  uint64_t *dfree = dready + 2;   // [2]
  uint64_t *pfull = dfree + 2;
  uint64_t *done = pfull + 1;
  int *misc = reinterpret_cast<int *>(smem + lay.misc_off);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(misc);
  int *abort_flag = misc + 1;
  int *nb_count = misc + 2;
  int *last_chunk = misc + 4;     // [kNtBSlots] last chunk whose copies were issued into each slot
  int *nb_first = misc + 12;      // [27] first block of each non-empty neighbour leaf
  int *nb_prefix = nb_first + 27; // [28] neighbourhood block prefix
  float *nb_off = reinterpret_cast<float *>(nb_prefix + 28); // [27][3] neighbour centre - this centre

  const int4 unit = a.work[blockIdx.x];
  const int leaf = unit.x;
  const int t0 = unit.y;
  const int nt = unit.z;
  const uint32_t blk_bytes = 96u * static_cast<uint32_t>(N); // hi and lo of one block

  if (tid == 0) {
    for (int s = 0; s < SB; ++s) {
      mbar_init(&bfull[s], 1);
      mbar_init(&bempty[s], 1);
    }
    for (int s = 0; s < SA; ++s) {
      mbar_init(&aready[s], 4);
      mbar_init(&aempty[s], 1);
    }
    for (int d = 0; d < 2; ++d) {
      mbar_init(&dready[d], 1);
      mbar_init(&dfree[d], 4);
    }
    mbar_init(pfull, 1);
    mbar_init(done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < kNtBSlots) last_chunk[tid] = -1;
  if (warp == kNtCopyWarp) {
    // The clipped 3x3x3 neighbourhood, z outermost and x fastest; the
    // leaves with sources compacted in that order with their block counts.
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
  if (warp == kNtMmaWarp) tmem_alloc(tmem_slot, kNtTmemCols);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int n_nb = *nb_count;
  const int n_blk = nb_prefix[n_nb];
  const int chunks = (n_blk + kNtCB - 1) / kNtCB;
  const int groups = (chunks + G - 1) / G;
  const bool staged = n_blk <= kNtPosCap; // positions in shared memory (else read from global memory)
  const uint32_t acc_cols = static_cast<uint32_t>(nt_acc_cols(N));
  const uint32_t acol0 = kNtDBuf * acc_cols; // first A slot column

  if (warp == kNtCopyWarp) {
    // Copies: the neighbourhood's positions once (one bulk copy per leaf),
    // then chunk i's moment blocks (2i, 2i + 1; the empty block pads an odd
    // count) into ring slot i % SB once the MMAs of chunk i - SB released it.
    if (staged) {
      if (lane == 0) mbar_expect_tx(pfull, static_cast<uint32_t>(n_blk) * 64u);
      __syncwarp();
      if (lane < n_nb) {
        const int cnt = nb_prefix[lane + 1] - nb_prefix[lane];
        bulk_g2s(spos + 4 * nb_prefix[lane], a.blk_pos + 4LL * nb_first[lane], static_cast<uint32_t>(cnt) * 64u, pfull);
      }
    }
    int nbi = 0;
    for (int i = 0; i < chunks; ++i) {
      const int s = i % SB;
      int ok = 1;
      if (lane == 0) {
        if (i >= SB && !nt_wait(&bempty[s], static_cast<uint32_t>((i / SB) - 1) & 1u, a.wait_limit))
          nt_abort(abort_flag, a.error_flag, 4);
        ok = !nt_aborted(abort_flag);
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      // block of this lane (lanes < kNtCB): neighbourhood block CB i + lane
      int blk = a.zero_block;
      for (int b = 0; b < kNtCB; ++b) {
        const int g = kNtCB * i + b;
        if (g < n_blk) {
          while (nbi + 1 < n_nb && nb_prefix[nbi + 1] <= g) ++nbi;
          if (lane == b) blk = nb_first[nbi] + (g - nb_prefix[nbi]);
        }
      }
      uint8_t *st = smem + static_cast<uint32_t>(s) * lay.slot_bytes;
      if (lane == 0) mbar_expect_tx(&bfull[s], kNtCB * blk_bytes);
      __syncwarp();
      if (lane < kNtCB)
        bulk_g2s(st + static_cast<uint32_t>(lane) * blk_bytes, a.b_ops + static_cast<size_t>(blk) * blk_bytes, blk_bytes,
                 &bfull[s]);
      __syncwarp();
      if (lane == 0) last_chunk[s] = i;
    }
  } else if (warp == kNtMmaWarp) {
    // MMA issuer: chunk i adds A_(i % SA) x B_(i % SB) into accumulator
    // (i / G) % kNtDBuf, which a group's first MMA overwrites once the drain
    // of that buffer's previous group freed it.  Per k-step of 8 two MMAs:
    // A_hi x [B_hi | B_lo] (N = 2 N: columns [0, N) hi x hi, [N, 2 N)
    // hi x lo) and A_lo x B_hi (N, onto columns [0, N)); the drain adds the
    // halves.  B descriptors: core matrices 8 states x 4 sources, the
    // 16 hi and lo state groups 128 bytes apart (SBO), K-adjacent core
    // matrices 32 N bytes apart (LBO).
    if (lane == 0) {
      const uint32_t idesc = instr_desc_tf32(N);
      const uint32_t idesc2 = instr_desc_tf32(2 * N);
      const uint64_t desc0 = smem_desc(smem_u32(smem), 32u * static_cast<uint32_t>(N), 128u);
      for (int i = 0; i < chunks; ++i) {
        const int sb = i % SB;
        const int sa = i % SA;
        const int gi = i / G;
        const int db = gi % kNtDBuf;
        const bool first = i % G == 0;
        if (first && gi >= kNtDBuf &&
            !nt_wait(&dfree[db], static_cast<uint32_t>((gi / kNtDBuf) - 1) & 1u, a.wait_limit)) {
          nt_abort(abort_flag, a.error_flag, 5);
          break;
        }
        if (!nt_wait(&bfull[sb], static_cast<uint32_t>(i / SB) & 1u, a.wait_limit) ||
            !nt_wait(&aready[sa], static_cast<uint32_t>(i / SA) & 1u, a.wait_limit)) {
          nt_abort(abort_flag, a.error_flag, 5);
          break;
        }
        tc_fence_after();
        const uint32_t dcol = tmem + static_cast<uint32_t>(db) * acc_cols;
        const uint64_t bd = desc0 + ((static_cast<uint32_t>(sb) * lay.slot_bytes) >> 4);
        const uint32_t acol = tmem + acol0 + kNtAW * static_cast<uint32_t>(sa);
#pragma unroll
        for (int j = 0; j < 3 * kNtCB / 2; ++j) {
          const uint64_t bj = bd + ((2u * static_cast<uint32_t>(j) * 32u * static_cast<uint32_t>(N)) >> 4);
          const uint32_t ah = acol + 8u * static_cast<uint32_t>(j);
          const uint32_t al = ah + 12u * kNtCB;
          if (kNtFuse) {
            mma_tf32_ts(dcol, ah, bj, idesc2, (first && j == 0) ? 0u : 1u);
          } else {
            mma_tf32_ts(dcol, ah, bj, idesc, (first && j == 0) ? 0u : 1u);
            mma_tf32_ts(dcol, ah, bj + ((16u * static_cast<uint32_t>(N)) >> 4), idesc, 1); // B_lo
          }
          mma_tf32_ts(dcol, al, bj, idesc, 1);
        }
        mma_commit(&bempty[sb]);
        mma_commit(&aempty[sa]);
        if (i % G == G - 1 || i == chunks - 1) mma_commit(&dready[db]);
      }
      // arrives once every MMA issued above has completed
      mma_commit(done);
    }
    __syncwarp();
  } else if (warp < 4 * kNtWg) {
    // Pair tensors: warpgroup wg takes chunks wg, wg + kNtWg, ...; in it
    // warp c forms the row block of component c, lane t target t.
    const int c = warp & 3;
    const int wg = warp >> 2;
    const int it = t0 + (lane < nt ? lane : 0); // lanes beyond the unit's targets: rows never stored
    const float4 tp = a.tgt_rel[it];
    const float ntx = -tp.x, nty = -tp.y, ntz = -tp.z;
    const int self = (a.self_idx != nullptr && lane < nt) ? a.self_idx[it] : -2;
    const uint32_t lane_base = static_cast<uint32_t>(32 * c) << 16;
    bool ok = true;
    if (staged && chunks > 0) ok = nt_wait(pfull, 0, a.wait_limit);
    ok = __all_sync(0xffffffffu, ok);
    if (!ok && lane == 0) nt_abort(abort_flag, a.error_flag, 6);
    const int at = tid; // 0 .. 128 kNtWg - 1 over the pair-tensor warps
    if (staged) {
      // Staged positions += their leaf's offset (as the FP32 near field
      // forms source positions), and an empty block after the last one.
      if (ok)
        for (int e = at; e < 4 * n_blk; e += 128 * kNtWg) {
          const int g = e >> 2;
          int n = 0;
          while (n + 1 < n_nb && nb_prefix[n + 1] <= g) ++n;
          const float4 q = spos[e];
          spos[e] = make_float4(q.x + nb_off[3 * n], q.y + nb_off[3 * n + 1], q.z + nb_off[3 * n + 2], q.w);
        }
      if (at < 4 * kNtCB) spos[4 * n_blk + at] = far_slot();
      agen_bar();
    }
    float4 *scratch = spos + 4 * (kNtPosCap + kNtCB) + 8 * warp; // this warp's 8 positions (unstaged)
    for (int i = wg; ok && i < chunks; i += kNtWg) {
      const int sa = i % SA;
      // the MMAs that read this slot's previous A (chunk i - SA) have completed
      bool free_slot = i < SA || nt_wait(&aempty[sa], static_cast<uint32_t>((i / SA) - 1) & 1u, a.wait_limit);
      free_slot = __all_sync(0xffffffffu, free_slot);
      int go = free_slot ? 1 : 0;
      if (lane == 0) {
        if (!free_slot) nt_abort(abort_flag, a.error_flag, 6);
        go = go && !nt_aborted(abort_flag);
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
      tc_fence_after();
      const uint32_t ta = tmem + lane_base + acol0 + kNtAW * static_cast<uint32_t>(sa);
      // the chunk in sub-chunks of 8 sources (2 blocks): k columns 24 h ...
      for (int h = 0; h < kNtCB / 2; ++h) {
        const int g0 = kNtCB * i + 2 * h; // first block of the sub-chunk
        const float4 *p8 = spos + 4 * g0;
        if (!staged) {
          // a neighbourhood beyond the staging capacity: lane q < 8 forms
          // position q of the sub-chunk from global memory
          if (lane < 8) {
            const int g = g0 + (lane >> 2);
            float4 q = far_slot();
            if (g < n_blk) {
              int n = 0;
              while (n + 1 < n_nb && nb_prefix[n + 1] <= g) ++n;
              q = a.blk_pos[4LL * (nb_first[n] + (g - nb_prefix[n])) + (lane & 3)];
              q = make_float4(q.x + nb_off[3 * n], q.y + nb_off[3 * n + 1], q.z + nb_off[3 * n + 2], q.w);
            }
            scratch[lane] = q;
          }
          __syncwarp();
          p8 = scratch;
        }
        float hv[24], lv[24];
        switch (c) {
        case 0: chunk_tensors<0>(p8, ntx, nty, ntz, self, hv, lv); break;
        case 1: chunk_tensors<1>(p8, ntx, nty, ntz, self, hv, lv); break;
        case 2: chunk_tensors<2>(p8, ntx, nty, ntz, self, hv, lv); break;
        default: chunk_tensors<3>(p8, ntx, nty, ntz, self, hv, lv); break;
        }
        if (!staged) __syncwarp(); // scratch reads done before the next sub-chunk overwrites it
        const uint32_t th = ta + 24u * static_cast<uint32_t>(h);
        tmem_st16(th, hv);
        tmem_st8(th + 16u, hv + 16);
        tmem_st16(th + 12u * kNtCB, lv);
        tmem_st8(th + 12u * kNtCB + 16u, lv + 16);
      }
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&aready[sa]);
    }
  } else if (warp >= kNtDrainWarp) {
    // Drains: warp kNtDrainWarp + r reads the rows of tensor-memory
    // sub-partition c = warp % 4 (component c of targets = lanes) and adds each
    // group's accumulator into FP32 registers; then the epilogue stores
    // near[t][k] = (phi, Hx, Hy, Hz) / 4 pi through a shared-memory transpose.
    const int c = warp & 3;
    const uint32_t lane_base = static_cast<uint32_t>(32 * c) << 16;
    float acc[4][16];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int kk = 0; kk < 16; ++kk) acc[q][kk] = 0.0F;
    for (int gi = 0; gi < groups; ++gi) {
      const int db = gi % kNtDBuf;
      bool ok = nt_wait(&dready[db], static_cast<uint32_t>(gi / kNtDBuf) & 1u, a.wait_limit);
      ok = __all_sync(0xffffffffu, ok);
      int go = ok ? 1 : 0;
      if (lane == 0) {
        if (!ok) nt_abort(abort_flag, a.error_flag, 7);
        go = go && !nt_aborted(abort_flag);
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
      tc_fence_after();
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (16 * q < N) {
#pragma unroll
          for (int h = 0; h < (kNtFuse ? 2 : 1); ++h) {
            float v[16];
            tmem_ld16(tmem + lane_base + static_cast<uint32_t>(db) * acc_cols + static_cast<uint32_t>(h * N + 16 * q), v);
#pragma unroll
            for (int kk = 0; kk < 16; ++kk) acc[q][kk] += v[kk];
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&dfree[db]);
    }
    // every MMA has completed (full limit: the accumulators must be quiet
    // before the tensor memory is freed)
    bool quiet = mbar_wait(done, 0, kTcWaitLimit);
    quiet = __all_sync(0xffffffffu, quiet);
    int poison = quiet ? 0 : 1;
    if (lane == 0) {
      if (!quiet) nt_abort(abort_flag, a.error_flag, 7);
      poison = poison || nt_aborted(abort_flag);
    }
    poison = __shfl_sync(0xffffffffu, poison, 0);
    const float scale = (c == 0 && !a.want_phi) ? 0.0F : kInvFourPiF;
    const int et = tid - 32 * kNtDrainWarp; // 0..127 over the drain warps
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (16 * q < N) {
#pragma unroll
        for (int kk = 0; kk < 16; ++kk)
          stage[(c * 16 + kk) * kNtStageStride + lane] = poison ? __int_as_float(0x7fc00000) : acc[q][kk] * scale;
        drain_bar();
        for (int e = et; e < 32 * 16; e += 128) {
          const int tt = e >> 4;
          const int kk = e & 15;
          const int k = 16 * q + kk;
          if (tt < nt && k < a.K)
            a.near[static_cast<long long>(t0 + tt) * a.K + k] =
                make_float4(stage[kk * kNtStageStride + tt], stage[(16 + kk) * kNtStageStride + tt],
                            stage[(32 + kk) * kNtStageStride + tt], stage[(48 + kk) * kNtStageStride + tt]);
        }
        drain_bar();
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (nt_aborted(abort_flag) && tid < 32) {
    // Abort: copies issued and never consumed may still be in flight; wait
    // for them (full limit) before the shared memory is released.
    if (tid < SB) {
      const int u = last_chunk[tid];
      if (u >= 0) mbar_wait(&bfull[tid], static_cast<uint32_t>(u / SB) & 1u, kTcWaitLimit);
    }
    if (tid == SB && staged && chunks > 0) mbar_wait(pfull, 0, kTcWaitLimit);
  }
  __syncthreads();
  if (warp == kNtMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem, kNtTmemCols);
  }
}

// Moments -> TF32 hi / lo blocks [block][3 components][hi, lo][N states][4
// sources]; states k >= K and empty slots are zero.  Thread per (block,
// component, state): one float4 of each of hi and lo (consecutive threads
// write consecutive 16 bytes).
template <bool PAIRED>
__global__ void __launch_bounds__(256) near_tc_pack_kernel(const float4 *__restrict__ mom,
                                                           const int *__restrict__ blk_src, long long total, int K,
                                                           int N, float4 *__restrict__ ops) {
  const long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const int k = static_cast<int>(e % N);
  const long long bd = e / N;
  const int d = static_cast<int>(bd % 3);
  const long long b = bd / 3;
  float v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int j = blk_src[4 * b + q];
    float m = 0.0F;
    if (j >= 0 && k < K) {
      if constexpr (PAIRED) {
        const float4 *row = mom + static_cast<long long>(j) * ((K + 1) & ~1) + (k & ~1);
        if (d < 2) {
          const float4 r0 = row[0];
          m = d == 0 ? ((k & 1) ? r0.y : r0.x) : ((k & 1) ? r0.w : r0.z);
        } else {
          const float4 r1 = row[1];
          m = (k & 1) ? r1.y : r1.x;
        }
      } else {
        const float4 r = mom[static_cast<long long>(j) * K + k];
        m = d == 0 ? r.x : (d == 1 ? r.y : r.z);
      }
    }
    v[q] = m;
  }
  float h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    h[q] = tf32_hi(v[q]);
    l[q] = tf32_hi(v[q] - h[q]);
  }
  ops[2 * bd * N + k] = make_float4(h[0], h[1], h[2], h[3]);
  ops[(2 * bd + 1) * N + k] = make_float4(l[0], l[1], l[2], l[3]);
}

__global__ void __launch_bounds__(256) near_tc_positions_kernel(const float4 *__restrict__ src_rel,
                                                                const int *__restrict__ blk_src, int slots,
                                                                float4 *__restrict__ blk_pos) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= slots) return;
  const int j = blk_src[e];
  if (j >= 0) {
    const float4 p = src_rel[j];
    blk_pos[e] = make_float4(p.x, p.y, p.z, __int_as_float(j));
  } else {
    // an empty slot lies far from every target: its pair tensor underflows to 0
    blk_pos[e] = make_float4(3.0e18F, 3.0e18F, 3.0e18F, __int_as_float(-1));
  }
}

} // namespace

NearTcLayout near_tc_layout(const int *src_off, const int *tgt_off, int depth) {
  NearTcLayout lay;
  const int leaves = 1 << (3 * depth);
  lay.blk_off.assign(static_cast<size_t>(leaves) + 1, 0);
  for (int l = 0; l < leaves; ++l) {
    const int cnt = src_off[l + 1] - src_off[l];
    lay.blk_off[static_cast<size_t>(l) + 1] = lay.blk_off[static_cast<size_t>(l)] + (cnt + kNearTcSlots - 1) / kNearTcSlots;
  }
  lay.n_blocks = lay.blk_off[static_cast<size_t>(leaves)];
  lay.blk_src.assign(static_cast<size_t>(lay.n_blocks + 1) * kNearTcSlots, -1);
  for (int l = 0; l < leaves; ++l)
    for (int j = src_off[l]; j < src_off[l + 1]; ++j) {
      const int q = j - src_off[l];
      lay.blk_src[static_cast<size_t>(lay.blk_off[static_cast<size_t>(l)]) * kNearTcSlots + static_cast<size_t>(q)] = j;
    }
  // Work units of <= 32 targets; cost = neighbourhood blocks (MMA work).
  const int side = 1 << depth;
  for (int l = 0; l < leaves; ++l) {
    const int tn = tgt_off[l + 1] - tgt_off[l];
    if (tn == 0) continue;
    int ix, iy, iz;
    demorton3(static_cast<uint32_t>(l), ix, iy, iz);
    int cost = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = ix + dx, y = iy + dy, z = iz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= side || y >= side || z >= side) continue;
          const uint32_t m = morton3(static_cast<uint32_t>(x), static_cast<uint32_t>(y), static_cast<uint32_t>(z));
          cost += lay.blk_off[m + 1] - lay.blk_off[m];
        }
    for (int t = 0; t < tn; t += kNearTcTargets) {
      lay.work.push_back(make_int4(l, tgt_off[l] + t, std::min(kNearTcTargets, tn - t), cost));
      lay.k_cols += 3u * 4u * static_cast<uint64_t>(kNtCB) * static_cast<uint64_t>((cost + kNtCB - 1) / kNtCB);
    }
  }
  return lay;
}

size_t near_tc_operand_bytes(int n_blocks, int K) {
  return static_cast<size_t>(n_blocks + 1) * 96u * static_cast<size_t>(nt_N(std::max(K, 1)));
}

void launch_near_tc_positions(const float4 *src_rel, const int *blk_src, int n_blocks, float4 *blk_pos,
                              cudaStream_t s) {
  const int slots = (n_blocks + 1) * kNearTcSlots;
  near_tc_positions_kernel<<<(slots + 255) / 256, 256, 0, s>>>(src_rel, blk_src, slots, blk_pos);
}

void launch_near_tc_pack(const NearTcLaunch &a, const float4 *mom, int K, cudaStream_t s) {
  if (K < kNearTcMinStates || K > kNearTcMaxStates) return;
  const int N = nt_N(K);
  const long long total = static_cast<long long>(a.n_blocks + 1) * 3 * N;
  const unsigned grid = static_cast<unsigned>((total + 255) / 256);
  near_tc_pack_kernel<true><<<grid, 256, 0, s>>>(mom, a.blk_src, total, K, N, static_cast<float4 *>(a.b_ops));
}

void launch_near_tc(const NearTcLaunch &a, const float4 *mom, const float4 *tgt_rel, const int *self_idx, int depth,
                    int K, bool want_phi, float4 *near, cudaStream_t s) {
  if (a.n_work == 0 || K < kNearTcMinStates || K > kNearTcMaxStates) return;
  const int N = nt_N(K);
  if (!a.packed) launch_near_tc_pack(a, mom, K, s);
  NtArgs args{};
  args.blk_pos = a.blk_pos;
  args.blk_off = a.blk_off;
  args.b_ops = static_cast<const uint8_t *>(a.b_ops);
  args.work = a.work;
  args.tgt_rel = tgt_rel;
  args.self_idx = self_idx;
  args.near = near;
  args.error_flag = a.error_flag;
  args.depth = depth;
  args.K = K;
  args.N = N;
  args.slots = nt_slots(N);
  args.want_phi = want_phi ? 1 : 0;
  args.zero_block = a.n_blocks;
  args.wait_limit = a.wait_limit;
  // Enough shared memory per CTA that no more CTAs than the tensor memory
  // holds share an SM (the extra one's allocation would wait for ours).
  const size_t smem = std::max<size_t>(nt_smem(N, args.slots).total, kNtCtasPerSm == 2 ? 80 * 1024 : 116 * 1024);
  near_tc_kernel<<<a.n_work, kNtThreads, smem, s>>>(args);
}

bool configure_near_tc(size_t max_smem) {
  prefer_max_shared_carveout(near_tc_kernel);
  return allow_dynamic_smem(near_tc_kernel, max_smem);
}

} // namespace cdfmm_b200
