// M2L on the 5th-generation tensor cores (tcgen05), split BF16 with FP32
// accumulation in tensor memory (K states per call; fewer than 8 fill an
// 8-row group of each MMA tile with zero rows).
//
// For one level, parity class c and a tile of T targets (rows = target x
// state, 128 rows = one MMA M tile), the kernel accumulates over the 189 list2
// offsets o of class c (implicit list2, see m2l_simt.cu):
//
//   D[(t, k), beta] += sum_alpha A_o[(t, k), alpha] * B_o[beta, alpha]
//   A_o[(t, k), alpha] = 2^(l|alpha|) M'_alpha(t - o, state k)   (exact scaling)
//   B_o[beta, alpha]   = T^(o)[beta][alpha] = D^{alpha+beta} G(o)
//
// on the traceless-reduced operator (M2lTraceless): alpha runs over the
// (p+1)^2 - 1 folded moments M' (alpha_z <= 1, the monopole left out) and
// beta over the (p+1)^2 locals with beta_z <= 1, an exact sub-block of the
// full matrix; each operand is split x = hi + lo in BF16 with three products
// A_hi*B_hi + A_hi*B_lo + A_lo*B_hi (the dropped lo*lo term is ~2^-16 of the
// product), then the epilogue forms the other locals from the trace
// relations and stores L = 2^(l(|beta|+1)) D for all n coefficients
// (upstream math: docs/math.md "M2L normalisation and cross-level reuse").
//
// Data movement: a producer warp issues bulk async copies (cp.async.bulk, TMA
// engine) of each source box's rows (contiguous, already in the canonical
// no-swizzle K-major core-matrix layout written by the pack kernel) and of the
// offset's B tile (pre-tiled on the host), completing on the stage's "full"
// mbarrier; one thread issues tcgen05.mma from shared memory into the TMEM
// accumulators and commits to the stage's "empty" mbarrier, which frees it.
// A pipeline unit is one offset and one 32-wide alpha chunk, so 4-8 stages
// fit in shared memory and copies run several units ahead of the MMAs.
// Every wait is bounded: on expiry the kernel records an error code, stops
// issuing, drains what it issued (those waits always keep the full limit, so
// no copy or MMA is still in flight when the CTA exits), writes NaN into its
// targets' locals (stale values of an earlier call never pass for results),
// frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "far_kernels.hpp"
#include "kernels.cuh"
#include "m2l_tc.hpp"
#include "tcgen05.cuh"

namespace cdfmm_b200 {

namespace {

constexpr int kTcThreads = 128;
constexpr uint32_t kWaitLimit = kTcWaitLimit; // ~2 s with the back-off below
constexpr int kKChunk = 32;               // alphas per pipeline unit

using tc::bulk_g2s;
using tc::fence_proxy_async;
using tc::instr_desc_bf16;
using tc::mbar_expect_tx;
using tc::mbar_init;
using tc::mma_bf16;
using tc::mma_commit;
using tc::smem_desc;
using tc::smem_u32;
using tc::tc_fence_after;
using tc::tc_fence_before;
using tc::tmem_ld16;

// Bounded wait (by default with the full limit).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = kWaitLimit) {
  return tc::mbar_wait(bar, parity, limit);
}

// Pipeline unit = (offset, alpha chunk of kKChunk = 32, the last chunk
// possibly 16 wide): up to two MMA k-steps on each of the CTA's m_tiles
// accumulators, which share the unit's B tile.  Shared-memory operand layout
// of a chunk of width w (no swizzle, K-major, 8x16-byte core matrices):
//   [row group][w/8 column blocks][8 rows][8 alphas]  -> LBO 128 B, SBO w*16 B
// for A (128 rows per M tile) and for B (Npad rows = betas).  Stage =
// [A_hi x m_tiles][A_lo x m_tiles][B_hi][B_lo].  Global operands hold each
// chunk in the same order, so one source box's rows of one chunk are one
// contiguous bulk copy; lanes of the producer warp issue a unit's copies in
// parallel.
template <int MT>
__global__ void __launch_bounds__(kTcThreads, 1) m2l_tc_kernel(const TcArgs args) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int4 tile = args.tiles[blockIdx.x];
  const int level = tile.x;
  const int cls = tile.y;
  const int p_first = tile.z; // first parent (Morton index at level-1) of this tile
  const int count = tile.w;   // targets in this tile (<= m_tiles * 128 / Kp)
  const int cx = cls & 1, cy = (cls >> 1) & 1, cz = (cls >> 2) & 1;
  const int side = 1 << level;
  const int S = args.stages;
  const int T = 128 / args.Kp;                                      // targets per M tile
  const int m_active = (count + T - 1) / T;
  const int nkc = (args.Kpad + kKChunk - 1) / kKChunk;

  const uint32_t a_tile = 128u * kKChunk * 2u;                      // one M tile, one of hi / lo
  const uint32_t a_bytes = a_tile * static_cast<uint32_t>(MT);
  const uint32_t b_bytes = static_cast<uint32_t>(args.Npad) * kKChunk * 2u;
  const uint32_t stage_bytes = 2u * a_bytes + 2u * b_bytes;
  uint8_t *stage0 = smem;
  // the stages, reused after the last MMA by the epilogue's full-basis rows
  const uint32_t epi_bytes = (128u * static_cast<uint32_t>(args.n) * 4u + 15u) & ~15u;
  const uint32_t pipe_bytes = max(static_cast<uint32_t>(S) * stage_bytes, epi_bytes);
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + pipe_bytes);
  uint64_t *empty = full + S;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(empty + S);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
  int *tgt_node = abort_flag + 1;            // [kTcMaxTargets]
  int *tgt_xyz = tgt_node + kTcMaxTargets;   // [kTcMaxTargets] packed coordinates
  int *act = tgt_xyz + kTcMaxTargets;        // [216] offset positions that reach a source box in the grid
  int *n_act = act + 216;                    // their count
  int *last_unit = n_act + 1;                // [8] per stage: the last pipeline unit issued into it

  // Zero every stage once: A rows beyond a tile's targets are never written.
  for (uint32_t q = tid; q < S * stage_bytes / 16u; q += kTcThreads)
    reinterpret_cast<uint4 *>(stage0)[q] = make_uint4(0, 0, 0, 0);
  if (tid < count) {
    int px, py, pz;
    demorton3(static_cast<uint32_t>(p_first + tid), px, py, pz);
    const int tx = 2 * px + cx, ty = 2 * py + cy, tz = 2 * pz + cz;
    tgt_node[tid] = level_offset_d(level) + static_cast<int>(morton3(tx, ty, tz));
    tgt_xyz[tid] = tx | (ty << 10) | (tz << 20);
  }
  if (tid < 8) last_unit[tid] = -1;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // list2 offsets of class (cx, cy, cz): o in [c-3, c+2]^3 minus |o| <= 1, x
  // fastest; an offset whose source box lies outside the grid for every
  // target of the tile (zero multipoles) is dropped from the pipeline.
  for (int i = tid; i < 216; i += kTcThreads) {
    const int ox = cx - 3 + i % 6, oy = cy - 3 + (i / 6) % 6, oz = cz - 3 + i / 36;
    bool use = !(ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1 && oz >= -1 && oz <= 1);
    if (use) {
      use = false;
      for (int t = 0; t < count && !use; ++t) {
        const int xyz = tgt_xyz[t];
        const int sx = (xyz & 1023) - ox, sy = ((xyz >> 10) & 1023) - oy, sz = ((xyz >> 20) & 1023) - oz;
        use = sx >= 0 && sy >= 0 && sz >= 0 && sx < side && sy < side && sz < side;
      }
    }
    act[i] = use ? 1 : 0;
  }
  __syncthreads();
  if (tid == 0) {
    int c = 0;
    for (int i = 0; i < 216; ++i)
      if (act[i]) act[c++] = i;
    *n_act = c;
  }
  fence_proxy_async();
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(args.tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const int units = *n_act * nkc;

  if (tid >= 32) {
    // Producer warps 1..npw: warp 1 + w issues the bulk copies of units
    // u = w, w + npw, ... (an (offset, chunk) pair each) into stage u % S.
    // Several warps overlap the address arithmetic and copy issue of
    // consecutive units.  npw <= S: a producer waiting for the previous use
    // (u - S) of its stage knows that its own previous unit's stage wait
    // (u - npw - S) completed, so every unit up to u - 2S has completed and
    // the stage's empty barrier is at most one phase behind (a parity wait
    // cannot alias an older phase).
    const int npw = min(kTcThreads / 32 - 1, S);
    const int pw = (tid >> 5) - 1;
    const size_t btile = static_cast<size_t>(args.Npad) * kKChunk * 2u; // stride of one B chunk tile
    for (int u = pw; pw < npw && u < units; u += npw) {
      const int s = u % S;
      int ok = 1;
      if (lane == 0) {
        if (u >= S && !mbar_wait(&empty[s], ((u / S) - 1) & 1, args.wait_limit)) {
          *abort_flag = 1;
          atomicExch(args.error_flag, 1);
        }
        ok = *reinterpret_cast<volatile int *>(abort_flag) == 0;
      }
      ok = __shfl_sync(0xffffffffu, ok, 0);
      if (!ok) break;
      const int kc = u % nkc;
      const int i = act[u / nkc];
      const int ox = cx - 3 + i % 6, oy = cy - 3 + (i / 6) % 6, oz = cz - 3 + i / 36;
      const int slot = (ox + 3) * 49 + (oy + 3) * 7 + (oz + 3);
      const int kcw = min(kKChunk, args.Kpad - kc * kKChunk);
      const uint32_t box_chunk = static_cast<uint32_t>(args.Kp * kcw * 2); // one box's rows of this chunk
      uint8_t *st = stage0 + s * stage_bytes;
      const int n_a = count * 2;
      if (lane == 0)
        mbar_expect_tx(&full[s], static_cast<uint32_t>(n_a) * box_chunk + 2u * static_cast<uint32_t>(args.Npad) * kcw * 2u);
      __syncwarp();
      for (int c = lane; c < n_a + 2; c += 32) {
        if (c < n_a) {
          const int h = c & 1;
          const int t = c >> 1;
          const int m = t / T;
          const int xyz = tgt_xyz[t];
          const int sx = (xyz & 1023) - ox, sy = ((xyz >> 10) & 1023) - oy, sz = ((xyz >> 20) & 1023) - oz;
          int src = args.zero_node;
          if (sx >= 0 && sy >= 0 && sz >= 0 && sx < side && sy < side && sz < side)
            src = level_offset_d(level) + static_cast<int>(morton3(sx, sy, sz)) - args.node_base;
          const size_t goff = static_cast<size_t>(src) * args.box_bytes +
                              static_cast<size_t>(kc) * static_cast<size_t>(args.Kp * kKChunk * 2);
          const uint32_t soff = static_cast<uint32_t>(h) * a_bytes + static_cast<uint32_t>(m) * a_tile +
                                static_cast<uint32_t>(t - m * T) * box_chunk;
          bulk_g2s(st + soff, (h ? args.a_lo : args.a_hi) + goff, box_chunk, &full[s]);
        } else {
          const int h = c - n_a;
          const uint8_t *bsrc = args.b_tiles + (static_cast<size_t>(slot) * nkc + kc) * 2u * btile + h * btile;
          // B_lo right after B_hi (both kcw wide): the 2 Npad rows form one
          // operand of uniform row-group stride for the fused-N MMA
          const uint32_t bw = static_cast<uint32_t>(args.Npad) * kcw * 2u;
          bulk_g2s(st + 2 * a_bytes + h * bw, bsrc, bw, &full[s]);
        }
      }
      __syncwarp();
      if (lane == 0) atomicMax(&last_unit[s], u);
    }
  } else if (tid == 0) {
    // MMA issuer: waits for each unit's operands, issues its MMAs, commits
    // to the unit's empty barrier (arrives when those MMAs completed).  The
    // shared-memory descriptors are built once: a byte offset o < 256 KB is
    // added to a descriptor as o >> 4 in its 14-bit start-address field.
    const uint32_t idesc = instr_desc_bf16(args.Npad);
    const uint32_t idesc2 = instr_desc_bf16(2 * args.Npad); // fused: N = [B_hi | B_lo]
    const bool fuse = args.fuse_n != 0;
    const uint64_t desc_full = smem_desc(smem_u32(stage0), 128u, kKChunk * 16u); // SBO = chunk width * 16 B
    const uint64_t desc_half = smem_desc(smem_u32(stage0), 128u, 16u * 16u);     // last chunk 16 wide
    const uint64_t o_alo = a_bytes >> 4, o_bhi = (2u * a_bytes) >> 4;
    uint32_t accumulate = 0;
    int issued = 0;
    int s = 0, kc = 0;
    uint32_t phase = 0;
    for (int u = 0; u < units; ++u) {
      if (!mbar_wait(&full[s], phase, args.wait_limit)) {
        *abort_flag = 1;
        atomicExch(args.error_flag, 2);
        break;
      }
      tc_fence_after();
      const int kcw = min(kKChunk, args.Kpad - kc * kKChunk);
      const uint64_t base = (kcw == kKChunk ? desc_full : desc_half) + ((static_cast<uint32_t>(s) * stage_bytes) >> 4);
      const uint64_t o_blo = (2u * a_bytes + static_cast<uint32_t>(args.Npad) * kcw * 2u) >> 4;
#pragma unroll
      for (int ks = 0; ks < kKChunk / 16; ++ks) {
        if (ks * 16 < kcw) {
          const uint64_t o = base + static_cast<uint64_t>(ks * 16); // 2 core matrices = 256 B
#pragma unroll
          for (int m = 0; m < MT; ++m) {
            if (m < m_active) {
              const uint32_t d = tmem + static_cast<uint32_t>(m * args.acc_stride);
              const uint64_t ah = o + ((static_cast<uint32_t>(m) * a_tile) >> 4);
              if (fuse) {
                // columns [0, Npad): hi*hi + lo*hi; [Npad, 2 Npad): hi*lo
                mma_bf16(d, ah, o + o_bhi, idesc2, accumulate);
                mma_bf16(d, ah + o_alo, o + o_bhi, idesc, 1);
              } else {
                mma_bf16(d, ah, o + o_bhi, idesc, accumulate);
                mma_bf16(d, ah, o + o_blo, idesc, 1);
                mma_bf16(d, ah + o_alo, o + o_bhi, idesc, 1);
              }
            }
          }
          accumulate = 1;
        }
      }
      mma_commit(&empty[s]);
      issued = u + 1;
      if (++s == S) {
        s = 0;
        phase ^= 1u;
      }
      if (++kc == nkc) kc = 0;
    }
    // The last commit arrives once every MMA issued before it has completed.
    if (issued > 0 && !mbar_wait(&empty[(issued - 1) % S], ((issued - 1) / S) & 1)) {
      *abort_flag = 1;
      atomicExch(args.error_flag, 3);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (*abort_flag != 0 && tid < S) {
    // Abort: the copies of the last unit issued into each stage may still be
    // in flight (earlier units of a stage completed before it was reused).
    // Wait for them with the full limit before the CTA's shared memory is
    // released.
    const int u = last_unit[tid];
    if (u >= 0) mbar_wait(&full[tid], static_cast<uint32_t>(u / S) & 1u);
  }

  // Epilogue: warp w owns TMEM lanes 32w..32w+31 (rows of every M tile).
  // A row's n_out reduced locals go to its column of the (now idle) stage
  // memory at their full ranks, the other locals follow from the trace
  // relations, and all n are scaled by D_L and stored.  After an expired
  // wait the accumulators are incomplete: the tile's locals are written as
  // NaN instead.
  if (*abort_flag != 0) {
    const int tr = tid / args.Kp;
    const int k = tid - tr * args.Kp;
    for (int m = 0; m < m_active; ++m) {
      const int tt = m * T + tr;
      if (tr < T && tt < count && k < args.K) {
        const long long base = static_cast<long long>(tgt_node[tt]) * args.n * args.K + k;
        for (int b = 0; b < args.n; ++b) {
          if (args.L_list != nullptr)
            args.L_list[k][static_cast<long long>(tgt_node[tt]) * args.n + b] = __int_as_float(0x7fc00000);
          else
            args.L[base + static_cast<long long>(b) * args.K] = __int_as_float(0x7fc00000);
        }
      }
    }
  } else {
    const int warp = tid >> 5;
    const int row = tid;
    const int tr = row / args.Kp;
    const int k = row - tr * args.Kp;
    const float *sl = args.scale_l + level * args.n;
    float *const ep = reinterpret_cast<float *>(smem) + tid; // this row's locals, stride kTcThreads floats
    for (int m = 0; m < m_active; ++m) {
      const int tt = m * T + tr;
      const bool valid = tr < T && tt < count && k < args.K;
      const int node = valid ? tgt_node[tt] : 0;
      const long long base = static_cast<long long>(node) * args.n * args.K + k;
      float *const out_k = (args.L_list != nullptr && valid) ? args.L_list[k] + static_cast<long long>(node) * args.n
                                                              : nullptr;
      for (int c0 = 0; c0 < args.Npad; c0 += 16) {
        float v[16];
        const uint32_t tcol = tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(m * args.acc_stride + c0);
        tmem_ld16(tcol, v);
        if (args.fuse_n) {
          float w[16];
          tmem_ld16(tcol + static_cast<uint32_t>(args.Npad), w);
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] += w[j];
        }
        if (units == 0) {
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = 0.0F; // no source box in the grid: no MMA wrote the accumulator
        }
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (c0 + j < args.n_out) ep[__ldg(args.expand + c0 + j) * kTcThreads] = v[j];
      }
      for (int i = 0; i < args.n_derived; ++i) {
        const int e = __ldg(args.expand + args.n_out + i);
        ep[(e & 1023) * kTcThreads] = -(ep[((e >> 10) & 1023) * kTcThreads] + ep[(e >> 20) * kTcThreads]);
      }
      if (valid) {
        for (int b = 0; b < args.n; ++b) {
          const float x = ep[b * kTcThreads] * sl[b];
          if (out_k != nullptr)
            out_k[b] = x;
          else
            args.L[base + static_cast<long long>(b) * args.K] = x;
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(args.tmem_cols));
  }
}

// Pack: scaled multipoles of levels 2..depth -> BF16 hi/lo boxes.  A box is
// Kp rows (states) x Kpad alphas stored chunk by chunk (32 alphas; the last
// chunk may be 16), each chunk as [Kp/8 row groups][w/8 column blocks][8][8]
// so one box's rows of one chunk are contiguous.  One extra all-zero box
// (index n_boxes) stands for sources outside the grid.  One CTA per box: a
// chunk's 32 alphas x Kp states are read along the states (coalesced rows
// of M[node][alpha][k]) into a shared tile, then written as 16-byte runs of
// 8 alphas (one core-matrix row of hi and of lo).
constexpr int kPackThreads = 256;
constexpr int kPackMaxKp = 128;

__global__ void __launch_bounds__(kPackThreads) m2l_pack_kernel(const float *__restrict__ M,
                                                                const float *const *__restrict__ M_list,
                                                                const float *__restrict__ scale_m,
                                                                const int *__restrict__ fold_off,
                                                                const int *__restrict__ fold, int n_in,
                                                                uint4 *__restrict__ hi, uint4 *__restrict__ lo, int n,
                                                                int K, int Kp, int Kpad, int depth, int node_base,
                                                                int n_boxes) {
  __shared__ float tile[kKChunk][kPackMaxKp + 1]; // [alpha in chunk][state]
  const int box = blockIdx.x;
  const int tid = threadIdx.x;
  const int node = node_base + box;
  int level = 0;
  while (level < depth && level_offset_d(level + 1) <= node) ++level;
  const float *src = M != nullptr ? M + static_cast<long long>(node) * n * K : nullptr;
  const long long box_vec = static_cast<long long>(box) * Kp * Kpad / 8; // 16-byte vectors before this box
  const int nkc = (Kpad + kKChunk - 1) / kKChunk;
  for (int kc = 0; kc < nkc; ++kc) {
    const int w = min(kKChunk, Kpad - kc * kKChunk);
    const int ncj = w / 8;
    __syncthreads();
    for (int e = tid; e < w * Kp; e += kPackThreads) {
      const int al = e / Kp;
      const int k = e - al * Kp;
      const int j = kc * kKChunk + al;
      // folded input j: sum of c M_a over its fold entries (all of one
      // degree, the first one its own rank), then scaled (scale_m is one
      // power of two per degree).  Padding inputs (j >= n_in), padding
      // states (k >= K) and the zero box are zero.
      float m = 0.0F;
      if (box < n_boxes && j < n_in && k < K) {
        const int f0 = __ldg(fold_off + j), f1 = __ldg(fold_off + j + 1);
        for (int f = f0; f < f1; ++f) {
          const int ent = __ldg(fold + f);
          const int a = ent & 0xffff;
          const float x =
              M_list != nullptr ? M_list[k][static_cast<long long>(node) * n + a] : src[static_cast<long long>(a) * K + k];
          m = fmaf(static_cast<float>((ent >> 16) - 64), x, m);
        }
        m *= scale_m[level * n + (__ldg(fold + f0) & 0xffff)];
      }
      tile[al][k] = m;
    }
    __syncthreads();
    const long long chunk_vec = box_vec + static_cast<long long>(kc) * Kp * kKChunk / 8;
    for (int v = tid; v < Kp * w / 8; v += kPackThreads) {
      const int x = v >> 3;
      const int r8 = v & 7;
      const int cjl = x % ncj;
      const int k = (x / ncj) * 8 + r8;
      uint32_t h[4], l[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float v0 = tile[cjl * 8 + 2 * j][k], v1 = tile[cjl * 8 + 2 * j + 1][k];
        const __nv_bfloat16 h0 = __float2bfloat16_rn(v0), h1 = __float2bfloat16_rn(v1);
        const __nv_bfloat16 l0 = __float2bfloat16_rn(v0 - __bfloat162float(h0));
        const __nv_bfloat16 l1 = __float2bfloat16_rn(v1 - __bfloat162float(h1));
        h[j] = static_cast<uint32_t>(__bfloat16_as_ushort(h0)) | (static_cast<uint32_t>(__bfloat16_as_ushort(h1)) << 16);
        l[j] = static_cast<uint32_t>(__bfloat16_as_ushort(l0)) | (static_cast<uint32_t>(__bfloat16_as_ushort(l1)) << 16);
      }
      hi[chunk_vec + v] = make_uint4(h[0], h[1], h[2], h[3]);
      lo[chunk_vec + v] = make_uint4(l[0], l[1], l[2], l[3]);
    }
  }
}

} // namespace

size_t m2l_tc_smem_bytes(int Npad, int m_tiles, int stages, int n) {
  const size_t a = 128u * kKChunk * 2u * static_cast<size_t>(m_tiles);
  const size_t b = static_cast<size_t>(Npad) * kKChunk * 2u;
  const size_t epi = (static_cast<size_t>(kTcThreads) * n * 4u + 15u) & ~static_cast<size_t>(15);
  return std::max(static_cast<size_t>(stages) * (2 * a + 2 * b), epi) + 2 * stages * sizeof(uint64_t) + 8 +
         (2 * kTcMaxTargets + 216 + 1 + 8) * sizeof(int);
}

void launch_m2l_pack(const float *M, const float *scale_m, const int *fold_off, const int *fold, int n_in, void *hi,
                     void *lo, int n, int K, int Kp, int Kpad, int depth, int node_base, int n_boxes, cudaStream_t s,
                     const float *const *M_list) {
  if (Kp > kPackMaxKp || Kp % 8 != 0 || Kpad % 16 != 0) return; // the plan keeps Kp <= 128, multiples of 8
  m2l_pack_kernel<<<n_boxes + 1, kPackThreads, 0, s>>>(M, M_list, scale_m, fold_off, fold, n_in,
                                                        static_cast<uint4 *>(hi), static_cast<uint4 *>(lo), n, K, Kp,
                                                        Kpad, depth, node_base, n_boxes);
}

void launch_m2l_tc(const TcArgs &args, int n_tiles, cudaStream_t s) {
  if (n_tiles == 0) return;
  size_t smem = m2l_tc_smem_bytes(args.Npad, args.m_tiles, args.stages, args.n);
  // More than half of TMEM per CTA: request enough shared memory that a
  // second CTA never shares the SM (its tcgen05.alloc would wait for ours).
  if (args.tmem_cols > 256) smem = std::max<size_t>(smem, 120 * 1024);
  if (args.m_tiles == 4)
    m2l_tc_kernel<4><<<n_tiles, kTcThreads, smem, s>>>(args);
  else if (args.m_tiles == 2)
    m2l_tc_kernel<2><<<n_tiles, kTcThreads, smem, s>>>(args);
  else
    m2l_tc_kernel<1><<<n_tiles, kTcThreads, smem, s>>>(args);
}

// Self-test of the bounded-wait path: one thread waits on an mbarrier whose
// phase nothing completes, with a short limit; the wait must give up and the
// kernel record the same error code the M2L pipeline records and return.
__global__ void bounded_wait_selftest_kernel(int *error_flag, uint32_t limit) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (!mbar_wait(&bar, 0, limit)) atomicExch(error_flag, 2);
  }
}

void launch_bounded_wait_selftest(int *error_flag, cudaStream_t s) {
  bounded_wait_selftest_kernel<<<1, 32, 0, s>>>(error_flag, 1u << 12);
}

bool configure_m2l_tc(size_t max_smem) {
  prefer_max_shared_carveout(m2l_tc_kernel<1>);
  prefer_max_shared_carveout(m2l_tc_kernel<2>);
  prefer_max_shared_carveout(m2l_tc_kernel<4>);
  return allow_dynamic_smem(m2l_tc_kernel<1>, max_smem) && allow_dynamic_smem(m2l_tc_kernel<2>, max_smem) &&
         allow_dynamic_smem(m2l_tc_kernel<4>, max_smem);
}

// Host: B tiles [slot][alpha chunk][hi, lo][Npad x 32 stride] BF16 from FP64
// matrices T[slot][alpha][beta] (symmetric in alpha, beta); a chunk of width w
// is stored as [beta group][w/8 column blocks][8 betas][8 alphas].
std::vector<uint16_t> pack_m2l_b_tiles(const std::vector<double> &T64, int n, const M2lTraceless &red, int Npad,
                                       int Kpad) {
  const int nkc = (Kpad + kKChunk - 1) / kKChunk;
  const size_t btile = static_cast<size_t>(Npad) * kKChunk;
  std::vector<uint16_t> out(static_cast<size_t>(343) * nkc * 2 * btile, 0);
  auto bf16_bits = [](float f) -> uint16_t {
    const __nv_bfloat16 h = __float2bfloat16_rn(f);
    uint16_t b;
    std::memcpy(&b, &h, 2);
    return b;
  };
  for (int slot = 0; slot < 343; ++slot) {
    const double *Ts = T64.data() + static_cast<size_t>(slot) * n * n;
    const int n_out = static_cast<int>(red.out_set.size()), n_in = static_cast<int>(red.in_set.size());
    for (int beta = 0; beta < n_out; ++beta)
      for (int alpha = 0; alpha < n_in; ++alpha) {
        const double v = Ts[static_cast<size_t>(red.in_set[static_cast<size_t>(alpha)]) * n +
                            red.out_set[static_cast<size_t>(beta)]];
        const __nv_bfloat16 h = __float2bfloat16_rn(static_cast<float>(v));
        const float l = static_cast<float>(v - static_cast<double>(__bfloat162float(h)));
        const int kc = alpha / kKChunk;
        const int al = alpha - kc * kKChunk;
        const int ncj = std::min(kKChunk, Kpad - kc * kKChunk) / 8;
        uint16_t *hi = out.data() + (static_cast<size_t>(slot) * nkc + kc) * 2 * btile;
        uint16_t *lo = hi + btile;
        const size_t at = ((static_cast<size_t>(beta / 8) * ncj + al / 8) * 8 + beta % 8) * 8 + al % 8;
        hi[at] = bf16_bits(static_cast<float>(v));
        lo[at] = bf16_bits(l);
      }
  }
  return out;
}

M2lTraceless m2l_traceless(int p) {
  const int n = basis_size_d(p);
  std::vector<int> ex(static_cast<size_t>(n)), ey(static_cast<size_t>(n)), ez(static_cast<size_t>(n));
  for (int d = 0; d <= p; ++d)
    for (int a = 0; a <= d; ++a)
      for (int b = 0; a + b <= d; ++b) {
        const size_t r = static_cast<size_t>(rank3(a, b, d - a - b));
        ex[r] = a;
        ey[r] = b;
        ez[r] = d - a - b;
      }
  M2lTraceless t;
  std::vector<int> in_pos(static_cast<size_t>(n), -1);
  for (int r = 0; r < n; ++r) {
    if (ez[static_cast<size_t>(r)] > 1) continue;
    t.out_set.push_back(r);
    if (r > 0) {
      in_pos[static_cast<size_t>(r)] = static_cast<int>(t.in_set.size());
      t.in_set.push_back(r);
    }
  }
  // fold every moment a >= 1 onto the reduced inputs: repeatedly move the
  // weight on an exponent with z >= 2 to (x + 2, z - 2) and (y + 2, z - 2)
  // with the sign flipped, from the highest z down
  std::vector<std::vector<std::pair<int, int>>> per_in(t.in_set.size());
  for (int a = 1; a < n; ++a) {
    std::vector<int> w(static_cast<size_t>(n), 0);
    w[static_cast<size_t>(a)] = 1;
    for (int z = p; z >= 2; --z)
      for (int r = 0; r < n; ++r) {
        const size_t rr = static_cast<size_t>(r);
        if (ez[rr] != z || w[rr] == 0) continue;
        w[static_cast<size_t>(rank3(ex[rr] + 2, ey[rr], z - 2))] -= w[rr];
        w[static_cast<size_t>(rank3(ex[rr], ey[rr] + 2, z - 2))] -= w[rr];
        w[rr] = 0;
      }
    for (int r = 0; r < n; ++r)
      if (w[static_cast<size_t>(r)] != 0) per_in[static_cast<size_t>(in_pos[static_cast<size_t>(r)])].push_back({a, w[static_cast<size_t>(r)]});
  }
  t.fold_off.push_back(0);
  for (size_t j = 0; j < per_in.size(); ++j) {
    // its own rank first (coefficient 1), then the folded ranks ascending
    std::stable_sort(per_in[j].begin(), per_in[j].end(), [&](const std::pair<int, int> &x, const std::pair<int, int> &y) {
      const bool xs = x.first == t.in_set[j], ys = y.first == t.in_set[j];
      return xs != ys ? xs : x.first < y.first;
    });
    for (const auto &e : per_in[j]) t.fold.push_back(e.first | ((e.second + 64) << 16));
    t.fold_off.push_back(static_cast<int>(t.fold.size()));
  }
  t.expand = t.out_set;
  for (int z = 2; z <= p; ++z)
    for (int r = 0; r < n; ++r) {
      const size_t rr = static_cast<size_t>(r);
      if (ez[rr] != z) continue;
      const int s1 = rank3(ex[rr] + 2, ey[rr], z - 2), s2 = rank3(ex[rr], ey[rr] + 2, z - 2);
      t.expand.push_back(r | (s1 << 10) | (s2 << 20));
      ++t.n_derived;
    }
  return t;
}

} // namespace cdfmm_b200
