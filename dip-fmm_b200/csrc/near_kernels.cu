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

#include <algorithm>
#include <cmath>
#include <vector>

#include "far_kernels.hpp"
#include "kernels.cuh"
#include "near_tc.hpp"

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
// offset (neighbour centre - this centre) in normalised units.  Run by one
// full warp: lane l < 27 looks up neighbour (dx, dy, dz) = (l % 3, l / 3 % 3,
// l / 9) - 1 (z outermost, x fastest), and the non-empty ones are compacted
// in that order with a ballot and a shuffle scan of their source counts.
__device__ void build_neighbours(Neighbours &nb, int leaf, int depth, const int *src_off, int lane) {
  int ix, iy, iz;
  demorton3(static_cast<uint32_t>(leaf), ix, iy, iz);
  const int side = 1 << depth;
  const float w = 1.0F / static_cast<float>(side);
  const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
  const int x = ix + dx, y = iy + dy, z = iz + dz;
  int b = 0, e = 0;
  if (lane < 27 && x >= 0 && y >= 0 && z >= 0 && x < side && y < side && z < side) {
    const uint32_t m = morton3(x, y, z);
    b = src_off[m];
    e = src_off[m + 1];
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
    nb.begin[slot] = b;
    nb.sx[slot] = static_cast<float>(dx) * w;
    nb.sy[slot] = static_cast<float>(dy) * w;
    nb.sz[slot] = static_cast<float>(dz) * w;
    nb.prefix[slot + 1] = incl;
  }
  if (lane == 0) {
    nb.prefix[0] = 0;
    nb.count = __popc(mask);
  }
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

// Close pairs.  Positions are kept in FP32 relative to their leaf centre,
// an absolute error of about 2^-25 leaf widths; for a pair much closer than
// a leaf that error is no longer small against |r| (the reference builds its
// pair tensors from FP64 positions).  The near-field kernels treat every
// pair alike; the plan lists the pairs closer than a leaf width / 2^k (k >= 4,
// chosen so the list stays within a few entries per target) with both the
// FP32 r the kernels form and r from the FP64 positions, and a correction
// pass after each near-field launch adds, per listed pair, its field at the
// exact r minus its field at the FP32 r.  An exact zero r^2 in FP32 (the
// self pair, or coincident points) is never listed.

// One staged source pair (components .x, .y: two sources) against one
// target in packed FP32x2 arithmetic.  With d = source - target (= -r) and
// v = 1/|r|^3 the pair adds
//   P += (m.d) v                          (phi = -P)
//   G += v (m - 3 (m.d) / |d|^2 d)        (H = -G)
// so the target's coordinates enter negated and no operand needs a sign
// flip inside the loop.  SELF: the sources' sorted indices are compared with
// the target's self index; the self pair gets 1/|r| = 0 (no contribution).
// A coincident non-self pair gives 1/|r| = inf and NaN, as in the reference.
template <bool PHI, bool SELF>
__device__ __forceinline__ void pair_k1_x2(const float2 &ntx, const float2 &nty, const float2 &ntz, int self,
                                           const float4 &pxy, const float4 &pzj, const float4 &mxy,
                                           const float2 &mz, float2 (&acc)[4]) {
  const float2 dx = __fadd2_rn(make_float2(pxy.x, pxy.y), ntx);
  const float2 dy = __fadd2_rn(make_float2(pxy.z, pxy.w), nty);
  const float2 dz = __fadd2_rn(make_float2(pzj.x, pzj.y), ntz);
  const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
  float2 rinv = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
  if (SELF) {
    rinv.x = __float_as_int(pzj.z) == self ? 0.0F : rinv.x;
    rinv.y = __float_as_int(pzj.w) == self ? 0.0F : rinv.y;
  }
  const float2 rinv2 = __fmul2_rn(rinv, rinv);
  const float2 rinv3 = __fmul2_rn(rinv2, rinv);
  const float2 mx = make_float2(mxy.x, mxy.y), my = make_float2(mxy.z, mxy.w);
  const float2 md = __ffma2_rn(mx, dx, __ffma2_rn(my, dy, __fmul2_rn(mz, dz)));
  if (PHI) acc[0] = __ffma2_rn(md, rinv3, acc[0]);
  const float2 nb = __fmul2_rn(__fmul2_rn(md, make_float2(-3.0F, -3.0F)), rinv2);
  acc[1] = __ffma2_rn(rinv3, __ffma2_rn(nb, dx, mx), acc[1]);
  acc[2] = __ffma2_rn(rinv3, __ffma2_rn(nb, dy, my), acc[2]);
  acc[3] = __ffma2_rn(rinv3, __ffma2_rn(nb, dz, mz), acc[3]);
}

constexpr int kK1Chunk = 1024;               // staged sources per pass
constexpr int kK1Pairs = kK1Chunk / 2;
constexpr int kK1TargetChunk = kP2pUnitTargets;

// Staged source pairs [pa, pb) against a warp's 4 targets, lane l taking
// pa + l, pa + l + 32, ...
template <bool PHI, bool SELF>
__device__ __forceinline__ void k1_segment(const float2 (&nt)[4][3], const int (&self)[4], const float4 *sPxy,
                                           const float4 *sPzj, const float4 *sMxy, const float2 *sMz, int pa,
                                           int pb, int lane, float2 (&acc)[4][4]) {
  for (int q = pa + lane; q < pb; q += 32) {
    const float4 pxy = sPxy[q];
    const float4 pzj = sPzj[q];
    const float4 mxy = sMxy[q];
    const float2 mz = sMz[q];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      pair_k1_x2<PHI, SELF>(nt[u][0], nt[u][1], nt[u][2], self[u], pxy, pzj, mxy, mz, acc[u]);
  }
}

// K = 1: one CTA per work unit (up to 128 targets of one leaf), the
// neighbourhood sources staged in shared memory kK1Chunk at a time as pairs
// of consecutive sources in structure-of-arrays form (x0 x1 y0 y1 | z0 z1 j0
// j1 | mx0 mx1 my0 my1 | mz0 mz1; an odd chunk is padded with a zero moment
// 1e18 away), so each lane reads two sources' operands ready for packed
// FP32x2 arithmetic; each warp owns 4 targets at a time, lanes stride over
// the staged pairs and the partial sums are combined with warp shuffles.
// Only the staged positions of the sources between the lowest and highest
// self source of the leaf's targets are compared against the self indices
// (the own leaf's, when sources and targets are the same points).
template <bool PHI>
__global__ void __launch_bounds__(128) p2p_k1_kernel(const float4 *__restrict__ src_rel,
                                                     const float4 *__restrict__ mom,
                                                     const int *__restrict__ src_off,
                                                     const float4 *__restrict__ tgt_rel,
                                                     const int4 *__restrict__ work,
                                                     const int *__restrict__ self_idx,
                                                     const int2 *__restrict__ leaf_self, int depth,
                                                     float4 *__restrict__ near) {
  __shared__ float4 sPxy[kK1Pairs];
  __shared__ float4 sPzj[kK1Pairs];
  __shared__ float4 sMxy[kK1Pairs];
  __shared__ float2 sMz[kK1Pairs];
  __shared__ float4 sAcc[kK1TargetChunk];
  __shared__ Neighbours nb;
  __shared__ int sSelf[2]; // staged positions [lo, hi] of the leaf's self-source range
  const int4 unit = work[blockIdx.x];
  const int leaf = unit.x;
  const int t0 = unit.y;
  const int t1 = unit.y + unit.z;
  if (threadIdx.x < 32) build_neighbours(nb, leaf, depth, src_off, threadIdx.x);
  __syncthreads();
  if (threadIdx.x == 0) {
    // staged positions of the leaf's self-source range (the whole leaf's, so
    // a target's sum does not depend on how its leaf is cut into units)
    int lo = 0x7fffffff, hi = -1;
    if (self_idx != nullptr) {
      const int2 r = leaf_self[leaf];
      for (int c = 0; c < nb.count; ++c) {
        const int b = nb.begin[c], len = nb.prefix[c + 1] - nb.prefix[c];
        const int a0 = max(r.x, b), a1 = min(r.y, b + len - 1);
        if (a0 <= a1) {
          lo = min(lo, nb.prefix[c] + a0 - b);
          hi = max(hi, nb.prefix[c] + a1 - b);
        }
      }
    }
    sSelf[0] = lo;
    sSelf[1] = hi;
  }
  __syncthreads();
  const int total = nb.prefix[nb.count];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  for (int tc = t0; tc < t1; tc += kK1TargetChunk) {
    const int tn = min(kK1TargetChunk, t1 - tc);
    for (int q = threadIdx.x; q < tn; q += blockDim.x) sAcc[q] = make_float4(0, 0, 0, 0);
    for (int sc = 0; sc < total; sc += kK1Chunk) {
      const int sn = min(kK1Chunk, total - sc);
      const int np = (sn + 1) / 2;
      __syncthreads();
      for (int q = threadIdx.x; q < np; q += blockDim.x) {
        float4 p0, p1 = make_float4(1.0e18F, 1.0e18F, 1.0e18F, __int_as_float(-1));
        float4 m0, m1 = make_float4(0.0F, 0.0F, 0.0F, 0.0F);
        int j;
        stage_source(nb, sc + 2 * q, src_rel, p0, j);
        m0 = mom[j];
        if (2 * q + 1 < sn) {
          stage_source(nb, sc + 2 * q + 1, src_rel, p1, j);
          m1 = mom[j];
        }
        sPxy[q] = make_float4(p0.x, p1.x, p0.y, p1.y);
        sPzj[q] = make_float4(p0.z, p1.z, p0.w, p1.w);
        sMxy[q] = make_float4(m0.x, m1.x, m0.y, m1.y);
        sMz[q] = make_float2(m0.z, m1.z);
      }
      __syncthreads();
      // pairs [0, pa) and [pb, np) hold no self source of the leaf's targets
      const int qa = min(max(sSelf[0] - sc, 0), sn);
      const int qb = max(min(sSelf[1] + 1 - sc, sn), qa);
      const int pa = qa / 2, pb = max((qb + 1) / 2, pa);
      for (int tb = warp * 4; tb < tn; tb += 16) {
        float2 nt[4][3];
        int self[4];
        float2 acc2[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int i = tc + min(tb + u, tn - 1);
          const float4 t = tgt_rel[i];
          nt[u][0] = make_float2(-t.x, -t.x);
          nt[u][1] = make_float2(-t.y, -t.y);
          nt[u][2] = make_float2(-t.z, -t.z);
          self[u] = self_idx != nullptr ? self_idx[i] : -1;
          acc2[u][0] = acc2[u][1] = acc2[u][2] = acc2[u][3] = make_float2(0.0F, 0.0F);
        }
        k1_segment<PHI, false>(nt, self, sPxy, sPzj, sMxy, sMz, 0, pa, lane, acc2);
        k1_segment<PHI, true>(nt, self, sPxy, sPzj, sMxy, sMz, pa, pb, lane, acc2);
        k1_segment<PHI, false>(nt, self, sPxy, sPzj, sMxy, sMz, pb, np, lane, acc2);
        float acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            acc[u][c] = -(acc2[u][c].x + acc2[u][c].y); // phi = -P, H = -G
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[u][c] += __shfl_xor_sync(0xffffffffu, acc[u][c], o);
          }
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

// K > 1.  One CTA per work unit (up to 128 targets of one leaf).  Work
// items are (target, group of KG states); a lane owns one item and computes
// a pair's geometry once --
// r, v = 1/|r|^3, u = 3 r / |r|^5, w = |r|^2 / 3 -- applying it to its KG
// states:
//   s = m.u,  phi += s w,  H += s r - v m          (10 FP ops per pair-state)
// A self pair gets u = v = w = 0; a coincident non-self pair gives u = NaN
// (0 * inf), hence NaN results, as in the reference.
//
// Load balance: the items of a unit are processed in rounds of 256 lanes; a
// round gives each of its r items F = 2^j <= 8 lanes that split the sources
// (lane f takes sources f, f + F, ...) and are summed with warp shuffles at
// the end of the round.  Each round takes the F (and r = min(remaining,
// 256 / F)) that keeps the most lanes busy, so a unit whose item count is
// not a multiple of 256 -- fewer than 32 targets, or a narrow state window
// -- does not leave lanes idle.
//
// Staging: the neighbourhood positions (relative to this leaf's centre) and
// sorted source indices are staged once; the moments of the round's state
// window stream through a kBufs-buffered cp.async pipeline in chunks of
// kChunkB sources, one barrier per chunk: the copy of chunk c + kBufs - 1 is
// issued after the barrier that ends every thread's use of chunk c - 1,
// whose buffer it overwrites.  (Three buffers of 24 sources, which fit two
// CTAs per SM, measured slower than two of 32.)  Within a moment row, state k sits at k + k/8 (one pad
// float4 per 8 states), so lanes of one warp that read the same source for
// two state groups hit different banks; the row stride Kr is 1 mod 8 (in
// float4) so the F lanes of one item, reading different sources, do too.
constexpr int kChunkB = 32;         // sources per moment chunk
constexpr int kBufs = 2;            // moment chunk buffers (copies run kBufs - 1 chunks ahead)
constexpr int kNeighbourCap = 1024; // staged neighbourhood size per pass
constexpr int kStateBlock = 64;     // states per state block (bounds shared memory)
constexpr int kKbThreads = 256;
// Co-resident form: two CTAs of this kernel leave room on every SM for one
// CTA of a far-field kernel (the tensor-core M2L: 128 threads, <= 56
// registers, up to ~105 KB of shared memory), so the near field and the far
// field run side by side instead of taking SMs from each other: state blocks
// of 32 (58 KB of shared memory per CTA; moment chunks of 24 sources, 47.5
// KB, were measured slower with no gain for the M2L beside them) and at most
// 112 registers per thread (2 x 256 x 112 + 128 x 56 <= 65,536).
constexpr int kStateBlockCorun = 32;
constexpr int kChunkCorun = 32;
constexpr int kKbRegsCorun = 112;

// Shared-memory position of state k within a staged moment row (one pad
// float4 after every group of KG states), and the row stride for a window of
// Kw states (1 mod 8 float4).
template <int KG> __host__ __device__ __forceinline__ int mrow_pos(int k) { return k + k / KG; }
template <int KG> __host__ __device__ __forceinline__ int mrow_stride(int Kw) {
  return ((Kw + (Kw - 1) / KG + 6) / 8) * 8 + 1;
}

// Sources q = qbeg, qbeg + F, ... < sn of one staged chunk; m_row0 points at
// this item's first state in source row 0 (its KG states are contiguous:
// groups start at multiples of 8), rows Kr float4 apart.  FULL: all KG states
// valid (no per-state predicate).
template <int KG, bool PHI, bool FULL>
__device__ __forceinline__ void p2p_kb_chunk(const float4 &ti, int self, const float4 *sPos,
                                             const float4 *m_row0, int Kr, int qbeg, int sn, int F, int kvalid,
                                             float (&acc)[KG][4]) {
#pragma unroll 2
  for (int q = qbeg; q < sn; q += F) {
    const float4 s = sPos[q];
    const float dx = ti.x - s.x, dy = ti.y - s.y, dz = ti.z - s.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const bool is_self = __float_as_int(s.w) == self;
    const float rinv = is_self ? 0.0F : rsqrtf(r2);
    const float v = rinv * rinv * rinv;
    const float f = 3.0F * v * rinv * rinv;
    const float ux = f * dx, uy = f * dy, uz = f * dz;
    const float w = is_self ? 0.0F : r2 * (1.0F / 3.0F);
    const float4 *mq = m_row0 + q * Kr;
#pragma unroll
    for (int st = 0; st < KG; ++st) {
      if (FULL || st < kvalid) {
        const float4 m = mq[st];
        const float sd = fmaf(m.x, ux, fmaf(m.y, uy, m.z * uz));
        if (PHI) acc[st][0] = fmaf(sd, w, acc[st][0]);
        acc[st][1] = fmaf(-v, m.x, fmaf(sd, dx, acc[st][1]));
        acc[st][2] = fmaf(-v, m.y, fmaf(sd, dy, acc[st][2]));
        acc[st][3] = fmaf(-v, m.z, fmaf(sd, dz, acc[st][3]));
      }
    }
  }
}

// Paired states (K >= 4): the staged row holds state pairs as
// (x_a, x_b, y_a, y_b), (z_a, z_b, 0, 0) and the per-state arithmetic runs on
// packed FP32x2 FMAs, one instruction for two states (same FP32 throughput,
// half the issue slots).  The self source is recognised by its position in
// the staged chunk (self_q, computed once per item; out of range when it is
// not in this chunk), and the self pair needs no zeroed w: with 1/|r| = 0
// the pair's s = m.u is 0.
template <int KG, bool PHI, bool FULL>
__device__ __forceinline__ void p2p_kb_chunk_x2(const float4 &ti, int self_q, const float4 *sPos,
                                                const float4 *m_row0, int Kr, int qbeg, int sn, int F, int kvalid,
                                                float2 (&acc)[KG / 2][4]) {
#pragma unroll 2
  for (int q = qbeg; q < sn; q += F) {
    const float4 s = sPos[q];
    const float dx = ti.x - s.x, dy = ti.y - s.y, dz = ti.z - s.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const float rinv = q == self_q ? 0.0F : rsqrtf(r2);
    const float v = rinv * rinv * rinv;
    const float f = 3.0F * v * rinv * rinv;
    const float w = r2 * (1.0F / 3.0F);
    const float2 UX = make_float2(f * dx, f * dx), UY = make_float2(f * dy, f * dy), UZ = make_float2(f * dz, f * dz);
    const float2 DX = make_float2(dx, dx), DY = make_float2(dy, dy), DZ = make_float2(dz, dz);
    const float2 NV = make_float2(-v, -v), W2 = make_float2(w, w);
    const float4 *mq = m_row0 + q * Kr;
#pragma unroll
    for (int pr = 0; pr < KG / 2; ++pr) {
      if (FULL || 2 * pr < kvalid) {
        const float4 a = mq[2 * pr], b = mq[2 * pr + 1];
        const float2 X = make_float2(a.x, a.y), Y = make_float2(a.z, a.w), Z = make_float2(b.x, b.y);
        float2 sd = __fmul2_rn(X, UX);
        sd = __ffma2_rn(Y, UY, sd);
        sd = __ffma2_rn(Z, UZ, sd);
        if (PHI) acc[pr][0] = __ffma2_rn(sd, W2, acc[pr][0]);
        acc[pr][1] = __ffma2_rn(NV, X, __ffma2_rn(sd, DX, acc[pr][1]));
        acc[pr][2] = __ffma2_rn(NV, Y, __ffma2_rn(sd, DY, acc[pr][2]));
        acc[pr][3] = __ffma2_rn(NV, Z, __ffma2_rn(sd, DZ, acc[pr][3]));
      }
    }
  }
}

// Position gradient of w.H for a target over one staged chunk (summed over
// the item's KG states): with a = m.r, b = w.r, f5 = 3/|r|^5, f7 = 15/|r|^7,
//   grad_x [w.K(r) m] = f5 [b m + a w + (w.m) r] - f7 a b r       (times 1/(4 pi))
// accumulated per pair as g += f5 V + (f5 C - f7 P) r with V = sum(b m + a w),
// C = sum(w.m), P = sum(a b) over the states.  Self pairs give zero; a
// coincident non-self pair gives NaN like the forward field.
template <int KG, bool FULL, bool PAIRED>
__device__ __forceinline__ void p2p_grad_chunk(const float4 &ti, int self, const float4 *sPos,
                                               const float4 *m_row0, int Kr, int qbeg, int sn, int F, int kvalid,
                                               const float (&w)[KG][3], float (&g)[3]) {
#pragma unroll 2
  for (int q = qbeg; q < sn; q += F) {
    const float4 s = sPos[q];
    const float dx = ti.x - s.x, dy = ti.y - s.y, dz = ti.z - s.z;
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    const bool is_self = __float_as_int(s.w) == self;
    const float rinv = is_self ? 0.0F : rsqrtf(r2);
    const float r2inv = rinv * rinv;
    const float f5 = 3.0F * r2inv * r2inv * rinv;
    const float f7 = 5.0F * f5 * r2inv;
    const float4 *mq = m_row0 + q * Kr;
    float vx = 0.0F, vy = 0.0F, vz = 0.0F, C = 0.0F, P = 0.0F;
#pragma unroll
    for (int st = 0; st < KG; ++st) {
      if (FULL || st < kvalid) {
        float4 m;
        if constexpr (PAIRED) {
          const float4 pa = mq[st & ~1], pb = mq[st | 1];
          m = (st & 1) ? make_float4(pa.y, pa.w, pb.y, 0.0F) : make_float4(pa.x, pa.z, pb.x, 0.0F);
        } else {
          m = mq[st];
        }
        const float a = fmaf(m.x, dx, fmaf(m.y, dy, m.z * dz));
        const float b = fmaf(w[st][0], dx, fmaf(w[st][1], dy, w[st][2] * dz));
        C = fmaf(w[st][0], m.x, fmaf(w[st][1], m.y, fmaf(w[st][2], m.z, C)));
        P = fmaf(a, b, P);
        vx = fmaf(b, m.x, fmaf(a, w[st][0], vx));
        vy = fmaf(b, m.y, fmaf(a, w[st][1], vy));
        vz = fmaf(b, m.z, fmaf(a, w[st][2], vz));
      }
    }
    const float coef = fmaf(f5, C, -f7 * P);
    g[0] = fmaf(f5, vx, fmaf(coef, dx, g[0]));
    g[1] = fmaf(f5, vy, fmaf(coef, dy, g[1]));
    g[2] = fmaf(f5, vz, fmaf(coef, dz, g[2]));
  }
}

// MODE 0: field; 1: field and potential (near[nt][K] = (phi, H) / 4 pi);
// 2: position gradient of sum_k w_k . H_k, partial sums per state group
//    gpart[nt][G] (G = ceil(K / KG)) from the weights W[nt][K] (plain layout).
// PAIRED: the sorted moments use the paired layout (rows of round_up(K, 2)
// float4), K >= 4.
// SB: states per state block, CB: sources per moment chunk at the widest
// state window (kStateBlock, kChunkB; or kStateBlockCorun, kChunkCorun for
// the co-resident form).
template <int KG, int MODE, bool PAIRED, int SB, int CB>
__device__ __forceinline__ void p2p_kb_body(const float4 *__restrict__ src_rel, const float4 *__restrict__ mom,
                                            const int *__restrict__ src_off, const float4 *__restrict__ tgt_rel,
                                            const int4 *__restrict__ work, const int *__restrict__ self_idx,
                                            int depth, int K, float4 *__restrict__ near,
                                            const float4 *__restrict__ W, int k_begin, int k_end, int accumulate,
                                            float acc_phi_scale, int unit_index) {
  constexpr bool PHI = MODE == 1;
  constexpr bool GRAD = MODE == 2;
  extern __shared__ float4 dynb[];
  float4 *sPos = dynb;                                            // [kNeighbourCap]
  float4 *sMom = sPos + kNeighbourCap;                            // [kBufs][CB][Kr <= SB + 9]
  __shared__ Neighbours nb;
  const int4 unit = work[unit_index];
  const int leaf = unit.x;
  const int t0 = unit.y;
  const int nt = unit.z;
  if (threadIdx.x < 32) build_neighbours(nb, leaf, depth, src_off, threadIdx.x);
  __syncthreads();
  const int total = nb.prefix[nb.count];
  const int tid = threadIdx.x;
  bool staged = false; // positions of the single pass already in shared memory
  for (int kblk = k_begin; kblk < k_end; kblk += SB) {
    const int Kc = min(SB, k_end - kblk);
    const int G = (Kc + KG - 1) / KG;
    const int items = nt * G;
    for (int ib = 0, r = 0; ib < items; ib += r) {
      // This round's items r and lanes per item F (a power of two <= 8):
      // the F that keeps the most of the 256 lanes busy (the fewest lanes
      // per item among equals), e.g. 72 items -> 64 items x 4 lanes, then
      // 8 x 8, instead of 72 x 2 with 112 lanes idle.
      int F = 1, busy = 0;
      for (int fc = 1; fc <= 8; fc <<= 1) {
        const int lanes = min(items - ib, kKbThreads / fc) * fc;
        if (lanes > busy) {
          busy = lanes;
          F = fc;
        }
      }
      r = min(items - ib, kKbThreads / F);
      const int li = tid / F;
      const int f = tid - li * F;
      const bool valid = li < r;
      const int item = ib + (valid ? li : 0);
      const int g = item / nt;
      const int t = item - g * nt;
      const int kb = g * KG;                 // within the state block
      const int kvalid = min(KG, Kc - kb);
      const int k_lo = (ib / nt) * KG;       // the round's state window [k_lo, k_hi)
      const int k_hi = min(Kc, ((ib + r - 1) / nt + 1) * KG);
      const int Kw = PAIRED ? (k_hi - k_lo + 1) & ~1 : k_hi - k_lo; // staged float4 units per source
      const int Kr = mrow_stride<KG>(Kw);
      // sources per chunk: CB at the widest window, more for narrower
      // windows (a chunk buffer holds CB rows of the widest stride), so
      // each chunk carries about the same work between barriers
      const int chunkB = CB * (mrow_stride<KG>((min(K, SB) + 1) & ~1) / Kr);
      const int mrow = PAIRED ? (K + 1) & ~1 : K;                   // global row length (float4)
      const int i = t0 + t;
      const float4 ti = tgt_rel[i];
      const int self = self_idx != nullptr ? self_idx[i] : -1;
      // staged position of the self source in the neighbourhood (-1: none)
      int self_g = -1;
      if (self >= 0)
        for (int c = 0; c < nb.count; ++c) {
          const int off = self - nb.begin[c];
          if (off >= 0 && off < nb.prefix[c + 1] - nb.prefix[c]) self_g = nb.prefix[c] + off;
        }
      float acc[KG][4];
#pragma unroll
      for (int st = 0; st < KG; ++st) acc[st][0] = acc[st][1] = acc[st][2] = acc[st][3] = 0.0F;
      float2 acc2[KG / 2][4];
#pragma unroll
      for (int pr = 0; pr < KG / 2; ++pr) acc2[pr][0] = acc2[pr][1] = acc2[pr][2] = acc2[pr][3] = make_float2(0, 0);
      float wreg[KG][3];
      float gacc[3] = {0.0F, 0.0F, 0.0F};
      if constexpr (GRAD) {
#pragma unroll
        for (int st = 0; st < KG; ++st) {
          const float4 wv = st < kvalid ? W[static_cast<long long>(i) * K + kblk + kb + st] : make_float4(0, 0, 0, 0);
          wreg[st][0] = wv.x;
          wreg[st][1] = wv.y;
          wreg[st][2] = wv.z;
        }
      }
      for (int pass = 0; pass < total; pass += kNeighbourCap) {
        const int pn = min(kNeighbourCap, total - pass);
        if (!staged || total > kNeighbourCap) {
          __syncthreads();
          for (int q = tid; q < pn; q += kKbThreads) {
            float4 pos;
            int j;
            stage_source(nb, pass + q, src_rel, pos, j);
            sPos[q] = pos;
          }
          __syncthreads();
          staged = true;
        }
        const int chunks = (pn + chunkB - 1) / chunkB;
        // Copy element e = q * Kw + k of a chunk; each thread walks e = tid,
        // tid + 256, ... incrementally (no division in the loop).
        const int cq0 = tid / Kw, ck0 = tid - cq0 * Kw;
        const int cqs = kKbThreads / Kw, cks = kKbThreads - cqs * Kw;
        auto issue = [&](int c) {
          const int q0 = c * chunkB;
          const int sn = min(chunkB, pn - q0);
          float4 *dst = sMom + (c % kBufs) * chunkB * Kr;
          int q = cq0, k = ck0;
          while (q < sn) {
            cp_async16(dst + q * Kr + mrow_pos<KG>(k),
                       mom + static_cast<long long>(__float_as_int(sPos[q0 + q].w)) * mrow + kblk + k_lo + k);
            q += cqs;
            k += cks;
            if (k >= Kw) {
              k -= Kw;
              ++q;
            }
          }
          cp_async_commit();
        };
        for (int j = 0; j < kBufs - 1; ++j) {
          if (j < chunks)
            issue(j);
          else
            cp_async_commit(); // one group per step keeps the wait count uniform
        }
        for (int c = 0; c < chunks; ++c) {
          cp_async_wait<kBufs - 2>(); // chunk c has landed (this thread's copies)
          __syncthreads();            // ... and every thread's; all are done with chunk c - 1
          if (c + kBufs - 1 < chunks)
            issue(c + kBufs - 1); // into the buffer chunk c - 1 used
          else
            cp_async_commit();
          const int q0 = c * chunkB;
          const int sn = min(chunkB, pn - q0);
          if (valid) {
            const float4 *m_row0 = sMom + (c % kBufs) * chunkB * Kr + mrow_pos<KG>(kb - k_lo);
            if constexpr (GRAD) {
              if (kvalid == KG)
                p2p_grad_chunk<KG, true, PAIRED>(ti, self, sPos + q0, m_row0, Kr, f, sn, F, kvalid, wreg,
                                                 gacc);
              else
                p2p_grad_chunk<KG, false, PAIRED>(ti, self, sPos + q0, m_row0, Kr, f, sn, F, kvalid, wreg,
                                                  gacc);
            } else if constexpr (PAIRED) {
              const int self_q = self_g >= 0 ? self_g - pass - q0 : -1;
              if (kvalid == KG)
                p2p_kb_chunk_x2<KG, PHI, true>(ti, self_q, sPos + q0, m_row0, Kr, f, sn, F, kvalid, acc2);
              else
                p2p_kb_chunk_x2<KG, PHI, false>(ti, self_q, sPos + q0, m_row0, Kr, f, sn, F, kvalid, acc2);
            } else {
              if (kvalid == KG)
                p2p_kb_chunk<KG, PHI, true>(ti, self, sPos + q0, m_row0, Kr, f, sn, F, kvalid, acc);
              else
                p2p_kb_chunk<KG, PHI, false>(ti, self, sPos + q0, m_row0, Kr, f, sn, F, kvalid, acc);
            }
          }
        }
        __syncthreads(); // the next pass or round refills the buffers
      }
      if constexpr (GRAD) {
        for (int o = 1; o < F; o <<= 1)
#pragma unroll
          for (int c = 0; c < 3; ++c) gacc[c] += __shfl_xor_sync(0xffffffffu, gacc[c], o);
        if (valid && f == 0)
          near[static_cast<long long>(i) * ((K + KG - 1) / KG) + kblk / KG + g] =
              make_float4(gacc[0] * kInvFourPiF, gacc[1] * kInvFourPiF, gacc[2] * kInvFourPiF, 0.0F);
        continue;
      }
      if constexpr (PAIRED) {
#pragma unroll
        for (int st = 0; st < KG; ++st)
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[st][c] = (st & 1) ? acc2[st >> 1][c].y : acc2[st >> 1][c].x;
      }
      if (F > 1) {
#pragma unroll
        for (int st = 0; st < KG; ++st)
#pragma unroll
          for (int c = 0; c < 4; ++c)
            for (int o = 1; o < F; o <<= 1) acc[st][c] += __shfl_xor_sync(0xffffffffu, acc[st][c], o);
      }
      if (valid && f == 0) {
        float4 *out = near + static_cast<long long>(i) * K + kblk + kb;
#pragma unroll
        for (int st = 0; st < KG; ++st)
          if (st < kvalid) {
            const float4 v = make_float4(acc[st][0] * kInvFourPiF, acc[st][1] * kInvFourPiF, acc[st][2] * kInvFourPiF,
                                         acc[st][3] * kInvFourPiF);
            if (accumulate) {
              // onto the far-field results: phi = (far + near) * phi_scale,
              // H = near - grad far (accumulate == 2: potential only, H stays 0)
              const float4 o = out[st];
              out[st] = accumulate == 1 ? make_float4(fmaf(v.x, acc_phi_scale, o.x), o.y + v.y, o.z + v.z, o.w + v.w)
                                        : make_float4(fmaf(v.x, acc_phi_scale, o.x), o.y, o.z, o.w);
            } else {
              out[st] = v;
            }
          }
      }
    }
  }
}

template <int KG, int MODE, bool PAIRED>
__global__ void __launch_bounds__(kKbThreads, 2)
    p2p_kb_kernel(const float4 *__restrict__ src_rel, const float4 *__restrict__ mom,
                  const int *__restrict__ src_off, const float4 *__restrict__ tgt_rel,
                  const int4 *__restrict__ work, const int *__restrict__ self_idx, int depth, int K,
                  float4 *__restrict__ near, const float4 *__restrict__ W, int k_begin, int k_end, int accumulate,
                  float acc_phi_scale) {
  p2p_kb_body<KG, MODE, PAIRED, kStateBlock, kChunkB>(src_rel, mom, src_off, tgt_rel, work, self_idx, depth, K, near, W,
                                             k_begin, k_end, accumulate, acc_phi_scale, blockIdx.x);
}

// The co-resident form (see kStateBlockCorun), persistent: the grid is two
// CTAs per SM, each taking work units from `next_unit` (zero at launch) until
// none are left.  A kernel with CTAs still waiting to be placed keeps a
// lower-priority kernel's CTAs off the SMs even where they would fit, so the
// near field leaves nothing waiting: every CTA is placed at launch and the
// far field's CTAs take the room left beside them.
template <int KG, int MODE, bool PAIRED>
__global__ void __maxnreg__(kKbRegsCorun)
    p2p_kb_corun_kernel(const float4 *__restrict__ src_rel, const float4 *__restrict__ mom,
                        const int *__restrict__ src_off, const float4 *__restrict__ tgt_rel,
                        const int4 *__restrict__ work, int n_work, int *__restrict__ next_unit,
                        const int *__restrict__ self_idx, int depth, int K, float4 *__restrict__ near,
                        const float4 *__restrict__ W, int k_begin, int k_end, int accumulate, float acc_phi_scale) {
  __shared__ int s_unit;
  for (;;) {
    __syncthreads(); // the previous unit is done with shared memory (and s_unit)
    if (threadIdx.x == 0) s_unit = atomicAdd(next_unit, 1);
    __syncthreads();
    const int u = s_unit;
    if (u >= n_work) break;
    p2p_kb_body<KG, MODE, PAIRED, kStateBlockCorun, kChunkCorun>(src_rel, mom, src_off, tgt_rel, work, self_idx, depth, K, near,
                                                    W, k_begin, k_end, accumulate, acc_phi_scale, u);
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

// FP64 direct position gradient of w_i . H_i (validation reference of the
// reverse mode): g_i = sum_{j != self_i} (1/(4 pi)) { (3/|r|^5)[(w.r) m + (m.r) w
// + (w.m) r] - 15 (m.r)(w.r) r / |r|^7 },  r = x_i - y_j.
__global__ void __launch_bounds__(256) direct_grad_fp64_kernel(const double *__restrict__ src,
                                                               const double *__restrict__ mom, int ns,
                                                               const double *__restrict__ tgt, int nt,
                                                               const int *__restrict__ self,
                                                               const double *__restrict__ w,
                                                               double *__restrict__ grad) {
  __shared__ double sp[256][3];
  __shared__ double sm[256][3];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < nt;
  double x = 0, y = 0, z = 0, wx = 0, wy = 0, wz = 0;
  int me = -1;
  if (active) {
    x = tgt[3 * i];
    y = tgt[3 * i + 1];
    z = tgt[3 * i + 2];
    wx = w[3 * i];
    wy = w[3 * i + 1];
    wz = w[3 * i + 2];
    me = self != nullptr ? self[i] : -1;
  }
  double gx = 0, gy = 0, gz = 0;
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
        const double rinv5 = rinv * rinv * rinv * rinv * rinv;
        const double a = sm[q][0] * rx + sm[q][1] * ry + sm[q][2] * rz;
        const double b = wx * rx + wy * ry + wz * rz;
        const double c = wx * sm[q][0] + wy * sm[q][1] + wz * sm[q][2];
        const double f5 = 3.0 * rinv5, f7 = 15.0 * rinv5 * rinv * rinv * a * b;
        gx += f5 * (b * sm[q][0] + a * wx + c * rx) - f7 * rx;
        gy += f5 * (b * sm[q][1] + a * wy + c * ry) - f7 * ry;
        gz += f5 * (b * sm[q][2] + a * wz + c * rz) - f7 * rz;
      }
    }
  }
  if (active) {
    const double k = 1.0 / (4.0 * 3.14159265358979323846);
    grad[3 * i] = gx * k;
    grad[3 * i + 1] = gy * k;
    grad[3 * i + 2] = gz * k;
  }
}

template <int KG> size_t p2p_kb_smem_bytes(int K, int state_block, int chunk) {
  const int Kc = (std::min(K, state_block) + 1) & ~1; // widest window (paired rows round up)
  const int Kr = mrow_stride<KG>(Kc);
  return sizeof(float4) * kNeighbourCap + sizeof(float4) * kBufs * chunk * static_cast<size_t>(Kr);
}

template <int KG, bool PAIRED, int MODE>
void launch_kb_mode(const float4 *src_rel, const float4 *mom, const int *src_off, const float4 *tgt_rel,
                    const int4 *work, int n_work, const int *self_idx, int depth, int K, float4 *near,
                    const float4 *W, cudaStream_t s, int k_begin, int k_end, int accumulate, float acc_phi_scale,
                    const CorunLaunch *corun) {
  if (corun != nullptr) {
    cudaMemsetAsync(corun->next_unit, 0, sizeof(int), s);
    const int grid = std::min(n_work, corun->ctas);
    p2p_kb_corun_kernel<KG, MODE, PAIRED><<<grid, kKbThreads, p2p_kb_smem_bytes<KG>(K, kStateBlockCorun, kChunkCorun), s>>>(
        src_rel, mom, src_off, tgt_rel, work, n_work, corun->next_unit, self_idx, depth, K, near, W, k_begin, k_end,
        accumulate, acc_phi_scale);
  } else
    p2p_kb_kernel<KG, MODE, PAIRED><<<n_work, kKbThreads, p2p_kb_smem_bytes<KG>(K, kStateBlock, kChunkB), s>>>(
        src_rel, mom, src_off, tgt_rel, work, self_idx, depth, K, near, W, k_begin, k_end, accumulate, acc_phi_scale);
}

template <int KG, bool PAIRED>
void launch_kb(const float4 *src_rel, const float4 *mom, const int *src_off, const float4 *tgt_rel,
               const int4 *work, int n_work, const int *self_idx, int depth, int K, int mode, float4 *near, const float4 *W,
               cudaStream_t s, int k_begin, int k_end, int accumulate, float acc_phi_scale, const CorunLaunch *corun) {
  if (n_work == 0) return;
  if (mode == 1)
    launch_kb_mode<KG, PAIRED, 1>(src_rel, mom, src_off, tgt_rel, work, n_work, self_idx, depth, K, near, W, s, k_begin,
                                  k_end, accumulate, acc_phi_scale, corun);
  else if (mode == 2)
    launch_kb_mode<KG, PAIRED, 2>(src_rel, mom, src_off, tgt_rel, work, n_work, self_idx, depth, K, near, W, s, k_begin,
                                  k_end, accumulate, acc_phi_scale, corun);
  else
    launch_kb_mode<KG, PAIRED, 0>(src_rel, mom, src_off, tgt_rel, work, n_work, self_idx, depth, K, near, W, s, k_begin,
                                  k_end, accumulate, acc_phi_scale, corun);
}

// K >= 8: groups of 8 states, paired layout; 4 <= K < 8: groups of 4,
// paired; K = 2, 3: groups of 4, plain layout.  (Groups of 16 were measured
// slower at K = 64: the accumulators no longer fit the register budget.)
void launch_kb_any(const float4 *src_rel, const float4 *mom, const int *src_off, const float4 *tgt_rel,
                   const int4 *work, int n_work, const int *self_idx, int depth, int K, int mode, float4 *near, const float4 *W,
                   cudaStream_t s, int k_begin = 0, int k_end = -1, int accumulate = 0,
                   float acc_phi_scale = 1.0F, const CorunLaunch *corun = nullptr) {
  if (k_end < 0) k_end = K;
  if (K >= 8)
    launch_kb<8, true>(src_rel, mom, src_off, tgt_rel, work, n_work, self_idx, depth, K, mode, near, W, s, k_begin, k_end, accumulate, acc_phi_scale, corun);
  else if (K >= 4)
    launch_kb<4, true>(src_rel, mom, src_off, tgt_rel, work, n_work, self_idx, depth, K, mode, near, W, s, k_begin, k_end, accumulate, acc_phi_scale, corun);
  else
    launch_kb<4, false>(src_rel, mom, src_off, tgt_rel, work, n_work, self_idx, depth, K, mode, near, W, s, k_begin, k_end, accumulate, acc_phi_scale, corun);
}

} // namespace

std::vector<int4> p2p_work_units(const int *src_off, const int *tgt_off, int depth, int sm_count, bool cap_cost) {
  const int side = 1 << depth;
  const int leaves = 1 << (3 * depth);
  std::vector<long long> sources(static_cast<size_t>(leaves), 0);
  long long total = 0;
  for (int m = 0; m < leaves; ++m) {
    const int nt = tgt_off[m + 1] - tgt_off[m];
    if (nt == 0) continue;
    int ix, iy, iz;
    demorton3(static_cast<uint32_t>(m), ix, iy, iz);
    long long sn = 0;
    for (int z = std::max(iz - 1, 0); z <= std::min(iz + 1, side - 1); ++z)
      for (int y = std::max(iy - 1, 0); y <= std::min(iy + 1, side - 1); ++y)
        for (int x = std::max(ix - 1, 0); x <= std::min(ix + 1, side - 1); ++x) {
          const uint32_t b = morton3(static_cast<uint32_t>(x), static_cast<uint32_t>(y), static_cast<uint32_t>(z));
          sn += src_off[b + 1] - src_off[b];
        }
    sources[static_cast<size_t>(m)] = sn;
    total += nt * sn;
  }
  // unit cost cap: total / (kP2pUnitsPerSm x SMs) pairs
  const long long cap = std::max(1LL, total / (static_cast<long long>(kP2pUnitsPerSm) * std::max(sm_count, 1)));
  std::vector<int4> units;
  std::vector<long long> cost;
  for (int m = 0; m < leaves; ++m) {
    const int nt = tgt_off[m + 1] - tgt_off[m];
    if (nt == 0) continue;
    const long long sn = sources[static_cast<size_t>(m)];
    int width = kP2pUnitTargets;
    if (cap_cost && sn > 0 && width * sn > cap)
      width = static_cast<int>(std::max<long long>(kP2pUnitMinTargets, cap / sn / kP2pUnitMinTargets * kP2pUnitMinTargets));
    for (int t = 0; t < nt; t += width) {
      const int tn = std::min(width, nt - t);
      units.push_back(make_int4(m, tgt_off[m] + t, tn, 0));
      cost.push_back(static_cast<long long>(tn) * sn);
    }
  }
  const long long n = static_cast<long long>(units.size());
  std::vector<int> order(units.size());
  for (size_t u = 0; u < order.size(); ++u) order[u] = static_cast<int>(u);
  // heavy: cost >= 4 x mean
  const auto heavy_end = std::stable_partition(order.begin(), order.end(),
                                               [&](int u) { return cost[static_cast<size_t>(u)] * n >= 4 * total; });
  std::stable_sort(order.begin(), heavy_end,
                   [&](int a, int b) { return cost[static_cast<size_t>(a)] > cost[static_cast<size_t>(b)]; });
  std::vector<int4> out(units.size());
  for (size_t u = 0; u < order.size(); ++u) out[u] = units[static_cast<size_t>(order[u])];
  return out;
}

namespace {

// Moment of state k of sorted source j (paired rows for K >= 4, else plain).
template <bool PAIRED>
__device__ __forceinline__ float3 moment_of(const float4 *mom, int j, int K, int k) {
  if constexpr (PAIRED) {
    const float4 *row = mom + static_cast<long long>(j) * ((K + 1) & ~1) + (k & ~1);
    const float4 a = row[0], b = row[1];
    return (k & 1) ? make_float3(a.y, a.w, b.y) : make_float3(a.x, a.z, b.x);
  } else {
    const float4 m = mom[static_cast<long long>(j) * K + k];
    return make_float3(m.x, m.y, m.z);
  }
}

// Pair field at r (= target - source) for moment m: (phi, H) times 4 pi.
__device__ __forceinline__ float4 pair_field(float rx, float ry, float rz, float3 m) {
  const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
  const float rinv = rsqrtf(r2);
  const float v = rinv * rinv * rinv;
  const float mr = fmaf(m.x, rx, fmaf(m.y, ry, m.z * rz));
  const float f = 3.0F * mr * v * rinv * rinv;
  return make_float4(mr * v, fmaf(f, rx, -v * m.x), fmaf(f, ry, -v * m.y), fmaf(f, rz, -v * m.z));
}
// Position gradient of w . H (times 4 pi) at r for moment m.
__device__ __forceinline__ float3 pair_grad(float rx, float ry, float rz, float3 m, float3 w) {
  const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
  const float rinv = rsqrtf(r2);
  const float r2inv = rinv * rinv;
  const float f5 = 3.0F * r2inv * r2inv * rinv, f7 = 5.0F * f5 * r2inv;
  const float a = fmaf(m.x, rx, fmaf(m.y, ry, m.z * rz)), b = fmaf(w.x, rx, fmaf(w.y, ry, w.z * rz));
  const float c = fmaf(w.x, m.x, fmaf(w.y, m.y, w.z * m.z));
  const float coef = fmaf(f5, c, -f7 * a * b);
  return make_float3(fmaf(f5, fmaf(b, m.x, a * w.x), coef * rx), fmaf(f5, fmaf(b, m.y, a * w.y), coef * ry),
                     fmaf(f5, fmaf(b, m.z, a * w.z), coef * rz));
}

// Close-pair correction (see above): one warp per listed target, which walks
// its pairs (skipping its current self source); the lanes take the states
// k_begin + lane, + 32, ... and add (field at the exact r) - (field at the
// FP32 r), times 1 / (4 pi), to the near-field result in the form the
// kernel wrote it:
//   MODE 0 / 1: field / field and potential, near[i][K] (accumulate 1: onto
//     the far field, potential times phi_scale; accumulate 2: potential only);
//   MODE 2: the position gradient summed over the states, added to the
//     partial sum of state group 0, gpart[i][G].
// Both fields are formed in FP32 at their own r; at a close pair's r the
// exact one is as accurate as FP32 arithmetic allows.
template <int MODE, bool PAIRED>
__global__ void __launch_bounds__(256) p2p_close_correction_kernel(const float4 *__restrict__ mom, CloseGeometry cg,
                                                                   const int *__restrict__ self_idx, int K,
                                                                   float4 *__restrict__ near,
                                                                   const float4 *__restrict__ W, int G, int k_begin,
                                                                   int k_end, int accumulate, float acc_phi_scale) {
  const int lane = threadIdx.x & 31;
  const int entry = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (entry >= cg.n_targets) return;
  const int4 ct = cg.targets[entry]; // (target, first pair, pairs, 0)
  const int i = ct.x;
  const int self = self_idx != nullptr ? self_idx[i] : -1;
  float3 gsum = make_float3(0.0F, 0.0F, 0.0F);
  for (int q = ct.y; q < ct.y + ct.z; ++q) {
    const float4 rf = cg.r_fp32[q]; // .w: sorted source index
    const float4 re = cg.r_exact[q];
    const int j = __float_as_int(rf.w);
    if (j == self) continue;
    for (int k = k_begin + lane; k < k_end; k += 32) {
      const float3 mk = moment_of<PAIRED>(mom, j, K, k);
      if constexpr (MODE == 2) {
        const float4 wv = W[static_cast<long long>(i) * K + k];
        const float3 wk = make_float3(wv.x, wv.y, wv.z);
        const float3 ge = pair_grad(re.x, re.y, re.z, mk, wk);
        const float3 gf = pair_grad(rf.x, rf.y, rf.z, mk, wk);
        gsum.x += ge.x - gf.x;
        gsum.y += ge.y - gf.y;
        gsum.z += ge.z - gf.z;
      } else {
        const float4 fe = pair_field(re.x, re.y, re.z, mk);
        const float4 ff = pair_field(rf.x, rf.y, rf.z, mk);
        const float dphi = (fe.x - ff.x) * kInvFourPiF;
        const float dhx = (fe.y - ff.y) * kInvFourPiF, dhy = (fe.z - ff.z) * kInvFourPiF;
        const float dhz = (fe.w - ff.w) * kInvFourPiF;
        float4 &o = near[static_cast<long long>(i) * K + k];
        float4 v = o;
        if (accumulate != 0) {
          if (MODE == 1) v.x = fmaf(dphi, acc_phi_scale, v.x);
          if (accumulate == 1) {
            v.y += dhx;
            v.z += dhy;
            v.w += dhz;
          }
        } else {
          if (MODE == 1) v.x += dphi;
          v.y += dhx;
          v.z += dhy;
          v.w += dhz;
        }
        o = v;
      }
    }
  }
  if constexpr (MODE == 2) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      gsum.x += __shfl_xor_sync(0xffffffffu, gsum.x, o);
      gsum.y += __shfl_xor_sync(0xffffffffu, gsum.y, o);
      gsum.z += __shfl_xor_sync(0xffffffffu, gsum.z, o);
    }
    if (lane == 0) {
      float4 &g = near[static_cast<long long>(i) * G];
      g = make_float4(fmaf(gsum.x, kInvFourPiF, g.x), fmaf(gsum.y, kInvFourPiF, g.y), fmaf(gsum.z, kInvFourPiF, g.z),
                      g.w);
    }
  }
}

template <int MODE>
void launch_close_correction(const float4 *mom, const CloseGeometry &cg, const int *self_idx, int K, float4 *near,
                             const float4 *W, int G, int k_begin, int k_end, int accumulate, float acc_phi_scale,
                             cudaStream_t s) {
  if (cg.n_targets == 0) return;
  const int grid = (cg.n_targets + 7) / 8;
  if (K >= 4)
    p2p_close_correction_kernel<MODE, true><<<grid, 256, 0, s>>>(mom, cg, self_idx, K, near, W, G, k_begin, k_end,
                                                                 accumulate, acc_phi_scale);
  else
    p2p_close_correction_kernel<MODE, false><<<grid, 256, 0, s>>>(mom, cg, self_idx, K, near, W, G, k_begin, k_end,
                                                                  accumulate, acc_phi_scale);
}

} // namespace

// ---------------------------------------------------------------------------
// Uniformly magnetised cuboid sources (upstream SourceGeometry::UniformCuboid:
// src/cuboid.cpp:150-180 for the tensor, src/static_operators.cpp:405-470 for
// the near-field pairs).  A source j is a cuboid of side lengths h centred at
// x_j carrying the total moment m_j (magnetisation m_j / V).  Its field at a
// point r = x - x_j is H = T(r) m_j with T the cuboid's moment-to-field
// tensor, from the magnetic surface charges of the faces (the classical
// closed form of the prism's demagnetising tensor):
//   T_xx = 1/(4 pi V) sum_corners s atan(Y Z / (X R))
//   T_xy = -1/(4 pi V) sum_corners s asinh(Z / hypot(X, Y))   (xz: Y / hypot(X, Z), yz: X / hypot(Y, Z))
// over the corners (X, Y, Z) = r - (sx hx, sy hy, sz hz) / 2, sx, sy, sz = +-1,
// s = sx sy sz, R = |(X, Y, Z)|, with the limiting values 0 (0/0) and
// +-pi/2 (X = 0) the reference uses on faces and edges.  Self pairs are
// included (a cube's own field at its centre is -m / (3 V)); the potential
// is the point dipole's, (m.r) / (4 pi |r|^3), and 0 at r = 0, as upstream.
// The tensors are computed once per plan in FP64 and stored in FP32 (the
// reference's FP32 static plan stores the same), then applied by an FP32
// kernel in every evaluation.
namespace {

__device__ inline double atan_limit(double num, double den) {
  if (den != 0.0) return atan(num / den);
  if (num == 0.0) return 0.0;
  return copysign(1.5707963267948966, num);
}

__device__ inline double asinh_limit(double num, double a, double b) {
  const double d = hypot(a, b);
  return d == 0.0 ? 0.0 : asinh(num / d);
}

// Tensor (xx, xy, xz, yy, yz, zz) at r of a cuboid with half sides (a, b, c),
// times 4 pi V.
__device__ void cuboid_tensor_4piV(double x, double y, double z, double a, double b, double c, double (&t)[6]) {
  for (int q = 0; q < 6; ++q) t[q] = 0.0;
  for (int corner = 0; corner < 8; ++corner) {
    const double sx = (corner & 1) ? 1.0 : -1.0, sy = (corner & 2) ? 1.0 : -1.0, sz = (corner & 4) ? 1.0 : -1.0;
    const double X = x - sx * a, Y = y - sy * b, Z = z - sz * c;
    const double s = sx * sy * sz;
    const double R = sqrt(X * X + Y * Y + Z * Z);
    t[0] += s * atan_limit(Y * Z, X * R);
    t[3] += s * atan_limit(X * Z, Y * R);
    t[5] += s * atan_limit(X * Y, Z * R);
    t[1] -= s * asinh_limit(Z, X, Y);
    t[2] -= s * asinh_limit(Y, X, Z);
    t[4] -= s * asinh_limit(X, Y, Z);
  }
}

// One CTA per work unit, one thread per target: walks the unit's flattened
// neighbourhood and writes each pair's tensor.
__global__ void __launch_bounds__(128) cuboid_tensor_kernel(const int4 *__restrict__ work,
                                                            const long long *__restrict__ base,
                                                            const int *__restrict__ src_off, int depth,
                                                            const double *__restrict__ src_pos,
                                                            const double *__restrict__ tgt_pos, double inv_scale,
                                                            const double *__restrict__ size, int size_step,
                                                            float *__restrict__ T) {
  __shared__ Neighbours nb;
  const int4 unit = work[blockIdx.x];
  if (threadIdx.x < 32) build_neighbours(nb, unit.x, depth, src_off, threadIdx.x);
  __syncthreads();
  const int t = threadIdx.x;
  if (t >= unit.z) return;
  const int i = unit.y + t;
  const double xt = tgt_pos[3LL * i], yt = tgt_pos[3LL * i + 1], zt = tgt_pos[3LL * i + 2];
  const int total = nb.prefix[nb.count];
  float *out = T + base[blockIdx.x];
  int b = 0;
  for (int g = 0; g < total; ++g) {
    while (b + 1 < nb.count && nb.prefix[b + 1] <= g) ++b;
    const int j = nb.begin[b] + (g - nb.prefix[b]);
    const double *h = size + 3LL * j * size_step;
    const double rx = (xt - src_pos[3LL * j]) * inv_scale, ry = (yt - src_pos[3LL * j + 1]) * inv_scale,
                 rz = (zt - src_pos[3LL * j + 2]) * inv_scale;
    double v[6];
    cuboid_tensor_4piV(rx, ry, rz, 0.5 * h[0], 0.5 * h[1], 0.5 * h[2], v);
    const double f = 1.0 / (4.0 * 3.14159265358979323846 * h[0] * h[1] * h[2]);
    for (int q = 0; q < 6; ++q) out[(static_cast<long long>(g) * 6 + q) * unit.z + t] = static_cast<float>(v[q] * f);
  }
}

constexpr int kCuboidChunk = 128; // staged sources per pass

// Near field of cuboid sources: one CTA per work unit, one thread per target,
// states in blocks of KC (sources staged in chunks; each pair's tensor is
// read once per state block).  Output as the point kernels write it (see
// p2p_close_correction_kernel for `accumulate`).
template <bool PHI, bool PAIRED, int KC>
__global__ void __launch_bounds__(128) p2p_cuboid_kernel(const float4 *__restrict__ src_rel,
                                                         const float4 *__restrict__ mom,
                                                         const int *__restrict__ src_off,
                                                         const float4 *__restrict__ tgt_rel,
                                                         const int4 *__restrict__ work,
                                                         const long long *__restrict__ base,
                                                         const float *__restrict__ T, int depth, int K,
                                                         float4 *__restrict__ near, int k_begin, int k_end,
                                                         int accumulate, float acc_phi_scale) {
  __shared__ Neighbours nb;
  __shared__ float4 sPos[kCuboidChunk];
  __shared__ float4 sMom[kCuboidChunk * KC];
  const int4 unit = work[blockIdx.x];
  if (threadIdx.x < 32) build_neighbours(nb, unit.x, depth, src_off, threadIdx.x);
  __syncthreads();
  const int total = nb.prefix[nb.count];
  const int t = threadIdx.x;
  const bool mine = t < unit.z;
  const int i = unit.y + (mine ? t : 0);
  const float4 tp = tgt_rel[i];
  const float *Tu = T + base[blockIdx.x];
  for (int k0 = k_begin; k0 < k_end; k0 += KC) {
    float acc[KC][4];
#pragma unroll
    for (int kk = 0; kk < KC; ++kk) acc[kk][0] = acc[kk][1] = acc[kk][2] = acc[kk][3] = 0.0F;
    for (int sc = 0; sc < total; sc += kCuboidChunk) {
      const int sn = min(kCuboidChunk, total - sc);
      __syncthreads();
      for (int q = threadIdx.x; q < sn; q += blockDim.x) {
        float4 pos;
        int j;
        stage_source(nb, sc + q, src_rel, pos, j);
        sPos[q] = pos;
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
          const int k = k0 + kk;
          const float3 m = k < k_end ? moment_of<PAIRED>(mom, j, K, k) : make_float3(0.0F, 0.0F, 0.0F);
          sMom[q * KC + kk] = make_float4(m.x, m.y, m.z, 0.0F);
        }
      }
      __syncthreads();
      if (!mine) continue;
      for (int q = 0; q < sn; ++q) {
        const long long g6 = static_cast<long long>(sc + q) * 6 * unit.z + t;
        const float txx = Tu[g6], txy = Tu[g6 + unit.z], txz = Tu[g6 + 2 * unit.z];
        const float tyy = Tu[g6 + 3 * unit.z], tyz = Tu[g6 + 4 * unit.z], tzz = Tu[g6 + 5 * unit.z];
        float rx = 0.0F, ry = 0.0F, rz = 0.0F, v = 0.0F;
        if (PHI) {
          const float4 p = sPos[q];
          rx = tp.x - p.x;
          ry = tp.y - p.y;
          rz = tp.z - p.z;
          const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
          const float rinv = r2 > 0.0F ? rsqrtf(r2) : 0.0F;
          v = rinv * rinv * rinv * kInvFourPiF;
        }
#pragma unroll
        for (int kk = 0; kk < KC; ++kk) {
          const float4 m = sMom[q * KC + kk];
          if (PHI) acc[kk][0] = fmaf(fmaf(m.x, rx, fmaf(m.y, ry, m.z * rz)), v, acc[kk][0]);
          acc[kk][1] = fmaf(txx, m.x, fmaf(txy, m.y, fmaf(txz, m.z, acc[kk][1])));
          acc[kk][2] = fmaf(txy, m.x, fmaf(tyy, m.y, fmaf(tyz, m.z, acc[kk][2])));
          acc[kk][3] = fmaf(txz, m.x, fmaf(tyz, m.y, fmaf(tzz, m.z, acc[kk][3])));
        }
      }
    }
    if (mine) {
#pragma unroll
      for (int kk = 0; kk < KC; ++kk) {
        const int k = k0 + kk;
        if (k >= k_end) continue;
        float4 &o = near[static_cast<long long>(i) * K + k];
        if (accumulate != 0) {
          float4 w = o;
          if (PHI) w.x = fmaf(acc[kk][0], acc_phi_scale, w.x);
          if (accumulate == 1) {
            w.y += acc[kk][1];
            w.z += acc[kk][2];
            w.w += acc[kk][3];
          }
          o = w;
        } else {
          o = make_float4(PHI ? acc[kk][0] : 0.0F, acc[kk][1], acc[kk][2], acc[kk][3]);
        }
      }
    }
  }
}

template <bool PHI, bool PAIRED>
void launch_cuboid_kb(const float4 *src_rel, const float4 *mom, const int *src_off, const float4 *tgt_rel,
                      const CuboidNear &c, int depth, int K, float4 *near, int kb, int ke, int accumulate,
                      float phi_scale, cudaStream_t s) {
  if (ke - kb >= 8)
    p2p_cuboid_kernel<PHI, PAIRED, 8><<<c.n_work, 128, 0, s>>>(src_rel, mom, src_off, tgt_rel, c.work, c.base, c.T,
                                                              depth, K, near, kb, ke, accumulate, phi_scale);
  else if (ke - kb >= 4)
    p2p_cuboid_kernel<PHI, PAIRED, 4><<<c.n_work, 128, 0, s>>>(src_rel, mom, src_off, tgt_rel, c.work, c.base, c.T,
                                                              depth, K, near, kb, ke, accumulate, phi_scale);
  else
    p2p_cuboid_kernel<PHI, PAIRED, 1><<<c.n_work, 128, 0, s>>>(src_rel, mom, src_off, tgt_rel, c.work, c.base, c.T,
                                                              depth, K, near, kb, ke, accumulate, phi_scale);
}

} // namespace

void launch_cuboid_tensors(const int4 *work, int n_work, const long long *base, const int *src_off, int depth,
                           const double *src_pos, const double *tgt_pos, double inv_scale, const double *size,
                           int size_step, float *T, cudaStream_t s) {
  if (n_work == 0) return;
  cuboid_tensor_kernel<<<n_work, 128, 0, s>>>(work, base, src_off, depth, src_pos, tgt_pos, inv_scale, size,
                                              size_step, T);
}

std::vector<long long> cuboid_unit_sources(const int *src_off, const std::vector<int4> &work, int depth) {
  std::vector<long long> out(work.size(), 0);
  const int side = 1 << depth;
  for (size_t u = 0; u < work.size(); ++u) {
    int ix, iy, iz;
    demorton3(static_cast<uint32_t>(work[u].x), ix, iy, iz);
    long long n = 0;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          const int x = ix + dx, y = iy + dy, z = iz + dz;
          if (x < 0 || y < 0 || z < 0 || x >= side || y >= side || z >= side) continue;
          const uint32_t m = morton3(x, y, z);
          n += src_off[m + 1] - src_off[m];
        }
    out[u] = n;
  }
  return out;
}

void launch_p2p(const float4 *src_rel, const float4 *mom, const int *src_off,
                const float4 *tgt_rel, const int4 *work, int n_work, const int *self_idx,
                const int2 *leaf_self, const CloseGeometry &cg, int depth, int K,
                bool want_phi, float4 *near, cudaStream_t s, int k_begin, int k_end, int accumulate,
                float phi_scale, const CorunLaunch *corun, const NearTcLaunch *tc) {
  if (cg.cuboid.T != nullptr) {
    const int kb = k_begin, ke = k_end < 0 ? K : k_end;
    if (cg.cuboid.n_work == 0 || ke <= kb) return;
    if (K >= 4) {
      if (want_phi)
        launch_cuboid_kb<true, true>(src_rel, mom, src_off, tgt_rel, cg.cuboid, depth, K, near, kb, ke, accumulate,
                                     phi_scale, s);
      else
        launch_cuboid_kb<false, true>(src_rel, mom, src_off, tgt_rel, cg.cuboid, depth, K, near, kb, ke, accumulate,
                                      phi_scale, s);
    } else {
      if (want_phi)
        launch_cuboid_kb<true, false>(src_rel, mom, src_off, tgt_rel, cg.cuboid, depth, K, near, kb, ke, accumulate,
                                      phi_scale, s);
      else
        launch_cuboid_kb<false, false>(src_rel, mom, src_off, tgt_rel, cg.cuboid, depth, K, near, kb, ke,
                                       accumulate, phi_scale, s);
    }
    return;
  }
  if (n_work == 0) return;
  if (K == 1) {
    if (want_phi)
      p2p_k1_kernel<true><<<n_work, 128, 0, s>>>(src_rel, mom, src_off, tgt_rel, work, self_idx, leaf_self, depth,
                                                 near);
    else
      p2p_k1_kernel<false><<<n_work, 128, 0, s>>>(src_rel, mom, src_off, tgt_rel, work, self_idx, leaf_self, depth,
                                                  near);
  } else if (tc != nullptr && K >= kNearTcMinStates && K <= kNearTcMaxStates && k_begin == 0 &&
             (k_end < 0 || k_end == K) && accumulate == 0) {
    launch_near_tc(*tc, mom, tgt_rel, self_idx, depth, K, want_phi, near, s);
  } else {
    launch_kb_any(src_rel, mom, src_off, tgt_rel, work, n_work, self_idx, depth, K, want_phi ? 1 : 0, near, nullptr, s,
                  k_begin, k_end, accumulate, phi_scale, corun);
  }
  const int kb = k_begin, ke = k_end < 0 ? K : k_end;
  if (want_phi)
    launch_close_correction<1>(mom, cg, self_idx, K, near, nullptr, 0, kb, ke, accumulate, phi_scale, s);
  else
    launch_close_correction<0>(mom, cg, self_idx, K, near, nullptr, 0, kb, ke, accumulate, phi_scale, s);
}

int p2p_grad_groups(int K) { return K >= 8 ? (K + 7) / 8 : (K + 3) / 4; }

void launch_p2p_grad_close(const float4 *mom, const CloseGeometry &cg, const int *self_idx, int K, const float4 *W,
                           float4 *gpart, cudaStream_t s) {
  launch_close_correction<2>(mom, cg, self_idx, K, gpart, W, p2p_grad_groups(K), 0, K, 0, 1.0F, s);
}

void launch_p2p_grad(const float4 *src_rel, const float4 *mom, const int *src_off, const float4 *tgt_rel,
                     const int4 *work, int n_work, const int *self_idx, const CloseGeometry &cg, int depth, int K,
                     const float4 *W, float4 *gpart, cudaStream_t s, const CorunLaunch *corun) {
  launch_kb_any(src_rel, mom, src_off, tgt_rel, work, n_work, self_idx, depth, K, 2, gpart, W, s, 0, -1, 0, 1.0F,
                corun);
  launch_close_correction<2>(mom, cg, self_idx, K, gpart, W, p2p_grad_groups(K), 0, K, 0, 1.0F, s);
}

namespace {

// Close-pair search over every target's list 1, with r formed in FP32
// exactly as the near-field kernels form it (staged source = leaf-relative
// position + neighbour offset; exactly coincident points excluded).  COUNT:
// counts[i][l] = pairs with r^2 below thresholds[l] (l < kCloseLevels);
// else: writes the pairs of threshold r2_max from out_first[i] on, as
// (FP32 r, source index in .w) and r from the FP64 root-normalised positions.
// One CTA per work unit (at most 128 targets, one thread each), the
// neighbourhood staged in chunks of kSearchChunk.
constexpr int kSearchChunk = 512;

template <bool COUNT>
__global__ void __launch_bounds__(128) p2p_close_search_kernel(
    const float4 *__restrict__ src_rel, const int *__restrict__ src_off, const float4 *__restrict__ tgt_rel,
    const int4 *__restrict__ work, int depth, float4 thresholds, int *__restrict__ counts, float r2_max,
    const int *__restrict__ out_first, const double *__restrict__ src_abs, const double *__restrict__ tgt_abs,
    float4 *__restrict__ r_fp32, float4 *__restrict__ r_exact) {
  __shared__ Neighbours nb;
  __shared__ float4 sPos[kSearchChunk];
  const int4 unit = work[blockIdx.x];
  if (threadIdx.x < 32) build_neighbours(nb, unit.x, depth, src_off, threadIdx.x);
  __syncthreads();
  const int total = nb.prefix[nb.count];
  const bool mine = static_cast<int>(threadIdx.x) < unit.z;
  const int i = unit.y + (mine ? static_cast<int>(threadIdx.x) : 0);
  const float4 t = tgt_rel[i];
  int c0 = 0, c1 = 0, c2 = 0, c3 = 0;
  int out = (!COUNT && mine) ? out_first[i] : 0;
  for (int sc = 0; sc < total; sc += kSearchChunk) {
    const int sn = min(kSearchChunk, total - sc);
    __syncthreads();
    for (int q = threadIdx.x; q < sn; q += blockDim.x) {
      float4 p;
      int j;
      stage_source(nb, sc + q, src_rel, p, j);
      sPos[q] = p;
    }
    __syncthreads();
    if (!mine) continue;
    for (int q = 0; q < sn; ++q) {
      const float4 p = sPos[q];
      const float rx = t.x - p.x, ry = t.y - p.y, rz = t.z - p.z;
      const float r2 = fmaf(rx, rx, fmaf(ry, ry, rz * rz));
      if (!(r2 > 0.0F)) continue;
      if constexpr (COUNT) {
        c0 += r2 < thresholds.x;
        c1 += r2 < thresholds.y;
        c2 += r2 < thresholds.z;
        c3 += r2 < thresholds.w;
      } else if (r2 < r2_max) {
        const int j = __float_as_int(p.w);
        r_fp32[out] = make_float4(rx, ry, rz, p.w);
        r_exact[out] = make_float4(static_cast<float>(tgt_abs[3LL * i] - src_abs[3LL * j]),
                                   static_cast<float>(tgt_abs[3LL * i + 1] - src_abs[3LL * j + 1]),
                                   static_cast<float>(tgt_abs[3LL * i + 2] - src_abs[3LL * j + 2]), 0.0F);
        ++out;
      }
    }
  }
  if (COUNT && mine) {
    counts[4 * i] = c0;
    counts[4 * i + 1] = c1;
    counts[4 * i + 2] = c2;
    counts[4 * i + 3] = c3;
  }
}

} // namespace

void launch_p2p_close_count(const float4 *src_rel, const int *src_off, const float4 *tgt_rel, const int4 *work,
                            int n_work, int depth, const float (&thresholds)[kCloseLevels], int *counts,
                            cudaStream_t s) {
  if (n_work == 0) return;
  p2p_close_search_kernel<true><<<n_work, 128, 0, s>>>(
      src_rel, src_off, tgt_rel, work, depth, make_float4(thresholds[0], thresholds[1], thresholds[2], thresholds[3]),
      counts, 0.0F, nullptr, nullptr, nullptr, nullptr, nullptr);
}

void launch_p2p_close_write(const float4 *src_rel, const int *src_off, const float4 *tgt_rel, const int4 *work,
                            int n_work, int depth, float r2_max, const int *out_first, const double *src_abs,
                            const double *tgt_abs, float4 *r_fp32, float4 *r_exact, cudaStream_t s) {
  if (n_work == 0) return;
  p2p_close_search_kernel<false><<<n_work, 128, 0, s>>>(src_rel, src_off, tgt_rel, work, depth,
                                                        make_float4(0.0F, 0.0F, 0.0F, 0.0F), nullptr, r2_max,
                                                        out_first, src_abs, tgt_abs, r_fp32, r_exact);
}

template <int KG, bool PAIRED> void configure_p2p_kb(size_t max_smem) {
  allow_dynamic_smem(p2p_kb_kernel<KG, 0, PAIRED>, max_smem);
  allow_dynamic_smem(p2p_kb_kernel<KG, 1, PAIRED>, max_smem);
  allow_dynamic_smem(p2p_kb_kernel<KG, 2, PAIRED>, max_smem);
  allow_dynamic_smem(p2p_kb_corun_kernel<KG, 0, PAIRED>, max_smem);
  allow_dynamic_smem(p2p_kb_corun_kernel<KG, 1, PAIRED>, max_smem);
  allow_dynamic_smem(p2p_kb_corun_kernel<KG, 2, PAIRED>, max_smem);
  // the co-resident form shares its SMs with a far-field CTA
  prefer_max_shared_carveout(p2p_kb_corun_kernel<KG, 0, PAIRED>);
  prefer_max_shared_carveout(p2p_kb_corun_kernel<KG, 1, PAIRED>);
  prefer_max_shared_carveout(p2p_kb_corun_kernel<KG, 2, PAIRED>);
}

size_t p2p_corun_cta_smem(int K) {
  cudaFuncAttributes attr{};
  if (K >= 8) {
    cudaFuncGetAttributes(&attr, p2p_kb_corun_kernel<8, 1, true>);
    return p2p_kb_smem_bytes<8>(K, kStateBlockCorun, kChunkCorun) + attr.sharedSizeBytes;
  }
  cudaFuncGetAttributes(&attr, p2p_kb_corun_kernel<4, 1, true>);
  return p2p_kb_smem_bytes<4>(K, kStateBlockCorun, kChunkCorun) + attr.sharedSizeBytes;
}

void configure_p2p(size_t max_smem) {
  configure_p2p_kb<8, true>(max_smem);
  configure_p2p_kb<4, true>(max_smem);
  configure_p2p_kb<4, false>(max_smem);
}

void launch_direct_grad_fp64(const double *src, const double *mom, int ns, const double *tgt, int nt,
                             const int *self, const double *w, double *grad, cudaStream_t s) {
  if (nt == 0) return;
  direct_grad_fp64_kernel<<<(nt + 255) / 256, 256, 0, s>>>(src, mom, ns, tgt, nt, self, w, grad);
}

void launch_direct_fp64(const double *src, const double *mom, int ns, const double *tgt, int nt,
                        const int *self, double *phi, double *field, cudaStream_t s) {
  if (nt == 0) return;
  direct_fp64_kernel<<<(nt + 255) / 256, 256, 0, s>>>(src, mom, ns, tgt, nt, self, phi, field);
}

} // namespace cdfmm_b200
