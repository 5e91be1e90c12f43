// M2L on the 5th-generation tensor cores (tcgen05), split BF16 with FP32
// accumulation in tensor memory -- the batched (K >= 8 states) path.
//
// For one level, parity class c and a tile of T targets (rows = target x
// state, 128 rows = one MMA M tile), the kernel accumulates over the 189 list2
// offsets o of class c (implicit list2, see m2l_simt.cu):
//
//   D[(t, k), beta] += sum_alpha A_o[(t, k), alpha] * B_o[beta, alpha]
//   A_o[(t, k), alpha] = 2^(l|alpha|) M_alpha(t - o, state k)   (exact scaling)
//   B_o[beta, alpha]   = T^(o)[beta][alpha] = D^{alpha+beta} G(o)
//
// with each operand split x = hi + lo in BF16 and three products
// A_hi*B_hi + A_hi*B_lo + A_lo*B_hi (the dropped lo*lo term is ~2^-16 of the
// product), then L = 2^(l(|beta|+1)) D in the epilogue (upstream math:
// docs/math.md "M2L normalisation and cross-level reuse").
//
// Data movement: one thread issues bulk async copies (cp.async.bulk, TMA
// engine) of each source box's K-row block (contiguous, already in the
// canonical no-swizzle K-major core-matrix layout written by the pack kernel)
// and of the offset's B tile (pre-tiled on the host), completing on an
// mbarrier; the same thread issues tcgen05.mma from shared memory into the
// TMEM accumulator and commits to a second mbarrier that frees the stage.
// Stages are double buffered so copies of offset o+1 overlap the MMAs of o.
// Every wait is bounded: on expiry the kernel records an error code, stops
// issuing, drains what it issued, frees its TMEM and returns.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "far_kernels.hpp"
#include "kernels.cuh"
#include "m2l_tc.hpp"

namespace cdfmm_b200 {

namespace {

constexpr int kTcThreads = 128;
constexpr uint32_t kWaitLimit = 1u << 26; // ~2 s with the back-off below

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (i > 64) __nanosleep(32);
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(smem_dst)),
               "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Shared-memory matrix descriptor, K-major, no swizzle: 8x16-byte core
// matrices; lbo = byte distance between K-adjacent core matrices, sbo =
// between 8-row groups (both multiples of 16); version 1 (sm_100).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= static_cast<uint64_t>((addr >> 4) & 0x3fffu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3fffu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3fffu) << 32;
  d |= static_cast<uint64_t>(1u) << 46; // version
  // base offset 0, lbo mode 0, layout type 0 (SWIZZLE_NONE)
  return d;
}

// Instruction descriptor: kind::f16, A = B = BF16, D = F32, K-major A and B, M = 128.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(kTcThreads, 1) m2l_tc_kernel(const TcArgs args) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const int tid = threadIdx.x;
  const int4 tile = args.tiles[blockIdx.x];
  const int level = tile.x;
  const int cls = tile.y;
  const int p_first = tile.z; // first parent (Morton index at level-1) of this tile
  const int count = tile.w;   // targets in this tile (<= T)
  const int cx = cls & 1, cy = (cls >> 1) & 1, cz = (cls >> 2) & 1;
  const int side = 1 << level;

  const uint32_t a_bytes = 128u * static_cast<uint32_t>(args.Kpad) * 2u;
  const uint32_t b_bytes = static_cast<uint32_t>(args.Npad) * static_cast<uint32_t>(args.Kpad) * 2u;
  const uint32_t stage_bytes = 2u * a_bytes + 2u * b_bytes;
  uint8_t *stage0 = smem;
  uint64_t *full = reinterpret_cast<uint64_t *>(smem + args.stages * stage_bytes);
  uint64_t *empty = full + args.stages;
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(empty + args.stages);
  int *abort_flag = reinterpret_cast<int *>(tmem_slot + 1);
  int *tgt_node = abort_flag + 1; // [T]
  int *tgt_xyz = tgt_node + 16;   // [T] packed coordinates

  // Zero both stages' A buffers once: rows beyond count*Kp stay zero.
  for (uint32_t q = tid; q < args.stages * stage_bytes / 16u; q += kTcThreads)
    reinterpret_cast<uint4 *>(stage0)[q] = make_uint4(0, 0, 0, 0);
  if (tid < count) {
    int px, py, pz;
    demorton3(static_cast<uint32_t>(p_first + tid), px, py, pz);
    const int tx = 2 * px + cx, ty = 2 * py + cy, tz = 2 * pz + cz;
    tgt_node[tid] = level_offset_d(level) + static_cast<int>(morton3(tx, ty, tz));
    tgt_xyz[tid] = tx | (ty << 10) | (tz << 20);
  }
  if (tid == 0) {
    for (int s = 0; s < args.stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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

  if (tid == 0) {
    const uint32_t idesc = instr_desc_bf16(args.Npad);
    const uint32_t sbo = static_cast<uint32_t>(args.Kpad) * 16u;
    const int ksteps = args.Kpad / 16;
    const uint32_t expect = 2u * static_cast<uint32_t>(count) * args.box_bytes + 2u * b_bytes;
    // the 189 offsets of this class in a fixed order
    int units = 0;
    int o_list[189];
    for (int oz = cz - 3; oz <= cz + 2; ++oz)
      for (int oy = cy - 3; oy <= cy + 2; ++oy)
        for (int ox = cx - 3; ox <= cx + 2; ++ox) {
          if (ox >= -1 && ox <= 1 && oy >= -1 && oy <= 1 && oz >= -1 && oz <= 1) continue;
          o_list[units++] = (ox + 3) * 49 + (oy + 3) * 7 + (oz + 3);
        }
    bool ok = true;
    uint32_t accumulate = 0;
    int issued = 0; // units whose MMAs were committed
    for (int step = 0; step < units + args.stages - 1 && ok; ++step) {
      if (step < units) { // produce unit `step`
        const int s = step % args.stages;
        if (step >= args.stages) ok = mbar_wait(&empty[s], ((step / args.stages) - 1) & 1);
        if (!ok) break;
        const int slot = o_list[step];
        const int ox = slot / 49 - 3, oy = (slot / 7) % 7 - 3, oz = slot % 7 - 3;
        uint8_t *st = stage0 + s * stage_bytes;
        mbar_expect_tx(&full[s], expect);
        for (int t = 0; t < count; ++t) {
          const int xyz = tgt_xyz[t];
          const int sx = (xyz & 1023) - ox, sy = ((xyz >> 10) & 1023) - oy, sz = ((xyz >> 20) & 1023) - oz;
          int src = args.zero_node;
          if (sx >= 0 && sy >= 0 && sz >= 0 && sx < side && sy < side && sz < side)
            src = level_offset_d(level) + static_cast<int>(morton3(sx, sy, sz)) - args.node_base;
          const size_t off = static_cast<size_t>(src) * args.box_bytes;
          bulk_g2s(st + t * args.box_bytes, args.a_hi + off, args.box_bytes, &full[s]);
          bulk_g2s(st + a_bytes + t * args.box_bytes, args.a_lo + off, args.box_bytes, &full[s]);
        }
        const uint8_t *bsrc = args.b_tiles + static_cast<size_t>(slot) * 2u * b_bytes;
        bulk_g2s(st + 2 * a_bytes, bsrc, b_bytes, &full[s]);
        bulk_g2s(st + 2 * a_bytes + b_bytes, bsrc + b_bytes, b_bytes, &full[s]);
      }
      const int c = step - (args.stages - 1);
      if (c >= 0) { // consume unit c
        const int s = c % args.stages;
        ok = mbar_wait(&full[s], (c / args.stages) & 1);
        if (!ok) break;
        tc_fence_after();
        const uint32_t a_hi = smem_u32(stage0 + s * stage_bytes);
        const uint32_t a_lo = a_hi + a_bytes;
        const uint32_t b_hi = a_hi + 2 * a_bytes;
        const uint32_t b_lo = b_hi + b_bytes;
        for (int ks = 0; ks < ksteps; ++ks) {
          const uint32_t koff = static_cast<uint32_t>(ks) * 256u;
          const uint64_t dah = smem_desc(a_hi + koff, 128u, sbo);
          const uint64_t dal = smem_desc(a_lo + koff, 128u, sbo);
          const uint64_t dbh = smem_desc(b_hi + koff, 128u, sbo);
          const uint64_t dbl = smem_desc(b_lo + koff, 128u, sbo);
          mma_bf16(tmem, dah, dbh, idesc, accumulate);
          accumulate = 1;
          mma_bf16(tmem, dah, dbl, idesc, 1);
          mma_bf16(tmem, dal, dbh, idesc, 1);
        }
        mma_commit(&empty[s]);
        issued = c + 1;
      }
    }
    if (!ok) {
      *abort_flag = 1;
      atomicExch(args.error_flag, 1);
    }
    // The last commit arrives once every MMA issued before it has completed.
    if (issued > 0) {
      const int last = issued - 1;
      if (!mbar_wait(&empty[last % args.stages], (last / args.stages) & 1)) {
        *abort_flag = 1;
        atomicExch(args.error_flag, 2);
      }
    }
    // Drain copies that were issued but never consumed (only after an abort).
    if (*abort_flag) {
      for (int u = issued; u < units && u < issued + args.stages; ++u) mbar_wait(&full[u % args.stages], (u / args.stages) & 1);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  // Epilogue: warp w owns TMEM lanes 32w..32w+31 (rows); scale by D_L and store.
  if (*abort_flag == 0) {
    const int warp = tid >> 5;
    const int row = tid;
    const int tt = row / args.Kp;
    const int k = row - tt * args.Kp;
    const bool valid = tt < count && k < args.K;
    const int node = valid ? tgt_node[tt] : 0;
    const long long base = static_cast<long long>(node) * args.n * args.K + k;
    const float *sl = args.scale_l + level * args.n;
    for (int c0 = 0; c0 < args.Npad; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + static_cast<uint32_t>(c0), v);
      if (valid) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int b = c0 + j;
          if (b < args.n) args.L[base + static_cast<long long>(b) * args.K] = v[j] * sl[b];
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

// Pack: scaled multipoles of levels 2..depth -> BF16 hi/lo boxes
// [box][Kp/8][Kpad/8][8 rows][8 alphas] (rows = states), the no-swizzle
// K-major core-matrix layout the MMA reads directly.  One extra all-zero box
// (index n_boxes) stands for sources outside the grid.
__global__ void m2l_pack_kernel(const float *__restrict__ M, const float *__restrict__ scale_m,
                                const int8_t *__restrict__ basis, __nv_bfloat16 *__restrict__ hi,
                                __nv_bfloat16 *__restrict__ lo, int n, int K, int Kp, int Kpad, int depth,
                                int node_base, int n_boxes) {
  const long long per_box = static_cast<long long>(Kp) * Kpad;
  const long long total = (static_cast<long long>(n_boxes) + 1) * per_box;
  for (long long q = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; q < total;
       q += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long box = q / per_box;
    const int e = static_cast<int>(q - box * per_box);
    // e enumerates [rg][cj][r8][a8]
    const int a8 = e & 7;
    const int r8 = (e >> 3) & 7;
    const int rest = e >> 6;
    const int cj = rest % (Kpad / 8);
    const int rg = rest / (Kpad / 8);
    const int k = rg * 8 + r8;
    const int a = cj * 8 + a8;
    float v = 0.0F;
    if (box < n_boxes && k < K && a < n) {
      const int node = node_base + static_cast<int>(box);
      int level = 0;
      while (level < depth && level_offset_d(level + 1) <= node) ++level;
      v = M[static_cast<long long>(node) * n * K + static_cast<long long>(a) * K + k] * scale_m[level * n + a];
    }
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[q] = h;
    lo[q] = __float2bfloat16_rn(v - __bfloat162float(h));
  }
}

} // namespace

size_t m2l_tc_smem_bytes(int Kpad, int Npad, int stages) {
  const size_t a = 128u * static_cast<size_t>(Kpad) * 2u;
  const size_t b = static_cast<size_t>(Npad) * Kpad * 2u;
  return static_cast<size_t>(stages) * (2 * a + 2 * b) + 2 * stages * sizeof(uint64_t) + 8 + 32 * sizeof(int) + 1024;
}

void launch_m2l_pack(const float *M, const float *scale_m, const int8_t *basis, void *hi, void *lo, int n, int K,
                     int Kp, int Kpad, int depth, int node_base, int n_boxes, cudaStream_t s) {
  const long long total = (static_cast<long long>(n_boxes) + 1) * Kp * Kpad;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148LL * 64));
  m2l_pack_kernel<<<blocks, 256, 0, s>>>(M, scale_m, basis, static_cast<__nv_bfloat16 *>(hi),
                                          static_cast<__nv_bfloat16 *>(lo), n, K, Kp, Kpad, depth, node_base, n_boxes);
}

void launch_m2l_tc(const TcArgs &args, int n_tiles, cudaStream_t s) {
  if (n_tiles == 0) return;
  const size_t smem = m2l_tc_smem_bytes(args.Kpad, args.Npad, args.stages);
  m2l_tc_kernel<<<n_tiles, kTcThreads, smem, s>>>(args);
}

bool configure_m2l_tc(size_t max_smem) { return allow_dynamic_smem(m2l_tc_kernel, max_smem); }

// Host: B tiles [slot][hi, lo][Npad/8][Kpad/8][8][8] BF16 from FP64 matrices
// T[slot][alpha][beta] (symmetric in alpha, beta).
std::vector<uint16_t> pack_m2l_b_tiles(const std::vector<double> &T64, int n, int Npad, int Kpad) {
  const size_t tile = static_cast<size_t>(Npad) * Kpad;
  std::vector<uint16_t> out(343 * 2 * tile, 0);
  auto bf16_bits = [](float f) -> uint16_t {
    const __nv_bfloat16 h = __float2bfloat16_rn(f);
    uint16_t b;
    std::memcpy(&b, &h, 2);
    return b;
  };
  for (int slot = 0; slot < 343; ++slot) {
    const double *Ts = T64.data() + static_cast<size_t>(slot) * n * n;
    uint16_t *hi = out.data() + static_cast<size_t>(slot) * 2 * tile;
    uint16_t *lo = hi + tile;
    for (int beta = 0; beta < n; ++beta)
      for (int alpha = 0; alpha < n; ++alpha) {
        const double v = Ts[static_cast<size_t>(alpha) * n + beta];
        const __nv_bfloat16 h = __float2bfloat16_rn(static_cast<float>(v));
        const float l = static_cast<float>(v - static_cast<double>(__bfloat162float(h)));
        const size_t at = ((static_cast<size_t>(beta / 8) * (Kpad / 8) + alpha / 8) * 8 + beta % 8) * 8 + alpha % 8;
        hi[at] = bf16_bits(static_cast<float>(v));
        lo[at] = bf16_bits(l);
      }
  }
  return out;
}

} // namespace cdfmm_b200
