// Tensor-core (tcgen05) M2L: launch interface.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

namespace cdfmm_b200 {

struct TcArgs {
  const uint8_t *a_hi;     // packed BF16 hi boxes [box][32-alpha chunk][Kp/8][w/8][8][8]
  const uint8_t *a_lo;     // packed BF16 lo boxes
  const uint8_t *b_tiles;  // [343 slots][32-alpha chunk][hi, lo][Npad/8][w/8][8][8]
  const int4 *tiles;       // per CTA: (level, class, first parent Morton index, target count)
  const float *scale_l;    // [depth+1][n] exact powers of two
  float *L;                // [node][n][K] FP32 locals (overwritten)
  float *const *L_list;    // or (stacked problems, one state each): state k's locals at L_list[k][node][n]
  int *error_flag;         // set nonzero if a bounded wait expired
  int n, K, Kp, Kpad, Npad;
  int node_base;           // flat node index of packed box 0
  int zero_node;           // packed index of the all-zero box
  int stages;
  int m_tiles;             // 128-row accumulators per CTA sharing each B tile
  int acc_stride;          // TMEM columns between accumulators (multiple of 32)
  int fuse_n;              // 1: A_hi x [B_hi | B_lo] as one N = 2 Npad MMA (acc_stride >= 2 Npad)
  uint32_t tmem_cols;
  uint32_t box_bytes;      // Kp * Kpad * 2
  uint32_t wait_limit;     // iterations of each pipeline progress wait (kTcWaitLimit; 0 = expire at once)
};

// Default iterations of a bounded mbarrier wait (about 2 s with the back-off).
constexpr uint32_t kTcWaitLimit = 1u << 26;

// Largest target count of one CTA: m_tiles (<= 4) x 128 / Kp with Kp >= 8.
constexpr int kTcMaxTargets = 64;

size_t m2l_tc_smem_bytes(int Npad, int m_tiles, int stages);
void launch_m2l_pack(const float *M, const float *scale_m, const int8_t *basis, void *hi, void *lo, int n, int K,
                     int Kp, int Kpad, int depth, int node_base, int n_boxes, cudaStream_t s,
                     const float *const *M_list = nullptr);
void launch_m2l_tc(const TcArgs &args, int n_tiles, cudaStream_t s);
bool configure_m2l_tc(size_t max_smem);
// Runs a kernel whose bounded mbarrier wait must expire (nothing arrives)
// and set *error_flag = 2, exactly as an expired wait of the M2L pipeline.
void launch_bounded_wait_selftest(int *error_flag, cudaStream_t s);
std::vector<uint16_t> pack_m2l_b_tiles(const std::vector<double> &T64, int n, int Npad, int Kpad);

} // namespace cdfmm_b200
