// List-1 near field on the tensor cores (tcgen05, kind::tf32, three products
// of TF32 hi / lo splits): launch interface.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

namespace cdfmm_b200 {

// Sources are grouped per leaf into blocks of 4 (the last block of a leaf
// padded with empty slots); a block is the unit of the moment operand.
constexpr int kNearTcSlots = 4;      // sources per block
constexpr int kNearTcTargets = 32;   // targets per work unit (128 rows = 4 components x 32)
constexpr int kNearTcMinStates = 8;  // K range served (MMA N = K rounded up to 16, <= 64)
constexpr int kNearTcMaxStates = 64;

// Per plan: blocks and work units (built once, on the host, from the leaf
// offsets).
struct NearTcLayout {
  std::vector<int> blk_off; // [leaves + 1] first block of each leaf
  std::vector<int> blk_src; // [(n_blocks + 1) * 4] sorted source index of each slot, -1: empty
  std::vector<int4> work;   // (leaf, first target, targets <= 32, neighbourhood blocks) in leaf order
  int n_blocks = 0;         // block n_blocks is the all-empty block
  uint64_t k_cols = 0;      // sum over units of the MMA reduction length (3 x chunk-padded sources)
};
NearTcLayout near_tc_layout(const int *src_off, const int *tgt_off, int depth);

// Device arrays of one plan and per-call scratch.
struct NearTcLaunch {
  const float4 *blk_pos; // [(n_blocks + 1) * 4] leaf-relative positions, .w: sorted index (-1: empty)
  const int *blk_off;
  const int *blk_src;
  int n_blocks;
  const int4 *work;
  int n_work;
  void *b_ops;           // [(n_blocks + 1)][3][hi, lo][N][4] TF32 moments (96 N bytes per block)
  int *error_flag;
  uint32_t wait_limit;
  bool packed;           // b_ops already holds this call's moments (launch_near_tc_pack ran)
};

// Bytes of b_ops for states up to K.
size_t near_tc_operand_bytes(int n_blocks, int K);
// Block positions from the leaf-relative source positions.
void launch_near_tc_positions(const float4 *src_rel, const int *blk_src, int n_blocks, float4 *blk_pos,
                              cudaStream_t s);
// Moments (sorted, scaled; paired rows for K >= 4) -> TF32 hi / lo blocks.
void launch_near_tc_pack(const NearTcLaunch &a, const float4 *mom, int K, cudaStream_t s);
// The blocks (unless a.packed), then the near field near[nt][K] =
// (phi, H) / 4 pi of every target.
void launch_near_tc(const NearTcLaunch &a, const float4 *mom, const float4 *tgt_rel, const int *self_idx, int depth,
                    int K, bool want_phi, float4 *near, cudaStream_t s);
bool configure_near_tc(size_t max_smem);

} // namespace cdfmm_b200
