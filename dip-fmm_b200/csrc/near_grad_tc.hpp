// Position gradient of the list-1 near field on the tensor cores: launch
// interface (kind::tf32, three products of TF32 hi / lo splits).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "near_tc.hpp"

namespace cdfmm_b200 {

constexpr int kNearGradSources = 16; // sources per block (one pipeline chunk)

// Per plan: sources grouped per leaf into blocks of 16 (the last block of a
// leaf padded with empty slots); block n_blocks is the all-empty block.
struct NearGradLayout {
  std::vector<int> blk_off; // [leaves + 1]
  std::vector<int> blk_src; // [(n_blocks + 1) * 16] sorted source index, -1: empty
  int n_blocks = 0;
};
NearGradLayout near_grad_layout(const int *src_off, int depth);

struct NearGradLaunch {
  const float4 *blk_pos; // [(n_blocks + 1) * 16] leaf-relative positions, .w: sorted index (-1: empty)
  const int *blk_off;
  const int *blk_src;
  int n_blocks;
  const int4 *work;      // the forward tensor-core near field's units (<= 32 targets)
  int n_work;
  void *b_ops;           // near_grad_operand_bytes
  int *error_flag;
  uint32_t wait_limit;
};

size_t near_grad_operand_bytes(int n_blocks, int K);
void launch_near_grad_positions(const float4 *src_rel, const int *blk_src, int n_blocks, float4 *blk_pos,
                                cudaStream_t s);
// Moments (sorted, scaled, paired rows) and weights W[nt][K] -> the near
// field's position gradient of sum_k w_k . H_k per target, written as
// gpart[nt][G] (group 0 the whole sum, the other groups zero).
void launch_near_grad_tc(const NearGradLaunch &a, const float4 *mom, const float4 *tgt_rel, const int *self_idx,
                         int depth, int K, const float4 *W, float4 *gpart, int G, cudaStream_t s);
bool configure_near_grad_tc(size_t max_smem);

} // namespace cdfmm_b200
