// Leaf multipoles (P2M) on the tensor cores: launch interface.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "near_tc.hpp"

namespace cdfmm_b200 {

// Orders with n <= 128 coefficients (p <= 7) and the state range of the
// tensor-core near field, whose packed moment blocks it reads.
bool p2m_tc_supported(int n, int K);
// Leaf multipoles M[leaf][n][K] from the near field's packed moment blocks
// (ntc.b_ops, packed for these K states before this launch) and block
// positions; the same sums as the FP32 P2M (upstream src/far_field.cpp P2M).
void launch_p2m_tc(const NearTcLaunch &ntc, const int8_t *basis, float *M, int n, int p, int K, int depth,
                   cudaStream_t s);
bool configure_p2m_tc(size_t max_smem);

} // namespace cdfmm_b200
