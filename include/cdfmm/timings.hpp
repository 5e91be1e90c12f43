// Timing and statistics records exposed by UniformFmm.
//
// Field names follow the upstream records (include/cdfmm/timings.hpp:15-223 in
// dip-fmm) so code reading last_timings(), static_plan_statistics() or
// cuda_plan_statistics() keeps compiling.  Fields that describe upstream
// storage this backend does not have (per-pair P2P tensors, BSR blocks,
// oneMKL scratch) stay zero.
#pragma once

#include <cstddef>
#include <cstdint>

namespace cdfmm {

struct PhaseTiming {
  double total_seconds{0.0};
  std::uint64_t calls{0};

  void add(double seconds) {
    total_seconds += seconds;
    ++calls;
  }
};

struct TreeBuildTimings {
  PhaseTiming root_bounds{};
  PhaseTiming node_construction{};
  PhaseTiming topology{};
  PhaseTiming source_morton{};
  PhaseTiming source_sorting{};
  PhaseTiming target_morton{};
  PhaseTiming target_sorting{};
  PhaseTiming ranges{};
  PhaseTiming interaction_lists{};
  PhaseTiming total{};
};

struct EvaluationTimings {
  PhaseTiming moment_permutation{};
  PhaseTiming multipole_reset{};
  PhaseTiming p2m{};
  PhaseTiming m2m{};
  PhaseTiming local_reset{};
  PhaseTiming l2l{};
  PhaseTiming m2l{};
  PhaseTiming m2l_scale{};
  PhaseTiming m2l_gather{};
  PhaseTiming m2l_multiply{};
  PhaseTiming m2l_scatter{};
  PhaseTiming l2p{};
  PhaseTiming p2p{};
  PhaseTiming result_unpermutation{};
  PhaseTiming cuda_h2d{};
  PhaseTiming cuda_kernel{};
  PhaseTiming cuda_d2h{};
  PhaseTiming cuda_m2l_h2d{};
  PhaseTiming cuda_m2l_d2h{};
  PhaseTiming cuda_p2p_h2d{};
  PhaseTiming cuda_p2p_kernel{};
  PhaseTiming cuda_p2p_d2h{};
  PhaseTiming cuda_p2p_wait{};
  PhaseTiming total{};
  std::uint64_t evaluations{0};
};

struct StaticPlanStatistics {
  std::size_t scalar_bytes{sizeof(float)};
  static constexpr std::size_t theoretical_maximum_m2l_classes = 316;
  PhaseTiming p2m_plan{};
  PhaseTiming m2m_plan{};
  PhaseTiming m2l_plan{};
  PhaseTiming l2l_plan{};
  PhaseTiming l2p_plan{};
  PhaseTiming p2p_tensor_plan{};
  PhaseTiming transfer_discovery{};
  PhaseTiming operator_construction{};
  PhaseTiming buffer_allocation{};
  PhaseTiming total{};
  std::size_t transfer_classes{0};
  std::size_t interactions{0};
  std::size_t operator_bytes{0};
  std::size_t interaction_bytes{0};
  std::size_t scratch_bytes{0};
  std::size_t state_bytes{0};
  std::size_t m2m_operators{0};
  std::size_t m2m_theoretical_interactions{0};
  std::size_t m2m_operator_bytes{0};
  std::size_t m2l_operators{0};
  std::size_t m2l_operator_bytes{0};
  std::size_t m2l_interaction_bytes{0};
  std::size_t l2l_operators{0};
  std::size_t l2l_theoretical_interactions{0};
  std::size_t l2l_operator_bytes{0};
  bool dense{true};
  bool sparse{false};
  bool numerically_pruned{false};
  bool symmetry_compressed{false};
  std::size_t p2p_interactions{0};
  std::size_t p2p_value_bytes{0};
  std::size_t p2p_index_bytes{0};
  std::uint64_t construction_count{0};

  std::size_t translation_operator_bytes() const {
    return m2m_operator_bytes + m2l_operator_bytes + l2l_operator_bytes;
  }
  std::size_t total_bytes() const {
    return operator_bytes + interaction_bytes + scratch_bytes + state_bytes;
  }
};

struct CudaPlanStatistics {
  std::size_t scalar_bytes{sizeof(float)};
  std::size_t m2m_unique_matrix_count{0};
  std::size_t m2m_matrix_bytes{0};
  std::size_t m2l_unique_matrix_count{0};
  std::size_t m2l_matrix_bytes{0};
  std::size_t m2l_interaction_metadata_bytes{0};
  std::size_t m2l_interaction_count{0};
  std::size_t m2l_active_row_count{0};
  std::size_t m2l_scratch_bytes{0};
  int m2l_threads_per_block{0};
  std::size_t l2l_unique_matrix_count{0};
  std::size_t l2l_matrix_bytes{0};
  std::size_t p2p_interaction_count{0};
  std::size_t p2p_tensor_bytes{0};
  std::size_t p2p_index_bytes{0};
  std::size_t p2p_row_metadata_bytes{0};
  std::size_t p2p_leaf_metadata_bytes{0};
  std::size_t p2p_identity_bytes{0};
  std::size_t p2p_scratch_bytes{0};
  int p2p_threads_per_block{0};
  std::size_t setup_h2d_bytes{0};
  std::size_t evaluation_h2d_bytes{0};
  std::size_t evaluation_d2h_bytes{0};
  std::uint64_t evaluation_h2d_calls{0};
  std::uint64_t evaluation_d2h_calls{0};
  std::size_t persistent_device_bytes{0};
  std::uint64_t plan_generation_count{0};
  std::uint64_t static_upload_count{0};
  std::uint64_t static_m2l_upload_count{0};
  std::uint64_t static_p2p_upload_count{0};
  std::uint64_t geometry_upload_count{0};
};

} // namespace cdfmm
