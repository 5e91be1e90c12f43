// cdfmm::UniformFmm -- static-geometry uniform-octree dipole FMM evaluated on
// one B200 through the C ABI of include/cdfmm_b200.h.
//
// Drop-in surface: the constructors, evaluate / evaluate_into /
// evaluate_float32 / evaluate_into_float32, the options record, the enums,
// the identity-map contract and the inspection accessors keep the names,
// argument meaning and exceptions of upstream dip-fmm
// (include/cdfmm/uniform_fmm.hpp:22-442 there).  The one new backend value is
// ExecutionBackend::CudaB200, which is also what Auto resolves to: this
// library evaluates every stage on the GPU and has no CPU executor, so the
// upstream CPU/CUDA backend values raise std::runtime_error ("unavailable in
// this build") exactly as an upstream build without that backend does.
//
// Extensions (no upstream counterpart): K moment states per call
// (evaluate_states_float32), device-resident input/output
// (evaluate_device), and UniformFmmOptions::max_states / b200_m2l / device.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>
#include <optional>
#include <span>
#include <string>
#include <vector>

#include "cdfmm/multi_index.hpp"
#include "cdfmm/output_flags.hpp"
#include "cdfmm/precision.hpp"
#include "cdfmm/timings.hpp"
#include "cdfmm/uniform_tree.hpp"

struct cdfmm_b200_plan;

namespace cdfmm {

enum class ExecutionBackend {
  Auto,
  CpuReference,
  CpuStatic,
  CudaM2LP2P,
  CudaPartial = CudaM2LP2P,
  CudaFull,
  CudaM2L = CudaM2LP2P,
  CudaM2LStaticP2P = CudaM2LP2P,
  CudaB200
};

enum class StaticMatrixBackend { Portable, OneMkl };
enum class StaticOperatorExecutor { Reference, Portable, OneMkl, Cuda };
/// OnTheFly: pair tensors recomputed from positions in every evaluation.
enum class P2PExecutionPacking { Reference, CanonicalAos, ParticleRowSoa, CudaBsr3, OnTheFly };

struct StaticExecutionPlan {
  StaticOperatorExecutor p2m{StaticOperatorExecutor::Cuda};
  StaticOperatorExecutor m2m{StaticOperatorExecutor::Cuda};
  StaticOperatorExecutor m2l{StaticOperatorExecutor::Cuda};
  StaticOperatorExecutor l2l{StaticOperatorExecutor::Cuda};
  StaticOperatorExecutor l2p{StaticOperatorExecutor::Cuda};
  StaticOperatorExecutor p2p{StaticOperatorExecutor::Cuda};
};

/// Physical model of a source (upstream include/cdfmm/cuboid.hpp): point
/// dipoles, or uniformly magnetised axis-aligned cuboids (total moments;
/// side lengths in UniformFmmOptions.source_sizes).
enum class SourceGeometry { PointDipole, UniformCuboid };
struct CuboidSize {
  double hx{0.0};
  double hy{0.0};
  double hz{0.0};
};

/// Arithmetic of the M2L contraction on the B200.
enum class B200M2L { Auto, Float32, SplitBf16 };

bool one_mkl_available() noexcept;
bool cuda_compiled() noexcept;
bool cuda_available() noexcept;
bool cuda_direct_available() noexcept;
bool cuda_m2l_p2p_available() noexcept;
bool cuda_m2l_available() noexcept;
bool cuda_full_available() noexcept;
bool cuda_b200_available() noexcept;
std::string cuda_device_description();

struct UniformFmmOptions {
  StaticPrecision precision{StaticPrecision::Float32};
  int expansion_order{4};
  UniformTreeOptions tree{};
  enum class M2LBackend { Static, Reference } m2l_backend{M2LBackend::Static};
  StaticMatrixBackend static_matrix_backend{StaticMatrixBackend::Portable};
  ExecutionBackend backend{ExecutionBackend::Auto};
  SourceGeometry source_geometry{SourceGeometry::PointDipole};
  std::vector<CuboidSize> source_sizes{};
  bool use_cuboid_p2m{true};
  /// Immutable target -> source identity map in user order (-1 = none).
  std::optional<std::vector<int>> fixed_target_source_indices{};
  /// Kept for source compatibility; the B200 backend stores no pair tensors.
  std::size_t cuda_p2p_bsr_max_bytes{20ULL * 1024ULL * 1024ULL * 1024ULL};
  /// Largest number of moment states passed to one evaluate call.
  int max_states{1};
  B200M2L b200_m2l{B200M2L::Auto};
  int device{0};
};

using M2LBackend = UniformFmmOptions::M2LBackend;

class UniformFmm {
public:
  ~UniformFmm();
  UniformFmm(UniformFmm &&) noexcept;
  UniformFmm &operator=(UniformFmm &&) noexcept;
  UniformFmm(const UniformFmm &) = delete;
  UniformFmm &operator=(const UniformFmm &) = delete;

  /// Source-only geometry: no targets, so evaluate returns no results; the
  /// multipoles of upward_pass are the product (upstream semantics).
  UniformFmm(const std::vector<Vec3> &source_positions, const UniformFmmOptions &options = {});
  UniformFmm(const std::vector<Vec3> &source_positions, const std::vector<Vec3> &target_positions,
             const UniformFmmOptions &options = {});

  /// P2M + M2M on the device for one state (multipoles readable afterwards).
  void upward_pass(std::span<const Vec3> dipole_moments);
  /// M2L + L2L of the last upward pass (locals readable afterwards).
  void downward_pass();

  std::vector<PotentialField> evaluate(std::span<const Vec3> dipole_moments,
                                       OutputFlags output = OutputFlags::Field,
                                       std::span<const int> target_source_indices = {});
  void evaluate_into(std::span<const Vec3> dipole_moments, std::span<PotentialField> results,
                     OutputFlags output = OutputFlags::Field,
                     std::span<const int> target_source_indices = {});
  std::vector<FloatPotentialField> evaluate_float32(std::span<const Vec3> dipole_moments,
                                                    OutputFlags output = OutputFlags::Field,
                                                    std::span<const int> target_source_indices = {});
  void evaluate_into_float32(std::span<const Vec3> dipole_moments,
                             std::span<FloatPotentialField> results,
                             OutputFlags output = OutputFlags::Field,
                             std::span<const int> target_source_indices = {});
  std::vector<PotentialField> evaluate_float64(std::span<const Vec3> dipole_moments,
                                               OutputFlags output = OutputFlags::Field,
                                               std::span<const int> target_source_indices = {});

  /// K states in one call.  moments: [K][n_sources][3] float32 host memory,
  /// user order, physical units.  field: [K][n_targets][3] (may be empty when
  /// only the potential is requested); potential: [K][n_targets] (may be empty
  /// when only the field is requested).
  void evaluate_states_float32(std::span<const float> moments, int n_states,
                               std::span<float> field, std::span<float> potential,
                               OutputFlags output = OutputFlags::Field,
                               std::span<const int> target_source_indices = {});

  /// K states with device-resident arrays (CUDA device pointers) on `stream`
  /// (a cudaStream_t, or nullptr for the plan's stream); returns without
  /// waiting for the GPU.  Layout as evaluate_states_float32.
  void evaluate_device(const float *moments, int n_states, float *field, float *potential,
                       OutputFlags output, void *stream);

  const EvaluationTimings &last_timings() const { return last_timings_; }
  const EvaluationTimings &aggregate_timings() const { return aggregate_timings_; }
  void reset_timings() { aggregate_timings_ = {}; }

  const UniformTree &tree() const { return tree_; }
  const MultiIndexSet &basis() const { return basis_; }
  M2LBackend m2l_backend() const { return M2LBackend::Static; }
  StaticMatrixBackend static_matrix_backend() const { return StaticMatrixBackend::Portable; }
  ExecutionBackend backend() const { return ExecutionBackend::CudaB200; }
  StaticPrecision precision() const noexcept { return StaticPrecision::Float32; }
  StaticExecutionPlan execution_plan() const noexcept { return {}; }
  P2PExecutionPacking p2p_execution_packing() const noexcept { return P2PExecutionPacking::OnTheFly; }
  const CudaPlanStatistics &cuda_plan_statistics() const;
  const StaticPlanStatistics &static_plan_statistics() const { return static_stats_; }
  B200M2L b200_m2l() const noexcept { return m2l_mode_; }
  int max_states() const noexcept { return max_states_; }

  std::span<const double> multipole(int node_index) const;
  std::span<const double> local(int node_index) const;
  std::span<const double> root_multipole() const { return multipole(0); }
  std::span<const float> multipole_float32(int node_index) const;
  std::span<const float> local_float32(int node_index) const;
  std::span<const float> root_multipole_float32() const { return multipole_float32(0); }
  std::span<const double> multipole_float64(int node_index) const;
  std::span<const double> local_float64(int node_index) const;
  std::span<const double> root_multipole_float64() const { return multipole_float64(0); }

  /// The underlying C-ABI plan (borrowed; owned by this object).
  cdfmm_b200_plan *device_plan() const noexcept { return plan_.get(); }

private:
  struct PlanDeleter {
    void operator()(cdfmm_b200_plan *p) const noexcept;
  };
  void construct(const UniformFmmOptions &options);
  void bind_identities(std::span<const int> target_source_indices, std::size_t moment_count);
  void run(const void *moments, int dtype, int n_states, OutputFlags output, int layout,
           float *field, float *potential, unsigned memory, bool synchronize);
  void refresh_expansions(int which) const;

  UniformTree tree_;
  MultiIndexSet basis_;
  B200M2L m2l_mode_{B200M2L::Auto};
  int max_states_{1};
  std::unique_ptr<cdfmm_b200_plan, PlanDeleter> plan_;
  std::optional<std::vector<int>> fixed_identities_{};
  std::vector<int> fixed_sorted_self_{};
  bool identities_bound_{false};
  bool cuboid_sources_{false}; // identity maps do not apply to cuboid sources
  StaticPlanStatistics static_stats_{};
  mutable CudaPlanStatistics cuda_stats_{};
  EvaluationTimings last_timings_{};
  EvaluationTimings aggregate_timings_{};
  bool upward_only_{false};
  mutable std::vector<float> expansion_cache_[2];
  mutable bool expansion_valid_[2]{false, false};
  mutable std::vector<double> widened_{};
};

} // namespace cdfmm
