// cdfmm::UniformFmm on the B200 C ABI.
//
// Argument validation, the identity-map contract and the exception types
// follow upstream src/uniform_fmm.cpp (constructor checks :100-123, identity
// policy :265-295 and :1028-1063, size checks :1281-1311).  Evaluation is a
// single cdfmm_b200_evaluate call: the FP64 user moments go to the device
// as they are, where they are divided by scale^3 in FP64 exactly as the
// reference does on the host (:1315-1323), and the FP32 results come back
// already combined and unsorted, directly into the caller's
// FloatPotentialField array.
#include "cdfmm/uniform_fmm.hpp"

#include <algorithm>
#include <chrono>
#include <stdexcept>
#include <string>

#include "cdfmm_b200.h"

namespace cdfmm {

namespace {

using Clock = std::chrono::steady_clock;

[[noreturn]] void throw_status(int status, const char *message) {
  const std::string m = message != nullptr ? message : "unknown error";
  if (status == CDFMM_B200_ERR_INVALID_ARGUMENT) throw std::invalid_argument(m);
  if (status == CDFMM_B200_ERR_LOGIC) throw std::logic_error(m);
  throw std::runtime_error(m);
}

void check_plan(int status, const cdfmm_b200_plan *plan) {
  if (status != CDFMM_B200_OK) throw_status(status, cdfmm_b200_last_error(plan));
}

int device_count() {
  int32_t c = 0;
  cdfmm_b200_device_count(&c);
  return c;
}

const char *backend_name(ExecutionBackend b) {
  switch (b) {
  case ExecutionBackend::CpuReference: return "CpuReference";
  case ExecutionBackend::CpuStatic: return "CpuStatic";
  case ExecutionBackend::CudaM2LP2P: return "CudaM2LP2P";
  case ExecutionBackend::CudaFull: return "CudaFull";
  default: return "backend";
  }
}

} // namespace

bool one_mkl_available() noexcept { return false; }
bool cuda_compiled() noexcept { return true; }
bool cuda_available() noexcept { return device_count() > 0; }
bool cuda_direct_available() noexcept { return device_count() > 0; }
bool cuda_m2l_p2p_available() noexcept { return false; }
bool cuda_m2l_available() noexcept { return false; }
bool cuda_full_available() noexcept { return false; }
bool cuda_b200_available() noexcept {
  if (device_count() == 0) return false;
  int32_t major = 0, minor = 0;
  if (cdfmm_b200_device_info(0, nullptr, 0, &major, &minor) != CDFMM_B200_OK) return false;
  return major == 10;
}
std::string cuda_device_description() {
  if (device_count() == 0) return "no CUDA device";
  char name[256];
  int32_t major = 0, minor = 0;
  if (cdfmm_b200_device_info(0, name, sizeof(name), &major, &minor) != CDFMM_B200_OK) return "no CUDA device";
  return std::string(name) + " (sm_" + std::to_string(major) + std::to_string(minor) + ")";
}

void UniformFmm::PlanDeleter::operator()(cdfmm_b200_plan *p) const noexcept { cdfmm_b200_plan_destroy(p); }

UniformFmm::~UniformFmm() = default;
UniformFmm::UniformFmm(UniformFmm &&) noexcept = default;
UniformFmm &UniformFmm::operator=(UniformFmm &&) noexcept = default;

UniformFmm::UniformFmm(const std::vector<Vec3> &source_positions, const UniformFmmOptions &options)
    : tree_(source_positions, options.tree), basis_(options.expansion_order) {
  construct(options);
}

UniformFmm::UniformFmm(const std::vector<Vec3> &source_positions,
                       const std::vector<Vec3> &target_positions, const UniformFmmOptions &options)
    : tree_(source_positions, target_positions, options.tree), basis_(options.expansion_order) {
  construct(options);
}

void UniformFmm::construct(const UniformFmmOptions &options) {
  const auto t0 = Clock::now();
  if (options.expansion_order < 0) {
    throw std::invalid_argument("UniformFmmOptions.expansion_order must be >= 0");
  }
  if (options.expansion_order > 10) {
    throw std::invalid_argument("UniformFmmOptions.expansion_order must be <= 10 on the B200 backend");
  }
  if (options.backend != ExecutionBackend::Auto && options.backend != ExecutionBackend::CudaB200) {
    throw std::runtime_error(std::string(backend_name(options.backend)) + " is unavailable in this build");
  }
  if (options.precision != StaticPrecision::Float32) {
    throw std::invalid_argument("the B200 backend evaluates FP32 plans; set precision to Float32");
  }
  // Source geometry (upstream src/uniform_fmm.cpp:296-328).
  cuboid_sources_ = options.source_geometry == SourceGeometry::UniformCuboid;
  if (!cuboid_sources_ && !options.source_sizes.empty()) {
    throw std::invalid_argument("point-dipole sources do not accept cuboid sizes");
  }
  if (cuboid_sources_ && options.source_sizes.size() != 1 &&
      options.source_sizes.size() != tree_.sorted_source_positions().size()) {
    throw std::invalid_argument("cuboid sizes must contain one or one per source");
  }
  if (options.max_states < 1) {
    throw std::invalid_argument("UniformFmmOptions.max_states must be >= 1");
  }
  if (tree_.max_level() > 8) {
    throw std::invalid_argument("UniformTreeOptions.max_level must be <= 8 on the B200 backend");
  }
  const std::size_t nt = tree_.sorted_target_positions().size();
  const std::size_t ns = tree_.sorted_source_positions().size();
  if (options.fixed_target_source_indices.has_value()) {
    const std::vector<int> &ids = options.fixed_target_source_indices.value();
    if (ids.size() != nt) {
      throw std::invalid_argument("fixed_target_source_indices must contain one entry per target");
    }
    for (int s : ids) {
      if (s < -1 || s >= static_cast<int>(ns)) {
        throw std::invalid_argument("fixed_target_source_indices contains an invalid source index");
      }
    }
    // finite cuboid self fields are physical: the map is checked, not kept
    if (!cuboid_sources_) fixed_identities_ = ids;
  }
  m2l_mode_ = options.b200_m2l;
  max_states_ = options.max_states;

  const auto src_off = tree_.leaf_source_offsets();
  const auto tgt_off = tree_.leaf_target_offsets();
  std::vector<double> spos(3 * ns), tpos(3 * nt);
  for (std::size_t i = 0; i < ns; ++i) {
    const Vec3 &p = tree_.sorted_source_positions()[i];
    spos[3 * i] = p.x;
    spos[3 * i + 1] = p.y;
    spos[3 * i + 2] = p.z;
  }
  for (std::size_t i = 0; i < nt; ++i) {
    const Vec3 &p = tree_.sorted_target_positions()[i];
    tpos[3 * i] = p.x;
    tpos[3 * i + 1] = p.y;
    tpos[3 * i + 2] = p.z;
  }
  cdfmm_b200_plan_desc d{};
  d.struct_size = sizeof(d);
  d.n_sources = static_cast<int32_t>(ns);
  d.n_targets = static_cast<int32_t>(nt);
  d.order = options.expansion_order;
  d.depth = tree_.max_level();
  d.max_states = options.max_states;
  d.m2l_mode = options.b200_m2l == B200M2L::Float32   ? CDFMM_B200_M2L_FP32
               : options.b200_m2l == B200M2L::SplitBf16 ? CDFMM_B200_M2L_BF16X3
                                                      : CDFMM_B200_M2L_AUTO;
  d.device = options.device;
  d.root_centre[0] = tree_.root_centre().x;
  d.root_centre[1] = tree_.root_centre().y;
  d.root_centre[2] = tree_.root_centre().z;
  d.root_half_width = tree_.root_half_width();
  d.sorted_source_positions = spos.data();
  d.sorted_target_positions = tpos.data();
  d.source_permutation = tree_.source_permutation().data();
  d.target_permutation = tree_.target_permutation().data();
  d.leaf_source_offsets = src_off.data();
  d.leaf_target_offsets = tgt_off.data();
  cdfmm_b200_plan *raw = nullptr;
  const int status = cdfmm_b200_plan_create(&d, &raw);
  if (status != CDFMM_B200_OK) throw_status(status, cdfmm_b200_last_error(nullptr));
  plan_.reset(raw);
  if (cuboid_sources_) {
    std::vector<double> sizes;
    sizes.reserve(3 * options.source_sizes.size());
    for (const CuboidSize &h : options.source_sizes) {
      sizes.push_back(h.hx);
      sizes.push_back(h.hy);
      sizes.push_back(h.hz);
    }
    check_plan(cdfmm_b200_set_source_cuboids(plan_.get(), sizes.data(), static_cast<int32_t>(options.source_sizes.size()),
                                             options.use_cuboid_p2m ? 1 : 0),
               plan_.get());
  }

  if (fixed_identities_.has_value()) {
    bind_identities(fixed_identities_.value(), ns);
  }

  cdfmm_b200_stats st{};
  cdfmm_b200_get_stats(plan_.get(), &st);
  static_stats_ = {};
  static_stats_.scalar_bytes = sizeof(float);
  static_stats_.transfer_classes = st.m2l_classes;
  static_stats_.interactions = st.m2l_interactions;
  static_stats_.m2l_operators = st.m2l_classes;
  static_stats_.m2l_operator_bytes = st.m2l_matrix_bytes;
  static_stats_.operator_bytes = st.m2l_matrix_bytes;
  static_stats_.m2m_operators = 8 * static_cast<std::size_t>(tree_.max_level());
  static_stats_.l2l_operators = static_stats_.m2m_operators;
  static_stats_.m2m_theoretical_interactions = tree_.nodes().empty() ? 0 : tree_.nodes().size() - 1;
  static_stats_.l2l_theoretical_interactions = static_stats_.m2m_theoretical_interactions;
  static_stats_.p2p_interactions = st.p2p_pairs;
  static_stats_.state_bytes = st.persistent_device_bytes;
  static_stats_.total.add(std::chrono::duration<double>(Clock::now() - t0).count());
  static_stats_.construction_count = 1;
}

// Resolves the identity map like the reference (src/uniform_fmm.cpp:1045-1063,
// :1290-1305) and uploads its sorted form when it differs from the bound one
// (src/uniform_fmm.cpp:1028-1043 builds the same sorted map).
void UniformFmm::bind_identities(std::span<const int> ids, std::size_t moment_count) {
  // cuboid sources: identities are not applied (upstream resolve_self_indices)
  if (cuboid_sources_) {
    identities_bound_ = true;
    return;
  }
  const std::size_t nt = tree_.sorted_target_positions().size();
  if (fixed_identities_.has_value()) {
    const std::vector<int> &fixed = fixed_identities_.value();
    if (ids.empty()) {
      ids = fixed;
    } else if (!std::equal(ids.begin(), ids.end(), fixed.begin(), fixed.end())) {
      throw std::invalid_argument("fixed target-to-source identity map changed; rebuild the FMM plan");
    }
  }
  if (!ids.empty() && ids.size() != nt) {
    throw std::invalid_argument("UniformFmm::evaluate identity map has incorrect length");
  }
  for (int s : ids) {
    if (s < -1 || s >= static_cast<int>(moment_count)) {
      throw std::invalid_argument("UniformFmm::evaluate identity map contains an invalid index");
    }
  }
  std::vector<int> sorted(nt, -1);
  const auto tperm = tree_.target_permutation();
  const auto sinv = tree_.source_inverse_permutation();
  if (!ids.empty()) {
    for (std::size_t t = 0; t < nt; ++t) {
      const int s = ids[static_cast<std::size_t>(tperm[t])];
      if (s >= 0) sorted[t] = sinv[static_cast<std::size_t>(s)];
    }
  }
  if (identities_bound_ && sorted == fixed_sorted_self_) return;
  check_plan(cdfmm_b200_set_self_indices(plan_.get(), sorted.data()), plan_.get());
  fixed_sorted_self_ = std::move(sorted);
  identities_bound_ = true;
}

void UniformFmm::run(const void *moments, int dtype, int n_states, OutputFlags output, int layout,
                     float *field, float *potential, unsigned memory, bool synchronize) {
  const auto t0 = Clock::now();
  cdfmm_b200_eval_args a{};
  a.moments = moments;
  a.moments_dtype = dtype;
  a.n_states = n_states;
  a.output = static_cast<unsigned>(output);
  a.layout = layout;
  a.field = field;
  a.potential = potential;
  a.memory = memory;
  a.stream = nullptr;
  a.synchronize = synchronize ? 1 : 0;
  check_plan(cdfmm_b200_evaluate(plan_.get(), &a), plan_.get());
  expansion_valid_[0] = expansion_valid_[1] = false;
  last_timings_ = {};
  cdfmm_b200_stats st{};
  cdfmm_b200_get_stats(plan_.get(), &st);
  if (st.timing_enabled) {
    last_timings_.moment_permutation.add(st.ms_gather * 1e-3);
    last_timings_.p2m.add(st.ms_p2m * 1e-3);
    last_timings_.m2m.add(st.ms_m2m * 1e-3);
    last_timings_.m2l.add(st.ms_m2l * 1e-3);
    last_timings_.l2l.add(st.ms_l2l * 1e-3);
    last_timings_.l2p.add(st.ms_l2p * 1e-3);
    last_timings_.p2p.add(st.ms_p2p * 1e-3);
    last_timings_.cuda_p2p_kernel.add(st.ms_p2p * 1e-3);
    last_timings_.cuda_kernel.add(st.ms_total * 1e-3);
  }
  last_timings_.total.add(std::chrono::duration<double>(Clock::now() - t0).count());
  last_timings_.evaluations = static_cast<std::uint64_t>(n_states);
  auto acc = [](PhaseTiming &a2, const PhaseTiming &b) {
    a2.total_seconds += b.total_seconds;
    a2.calls += b.calls;
  };
  acc(aggregate_timings_.moment_permutation, last_timings_.moment_permutation);
  acc(aggregate_timings_.p2m, last_timings_.p2m);
  acc(aggregate_timings_.m2m, last_timings_.m2m);
  acc(aggregate_timings_.m2l, last_timings_.m2l);
  acc(aggregate_timings_.l2l, last_timings_.l2l);
  acc(aggregate_timings_.l2p, last_timings_.l2p);
  acc(aggregate_timings_.p2p, last_timings_.p2p);
  acc(aggregate_timings_.cuda_kernel, last_timings_.cuda_kernel);
  acc(aggregate_timings_.total, last_timings_.total);
  aggregate_timings_.evaluations += last_timings_.evaluations;
}

void UniformFmm::upward_pass(std::span<const Vec3> dipole_moments) {
  if (dipole_moments.size() != tree_.sorted_source_positions().size()) {
    throw std::invalid_argument("UniformFmm::upward_pass requires one dipole moment per source position");
  }
  // One device evaluation produces every expansion; the multipoles of this
  // state are then readable through multipole()/multipole_float32().
  std::vector<FloatPotentialField> scratch(tree_.sorted_target_positions().size());
  bind_identities({}, dipole_moments.size());
  run(dipole_moments.data(), 1, 1, OutputFlags::Field, CDFMM_B200_LAYOUT_INTERLEAVED,
      reinterpret_cast<float *>(scratch.data()), nullptr, CDFMM_B200_MOMENTS_ON_HOST | CDFMM_B200_RESULTS_ON_HOST,
      true);
  upward_only_ = true;
}

void UniformFmm::downward_pass() {
  // Locals were produced by the same device evaluation as the multipoles.
  upward_only_ = false;
}

std::vector<PotentialField> UniformFmm::evaluate(std::span<const Vec3> dipole_moments, OutputFlags output,
                                                 std::span<const int> ids) {
  std::vector<PotentialField> results(tree_.sorted_target_positions().size());
  evaluate_into(dipole_moments, results, output, ids);
  return results;
}

void UniformFmm::evaluate_into(std::span<const Vec3> dipole_moments, std::span<PotentialField> results,
                               OutputFlags output, std::span<const int> ids) {
  std::vector<FloatPotentialField> f(results.size());
  evaluate_into_float32(dipole_moments, f, output, ids);
  for (std::size_t i = 0; i < results.size(); ++i) {
    results[i].phi = static_cast<double>(f[i].phi);
    results[i].H = {static_cast<double>(f[i].H.x), static_cast<double>(f[i].H.y), static_cast<double>(f[i].H.z)};
  }
}

std::vector<FloatPotentialField> UniformFmm::evaluate_float32(std::span<const Vec3> dipole_moments,
                                                              OutputFlags output, std::span<const int> ids) {
  std::vector<FloatPotentialField> results(tree_.sorted_target_positions().size());
  evaluate_into_float32(dipole_moments, results, output, ids);
  return results;
}

void UniformFmm::evaluate_into_float32(std::span<const Vec3> dipole_moments,
                                       std::span<FloatPotentialField> results, OutputFlags output,
                                       std::span<const int> ids) {
  const std::size_t nt = tree_.sorted_target_positions().size();
  if (results.size() != nt) {
    throw std::invalid_argument("UniformFmm::evaluate_into_float32 requires one result per target");
  }
  if (dipole_moments.size() != tree_.sorted_source_positions().size()) {
    throw std::invalid_argument("UniformFmm::upward_pass requires one dipole moment per source position");
  }
  bind_identities(ids, dipole_moments.size());
  if (output == OutputFlags::None || nt == 0) {
    std::fill(results.begin(), results.end(), FloatPotentialField{});
    if (nt == 0 && !dipole_moments.empty() && output != OutputFlags::None) {
      std::vector<FloatPotentialField> none(1);
      run(dipole_moments.data(), 1, 1, output, CDFMM_B200_LAYOUT_INTERLEAVED,
          reinterpret_cast<float *>(none.data()), nullptr,
          CDFMM_B200_MOMENTS_ON_HOST | CDFMM_B200_RESULTS_ON_HOST, true);
    }
    return;
  }
  run(dipole_moments.data(), 1, 1, output, CDFMM_B200_LAYOUT_INTERLEAVED,
      reinterpret_cast<float *>(results.data()), nullptr, CDFMM_B200_MOMENTS_ON_HOST | CDFMM_B200_RESULTS_ON_HOST,
      true);
}

std::vector<PotentialField> UniformFmm::evaluate_float64(std::span<const Vec3>, OutputFlags, std::span<const int>) {
  throw std::logic_error("evaluate_float64 requires an FP64 FMM plan");
}

void UniformFmm::evaluate_states_float32(std::span<const float> moments, int n_states, std::span<float> field,
                                         std::span<float> potential, OutputFlags output,
                                         std::span<const int> ids) {
  const std::size_t ns = tree_.sorted_source_positions().size();
  const std::size_t nt = tree_.sorted_target_positions().size();
  if (n_states < 1 || n_states > max_states_) {
    throw std::invalid_argument("n_states must be in [1, max_states]");
  }
  if (moments.size() != static_cast<std::size_t>(n_states) * ns * 3) {
    throw std::invalid_argument("moments must hold n_states * n_sources * 3 values");
  }
  const bool want_h = has_flag(output, OutputFlags::Field);
  const bool want_phi = has_flag(output, OutputFlags::Potential);
  if (want_h && field.size() != static_cast<std::size_t>(n_states) * nt * 3) {
    throw std::invalid_argument("field must hold n_states * n_targets * 3 values");
  }
  if (want_phi && potential.size() != static_cast<std::size_t>(n_states) * nt) {
    throw std::invalid_argument("potential must hold n_states * n_targets values");
  }
  bind_identities(ids, ns);
  if (output == OutputFlags::None || nt == 0) return;
  run(moments.data(), 0, n_states, output, CDFMM_B200_LAYOUT_SEPARATE, want_h ? field.data() : nullptr,
      want_phi ? potential.data() : nullptr, CDFMM_B200_MOMENTS_ON_HOST | CDFMM_B200_RESULTS_ON_HOST, true);
}

void UniformFmm::evaluate_device(const float *moments, int n_states, float *field, float *potential,
                                 OutputFlags output, void *stream) {
  if (n_states < 1 || n_states > max_states_) {
    throw std::invalid_argument("n_states must be in [1, max_states]");
  }
  if (!identities_bound_) bind_identities({}, tree_.sorted_source_positions().size());
  if (output == OutputFlags::None || tree_.sorted_target_positions().empty()) return;
  cdfmm_b200_eval_args a{};
  a.moments = moments;
  a.moments_dtype = 0;
  a.n_states = n_states;
  a.output = static_cast<unsigned>(output);
  a.layout = CDFMM_B200_LAYOUT_SEPARATE;
  a.field = field;
  a.potential = potential;
  a.memory = 0;
  a.stream = stream;
  a.synchronize = 0;
  check_plan(cdfmm_b200_evaluate(plan_.get(), &a), plan_.get());
  expansion_valid_[0] = expansion_valid_[1] = false;
}

const CudaPlanStatistics &UniformFmm::cuda_plan_statistics() const {
  cdfmm_b200_stats st{};
  cdfmm_b200_get_stats(plan_.get(), &st);
  cuda_stats_ = {};
  cuda_stats_.scalar_bytes = sizeof(float);
  cuda_stats_.m2l_unique_matrix_count = st.m2l_classes;
  cuda_stats_.m2l_matrix_bytes = st.m2l_matrix_bytes;
  cuda_stats_.m2l_interaction_count = st.m2l_interactions;
  cuda_stats_.m2m_unique_matrix_count = 8 * static_cast<std::size_t>(tree_.max_level());
  cuda_stats_.l2l_unique_matrix_count = cuda_stats_.m2m_unique_matrix_count;
  cuda_stats_.p2p_interaction_count = st.p2p_pairs;
  cuda_stats_.setup_h2d_bytes = st.setup_h2d_bytes;
  cuda_stats_.evaluation_h2d_bytes = st.evaluation_h2d_bytes;
  cuda_stats_.evaluation_d2h_bytes = st.evaluation_d2h_bytes;
  cuda_stats_.evaluation_h2d_calls = st.evaluation_h2d_calls;
  cuda_stats_.evaluation_d2h_calls = st.evaluation_d2h_calls;
  cuda_stats_.persistent_device_bytes = st.persistent_device_bytes;
  cuda_stats_.plan_generation_count = 1;
  cuda_stats_.static_upload_count = 1;
  cuda_stats_.geometry_upload_count = 1;
  return cuda_stats_;
}

void UniformFmm::refresh_expansions(int which) const {
  if (expansion_valid_[which]) return;
  const std::size_t count = tree_.nodes().size() * static_cast<std::size_t>(basis_.size());
  std::vector<float> &dst = expansion_cache_[which];
  dst.assign(count, 0.0F);
  cdfmm_b200_stats st{};
  cdfmm_b200_get_stats(plan_.get(), &st);
  if (st.evaluations > 0 && count > 0) {
    check_plan(cdfmm_b200_read_expansions(plan_.get(), which, 0, dst.data(), dst.size()), plan_.get());
  }
  if (which == 1 && upward_only_) std::fill(dst.begin(), dst.end(), 0.0F);
  // The reference never forms locals of boxes without targets (nor
  // multipoles of boxes without sources): they read as zero there.
  const std::size_t n = static_cast<std::size_t>(basis_.size());
  for (const TreeNode &node : tree_.nodes()) {
    const bool empty = which == 0 ? node.source_count() == 0 : node.target_count() == 0;
    if (empty) std::fill_n(dst.begin() + static_cast<std::ptrdiff_t>(node.index * n), n, 0.0F);
  }
  expansion_valid_[which] = true;
}

std::span<const float> UniformFmm::multipole_float32(int node_index) const {
  if (node_index < 0 || node_index >= static_cast<int>(tree_.nodes().size())) {
    throw std::out_of_range("node index out of range");
  }
  refresh_expansions(0);
  const std::size_t n = static_cast<std::size_t>(basis_.size());
  return std::span<const float>(expansion_cache_[0]).subspan(static_cast<std::size_t>(node_index) * n, n);
}

std::span<const float> UniformFmm::local_float32(int node_index) const {
  if (node_index < 0 || node_index >= static_cast<int>(tree_.nodes().size())) {
    throw std::out_of_range("node index out of range");
  }
  refresh_expansions(1);
  const std::size_t n = static_cast<std::size_t>(basis_.size());
  return std::span<const float>(expansion_cache_[1]).subspan(static_cast<std::size_t>(node_index) * n, n);
}

std::span<const double> UniformFmm::multipole(int node_index) const {
  const auto f = multipole_float32(node_index);
  widened_.assign(f.begin(), f.end());
  return widened_;
}

std::span<const double> UniformFmm::local(int node_index) const {
  const auto f = local_float32(node_index);
  widened_.assign(f.begin(), f.end());
  return widened_;
}

std::span<const double> UniformFmm::multipole_float64(int) const {
  throw std::logic_error("multipole_float64 requires an FP64 FMM plan");
}

std::span<const double> UniformFmm::local_float64(int) const {
  throw std::logic_error("local_float64 requires an FP64 FMM plan");
}

} // namespace cdfmm
