// Internal declarations of the B200 evaluator (not part of the public ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
#include <memory>
#include <vector>

#include "cdfmm_b200.h"

namespace cdfmm_b200 {

constexpr int kMaxOrder = 10;
constexpr int kMaxDepth = 8;
constexpr int kMaxCoef = (kMaxOrder + 1) * (kMaxOrder + 2) * (kMaxOrder + 3) / 6; // 286
// Pairs closer than a leaf width / 2^kCloseShift (or a smaller threshold in
// dense clusters) have their near field corrected with r from the FP64
// positions: FP32 coordinates relative to a leaf centre carry an absolute
// error of about 2^-25 leaf widths, which for such pairs is no longer small
// against their distance.
constexpr int kCloseShift = 4;

inline int basis_size(int p) { return p < 0 ? 0 : (p + 1) * (p + 2) * (p + 3) / 6; }
inline int level_offset(int level) {
  long long p = 1;
  for (int i = 0; i < level; ++i) p *= 8;
  return static_cast<int>((p - 1) / 7);
}
inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// Host tables of the expansion basis and of every geometry-dependent operator.
// All values are computed in FP64 (long double for the derivative recurrence)
// and rounded once to FP32, as the reference FP32 plan rounds its FP64 operator
// entries once (src/uniform_fmm.cpp:719-824 upstream).
struct HostOperators {
  int p = 0;
  int n = 0;       // coefficients per expansion
  int depth = 0;
  std::vector<int> ax, ay, az; // basis multi-indices in basis order

  // M2M / L2L: for output coefficient a, pairs [off[a], off[a+1]) of
  // (monomial index g, input coefficient index).  Coefficient value for
  // (level, child class, g) is coef[(level * 8 + class) * n + g].
  std::vector<int> m2m_off, l2l_off;
  std::vector<int> m2m_pair_g, m2m_pair_in, l2l_pair_g, l2l_pair_in;
  std::vector<float> m2m_coef, l2l_coef; // [(depth+1) * 8][n]

  // Normalised M2L matrices T^(t)[beta][alpha] = D^{alpha+beta} G(t) for the
  // 7x7x7 integer translation stencil (slot = (tx+3)*49 + (ty+3)*7 + (tz+3));
  // slots inside the 3x3x3 near stencil are zero and never used.
  // Stored FP32 as [slot][alpha][beta_pad] with beta_pad = m2l_ld.  Both
  // tables depend on the order alone and are shared by every plan of that
  // order (see m2l_matrices); null for depth < 2 (no M2L).
  int m2l_ld = 0;
  std::shared_ptr<const std::vector<float>> m2l_T;
  // The same matrices in FP64, [slot][alpha][beta] with leading dimension n
  // (input of the BF16 hi/lo split of the tensor-core path).
  std::shared_ptr<const std::vector<double>> m2l_T64;
};

HostOperators build_host_operators(int p, int depth, int m2l_ld_multiple);

// Where m2l_matrices found the tables of an order.
enum class OperatorSource { Computed = 0, Process = 1, Disk = 2 };

// The normalised FP64 M2L matrices of order p ([343][n][n], near-stencil
// slots zero).  Computed once per process and order; when the environment
// variable CDFMM_B200_OPERATOR_CACHE names a directory they are also kept
// there, one file per order, and read back by later processes (a file whose
// header, size or checksum does not match is ignored and rewritten).
std::shared_ptr<const std::vector<double>> m2l_matrices(int p, OperatorSource *source = nullptr);
// Their FP32 copy with rows padded to ld (zero padding), also shared.
std::shared_ptr<const std::vector<float>> m2l_matrices_fp32(int p, int ld,
                                                            const std::shared_ptr<const std::vector<double>> &T64);

// D^gamma G(R) for G = 1/(4 pi |R|) and every gamma of total degree <= order,
// in basis order (FP64).  Cartesian recurrence for the Taylor coefficients
// of 1/|R|:  |g| r^2 a_g + (2|g|-1) sum_i R_i a_{g-e_i} + (|g|-1) sum_i a_{g-2e_i} = 0.
std::vector<double> laplace_derivatives(int order, const double R[3]);

struct Plan;

} // namespace cdfmm_b200

// Records `msg` as the last error of `plan` (may be NULL) and of this thread,
// as reported by cdfmm_b200_last_error.
void cdfmm_b200_record_error(cdfmm_b200_plan *plan, const std::string &msg);

// Enqueues on `s` the move of the plan's device error flag into its host
// status record, tagged with call number `call` (the last work of a call).
cudaError_t cdfmm_b200_collect_status(cdfmm_b200_plan *plan, cudaStream_t s, unsigned long long call);
// After the stream of call number `call` was synchronised: an empty string if
// that call's work recorded no expired wait, else the error message (and the
// record counts as reported).  Failures of earlier calls are left for
// cdfmm_b200_poll_status.
std::string cdfmm_b200_own_status(cdfmm_b200_plan *plan, unsigned long long call);

// Near-field geometry of a plan as launch_p2p takes it: the close pairs and,
// for cuboid sources, the pair tensors.
namespace cdfmm_b200 {
struct CloseGeometry;
}
cdfmm_b200::CloseGeometry cdfmm_b200_near_geometry(const cdfmm_b200_plan *plan);

// Batch building blocks: a one-state evaluation (device arrays, already
// validated by a plain evaluate of the same arguments) split around its M2L,
// which the batch runs for several plans of one depth and order at once
// (their multipoles stacked as the states of one tensor-core M2L).  upward:
// gather, the near field (forked onto the plan's near stream), P2M, M2M on s;
// downward: L2L, the join with the near field, L2P, the status record, on s.
namespace cdfmm_b200 {
// Tensor-core M2L work tiles (per level, deepest first: runs of T parents, the
// 8 parity classes of a run adjacent) and the TMEM columns of m_tiles
// accumulators acc_stride apart.
std::vector<int4> tc_work_tiles(int depth, int T);
uint32_t tc_tmem_columns(int m_tiles, int acc_stride);
} // namespace cdfmm_b200

extern "C" {
void cdfmm_b200_stacked_upward(cdfmm_b200_plan *plan, const cdfmm_b200_eval_args *a, cudaStream_t s);
void cdfmm_b200_stacked_downward(cdfmm_b200_plan *plan, const cdfmm_b200_eval_args *a, cudaStream_t s);
}

// The opaque ABI handle.
struct cdfmm_b200_plan {
  int device = 0;
  int ns = 0, nt = 0, p = 0, n = 0, depth = 0, n_leaves = 0, n_nodes = 0;
  int max_states = 1;
  int m2l_mode = CDFMM_B200_M2L_FP32;
  double root_centre[3] = {0, 0, 0};
  double root_half_width = 1.0;
  double scale = 2.0;         // root width: FP32 coordinates are (x - c) / scale
  float inv_scale3 = 1.0F;    // moments are multiplied by 1 / scale^3
  float phi_scale = 1.0F;     // potential is multiplied by scale
  bool has_self = false;
  bool timing = false;
  std::string last_error;

  cdfmm_b200::HostOperators ops;

  cudaStream_t stream = nullptr;   // far-field / main stream
  cudaStream_t near_stream = nullptr;
  cudaStream_t far_stream = nullptr;                // far field, high priority (overlaps the near field)
  cudaEvent_t ev_far = nullptr;
  cudaStream_t io_in = nullptr, io_out = nullptr;  // host-memory copies overlapping the evaluation
  std::vector<cudaEvent_t> io_events;               // chunk pipeline events
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_t[20] = {};
  bool trace = false;                               // concurrent trace events (timing mode 2)
  int schedule = CDFMM_B200_SCHEDULE_AUTO;          // near/far schedule of K > 1 evaluations
  int last_schedule = CDFMM_B200_SCHEDULE_SEPARATE;

  // geometry (device)
  float4 *src_rel = nullptr;   // [ns] (x - leaf centre) normalised, .w unused
  float4 *tgt_rel = nullptr;   // [nt]
  // close pairs (closer than a leaf width / 2^close_shift; see CloseGeometry)
  int4 *close_targets = nullptr;  // [n_close_targets] (sorted target, first pair, pairs, 0)
  int n_close_targets = 0;
  float4 *close_r_fp32 = nullptr; // [pairs] r as the near-field kernels form it, .w = source index
  float4 *close_r_exact = nullptr; // [pairs] r from the FP64 positions
  uint64_t close_pairs = 0;
  int close_shift = 0;
  int *src_off = nullptr;      // [n_leaves + 1]
  int *tgt_off = nullptr;      // [n_leaves + 1]
  int *src_perm = nullptr;     // [ns] sorted -> user
  int *tgt_perm = nullptr;     // [nt]
  int *src_inv = nullptr;      // [ns] user -> sorted
  int *tgt_inv = nullptr;      // [nt]
  int *self_idx = nullptr;     // [nt] sorted target -> sorted source, -1 none
  int2 *leaf_self = nullptr;   // [n_leaves] lowest, highest self source of each leaf's targets ((INT_MAX, -1): none)
  int4 *p2p_work = nullptr;    // [n_p2p_work] list1 work units (leaf, first target, targets, 0)
  int n_p2p_work = 0;
  int *p2p_next_unit = nullptr; // work-unit counter of the persistent co-resident near field
  int sm_count = 0;
  // Units of up to 128 targets without the per-unit cost cap (the same array
  // as p2p_work when no unit was capped): used while the plan is captured
  // into a batch graph, where the other geometries' work runs beside a long
  // unit and the cap's extra staging only costs time.
  int4 *p2p_work_wide = nullptr;
  int n_p2p_work_wide = 0;
  bool in_batch = false;
  // tensor-core near field (states 8..128): sources in blocks of 4 per leaf,
  // work units of <= 32 targets, TF32 hi / lo moment operands; built on
  // first use
  int near_mode = CDFMM_B200_NEAR_AUTO;
  bool ntc_supported = false;
  bool ntc_built = false;
  int *ntc_blk_off = nullptr;
  int *ntc_blk_src = nullptr;
  float4 *ntc_blk_pos = nullptr;
  int4 *ntc_work = nullptr;
  int ntc_n_blocks = 0, ntc_n_work = 0;
  void *ntc_b = nullptr;
  // tensor-core position gradient of the near field: blocks of 16 sources
  bool ngt_supported = false;
  bool ngt_built = false;
  int *ngt_blk_off = nullptr;
  int *ngt_blk_src = nullptr;
  float4 *ngt_blk_pos = nullptr;
  int ngt_n_blocks = 0;
  void *ngt_b = nullptr;

  // operators (device)
  int *m2m_off = nullptr, *m2m_pair = nullptr; // pair = g | (in << 16)
  int *l2l_off = nullptr, *l2l_pair = nullptr;
  float *m2m_coef = nullptr, *l2l_coef = nullptr;
  float *m2l_T = nullptr;            // traceless FP32 sub-blocks [343][tc_n_in][m2l_ld_red] (SIMT M2L)
  int m2l_ld_red = 0;
  float *m2l_fold_buf = nullptr;     // [levels 2..depth boxes][tc_n_in][max_states] folded moments (SIMT M2L)
  float *scale_m = nullptr;    // [depth+1][n] 2^(level*|alpha|)   (exact)
  float *scale_l = nullptr;    // [depth+1][n] 2^(level*(|beta|+1)) (exact)
  int4 *m2l_tiles = nullptr;   // SIMT M2L work tiles (level, class, packed parent origin)
  int n_tiles = 0;
  int8_t *basis = nullptr;     // [n][4] ax, ay, az, degree
  int p2m_chunk = 64;
  int last_K = 0;              // states whose expansions M, L hold (from state exp_state0)
  int exp_state0 = 0;

  // tensor-core M2L (split BF16): availability, shapes, buffers, tiles
  bool tc_supported = false;
  int tc_Kpad = 0, tc_Npad = 0, tc_stages = 0, tc_Kp_max = 0;
  int tc_m_tiles = 1, tc_acc_stride = 0; // accumulators per CTA, TMEM columns apart
  int tc_fuse = 0;                        // 1: A_hi x [B_hi | B_lo] as one N = 2 Npad MMA
  bool tc_pinned = false;                 // shape set by cdfmm_b200_set_m2l_shape: no autotuning
  size_t tc_tuned_budget = 0;             // shared-memory budget the current shape was chosen for
  struct TcShape {
    int m_tiles, stages, fuse;
  };
  std::vector<TcShape> tc_candidates;     // pipeline shapes the autotuner tries
  uint32_t tc_tmem_cols = 0;
  void *tc_a_hi = nullptr, *tc_a_lo = nullptr; // [boxes + 1][Kp_max * Kpad] BF16
  void *tc_b = nullptr;                        // [343][Kpad/32][2][Npad * 32] BF16 (reduced operator)
  bool p2m_tc_ok = false;                      // tensor-core P2M configured (beside the tensor-core near field)
  int *tc_fold_off = nullptr, *tc_fold = nullptr, *tc_expand = nullptr; // traceless reduction tables
  int tc_n_in = 0, tc_n_out = 0, tc_n_derived = 0;
  int4 *tc_tiles = nullptr;
  size_t tc_tiles_capacity = 0;
  int tc_tiles_Kp = 0, tc_n_tiles = 0;
  int *error_flag = nullptr;                   // device: nonzero after an expired bounded wait
  bool last_m2l_tc = false;
  uint32_t tc_wait_limit = 0;                  // iterations of each M2L pipeline progress wait

  // Expired bounded waits, as seen by the host: every call ends with a
  // one-thread kernel on its stream that moves a nonzero device error flag
  // into this record (pinned host memory mapped into the device address
  // space) and clears the flag, so a failure is attributed to the call whose
  // work raised it even when that call did not wait for its results.
  struct StatusRecord {
    int code;                  // error code of the last expired wait
    int count;                 // calls whose GPU work recorded an expired wait
    unsigned long long call;   // call number (call_seq) of the last such call
  };
  StatusRecord *status = nullptr;              // host address
  StatusRecord *status_dev = nullptr;          // device address of the same record
  int status_seen = 0;                         // `count` already reported to the caller
  unsigned long long call_seq = 0;             // evaluate / backward / noalloc calls so far

  // state (device), sized for max_states
  float4 *mom = nullptr;       // [ns][K] sorted scaled moments
  float *M = nullptr;          // [n_nodes][n][K]
  float *L = nullptr;          // [n_nodes][n][K]
  float4 *near = nullptr;      // [nt][K] (phi, Hx, Hy, Hz) near field
  void *stage_in = nullptr;    // device copy of host moments
  size_t stage_in_bytes = 0;
  void *stage_out = nullptr;   // device results before D2H
  size_t stage_out_bytes = 0;

  // Uniformly magnetised cuboid sources (cdfmm_b200_set_source_cuboids):
  // root-normalised side lengths (FP32 for the P2M, FP64 for the pair
  // tensors; one entry for all sources when size_step is 0, else one per
  // sorted source), whether the P2M averages over them, and the near-field
  // pair tensors of the work units p2p_work (see CuboidNear).
  bool cuboid = false;
  bool cuboid_p2m = false;
  int size_step = 0;
  float4 *src_size = nullptr;
  double *src_size64 = nullptr;
  float *cuboid_T = nullptr;
  long long *cuboid_base = nullptr;
  uint64_t cuboid_T_bytes = 0;
  // Morton-sorted FP64 positions (device, [n][3]): the exact geometry of the
  // close pairs and the input of the transposed plan; host copy of the leaf
  // ranges
  double *src_pos64 = nullptr, *tgt_pos64 = nullptr;
  std::vector<int> h_src_off, h_tgt_off;
  // reverse mode: the transposed plan (built on first use; its sources are
  // this plan's targets and vice versa) and the buffers of the position
  // gradient
  std::vector<int> h_self;                     // sorted self map as last set (empty: none)
  int self_version = 0;                        // bumped by every set_self_indices
  cdfmm_b200_plan *adjoint = nullptr;
  int adjoint_self_version = -1;
  float4 *wbuf = nullptr;                      // [nt][K] sorted dL/dH weights
  float4 *gpart = nullptr;                     // [nt][groups] near gradient partial sums
  size_t wbuf_count = 0, gpart_count = 0;
  void *stage_grad = nullptr;                  // device staging of host gradient inputs / outputs
  size_t stage_grad_bytes = 0;

  cdfmm_b200_stats stats{};
};
