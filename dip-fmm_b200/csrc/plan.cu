// C ABI of the B200 evaluator: plan construction and the evaluate pipeline.
//
// Pipeline of one evaluate call (K states), stream-ordered:
//   [H2D moments] -> gather (user -> Morton order, / scale^3)
//   far stream : P2M -> M2M (levels d-1..0) -> M2L (levels 2..d) -> L2L (3..d)
//   near stream: list1 P2P                       (runs concurrently with far)
//   join -> L2P + near/far combine + unsort to user order -> [D2H results]
// (upstream src/cuda_fmm.cu:3457-3655 orders the same stages with a far and a
// near stream and an event join before the combine).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "cdfmm_b200.h"
#include "far_kernels.hpp"
#include "fmm_internal.hpp"
#include "geometry.hpp"
#include "kernels.cuh"
#include "m2l_tc.hpp"
#include "p2m_tc.hpp"
#include "near_grad_tc.hpp"
#include "near_tc.hpp"

namespace {

using namespace cdfmm_b200;

thread_local std::string g_last_error;

struct AbiError : std::runtime_error {
  int code;
  AbiError(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void check(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    const int code = e == cudaErrorMemoryAllocation ? CDFMM_B200_ERR_OUT_OF_MEMORY : CDFMM_B200_ERR_RUNTIME;
    throw AbiError(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

void require(bool ok, const std::string &what) {
  if (!ok) throw AbiError(CDFMM_B200_ERR_INVALID_ARGUMENT, what);
}

template <typename T> T *dalloc(size_t count, uint64_t &bytes) {
  void *p = nullptr;
  if (count == 0) count = 1;
  check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
  bytes += count * sizeof(T);
  return static_cast<T *>(p);
}

// Host -> device copy that has landed when it returns.  cudaMemcpy from
// pageable host memory may return once the data is in the driver's staging
// buffer, before the DMA into device memory is done; it is ordered only on
// the legacy default stream, and the evaluator's kernels run on non-blocking
// streams that do not wait for that stream.
void copy_to_device(void *dst, const void *src, size_t bytes, const char *what) {
  if (bytes == 0) return;
  check(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice), what);
  check(cudaStreamSynchronize(cudaStreamLegacy), what);
}

template <typename T> void upload(T *dst, const T *src, size_t count, uint64_t &bytes) {
  if (count == 0) return;
  copy_to_device(dst, src, count * sizeof(T), "cudaMemcpy H2D");
  bytes += count * sizeof(T);
}

// Events of the concurrent trace (cdfmm_b200_set_timing mode 2).
constexpr int kTraceBegin = 12, kTraceP2pBegin = 13, kTraceP2pEnd = 14, kTraceFarBegin = 15, kTraceM2lBegin = 16,
              kTraceFarEnd = 17, kTraceEnd = 18;

// Grows a device buffer to at least `need` bytes (contents not kept).
template <typename T> T *grow_bytes(T *&buf, size_t &have, size_t need, const char *what) {
  if (have < need) {
    if (buf) cudaFree(buf);
    buf = nullptr;
    have = 0;
    check(cudaMalloc(reinterpret_cast<void **>(&buf), need), what);
    have = need;
  }
  return buf;
}

// TMEM columns for m_tiles accumulators acc_stride apart (a power of two >= 32).
uint32_t tmem_columns(int m_tiles, int acc_stride) {
  uint32_t cols = 32;
  while (cols < static_cast<uint32_t>(m_tiles * acc_stride)) cols <<= 1;
  return cols;
}

// Grows a device buffer to at least `need` elements (contents not kept).
template <typename T> T *grow(T *&buf, size_t &have, size_t need, const char *what) {
  if (have < need) {
    if (buf) cudaFree(buf);
    buf = nullptr;
    have = 0;
    check(cudaMalloc(reinterpret_cast<void **>(&buf), need * sizeof(T)), what);
    have = need;
  }
  return buf;
}

void free_plan(cdfmm_b200_plan *p) {
  if (p == nullptr) return;
  void *ptrs[] = {p->src_rel, p->tgt_rel, p->src_off, p->tgt_off, p->src_perm, p->tgt_perm, p->src_inv, p->tgt_inv,
                  p->self_idx, p->leaf_self, p->p2p_work, p->m2m_off, p->m2m_pair, p->l2l_off, p->l2l_pair, p->m2m_coef,
                  p->l2l_coef, p->m2l_T, p->basis, p->mom, p->M, p->L, p->near, p->stage_in,
                  p->stage_out, p->scale_m, p->scale_l, p->m2l_tiles, p->tc_a_hi, p->tc_a_lo,
                  p->tc_b, p->m2l_fold_buf, p->tc_fold_off, p->tc_fold, p->tc_expand, p->tc_tiles, p->error_flag, p->wbuf, p->gpart, p->stage_grad, p->p2p_next_unit,
                  p->close_targets, p->close_r_fp32, p->close_r_exact, p->src_pos64, p->tgt_pos64,
                  p->src_size, p->src_size64, p->cuboid_T, p->cuboid_base, p->ntc_blk_off, p->ntc_blk_src,
                  p->ntc_blk_pos, p->ntc_work, p->ntc_b, p->ngt_blk_off, p->ngt_blk_src, p->ngt_blk_pos,
                  p->ngt_b};
  for (void *q : ptrs)
    if (q != nullptr) cudaFree(q);
  if (p->p2p_work_wide != nullptr && p->p2p_work_wide != p->p2p_work) cudaFree(p->p2p_work_wide);
  if (p->status != nullptr) cudaFreeHost(p->status);
  if (p->adjoint != nullptr) free_plan(p->adjoint);
  if (p->ev_fork) cudaEventDestroy(p->ev_fork);
  if (p->ev_join) cudaEventDestroy(p->ev_join);
  for (cudaEvent_t &e : p->ev_t)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : p->io_events)
    if (e) cudaEventDestroy(e);
  if (p->io_in) cudaStreamDestroy(p->io_in);
  if (p->io_out) cudaStreamDestroy(p->io_out);
  if (p->near_stream) cudaStreamDestroy(p->near_stream);
  if (p->far_stream) cudaStreamDestroy(p->far_stream);
  if (p->ev_far) cudaEventDestroy(p->ev_far);
  if (p->stream) cudaStreamDestroy(p->stream);
  delete p;
}

int fail(cdfmm_b200_plan *plan, int code, const std::string &msg) {
  if (plan != nullptr) plan->last_error = msg;
  g_last_error = msg;
  return code;
}

size_t device_smem_optin(int device) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  return static_cast<size_t>(v);
}

// Moves a nonzero device error flag into the host status record (one thread).
__global__ void collect_status_kernel(int *flag, cdfmm_b200_plan::StatusRecord *rec, unsigned long long call) {
  const int f = *reinterpret_cast<volatile int *>(flag);
  if (f != 0) {
    *flag = 0;
    volatile cdfmm_b200_plan::StatusRecord *r = rec;
    r->code = f;
    r->call = call;
    r->count = r->count + 1;
    __threadfence_system();
  }
}

std::string timeout_message(int code, int calls, bool own) {
  std::string m = "tensor-core M2L: a bounded wait expired (code " + std::to_string(code) + ")";
  if (own) {
    m += "; the results of this call are invalid (the affected local expansions were set to NaN)";
    if (calls > 1) m += "; " + std::to_string(calls - 1) + " earlier call(s) on this plan failed the same way";
  } else {
    m += " in " + std::to_string(calls) + " call(s) on this plan since the last report; their results are invalid "
         "(the affected local expansions were set to NaN)";
  }
  return m;
}

} // namespace

cudaError_t cdfmm_b200_collect_status(cdfmm_b200_plan *plan, cudaStream_t s, unsigned long long call) {
  collect_status_kernel<<<1, 1, 0, s>>>(plan->error_flag, plan->status_dev, call);
  return cudaGetLastError();
}

std::string cdfmm_b200_own_status(cdfmm_b200_plan *plan, unsigned long long call) {
  const volatile cdfmm_b200_plan::StatusRecord *r = plan->status;
  const int count = r->count;
  if (count == plan->status_seen || r->call != call) return std::string();
  const int calls = count - plan->status_seen;
  plan->status_seen = count;
  return timeout_message(r->code, calls, true);
}

// The plan's close-pair list (see CloseGeometry): counts every target's
// pairs below four thresholds (leaf width / 2^k, k = kCloseShift .. + 3),
// takes the largest threshold whose list holds at most 4 pairs per target
// on average (dense clusters get a smaller one; the closest pairs, which
// need the exact r most, are always inside it), and writes the list.  A
// geometry with more than 64 pairs per target even at the smallest
// threshold keeps no list (close_shift = -1).
static void build_close_pairs(cdfmm_b200_plan *plan, uint64_t &bytes, uint64_t &h2d) {
  plan->n_close_targets = 0;
  plan->close_pairs = 0;
  plan->close_shift = -1;
  if (plan->nt == 0 || plan->ns == 0 || plan->n_p2p_work_wide == 0) return;
  float thr[kCloseLevels];
  for (int l = 0; l < kCloseLevels; ++l)
    thr[l] = static_cast<float>(std::ldexp(1.0, -2 * (plan->depth + kCloseShift + l)));
  uint64_t tmp = 0;
  int *counts = dalloc<int>(4 * static_cast<size_t>(plan->nt), tmp);
  launch_p2p_close_count(plan->src_rel, plan->src_off, plan->tgt_rel, plan->p2p_work_wide, plan->n_p2p_work_wide,
                         plan->depth, thr, counts, nullptr);
  std::vector<int> h(4 * static_cast<size_t>(plan->nt));
  cudaError_t e = cudaMemcpy(h.data(), counts, sizeof(int) * h.size(), cudaMemcpyDeviceToHost);
  cudaFree(counts);
  check(e, "close-pair count");
  long long total[kCloseLevels] = {};
  for (int i = 0; i < plan->nt; ++i)
    for (int l = 0; l < kCloseLevels; ++l) total[l] += h[4 * static_cast<size_t>(i) + l];
  int level = kCloseLevels - 1;
  for (int l = 0; l < kCloseLevels; ++l)
    if (total[l] <= 4LL * plan->nt + 1024) {
      level = l;
      break;
    }
  if (total[level] > 64LL * plan->nt + 1024) return;
  plan->close_shift = kCloseShift + level;
  if (total[level] == 0) return;
  std::vector<int4> targets;
  std::vector<int> first(static_cast<size_t>(plan->nt), 0);
  int run = 0;
  for (int i = 0; i < plan->nt; ++i) {
    const int c = h[4 * static_cast<size_t>(i) + level];
    first[static_cast<size_t>(i)] = run;
    if (c > 0) targets.push_back(make_int4(i, run, c, 0));
    run += c;
  }
  double *d_sabs = dalloc<double>(3 * static_cast<size_t>(plan->ns), tmp);
  double *d_tabs = dalloc<double>(3 * static_cast<size_t>(plan->nt), tmp);
  int *d_first = dalloc<int>(first.size(), tmp);
  plan->close_r_fp32 = dalloc<float4>(static_cast<size_t>(run), bytes);
  plan->close_r_exact = dalloc<float4>(static_cast<size_t>(run), bytes);
  launch_normalised_positions(plan->src_pos64, plan->ns, plan->root_centre, 1.0 / plan->scale, d_sabs, nullptr);
  launch_normalised_positions(plan->tgt_pos64, plan->nt, plan->root_centre, 1.0 / plan->scale, d_tabs, nullptr);
  upload(d_first, first.data(), first.size(), h2d);
  launch_p2p_close_write(plan->src_rel, plan->src_off, plan->tgt_rel, plan->p2p_work_wide, plan->n_p2p_work_wide,
                         plan->depth, thr[level], d_first, d_sabs, d_tabs, plan->close_r_fp32, plan->close_r_exact,
                         nullptr);
  e = cudaDeviceSynchronize();
  cudaFree(d_sabs);
  cudaFree(d_tabs);
  cudaFree(d_first);
  check(e, "close-pair write");
  plan->close_targets = dalloc<int4>(targets.size(), bytes);
  upload(plan->close_targets, targets.data(), targets.size(), h2d);
  plan->n_close_targets = static_cast<int>(targets.size());
  plan->close_pairs = static_cast<uint64_t>(run);
}

void cdfmm_b200_record_error(cdfmm_b200_plan *plan, const std::string &msg) {
  if (plan != nullptr) plan->last_error = msg;
  g_last_error = msg;
}

extern "C" {

int cdfmm_b200_device_count(int32_t *count) {
  if (count == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "count is NULL");
  int c = 0;
  const cudaError_t e = cudaGetDeviceCount(&c);
  if (e != cudaSuccess) {
    cudaGetLastError();
    c = 0;
  }
  *count = c;
  return CDFMM_B200_OK;
}

int cdfmm_b200_device_info(int32_t device, char *name, size_t name_len, int32_t *cc_major,
                           int32_t *cc_minor) {
  cudaDeviceProp prop{};
  const cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(nullptr, CDFMM_B200_ERR_NO_DEVICE, std::string("cudaGetDeviceProperties: ") + cudaGetErrorString(e));
  }
  if (name != nullptr && name_len > 0) {
    std::strncpy(name, prop.name, name_len - 1);
    name[name_len - 1] = '\0';
  }
  if (cc_major) *cc_major = prop.major;
  if (cc_minor) *cc_minor = prop.minor;
  return CDFMM_B200_OK;
}

static size_t corun_m2l_smem_budget(const cdfmm_b200_plan *plan, int K);

// BF16 hi/lo B tiles of the tensor-core M2L per (order, Npad, Kpad), packed
// once per process and shared by the plans of that order.
static std::shared_ptr<const std::vector<uint16_t>> packed_b_tiles(int p, const HostOperators &ops,
                                                                    const M2lTraceless &red, int Npad, int Kpad) {
  static std::mutex mutex;
  static std::map<std::tuple<int, int, int>, std::shared_ptr<const std::vector<uint16_t>>> cache;
  std::lock_guard<std::mutex> lock(mutex);
  auto &slot = cache[std::make_tuple(p, Npad, Kpad)];
  if (!slot) slot = std::make_shared<const std::vector<uint16_t>>(pack_m2l_b_tiles(*ops.m2l_T64, ops.n, red, Npad, Kpad));
  return slot;
}

// A new plan's sizes, streams and events (root cube, geometry, operators
// and buffers are set by the creators below).
static cdfmm_b200_plan *new_plan(int ns, int nt, int order, int depth, int max_states, int device) {
  cdfmm_b200_plan *plan = new cdfmm_b200_plan();
  try {
    plan->device = device;
    plan->ns = ns;
    plan->nt = nt;
    plan->p = order;
    plan->depth = depth;
    plan->n_leaves = 1 << (3 * depth);
    plan->n_nodes = level_offset(depth + 1);
    plan->max_states = max_states;
    plan->m2l_mode = CDFMM_B200_M2L_FP32; // tensor-core M2L is selected in finish_plan when available

    check(cudaStreamCreateWithFlags(&plan->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaStreamCreateWithFlags(&plan->near_stream, cudaStreamNonBlocking), "cudaStreamCreate");
    {
      // The far field runs on a high-priority stream so its CTAs are
      // dispatched into SM slots as they free up while the (FP32-bound) near
      // field runs at the default priority: tensor-core M2L and P2P overlap.
      int least = 0, greatest = 0;
      check(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
      check(cudaStreamCreateWithPriority(&plan->far_stream, cudaStreamNonBlocking, greatest), "cudaStreamCreate");
      check(cudaEventCreateWithFlags(&plan->ev_far, cudaEventDisableTiming), "cudaEventCreate");
    }
    check(cudaStreamCreateWithFlags(&plan->io_in, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaStreamCreateWithFlags(&plan->io_out, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaEventCreateWithFlags(&plan->ev_fork, cudaEventDisableTiming), "cudaEventCreate");
    check(cudaEventCreateWithFlags(&plan->ev_join, cudaEventDisableTiming), "cudaEventCreate");
    for (cudaEvent_t &e : plan->ev_t) check(cudaEventCreate(&e), "cudaEventCreate");
  } catch (...) {
    free_plan(plan);
    throw;
  }
  return plan;
}

static void set_root(cdfmm_b200_plan *plan, const double centre[3], double half_width) {
  for (int a = 0; a < 3; ++a) plan->root_centre[a] = centre[a];
  plan->root_half_width = half_width;
  plan->scale = 2.0 * half_width;
  plan->inv_scale3 = static_cast<float>(1.0 / (plan->scale * plan->scale * plan->scale));
  plan->phi_scale = static_cast<float>(plan->scale);
}

// Everything that follows from the plan's Morton-ordered geometry (src_pos64,
// tgt_pos64, src_perm, tgt_perm, src_off, tgt_off on the device, h_src_off,
// h_tgt_off on the host): leaf-relative FP32 positions, inverse
// permutations, near-field work units, close pairs, operators, interaction
// statistics, state buffers and the tensor-core M2L set-up.
static void finish_plan(cdfmm_b200_plan *plan, int m2l_mode) {
  const int n_leaves = plan->n_leaves;
  auto mark = std::chrono::steady_clock::now();
  auto lap = [&mark](double &slot) {
    const auto now = std::chrono::steady_clock::now();
    slot += std::chrono::duration<double, std::milli>(now - mark).count();
    mark = now;
  };

  HostOperators &ops = plan->ops;
  ops = build_host_operators(plan->p, plan->depth, 16);
  plan->n = ops.n;
  const int n = ops.n;
  const int J = m2l_simt_beta_per_thread(n);
  if (ops.m2l_ld < 16 * J) {
    ops = build_host_operators(plan->p, plan->depth, 16 * J);
  }
  uint64_t &bytes = plan->stats.persistent_device_bytes;
  uint64_t &h2d = plan->stats.setup_h2d_bytes;
  lap(plan->stats.setup_ms_operators);

  // geometry: leaf-relative positions and inverse permutations on the device
  {
    const double inv_scale = 1.0 / plan->scale;
    plan->src_rel = dalloc<float4>(plan->ns, bytes);
    plan->tgt_rel = dalloc<float4>(plan->nt, bytes);
    launch_relative_positions(plan->src_pos64, plan->src_off, n_leaves, plan->ns, plan->depth, plan->root_centre,
                              plan->root_half_width, inv_scale, plan->src_rel, nullptr);
    launch_relative_positions(plan->tgt_pos64, plan->tgt_off, n_leaves, plan->nt, plan->depth, plan->root_centre,
                              plan->root_half_width, inv_scale, plan->tgt_rel, nullptr);
    plan->src_inv = dalloc<int>(plan->ns, bytes);
    plan->tgt_inv = dalloc<int>(plan->nt, bytes);
    check(cudaMemset(plan->src_inv, 0xff, sizeof(int) * std::max(plan->ns, 1)), "cudaMemset");
    check(cudaMemset(plan->tgt_inv, 0xff, sizeof(int) * std::max(plan->nt, 1)), "cudaMemset");
    uint64_t tmp = 0;
    int *flags = dalloc<int>(2, tmp);
    int h_flags[2] = {0, 0};
    cudaError_t e = cudaMemset(flags, 0, 2 * sizeof(int));
    if (e == cudaSuccess) {
      launch_inverse_permutation(plan->src_perm, plan->ns, plan->src_inv, flags, nullptr);
      launch_inverse_permutation(plan->tgt_perm, plan->nt, plan->tgt_inv, flags + 1, nullptr);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(h_flags, flags, sizeof h_flags, cudaMemcpyDeviceToHost);
    cudaFree(flags);
    check(e, "plan geometry");
    require((h_flags[0] & 1) == 0, "source_permutation out of range");
    require((h_flags[1] & 1) == 0, "target_permutation out of range");
    require((h_flags[0] & 2) == 0, "source_permutation is not a permutation");
    require((h_flags[1] & 2) == 0, "target_permutation is not a permutation");
    plan->self_idx = dalloc<int>(plan->nt, bytes);
    plan->leaf_self = dalloc<int2>(n_leaves, bytes);
  }
  lap(plan->stats.setup_ms_geometry);

  {
    int sms = 0;
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, plan->device), "device attribute");
    plan->sm_count = sms;
    plan->p2p_next_unit = dalloc<int>(1, bytes);
    const std::vector<int4> work =
        p2p_work_units(plan->h_src_off.data(), plan->h_tgt_off.data(), plan->depth, sms, true);
    const std::vector<int4> wide =
        p2p_work_units(plan->h_src_off.data(), plan->h_tgt_off.data(), plan->depth, sms, false);
    plan->n_p2p_work = static_cast<int>(work.size());
    plan->n_p2p_work_wide = static_cast<int>(wide.size());
    if (!work.empty()) {
      plan->p2p_work = dalloc<int4>(work.size(), bytes);
      upload(plan->p2p_work, work.data(), work.size(), h2d);
    }
    if (wide.size() == work.size()) {
      plan->p2p_work_wide = plan->p2p_work; // no unit was capped: the same units
    } else {
      plan->p2p_work_wide = dalloc<int4>(wide.size(), bytes);
      upload(plan->p2p_work_wide, wide.data(), wide.size(), h2d);
    }
    build_close_pairs(plan, bytes, h2d);
  }
  lap(plan->stats.setup_ms_near);

  // operators
  std::vector<int8_t> basis(static_cast<size_t>(n) * 4);
  for (int a = 0; a < n; ++a) {
    basis[4 * a] = static_cast<int8_t>(ops.ax[a]);
    basis[4 * a + 1] = static_cast<int8_t>(ops.ay[a]);
    basis[4 * a + 2] = static_cast<int8_t>(ops.az[a]);
    basis[4 * a + 3] = static_cast<int8_t>(ops.ax[a] + ops.ay[a] + ops.az[a]);
  }
  std::vector<int> m2m_pair(ops.m2m_pair_g.size()), l2l_pair(ops.l2l_pair_g.size());
  for (size_t e = 0; e < m2m_pair.size(); ++e) m2m_pair[e] = ops.m2m_pair_g[e] | (ops.m2m_pair_in[e] << 16);
  for (size_t e = 0; e < l2l_pair.size(); ++e) l2l_pair[e] = ops.l2l_pair_g[e] | (ops.l2l_pair_in[e] << 16);
  plan->basis = dalloc<int8_t>(basis.size(), bytes);
  plan->m2m_off = dalloc<int>(ops.m2m_off.size(), bytes);
  plan->l2l_off = dalloc<int>(ops.l2l_off.size(), bytes);
  plan->m2m_pair = dalloc<int>(m2m_pair.size(), bytes);
  plan->l2l_pair = dalloc<int>(l2l_pair.size(), bytes);
  plan->m2m_coef = dalloc<float>(ops.m2m_coef.size(), bytes);
  plan->l2l_coef = dalloc<float>(ops.l2l_coef.size(), bytes);
  upload(plan->basis, basis.data(), basis.size(), h2d);
  upload(plan->m2m_off, ops.m2m_off.data(), ops.m2m_off.size(), h2d);
  upload(plan->l2l_off, ops.l2l_off.data(), ops.l2l_off.size(), h2d);
  upload(plan->m2m_pair, m2m_pair.data(), m2m_pair.size(), h2d);
  upload(plan->l2l_pair, l2l_pair.data(), l2l_pair.size(), h2d);
  upload(plan->m2m_coef, ops.m2m_coef.data(), ops.m2m_coef.size(), h2d);
  upload(plan->l2l_coef, ops.l2l_coef.data(), ops.l2l_coef.size(), h2d);

  // M2L: matrices, exact power-of-two level scalings, and the work tiles.
  std::vector<float> sm(static_cast<size_t>(plan->depth + 1) * n), sl(sm.size());
  for (int level = 0; level <= plan->depth; ++level)
    for (int a = 0; a < n; ++a) {
      const int deg = ops.ax[a] + ops.ay[a] + ops.az[a];
      sm[static_cast<size_t>(level) * n + a] = std::ldexp(1.0F, level * deg);
      sl[static_cast<size_t>(level) * n + a] = std::ldexp(1.0F, level * (deg + 1));
    }
  std::vector<int4> tiles;
  for (int level = plan->depth; level >= 2; --level) {
    const int pside = 1 << (level - 1);
    for (int cls = 0; cls < 8; ++cls)
      for (int pz = 0; pz < pside; pz += 4)
        for (int py = 0; py < pside; py += 4)
          for (int px = 0; px < pside; px += 4) tiles.push_back(make_int4(level, cls, px | (py << 10) | (pz << 20), 0));
  }
  plan->n_tiles = static_cast<int>(tiles.size());
  plan->scale_m = dalloc<float>(sm.size(), bytes);
  plan->scale_l = dalloc<float>(sl.size(), bytes);
  plan->m2l_tiles = dalloc<int4>(tiles.size(), bytes);
  upload(plan->scale_m, sm.data(), sm.size(), h2d);
  upload(plan->scale_l, sl.data(), sl.size(), h2d);
  upload(plan->m2l_tiles, tiles.data(), tiles.size(), h2d);
  if (plan->depth >= 2) {
    // the traceless reduction (both M2L paths): fold and expansion tables,
    // and the FP32 sub-blocks [343][n_in][ld] the SIMT M2L applies
    const M2lTraceless red = m2l_traceless(plan->p);
    plan->tc_n_in = static_cast<int>(red.in_set.size());
    plan->tc_n_out = static_cast<int>(red.out_set.size());
    plan->tc_n_derived = red.n_derived;
    plan->tc_fold_off = dalloc<int>(red.fold_off.size(), bytes);
    upload(plan->tc_fold_off, red.fold_off.data(), red.fold_off.size(), h2d);
    plan->tc_fold = dalloc<int>(std::max<size_t>(red.fold.size(), 1), bytes);
    upload(plan->tc_fold, red.fold.data(), red.fold.size(), h2d);
    plan->tc_expand = dalloc<int>(red.expand.size(), bytes);
    upload(plan->tc_expand, red.expand.data(), red.expand.size(), h2d);
    plan->m2l_ld_red = 16 * m2l_simt_beta_per_thread(plan->tc_n_out);
    const std::vector<double> &T64 = *ops.m2l_T64;
    std::vector<float> Tr(static_cast<size_t>(343) * std::max(plan->tc_n_in, 1) * plan->m2l_ld_red, 0.0F);
    for (size_t slot = 0; slot < 343; ++slot)
      for (int j = 0; j < plan->tc_n_in; ++j)
        for (int i = 0; i < plan->tc_n_out; ++i)
          Tr[(slot * plan->tc_n_in + static_cast<size_t>(j)) * plan->m2l_ld_red + static_cast<size_t>(i)] =
              static_cast<float>(T64[(slot * n + static_cast<size_t>(red.in_set[static_cast<size_t>(j)])) * n +
                                     static_cast<size_t>(red.out_set[static_cast<size_t>(i)])]);
    plan->m2l_T = dalloc<float>(Tr.size(), bytes);
    upload(plan->m2l_T, Tr.data(), Tr.size(), h2d);
    plan->stats.m2l_matrix_bytes = Tr.size() * sizeof(float);
  }

  lap(plan->stats.setup_ms_operators);
  // statistics of the implicit interaction lists (counted on the host)
  {
    uint64_t classes = 0, inter = 0, pairs = 0;
    bool used[343] = {};
    const int32_t *so = plan->h_src_off.data();
    const int32_t *to = plan->h_tgt_off.data();
    // occupancy of every level for sources and targets
    std::vector<std::vector<int>> socc(plan->depth + 1), tocc(plan->depth + 1);
    for (int level = 0; level <= plan->depth; ++level) {
      socc[level].assign(static_cast<size_t>(1) << (3 * level), 0);
      tocc[level].assign(static_cast<size_t>(1) << (3 * level), 0);
    }
    for (int m = 0; m < n_leaves; ++m) {
      for (int level = 0; level <= plan->depth; ++level) {
        const int shift = 3 * (plan->depth - level);
        socc[level][m >> shift] += so[m + 1] - so[m];
        tocc[level][m >> shift] += to[m + 1] - to[m];
      }
    }
    for (int level = 2; level <= plan->depth; ++level) {
      const int side = 1 << level;
      for (int t = 0; t < side * side * side; ++t) {
        if (tocc[level][t] == 0) continue;
        int tx, ty, tz;
        demorton3(static_cast<uint32_t>(t), tx, ty, tz);
        for (int sz = 2 * (tz >> 1) - 2; sz <= 2 * (tz >> 1) + 3; ++sz)
          for (int sy = 2 * (ty >> 1) - 2; sy <= 2 * (ty >> 1) + 3; ++sy)
            for (int sx = 2 * (tx >> 1) - 2; sx <= 2 * (tx >> 1) + 3; ++sx) {
              if (sx < 0 || sy < 0 || sz < 0 || sx >= side || sy >= side || sz >= side) continue;
              if (std::abs(sx - tx) <= 1 && std::abs(sy - ty) <= 1 && std::abs(sz - tz) <= 1) continue;
              if (socc[level][morton3(sx, sy, sz)] == 0) continue;
              ++inter;
              const int slot = (tx - sx + 3) * 49 + (ty - sy + 3) * 7 + (tz - sz + 3);
              if (!used[slot]) {
                used[slot] = true;
                ++classes;
              }
            }
      }
    }
    const int side = 1 << plan->depth;
    for (int m = 0; m < n_leaves; ++m) {
      const int nt_leaf = to[m + 1] - to[m];
      if (nt_leaf == 0) continue;
      int x, y, z;
      demorton3(static_cast<uint32_t>(m), x, y, z);
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            const int a = x + dx, b = y + dy, c = z + dz;
            if (a < 0 || b < 0 || c < 0 || a >= side || b >= side || c >= side) continue;
            const uint32_t q = morton3(a, b, c);
            pairs += static_cast<uint64_t>(nt_leaf) * static_cast<uint64_t>(so[q + 1] - so[q]);
          }
    }
    plan->stats.m2l_classes = classes;
    plan->stats.m2l_interactions = inter;
    plan->stats.p2p_pairs = pairs;
  }

  lap(plan->stats.setup_ms_statistics);
  // state buffers sized for max_states
  const size_t K = static_cast<size_t>(plan->max_states);
  plan->mom = dalloc<float4>(static_cast<size_t>(plan->ns) * ((K + 1) & ~static_cast<size_t>(1)), bytes); // paired rows
  plan->M = dalloc<float>(static_cast<size_t>(plan->n_nodes) * n * K, bytes);
  plan->L = dalloc<float>(static_cast<size_t>(plan->n_nodes) * n * K, bytes);
  plan->near = dalloc<float4>(static_cast<size_t>(plan->nt) * K, bytes);
  check(cudaMemset(plan->M, 0, static_cast<size_t>(plan->n_nodes) * n * K * sizeof(float)), "cudaMemset");
  check(cudaMemset(plan->L, 0, static_cast<size_t>(plan->n_nodes) * n * K * sizeof(float)), "cudaMemset");
  check(cudaMemset(plan->near, 0, static_cast<size_t>(std::max(plan->nt, 1)) * K * sizeof(float4)), "cudaMemset");

  const size_t smem = device_smem_optin(plan->device);
  configure_far_kernels(smem);
  configure_m2l_simt(smem);
  configure_p2p(smem);
  plan->p2m_chunk = 64;
  while (plan->p2m_chunk > 8 && p2m_smem_bytes(n, plan->p, static_cast<int>(K), plan->p2m_chunk) > smem) plan->p2m_chunk /= 2;
  require(p2m_smem_bytes(n, plan->p, 4, plan->p2m_chunk) <= smem && l2p_smem_bytes(n, plan->p, 4) <= smem,
          "order exceeds the shared-memory budget of one CTA");
  check(cudaDeviceSynchronize(), "plan upload");
  plan->error_flag = dalloc<int>(1, bytes);
  check(cudaMemset(plan->error_flag, 0, sizeof(int)), "cudaMemset");
  check(cudaHostAlloc(reinterpret_cast<void **>(&plan->status), sizeof(cdfmm_b200_plan::StatusRecord),
                      cudaHostAllocMapped), "cudaHostAlloc");
  std::memset(plan->status, 0, sizeof(cdfmm_b200_plan::StatusRecord));
  check(cudaHostGetDevicePointer(reinterpret_cast<void **>(&plan->status_dev), plan->status, 0),
        "cudaHostGetDevicePointer");
  plan->tc_wait_limit = kTcWaitLimit;

  lap(plan->stats.setup_ms_buffers);
  // Tensor-core M2L: sm_100 devices and at least two pipeline stages in
  // shared memory (the traceless operator's N = 16 ceil((p+1)^2 / 16) <= 128
  // accumulator columns for every order up to 10).  AUTO keeps order 10 on
  // the FP32 SIMT M2L, whose products are exact FP32.
  {
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, plan->device);
    // traceless reduction: (p+1)^2 - 1 folded moments in, (p+1)^2 locals out
    const M2lTraceless red = m2l_traceless(plan->p);
    const int Kpad = std::max(16, round_up(static_cast<int>(red.in_set.size()), 16));
    const int Npad = round_up(static_cast<int>(red.out_set.size()), 16);
    // Pipeline shapes: 1, 2 or 4 128-row accumulators per CTA sharing each
    // B tile, with as many stages as fit one CTA per SM, or half / a third
    // of that for two / three CTAs per SM; each with the three products as
    // three MMAs of N = Npad, or (when 2 Npad <= 256) A_hi x [B_hi | B_lo]
    // fused into one MMA of N = 2 Npad plus A_lo x B_hi (two larger MMAs
    // instead of three: fewer instructions for the one issuing thread;
    // twice the TMEM columns).  Default: two accumulators, two CTAs per SM,
    // three MMAs; the autotuner times the candidates on first use for
    // each K.
    auto acc_stride_of = [&](int fuse) { return round_up(fuse ? 2 * Npad : Npad, 32); };
    auto max_stages = [&](int mt, size_t budget) {
      int st = 0;
      while (st < 8 && m2l_tc_smem_bytes(Npad, mt, st + 1, n) <= budget) ++st;
      return st;
    };
    const size_t one_cta = std::min<size_t>(smem, 224 * 1024), two_cta = 112 * 1024, three_cta = 74 * 1024;
    // one CTA beside two co-resident near-field CTAs (schedule CORUN)
    const size_t corun_cta = corun_m2l_smem_budget(plan, std::min(plan->max_states, 64));
    plan->tc_candidates.clear();
    for (int fuse : {0, 1}) {
      if (fuse && 2 * Npad > 256) continue; // MMA N <= 256
      const int acc = acc_stride_of(fuse);
      for (int mt : {2, 1, 4}) {
        if (mt * acc > 512) continue;
        const int s1 = max_stages(mt, one_cta);
        const int s2 = max_stages(mt, two_cta);
        const int s3 = max_stages(mt, three_cta);
        const int sc = max_stages(mt, corun_cta);
        if (s2 >= 2 && s2 < s1 && tmem_columns(mt, acc) <= 256) plan->tc_candidates.push_back({mt, s2, fuse});
        if (s1 >= 2) plan->tc_candidates.push_back({mt, s1, fuse});
        if (s3 >= 2 && s3 < s2 && 3 * tmem_columns(mt, acc) <= 512) plan->tc_candidates.push_back({mt, s3, fuse});
        if (sc >= 2 && sc != s1 && sc != s2 && sc != s3) plan->tc_candidates.push_back({mt, sc, fuse});
      }
    }
    const int m_tiles = plan->tc_candidates.empty() ? 1 : plan->tc_candidates.front().m_tiles;
    const int stages = plan->tc_candidates.empty() ? 0 : plan->tc_candidates.front().stages;
    const int fuse0 = plan->tc_candidates.empty() ? 0 : plan->tc_candidates.front().fuse;
    const int acc_stride = acc_stride_of(fuse0);
    // AUTO and BF16X3 run the M2L on the tensor cores for any K (fewer
    // than 8 states fill 8-row groups of the MMA tile with zero rows: the
    // tensor cores still beat the FP32 SIMT M2L several times over);
    // FP32 keeps the SIMT M2L (the plain per-state path).
    const bool wanted = m2l_mode == CDFMM_B200_M2L_BF16X3 || (m2l_mode == CDFMM_B200_M2L_AUTO && plan->p <= 9);
    plan->tc_supported = major == 10 && plan->depth >= 2 && Npad <= 256 && stages >= 2 && wanted &&
                         configure_m2l_tc(smem);
    if (plan->tc_supported) {
      plan->tc_Kpad = Kpad;
      plan->tc_Npad = Npad;
      plan->tc_stages = stages;
      plan->tc_m_tiles = m_tiles;
      plan->tc_acc_stride = acc_stride;
      plan->tc_fuse = fuse0;
      plan->tc_tmem_cols = tmem_columns(m_tiles, acc_stride);
      plan->tc_Kp_max = round_up(std::min(plan->max_states, 128), 8);
      const size_t boxes = static_cast<size_t>(plan->n_nodes - level_offset(2)) + 1;
      const size_t box_elems = static_cast<size_t>(plan->tc_Kp_max) * Kpad;
      plan->tc_a_hi = dalloc<uint16_t>(boxes * box_elems, bytes);
      plan->tc_a_lo = dalloc<uint16_t>(boxes * box_elems, bytes);
      const std::shared_ptr<const std::vector<uint16_t>> bt = packed_b_tiles(plan->p, ops, red, Npad, Kpad);
      plan->tc_b = dalloc<uint16_t>(bt->size(), bytes);
      upload(static_cast<uint16_t *>(plan->tc_b), bt->data(), bt->size(), h2d);
    } else if (m2l_mode == CDFMM_B200_M2L_BF16X3) {
      throw AbiError(CDFMM_B200_ERR_RUNTIME,
                     "split-BF16 tensor-core M2L needs an sm_100 device and depth >= 2");
    }
    // tensor-core near field: sm_100 devices (layout and buffers on first use)
    // folded moments of the SIMT M2L, for plans that can take that path
    if (plan->depth >= 2 && (!plan->tc_supported || plan->max_states > 128))
      plan->m2l_fold_buf = dalloc<float>(static_cast<size_t>(plan->n_nodes - level_offset(2)) *
                                             static_cast<size_t>(std::max(plan->tc_n_in, 1)) * plan->max_states,
                                         bytes);
    plan->ntc_supported = major == 10 && configure_near_tc(smem);
    plan->ngt_supported = plan->ntc_supported && configure_near_grad_tc(smem);
    plan->p2m_tc_ok = plan->ntc_supported && configure_p2m_tc(smem);
  }
  ops.m2l_T64.reset();
  // every set-up copy, memset and kernel (legacy default stream) is complete
  // before the plan's non-blocking streams can read what they wrote
  check(cudaDeviceSynchronize(), "plan set-up");
  lap(plan->stats.setup_ms_m2l);
  plan->m2l_mode = m2l_mode;
  plan->stats.m2l_mode_resolved = plan->tc_supported ? (m2l_mode == CDFMM_B200_M2L_FP32 ? CDFMM_B200_M2L_FP32 : CDFMM_B200_M2L_BF16X3)
                                                     : CDFMM_B200_M2L_FP32;
}

int cdfmm_b200_plan_create(const cdfmm_b200_plan_desc *desc, cdfmm_b200_plan **out_plan) {
  cdfmm_b200_plan *plan = nullptr;
  const auto t_begin = std::chrono::steady_clock::now();
  try {
    require(desc != nullptr && out_plan != nullptr, "desc and out_plan must not be NULL");
    *out_plan = nullptr;
    require(desc->struct_size == static_cast<int32_t>(sizeof(cdfmm_b200_plan_desc)), "desc.struct_size mismatch");
    require(desc->n_sources >= 0 && desc->n_targets >= 0, "negative population size");
    require(desc->order >= 0 && desc->order <= kMaxOrder, "order must be in [0, 10]");
    require(desc->depth >= 0 && desc->depth <= kMaxDepth, "depth must be in [0, 8]");
    require(desc->max_states >= 1 && desc->max_states <= 1024, "max_states must be in [1, 1024]");
    require(desc->root_half_width > 0.0 && std::isfinite(desc->root_half_width), "root_half_width must be positive");
    require(desc->m2l_mode >= CDFMM_B200_M2L_AUTO && desc->m2l_mode <= CDFMM_B200_M2L_BF16X3, "unknown m2l_mode");
    const int n_leaves = 1 << (3 * desc->depth);
    require(desc->leaf_source_offsets != nullptr && desc->leaf_target_offsets != nullptr, "leaf offsets are required");
    require(desc->leaf_source_offsets[0] == 0 && desc->leaf_source_offsets[n_leaves] == desc->n_sources,
            "leaf_source_offsets must span [0, n_sources]");
    require(desc->leaf_target_offsets[0] == 0 && desc->leaf_target_offsets[n_leaves] == desc->n_targets,
            "leaf_target_offsets must span [0, n_targets]");
    for (int m = 0; m < n_leaves; ++m) {
      require(desc->leaf_source_offsets[m + 1] >= desc->leaf_source_offsets[m], "leaf_source_offsets must be non-decreasing");
      require(desc->leaf_target_offsets[m + 1] >= desc->leaf_target_offsets[m], "leaf_target_offsets must be non-decreasing");
    }
    require(desc->n_sources == 0 || (desc->sorted_source_positions && desc->source_permutation), "source arrays are required");
    require(desc->n_targets == 0 || (desc->sorted_target_positions && desc->target_permutation), "target arrays are required");

    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
      cudaGetLastError();
      throw AbiError(CDFMM_B200_ERR_NO_DEVICE, "no CUDA device is available");
    }
    require(desc->device >= 0 && desc->device < devices, "device ordinal out of range");
    check(cudaSetDevice(desc->device), "cudaSetDevice");

    plan = new_plan(desc->n_sources, desc->n_targets, desc->order, desc->depth, desc->max_states, desc->device);
    set_root(plan, desc->root_centre, desc->root_half_width);
    uint64_t &bytes = plan->stats.persistent_device_bytes;
    uint64_t &h2d = plan->stats.setup_h2d_bytes;
    plan->src_pos64 = dalloc<double>(3 * static_cast<size_t>(plan->ns), bytes);
    plan->tgt_pos64 = dalloc<double>(3 * static_cast<size_t>(plan->nt), bytes);
    plan->src_perm = dalloc<int>(plan->ns, bytes);
    plan->tgt_perm = dalloc<int>(plan->nt, bytes);
    plan->src_off = dalloc<int>(n_leaves + 1, bytes);
    plan->tgt_off = dalloc<int>(n_leaves + 1, bytes);
    upload(plan->src_pos64, desc->sorted_source_positions, 3 * static_cast<size_t>(plan->ns), h2d);
    upload(plan->tgt_pos64, desc->sorted_target_positions, 3 * static_cast<size_t>(plan->nt), h2d);
    upload(plan->src_perm, desc->source_permutation, static_cast<size_t>(plan->ns), h2d);
    upload(plan->tgt_perm, desc->target_permutation, static_cast<size_t>(plan->nt), h2d);
    upload(plan->src_off, desc->leaf_source_offsets, static_cast<size_t>(n_leaves) + 1, h2d);
    upload(plan->tgt_off, desc->leaf_target_offsets, static_cast<size_t>(n_leaves) + 1, h2d);
    plan->h_src_off.assign(desc->leaf_source_offsets, desc->leaf_source_offsets + n_leaves + 1);
    plan->h_tgt_off.assign(desc->leaf_target_offsets, desc->leaf_target_offsets + n_leaves + 1);
    plan->stats.setup_ms_geometry =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count();
    finish_plan(plan, desc->m2l_mode);
    plan->stats.setup_ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count();

    *out_plan = plan;
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    free_plan(plan);
    return fail(nullptr, e.code, e.what());
  } catch (const std::bad_alloc &) {
    free_plan(plan);
    return fail(nullptr, CDFMM_B200_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception &e) {
    free_plan(plan);
    return fail(nullptr, CDFMM_B200_ERR_RUNTIME, e.what());
  }
}

int cdfmm_b200_plan_create_from_points(const cdfmm_b200_points_desc *desc, cdfmm_b200_plan **out_plan) {
  const auto t_begin = std::chrono::steady_clock::now();
  cdfmm_b200_plan *plan = nullptr;
  void *staged = nullptr;
  SortedPopulation src, tgt;
  auto release = [&]() {
    for (void *q : {static_cast<void *>(src.positions), static_cast<void *>(src.permutation),
                    static_cast<void *>(src.offsets), static_cast<void *>(tgt.positions),
                    static_cast<void *>(tgt.permutation), static_cast<void *>(tgt.offsets), staged})
      if (q != nullptr) cudaFree(q);
    free_plan(plan);
  };
  try {
    require(desc != nullptr && out_plan != nullptr, "desc and out_plan must not be NULL");
    *out_plan = nullptr;
    require(desc->struct_size == static_cast<int32_t>(sizeof(cdfmm_b200_points_desc)), "desc.struct_size mismatch");
    require(desc->n_sources >= 0 && desc->n_targets >= 0, "negative population size");
    require(desc->order >= 0 && desc->order <= kMaxOrder, "order must be in [0, 10]");
    require(desc->depth >= 0 && desc->depth <= kMaxDepth, "depth must be in [0, 8]");
    require(desc->max_states >= 1 && desc->max_states <= 1024, "max_states must be in [1, 1024]");
    require(desc->m2l_mode >= CDFMM_B200_M2L_AUTO && desc->m2l_mode <= CDFMM_B200_M2L_BF16X3, "unknown m2l_mode");
    require(desc->root_flags >= 0 && desc->root_flags <= (CDFMM_B200_ROOT_CENTRE | CDFMM_B200_ROOT_HALF_WIDTH),
            "unknown root_flags");
    require((desc->root_flags & CDFMM_B200_ROOT_HALF_WIDTH) == 0 ||
                (desc->root_half_width > 0.0 && std::isfinite(desc->root_half_width)),
            "UniformTreeOptions.root_half_width must be positive");
    const bool same = desc->target_positions == nullptr;
    require(desc->n_sources == 0 || desc->source_positions != nullptr, "source_positions are required");
    require(same || desc->n_targets == 0 || desc->target_positions != nullptr, "target_positions are required");
    require(desc->self_map == 0 || same, "the identity self map needs targets == sources (target_positions NULL)");
    const int ns = desc->n_sources;
    const int nt = same ? ns : desc->n_targets;

    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
      cudaGetLastError();
      throw AbiError(CDFMM_B200_ERR_NO_DEVICE, "no CUDA device is available");
    }
    require(desc->device >= 0 && desc->device < devices, "device ordinal out of range");
    check(cudaSetDevice(desc->device), "cudaSetDevice");

    cudaGetLastError(); // a stale error of an earlier call must not fail this one's checks
    plan = new_plan(ns, nt, desc->order, desc->depth, desc->max_states, desc->device);
    const auto t_tree = std::chrono::steady_clock::now();
    uint64_t &bytes = plan->stats.persistent_device_bytes;
    uint64_t &h2d = plan->stats.setup_h2d_bytes;
    const double *sp = desc->source_positions;
    const double *tp = same ? nullptr : desc->target_positions;
    if (desc->positions_on_host) {
      const size_t sb = 24 * static_cast<size_t>(ns), tb = same ? 0 : 24 * static_cast<size_t>(nt);
      check(cudaMalloc(&staged, std::max<size_t>(sb + tb, 8)), "cudaMalloc positions");
      char *d = static_cast<char *>(staged);
      if (sb) check(cudaMemcpyAsync(d, sp, sb, cudaMemcpyHostToDevice, plan->stream), "H2D positions");
      if (tb) check(cudaMemcpyAsync(d + sb, tp, tb, cudaMemcpyHostToDevice, plan->stream), "H2D positions");
      h2d += sb + tb;
      sp = reinterpret_cast<const double *>(d);
      tp = same ? nullptr : reinterpret_cast<const double *>(d + sb);
    }
    RootRequest root;
    root.has_centre = (desc->root_flags & CDFMM_B200_ROOT_CENTRE) != 0;
    root.has_half_width = (desc->root_flags & CDFMM_B200_ROOT_HALF_WIDTH) != 0;
    for (int a = 0; a < 3; ++a) root.centre[a] = desc->root_centre[a];
    root.half_width = desc->root_half_width;
    double centre[3], half_width = 0.0;
    const std::string err =
        build_device_tree(sp, ns, tp, same ? 0 : nt, desc->depth, root, centre, half_width, src, tgt, plan->stream);
    if (staged != nullptr) {
      cudaFree(staged);
      staged = nullptr;
    }
    require(err.empty(), err);
    require(half_width > 0.0 && std::isfinite(half_width),
            "the points span no volume (root half width 0); give root_half_width explicitly");
    set_root(plan, centre, half_width);
    plan->src_pos64 = src.positions;
    plan->src_perm = src.permutation;
    plan->src_off = src.offsets;
    plan->tgt_pos64 = tgt.positions;
    plan->tgt_perm = tgt.permutation;
    plan->tgt_off = tgt.offsets;
    plan->h_src_off = std::move(src.host_offsets);
    plan->h_tgt_off = std::move(tgt.host_offsets);
    src = SortedPopulation();
    tgt = SortedPopulation();
    bytes += 28 * (static_cast<uint64_t>(ns) + static_cast<uint64_t>(nt)) +
             8 * (static_cast<uint64_t>(plan->n_leaves) + 1);
    plan->stats.setup_ms_tree =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_tree).count();
    finish_plan(plan, desc->m2l_mode);
    if (desc->self_map != 0) {
      launch_identity_self(nt, plan->tgt_off, plan->n_leaves, plan->self_idx, plan->leaf_self, nullptr);
      check(cudaGetLastError(), "identity self map");
      check(cudaDeviceSynchronize(), "identity self map");
      plan->h_self.resize(static_cast<size_t>(nt));
      for (int i = 0; i < nt; ++i) plan->h_self[static_cast<size_t>(i)] = i;
      plan->has_self = true;
      plan->self_version += 1;
    }
    plan->stats.setup_ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_begin).count();
    *out_plan = plan;
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    release();
    return fail(nullptr, e.code, e.what());
  } catch (const std::bad_alloc &) {
    release();
    return fail(nullptr, CDFMM_B200_ERR_OUT_OF_MEMORY, "allocation failed");
  } catch (const std::exception &e) {
    release();
    return fail(nullptr, CDFMM_B200_ERR_RUNTIME, e.what());
  }
}

int cdfmm_b200_plan_tree(cdfmm_b200_plan *plan, double *root, int32_t *source_permutation,
                         int32_t *target_permutation, int32_t *leaf_source_offsets, int32_t *leaf_target_offsets,
                         double *sorted_source_positions, double *sorted_target_positions) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  try {
    check(cudaSetDevice(plan->device), "cudaSetDevice");
    if (root != nullptr) {
      for (int a = 0; a < 3; ++a) root[a] = plan->root_centre[a];
      root[3] = plan->root_half_width;
    }
    const size_t ns = static_cast<size_t>(plan->ns), nt = static_cast<size_t>(plan->nt);
    const size_t nl = static_cast<size_t>(plan->n_leaves) + 1;
    if (leaf_source_offsets) std::memcpy(leaf_source_offsets, plan->h_src_off.data(), nl * sizeof(int32_t));
    if (leaf_target_offsets) std::memcpy(leaf_target_offsets, plan->h_tgt_off.data(), nl * sizeof(int32_t));
    check(cudaDeviceSynchronize(), "sync");
    if (source_permutation && ns)
      check(cudaMemcpy(source_permutation, plan->src_perm, ns * sizeof(int32_t), cudaMemcpyDeviceToHost), "D2H");
    if (target_permutation && nt)
      check(cudaMemcpy(target_permutation, plan->tgt_perm, nt * sizeof(int32_t), cudaMemcpyDeviceToHost), "D2H");
    if (sorted_source_positions && ns)
      check(cudaMemcpy(sorted_source_positions, plan->src_pos64, 3 * ns * sizeof(double), cudaMemcpyDeviceToHost),
            "D2H");
    if (sorted_target_positions && nt)
      check(cudaMemcpy(sorted_target_positions, plan->tgt_pos64, 3 * nt * sizeof(double), cudaMemcpyDeviceToHost),
            "D2H");
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(plan, e.code, e.what());
  }
}

void cdfmm_b200_plan_destroy(cdfmm_b200_plan *plan) {
  if (plan == nullptr) return;
  cudaSetDevice(plan->device);
  cudaDeviceSynchronize();
  free_plan(plan);
}

int cdfmm_b200_set_source_cuboids(cdfmm_b200_plan *plan, const double *sizes, int32_t count, int32_t cuboid_p2m) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  try {
    require(count == 0 || count == 1 || count == plan->ns, "cuboid sizes must contain one or one per source");
    require(count == 0 || sizes != nullptr, "sizes must not be NULL");
    for (int64_t i = 0; i < 3 * static_cast<int64_t>(count); ++i)
      require(std::isfinite(sizes[i]) && sizes[i] > 0.0, "source cuboid dimensions must be positive");
    check(cudaSetDevice(plan->device), "cudaSetDevice");
    check(cudaDeviceSynchronize(), "sync");
    uint64_t &bytes = plan->stats.persistent_device_bytes;
    for (void *q : {static_cast<void *>(plan->src_size), static_cast<void *>(plan->src_size64),
                    static_cast<void *>(plan->cuboid_T), static_cast<void *>(plan->cuboid_base)})
      if (q != nullptr) cudaFree(q);
    plan->src_size = nullptr;
    plan->src_size64 = nullptr;
    plan->cuboid_T = nullptr;
    plan->cuboid_base = nullptr;
    bytes -= std::min(bytes, plan->cuboid_T_bytes);
    plan->cuboid_T_bytes = 0;
    plan->cuboid = false;
    plan->cuboid_p2m = false;
    if (count == 0) return CDFMM_B200_OK;

    // side lengths in sorted order, normalised by the root width
    const int m = count == 1 ? 1 : plan->ns;
    std::vector<int> perm(static_cast<size_t>(plan->ns));
    if (count > 1 && plan->ns > 0)
      check(cudaMemcpy(perm.data(), plan->src_perm, sizeof(int) * perm.size(), cudaMemcpyDeviceToHost), "D2H");
    const double inv = 1.0 / plan->scale;
    std::vector<double> h64(3 * static_cast<size_t>(m));
    std::vector<float4> h32(static_cast<size_t>(m));
    for (int j = 0; j < m; ++j) {
      const size_t u = count == 1 ? 0 : static_cast<size_t>(perm[static_cast<size_t>(j)]);
      for (int c = 0; c < 3; ++c) h64[3 * static_cast<size_t>(j) + c] = sizes[3 * u + c] * inv;
      h32[static_cast<size_t>(j)] = make_float4(static_cast<float>(h64[3 * j]), static_cast<float>(h64[3 * j + 1]),
                                                static_cast<float>(h64[3 * j + 2]), 0.0F);
    }
    // pair tensors of the near-field work units
    std::vector<int4> work(static_cast<size_t>(plan->n_p2p_work));
    if (!work.empty())
      check(cudaMemcpy(work.data(), plan->p2p_work, sizeof(int4) * work.size(), cudaMemcpyDeviceToHost), "D2H");
    const std::vector<long long> sources = cuboid_unit_sources(plan->h_src_off.data(), work, plan->depth);
    std::vector<long long> base(work.size() + 1, 0);
    for (size_t u = 0; u < work.size(); ++u) base[u + 1] = base[u] + 6 * sources[u] * work[u].z;
    const uint64_t tensor_bytes = sizeof(float) * static_cast<uint64_t>(base.back());
    size_t free_b = 0, total_b = 0;
    check(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    if (tensor_bytes > free_b / 10 * 9)
      throw AbiError(CDFMM_B200_ERR_OUT_OF_MEMORY,
                     "the cuboid near-field pair tensors need " + std::to_string(tensor_bytes >> 20) + " MiB (" +
                         std::to_string(free_b >> 20) + " MiB free)");
    uint64_t added = 0;
    plan->src_size = dalloc<float4>(h32.size(), added);
    plan->src_size64 = dalloc<double>(h64.size(), added);
    plan->cuboid_base = dalloc<long long>(base.size(), added);
    plan->cuboid_T = dalloc<float>(static_cast<size_t>(base.back()), added);
    upload(plan->src_size, h32.data(), h32.size(), plan->stats.setup_h2d_bytes);
    upload(plan->src_size64, h64.data(), h64.size(), plan->stats.setup_h2d_bytes);
    upload(plan->cuboid_base, base.data(), base.size(), plan->stats.setup_h2d_bytes);
    launch_cuboid_tensors(plan->p2p_work, plan->n_p2p_work, plan->cuboid_base, plan->src_off, plan->depth,
                          plan->src_pos64, plan->tgt_pos64, inv, plan->src_size64, count == 1 ? 0 : 1,
                          plan->cuboid_T, nullptr);
    check(cudaGetLastError(), "cuboid tensors");
    check(cudaDeviceSynchronize(), "cuboid tensors");
    plan->cuboid_T_bytes = added;
    bytes += added;
    plan->size_step = count == 1 ? 0 : 1;
    plan->cuboid = true;
    plan->cuboid_p2m = cuboid_p2m != 0;
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(plan, e.code, e.what());
  } catch (const std::bad_alloc &) {
    return fail(plan, CDFMM_B200_ERR_OUT_OF_MEMORY, "host allocation failed");
  }
}

int cdfmm_b200_set_self_indices(cdfmm_b200_plan *plan, const int32_t *sorted_self) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  try {
    check(cudaSetDevice(plan->device), "cudaSetDevice");
    plan->self_version += 1;
    if (sorted_self == nullptr) {
      plan->has_self = false;
      plan->h_self.clear();
      return CDFMM_B200_OK;
    }
    for (int i = 0; i < plan->nt; ++i)
      require(sorted_self[i] >= -1 && sorted_self[i] < plan->ns, "self index out of range");
    check(cudaDeviceSynchronize(), "sync");
    if (plan->nt > 0)
      copy_to_device(plan->self_idx, sorted_self, sizeof(int) * plan->nt, "cudaMemcpy");
    {
      // per leaf: the lowest and highest self source of its targets
      std::vector<int2> range(static_cast<size_t>(plan->n_leaves), make_int2(0x7fffffff, -1));
      for (int m = 0; m < plan->n_leaves; ++m)
        for (int i = plan->h_tgt_off[static_cast<size_t>(m)]; i < plan->h_tgt_off[static_cast<size_t>(m) + 1]; ++i)
          if (sorted_self[i] >= 0) {
            int2 &r = range[static_cast<size_t>(m)];
            r.x = std::min(r.x, sorted_self[i]);
            r.y = std::max(r.y, sorted_self[i]);
          }
      copy_to_device(plan->leaf_self, range.data(), sizeof(int2) * range.size(), "cudaMemcpy");
    }
    plan->h_self.assign(sorted_self, sorted_self + plan->nt);
    plan->has_self = true;
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(plan, e.code, e.what());
  }
}

// Tensor-core M2L work tiles: per level (deepest first), runs of
// T = m_tiles * (128 / Kp) consecutive parents in Morton order, the 8 parity
// classes of a run adjacent so that CTAs running together read the same
// source boxes (the run's parents' neighbours' children) from L2.
static std::vector<int4> build_tc_tiles(int depth, int T) {
  std::vector<int4> tiles;
  for (int level = depth; level >= 2; --level) {
    const int parents = 1 << (3 * (level - 1));
    for (int p0 = 0; p0 < parents; p0 += T)
      for (int cls = 0; cls < 8; ++cls) tiles.push_back(make_int4(level, cls, p0, std::min(T, parents - p0)));
  }
  return tiles;
}

static void upload_tc_tiles(cdfmm_b200_plan *plan, int Kp) {
  const std::vector<int4> tiles = build_tc_tiles(plan->depth, plan->tc_m_tiles * (128 / Kp));
  grow(plan->tc_tiles, plan->tc_tiles_capacity, tiles.size(), "cudaMalloc tiles");
  copy_to_device(plan->tc_tiles, tiles.data(), tiles.size() * sizeof(int4), "tiles");
  plan->tc_tiles_Kp = Kp;
  plan->tc_n_tiles = static_cast<int>(tiles.size());
}

// Autotuner of the tensor-core M2L pipeline shape (accumulators per CTA,
// stages, fused hi/lo B operand): times every candidate on this call's
// packed operands (device events, second of two launches) and keeps the
// fastest.  Candidates trade B reuse (more accumulators per CTA) against
// pipeline depth, CTAs per SM and MMA size.  Shapes with the same fusion
// give bit-identical results (the per-row MMA sequence is the same); the
// fused form sums the hi*lo product in its own accumulator, a difference at
// FP32 rounding level.
static void tune_m2l_tc(cdfmm_b200_plan *plan, int K, cudaStream_t s, size_t smem_budget) {
  const int Kp = round_up(K, 8);
  const int node_base = level_offset(2);
  TcArgs ta{};
  ta.a_hi = static_cast<const uint8_t *>(plan->tc_a_hi);
  ta.a_lo = static_cast<const uint8_t *>(plan->tc_a_lo);
  ta.b_tiles = static_cast<const uint8_t *>(plan->tc_b); set_m2l_reduction(ta, plan);
  ta.scale_l = plan->scale_l;
  ta.L = plan->L;
  ta.error_flag = plan->error_flag;
  ta.n = plan->n;
  ta.K = K;
  ta.Kp = Kp;
  ta.Kpad = plan->tc_Kpad;
  ta.Npad = plan->tc_Npad;
  ta.node_base = node_base;
  ta.zero_node = plan->n_nodes - node_base;
  ta.box_bytes = static_cast<uint32_t>(Kp) * static_cast<uint32_t>(plan->tc_Kpad) * 2u;
  ta.wait_limit = plan->tc_wait_limit;
  float best = 0.0F;
  int best_i = -1;
  // candidates within the budget (all of them if none fits)
  auto launch_smem = [&](const cdfmm_b200_plan::TcShape &c) {
    const int acc = round_up(c.fuse ? 2 * plan->tc_Npad : plan->tc_Npad, 32);
    size_t b = m2l_tc_smem_bytes(plan->tc_Npad, c.m_tiles, c.stages, plan->n);
    if (tmem_columns(c.m_tiles, acc) > 256) b = std::max<size_t>(b, 120 * 1024);
    return b;
  };
  bool any_fits = false;
  for (const cdfmm_b200_plan::TcShape &c : plan->tc_candidates) any_fits = any_fits || launch_smem(c) <= smem_budget;

  for (size_t c = 0; c < plan->tc_candidates.size(); ++c) {
    if (any_fits && launch_smem(plan->tc_candidates[c]) > smem_budget) continue;
    const int mt = plan->tc_candidates[c].m_tiles;
    const std::vector<int4> tiles = build_tc_tiles(plan->depth, mt * (128 / Kp));
    grow(plan->tc_tiles, plan->tc_tiles_capacity, tiles.size(), "cudaMalloc tiles");
    copy_to_device(plan->tc_tiles, tiles.data(), tiles.size() * sizeof(int4), "tiles");
    ta.tiles = plan->tc_tiles;
    ta.m_tiles = mt;
    ta.stages = plan->tc_candidates[c].stages;
    ta.fuse_n = plan->tc_candidates[c].fuse;
    ta.acc_stride = round_up(ta.fuse_n ? 2 * plan->tc_Npad : plan->tc_Npad, 32);
    ta.tmem_cols = tmem_columns(mt, ta.acc_stride);
    // one warm-up launch, then the faster of two timed ones (single timings
    // of neighbouring shapes differ by less than their run-to-run noise)
    float ms = 0.0F;
    for (int rep = 0; rep < 3; ++rep) {
      check(cudaEventRecord(plan->ev_t[10], s), "event");
      launch_m2l_tc(ta, static_cast<int>(tiles.size()), s);
      check(cudaEventRecord(plan->ev_t[11], s), "event");
      check(cudaEventSynchronize(plan->ev_t[11]), "autotune");
      float t = 0.0F;
      check(cudaEventElapsedTime(&t, plan->ev_t[10], plan->ev_t[11]), "event");
      if (rep == 1 || (rep > 1 && t < ms)) ms = t;
    }
    if (best_i < 0 || ms < best) {
      best = ms;
      best_i = static_cast<int>(c);
    }
  }
  const cdfmm_b200_plan::TcShape &best_shape = plan->tc_candidates[static_cast<size_t>(best_i)];
  plan->tc_m_tiles = best_shape.m_tiles;
  plan->tc_stages = best_shape.stages;
  plan->tc_fuse = best_shape.fuse;
  plan->tc_acc_stride = round_up(best_shape.fuse ? 2 * plan->tc_Npad : plan->tc_Npad, 32);
  plan->tc_tmem_cols = tmem_columns(plan->tc_m_tiles, plan->tc_acc_stride);
  plan->tc_tiles_Kp = 0; // rebuilt for the chosen shape by the caller
}

// Upward pass for K states whose sorted, scaled moments are in plan->mom:
// P2M and M2M, leaving the multipoles in plan->M.  Returns the launch count.
// With `ntc` (the tensor-core near field's moment blocks, packed for these
// K states) the leaf multipoles run on the tensor cores where they can.
static int enqueue_upward(cdfmm_b200_plan *plan, int K, cudaStream_t s, bool timing,
                          const NearTcLaunch *ntc = nullptr) {
  const int n = plan->n;
  int launches = 0;
  if (ntc != nullptr && plan->p2m_tc_ok && !plan->cuboid_p2m && p2m_tc_supported(n, K))
    launch_p2m_tc(*ntc, plan->basis, plan->M, n, plan->p, K, plan->depth, s);
  else
    launch_p2m(plan->src_rel, plan->mom, plan->src_off, plan->basis, plan->M, n, plan->p, K, plan->depth,
               plan->p2m_chunk, s, plan->cuboid_p2m ? plan->src_size : nullptr, plan->size_step);
  ++launches;
  if (timing) check(cudaEventRecord(plan->ev_t[2], s), "event");
  for (int level = plan->depth - 1; level >= 0; --level) {
    launch_m2m(plan->M, plan->m2m_off, plan->m2m_pair, plan->m2m_coef, n, K, level,
               static_cast<int>(plan->ops.m2m_pair_g.size()), s);
    ++launches;
  }
  if (timing) check(cudaEventRecord(plan->ev_t[3], s), "event");
  return launches;
}

static CloseGeometry close_geometry(const cdfmm_b200_plan *plan) { return cdfmm_b200_near_geometry(plan); }

// Whether K states take the tensor-core M2L.
static bool m2l_on_tensor_cores(const cdfmm_b200_plan *plan, int K) {
  return plan->depth >= 2 && plan->tc_supported && K <= 128 &&
         (plan->m2l_mode == CDFMM_B200_M2L_BF16X3 || plan->m2l_mode == CDFMM_B200_M2L_AUTO);
}

// Whether an evaluation of K states takes the tensor-core near field.
static bool near_on_tensor_cores(const cdfmm_b200_plan *plan, int K) {
  return plan->ntc_supported && plan->near_mode != CDFMM_B200_NEAR_FP32 && K >= kNearTcMinStates &&
         K <= kNearTcMaxStates && !plan->cuboid && plan->n_p2p_work > 0;
}

// Blocks, work units and operand buffers of the tensor-core near field
// (once per plan, on first use).
static void ensure_near_tc(cdfmm_b200_plan *plan) {
  if (plan->ntc_built) return;
  const NearTcLayout lay = near_tc_layout(plan->h_src_off.data(), plan->h_tgt_off.data(), plan->depth);
  uint64_t bytes = 0, h2d = 0;
  plan->ntc_blk_off = dalloc<int>(lay.blk_off.size(), bytes);
  upload(plan->ntc_blk_off, lay.blk_off.data(), lay.blk_off.size(), h2d);
  plan->ntc_blk_src = dalloc<int>(lay.blk_src.size(), bytes);
  upload(plan->ntc_blk_src, lay.blk_src.data(), lay.blk_src.size(), h2d);
  plan->ntc_blk_pos = dalloc<float4>(lay.blk_src.size(), bytes);
  plan->ntc_work = dalloc<int4>(lay.work.size(), bytes);
  upload(plan->ntc_work, lay.work.data(), lay.work.size(), h2d);
  const size_t ob = near_tc_operand_bytes(lay.n_blocks, std::min(plan->max_states, kNearTcMaxStates));
  plan->ntc_b = dalloc<uint8_t>(ob, bytes);
  launch_near_tc_positions(plan->src_rel, plan->ntc_blk_src, lay.n_blocks, plan->ntc_blk_pos, plan->stream);
  check(cudaGetLastError(), "kernel launch");
  check(cudaStreamSynchronize(plan->stream), "near-field blocks");
  plan->ntc_n_blocks = lay.n_blocks;
  plan->ntc_n_work = static_cast<int>(lay.work.size());
  plan->stats.near_tc_k_cols = lay.k_cols;
  plan->stats.persistent_device_bytes += bytes;
  plan->stats.setup_h2d_bytes += h2d;
  plan->ntc_built = true;
}

// Blocks of 16 sources and the operand buffer of the tensor-core position
// gradient (once per plan, on first use; its work units are the forward's).
static void ensure_near_grad_tc(cdfmm_b200_plan *plan) {
  ensure_near_tc(plan);
  if (plan->ngt_built) return;
  const NearGradLayout lay = near_grad_layout(plan->h_src_off.data(), plan->depth);
  uint64_t bytes = 0, h2d = 0;
  plan->ngt_blk_off = dalloc<int>(lay.blk_off.size(), bytes);
  upload(plan->ngt_blk_off, lay.blk_off.data(), lay.blk_off.size(), h2d);
  plan->ngt_blk_src = dalloc<int>(lay.blk_src.size(), bytes);
  upload(plan->ngt_blk_src, lay.blk_src.data(), lay.blk_src.size(), h2d);
  plan->ngt_blk_pos = dalloc<float4>(lay.blk_src.size(), bytes);
  plan->ngt_b = dalloc<uint8_t>(near_grad_operand_bytes(lay.n_blocks, std::min(plan->max_states, kNearTcMaxStates)),
                                bytes);
  launch_near_grad_positions(plan->src_rel, plan->ngt_blk_src, lay.n_blocks, plan->ngt_blk_pos, plan->stream);
  check(cudaGetLastError(), "kernel launch");
  check(cudaStreamSynchronize(plan->stream), "near-field gradient blocks");
  plan->ngt_n_blocks = lay.n_blocks;
  plan->stats.persistent_device_bytes += bytes;
  plan->stats.setup_h2d_bytes += h2d;
  plan->ngt_built = true;
}

static NearTcLaunch near_tc_launch(const cdfmm_b200_plan *plan) {
  NearTcLaunch l{};
  l.blk_pos = plan->ntc_blk_pos;
  l.blk_off = plan->ntc_blk_off;
  l.blk_src = plan->ntc_blk_src;
  l.n_blocks = plan->ntc_n_blocks;
  l.work = plan->ntc_work;
  l.n_work = plan->ntc_n_work;
  l.b_ops = plan->ntc_b;
  l.error_flag = plan->error_flag;
  l.wait_limit = plan->tc_wait_limit;
  return l;
}

// Near/far schedule of one evaluation (cdfmm_b200_set_schedule): the
// co-resident schedule needs the tensor-core M2L (whose CTA fits beside two
// co-resident near-field CTAs) and runs only on request; AUTO and every
// other evaluation run SEPARATE.  (With the traceless M2L, a third of the
// full-basis one, overlapping it no longer repays the co-resident near
// field's smaller CTAs: at N = 1M, p = 6, K = 64 with the FP32 near field,
// 43.5 ms SEPARATE against 46.7 ms CORUN.)
static int resolved_schedule(const cdfmm_b200_plan *plan, int K) {
  // cuboid sources and the tensor-core near field: no co-resident form
  if (K <= 1 || !m2l_on_tensor_cores(plan, K) || plan->cuboid || near_on_tensor_cores(plan, K))
    return CDFMM_B200_SCHEDULE_SEPARATE;
  return plan->schedule == CDFMM_B200_SCHEDULE_CORUN ? CDFMM_B200_SCHEDULE_CORUN : CDFMM_B200_SCHEDULE_SEPARATE;
}

// Shared memory one tensor-core M2L CTA may use to sit beside two
// co-resident near-field CTAs on one SM.
static size_t corun_m2l_smem_budget(const cdfmm_b200_plan *plan, int K) {
  int per_sm = 0, reserved = 0;
  cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, plan->device);
  cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, plan->device);
  const size_t near = p2p_corun_cta_smem(K) + static_cast<size_t>(reserved);
  const size_t used = 2 * near + static_cast<size_t>(reserved);
  return static_cast<size_t>(per_sm) > used ? static_cast<size_t>(per_sm) - used : 0;
}

// Tensor-core M2L operands: packs the scaled multipoles into BF16 hi/lo boxes
// and, on the first use for this K (or after a schedule change), chooses the
// pipeline shape -- the fastest candidate whose shared memory fits beside
// the co-resident near field when K states run CORUN -- and builds its work
// tiles.  Every path of the plan (device or host arrays, backward) then
// uses that shape.  Returns the launch count.
static int prepare_m2l(cdfmm_b200_plan *plan, int K, cudaStream_t s) {
  if (!m2l_on_tensor_cores(plan, K)) return 0;
  const size_t smem_budget =
      resolved_schedule(plan, K) == CDFMM_B200_SCHEDULE_CORUN ? corun_m2l_smem_budget(plan, K) : SIZE_MAX;
  const int Kp = round_up(K, 8);
  const int node_base = level_offset(2);
  const int boxes = plan->n_nodes - node_base;
  launch_m2l_pack(plan->M, plan->scale_m, plan->tc_fold_off, plan->tc_fold, plan->tc_n_in, plan->tc_a_hi, plan->tc_a_lo,
                  plan->n, K, Kp, plan->tc_Kpad,
                  plan->depth, node_base, boxes, s);
  if (plan->tc_tiles_Kp != Kp || (!plan->tc_pinned && plan->tc_tuned_budget != smem_budget)) {
    check(cudaStreamSynchronize(s), "sync");
    if (plan->tc_candidates.size() > 1 && !plan->tc_pinned) tune_m2l_tc(plan, K, s, smem_budget);
    plan->tc_tuned_budget = smem_budget;
    upload_tc_tiles(plan, Kp);
  }
  return 1;
}

// Downward pass: M2L (tensor cores or FP32 SIMT) and L2L, leaving the leaf
// local expansions in plan->L.  prepared: prepare_m2l already ran for this
// evaluation.  Returns the launch count.
static int enqueue_downward(cdfmm_b200_plan *plan, int K, cudaStream_t s, bool timing, bool prepared = false) {
  const int n = plan->n;
  int launches = 0;
    const bool use_tc = m2l_on_tensor_cores(plan, K);
    if (use_tc) {
      if (!prepared) launches += prepare_m2l(plan, K, s);
      const int Kp = round_up(K, 8);
      const int node_base = level_offset(2);
      const int boxes = plan->n_nodes - node_base;
      TcArgs ta{};
      ta.a_hi = static_cast<const uint8_t *>(plan->tc_a_hi);
      ta.a_lo = static_cast<const uint8_t *>(plan->tc_a_lo);
      ta.b_tiles = static_cast<const uint8_t *>(plan->tc_b); set_m2l_reduction(ta, plan);
      ta.tiles = plan->tc_tiles;
      ta.scale_l = plan->scale_l;
      ta.L = plan->L;
      ta.error_flag = plan->error_flag;
      ta.n = n;
      ta.K = K;
      ta.Kp = Kp;
      ta.Kpad = plan->tc_Kpad;
      ta.Npad = plan->tc_Npad;
      ta.node_base = node_base;
      ta.zero_node = boxes;
      ta.stages = plan->tc_stages;
      ta.m_tiles = plan->tc_m_tiles;
      ta.acc_stride = plan->tc_acc_stride;
      ta.fuse_n = plan->tc_fuse;
      ta.tmem_cols = plan->tc_tmem_cols;
      ta.box_bytes = static_cast<uint32_t>(Kp) * static_cast<uint32_t>(plan->tc_Kpad) * 2u;
      ta.wait_limit = plan->tc_wait_limit;
      launch_m2l_tc(ta, plan->tc_n_tiles, s);
      launches += 1;
      plan->stats.m2l_tc_m_tiles = plan->tc_m_tiles;
      plan->stats.m2l_tc_stages = plan->tc_stages;
      plan->stats.m2l_tc_fused = plan->tc_fuse;
    } else if (plan->depth >= 2) {
      launch_m2l_simt(plan->M, plan->m2l_fold_buf, plan->L, plan->m2l_T, plan->scale_m, plan->scale_l,
                      plan->m2l_tiles, plan->n_tiles, n, plan->m2l_ld_red, K, plan->depth, plan->tc_fold_off,
                      plan->tc_fold, plan->tc_expand, plan->tc_n_in, plan->tc_n_out, plan->tc_n_derived, s);
      ++launches;
    }
    plan->last_m2l_tc = use_tc;
    if (timing) check(cudaEventRecord(plan->ev_t[4], s), "event");
    for (int level = 3; level <= plan->depth; ++level) {
      launch_l2l(plan->L, plan->l2l_off, plan->l2l_pair, plan->l2l_coef, n, K, level,
                 static_cast<int>(plan->ops.l2l_pair_g.size()), s);
      ++launches;
    }
  return launches;
}

// Upward and downward far-field passes (P2M, M2M, M2L, L2L).
static int enqueue_far(cdfmm_b200_plan *plan, int K, cudaStream_t s, bool timing) {
  const int launches = enqueue_upward(plan, K, s, timing);
  return launches + enqueue_downward(plan, K, s, timing);
}


// Enqueues one evaluation of K states on stream s: device-resident moments
// ([K][ns][3], dtype) -> gather -> (list-1 P2P on the near stream || P2M, M2M,
// M2L, L2L) -> L2P + combine + unsort into device results.  Returns the
// kernel launch count.
static int enqueue_evaluation(cdfmm_b200_plan *plan, const void *moments, int dtype, int K, unsigned output,
                              int layout, float *field, float *potential, cudaStream_t s, bool timing) {
  const bool want_phi = (output & CDFMM_B200_OUTPUT_POTENTIAL) != 0u;
  int launches = 0;
  if (timing) check(cudaEventRecord(plan->ev_t[0], s), "event");
  if (plan->trace && !timing) check(cudaEventRecord(plan->ev_t[kTraceBegin], s), "event");
  launch_gather_moments(moments, dtype, plan->src_inv, plan->ns, K, plan->scale, plan->mom, s, moments_paired(K));
  launches += plan->ns > 0 ? 1 : 0;
  if (timing) check(cudaEventRecord(plan->ev_t[1], s), "event");

  // Near field on its own stream, concurrent with the far field.  With
  // stage timing enabled it runs first on the main stream instead, so that
  // each stage's events measure that stage alone.
  //   SEPARATE: the full-size near-field kernel (two CTAs fill an SM) beside
  //     the far field on a high-priority stream (which in practice takes
  //     most SMs while it runs: the two share the GPU by turns);
  //   CORUN: P2M, M2M and the M2L operand pack run first on all SMs; then
  //     the co-resident near-field form on the high-priority stream -- two
  //     of its CTAs per SM, which leave room for exactly one tensor-core M2L
  //     CTA -- beside M2L and L2L on a normal-priority stream, so an M2L CTA
  //     only ever takes the slot the near field leaves free and the FP32
  //     near field and the tensor-core far field run side by side on every
  //     SM (the M2L's pipeline shape is chosen among those that fit there).
  const int schedule = timing ? CDFMM_B200_SCHEDULE_SEPARATE : resolved_schedule(plan, K);
  const bool corun = schedule == CDFMM_B200_SCHEDULE_CORUN;
  const bool trace = plan->trace && !timing;
  cudaStream_t ns = timing ? s : (corun ? plan->far_stream : plan->near_stream);
  cudaStream_t fs = timing ? s : (corun ? plan->near_stream : plan->far_stream);
  if (corun) {
    if (trace) check(cudaEventRecord(plan->ev_t[kTraceFarBegin], s), "event");
    launches += enqueue_upward(plan, K, s, false);
    launches += prepare_m2l(plan, K, s);
  }
  // Tensor-core near field: its moment blocks are packed once, before the
  // streams fork, for the near field and the tensor-core P2M (on the far
  // stream) alike; with stage timing the pack counts as near-field time.
  const bool near_tc = near_on_tensor_cores(plan, K);
  if (near_tc) ensure_near_tc(plan);
  NearTcLaunch near_tc_args = near_tc_launch(plan);
  near_tc_args.packed = near_tc;
  if (near_tc && !timing) {
    launch_near_tc_pack(near_tc_args, plan->mom, K, s);
    ++launches;
  }
  if (!timing) {
    check(cudaEventRecord(plan->ev_fork, s), "event");
    check(cudaStreamWaitEvent(ns, plan->ev_fork, 0), "wait");
    check(cudaStreamWaitEvent(fs, plan->ev_fork, 0), "wait");
  }
  if (timing) check(cudaEventRecord(plan->ev_t[8], ns), "event");
  if (trace) check(cudaEventRecord(plan->ev_t[kTraceP2pBegin], ns), "event");
  if (near_tc && timing) {
    launch_near_tc_pack(near_tc_args, plan->mom, K, ns);
    ++launches;
  }
  // Inside a batch graph the K = 1 near field takes the uncapped units
  // (same results bit for bit: a K = 1 target's sum does not depend on how
  // its leaf is cut into units).
  const bool wide = plan->in_batch && K == 1;
  const CorunLaunch corun_launch{2 * plan->sm_count, plan->p2p_next_unit};
  launch_p2p(plan->src_rel, plan->mom, plan->src_off, plan->tgt_rel, wide ? plan->p2p_work_wide : plan->p2p_work,
             wide ? plan->n_p2p_work_wide : plan->n_p2p_work, plan->has_self ? plan->self_idx : nullptr,
             plan->leaf_self, close_geometry(plan), plan->depth, K, want_phi, plan->near, ns, 0, -1, 0, 1.0F,
             corun ? &corun_launch : nullptr, near_tc ? &near_tc_args : nullptr);
  plan->stats.near_tc_last = near_tc ? 1 : 0;
  ++launches;
  if (timing) check(cudaEventRecord(plan->ev_t[9], ns), "event");
  if (trace) check(cudaEventRecord(plan->ev_t[kTraceP2pEnd], ns), "event");
  if (timing) check(cudaEventRecord(plan->ev_t[1], s), "event");
  if (!timing) check(cudaEventRecord(plan->ev_join, ns), "event");

  // far field
  if (corun) {
    if (trace) check(cudaEventRecord(plan->ev_t[kTraceM2lBegin], fs), "event");
    launches += enqueue_downward(plan, K, fs, false, true);
  } else {
    if (trace) check(cudaEventRecord(plan->ev_t[kTraceFarBegin], fs), "event");
    launches += enqueue_upward(plan, K, fs, timing, near_tc ? &near_tc_args : nullptr);
    if (trace) check(cudaEventRecord(plan->ev_t[kTraceM2lBegin], fs), "event");
    launches += enqueue_downward(plan, K, fs, timing);
  }
  if (trace) check(cudaEventRecord(plan->ev_t[kTraceFarEnd], fs), "event");
  plan->last_schedule = schedule;
  if (timing) check(cudaEventRecord(plan->ev_t[5], s), "event");
  if (!timing) {
    check(cudaEventRecord(plan->ev_far, fs), "event");
    check(cudaStreamWaitEvent(s, plan->ev_far, 0), "wait");
    check(cudaStreamWaitEvent(s, plan->ev_join, 0), "wait");
  }
  if (timing) check(cudaEventRecord(plan->ev_t[6], s), "event");
  launch_l2p(plan->L, plan->tgt_rel, plan->tgt_off, plan->tgt_perm, plan->tgt_inv, plan->near, plan->basis, plan->n,
             plan->p, K, plan->nt, plan->depth, output, layout, plan->phi_scale, field, potential, s);
  launches += (K >= 4 && plan->nt > 0) ? 2 : 1;
  check(cudaGetLastError(), "kernel launch");
  if (timing) check(cudaEventRecord(plan->ev_t[7], s), "event");
  if (trace) check(cudaEventRecord(plan->ev_t[kTraceEnd], s), "event");
  return launches;
}

void cdfmm_b200_stacked_upward(cdfmm_b200_plan *plan, const cdfmm_b200_eval_args *a, cudaStream_t s) {
  const bool want_phi = (a->output & CDFMM_B200_OUTPUT_POTENTIAL) != 0u;
  ++plan->call_seq;
  launch_gather_moments(a->moments, a->moments_dtype, plan->src_inv, plan->ns, 1, plan->scale, plan->mom, s, false);
  check(cudaEventRecord(plan->ev_fork, s), "event");
  check(cudaStreamWaitEvent(plan->near_stream, plan->ev_fork, 0), "wait");
  // inside a batch graph: the uncapped work units (see enqueue_evaluation)
  launch_p2p(plan->src_rel, plan->mom, plan->src_off, plan->tgt_rel, plan->p2p_work_wide, plan->n_p2p_work_wide,
             plan->has_self ? plan->self_idx : nullptr, plan->leaf_self, close_geometry(plan), plan->depth, 1, want_phi,
             plan->near, plan->near_stream);
  check(cudaEventRecord(plan->ev_join, plan->near_stream), "event");
  enqueue_upward(plan, 1, s, false);
  check(cudaGetLastError(), "kernel launch");
}

void cdfmm_b200_stacked_downward(cdfmm_b200_plan *plan, const cdfmm_b200_eval_args *a, cudaStream_t s) {
  for (int level = 3; level <= plan->depth; ++level)
    launch_l2l(plan->L, plan->l2l_off, plan->l2l_pair, plan->l2l_coef, plan->n, 1, level,
               static_cast<int>(plan->ops.l2l_pair_g.size()), s);
  check(cudaStreamWaitEvent(s, plan->ev_join, 0), "wait");
  launch_l2p(plan->L, plan->tgt_rel, plan->tgt_off, plan->tgt_perm, plan->tgt_inv, plan->near, plan->basis, plan->n,
             plan->p, 1, plan->nt, plan->depth, a->output, a->layout, plan->phi_scale, a->field, a->potential, s);
  check(cdfmm_b200_collect_status(plan, s, plan->call_seq), "status kernel launch");
  check(cudaGetLastError(), "kernel launch");
  plan->last_m2l_tc = true;
  plan->last_schedule = CDFMM_B200_SCHEDULE_SEPARATE;
  plan->exp_state0 = 0;
  plan->last_K = 1;
  plan->stats.evaluations += 1;
}

int cdfmm_b200_evaluate(cdfmm_b200_plan *plan, const cdfmm_b200_eval_args *a) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  try {
    require(a != nullptr, "args is NULL");
    require(a->n_states >= 1 && a->n_states <= plan->max_states, "n_states must be in [1, max_states]");
    require(a->moments_dtype == 0 || a->moments_dtype == 1, "moments_dtype must be 0 (float32) or 1 (float64)");
    require((a->output & 3u) != 0u && (a->output & ~3u) == 0u, "output must request potential and/or field");
    require(a->layout == CDFMM_B200_LAYOUT_SEPARATE || a->layout == CDFMM_B200_LAYOUT_INTERLEAVED, "unknown layout");
    require(plan->ns == 0 || a->moments != nullptr, "moments is NULL");
    const bool want_phi = (a->output & CDFMM_B200_OUTPUT_POTENTIAL) != 0u;
    const bool want_h = (a->output & CDFMM_B200_OUTPUT_FIELD) != 0u;
    if (a->layout == CDFMM_B200_LAYOUT_INTERLEAVED || want_h) require(plan->nt == 0 || a->field != nullptr, "field is NULL");
    if (a->layout == CDFMM_B200_LAYOUT_SEPARATE && want_phi) require(plan->nt == 0 || a->potential != nullptr, "potential is NULL");
    if (a->layout == CDFMM_B200_LAYOUT_INTERLEAVED && (a->memory & CDFMM_B200_RESULTS_ON_HOST) == 0u)
      require(reinterpret_cast<uintptr_t>(a->field) % 16 == 0, "interleaved device results need a 16-byte aligned field pointer");
    if ((a->memory & CDFMM_B200_MOMENTS_ON_HOST) == 0u)
      require(reinterpret_cast<uintptr_t>(a->moments) % (a->moments_dtype == 1 ? 8 : 4) == 0, "misaligned moments pointer");
    check(cudaSetDevice(plan->device), "cudaSetDevice");
    // A launch error reported below must come from these launches, not from
    // an earlier unrelated runtime call of the host process.
    (void)cudaGetLastError();

    const int K = a->n_states;
    const unsigned long long call = ++plan->call_seq;
    // NULL is the legacy default stream, as everywhere in CUDA (a torch tensor
    // on the default stream and our kernels are then ordered).
    cudaStream_t s = static_cast<cudaStream_t>(a->stream);
    const bool host_in = (a->memory & CDFMM_B200_MOMENTS_ON_HOST) != 0u;
    const bool host_out = (a->memory & CDFMM_B200_RESULTS_ON_HOST) != 0u;
    const size_t in_state = static_cast<size_t>(plan->ns) * 3 * (a->moments_dtype == 1 ? 8 : 4);
    const int width = a->layout == CDFMM_B200_LAYOUT_INTERLEAVED ? 4 : 3;
    const size_t field_state = static_cast<size_t>(plan->nt) * sizeof(float) * width;
    const bool field_out = want_h || a->layout == CDFMM_B200_LAYOUT_INTERLEAVED;
    const size_t phi_state = (a->layout == CDFMM_B200_LAYOUT_SEPARATE && want_phi) ? static_cast<size_t>(plan->nt) * sizeof(float) : 0;
    const bool timing = plan->timing;
    // a concurrent trace is read back once the call's work is done
    bool traced = false;

    // Device staging of host arrays: [K][ns][3] moments; results field then potential.
    const char *moments = static_cast<const char *>(a->moments);
    if (host_in && in_state > 0) moments = grow_bytes(reinterpret_cast<char *&>(plan->stage_in), plan->stage_in_bytes, in_state * K, "cudaMalloc staging");
    char *field = reinterpret_cast<char *>(a->field);
    char *potential = reinterpret_cast<char *>(a->potential);
    if (host_out) {
      char *out = grow_bytes(reinterpret_cast<char *&>(plan->stage_out), plan->stage_out_bytes,
                             (field_state + phi_state) * K + 16, "cudaMalloc staging");
      field = out;
      potential = phi_state > 0 ? out + field_state * K : nullptr;
    }

    // Host arrays and many states: states are cut into 64-state chunks so
    // that the H2D copy of chunk c + 1 and the D2H copy of chunk c - 1 (on
    // their own streams) overlap the evaluation of chunk c.  Below 128 states
    // a call stays whole: per-state device time grows as chunks shrink (1.04,
    // 1.16, 1.48 ms per state at 64, 32, 16 states on the 1M-point p = 6
    // workload), which costs more than the copies the overlap would hide.
    const int chunk = ((host_in || host_out) && !timing && K >= 128) ? 64 : K;
    const int n_chunks = (K + chunk - 1) / chunk;
    // Host arrays and 32 <= K < 128 states: one evaluation of all K states
    // (the far field keeps its full batch) whose host copies overlap it part
    // by part.  The states are cut into parts of about a quarter of them (a
    // multiple of 8; the first part half as long, as its copy-in is exposed,
    // and the last the remainder); the copies run on their own streams and
    // the kernels in one explicit order on the caller's stream (stream
    // priorities alone let the later near-field parts delay the far field):
    //   gather 0, P2P 0, gather 1, P2P 1, ..., far field, L2P (all states),
    //   unsort 0, unsort 1, P2P 2 (adding to L2P's far field), unsort 2, ...
    // (the first n_parts / 2 P2P parts before the far field, while the later
    // moments are still being copied in; part j's results are copied out as
    // soon as its unsort is done, while later parts are computed).
    const bool parts = (host_in || host_out) && !timing && K >= 32 && n_chunks == 1 && plan->ns > 0 && plan->nt > 0;
    int launches = 0;
    if (parts) {
      // Parts of `part` states, the first one half as long (the first copy in
      // and the last copy out are the exposed ones): 8, 16, 16, 16, 8 for K = 64.
      const int part = round_up((K + 3) / 4, 8);
      std::vector<int> bounds = {0};
      for (int k = std::min(K, round_up(part / 2, 8)); ; k = std::min(K, k + part)) {
        bounds.push_back(k);
        if (k == K) break;
      }
      const int n_parts = static_cast<int>(bounds.size()) - 1;
      // P2P parts before the far field: as many as run while the later
      // moments are still being copied in (the far field, which needs them
      // all, then starts as early as possible, and so do the copies out)
      const int early = std::max(1, n_parts / 2);
      while (static_cast<int>(plan->io_events.size()) < 2 * n_parts + 2) {
        cudaEvent_t e;
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        plan->io_events.push_back(e);
      }
      const bool want_phi_p = (a->output & CDFMM_B200_OUTPUT_POTENTIAL) != 0u;
      cudaEvent_t ev_start = plan->io_events[0], ev_end = plan->io_events[1];
      check(cudaEventRecord(ev_start, s), "event");
      check(cudaStreamWaitEvent(plan->io_in, ev_start, 0), "wait");
      check(cudaStreamWaitEvent(plan->io_out, ev_start, 0), "wait");
      // P2P of part j: the early parts write the near field; the later
      // ones run after the (single) L2P and add theirs onto its far field.
      auto near_part = [&](int j, bool accumulate) {
        const int k0 = bounds[j], kc = bounds[j + 1] - bounds[j];
        launch_p2p(plan->src_rel, plan->mom, plan->src_off, plan->tgt_rel, plan->p2p_work, plan->n_p2p_work,
                   plan->has_self ? plan->self_idx : nullptr, plan->leaf_self, close_geometry(plan), plan->depth, K,
                   want_phi_p, plan->near, s, k0, k0 + kc,
                   accumulate ? ((a->output & CDFMM_B200_OUTPUT_FIELD) != 0u ? 1 : 2) : 0, plan->phi_scale);
        ++launches;
      };
      auto finish_part = [&](int j) {
        const int k0 = bounds[j], kc = bounds[j + 1] - bounds[j];
        launch_unsort(plan->near, plan->tgt_inv, plan->nt, K, a->output, a->layout, reinterpret_cast<float *>(field),
                      reinterpret_cast<float *>(potential), s, k0, k0 + kc);
        ++launches;
        if (host_out) check(cudaEventRecord(plan->io_events[3 + 2 * j], s), "event");
      };
      // Copies out are enqueued after every kernel: a copy into pageable host
      // memory returns only when it is done and must not hold back the
      // enqueueing of later parts' kernels.
      auto copy_out = [&](int j) {
        const int k0 = bounds[j], kc = bounds[j + 1] - bounds[j];
        check(cudaStreamWaitEvent(plan->io_out, plan->io_events[3 + 2 * j], 0), "wait");
        if (field_out && field_state > 0) {
          check(cudaMemcpyAsync(reinterpret_cast<char *>(a->field) + field_state * k0, field + field_state * k0,
                                field_state * kc, cudaMemcpyDeviceToHost, plan->io_out), "D2H field");
          plan->stats.evaluation_d2h_bytes += field_state * kc;
          plan->stats.evaluation_d2h_calls += 1;
        }
        if (phi_state > 0) {
          check(cudaMemcpyAsync(reinterpret_cast<char *>(a->potential) + phi_state * k0, potential + phi_state * k0,
                                phi_state * kc, cudaMemcpyDeviceToHost, plan->io_out), "D2H potential");
          plan->stats.evaluation_d2h_bytes += phi_state * kc;
          plan->stats.evaluation_d2h_calls += 1;
        }
      };
      for (int j = 0; j < n_parts; ++j) {
        const int k0 = bounds[j], kc = bounds[j + 1] - bounds[j];
        if (host_in) {
          // (a copy from pageable memory blocks here while earlier parts compute)
          check(cudaMemcpyAsync(const_cast<char *>(moments) + in_state * k0, static_cast<const char *>(a->moments) + in_state * k0,
                                in_state * kc, cudaMemcpyHostToDevice, plan->io_in), "H2D moments");
          plan->stats.evaluation_h2d_bytes += in_state * kc;
          plan->stats.evaluation_h2d_calls += 1;
          check(cudaEventRecord(plan->io_events[2 + 2 * j], plan->io_in), "event");
          check(cudaStreamWaitEvent(s, plan->io_events[2 + 2 * j], 0), "wait");
        }
        launch_gather_moments(moments + in_state * k0, a->moments_dtype, plan->src_inv, plan->ns, kc, plan->scale,
                              plan->mom, s, moments_paired(K), k0, K);
        ++launches;
        if (j < early) near_part(j, false);
      }
      launches += enqueue_far(plan, K, s, false);
      // one L2P for all K states: combined with the near field of the early
      // parts, far field alone for the later ones
      launch_l2p(plan->L, plan->tgt_rel, plan->tgt_off, plan->tgt_perm, plan->tgt_inv, plan->near, plan->basis,
                 plan->n, plan->p, K, plan->nt, plan->depth, a->output, a->layout, plan->phi_scale,
                 reinterpret_cast<float *>(field), reinterpret_cast<float *>(potential), s, 0, K, bounds[early], false);
      ++launches;
      for (int j = 0; j < early; ++j) finish_part(j);
      for (int j = early; j < n_parts; ++j) {
        near_part(j, true);
        finish_part(j);
      }
      check(cudaGetLastError(), "kernel launch");
      if (host_out) {
        for (int j = 0; j < n_parts; ++j) copy_out(j);
        check(cudaEventRecord(ev_end, plan->io_out), "event");
        check(cudaStreamWaitEvent(s, ev_end, 0), "wait");
      }
      plan->exp_state0 = 0;
      plan->last_K = K;
    } else if (n_chunks > 1) {
      while (static_cast<int>(plan->io_events.size()) < 2 * n_chunks + 2) {
        cudaEvent_t e;
        check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        plan->io_events.push_back(e);
      }
      cudaEvent_t ev_start = plan->io_events[0], ev_end = plan->io_events[1];
      check(cudaEventRecord(ev_start, s), "event");
      check(cudaStreamWaitEvent(plan->io_in, ev_start, 0), "wait");
      check(cudaStreamWaitEvent(plan->io_out, ev_start, 0), "wait");
      for (int c = 0; c < n_chunks; ++c) {
        const int k0 = c * chunk, kc = std::min(chunk, K - k0);
        cudaEvent_t ev_in = plan->io_events[2 + 2 * c], ev_done = plan->io_events[3 + 2 * c];
        if (host_in && in_state > 0) {
          check(cudaMemcpyAsync(const_cast<char *>(moments) + in_state * k0, static_cast<const char *>(a->moments) + in_state * k0,
                                in_state * kc, cudaMemcpyHostToDevice, plan->io_in), "H2D moments");
          plan->stats.evaluation_h2d_bytes += in_state * kc;
          plan->stats.evaluation_h2d_calls += 1;
          check(cudaEventRecord(ev_in, plan->io_in), "event");
          check(cudaStreamWaitEvent(s, ev_in, 0), "wait");
        }
        launches += enqueue_evaluation(plan, moments + in_state * k0, a->moments_dtype, kc, a->output, a->layout,
                                       field ? reinterpret_cast<float *>(field + field_state * k0) : nullptr,
                                       potential ? reinterpret_cast<float *>(potential + phi_state * k0) : nullptr, s, false);
        if (host_out) {
          check(cudaEventRecord(ev_done, s), "event");
          check(cudaStreamWaitEvent(plan->io_out, ev_done, 0), "wait");
          if (field_out && field_state > 0) {
            check(cudaMemcpyAsync(reinterpret_cast<char *>(a->field) + field_state * k0, field + field_state * k0,
                                  field_state * kc, cudaMemcpyDeviceToHost, plan->io_out), "D2H field");
            plan->stats.evaluation_d2h_bytes += field_state * kc;
            plan->stats.evaluation_d2h_calls += 1;
          }
          if (phi_state > 0) {
            check(cudaMemcpyAsync(reinterpret_cast<char *>(a->potential) + phi_state * k0, potential + phi_state * k0,
                                  phi_state * kc, cudaMemcpyDeviceToHost, plan->io_out), "D2H potential");
            plan->stats.evaluation_d2h_bytes += phi_state * kc;
            plan->stats.evaluation_d2h_calls += 1;
          }
        }
      }
      check(cudaEventRecord(ev_end, plan->io_out), "event");
      check(cudaStreamWaitEvent(s, ev_end, 0), "wait");
      plan->exp_state0 = (n_chunks - 1) * chunk;
      plan->last_K = K - plan->exp_state0;
    } else {
      if (host_in && in_state > 0) {
        check(cudaMemcpyAsync(const_cast<char *>(moments), a->moments, in_state * K, cudaMemcpyHostToDevice, s), "H2D moments");
        plan->stats.evaluation_h2d_bytes += in_state * K;
        plan->stats.evaluation_h2d_calls += 1;
      }
      launches += enqueue_evaluation(plan, moments, a->moments_dtype, K, a->output, a->layout,
                                     reinterpret_cast<float *>(field), reinterpret_cast<float *>(potential), s, timing);
      traced = plan->trace && !timing;
      if (host_out) {
        if (field_out && field_state > 0) {
          check(cudaMemcpyAsync(a->field, field, field_state * K, cudaMemcpyDeviceToHost, s), "D2H field");
          plan->stats.evaluation_d2h_bytes += field_state * K;
          plan->stats.evaluation_d2h_calls += 1;
        }
        if (phi_state > 0) {
          check(cudaMemcpyAsync(a->potential, potential, phi_state * K, cudaMemcpyDeviceToHost, s), "D2H potential");
          plan->stats.evaluation_d2h_bytes += phi_state * K;
          plan->stats.evaluation_d2h_calls += 1;
        }
      }
      plan->exp_state0 = 0;
      plan->last_K = K;
    }
    check(cdfmm_b200_collect_status(plan, s, call), "status kernel launch");
    ++launches;
    if (a->synchronize || host_out || timing || traced) {
      check(cudaStreamSynchronize(s), "evaluate");
      const std::string own = cdfmm_b200_own_status(plan, call);
      if (!own.empty()) throw AbiError(CDFMM_B200_ERR_TIMEOUT, own);
    }
    if (traced) {
      auto at = [&](int i) {
        float v = 0.0F;
        cudaEventElapsedTime(&v, plan->ev_t[kTraceBegin], plan->ev_t[i]);
        return static_cast<double>(v);
      };
      plan->stats.trace_p2p_begin = at(kTraceP2pBegin);
      plan->stats.trace_p2p_end = at(kTraceP2pEnd);
      plan->stats.trace_far_begin = at(kTraceFarBegin);
      plan->stats.trace_m2l_begin = at(kTraceM2lBegin);
      plan->stats.trace_far_end = at(kTraceFarEnd);
      plan->stats.trace_end = at(kTraceEnd);
    }
    plan->stats.schedule_last = plan->last_schedule;
    plan->stats.m2l_mode_resolved = plan->last_m2l_tc ? CDFMM_B200_M2L_BF16X3 : CDFMM_B200_M2L_FP32;
    if (timing) {
      auto ms = [&](int i, int j) {
        float v = 0.0F;
        cudaEventElapsedTime(&v, plan->ev_t[i], plan->ev_t[j]);
        return static_cast<double>(v);
      };
      plan->stats.ms_gather = ms(0, 8);
      plan->stats.ms_p2m = ms(1, 2);
      plan->stats.ms_m2m = ms(2, 3);
      plan->stats.ms_m2l = ms(3, 4);
      plan->stats.ms_l2l = ms(4, 5);
      plan->stats.ms_p2p = ms(8, 9);
      plan->stats.ms_l2p = ms(6, 7);
      plan->stats.ms_total = ms(0, 7);
    }
    plan->stats.evaluations += 1;
    plan->stats.kernel_launches_last = static_cast<uint64_t>(launches);
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(plan, e.code, e.what());
  } catch (const std::exception &e) {
    return fail(plan, CDFMM_B200_ERR_RUNTIME, e.what());
  }
}

// The transposed plan: sources and targets swapped, self map inverted.  The
// exact transpose of the evaluated (discrete) FMM is the same FMM with the
// two point sets exchanged: the M2L matrices satisfy T_o = T_o^t and
// T_-o = S T_o S (S = diag((-1)^|alpha|)), P2M/L2P and M2M/L2L are transposes
// of each other up to S and a sign, list1 and list2 are symmetric relations in
// the uniform tree, and the dipole pair tensor is symmetric and even in r.
static void ensure_adjoint(cdfmm_b200_plan *plan) {
  if (plan->adjoint == nullptr) {
    cdfmm_b200_plan *adj = nullptr;
    try {
      adj = new_plan(plan->nt, plan->ns, plan->p, plan->depth, plan->max_states, plan->device);
      set_root(adj, plan->root_centre, plan->root_half_width);
      uint64_t &bytes = adj->stats.persistent_device_bytes;
      const size_t nl = static_cast<size_t>(plan->n_leaves) + 1;
      adj->src_pos64 = dalloc<double>(3 * static_cast<size_t>(adj->ns), bytes);
      adj->tgt_pos64 = dalloc<double>(3 * static_cast<size_t>(adj->nt), bytes);
      adj->src_perm = dalloc<int>(adj->ns, bytes);
      adj->tgt_perm = dalloc<int>(adj->nt, bytes);
      adj->src_off = dalloc<int>(nl, bytes);
      adj->tgt_off = dalloc<int>(nl, bytes);
      check(cudaDeviceSynchronize(), "sync");
      const cudaMemcpyKind dd = cudaMemcpyDeviceToDevice;
      check(cudaMemcpy(adj->src_pos64, plan->tgt_pos64, 24 * static_cast<size_t>(adj->ns), dd), "D2D");
      check(cudaMemcpy(adj->tgt_pos64, plan->src_pos64, 24 * static_cast<size_t>(adj->nt), dd), "D2D");
      check(cudaMemcpy(adj->src_perm, plan->tgt_perm, 4 * static_cast<size_t>(adj->ns), dd), "D2D");
      check(cudaMemcpy(adj->tgt_perm, plan->src_perm, 4 * static_cast<size_t>(adj->nt), dd), "D2D");
      check(cudaMemcpy(adj->src_off, plan->tgt_off, 4 * nl, dd), "D2D");
      check(cudaMemcpy(adj->tgt_off, plan->src_off, 4 * nl, dd), "D2D");
      adj->h_src_off = plan->h_tgt_off;
      adj->h_tgt_off = plan->h_src_off;
      finish_plan(adj, plan->m2l_mode);
    } catch (const AbiError &e) {
      free_plan(adj);
      throw AbiError(e.code, std::string("transposed plan: ") + e.what());
    } catch (...) {
      free_plan(adj);
      throw;
    }
    plan->adjoint = adj;
    plan->adjoint_self_version = -1;
  }
  if (plan->adjoint_self_version != plan->self_version) {
    int rc = CDFMM_B200_OK;
    if (plan->h_self.empty()) {
      rc = cdfmm_b200_set_self_indices(plan->adjoint, nullptr);
    } else {
      std::vector<int> inv(static_cast<size_t>(plan->ns), -1);
      for (int t = 0; t < plan->nt; ++t) {
        const int j = plan->h_self[static_cast<size_t>(t)];
        if (j < 0) continue;
        require(inv[static_cast<size_t>(j)] < 0,
                "backward needs a one-to-one self map (two targets name the same self source)");
        inv[static_cast<size_t>(j)] = t;
      }
      rc = cdfmm_b200_set_self_indices(plan->adjoint, inv.data());
    }
    if (rc != CDFMM_B200_OK) throw AbiError(rc, cdfmm_b200_last_error(plan->adjoint));
    plan->adjoint_self_version = plan->self_version;
  }
}

int cdfmm_b200_backward(cdfmm_b200_plan *plan, const cdfmm_b200_backward_args *a) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  try {
    require(a != nullptr, "args is NULL");
    require(a->struct_size == static_cast<int32_t>(sizeof(cdfmm_b200_backward_args)), "args.struct_size mismatch");
    require(a->n_states >= 1 && a->n_states <= plan->max_states, "n_states must be in [1, max_states]");
    require(a->grad_moments != nullptr || a->grad_target_positions != nullptr,
            "request grad_moments and/or grad_target_positions");
    require(plan->nt == 0 || a->grad_field != nullptr, "grad_field is NULL");
    if (plan->cuboid) throw AbiError(CDFMM_B200_ERR_LOGIC, "reverse mode supports point-dipole sources only");
    const bool want_x = a->grad_target_positions != nullptr;
    // The forward's sorted moments and leaf locals are still in the plan if
    // no evaluate ran since and that one held all K states.
    const bool reuse = a->forward_evaluation != 0 && a->forward_evaluation == plan->stats.evaluations &&
                       plan->exp_state0 == 0 && plan->last_K == a->n_states;
    if (want_x && !reuse) {
      require(plan->ns == 0 || a->moments != nullptr, "grad_target_positions needs the forward moments");
      require(a->moments_dtype == 0 || a->moments_dtype == 1, "moments_dtype must be 0 (float32) or 1 (float64)");
    }
    check(cudaSetDevice(plan->device), "cudaSetDevice");
    (void)cudaGetLastError();
    const int K = a->n_states;
    const unsigned long long call = ++plan->call_seq;
    cudaStream_t s = static_cast<cudaStream_t>(a->stream);
    const bool host_in = (a->memory & CDFMM_B200_MOMENTS_ON_HOST) != 0u;
    const bool host_out = (a->memory & CDFMM_B200_RESULTS_ON_HOST) != 0u;
    unsigned long long adjoint_call = 0;

    if (a->grad_moments != nullptr) {
      // dL/dm = A^t dL/dH: the transposed plan evaluated on the weights.
      ensure_adjoint(plan);
      plan->adjoint->near_mode = plan->near_mode;
      cdfmm_b200_eval_args e{};
      e.moments = a->grad_field;
      e.moments_dtype = 0;
      e.n_states = K;
      e.output = CDFMM_B200_OUTPUT_FIELD;
      e.layout = CDFMM_B200_LAYOUT_SEPARATE;
      e.field = a->grad_moments;
      e.memory = a->memory;
      e.stream = a->stream;
      e.synchronize = 0;
      const int rc = cdfmm_b200_evaluate(plan->adjoint, &e);
      if (rc != CDFMM_B200_OK) throw AbiError(rc, std::string("transposed evaluate: ") + cdfmm_b200_last_error(plan->adjoint));
      adjoint_call = plan->adjoint->call_seq;
    }

    if (want_x && plan->nt > 0) {
      // dL/dx_target: forward moments -> leaf locals (far pass), then the P2P
      // gradient partial sums and the L2P second-derivative kernel.
      const size_t mom_in_bytes = reuse ? 0 : static_cast<size_t>(K) * plan->ns * 3 * (a->moments_dtype == 1 ? 8 : 4);
      const size_t w_in_bytes = static_cast<size_t>(K) * plan->nt * 3 * sizeof(float);
      const size_t out_bytes = static_cast<size_t>(plan->nt) * 3 * sizeof(float);
      const void *moments = a->moments;
      const void *weights = a->grad_field;
      float *out = a->grad_target_positions;
      if (host_in || host_out) {
        const size_t need = (host_in ? mom_in_bytes + w_in_bytes : 0) + (host_out ? out_bytes : 0) + 64;
        char *stage = grow(reinterpret_cast<char *&>(plan->stage_grad), plan->stage_grad_bytes, need, "cudaMalloc staging");
        size_t off = 0;
        if (host_in) {
          if (mom_in_bytes > 0)
            check(cudaMemcpyAsync(stage, a->moments, mom_in_bytes, cudaMemcpyHostToDevice, s), "H2D moments");
          check(cudaMemcpyAsync(stage + mom_in_bytes, a->grad_field, w_in_bytes, cudaMemcpyHostToDevice, s),
                "H2D grad_field");
          plan->stats.evaluation_h2d_bytes += mom_in_bytes + w_in_bytes;
          plan->stats.evaluation_h2d_calls += mom_in_bytes > 0 ? 2 : 1;
          moments = stage;
          weights = stage + mom_in_bytes;
          off = (mom_in_bytes + w_in_bytes + 15) & ~static_cast<size_t>(15);
        }
        if (host_out) out = reinterpret_cast<float *>(stage + off);
      }
      const int G = p2p_grad_groups(K);
      float4 *W = grow(plan->wbuf, plan->wbuf_count, static_cast<size_t>(plan->nt) * K, "cudaMalloc weights");
      float4 *gpart = grow(plan->gpart, plan->gpart_count, static_cast<size_t>(plan->nt) * G, "cudaMalloc partials");
      if (!reuse)
        launch_gather_moments(moments, a->moments_dtype, plan->src_inv, plan->ns, K, plan->scale, plan->mom, s,
                              moments_paired(K));
      launch_gather_moments(weights, 0, plan->tgt_inv, plan->nt, K, 1.0, W, s, false);
      plan->stats.backward_reused_forward = reuse ? 1 : 0;
      // The recomputed far pass and the near-field gradient run one after the
      // other: side by side (as the forward's CORUN schedule runs its near
      // and far fields) measured 127.6 against 119.8 ms on the 1M-point
      // K = 64 bench workload.
      if (!reuse) enqueue_far(plan, K, s, false);
      if (plan->ngt_supported && near_on_tensor_cores(plan, K)) {
        ensure_near_grad_tc(plan);
        NearGradLaunch l{};
        l.blk_pos = plan->ngt_blk_pos;
        l.blk_off = plan->ngt_blk_off;
        l.blk_src = plan->ngt_blk_src;
        l.n_blocks = plan->ngt_n_blocks;
        l.work = plan->ntc_work;
        l.n_work = plan->ntc_n_work;
        l.b_ops = plan->ngt_b;
        l.error_flag = plan->error_flag;
        l.wait_limit = plan->tc_wait_limit;
        launch_near_grad_tc(l, plan->mom, plan->tgt_rel, plan->has_self ? plan->self_idx : nullptr, plan->depth, K, W,
                            gpart, G, s);
        launch_p2p_grad_close(plan->mom, close_geometry(plan), plan->has_self ? plan->self_idx : nullptr, K, W, gpart,
                              s);
      } else {
        launch_p2p_grad(plan->src_rel, plan->mom, plan->src_off, plan->tgt_rel, plan->p2p_work, plan->n_p2p_work,
                        plan->has_self ? plan->self_idx : nullptr, close_geometry(plan), plan->depth, K, W, gpart, s);
      }
      launch_l2p_grad(plan->L, plan->tgt_rel, plan->tgt_off, plan->tgt_perm, W, gpart, G, plan->n, plan->p, K,
                      plan->nt, plan->depth, static_cast<float>(1.0 / plan->scale), out, s);
      check(cudaGetLastError(), "kernel launch");
      if (host_out) {
        check(cudaMemcpyAsync(a->grad_target_positions, out, out_bytes, cudaMemcpyDeviceToHost, s), "D2H gradient");
        plan->stats.evaluation_d2h_bytes += out_bytes;
        plan->stats.evaluation_d2h_calls += 1;
      }
    }
    check(cdfmm_b200_collect_status(plan, s, call), "status kernel launch");
    if (a->synchronize || host_in || host_out) {
      check(cudaStreamSynchronize(s), "backward");
      std::string own = cdfmm_b200_own_status(plan, call);
      if (own.empty() && adjoint_call != 0) own = cdfmm_b200_own_status(plan->adjoint, adjoint_call);
      if (!own.empty()) throw AbiError(CDFMM_B200_ERR_TIMEOUT, own);
    }
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(plan, e.code, e.what());
  } catch (const std::exception &e) {
    return fail(plan, CDFMM_B200_ERR_RUNTIME, e.what());
  }
}

int cdfmm_b200_read_expansions(const cdfmm_b200_plan *plan, int32_t which, int32_t state, float *out,
                               size_t out_count) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  auto *mp = const_cast<cdfmm_b200_plan *>(plan);
  try {
    require(which == 0 || which == 1, "which must be 0 (multipoles) or 1 (locals)");
    require(state >= plan->exp_state0 && state < plan->exp_state0 + std::max(plan->last_K, 1),
            "state out of range (a host-memory evaluation of 128 or more states keeps the expansions of its last "
            "64-state chunk only)");
    const size_t need = static_cast<size_t>(plan->n_nodes) * plan->n;
    require(out != nullptr && out_count >= need, "output buffer too small");
    check(cudaSetDevice(plan->device), "cudaSetDevice");
    check(cudaDeviceSynchronize(), "sync");
    const int K = std::max(plan->last_K, 1);
    std::vector<float> all(need * K);
    check(cudaMemcpy(all.data(), which == 0 ? plan->M : plan->L, all.size() * sizeof(float), cudaMemcpyDeviceToHost),
          "D2H expansions");
    for (size_t q = 0; q < need; ++q) out[q] = all[q * K + (state - plan->exp_state0)];
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(mp, e.code, e.what());
  }
}

int cdfmm_b200_set_timing(cdfmm_b200_plan *plan, int32_t enabled) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (enabled < 0 || enabled > 2) return fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "timing mode must be 0, 1 or 2");
  plan->timing = enabled == 1;
  plan->trace = enabled == 2;
  plan->stats.timing_enabled = enabled;
  return CDFMM_B200_OK;
}

int cdfmm_b200_set_schedule(cdfmm_b200_plan *plan, int32_t schedule) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (schedule < CDFMM_B200_SCHEDULE_AUTO || schedule > CDFMM_B200_SCHEDULE_CORUN)
    return fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "unknown schedule");
  plan->schedule = schedule;
  return CDFMM_B200_OK;
}

int cdfmm_b200_set_near_mode(cdfmm_b200_plan *plan, int32_t mode) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (mode < CDFMM_B200_NEAR_AUTO || mode > CDFMM_B200_NEAR_TF32X3)
    return fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "unknown near-field mode");
  if (mode == CDFMM_B200_NEAR_TF32X3 && !plan->ntc_supported)
    return fail(plan, CDFMM_B200_ERR_RUNTIME, "the tensor-core near field needs an sm_100 device");
  plan->near_mode = mode;
  return CDFMM_B200_OK;
}

int cdfmm_b200_get_stats(const cdfmm_b200_plan *plan, cdfmm_b200_stats *out) {
  if (plan == nullptr || out == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan and out must not be NULL");
  *out = plan->stats;
  return CDFMM_B200_OK;
}

int cdfmm_b200_m2l_shapes(const cdfmm_b200_plan *plan, int32_t *out, int32_t capacity) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (capacity < 0 || (capacity > 0 && out == nullptr))
    return fail(const_cast<cdfmm_b200_plan *>(plan), CDFMM_B200_ERR_INVALID_ARGUMENT, "out is NULL");
  if (!plan->tc_supported) return 0;
  const int n = static_cast<int>(plan->tc_candidates.size());
  for (int i = 0; i < n && i < capacity; ++i) {
    out[3 * i] = plan->tc_candidates[static_cast<size_t>(i)].m_tiles;
    out[3 * i + 1] = plan->tc_candidates[static_cast<size_t>(i)].stages;
    out[3 * i + 2] = plan->tc_candidates[static_cast<size_t>(i)].fuse;
  }
  return n;
}

int cdfmm_b200_set_m2l_shape(cdfmm_b200_plan *plan, int32_t m_tiles, int32_t stages, int32_t fused) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (m_tiles == 0) {
    plan->tc_pinned = false;
    plan->tc_tiles_Kp = 0; // re-tune on the next tensor-core evaluate
    return CDFMM_B200_OK;
  }
  if (!plan->tc_supported)
    return fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "this plan has no tensor-core M2L (m2l_mode, order or device)");
  for (const cdfmm_b200_plan::TcShape &c : plan->tc_candidates) {
    if (c.m_tiles == m_tiles && c.stages == stages && c.fuse == (fused != 0 ? 1 : 0)) {
      plan->tc_m_tiles = c.m_tiles;
      plan->tc_stages = c.stages;
      plan->tc_fuse = c.fuse;
      plan->tc_acc_stride = round_up(c.fuse ? 2 * plan->tc_Npad : plan->tc_Npad, 32);
      plan->tc_tmem_cols = tmem_columns(plan->tc_m_tiles, plan->tc_acc_stride);
      plan->tc_pinned = true;
      plan->tc_tiles_Kp = 0; // work tiles rebuilt for this shape on the next evaluate
      return CDFMM_B200_OK;
    }
  }
  return fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT,
              "not a pipeline shape of this plan (cdfmm_b200_m2l_shapes lists them)");
}

int cdfmm_b200_poll_status(cdfmm_b200_plan *plan) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  int code = 0, calls = 0;
  for (cdfmm_b200_plan *q : {plan, plan->adjoint}) {
    if (q == nullptr || q->status == nullptr) continue;
    const volatile cdfmm_b200_plan::StatusRecord *r = q->status;
    const int count = r->count;
    if (count != q->status_seen) {
      calls += count - q->status_seen;
      code = r->code;
      q->status_seen = count;
    }
  }
  if (calls == 0) return CDFMM_B200_OK;
  return fail(plan, CDFMM_B200_ERR_TIMEOUT, timeout_message(code, calls, false));
}

int cdfmm_b200_set_wait_limit(cdfmm_b200_plan *plan, int64_t iterations) {
  if (plan == nullptr) return fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (iterations > static_cast<int64_t>(0xffffffffu))
    return fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "iterations must be below 2^32");
  const uint32_t limit = iterations < 0 ? kTcWaitLimit : static_cast<uint32_t>(iterations);
  plan->tc_wait_limit = limit;
  if (plan->adjoint != nullptr) plan->adjoint->tc_wait_limit = limit;
  return CDFMM_B200_OK;
}

int cdfmm_b200_selftest_bounded_wait(int32_t device) {
  int *flag = nullptr;
  try {
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
      cudaGetLastError();
      throw AbiError(CDFMM_B200_ERR_NO_DEVICE, "no CUDA device is available");
    }
    require(device >= 0 && device < devices, "device ordinal out of range");
    check(cudaSetDevice(device), "cudaSetDevice");
    check(cudaMalloc(&flag, sizeof(int)), "cudaMalloc");
    check(cudaMemset(flag, 0, sizeof(int)), "cudaMemset");
    launch_bounded_wait_selftest(flag, nullptr);
    check(cudaGetLastError(), "self-test launch");
    check(cudaDeviceSynchronize(), "self-test");
    int v = 0;
    check(cudaMemcpy(&v, flag, sizeof(int), cudaMemcpyDeviceToHost), "D2H");
    cudaFree(flag);
    flag = nullptr;
    if (v != 0)
      throw AbiError(CDFMM_B200_ERR_TIMEOUT, "bounded wait expired as intended (code " + std::to_string(v) +
                                                 "); the device context remains usable");
    throw AbiError(CDFMM_B200_ERR_LOGIC, "bounded-wait self-test: the wait did not expire");
  } catch (const AbiError &e) {
    if (flag) cudaFree(flag);
    return fail(nullptr, e.code, e.what());
  }
}

int cdfmm_b200_direct_grad_fp64(int32_t device, int32_t ns, const double *src, const double *mom, int32_t nt,
                                const double *tgt, const int32_t *self, const double *weights, double *grad) {
  void *buf[6] = {};
  try {
    require(ns >= 0 && nt >= 0, "negative population size");
    require(ns == 0 || (src && mom), "source arrays are required");
    require(nt == 0 || (tgt && weights && grad), "target positions, weights and grad are required");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
      cudaGetLastError();
      throw AbiError(CDFMM_B200_ERR_NO_DEVICE, "no CUDA device is available");
    }
    check(cudaSetDevice(device), "cudaSetDevice");
    if (nt == 0) return CDFMM_B200_OK;
    uint64_t bytes = 0, h2d = 0;
    double *dsrc = dalloc<double>(3 * static_cast<size_t>(ns), bytes);
    buf[0] = dsrc;
    double *dmom = dalloc<double>(3 * static_cast<size_t>(ns), bytes);
    buf[1] = dmom;
    double *dtgt = dalloc<double>(3 * static_cast<size_t>(nt), bytes);
    buf[2] = dtgt;
    double *dw = dalloc<double>(3 * static_cast<size_t>(nt), bytes);
    buf[3] = dw;
    double *dg = dalloc<double>(3 * static_cast<size_t>(nt), bytes);
    buf[4] = dg;
    int *dself = nullptr;
    if (self) {
      dself = dalloc<int>(nt, bytes);
      buf[5] = dself;
      upload(dself, self, nt, h2d);
    }
    upload(dsrc, src, 3 * static_cast<size_t>(ns), h2d);
    upload(dmom, mom, 3 * static_cast<size_t>(ns), h2d);
    upload(dtgt, tgt, 3 * static_cast<size_t>(nt), h2d);
    upload(dw, weights, 3 * static_cast<size_t>(nt), h2d);
    launch_direct_grad_fp64(dsrc, dmom, ns, dtgt, nt, dself, dw, dg, nullptr);
    check(cudaGetLastError(), "direct gradient kernel");
    check(cudaDeviceSynchronize(), "direct gradient kernel");
    check(cudaMemcpy(grad, dg, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost), "D2H");
    for (void *b : buf)
      if (b) cudaFree(b);
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    for (void *b : buf)
      if (b) cudaFree(b);
    return fail(nullptr, e.code, e.what());
  }
}

int cdfmm_b200_direct_fp64(int32_t device, int32_t ns, const double *src, const double *mom, int32_t nt,
                           const double *tgt, const int32_t *self, double *phi, double *field) {
  void *buf[6] = {};
  try {
    require(ns >= 0 && nt >= 0, "negative population size");
    require(ns == 0 || (src && mom), "source arrays are required");
    require(nt == 0 || tgt, "target positions are required");
    int devices = 0;
    if (cudaGetDeviceCount(&devices) != cudaSuccess || devices == 0) {
      cudaGetLastError();
      throw AbiError(CDFMM_B200_ERR_NO_DEVICE, "no CUDA device is available");
    }
    check(cudaSetDevice(device), "cudaSetDevice");
    if (nt == 0) return CDFMM_B200_OK;
    uint64_t bytes = 0, h2d = 0;
    double *dsrc = dalloc<double>(3 * static_cast<size_t>(ns), bytes);
    buf[0] = dsrc;
    double *dmom = dalloc<double>(3 * static_cast<size_t>(ns), bytes);
    buf[1] = dmom;
    double *dtgt = dalloc<double>(3 * static_cast<size_t>(nt), bytes);
    buf[2] = dtgt;
    int *dself = nullptr;
    if (self) {
      dself = dalloc<int>(nt, bytes);
      buf[3] = dself;
      upload(dself, self, nt, h2d);
    }
    double *dphi = phi ? dalloc<double>(nt, bytes) : nullptr;
    buf[4] = dphi;
    double *dfield = field ? dalloc<double>(3 * static_cast<size_t>(nt), bytes) : nullptr;
    buf[5] = dfield;
    upload(dsrc, src, 3 * static_cast<size_t>(ns), h2d);
    upload(dmom, mom, 3 * static_cast<size_t>(ns), h2d);
    upload(dtgt, tgt, 3 * static_cast<size_t>(nt), h2d);
    launch_direct_fp64(dsrc, dmom, ns, dtgt, nt, dself, dphi, dfield, nullptr);
    check(cudaGetLastError(), "direct kernel");
    check(cudaDeviceSynchronize(), "direct kernel");
    if (phi) check(cudaMemcpy(phi, dphi, sizeof(double) * nt, cudaMemcpyDeviceToHost), "D2H");
    if (field) check(cudaMemcpy(field, dfield, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost), "D2H");
    for (void *b : buf)
      if (b) cudaFree(b);
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    for (void *b : buf)
      if (b) cudaFree(b);
    return fail(nullptr, e.code, e.what());
  }
}

int cdfmm_b200_m2l_matrix(int32_t order, const double *R, double *out, size_t out_count) {
  try {
    require(order >= 0 && order <= kMaxOrder, "order must be in [0, 10]");
    require(R != nullptr && out != nullptr, "R and out must not be NULL");
    require(R[0] != 0.0 || R[1] != 0.0 || R[2] != 0.0, "R must be nonzero");
    const int n = basis_size(order);
    require(out_count >= static_cast<size_t>(n) * n, "output buffer too small");
    const HostOperators ops = build_host_operators(order, 0, 1);
    const std::vector<double> d = laplace_derivatives(2 * order, R);
    for (int a = 0; a < n; ++a)
      for (int b = 0; b < n; ++b) {
        const int r = rank3(ops.ax[a] + ops.ax[b], ops.ay[a] + ops.ay[b], ops.az[a] + ops.az[b]);
        out[static_cast<size_t>(b) + static_cast<size_t>(n) * a] = d[static_cast<size_t>(r)];
      }
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(nullptr, e.code, e.what());
  }
}

int cdfmm_b200_m2l_stencil(int32_t order, double *out, size_t out_count, int32_t *source) {
  try {
    require(order >= 0 && order <= kMaxOrder, "order must be in [0, 10]");
    const int n = basis_size(order);
    require(out == nullptr || out_count >= static_cast<size_t>(343) * n * n, "output buffer too small");
    OperatorSource from = OperatorSource::Computed;
    const std::shared_ptr<const std::vector<double>> T = m2l_matrices(order, &from);
    if (out != nullptr) std::memcpy(out, T->data(), T->size() * sizeof(double));
    if (source != nullptr) *source = static_cast<int32_t>(from);
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(nullptr, e.code, e.what());
  } catch (const std::exception &e) {
    return fail(nullptr, CDFMM_B200_ERR_RUNTIME, e.what());
  }
}

int cdfmm_b200_m2l_traceless(int32_t order, int32_t *counts, int32_t *in_ranks, int32_t *out_ranks,
                             int32_t *fold_offsets, int32_t *fold_ranks, int32_t *fold_coefficients,
                             int32_t *derived) {
  try {
    require(order >= 0 && order <= kMaxOrder, "order must be in [0, 10]");
    require(counts != nullptr, "counts is NULL");
    const M2lTraceless t = m2l_traceless(order);
    const int n_out = static_cast<int>(t.out_set.size());
    counts[0] = static_cast<int32_t>(t.in_set.size());
    counts[1] = n_out;
    counts[2] = static_cast<int32_t>(t.fold.size());
    counts[3] = t.n_derived;
    if (in_ranks != nullptr) std::copy(t.in_set.begin(), t.in_set.end(), in_ranks);
    if (out_ranks != nullptr) std::copy(t.out_set.begin(), t.out_set.end(), out_ranks);
    if (fold_offsets != nullptr) std::copy(t.fold_off.begin(), t.fold_off.end(), fold_offsets);
    for (size_t f = 0; f < t.fold.size(); ++f) {
      if (fold_ranks != nullptr) fold_ranks[f] = t.fold[f] & 0xffff;
      if (fold_coefficients != nullptr) fold_coefficients[f] = (t.fold[f] >> 16) - 64;
    }
    if (derived != nullptr)
      for (int i = 0; i < t.n_derived; ++i) {
        const int e = t.expand[static_cast<size_t>(n_out + i)];
        derived[3 * i] = e & 1023;
        derived[3 * i + 1] = (e >> 10) & 1023;
        derived[3 * i + 2] = e >> 20;
      }
    return CDFMM_B200_OK;
  } catch (const AbiError &e) {
    return fail(nullptr, e.code, e.what());
  } catch (const std::exception &e) {
    return fail(nullptr, CDFMM_B200_ERR_RUNTIME, e.what());
  }
}

const char *cdfmm_b200_last_error(const cdfmm_b200_plan *plan) {
  if (plan != nullptr) return plan->last_error.c_str();
  return g_last_error.c_str();
}

} // extern "C"

std::vector<int4> cdfmm_b200::tc_work_tiles(int depth, int T) { return build_tc_tiles(depth, T); }
uint32_t cdfmm_b200::tc_tmem_columns(int m_tiles, int acc_stride) { return tmem_columns(m_tiles, acc_stride); }

cdfmm_b200::CloseGeometry cdfmm_b200_near_geometry(const cdfmm_b200_plan *plan) {
  using cdfmm_b200::CloseGeometry;
  using cdfmm_b200::CuboidNear;
  CloseGeometry g{plan->close_targets, plan->n_close_targets, plan->close_r_fp32, plan->close_r_exact, CuboidNear{}};
  if (plan->cuboid) g.cuboid = CuboidNear{plan->cuboid_T, plan->cuboid_base, plan->p2p_work, plan->n_p2p_work};
  return g;
}
