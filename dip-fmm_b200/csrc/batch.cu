// Multi-geometry batches: many plans (independent geometries of uneven size)
// evaluated by one CUDA graph launch (no counterpart in the reference, which
// evaluates one UniformFmm per call).
//
// cdfmm_b200_batch_create runs each plan's evaluate once (which also builds
// its tensor-core work tiles and runs the M2L autotuner), then captures every
// plan's evaluate into one graph, each on its own stream forked from and
// joined back to a capture stream, so the geometries are independent branches
// that the GPU overlaps.  cdfmm_b200_batch_launch replays the graph: one
// cudaGraphLaunch for the whole batch.  Arguments are fixed at creation
// (device-resident arrays; a new set of pointers needs a new batch).
//
// Stacked M2L: plans of one depth and order evaluated with one state each
// share their normalised M2L operators (the translation matrices and the
// exact power-of-two level scalings do not depend on a problem's size or
// position; its physical scale enters only through the moments' 1 / scale^3
// and the results' scale factors).  Such a group runs ONE tensor-core M2L
// whose states are the group's problems: the graph branch of each member
// runs gather, its near field, P2M and M2M, the group's branch packs every
// member's multipoles as one state each and runs the M2L, writing each
// state's locals into its own plan, and each member's branch then runs L2L
// and L2P.  One M2L with 8-24 states keeps the tensor cores far busier than
// 8-24 one-state M2Ls (each an 8-row group with one real state).
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "far_kernels.hpp"
#include "fmm_internal.hpp"
#include "kernels.cuh"
#include "m2l_tc.hpp"

namespace {

using namespace cdfmm_b200;

// One stacked-M2L group: plans of one depth and order, one state each.
struct StackGroup {
  std::vector<int> members;          // indices into the batch's plans
  int Kp = 0;                        // stacked states rounded up to 8
  void *a_hi = nullptr, *a_lo = nullptr; // packed operands [boxes + 1][Kp * Kpad] BF16
  float **M_list = nullptr;          // device: member k's multipoles
  float **L_list = nullptr;          // device: member k's locals
  int4 *tiles = nullptr;
  int n_tiles = 0;
  cdfmm_b200_plan::TcShape shape{1, 2, 0};
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<cudaEvent_t> up;       // per member: its multipoles are complete
};

} // namespace

struct cdfmm_b200_batch {
  int device = 0;
  std::vector<cdfmm_b200_plan *> plans;
  std::vector<cdfmm_b200_eval_args> args;
  std::vector<int> group_of;         // per plan: its stacked group, or -1
  std::vector<StackGroup> groups;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t capture = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> joins;
  std::string last_error;
};

namespace {

void destroy_batch(cdfmm_b200_batch *b) {
  if (b == nullptr) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cudaEvent_t e : b->joins)
    if (e) cudaEventDestroy(e);
  for (StackGroup &g : b->groups) {
    for (void *q : {g.a_hi, g.a_lo, static_cast<void *>(g.M_list), static_cast<void *>(g.L_list),
                    static_cast<void *>(g.tiles)})
      if (q) cudaFree(q);
    for (cudaEvent_t e : g.up)
      if (e) cudaEventDestroy(e);
    if (g.done) cudaEventDestroy(g.done);
    if (g.stream) cudaStreamDestroy(g.stream);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->capture) cudaStreamDestroy(b->capture);
  delete b;
}

int batch_fail(int code, const std::string &msg) {
  cdfmm_b200_record_error(nullptr, msg);
  return code;
}

// Kernel arguments of a group's stacked M2L (its first plan's operators).
TcArgs stacked_args(const cdfmm_b200_batch *b, const StackGroup &g) {
  const cdfmm_b200_plan *p0 = b->plans[static_cast<size_t>(g.members.front())];
  const int node_base = level_offset(2);
  TcArgs ta{};
  ta.a_hi = static_cast<const uint8_t *>(g.a_hi);
  ta.a_lo = static_cast<const uint8_t *>(g.a_lo);
  ta.b_tiles = static_cast<const uint8_t *>(p0->tc_b);
  set_m2l_reduction(ta, p0);
  ta.tiles = g.tiles;
  ta.scale_l = p0->scale_l;
  ta.L = nullptr;
  ta.L_list = g.L_list;
  ta.error_flag = p0->error_flag;
  ta.n = p0->n;
  ta.K = static_cast<int>(g.members.size());
  ta.Kp = g.Kp;
  ta.Kpad = p0->tc_Kpad;
  ta.Npad = p0->tc_Npad;
  ta.node_base = node_base;
  ta.zero_node = p0->n_nodes - node_base;
  ta.stages = g.shape.stages;
  ta.m_tiles = g.shape.m_tiles;
  ta.fuse_n = g.shape.fuse;
  ta.acc_stride = round_up(g.shape.fuse ? 2 * p0->tc_Npad : p0->tc_Npad, 32);
  ta.tmem_cols = tc_tmem_columns(g.shape.m_tiles, ta.acc_stride);
  ta.box_bytes = static_cast<uint32_t>(g.Kp) * static_cast<uint32_t>(p0->tc_Kpad) * 2u;
  ta.wait_limit = p0->tc_wait_limit;
  return ta;
}

void enqueue_stacked_m2l(const cdfmm_b200_batch *b, const StackGroup &g, cudaStream_t s) {
  const cdfmm_b200_plan *p0 = b->plans[static_cast<size_t>(g.members.front())];
  const int node_base = level_offset(2);
  launch_m2l_pack(nullptr, p0->scale_m, p0->tc_fold_off, p0->tc_fold, p0->tc_n_in, g.a_hi, g.a_lo, p0->n,
                  static_cast<int>(g.members.size()), g.Kp,
                  p0->tc_Kpad, p0->depth, node_base, p0->n_nodes - node_base, s, g.M_list);
  launch_m2l_tc(stacked_args(b, g), g.n_tiles, s);
}

cudaError_t upload_tiles(StackGroup &g, int depth) {
  const std::vector<int4> t = tc_work_tiles(depth, g.shape.m_tiles * (128 / g.Kp));
  if (g.tiles) cudaFree(g.tiles);
  g.tiles = nullptr;
  cudaError_t e = cudaMalloc(reinterpret_cast<void **>(&g.tiles), t.size() * sizeof(int4));
  // (a pageable copy may return before its DMA lands: wait for it)
  if (e == cudaSuccess) e = cudaMemcpy(g.tiles, t.data(), t.size() * sizeof(int4), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
  g.n_tiles = static_cast<int>(t.size());
  return e;
}

// Sets up group g (buffers, pointer tables) and picks its pipeline shape by
// timing every candidate of its first plan on the group's own packed
// operands (the members' multipoles from the warm-up evaluations).
cudaError_t prepare_group(cdfmm_b200_batch *b, StackGroup &g) {
  cdfmm_b200_plan *p0 = b->plans[static_cast<size_t>(g.members.front())];
  const int K = static_cast<int>(g.members.size());
  g.Kp = round_up(K, 8);
  const size_t boxes = static_cast<size_t>(p0->n_nodes - level_offset(2)) + 1;
  const size_t bytes = boxes * static_cast<size_t>(g.Kp) * p0->tc_Kpad * 2;
  std::vector<float *> M(static_cast<size_t>(K)), L(static_cast<size_t>(K));
  for (int k = 0; k < K; ++k) {
    M[static_cast<size_t>(k)] = b->plans[static_cast<size_t>(g.members[static_cast<size_t>(k)])]->M;
    L[static_cast<size_t>(k)] = b->plans[static_cast<size_t>(g.members[static_cast<size_t>(k)])]->L;
  }
  cudaError_t e = cudaMalloc(&g.a_hi, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&g.a_lo, bytes);
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&g.M_list), K * sizeof(float *));
  if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&g.L_list), K * sizeof(float *));
  if (e == cudaSuccess) e = cudaMemcpy(g.M_list, M.data(), K * sizeof(float *), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(g.L_list, L.data(), K * sizeof(float *), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy); // the copies have landed
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming);
  g.up.assign(static_cast<size_t>(K), nullptr);
  for (int k = 0; k < K && e == cudaSuccess; ++k) e = cudaEventCreateWithFlags(&g.up[static_cast<size_t>(k)], cudaEventDisableTiming);
  if (e != cudaSuccess) return e;
  // shape: the fastest candidate on this group's operands (the kernel
  // overwrites the members' locals, which the capture rewrites anyway)
  const int node_base = level_offset(2);
  launch_m2l_pack(nullptr, p0->scale_m, p0->tc_fold_off, p0->tc_fold, p0->tc_n_in, g.a_hi, g.a_lo, p0->n, K, g.Kp,
                  p0->tc_Kpad, p0->depth, node_base,
                  p0->n_nodes - node_base, g.stream, g.M_list);
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  e = cudaEventCreate(&t0);
  if (e == cudaSuccess) e = cudaEventCreate(&t1);
  float best = 0.0F;
  int best_i = -1;
  for (size_t c = 0; c < p0->tc_candidates.size() && e == cudaSuccess; ++c) {
    g.shape = p0->tc_candidates[c];
    if (g.shape.m_tiles * (128 / g.Kp) > kTcMaxTargets) continue;
    e = upload_tiles(g, p0->depth);
    float ms = 0.0F;
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
      e = cudaEventRecord(t0, g.stream);
      launch_m2l_tc(stacked_args(b, g), g.n_tiles, g.stream);
      if (e == cudaSuccess) e = cudaEventRecord(t1, g.stream);
      if (e == cudaSuccess) e = cudaEventSynchronize(t1);
      if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
    }
    if (e == cudaSuccess && (best_i < 0 || ms < best)) {
      best = ms;
      best_i = static_cast<int>(c);
    }
  }
  if (t0) cudaEventDestroy(t0);
  if (t1) cudaEventDestroy(t1);
  if (e != cudaSuccess) return e;
  if (best_i < 0) return cudaErrorInvalidConfiguration;
  g.shape = p0->tc_candidates[static_cast<size_t>(best_i)];
  e = upload_tiles(g, p0->depth);
  if (e == cudaSuccess) e = cudaStreamSynchronize(g.stream);
  return e;
}

// Groups plans evaluated with one state each on the tensor-core M2L by
// (depth, order); groups of two or more (up to 128 states) are stacked.
void form_groups(cdfmm_b200_batch *b) {
  std::map<std::pair<int, int>, std::vector<int>> by_key;
  for (size_t i = 0; i < b->plans.size(); ++i) {
    const cdfmm_b200_plan *p = b->plans[i];
    const cdfmm_b200_eval_args &a = b->args[i];
    const bool tc = p->depth >= 2 && p->tc_supported &&
                    (p->m2l_mode == CDFMM_B200_M2L_AUTO || p->m2l_mode == CDFMM_B200_M2L_BF16X3);
    if (tc && a.n_states == 1 && p->ns > 0 && p->nt > 0) by_key[{p->depth, p->p}].push_back(static_cast<int>(i));
  }
  b->group_of.assign(b->plans.size(), -1);
  for (auto &kv : by_key) {
    const std::vector<int> &v = kv.second;
    for (size_t s = 0; s < v.size(); s += 128) {
      const size_t e = std::min(v.size(), s + 128);
      if (e - s < 2) continue;
      StackGroup g;
      g.members.assign(v.begin() + static_cast<long>(s), v.begin() + static_cast<long>(e));
      for (int m : g.members) b->group_of[static_cast<size_t>(m)] = static_cast<int>(b->groups.size());
      b->groups.push_back(g);
    }
  }
}

} // namespace

extern "C" {

int cdfmm_b200_batch_create(cdfmm_b200_plan *const *plans, const cdfmm_b200_eval_args *args, int32_t count,
                            cdfmm_b200_batch **out_batch) {
  if (plans == nullptr || args == nullptr || out_batch == nullptr || count < 1)
    return batch_fail(CDFMM_B200_ERR_INVALID_ARGUMENT, "plans, args and out_batch must be non-NULL and count >= 1");
  *out_batch = nullptr;
  for (int i = 0; i < count; ++i) {
    if (plans[i] == nullptr) return batch_fail(CDFMM_B200_ERR_INVALID_ARGUMENT, "plan " + std::to_string(i) + " is NULL");
    if (plans[i]->device != plans[0]->device)
      return batch_fail(CDFMM_B200_ERR_INVALID_ARGUMENT, "all plans of a batch must be on one device");
    if (args[i].memory != 0u)
      return batch_fail(CDFMM_B200_ERR_INVALID_ARGUMENT, "batched evaluation takes device-resident arrays only");
    for (int j = 0; j < i; ++j)
      if (plans[j] == plans[i])
        return batch_fail(CDFMM_B200_ERR_INVALID_ARGUMENT, "a plan may appear once per batch (its buffers are shared)");
  }
  auto *b = new cdfmm_b200_batch();
  b->device = plans[0]->device;
  b->plans.assign(plans, plans + count);
  b->args.assign(args, args + count);
  cudaError_t e = cudaSetDevice(b->device);
  // Warm-up evaluation of every plan (tiles, autotuning, error checks; the
  // multipoles the stacked groups time their M2L shapes on).
  for (int i = 0; i < count && e == cudaSuccess; ++i) {
    cdfmm_b200_eval_args a = args[i];
    a.synchronize = 1;
    const int rc = cdfmm_b200_evaluate(plans[i], &a);
    if (rc != CDFMM_B200_OK) {
      const std::string msg = std::string("batch warm-up of plan ") + std::to_string(i) + ": " +
                              cdfmm_b200_last_error(plans[i]);
      destroy_batch(b);
      return batch_fail(rc, msg);
    }
  }
  form_groups(b);
  for (StackGroup &g : b->groups)
    if (e == cudaSuccess) e = prepare_group(b, g);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  b->joins.assign(static_cast<size_t>(count), nullptr);
  for (int i = 0; i < count && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&b->joins[static_cast<size_t>(i)], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    destroy_batch(b);
    return batch_fail(CDFMM_B200_ERR_RUNTIME, std::string("batch set-up: ") + cudaGetErrorString(e));
  }
  for (cdfmm_b200_plan *p : b->plans) p->timing = p->trace = false;
  e = cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) e = cudaEventRecord(b->fork, b->capture);
  int failed_rc = CDFMM_B200_OK;
  std::string failed_msg;
  try {
    // plans outside a group: one whole evaluate each; group members: the
    // upward half, the group's stacked M2L, then the downward half
    for (int i = 0; i < count && e == cudaSuccess && failed_rc == CDFMM_B200_OK; ++i) {
      cdfmm_b200_plan *p = plans[i];
      e = cudaStreamWaitEvent(p->stream, b->fork, 0);
      if (e != cudaSuccess) break;
      const int gi = b->group_of[static_cast<size_t>(i)];
      if (gi >= 0) {
        StackGroup &g = b->groups[static_cast<size_t>(gi)];
        const size_t k = static_cast<size_t>(std::find(g.members.begin(), g.members.end(), i) - g.members.begin());
        cdfmm_b200_stacked_upward(p, &args[i], p->stream);
        e = cudaEventRecord(g.up[k], p->stream);
        continue;
      }
      cdfmm_b200_eval_args a = args[i];
      a.stream = p->stream;
      a.synchronize = 0;
      p->in_batch = true; // the wide P2P units: other geometries run beside a long unit
      const int rc = cdfmm_b200_evaluate(p, &a);
      p->in_batch = false;
      if (rc != CDFMM_B200_OK) {
        failed_rc = rc;
        failed_msg = std::string("capture of plan ") + std::to_string(i) + ": " + cdfmm_b200_last_error(p);
        break;
      }
      e = cudaEventRecord(b->joins[static_cast<size_t>(i)], p->stream);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(b->capture, b->joins[static_cast<size_t>(i)], 0);
    }
    for (StackGroup &g : b->groups) {
      if (e != cudaSuccess || failed_rc != CDFMM_B200_OK) break;
      for (cudaEvent_t u : g.up)
        if (e == cudaSuccess) e = cudaStreamWaitEvent(g.stream, u, 0);
      if (e != cudaSuccess) break;
      enqueue_stacked_m2l(b, g, g.stream);
      e = cudaEventRecord(g.done, g.stream);
      for (size_t k = 0; k < g.members.size() && e == cudaSuccess; ++k) {
        const int i = g.members[k];
        cdfmm_b200_plan *p = plans[i];
        e = cudaStreamWaitEvent(p->stream, g.done, 0);
        if (e != cudaSuccess) break;
        cdfmm_b200_stacked_downward(p, &args[i], p->stream);
        e = cudaEventRecord(b->joins[static_cast<size_t>(i)], p->stream);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->capture, b->joins[static_cast<size_t>(i)], 0);
      }
    }
  } catch (const std::exception &ex) {
    failed_rc = CDFMM_B200_ERR_RUNTIME;
    failed_msg = std::string("batch capture: ") + ex.what();
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t end = cudaStreamEndCapture(b->capture, &graph);
  b->graph = graph;
  if (failed_rc != CDFMM_B200_OK) {
    destroy_batch(b);
    return batch_fail(failed_rc, failed_msg);
  }
  if (e == cudaSuccess) e = end;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    destroy_batch(b);
    return batch_fail(CDFMM_B200_ERR_RUNTIME, std::string("batch graph capture: ") + cudaGetErrorString(e));
  }
  *out_batch = b;
  return CDFMM_B200_OK;
}

int cdfmm_b200_batch_launch(cdfmm_b200_batch *batch, void *stream, int32_t synchronize) {
  if (batch == nullptr) return batch_fail(CDFMM_B200_ERR_INVALID_ARGUMENT, "batch is NULL");
  cudaError_t e = cudaSetDevice(batch->device);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (e == cudaSuccess) e = cudaGraphLaunch(batch->exec, s);
  if (e == cudaSuccess && synchronize) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return batch_fail(CDFMM_B200_ERR_RUNTIME, std::string("batch launch: ") + cudaGetErrorString(e));
  // The launch rewrote every plan's moments and expansions: a backward call
  // holding an older evaluation number must not reuse them.
  for (cdfmm_b200_plan *p : batch->plans) p->stats.evaluations += 1;
  if (synchronize) {
    // Each plan's captured work ends with its status kernel, which moved an
    // expired wait's error code into the plan's host record.
    int failed = 0, code = 0;
    for (cdfmm_b200_plan *p : batch->plans) {
      const volatile cdfmm_b200_plan::StatusRecord *r = p->status;
      const int count = r->count;
      if (count != p->status_seen) {
        failed += 1;
        code = r->code;
        p->status_seen = count;
      }
    }
    if (failed > 0)
      return batch_fail(CDFMM_B200_ERR_TIMEOUT, "tensor-core M2L: a bounded wait expired (code " + std::to_string(code) +
                                                   ") in " + std::to_string(failed) +
                                                   " plan(s) of the batch; their results are invalid (NaN)");
  }
  return CDFMM_B200_OK;
}

int cdfmm_b200_batch_groups(const cdfmm_b200_batch *batch, int32_t *out, int32_t capacity) {
  if (batch == nullptr) return batch_fail(CDFMM_B200_ERR_INVALID_ARGUMENT, "batch is NULL");
  const int n = static_cast<int>(batch->plans.size());
  if (capacity < 0 || (capacity > 0 && out == nullptr)) return batch_fail(CDFMM_B200_ERR_INVALID_ARGUMENT, "out is NULL");
  for (int i = 0; i < n && i < capacity; ++i) out[i] = batch->group_of[static_cast<size_t>(i)];
  return n;
}

void cdfmm_b200_batch_destroy(cdfmm_b200_batch *batch) {
  if (batch == nullptr) return;
  cudaSetDevice(batch->device);
  cudaDeviceSynchronize();
  destroy_batch(batch);
}

} // extern "C"
