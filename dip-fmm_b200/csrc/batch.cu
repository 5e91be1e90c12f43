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
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "fmm_internal.hpp"

struct cdfmm_b200_batch {
  int device = 0;
  std::vector<cdfmm_b200_plan *> plans;
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
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->capture) cudaStreamDestroy(b->capture);
  delete b;
}

int batch_fail(int code, const std::string &msg) {
  cdfmm_b200_record_error(nullptr, msg);
  return code;
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
  cudaError_t e = cudaSetDevice(b->device);
  // Warm-up evaluation of every plan (tiles, autotuning, error checks).
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
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  b->joins.assign(static_cast<size_t>(count), nullptr);
  for (int i = 0; i < count && e == cudaSuccess; ++i) e = cudaEventCreateWithFlags(&b->joins[static_cast<size_t>(i)], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    destroy_batch(b);
    return batch_fail(CDFMM_B200_ERR_RUNTIME, std::string("batch set-up: ") + cudaGetErrorString(e));
  }
  for (cdfmm_b200_plan *p : b->plans) p->timing = false;
  e = cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) e = cudaEventRecord(b->fork, b->capture);
  int failed_rc = CDFMM_B200_OK;
  std::string failed_msg;
  for (int i = 0; i < count && e == cudaSuccess && failed_rc == CDFMM_B200_OK; ++i) {
    cdfmm_b200_plan *p = plans[i];
    e = cudaStreamWaitEvent(p->stream, b->fork, 0);
    if (e != cudaSuccess) break;
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

void cdfmm_b200_batch_destroy(cdfmm_b200_batch *batch) {
  if (batch == nullptr) return;
  cudaSetDevice(batch->device);
  cudaDeviceSynchronize();
  destroy_batch(batch);
}

} // extern "C"
