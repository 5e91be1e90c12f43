// Allocation-free evaluation: cdfmm_b200_evaluate_noalloc.
//
// Who needs it: code that must not call cudaMalloc/cudaFree at evaluation
// time -- a framework whose caching pool already owns the device memory a
// library would ask for, a program that reserves all its device memory up
// front, or a real-time loop that cannot afford the allocator's implicit
// synchronisation.  Such callers create the plan once
// (plan creation allocates) and then evaluate with device-resident arrays
// through this entry point, which allocates nothing.
//
// How: every per-evaluation scratch buffer (sorted moments, multipole and
// local expansions, near field, the packed BF16 operands and work tiles of
// the tensor-core M2L) is carved out of ONE file-scope device array of
// kNoAllocScratchBytes, instead of the plan's own buffers.  The array exists
// on every GPU that loads this library, for the lifetime of the process.
// Host code must not pass the array's symbol to a kernel (in host code it is
// only a stand-in, not a device address): the device address is fetched with
// cudaGetSymbolAddress, once per device, on the first call made on that
// device -- make that first call before any stream capture begins.
//
// All calls share the one array and it keeps the previous call's contents:
// regions that must start at zero are cleared by every call, and two calls
// whose GPU work overlaps (on different streams, plans or threads) race on
// it -- order them on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "cdfmm_b200.h"
#include "far_kernels.hpp"
#include "fmm_internal.hpp"
#include "kernels.cuh"
#include "m2l_tc.hpp"

namespace {

using namespace cdfmm_b200;

// Scratch limit of the allocation-free entry point (documented in
// include/cdfmm_b200.h).
constexpr size_t kNoAllocScratchBytes = size_t{64} << 20;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_address[kMaxDevices] = {};

int noalloc_fail(cdfmm_b200_plan *plan, int code, const std::string &msg) {
  cdfmm_b200_record_error(plan, msg);
  return code;
}

// Device address of the scratch array on `device` (which must be current).
cudaError_t scratch_address(int device, void **out) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_address[device] == nullptr) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_address[device] = p;
  }
  *out = g_scratch_address[device];
  return cudaSuccess;
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

// Tensor-core M2L work tiles, written on the device (no host copy, no host
// synchronisation): per level from `depth` down to 2, runs of T
// consecutive parents, the 8 parity classes of a run adjacent (the plan's order).
__global__ void noalloc_tiles_kernel(int4 *tiles, int depth, int T, int n_tiles) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_tiles) return;
  int rest = q;
  for (int level = depth; level >= 2; --level) {
    const int parents = 1 << (3 * (level - 1));
    const int per_class = (parents + T - 1) / T;
    if (rest < 8 * per_class) {
      const int cls = rest & 7;
      const int p0 = (rest >> 3) * T;
      tiles[q] = make_int4(level, cls, p0, min(T, parents - p0));
      return;
    }
    rest -= 8 * per_class;
  }
}

} // namespace

extern "C" int cdfmm_b200_evaluate_noalloc(cdfmm_b200_plan *plan, const cdfmm_b200_eval_args *a) {
  if (plan == nullptr) return noalloc_fail(nullptr, CDFMM_B200_ERR_INVALID_ARGUMENT, "plan is NULL");
  if (a == nullptr) return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "args is NULL");
  if (a->memory != 0u)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT,
                        "evaluate_noalloc takes device-resident moments and results only (memory must be 0)");
  if (a->n_states < 1 || a->n_states > plan->max_states)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "n_states must be in [1, max_states]");
  if (a->moments_dtype != 0 && a->moments_dtype != 1)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "moments_dtype must be 0 (float32) or 1 (float64)");
  if ((a->output & 3u) == 0u || (a->output & ~3u) != 0u)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "output must request potential and/or field");
  if (a->layout != CDFMM_B200_LAYOUT_SEPARATE && a->layout != CDFMM_B200_LAYOUT_INTERLEAVED)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "unknown layout");
  const bool want_phi = (a->output & CDFMM_B200_OUTPUT_POTENTIAL) != 0u;
  const bool want_h = (a->output & CDFMM_B200_OUTPUT_FIELD) != 0u;
  if (plan->ns > 0 && a->moments == nullptr) return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "moments is NULL");
  if (plan->nt > 0 && (a->layout == CDFMM_B200_LAYOUT_INTERLEAVED || want_h) && a->field == nullptr)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "field is NULL");
  if (plan->nt > 0 && a->layout == CDFMM_B200_LAYOUT_SEPARATE && want_phi && a->potential == nullptr)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "potential is NULL");
  if (a->layout == CDFMM_B200_LAYOUT_INTERLEAVED && reinterpret_cast<uintptr_t>(a->field) % 16 != 0)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "interleaved results need a 16-byte aligned field pointer");
  if (reinterpret_cast<uintptr_t>(a->moments) % (a->moments_dtype == 1 ? 8 : 4) != 0)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "misaligned moments pointer");
  if (plan->device < 0 || plan->device >= kMaxDevices)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT, "device ordinal beyond the supported range");

  const int K = a->n_states;
  const int n = plan->n;
  const bool use_tc = plan->depth >= 2 && plan->tc_supported && K <= 128 &&
                      (plan->m2l_mode == CDFMM_B200_M2L_BF16X3 || plan->m2l_mode == CDFMM_B200_M2L_AUTO);
  const int Kp = round_up(K, 8);
  const int node_base = level_offset(2);
  const int boxes = plan->n_nodes - node_base;
  const int T = plan->tc_m_tiles * (128 / Kp);
  int n_tiles = 0;
  if (use_tc)
    for (int level = plan->depth; level >= 2; --level) n_tiles += 8 * (((1 << (3 * (level - 1))) + T - 1) / T);
  // Carve the scratch regions (each 256-byte aligned).
  const size_t mom_bytes = align256(sizeof(float4) * static_cast<size_t>(plan->ns) * moment_row(K));
  const size_t exp_bytes = align256(sizeof(float) * static_cast<size_t>(plan->n_nodes) * n * K);
  const size_t near_bytes = align256(sizeof(float4) * static_cast<size_t>(plan->nt) * K);
  const size_t pack_bytes = use_tc ? align256(static_cast<size_t>(boxes + 1) * Kp * plan->tc_Kpad * 2) : 0;
  const size_t tile_bytes = align256(sizeof(int4) * static_cast<size_t>(n_tiles));
  const size_t fold_bytes =
      (!use_tc && plan->depth >= 2) ? align256(sizeof(float) * static_cast<size_t>(boxes) * plan->tc_n_in * K) : 0;
  const size_t need = mom_bytes + 2 * exp_bytes + near_bytes + 2 * pack_bytes + tile_bytes + fold_bytes;
  if (need > kNoAllocScratchBytes)
    return noalloc_fail(plan, CDFMM_B200_ERR_INVALID_ARGUMENT,
                        "evaluate_noalloc needs " + std::to_string(need) + " bytes of scratch for this plan and n_states; "
                        "its fixed scratch holds at most " + std::to_string(kNoAllocScratchBytes) +
                        " bytes (64 MiB) -- use cdfmm_b200_evaluate");

  cudaError_t e = cudaSetDevice(plan->device);
  void *base = nullptr;
  if (e == cudaSuccess) e = scratch_address(plan->device, &base);
  if (e != cudaSuccess)
    return noalloc_fail(plan, CDFMM_B200_ERR_RUNTIME, std::string("scratch set-up: ") + cudaGetErrorString(e));
  (void)cudaGetLastError();
  char *cursor = static_cast<char *>(base);
  auto take = [&](size_t bytes) {
    char *p = cursor;
    cursor += bytes;
    return p;
  };
  float4 *mom = reinterpret_cast<float4 *>(take(mom_bytes));
  float *M = reinterpret_cast<float *>(take(exp_bytes));
  float *L = reinterpret_cast<float *>(take(exp_bytes));
  float4 *near = reinterpret_cast<float4 *>(take(near_bytes));
  void *a_hi = take(pack_bytes);
  void *a_lo = take(pack_bytes);
  int4 *dtiles = reinterpret_cast<int4 *>(take(tile_bytes));
  float *Mf = reinterpret_cast<float *>(take(fold_bytes));

  cudaStream_t s = static_cast<cudaStream_t>(a->stream);
  const unsigned long long call = ++plan->call_seq;
  // Locals of levels 0 and 1 are never written (no M2L there) and must read
  // as zero; the array still holds the previous call's values.
  e = cudaMemsetAsync(L, 0, exp_bytes, s);
  if (e != cudaSuccess) return noalloc_fail(plan, CDFMM_B200_ERR_RUNTIME, std::string("scratch: ") + cudaGetErrorString(e));
  if (n_tiles > 0) noalloc_tiles_kernel<<<(n_tiles + 127) / 128, 128, 0, s>>>(dtiles, plan->depth, T, n_tiles);

  launch_gather_moments(a->moments, a->moments_dtype, plan->src_inv, plan->ns, K, plan->scale, mom, s,
                        moments_paired(K));
  cudaEventRecord(plan->ev_fork, s);
  cudaStreamWaitEvent(plan->near_stream, plan->ev_fork, 0);
  launch_p2p(plan->src_rel, mom, plan->src_off, plan->tgt_rel, plan->p2p_work, plan->n_p2p_work,
             plan->has_self ? plan->self_idx : nullptr, plan->leaf_self,
             cdfmm_b200_near_geometry(plan),
             plan->depth, K, want_phi, near,
             plan->near_stream);
  cudaEventRecord(plan->ev_join, plan->near_stream);
  launch_p2m(plan->src_rel, mom, plan->src_off, plan->basis, M, n, plan->p, K, plan->depth, plan->p2m_chunk, s,
             plan->cuboid_p2m ? plan->src_size : nullptr, plan->size_step);
  for (int level = plan->depth - 1; level >= 0; --level)
    launch_m2m(M, plan->m2m_off, plan->m2m_pair, plan->m2m_coef, n, K, level, static_cast<int>(plan->ops.m2m_pair_g.size()), s);
  if (use_tc) {
    launch_m2l_pack(M, plan->scale_m, plan->tc_fold_off, plan->tc_fold, plan->tc_n_in, a_hi, a_lo, n, K, Kp,
                    plan->tc_Kpad, plan->depth, node_base, boxes, s);
    TcArgs ta{};
    ta.a_hi = static_cast<const uint8_t *>(a_hi);
    ta.a_lo = static_cast<const uint8_t *>(a_lo);
    ta.b_tiles = static_cast<const uint8_t *>(plan->tc_b);
    set_m2l_reduction(ta, plan);
    ta.tiles = dtiles;
    ta.scale_l = plan->scale_l;
    ta.L = L;
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
    launch_m2l_tc(ta, n_tiles, s);
  } else if (plan->depth >= 2) {
    launch_m2l_simt(M, Mf, L, plan->m2l_T, plan->scale_m, plan->scale_l, plan->m2l_tiles, plan->n_tiles, n,
                    plan->m2l_ld_red, K, plan->depth, plan->tc_fold_off, plan->tc_fold, plan->tc_expand,
                    plan->tc_n_in, plan->tc_n_out, plan->tc_n_derived, s);
  }
  for (int level = 3; level <= plan->depth; ++level)
    launch_l2l(L, plan->l2l_off, plan->l2l_pair, plan->l2l_coef, n, K, level, static_cast<int>(plan->ops.l2l_pair_g.size()), s);
  cudaStreamWaitEvent(s, plan->ev_join, 0);
  launch_l2p(L, plan->tgt_rel, plan->tgt_off, plan->tgt_perm, plan->tgt_inv, near, plan->basis, n, plan->p, K, plan->nt, plan->depth, a->output,
             a->layout, plan->phi_scale, a->field, a->potential, s);
  e = cudaGetLastError();
  // The plan's error flag (set by an expired wait of the tensor-core M2L)
  // goes to the plan's host status record, tagged with this call.
  if (e == cudaSuccess) e = cdfmm_b200_collect_status(plan, s, call);
  if (e == cudaSuccess && a->synchronize) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return noalloc_fail(plan, CDFMM_B200_ERR_RUNTIME, std::string("evaluate_noalloc: ") + cudaGetErrorString(e));
  if (a->synchronize) {
    const std::string own = cdfmm_b200_own_status(plan, call);
    if (!own.empty()) return noalloc_fail(plan, CDFMM_B200_ERR_TIMEOUT, own);
  }
  return CDFMM_B200_OK;
}
