// Launchers of the evaluator kernels (host side).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace cdfmm_b200 {

// Sorted moments: for K >= 4 states, pairs of states are interleaved so the
// near field can use packed FP32x2 arithmetic: a row of round_up(K, 2) float4
// holds, per pair (k, k+1), (x_k, x_k1, y_k, y_k1) then (z_k, z_k1, 0, 0).  For
// K < 4 a row is K float4 (x, y, z, 0).
inline bool moments_paired(int K) { return K >= 4; }
inline int moment_row(int K) { return moments_paired(K) ? (K + 1) & ~1 : K; }

// inv: user index -> sorted index; paired: write the paired layout (used for
// the moments of K >= 4 states; gradient weights are always plain).
// K states of user moments (user points at the first) into states
// [k0, k0 + K) of sorted rows laid out for k_total states (default K); k0 is
// even in the paired layout.
void launch_gather_moments(const void *user, int dtype, const int *inv, int ns, int K,
                           double scale, float4 *mom, cudaStream_t s, bool paired, int k0 = 0, int k_total = -1);
size_t p2m_smem_bytes(int n, int p, int K, int chunk);
// size != nullptr: uniformly magnetised cuboid sources, the monomials
// averaged over each source's cuboid (normalised side lengths, size[j] per
// source when size_step is 1, size[0] for all when 0).
void launch_p2m(const float4 *src_rel, const float4 *mom, const int *src_off, const int8_t *basis,
                float *M, int n, int p, int K, int depth, int chunk, cudaStream_t s,
                const float4 *size = nullptr, int size_step = 0);
void launch_m2m(float *M, const int *pair_off, const int *pairs, const float *coef, int n, int K,
                int parent_level, int n_pairs, cudaStream_t s);
void launch_l2l(float *L, const int *pair_off, const int *pairs, const float *coef, int n, int K,
                int child_level, int n_pairs, cudaStream_t s);
size_t l2p_smem_bytes(int n, int p, int Kb);
// L2P + combine; K >= 4 writes the sorted results over `near` and then unsorts
// them to user order (2 launches), K < 4 writes user order directly.  A state
// range [k_begin, k_end) (K >= 4 only; default all K) processes those states
// of the K-state rows.  States from k_near_end on (default K) have no near
// field yet: L2P writes the far field alone there, and a later P2P in
// accumulate mode adds the near field; unsort = false leaves the results
// sorted (launch_unsort does that part).
void launch_l2p(const float *L, const float4 *tgt_rel, const int *tgt_off, const int *tgt_perm, const int *tgt_inv,
                float4 *near, const int8_t *basis, int n, int p, int K, int nt, int depth, unsigned output,
                int layout, float phi_scale, float *field, float *potential, cudaStream_t s, int k_begin = 0,
                int k_end = -1, int k_near_end = -1, bool unsort = true);
// Sorted combined results (near, K states per target) of states
// [k_begin, k_end) -> user order (the second launch of launch_l2p).
void launch_unsort(const float4 *res, const int *tgt_inv, int nt, int K, unsigned output, int layout, float *field,
                   float *potential, cudaStream_t s, int k_begin, int k_end);
void configure_far_kernels(size_t max_smem);

// M2L, FP32 SIMT, all levels 2..depth in one launch (overwrites L there),
// on the traceless-reduced operator: T = [343][n_in][ld] FP32 sub-blocks
// (rows the folded moments, columns the n_out reduced locals), fold and
// expansion tables as built by m2l_traceless(); Mf is scratch for the
// folded moments of levels 2..depth ([boxes][n_in][K] floats).
void launch_m2l_simt(const float *M, float *Mf, float *L, const float *T, const float *scale_m,
                     const float *scale_l, const int4 *tiles, int n_tiles, int n, int ld, int K, int depth,
                     const int *fold_off, const int *fold, const int *expand, int n_in, int n_out, int n_derived,
                     cudaStream_t s);
void configure_m2l_simt(size_t max_smem);
int m2l_simt_beta_per_thread(int n);

// list1 P2P work units, one CTA each: (leaf, first sorted target, targets,
// 0), so the targets of a dense leaf spread over many SMs.  A unit holds at
// most kP2pUnitTargets targets, and fewer (a multiple of kP2pUnitMinTargets,
// at least that) where its cost -- targets x neighbourhood sources -- would
// exceed the total over kP2pUnitsPerSm x sm_count units: one CTA shares its
// SM with several others, so a unit above that cap would outlast the rest
// of the launch.  Units costing at least 4x the mean come first, heaviest
// first, so they start before the light ones fill the machine; the rest
// keep the Morton order, in which CTAs that run together share
// neighbourhood sources in L2 (a uniform geometry large enough that no leaf
// reaches the cap has its leaves as units, in Morton order).  Built once per geometry from the host leaf offsets
// (n_leaves + 1 prefix sums each); cap_cost = false keeps every unit at
// kP2pUnitTargets targets.
constexpr int kP2pUnitTargets = 128;
constexpr int kP2pUnitMinTargets = 16;
constexpr int kP2pUnitsPerSm = 20;
std::vector<int4> p2p_work_units(const int *src_off, const int *tgt_off, int depth, int sm_count, bool cap_cost);

// list1 P2P near field over the work units; states [k_begin, k_end) of the
// K-state rows (default all; k_begin a multiple of 8 when K >= 8).
// accumulate (K > 1): add the near field (phi times phi_scale) to the
// combined far-field results already in `near` instead of writing it (1: phi
// and H, 2: phi only).
// leaf_self: per leaf, the lowest and highest self source of its targets
// (read when self_idx is given).  corun (K > 1, NULL otherwise): the
// co-resident form -- persistent, `ctas` CTAs (two per SM) taking work units
// from the device counter `next_unit`, each CTA leaving room on its SM for
// one far-field CTA (same results up to the summation order of the state
// blocks).
struct NearTcLaunch; // tensor-core near field (near_tc.hpp)
struct CorunLaunch {
  int ctas;        // grid size: two per SM
  int *next_unit;  // device counter (reset on the launch stream)
};
// Close pairs: the plan's list of (target, source) pairs closer than a leaf
// width / 2^k, with the FP32 r the near-field kernels form (.w: source
// index) and r from the FP64 positions; a correction pass after every
// near-field launch swaps each pair's field at the FP32 r for its field at
// the exact r.  targets: (sorted target, first pair, pairs, 0).
// Cuboid sources: the near field applies per-pair moment-to-field tensors
// of the plan (FP32, computed once in FP64 by launch_cuboid_tensors) over
// its own work units; T of unit u, neighbourhood source g (flattened in
// build_neighbours order), component c (xx, xy, xz, yy, yz, zz) and target
// t of the unit is at T[base[u] + (g * 6 + c) * targets(u) + t].
struct CuboidNear {
  const float *T = nullptr;
  const long long *base = nullptr;
  const int4 *work = nullptr;
  int n_work = 0;
};
struct CloseGeometry {
  const int4 *targets;
  int n_targets;
  const float4 *r_fp32;
  const float4 *r_exact;
  CuboidNear cuboid; // T == nullptr: point-dipole sources
};
// Pair tensors of cuboid sources (see CuboidNear) from the Morton-sorted FP64
// positions (r = (x_t - x_s) * inv_scale) and the root-normalised FP64 side
// lengths (size[3 j + c], j = 0 for one common size when size_step is 0).
void launch_cuboid_tensors(const int4 *work, int n_work, const long long *base, const int *src_off, int depth,
                           const double *src_pos, const double *tgt_pos, double inv_scale, const double *size,
                           int size_step, float *T, cudaStream_t s);
// Near-field work of a cuboid-source plan per unit: neighbourhood sources of
// each unit (the tensor storage needed is 6 floats per (source, target)).
std::vector<long long> cuboid_unit_sources(const int *src_off, const std::vector<int4> &work, int depth);
void launch_p2p(const float4 *src_rel, const float4 *mom, const int *src_off,
                const float4 *tgt_rel, const int4 *work, int n_work, const int *self_idx,
                const int2 *leaf_self, const CloseGeometry &cg, int depth, int K,
                bool want_phi, float4 *near, cudaStream_t s, int k_begin = 0, int k_end = -1,
                int accumulate = 0, float phi_scale = 1.0F, const CorunLaunch *corun = nullptr,
                const NearTcLaunch *tc = nullptr);
// Close-pair search (once per plan), over work units covering every
// target, with r formed as the near-field kernels form it.  Count pass:
// counts[i][l] = pairs of target i with 0 < r^2 < thresholds[l]; write pass:
// the pairs with r^2 < r2_max of target i from out_first[i] on (FP32 r with
// the source index in .w; r from the FP64 root-normalised positions [n][3]).
constexpr int kCloseLevels = 4;
void launch_p2p_close_count(const float4 *src_rel, const int *src_off, const float4 *tgt_rel, const int4 *work,
                            int n_work, int depth, const float (&thresholds)[kCloseLevels], int *counts,
                            cudaStream_t s);
void launch_p2p_close_write(const float4 *src_rel, const int *src_off, const float4 *tgt_rel, const int4 *work,
                            int n_work, int depth, float r2_max, const int *out_first, const double *src_abs,
                            const double *tgt_abs, float4 *r_fp32, float4 *r_exact, cudaStream_t s);
void configure_p2p(size_t max_smem);
// Shared memory (dynamic + static bytes) of one CTA of the co-resident
// near-field form for K states.
size_t p2p_corun_cta_smem(int K);
// Position gradient of sum_k W_k . H_k, near part: partial sums per state
// group, gpart[nt][p2p_grad_groups(K)] (normalised units, 1/(4 pi) applied).
int p2p_grad_groups(int K);
// The close-pair correction of the position gradient (added to gpart's
// group 0), for a gradient computed by another near-field kernel.
void launch_p2p_grad_close(const float4 *mom, const CloseGeometry &cg, const int *self_idx, int K, const float4 *W,
                           float4 *gpart, cudaStream_t s);
void launch_p2p_grad(const float4 *src_rel, const float4 *mom, const int *src_off, const float4 *tgt_rel,
                     const int4 *work, int n_work, const int *self_idx, const CloseGeometry &cg, int depth, int K,
                     const float4 *W, float4 *gpart, cudaStream_t s, const CorunLaunch *corun = nullptr);
// Far part (second derivatives of the leaf local expansions) plus the near
// partial sums, scaled by inv_scale, written as out[user target][3].
void launch_l2p_grad(const float *L, const float4 *tgt_rel, const int *tgt_off, const int *tgt_perm,
                     const float4 *W, const float4 *gpart, int G, int n, int p, int K, int nt, int depth,
                     float inv_scale, float *out, cudaStream_t s);

// FP64 direct position gradient of w . H (validation reference of the reverse mode).
void launch_direct_grad_fp64(const double *src, const double *mom, int ns, const double *tgt, int nt,
                             const int *self, const double *w, double *grad, cudaStream_t s);

// FP64 direct sum (validation reference).
void launch_direct_fp64(const double *src, const double *mom, int ns, const double *tgt, int nt,
                        const int *self, double *phi, double *field, cudaStream_t s);

} // namespace cdfmm_b200
