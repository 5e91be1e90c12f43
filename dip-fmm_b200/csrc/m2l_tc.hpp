// Tensor-core (tcgen05) M2L: launch interface.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <vector>

namespace cdfmm_b200 {

struct TcArgs {
  const uint8_t *a_hi;     // packed BF16 hi boxes [box][32-alpha chunk][Kp/8][w/8][8][8] (folded moments)
  const uint8_t *a_lo;     // packed BF16 lo boxes
  const uint8_t *b_tiles;  // [343 slots][32-alpha chunk][hi, lo][Npad/8][w/8][8][8] (reduced operator)
  const int4 *tiles;       // per CTA: (level, class, first parent Morton index, target count)
  const float *scale_l;    // [depth+1][n] exact powers of two
  float *L;                // [node][n][K] FP32 locals (overwritten)
  float *const *L_list;    // or (stacked problems, one state each): state k's locals at L_list[k][node][n]
  int *error_flag;         // set nonzero if a bounded wait expired
  int n, K, Kp, Kpad, Npad;
  int node_base;           // flat node index of packed box 0
  int zero_node;           // packed index of the all-zero box
  int stages;
  int m_tiles;             // 128-row accumulators per CTA sharing each B tile
  int acc_stride;          // TMEM columns between accumulators (multiple of 32)
  int fuse_n;              // 1: A_hi x [B_hi | B_lo] as one N = 2 Npad MMA (acc_stride >= 2 Npad)
  uint32_t tmem_cols;
  uint32_t box_bytes;      // Kp * Kpad * 2
  uint32_t wait_limit;     // iterations of each pipeline progress wait (kTcWaitLimit; 0 = expire at once)
  // traceless reduction (M2lTraceless): accumulator column j holds the
  // local of full rank expand[j] (j < n_out); expand[n_out + i] =
  // d | s1 << 10 | s2 << 20 gives the remaining locals L_d = -(L_s1 + L_s2)
  // in an order where both sources come first
  const int *expand;
  int n_out, n_derived;
};

// Traceless reduction of the M2L (Cartesian Taylor basis of order p, n
// coefficients).  The operator T[beta][alpha] = D^{alpha+beta} G with G
// harmonic, so D^{g + 2z} = -D^{g + 2x} - D^{g + 2y}:
//   * inputs: a moment M_alpha with alpha_z >= 2 acts exactly as -M on
//     alpha - 2z + 2x and on alpha - 2z + 2y; folded repeatedly, the moments
//     reduce to the (p+1)^2 components with alpha_z <= 1, and the dipole
//     monopole M_0 is identically zero (every moment is a gradient moment),
//     leaving n_in = (p+1)^2 - 1 inputs;
//   * outputs: L_beta for beta_z <= 1 (n_out = (p+1)^2) determine the rest
//     by L_beta = -L_{beta-2z+2x} - L_{beta-2z+2y}.
// The matrices T restricted to (in, out) are exact sub-blocks of the full
// ones; the reduction is exact in exact arithmetic.
struct M2lTraceless {
  std::vector<int> in_set;    // full ranks of the reduced inputs (ascending)
  std::vector<int> out_set;   // full ranks of the reduced outputs (ascending)
  std::vector<int> fold_off;  // [n_in + 1] CSR over reduced inputs
  std::vector<int> fold;      // per entry: full rank | (coefficient + 64) << 16
  std::vector<int> expand;    // out_set, then the packed derived triplets
  int n_derived = 0;
};
M2lTraceless m2l_traceless(int p);

// Default iterations of a bounded mbarrier wait (about 2 s with the back-off).
constexpr uint32_t kTcWaitLimit = 1u << 26;

// Largest target count of one CTA: m_tiles (<= 4) x 128 / Kp with Kp >= 8.
constexpr int kTcMaxTargets = 64;

// The reduction fields of a launch from the plan that owns the tables.
template <class Plan> inline void set_m2l_reduction(TcArgs &ta, const Plan *p) {
  ta.expand = p->tc_expand;
  ta.n_out = p->tc_n_out;
  ta.n_derived = p->tc_n_derived;
}

// Dynamic shared memory of the M2L kernel: the pipeline stages, or the
// epilogue's 128 full-basis rows of n coefficients when larger.
size_t m2l_tc_smem_bytes(int Npad, int m_tiles, int stages, int n);
// Scaled, folded multipoles -> BF16 hi/lo boxes (fold_off / fold from
// M2lTraceless, n_in reduced inputs, Kpad = 16 ceil(n_in / 16)).
void launch_m2l_pack(const float *M, const float *scale_m, const int *fold_off, const int *fold, int n_in, void *hi,
                     void *lo, int n, int K, int Kp, int Kpad, int depth, int node_base, int n_boxes, cudaStream_t s,
                     const float *const *M_list = nullptr);
void launch_m2l_tc(const TcArgs &args, int n_tiles, cudaStream_t s);
bool configure_m2l_tc(size_t max_smem);
// Runs a kernel whose bounded mbarrier wait must expire (nothing arrives)
// and set *error_flag = 2, exactly as an expired wait of the M2L pipeline.
void launch_bounded_wait_selftest(int *error_flag, cudaStream_t s);
// B tiles of the reduced operator: element (beta row i, alpha column j) =
// T[out_set[i]][in_set[j]] of the FP64 matrices T[slot][n][n].
std::vector<uint16_t> pack_m2l_b_tiles(const std::vector<double> &T64, int n, const M2lTraceless &red, int Npad,
                                       int Kpad);

} // namespace cdfmm_b200
