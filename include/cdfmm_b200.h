/*
 * cdfmm_b200 -- C ABI of the B200 (sm_100a) evaluator for the static-geometry
 * uniform-octree dipole FMM.
 *
 * This is the drop-in boundary for upstream dip-fmm's device executor.  In the
 * reference, UniformFmm hands its CPU-built static plan to
 *   CudaFullPlan::CudaFullPlan(const FloatCudaFullPlanData&)   src/cuda_fmm_plan.hpp:95-101
 *   CudaFullPlan::evaluate(moments, fields, sorted_self_indices) src/cuda_fmm_plan.hpp:103-108
 * (owned through UniformFmm::CudaFullPlanOwner, src/uniform_fmm_internal.hpp:27-32,
 * dispatched from src/uniform_fmm.cpp:1102-1136 and :1307-1349).  Here the
 * caller hands over only the Morton-sorted geometry; every operator is
 * generated inside the plan, and one evaluate call processes K moment states.
 *
 * Conventions
 *  - Plain C: pointers, sizes and status codes; no exceptions cross the ABI.
 *  - Every function returns CDFMM_B200_OK (0) or an error status; the message
 *    of the last failure is available from cdfmm_b200_last_error().
 *  - Moments and results use the caller's (user) source / target order; the
 *    plan applies the Morton permutations internally.
 *  - Positions, moments, potential and field are in physical units.  The plan
 *    evaluates in root-width-normalised FP32 coordinates exactly as the
 *    reference FP32 plan does (src/uniform_fmm.cpp:379-417, :1315-1323, :1448-1451).
 *  - A plan is not re-entrant: calls on one plan must not overlap.
 */
#ifndef CDFMM_B200_H
#define CDFMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The C++ wrapper maps INVALID_ARGUMENT to std::invalid_argument,
 * LOGIC to std::logic_error and the rest to std::runtime_error, which is how
 * the reference reports the same conditions (src/uniform_fmm.cpp:1290-1311,
 * src/cuda_fmm.cu:32-54). */
#define CDFMM_B200_OK 0
#define CDFMM_B200_ERR_INVALID_ARGUMENT 1
#define CDFMM_B200_ERR_RUNTIME 2
#define CDFMM_B200_ERR_OUT_OF_MEMORY 3
#define CDFMM_B200_ERR_LOGIC 4
#define CDFMM_B200_ERR_NO_DEVICE 5
#define CDFMM_B200_ERR_TIMEOUT 6

/* Output selection: same bit values as cdfmm::OutputFlags (include/cdfmm/output_flags.hpp:12-17 upstream). */
#define CDFMM_B200_OUTPUT_POTENTIAL 1u
#define CDFMM_B200_OUTPUT_FIELD 2u

/* M2L arithmetic. */
#define CDFMM_B200_M2L_AUTO 0        /* split-BF16 tensor cores on sm_100, depth >= 2, order <= 9 (any K), else FP32 */
#define CDFMM_B200_M2L_FP32 1        /* FP32 SIMT (the plain per-state path), on the same traceless-reduced
                                        operator; plans that can take this path keep a folded-moment buffer
                                        of (levels 2..depth boxes) x (p+1)^2 x max_states floats */
#define CDFMM_B200_M2L_BF16X3 2      /* tcgen05, BF16 hi/lo with three products, FP32 accumulate; applies the
                                        traceless-reduced operator ((p+1)^2 - 1 folded moments in, (p+1)^2
                                        locals out, the rest from the trace relations); any order */

/* Near-field arithmetic of evaluations of 8..128 states (cdfmm_b200_set_near_mode). */
#define CDFMM_B200_NEAR_AUTO 0       /* tensor cores where supported, else FP32 */
#define CDFMM_B200_NEAR_FP32 1       /* FP32 SIMT */
#define CDFMM_B200_NEAR_TF32X3 2     /* tcgen05, TF32 hi/lo with three products, FP32 accumulate */

/* Where the caller's arrays live (cdfmm_b200_eval_args.memory). */
#define CDFMM_B200_MOMENTS_ON_HOST 1u
#define CDFMM_B200_RESULTS_ON_HOST 2u

/* Near/far schedule of an evaluation of K > 1 states (cdfmm_b200_set_schedule). */
#define CDFMM_B200_SCHEDULE_AUTO 0      /* SEPARATE (CORUN runs only on request) */
#define CDFMM_B200_SCHEDULE_SEPARATE 1  /* full-size near-field CTAs beside a high-priority far field */
#define CDFMM_B200_SCHEDULE_CORUN 2     /* upward pass first; then near-field CTAs sized to leave one
                                           tensor-core M2L CTA per SM, the near field at high priority */

/* Result layout (cdfmm_b200_eval_args.layout). */
#define CDFMM_B200_LAYOUT_SEPARATE 0    /* field[K][Nt][3] and potential[K][Nt] */
#define CDFMM_B200_LAYOUT_INTERLEAVED 1 /* field[K][Nt][4] = {phi, Hx, Hy, Hz}: cdfmm::FloatPotentialField */

typedef struct cdfmm_b200_plan cdfmm_b200_plan;

/* Geometry of one problem, as produced by the host tree
 * (include/cdfmm/uniform_tree.hpp; upstream src/uniform_tree.cpp:129-523).
 * Replaces FloatCudaFullPlanData (src/cuda_fmm_plan.hpp:69-86 upstream). */
typedef struct cdfmm_b200_plan_desc {
  int32_t struct_size;             /* sizeof(cdfmm_b200_plan_desc) */
  int32_t n_sources;               /* >= 0 */
  int32_t n_targets;               /* >= 0 */
  int32_t order;                   /* expansion order p, 0..10 */
  int32_t depth;                   /* tree max_level, 0..8 */
  int32_t max_states;              /* largest K passed to one evaluate call, >= 1 */
  int32_t m2l_mode;                /* CDFMM_B200_M2L_* */
  int32_t device;                  /* CUDA device ordinal */
  double root_centre[3];           /* cubic root box (UniformTree::root_centre) */
  double root_half_width;          /* (UniformTree::root_half_width), > 0 */
  const double *sorted_source_positions; /* [n_sources][3], Morton-sorted (host memory) */
  const double *sorted_target_positions; /* [n_targets][3], Morton-sorted (host memory) */
  const int32_t *source_permutation;     /* [n_sources] sorted index -> user index */
  const int32_t *target_permutation;     /* [n_targets] sorted index -> user index */
  const int32_t *leaf_source_offsets;    /* [8^depth + 1], sources of Morton leaf m are [o[m], o[m+1]) */
  const int32_t *leaf_target_offsets;    /* [8^depth + 1] */
} cdfmm_b200_plan_desc;

/* One evaluate call: K moment states on the plan's fixed geometry.
 * Replaces CudaFullPlan::evaluate (src/cuda_fmm.cu:3457-3655 upstream), which
 * handles one state, field only, host memory and a blocking D2H. */
typedef struct cdfmm_b200_eval_args {
  const void *moments;   /* [n_states][n_sources][3], user source order, physical units */
  int32_t moments_dtype; /* 0 = float32, 1 = float64 */
  int32_t n_states;      /* K, 1..max_states */
  uint32_t output;       /* CDFMM_B200_OUTPUT_* bits; at least one */
  int32_t layout;        /* CDFMM_B200_LAYOUT_* */
  float *field;          /* see layout; required when FIELD is requested or layout is interleaved */
  float *potential;      /* [n_states][n_targets] for LAYOUT_SEPARATE with POTENTIAL, else unused */
  uint32_t memory;       /* CDFMM_B200_*_ON_HOST bits */
  void *stream;          /* cudaStream_t to order the work on; NULL = the legacy default stream */
  int32_t synchronize;   /* nonzero: return only after results are complete */
} cdfmm_b200_eval_args;

/* Per-plan counters (mirrors the reference's CudaPlanStatistics fields it has,
 * include/cdfmm/timings.hpp:182-223 upstream) and the device time of the last
 * evaluate per stage (milliseconds; filled only when timing is enabled). */
typedef struct cdfmm_b200_stats {
  uint64_t persistent_device_bytes;
  uint64_t setup_h2d_bytes;
  uint64_t evaluation_h2d_bytes;
  uint64_t evaluation_d2h_bytes;
  uint64_t evaluation_h2d_calls;
  uint64_t evaluation_d2h_calls;
  uint64_t evaluations;
  uint64_t m2l_classes;          /* distinct translation vectors used (<= 316) */
  uint64_t m2l_interactions;     /* list2 pairs summed over levels */
  uint64_t m2l_matrix_bytes;
  uint64_t p2p_pairs;            /* list1 (target, source) pairs, self included */
  uint64_t kernel_launches_last; /* kernels launched by the last evaluate */
  int32_t m2l_mode_resolved;
  int32_t timing_enabled;
  int32_t m2l_tc_m_tiles;        /* tensor-core M2L shape last used: accumulators per CTA */
  int32_t m2l_tc_stages;         /*   and pipeline stages (chosen by the autotuner in AUTO mode) */
  int32_t backward_reused_forward; /* last backward reused the forward's moments and locals */
  int32_t m2l_tc_fused;          /*   1: hi and lo translation tiles side by side in one wider MMA */
  double ms_gather, ms_p2m, ms_m2m, ms_m2l, ms_l2l, ms_l2p, ms_p2p, ms_total;
  /* Concurrent trace of the last evaluate (timing mode 2; ms from its start,
   * device events on the streams the stages ran on): near field begin / end,
   * far field begin (P2M), M2L begin, far field end (after L2L), end. */
  double trace_p2p_begin, trace_p2p_end, trace_far_begin, trace_m2l_begin, trace_far_end, trace_end;
  int32_t schedule_last;         /* CDFMM_B200_SCHEDULE_* the last evaluate ran */
  int32_t near_tc_last;          /* 1: the last evaluate's near field ran on the tensor cores */
  /* Plan construction, host wall-clock ms: the device octree (points plans),
   * positions / permutations, near-field work units and close pairs,
   * operators, interaction statistics, state buffers and kernel set-up, the
   * tensor-core M2L set-up, and the whole call. */
  double setup_ms_tree, setup_ms_geometry, setup_ms_near, setup_ms_operators, setup_ms_statistics,
      setup_ms_buffers, setup_ms_m2l, setup_ms_total;
  /* Tensor-core near field (set when its layout is built): the sum over work
   * units of the MMA reduction length, 3 x the unit's sources padded to whole
   * chunks.  Issued tensor work per evaluation = 2 x 128 rows x 3 products x
   * near_tc_k_cols x 16 ceil(K / 16) FLOP. */
  uint64_t near_tc_k_cols;
} cdfmm_b200_stats;

/* Library / device probing.  Returns OK and *count = 0 when no device. */
int cdfmm_b200_device_count(int32_t *count);

/* Name and compute capability of a device (the reference's
 * cuda_device_description, include/cdfmm/uniform_fmm.hpp:89-90 upstream). */
int cdfmm_b200_device_info(int32_t device, char *name, size_t name_len, int32_t *cc_major,
                           int32_t *cc_minor);

/* Build operators and upload the geometry (the reference's CudaFullPlan ctor,
 * src/cuda_fmm.cu:2937-3155 upstream).  Host arrays may be freed on return. */
int cdfmm_b200_plan_create(const cdfmm_b200_plan_desc *desc, cdfmm_b200_plan **out_plan);

/* Root cube parts a cdfmm_b200_points_desc gives explicitly
 * (UniformTreeOptions.root_centre / root_half_width, include/cdfmm/
 * uniform_tree.hpp upstream); parts not given come from the bounding box. */
#define CDFMM_B200_ROOT_CENTRE 1
#define CDFMM_B200_ROOT_HALF_WIDTH 2

/* Plan geometry given as raw user-order positions: the uniform octree is
 * built on the device.  The root cube, leaf keys, stable leaf ordering and
 * leaf ranges equal upstream UniformTree's (src/uniform_tree.cpp:129-357)
 * bit for bit, so the plan is the one cdfmm_b200_plan_create builds from the
 * host tree of the same points. */
typedef struct cdfmm_b200_points_desc {
  int32_t struct_size;             /* sizeof(cdfmm_b200_points_desc) */
  int32_t n_sources;               /* >= 0 */
  int32_t n_targets;               /* >= 0; ignored when target_positions is NULL */
  int32_t order;                   /* expansion order p, 0..10 */
  int32_t depth;                   /* tree max_level, 0..8 */
  int32_t max_states;              /* largest K passed to one evaluate call, >= 1 */
  int32_t m2l_mode;                /* CDFMM_B200_M2L_* */
  int32_t device;                  /* CUDA device ordinal */
  int32_t root_flags;              /* CDFMM_B200_ROOT_* bits */
  int32_t positions_on_host;       /* nonzero: positions are host arrays, else device arrays */
  double root_centre[3];           /* used with CDFMM_B200_ROOT_CENTRE */
  double root_half_width;          /* used with CDFMM_B200_ROOT_HALF_WIDTH, > 0 */
  const double *source_positions;  /* [n_sources][3] FP64, user order */
  const double *target_positions;  /* [n_targets][3] FP64, user order; NULL: the targets are the sources */
  int32_t self_map;                /* nonzero (targets NULL only): target i is source i, as upstream's
                                      identity policy sets it for targets == sources
                                      (src/uniform_fmm.cpp:1028-1043) */
  int32_t reserved0;
} cdfmm_b200_points_desc;

/* Builds the tree on the device and then the plan as cdfmm_b200_plan_create
 * does (the reference's UniformFmm constructor, src/uniform_fmm.cpp:370-717,
 * plus CudaFullPlan's set-up).  A point outside an explicit root box, or a
 * non-finite coordinate, is CDFMM_B200_ERR_INVALID_ARGUMENT ("Point lies
 * outside the requested root box", the host tree's message).  Device
 * positions must be complete when the call is made. */
int cdfmm_b200_plan_create_from_points(const cdfmm_b200_points_desc *desc, cdfmm_b200_plan **out_plan);

/* The plan's tree, for callers that built it with
 * cdfmm_b200_plan_create_from_points: root (centre x, y, z, half width),
 * permutations (sorted index -> user index), leaf offsets ([8^depth + 1])
 * and Morton-sorted FP64 positions ([n][3]).  Any NULL output is skipped. */
int cdfmm_b200_plan_tree(cdfmm_b200_plan *plan, double *root, int32_t *source_permutation,
                         int32_t *target_permutation, int32_t *leaf_source_offsets, int32_t *leaf_target_offsets,
                         double *sorted_source_positions, double *sorted_target_positions);

/* Releases every device allocation of the plan.  NULL is ignored. */
void cdfmm_b200_plan_destroy(cdfmm_b200_plan *plan);

/* Uniformly magnetised cuboid sources (upstream SourceGeometry::UniformCuboid,
 * include/cdfmm/cuboid.hpp; UniformFmmOptions.source_sizes / use_cuboid_p2m).
 * sizes: [count][3] side lengths (hx, hy, hz) > 0 in physical units, one per
 * source in USER order (count == n_sources) or one for all (count == 1);
 * count == 0 returns to point dipoles.  Moments stay total moments (m = V M).
 * The near field then applies each pair's exact cuboid -> point
 * moment-to-field tensor (upstream src/cuboid.cpp:150-180), computed once
 * here in FP64 from the FP64 positions and kept in FP32 on the device
 * (24 bytes per list-1 pair; ERR_OUT_OF_MEMORY when they do not fit); self
 * pairs are included (the self map is not applied, as upstream) and the
 * potential stays the point dipole's.  cuboid_p2m nonzero: the multipoles
 * average each source's monomials over its cuboid (upstream
 * src/static_operators.cpp:222-255), else they treat sources as points.
 * Reverse mode is refused for cuboid sources (ERR_LOGIC). */
int cdfmm_b200_set_source_cuboids(cdfmm_b200_plan *plan, const double *sizes, int32_t count, int32_t cuboid_p2m);

/* Sets the target -> source self-exclusion map in SORTED numbering
 * ([n_targets], -1 = no self source), or clears it when NULL.  The list1 P2P
 * skips exactly that source for each target (upstream
 * src/uniform_fmm.cpp:1028-1043 builds the same sorted map from user
 * identities).  Coordinate equality is never used as identity. */
int cdfmm_b200_set_self_indices(cdfmm_b200_plan *plan, const int32_t *sorted_self_indices);

/* Runs P2M -> M2M -> M2L -> L2L -> L2P plus list1 P2P for K states and writes
 * the results in user target order (the reference's UniformFmm::evaluate_into_float32
 * with CudaFull, src/uniform_fmm.cpp:1281-1349 upstream, generalised to K states,
 * potential output and device-resident arrays).
 * Expired bounded waits: the tensor-core M2L gives up a wait after about 2 s
 * (nothing faults or hangs); the locals it could not finish are set to NaN,
 * so the affected results are NaN, never stale values.  A call that waits for
 * its results (synchronize, host arrays or stage timing) returns
 * CDFMM_B200_ERR_TIMEOUT when its own work expired; for a call that returns
 * before its work is done, cdfmm_b200_poll_status reports it later. */
int cdfmm_b200_evaluate(cdfmm_b200_plan *plan, const cdfmm_b200_eval_args *args);

/* Non-blocking report of expired bounded waits (no counterpart in the
 * reference, whose evaluate always blocks): CDFMM_B200_ERR_TIMEOUT if the
 * completed GPU work of any evaluate, backward or noalloc call on this plan
 * (or on its transposed plan) recorded an expired wait that no synchronous
 * call has reported yet, else CDFMM_B200_OK.  Work still in flight is not
 * seen: synchronise the call's stream first to include it.  Each failure is
 * reported once. */
int cdfmm_b200_poll_status(cdfmm_b200_plan *plan);

/* Failure injection for tests (no counterpart in the reference): sets how
 * many times each pipeline progress wait of the tensor-core M2L polls its
 * mbarrier before it gives up (0: every such wait expires at once; negative:
 * the default, about 2 s).  The waits that drain copies and MMAs already in
 * flight after an expiry always keep the default, so an injected expiry ends
 * the kernel cleanly.  Applies to the plan and its transposed plan. */
int cdfmm_b200_set_wait_limit(cdfmm_b200_plan *plan, int64_t iterations);

/* Allocation-free variant of cdfmm_b200_evaluate (no counterpart in the
 * reference).  For callers that cannot call cudaMalloc/cudaFree while they
 * evaluate -- a framework whose memory pool owns the device memory, a program
 * that reserves all its device memory up front, a real-time loop that cannot
 * take the allocator's implicit synchronisation.  Same
 * arguments and results as cdfmm_b200_evaluate, with these limits:
 *  - moments and results must be device-resident (args->memory == 0);
 *  - all per-call scratch (sorted moments, expansions, near field, tensor-
 *    core operands) lives in one fixed 64 MiB device array built into the
 *    library, so the plan's size times n_states must fit in it; larger calls
 *    fail with CDFMM_B200_ERR_INVALID_ARGUMENT and a message giving the need;
 *  - the first call on a device looks up that array's device address
 *    (cudaGetSymbolAddress): make it before any stream capture starts;
 *  - every call shares the array: calls whose GPU work overlaps race, so
 *    order them on one stream;
 *  - the device address is looked up once per device for the life of the
 *    process: do not use this entry point after cudaDeviceReset (or any
 *    other reset of the device's primary context) in the same process;
 *  - its expansions stay in the scratch array: cdfmm_b200_read_expansions
 *    keeps returning those of the last cdfmm_b200_evaluate.
 * Expired waits are reported as for cdfmm_b200_evaluate (this call when it
 * synchronises, else cdfmm_b200_poll_status).
 * The plan itself is created (and allocated) by cdfmm_b200_plan_create. */
int cdfmm_b200_evaluate_noalloc(cdfmm_b200_plan *plan, const cdfmm_b200_eval_args *args);

/* Reverse mode (no counterpart in the reference, whose evaluate is not
 * differentiable).  For a loss L = sum_k sum_i w_ik . H_ik of the field of
 * cdfmm_b200_evaluate, with w = dL/dH given:
 *  - grad_moments[k][j][c] = dL/dm_jkc, the exact transpose of the evaluated
 *    (discrete, FP32) FMM applied to w: the same FMM with sources and targets
 *    exchanged, run by a transposed plan that the first call builds (it
 *    needs a one-to-one self map);
 *  - grad_target_positions[i][c] = dL/dx_ic summed over the states, from the
 *    second derivatives of the leaf local expansions (one Taylor order beyond
 *    L2P) and the analytic gradient of the list1 pair field; this needs the
 *    forward moments, whose far pass is recomputed.
 * Arrays use user order and physical units like cdfmm_b200_evaluate. */
typedef struct cdfmm_b200_backward_args {
  int32_t struct_size;          /* sizeof(cdfmm_b200_backward_args) */
  int32_t n_states;             /* K, 1..max_states */
  const float *grad_field;      /* [n_states][n_targets][3] dL/dH */
  const void *moments;          /* [n_states][n_sources][3] forward moments (for grad_target_positions) */
  int32_t moments_dtype;        /* 0 = float32, 1 = float64 */
  float *grad_moments;          /* [n_states][n_sources][3] output, or NULL */
  float *grad_target_positions; /* [n_targets][3] output (sum over states), or NULL */
  uint32_t memory;              /* MOMENTS_ON_HOST: grad_field and moments on the host;
                                   RESULTS_ON_HOST: the outputs on the host */
  void *stream;                 /* cudaStream_t; NULL = the legacy default stream */
  int32_t synchronize;          /* nonzero: return only after the outputs are complete */
  uint64_t forward_evaluation;  /* the plan's `evaluations` counter (cdfmm_b200_get_stats) read right
                                   after the forward evaluate of these moments, or 0.  If no evaluate
                                   on the plan happened since and that one kept all n_states (device
                                   arrays, or fewer than 128 states), its sorted moments and leaf
                                   locals are reused instead of recomputed (moments may then be NULL). */
} cdfmm_b200_backward_args;
int cdfmm_b200_backward(cdfmm_b200_plan *plan, const cdfmm_b200_backward_args *args);

/* Multi-geometry batches (no counterpart in the reference, which evaluates
 * one UniformFmm per call).  A batch evaluates `count` plans -- independent
 * geometries of any sizes, each with its own arguments -- with ONE CUDA graph
 * launch: cdfmm_b200_batch_create evaluates each plan once (building its
 * work tiles and tuning its M2L), then captures all the evaluations into one
 * graph whose per-geometry branches run concurrently.  Arguments are fixed at
 * creation and must be device-resident (memory == 0); a plan appears at most
 * once per batch and must not be evaluated by other calls while the batch is
 * in use (the batch replays into the plan's own buffers); stage timing is
 * switched off on the plans. */
typedef struct cdfmm_b200_batch cdfmm_b200_batch;
int cdfmm_b200_batch_create(cdfmm_b200_plan *const *plans, const cdfmm_b200_eval_args *args, int32_t count,
                            cdfmm_b200_batch **out_batch);
/* One graph launch on `stream` (NULL = legacy default stream); with
 * synchronize nonzero, waits and returns CDFMM_B200_ERR_TIMEOUT if a plan's
 * work recorded an expired bounded wait.  Each launch counts as one
 * evaluation of every plan of the batch (the `evaluations` counter), so a
 * backward call cannot reuse expansions from before the launch. */
int cdfmm_b200_batch_launch(cdfmm_b200_batch *batch, void *stream, int32_t synchronize);
/* Stacked M2L groups of a batch: plans evaluated with one state each whose
 * M2L runs on the tensor cores are grouped by (depth, order); a group of two
 * or more runs ONE M2L with its plans as the states (their normalised M2L
 * operators are the same), instead of one M2L per plan.  Writes each plan's
 * group (or -1: evaluated on its own) into out[capacity] and returns the
 * plan count.  A stacked plan's results may differ from its own evaluate at
 * FP32 rounding level (the group's M2L pipeline shape is chosen for the
 * group). */
int cdfmm_b200_batch_groups(const cdfmm_b200_batch *batch, int32_t *out, int32_t capacity);
void cdfmm_b200_batch_destroy(cdfmm_b200_batch *batch);

/* Copies the FP32 multipole (which = 0) or local (which = 1) expansions of one
 * state of the last cdfmm_b200_evaluate (cdfmm_b200_evaluate_noalloc keeps its
 * expansions in its scratch array and does not update these) to host memory
 * as out[node][coefficient], node in
 * flat level-wise Morton order and coefficients in the total-degree basis
 * order; the values are in the normalised units of the reference FP32 plan
 * (UniformFmm::multipole_float32 / local_float32, include/cdfmm/uniform_fmm.hpp:262-269 upstream). */
int cdfmm_b200_read_expansions(const cdfmm_b200_plan *plan, int32_t which, int32_t state,
                               float *out, size_t out_count);

/* Timing of evaluate: 0 off; 1 per-stage CUDA-event times (the stages run
 * one after another on the caller's stream, ms_* fields); 2 a trace of the
 * concurrent schedule as it normally runs (trace_* fields; the call then
 * waits for its work). */
int cdfmm_b200_set_timing(cdfmm_b200_plan *plan, int32_t enabled);

/* Near/far schedule for evaluations of K > 1 states (no counterpart in the
 * reference, which overlaps a cuSPARSE near field with its M2L on two
 * streams, src/cuda_fmm.cu:3295-3300, 3386-3391 upstream):
 * CDFMM_B200_SCHEDULE_*.  Both schedules compute the same sums; the near
 * field's summation order differs between them (state blocks of 64 vs 32)
 * and the M2L pipeline shape may too, at FP32 rounding level.  Evaluations
 * whose M2L runs on the FP32 SIMT path always run SEPARATE. */
int cdfmm_b200_set_schedule(cdfmm_b200_plan *plan, int32_t schedule);

/* Near-field arithmetic for evaluations of 8 <= K <= 128 states (no
 * counterpart in the reference, whose CudaFull near field is an FP32
 * cuSPARSE product with stored pair tensors, src/cuda_fmm.cu:3295-3300
 * upstream): CDFMM_B200_NEAR_*.  The tensor-core form computes the pair
 * tensors of each work unit of up to 32 targets on the fly and multiplies
 * them with the states' moments as TF32 hi/lo splits (three products, FP32
 * accumulation: FP32-level accuracy; results differ from the FP32 SIMT form
 * at rounding level).  It takes the evaluations that compute every state in
 * one near-field pass on the device (cdfmm_b200_evaluate with device arrays,
 * or host arrays of fewer than 32 states; a backward pass's transposed
 * evaluation and its near-field position gradient too); streamed host-array
 * evaluations, cuboid sources and cdfmm_b200_evaluate_noalloc keep the FP32
 * form.  Its
 * per-plan blocks and operand buffers (about 96 bytes per source and state)
 * are allocated on its first use. */
int cdfmm_b200_set_near_mode(cdfmm_b200_plan *plan, int32_t mode);

int cdfmm_b200_get_stats(const cdfmm_b200_plan *plan, cdfmm_b200_stats *out);

/* Tensor-core M2L pipeline shapes (no counterpart in the reference, whose
 * CudaFull M2L has one fixed shape).  cdfmm_b200_m2l_shapes writes up to
 * `capacity` shapes as (accumulators per CTA, stages, fused) triples into
 * `out` ([capacity][3], may be NULL with capacity 0) and returns how many the
 * plan supports (negative: an error code).  By default the first
 * tensor-core evaluate of each K times them all and keeps the fastest; shapes
 * that differ only in accumulators or stages give bit-identical results,
 * the fused form (A_hi x [B_hi | B_lo] in one MMA) differs at FP32 rounding,
 * so timing noise can switch results at that level between runs.
 * cdfmm_b200_set_m2l_shape pins one of the listed shapes (no timing, the
 * same results on every run); m_tiles = 0 returns to autotuning. */
int cdfmm_b200_m2l_shapes(const cdfmm_b200_plan *plan, int32_t *out, int32_t capacity);
int cdfmm_b200_set_m2l_shape(cdfmm_b200_plan *plan, int32_t m_tiles, int32_t stages, int32_t fused);

/* FP64 O(N*M) direct sum on the device with explicit self exclusion: the
 * oracle-grade reference field (upstream validation.cpp:71-111 on the CPU and
 * dipole_field_kernel, src/cuda_fmm.cu:518-569).  Host arrays in user order;
 * self_indices may be NULL; phi and/or H may be NULL to skip them. */
int cdfmm_b200_direct_fp64(int32_t device, int32_t n_sources, const double *source_positions,
                           const double *moments, int32_t n_targets,
                           const double *target_positions, const int32_t *self_indices,
                           double *phi, double *field);

/* Failure-detection self-test (no counterpart in the reference): launches a
 * kernel whose bounded mbarrier wait cannot complete (nothing arrives) with a
 * short iteration limit -- the mechanism every wait of the tensor-core M2L
 * uses -- and returns CDFMM_B200_ERR_TIMEOUT when the wait gave up, set the
 * device error flag and returned; the device context stays usable.  Nothing
 * faults, traps or hangs. */
int cdfmm_b200_selftest_bounded_wait(int32_t device);
/* FP64 O(N*M) direct position gradient: grad[i] = d/dx_i (weights_i . H_i) with
 * explicit self exclusion (no counterpart in the reference; the validation
 * reference of cdfmm_b200_backward's grad_target_positions).  Host arrays in
 * user order; self_indices may be NULL. */
int cdfmm_b200_direct_grad_fp64(int32_t device, int32_t n_sources, const double *source_positions,
                                const double *moments, int32_t n_targets, const double *target_positions,
                                const int32_t *self_indices, const double *weights, double *grad);
/* The FP64 M2L matrix the plan generates for translation R = target centre -
 * source centre: out[beta + n*alpha] = D^{alpha+beta} G(R), n = (p+1)(p+2)(p+3)/6
 * (the reference's build_static_m2l_matrix, src/static_operators.cpp:159-184,
 * and its Python static_m2l_matrix, python/bindings.cpp:932-943).  Host only. */
int cdfmm_b200_m2l_matrix(int32_t order, const double *R, double *out, size_t out_count);

/* The 343 normalised M2L matrices of one order as plans use them
 * ([343][n][n], slot (tx+3)*49 + (ty+3)*7 + (tz+3) for the translation
 * t = target box - source box; slots inside the 3x3x3 near stencil are zero).
 * They are computed once per process and order, and kept on disk, one file
 * per order, when the environment variable CDFMM_B200_OPERATOR_CACHE names a
 * directory (a file that fails its header or checksum check is recomputed
 * and rewritten).  *source (optional) = 0 computed, 1 from this process's
 * cache, 2 read from the directory.  Host only. */
int cdfmm_b200_m2l_stencil(int32_t order, double *out, size_t out_count, int32_t *source);

/* The traceless reduction both M2L paths apply at `order` (no counterpart in
 * the reference, which applies the full basis): counts[4] = {n_in, n_out,
 * fold entries, derived locals}; with non-NULL arrays (sized from a first
 * call with NULLs) also in_ranks[n_in] (full ranks of the folded moments),
 * out_ranks[n_out] (of the computed locals), fold_offsets[n_in + 1],
 * fold_ranks / fold_coefficients[fold entries] (folded moment j =
 * sum over its entries of coefficient x M[rank]) and derived[3 x derived
 * locals] (rank d, s1, s2: L_d = -(L_s1 + L_s2), in evaluation order).
 * Host only. */
int cdfmm_b200_m2l_traceless(int32_t order, int32_t *counts, int32_t *in_ranks, int32_t *out_ranks,
                             int32_t *fold_offsets, int32_t *fold_ranks, int32_t *fold_coefficients,
                             int32_t *derived);

/* Message of the last failure on this plan (or of the last failure of a call
 * without a plan, on this thread, when plan is NULL).  Never NULL. */
const char *cdfmm_b200_last_error(const cdfmm_b200_plan *plan);

#ifdef __cplusplus
}
#endif

#endif /* CDFMM_B200_H */
