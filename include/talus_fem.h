/*
 * talus_fem.h -- C ABI of the B200 deformable-body (tet FEM) step.
 *
 * This is the drop-in boundary for Talus's tet FEM step.  Each entry point
 * names the reference interface it replaces (paths relative to the
 * d-adel/talus project).  Plain pointers and sizes only; status codes, no
 * exceptions.  The caller owns every host buffer; the library owns device
 * memory behind opaque handles.  Implemented by talus_b200/libtalus_fem.so
 * with hand-written sm_100a kernels; there is no CPU fallback: without a
 * usable CUDA device every entry point that needs one returns
 * TL_ERR_NO_DEVICE.
 */
#ifndef TALUS_FEM_H
#define TALUS_FEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TL_ABI_VERSION 1

/* Status codes. */
#define TL_OK 0
#define TL_ERR_ARG 1            /* bad argument or size */
#define TL_ERR_CUDA 2           /* a CUDA call failed */
#define TL_ERR_NOT_CONVERGED 3  /* reported, not fatal: a PCG or Newton cap was hit */
#define TL_ERR_NONFINITE 4      /* a NaN/Inf reached the state (StepReport::nonFinite, solver.h:278) */
#define TL_ERR_TIMEOUT 5        /* a device-side wait ran out; the context stays usable */
#define TL_ERR_UNSUPPORTED 6    /* feature outside this library's scope (e.g. floating bodies) */
#define TL_ERR_NO_DEVICE 7      /* no CUDA device / extension unusable */
#define TL_ERR_TOO_LARGE 8      /* input exceeds a fixed capacity (tl_step_noalloc) */

/* Arithmetic of a resident system. */
#define TL_FP64 0        /* plain FP64 GPU step */
#define TL_FP32_MIXED 1  /* FP32 bulk; FP64 element kinematics, Dm^-1, J and reductions */

/* Element law. */
#define TL_LAW_COROTATED 0  /* reference tet law: corotated + J2 return map (material.cc:236-265, 978-1057) */
#define TL_LAW_SNH 1        /* stable neo-Hookean (neohookean.cc:41-47, 183-192) at one point per tet */

/* tl_settings.flags */
#define TL_FLAG_PROFILE 1u  /* time the element pass, node assembly and PCG launches with CUDA events */
#define TL_FLAG_TRACE 2u    /* record each PCG launch's iteration count (synchronises after every solve) */

/* Host buffer element type for state transfer. */
#define TL_DTYPE_F32 0
#define TL_DTYPE_F64 1

/* RigidSplit (solver.h:28-32). */
#define TL_RIGID_SPLIT_OFF 0
#define TL_RIGID_SPLIT_UNPROJECTED 1
#define TL_RIGID_SPLIT_PROJECTED 2

typedef struct tl_ctx tl_ctx;
typedef struct tl_system tl_system;

/* talus::PhysicalMaterial (src/talus/material.h:12-29): the fields the tet
 * step reads (solver.cc:39-55: elasticOf, plasticOf). */
typedef struct tl_material {
  double density;
  double youngs_modulus;
  double poissons_ratio;
  double stiffness_damping;  /* >0: rigid-motion-free stiffness damping, corotated law only (factor.cc:755-855);
                                tl_step_noalloc returns TL_ERR_UNSUPPORTED for it */
  double yield_stress;       /* +inf: never yields (material.cc:747-749) */
  double hardening_modulus;
} tl_material;

/* The tet fields of talus::PreparedMesh (src/talus/mesh.h:11-44) for one
 * body, plus two extensions: a per-element Young's modulus override and a
 * velocity for anchored nodes (zero reproduces the reference's fixed anchors,
 * solver.cc:3784-3789, 5833-5838). */
typedef struct tl_mesh_desc {
  uint32_t nodes;
  uint32_t tets;
  const double* rest_positions;      /* [3*nodes] PreparedMesh::restPositions */
  const double* node_mass;           /* [nodes]   PreparedMesh::nodeMass */
  const uint8_t* anchored;           /* [nodes]   PreparedMesh::anchored */
  const uint32_t* tet_nodes;         /* [4*tets]  PreparedTet::nodes */
  const double* rest_inverse;        /* [9*tets]  PreparedTet::restInverse, row-major */
  const double* volume;              /* [tets]    PreparedTet::volume */
  const uint32_t* material;          /* [tets]    PreparedTet::material (lane) */
  const tl_material* materials;      /* [lanes]   std::span<const PhysicalMaterial> */
  uint32_t lanes;
  const double* element_youngs;      /* [tets] or NULL */
  const double* prescribed_velocity; /* [3*nodes] or NULL */
} tl_mesh_desc;

/* talus::deformable::Settings (src/talus/deformable/solver/solver.h:51-107):
 * the fields the non-contact tet path reads. */
typedef struct tl_settings {
  uint32_t substeps;        /* 1   (solver.h:52) */
  uint32_t cg_iterations;   /* 64  (solver.h:53) */
  uint32_t plastic_passes;  /* 40  (solver.h:56) */
  uint32_t rigid_split;     /* TL_RIGID_SPLIT_PROJECTED (solver.h:66) */
  uint32_t law;             /* TL_LAW_* */
  uint32_t flags;           /* TL_FLAG_* */
  double tolerance;         /* 1e-3 (solver.h:64) */
  double spectral_radius;   /* 0.5  (solver.h:65) */
} tl_settings;

/* talus::deformable::StepReport (solver.h:211-311): the counters of the
 * non-contact tet path, per body, accumulated (+=) like the reference
 * (solver.cc:3612-3615, 5881-5882). */
typedef struct tl_step_report {
  uint32_t nodes;
  uint32_t elements;
  uint32_t substeps;
  uint32_t cg_iterations;
  uint32_t cg_capped_solves;
  uint32_t plastic_evaluations;
  uint32_t plastic_solves;
  uint32_t plastic_backtracks;
  uint32_t plastic_capped;
  uint32_t plastic_linear_reads;
  uint32_t plastic_handoffs;
  uint32_t plastic_fallbacks;
  uint32_t plastic_fallback_rejections;
  uint32_t operator_applications;
  uint32_t yielding;
  uint32_t plastic_growth;
  uint32_t non_finite;
  uint32_t kernel_launches;
  uint32_t cg_tangent_iterations;  /* PCG iterations run with the consistent plastic tangent */
  uint32_t cg_solves;
  double cg_worst_relative_residual;
  double plastic_worst_residual;
  double elastic_energy;
  double kinetic_energy;
  double min_volume_ratio;
  double device_seconds;
  double element_seconds;   /* TL_FLAG_PROFILE: element-pass kernels */
  double assemble_seconds;  /* TL_FLAG_PROFILE: node gather + balance kernels, and the single-body
                               PCG's block-matrix assembly */
  double pcg_seconds;       /* TL_FLAG_PROFILE: persistent PCG launches */
} tl_step_report;

/* Library version (TL_ABI_VERSION); works without a device. */
int32_t tl_abi_version(void);
const char* tl_status_string(int32_t status);

/* Device context: one CUDA device and one stream.  No reference
 * counterpart: Talus is CPU-only. */
int32_t tl_ctx_create(int32_t device, tl_ctx** out);
int32_t tl_ctx_destroy(tl_ctx* ctx);
const char* tl_ctx_last_error(const tl_ctx* ctx);

/* Failure-detection self test, no reference counterpart.  Launches one block
 * at the grid barrier of the persistent PCG kernels, waiting for an arrival
 * that never comes.  The wait is bounded (2 s), so it runs out and the call
 * returns TL_ERR_TIMEOUT, the status a stalled persistent kernel reports.
 * The context stays usable.  Exercises the timeout path without faulting or
 * hanging the GPU. */
int32_t tl_ctx_check_wait_limit(tl_ctx* ctx);

/* Failure injection on the host, no reference counterpart.  Arms the next
 * tl_step of `system` so that its PCG solve number `solve` (0 = the step's
 * first solve; < 0 disarms) is preceded by the same bounded wait as
 * tl_ctx_check_wait_limit on the system's barrier word: the wait runs out
 * (about 2 s) and records TL_ERR_TIMEOUT, that solve and every later solve of
 * the step leave at their first barrier, and the step returns TL_ERR_TIMEOUT.
 * The arming is used once.  The system stays usable: the next step clears the
 * record and runs normally.  No GPU fault or hang is involved. */
int32_t tl_system_expire_wait(tl_system* system, int32_t solve);

/* Upload one or more bodies (a batch when count > 1) into one resident
 * system.  Replaces buildMesh's output handling + refreshStiffness +
 * buildIncidence (solver.cc:453-507, 1065-1101): the node->element CSR
 * incidence is built here in the reference's element order.  A body must
 * look like buildMesh output (solver.cc:2352-2356): finite rest positions,
 * rest inverses and prescribed velocities, volumes > 0, masses >= 0, node
 * indices < nodes, lanes with a finite E >= 0; otherwise TL_ERR_ARG and
 * nothing is uploaded.  tl_step and tl_step_noalloc also refuse a dt that is
 * not finite and positive, and non-finite gravity. */
int32_t tl_system_create(tl_ctx* ctx, const tl_mesh_desc* bodies, uint32_t count, int32_t precision,
                         tl_system** out);
int32_t tl_system_destroy(tl_system* system);
int32_t tl_system_counts(const tl_system* system, uint32_t* bodies, uint64_t* nodes, uint64_t* tets);

/* Launch shape, no reference counterpart (chosen by talus_b200/autotune.py):
 * pcg_blocks_per_sm caps the blocks per SM of the persistent PCG grid (0 =
 * as many as can be resident); graph != 0 lets a batched system (count > 1)
 * capture its elastic step in a CUDA graph and replay it every step. */
int32_t tl_system_tune(tl_system* system, uint32_t pcg_blocks_per_sm, uint32_t graph);

/* Launch shape of the assembled-operator PCG, no reference counterpart
 * (chosen by talus_b200/autotune.py); results are bitwise the same for every
 * shape. TL_SHAPE_ROW_GROUP: column slots of a matrix row whose inputs and
 * blocks are requested per round trip, 2 or 4 (0 = the default: 4 in FP32
 * and 2 in FP64 for a single body, 2 for batches). TL_SHAPE_BATCH_BLOCKS:
 * resident 256-thread blocks per SM the batched kernels are compiled for,
 * 3 or 4 (0 = 4). Other values return TL_ERR_ARG. */
#define TL_SHAPE_ROW_GROUP 0u
#define TL_SHAPE_BATCH_BLOCKS 1u
int32_t tl_system_tune_shape(tl_system* system, uint32_t knob, uint32_t value);

/* Form of the PCG operator, no reference counterpart (the reference applies
 * it element by element, solver.cc:904-1048): TL_SOLVER_ASSEMBLED assembles
 * the 3x3 node blocks once per solve and iterates on that matrix (about 40
 * bytes per nonzero block in FP32, 76 in FP64);
 * TL_SOLVER_ELEMENTWISE always iterates element by element;
 * TL_SOLVER_AUTO (default) is ASSEMBLED for batched systems and for single
 * bodies of at least 32,768 tets, ELEMENTWISE for smaller single bodies.
 * Both forms apply the same operator; they differ in rounding.  On the
 * assembled matrix a batch (or a body too large for the single-body grid)
 * iterates in one of two orders with the same iterates in exact arithmetic:
 * TL_SOLVER_ASSEMBLED_TWO_PHASE, the textbook order with two grid barriers
 * per iteration, or TL_SOLVER_ASSEMBLED_PIPELINED, the pipelined order with
 * one barrier per iteration and its recurrences kept in FP64 (eight vectors
 * per node, in both precisions). ASSEMBLED and AUTO take the pipelined order
 * in FP64 and the two-phase order in FP32-mixed, the faster of each on the
 * 512-body batch. */
#define TL_SOLVER_AUTO 0u
#define TL_SOLVER_ASSEMBLED 1u
#define TL_SOLVER_ELEMENTWISE 2u
#define TL_SOLVER_ASSEMBLED_TWO_PHASE 3u
#define TL_SOLVER_ASSEMBLED_PIPELINED 4u
int32_t tl_system_set_solver(tl_system* system, uint32_t form);

/* The caller-held solver state of deformable::step (DeformableSolverState*,
 * factor.h:205-210; solver.cc:3606-3655, 3808-3910, 4258-4263), held by the
 * library for a one-body system.  While it is on, every step preconditions
 * its PCG with the FP64 Cholesky factor of (1 - alpha_m) M + h^2 sum R K R^T
 * made at the committed rotations of the last refresh (SystemFactor,
 * factor.cc:318-618), applied in the body's rotation since then
 * (bodyRotation, applyFactor, factor.cc:620-704).  The factor is made again
 * when it is empty or the step's h or (1 - alpha_m) changed, and, with a
 * second solve from the same start at the full iteration cap, when a solve
 * that may refresh reaches factor_budget iterations (Settings::factorBudget,
 * solver.h:54; 0: the iteration cap).  The factor is made on the host
 * (nested-dissection order, block up-looking Cholesky) and applied on the
 * device inside the PCG launch (kPcgFactor).  Needs a one-body system with
 * the assembled operator available and the corotated law on the small-strain
 * path (with or without stiffness damping, whose blocks the factor holds):
 * TL_ERR_UNSUPPORTED otherwise.  enable = 0 drops the state. */
int32_t tl_system_use_factor(tl_system* system, uint32_t enable, uint32_t factor_budget);

/* SolverStats (factor.h:28-38), the SystemFactor's size (factor.h:50-62) and
 * the StepReport factor counters (solver.h:211-311; counts summed over
 * steps, the spent / refreshed figures as last set).  factor_nonzeros counts
 * this library's L (its own ordering); system_nonzeros counts the full
 * scalar system as the reference's does. */
typedef struct tl_factor_stats {
  uint32_t factor_age;
  uint32_t refactor_count;
  uint32_t retry_count;
  uint32_t substeps_since_refresh;
  uint32_t refresh_requested;
  uint32_t fresh_retry_failed;
  double mean_iterations;
  uint32_t rows;
  uint32_t ready;
  uint64_t system_nonzeros;
  uint64_t generation;
  uint32_t refresh_requests;
  uint32_t refactors;
  uint32_t retries;
  uint32_t retries_failed;
  uint32_t wasted_iterations;
  uint32_t spent_before_refresh;
  uint32_t spent_after_refresh;
  uint32_t refreshed_at_age;
  uint32_t factor_applications;
  uint32_t reserved;
  uint64_t factor_nonzeros;
  double refactor_seconds;  /* host time spent making the factor */
} tl_factor_stats;
int32_t tl_system_factor_stats(tl_system* system, tl_factor_stats* out);

/* Plasticity of the yielding lanes.
 * TL_PLASTICITY_SMALL_STRAIN (default): the tet law's J2 return on the small
 * elastic strain inside the step, with the plastic Newton loop
 * (material.cc:594-683, 978-1057; solver.cc:3951-4250).
 * TL_PLASTICITY_HENCKY: the finite-strain flow of the reference's hex World
 * path (plasticflow.cc:96-150, 184-247), at one point per tet.  Each step is
 * elastic (corotated law) from the tet's plastic rest shape: Dm^-1 P and
 * volume V / det P (plasticRest, plasticflow.cc:263-300).  After the solve,
 * every yielding tet with det F > 0 returns F P radially in log-stretch
 * space.  The yield stress is blended as (start + r q) / (1 + r), with
 * r = H / (3 mu), and P and a hardening variable are kept per tet.  Crush
 * and plastic cap come from tl_system_set_flow_limits.
 * With HENCKY, the plastic slot of tl_state_set/get holds P (9 values,
 * row-major) and then the hardening variable.  tl_step_report::yielding
 * counts the tets that flowed.  Setting a mode resets every tet to P = I and
 * hardening 0.  HENCKY needs TL_LAW_COROTATED and no stiffness damping, and
 * does not run under rollouts (TL_ERR_UNSUPPORTED). */
#define TL_PLASTICITY_SMALL_STRAIN 0u
#define TL_PLASTICITY_HENCKY 1u
int32_t tl_system_set_plasticity(tl_system* system, uint32_t mode);

/* PhysicalMaterial's crushStress, crushLimit and plasticMax (material.h:16-29)
 * for material lane `lane` of body `body`, read by the finite-strain flow
 * only (plasticflow.cc:196-240).  A lane with a finite crush stress and a
 * crush limit < 1 compacts when squeezed below J = exp(-crushStress / K),
 * until det Fp reaches the crush limit.  A finite plasticMax caps the
 * Frobenius distance of Fp from I.  Defaults (no crush, no cap): +inf, 1,
 * +inf.  crush_stress > 0, crush_limit in (0, 1], plastic_max > 0, else
 * TL_ERR_ARG. */
int32_t tl_system_set_flow_limits(tl_system* system, uint32_t body, uint32_t lane, double crush_stress,
                                  double crush_limit, double plastic_max);

/* Diagnostics, no reference counterpart: iteration counts (body 0) of the
 * PCG launches made while TL_FLAG_TRACE was set, oldest first, since the
 * system was created.  Writes min(capacity, recorded) entries; *count gets
 * the number recorded. */
int32_t tl_system_trace(const tl_system* system, uint32_t* iterations, uint32_t capacity, uint32_t* count);

/* talus::DeformableState (mesh.h:56-62) transfer for one body.  position,
 * velocity, acceleration: [3*nodes]; rotation: [9*tets] row-major
 * CommittedTet::rotation or NULL; plastic: [10*tets] (PlasticPoint strain
 * row-major, then equivalent) or NULL.  restState (solver.cc:2420-2453) is
 * tl_state_set with rest positions and zero velocity/acceleration. */
int32_t tl_state_set(tl_system* system, uint32_t body, int32_t dtype, const void* position, const void* velocity,
                     const void* acceleration, const void* rotation, const void* plastic);
int32_t tl_state_get(tl_system* system, uint32_t body, int32_t dtype, void* position, void* velocity,
                     void* acceleration, void* rotation, void* plastic);

/* talus::deformable::step (solver.h:451-462, solver.cc:3472-5901) for every
 * body of the system, with no contacts, no rigid partners and no
 * DeformableSolverState (block-Jacobi PCG).  reports: [bodies] or NULL,
 * accumulated.  Returns TL_OK, or TL_ERR_NONFINITE when a body's state
 * became non-finite (the step still completes, like the reference's
 * nonFinite flag), or an error. */
int32_t tl_step(tl_system* system, const tl_settings* settings, const double gravity[3], double dt,
                tl_step_report* reports);

/* Page-locks a caller's host buffer (cudaHostRegister), no reference
 * counterpart: the element state of tl_state_set/get and tl_step_host then
 * moves by one DMA straight between that buffer and the device instead of
 * through the library's pinned staging.  Register whole buffers, once, and
 * unregister them before freeing them.  Either call may return TL_ERR_CUDA
 * (a range already registered, or one that was never registered). */
int32_t tl_host_register(tl_ctx* ctx, void* ptr, size_t bytes);
int32_t tl_host_unregister(tl_ctx* ctx, void* ptr);

/* Host-state convenience: upload the state, step, download it (the
 * reference's calling convention, where DeformableState lives in host
 * memory).  Same buffer layout as tl_state_set/get.  The rotations are
 * written, not read: a step sets every committed rotation before it uses
 * one (assembleElastic, solver.cc:1404-1547), so they are not uploaded and
 * tl_state_set callers may pass NULL for them before tl_step.  The plastic
 * slot crosses only when the step uses it (a yielding lane under the
 * corotated law, or TL_PLASTICITY_HENCKY); otherwise the caller's buffer is
 * left as it is, which is the state the step leaves. */
int32_t tl_step_host(tl_system* system, uint32_t body, int32_t dtype, void* position, void* velocity,
                     void* acceleration, void* rotation, void* plastic, const tl_settings* settings,
                     const double gravity[3], double dt, tl_step_report* report);

/* The last tl_step's per-substep solve records of one body: the reference's
 * StepReport::cgPerSubstep, cgStartResidual and cgEndResidual
 * (solver.h:299-301, pushed once per substep at solver.cc:4253-4256).  Per
 * substep: the PCG iterations summed over its solves, the first solve's
 * starting relative residual and the last solve's final one.  Writes
 * min(capacity, substeps, 16) entries of each non-NULL output; *count (or
 * NULL) gets the substeps the step took (0 before the first step). */
int32_t tl_step_substeps(const tl_system* system, uint32_t body, uint32_t* iterations, double* start_residual,
                         double* end_residual, uint32_t capacity, uint32_t* count);

/* Default settings (Settings{} in solver.h:51-107). */
void tl_settings_default(tl_settings* settings);

/* Internal forces of one body at the positions it holds: the element pass and
 * vertex force gather of assembleElastic (solver.cc:1354-1572) with
 * returnMapping on and no solve.  forces: [3*nodes] (N) or NULL; yielding:
 * [tets] 1 where the trial state lies outside the yield surface, else 0, or
 * NULL.  Changes no state (committed rotations and plastic points are kept).
 * For comparing the arithmetic of two systems at one configuration. */
int32_t tl_evaluate(tl_system* system, uint32_t body, const tl_settings* settings, double* forces,
                    uint8_t* yielding);

/* Per-element Young's modulus of one body ([tets], Pa), the
 * PreparedMesh-side override that tl_mesh_desc::element_youngs sets at
 * creation; lets a caller change E between rollouts without rebuilding the
 * system.  No reference counterpart (the reference reads E from the lane). */
int32_t tl_system_set_youngs(tl_system* system, uint32_t body, const double* youngs);

/* Differentiable rollout, no reference counterpart (the reference has no
 * differentiation).  A rollout is `steps` calls of tl_step on a one-body
 * system whose law is TL_LAW_SNH and whose materials do not yield, starting
 * from the state the system holds when tl_rollout_forward is called.  Each
 * step runs `newton_reads` linearised reads (the reference takes 3,
 * solver.cc:3914-3950) with the settings' PCG tolerance, so a tight
 * tolerance and >= 3 reads give a converged implicit step, which is what the
 * adjoint differentiates.  The forward keeps the state every
 * `checkpoint_every` steps; the adjoint recomputes each segment from its
 * checkpoint and runs the steps' vector-Jacobian products backwards (one
 * element pass, one PCG solve with the step's own operator and one node
 * update per step).  Steps that need more than one substep (predictor
 * inversion, solver.cc:3574-3583) are refused with TL_ERR_UNSUPPORTED. */
typedef struct tl_rollout tl_rollout;
typedef struct tl_rollout_desc {
  uint32_t steps;
  uint32_t checkpoint_every;  /* >= 1 */
  uint32_t newton_reads;      /* >= 1; 3 is the reference's count */
  uint32_t pad;
  double delta_time;
  double gravity[3];
} tl_rollout_desc;
int32_t tl_rollout_create(tl_system* system, const tl_rollout_desc* desc, const tl_settings* settings,
                          tl_rollout** out);
/* A rollout holds on to its system: destroy it before the system (the destroy
 * call itself touches only its own memory, so it is safe in any order). */
int32_t tl_rollout_destroy(tl_rollout* rollout);
/* Runs the rollout; the system ends in the final state.  report (or NULL) is
 * accumulated over the steps; *device_seconds (or NULL) gets the GPU time. */
int32_t tl_rollout_forward(tl_rollout* rollout, tl_step_report* report, double* device_seconds);
/* Cotangents of the last forward rollout.  dl_dx_final: dL/dx_T [3*nodes];
 * dl_dv_final: dL/dv_T [3*nodes] or NULL (zero).  Outputs: dl_dyoungs dL/dE
 * [tets] (per element), dl_dv0 dL/dv_0 [3*nodes], dl_dx0 dL/dx_0 [3*nodes];
 * each may be NULL.  The system is left in the final state of the forward. */
int32_t tl_rollout_adjoint(tl_rollout* rollout, const double* dl_dx_final, const double* dl_dv_final,
                           double* dl_dyoungs, double* dl_dv0, double* dl_dx0, double* device_seconds);

/* No counterpart in the reference.  One step of one small body that allocates
 * nothing, for callers that cannot call cudaMalloc: engines that run inside a
 * fixed GPU memory budget decided at start-up, and hosts that hand out device
 * memory only through their own pool and forbid libraries to allocate behind
 * their back.  Same meaning of arguments and results as tl_step_host, with
 * the mesh passed each call (per-element Young's moduli included); the
 * arithmetic is FP64.
 *
 * All device scratch lives in one fixed array inside the library
 * (TL_NOALLOC_ARENA_BYTES on every GPU that loads it, held until the process
 * exits); nothing is allocated on the device or the host heap.  Limits:
 * TL_NOALLOC_MAX_NODES nodes, TL_NOALLOC_MAX_TETS tets, TL_NOALLOC_MAX_LANES
 * material lanes (beyond them: TL_ERR_TOO_LARGE), no plastic Newton loop (a
 * yielding material with plastic_passes > 1) and no stiffness damping on a
 * lane an element uses (both TL_ERR_UNSUPPORTED).  The first call on a device
 * looks up the array's device address and loads the step's kernels (once per
 * device); make that first call before any stream capture begins.  Calls are
 * serialised inside the library; GPU work of two overlapping calls would race
 * on the shared array.  Issues its copies and kernels on the legacy default
 * stream (stream 0), synchronises it, and returns when the step has
 * finished. */
#define TL_NOALLOC_MAX_NODES 1024
#define TL_NOALLOC_MAX_TETS 4096
#define TL_NOALLOC_MAX_LANES 16
#define TL_NOALLOC_ARENA_BYTES 4194304
int32_t tl_step_noalloc(int32_t device, const tl_mesh_desc* mesh, int32_t dtype, void* position, void* velocity,
                        void* acceleration, void* rotation, void* plastic, const tl_settings* settings,
                        const double gravity[3], double dt, tl_step_report* report);

#ifdef __cplusplus
}
#endif

#endif /* TALUS_FEM_H */
