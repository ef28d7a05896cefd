/*
 * fem_oracle.h -- C API of the CPU oracle for the Talus tet FEM step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain C++ restatement of
 * talus::deformable::step (src/talus/deformable/solver/solver.cc:3472-5901,
 * contact block excluded) and of the tet element laws it calls
 * (src/talus/deformable/material/material.cc).  It exists so that tests,
 * the smoke check and the timed CPU baseline have something to compare the
 * CUDA path against.  Nothing in the product links or calls it.
 *
 * Parity status: the reference cannot be compiled here (GLM, Eigen and
 * Catch2 are fetched at configure time, CMakeLists.txt:16-39), so this
 * oracle is pinned by known-answer tests restated from the reference's own
 * law tests (tests/neohookean_tests.cc:115-199, tests/dynamics_tests.cc:
 * 119-336, tests/dynamics_strainstep_tests.cc:3090-3104) and by analytic
 * cases of the generalized-alpha integrator; results at the GLM/Eigen
 * boundary (glm::inverse, Eigen::JacobiSVD) are "parity unpinned".
 *
 * All arrays are caller-owned, row-major, double precision.  The
 * `precision` argument selects the arithmetic the restatement runs in:
 * OR_F32 reproduces the reference's own float arithmetic, OR_F64 is the
 * FP64 oracle.
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_F32 = 0, OR_F64 = 1 };
enum { OR_LAW_COROTATED = 0, OR_LAW_SNH = 1 };
enum { OR_ROTATION_POLAR = 0, OR_ROTATION_INVERTIBLE = 1 };
/* or_settings.plasticity: the tet law's small-strain J2 return inside the
 * step (material.cc:594-683, 978-1057), or the finite-strain (Hencky) flow of
 * the hex World path (plasticflow.cc:96-150, 184-247) after the step, from a
 * per-tet plastic rest shape. */
enum { OR_PLASTICITY_SMALL_STRAIN = 0, OR_PLASTICITY_HENCKY = 1 };

typedef struct or_material {
  double density;
  double youngs_modulus;
  double poissons_ratio;
  double stiffness_damping;
  double yield_stress;
  double hardening_modulus;
  /* finite-strain flow only (plasticflow.cc:196-240): PhysicalMaterial's
   * crushStress (+inf: none), crushLimit (1: none) and plasticMax (+inf) */
  double crush_stress;
  double crush_limit;
  double plastic_max;
} or_material;

typedef struct or_mesh {
  uint32_t nodes;
  uint32_t tets;
  const double* rest;          /* [3*nodes] */
  const double* node_mass;     /* [nodes] */
  const uint8_t* anchored;     /* [nodes] */
  const uint32_t* tet_nodes;   /* [4*tets] */
  const double* rest_inverse;  /* [9*tets], row-major Dm^-1 */
  const double* volume;        /* [tets] */
  const uint32_t* lane;        /* [tets] */
  const double* element_youngs;/* [tets] or NULL: per-element E override */
  const double* prescribed;    /* [3*nodes] or NULL: velocity of anchored nodes */
} or_mesh;

typedef struct or_settings {
  uint32_t substeps;        /* Settings::substeps (solver.h:52) */
  uint32_t cg_iterations;   /* Settings::cgIterations (solver.h:53) */
  uint32_t plastic_passes;  /* Settings::plasticPasses (solver.h:56) */
  uint32_t law;             /* OR_LAW_* */
  double tolerance;         /* Settings::tolerance (solver.h:64) */
  double spectral_radius;   /* Settings::spectralRadius (solver.h:65) */
  uint32_t rigid_split;     /* Settings::rigidSplit (solver.h:66): 0 = Off */
  uint32_t plasticity;      /* OR_PLASTICITY_*; with HENCKY the state's plastic
                               slot holds the plastic rest map P = Fp^-1
                               row-major (9) and the hardening variable */
} or_settings;

typedef struct or_state {
  double* position;      /* [3*nodes] */
  double* velocity;      /* [3*nodes] */
  double* acceleration;  /* [3*nodes] */
  double* rotation;      /* [9*tets] row-major CommittedTet::rotation */
  double* plastic;       /* [10*tets]: strain row-major (9) + equivalent */
} or_state;

typedef struct or_report {
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
  uint32_t reserved;
  double cg_worst_relative_residual;
  double plastic_worst_residual;
  double elastic_energy;
  double kinetic_energy;
  double seconds;
} or_report;

/* Synthetic Kuhn box grid: buildMesh (solver.cc:2185-2418) for a lattice whose
 * every cell has fill 1.  Sizes: nodes = counted by or_grid_counts. */
typedef struct or_grid {
  uint32_t cells[3];
  double voxel;            /* cube edge (m) */
  double origin[3];
  double jitter;           /* uniform +-jitter*voxel per coordinate */
  uint64_t seed;
  double density;
  uint32_t anchor_axis;    /* 0,1,2; 3 = none */
  uint32_t anchor_side;    /* 0 = low face, 1 = high face */
} or_grid;

int or_grid_counts(const or_grid* grid, uint32_t* nodes, uint32_t* tets);
int or_grid_build(const or_grid* grid, double* rest, double* node_mass,
                  uint8_t* anchored, uint32_t* tet_nodes, double* rest_inverse,
                  double* volume, uint32_t* lane, uint32_t* grid_index);

/* One talus::deformable::step (solver.cc:3472) with no contacts/partners. */
/* A caller-held solver state (talus::deformable::DeformableSolverState,
 * factor.h:205-210): the FP64 Cholesky preconditioner SystemFactor and its
 * SolverStats.  factor_budget is Settings::factorBudget (solver.h:54). */
typedef struct or_solver or_solver;

typedef struct or_solver_stats {
  /* SolverStats (factor.h:30-40) */
  uint32_t factor_age;
  uint32_t refactor_count;
  uint32_t retry_count;
  uint32_t substeps_since_refresh;
  uint32_t refresh_requested;
  uint32_t fresh_retry_failed;
  double mean_iterations;
  /* SystemFactor (factor.h:50-62) */
  uint32_t rows;
  uint32_t ready;
  uint64_t system_nonzeros;
  uint64_t generation;
  /* StepReport's factor counters (solver.h:211-311): the counts summed over
   * steps, the spent/refreshed figures as last set */
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
} or_solver_stats;

or_solver* or_solver_create(uint32_t factor_budget);
void or_solver_destroy(or_solver* solver);
int or_solver_get_stats(const or_solver* solver, or_solver_stats* out);

/* or_step with a solver state (NULL: or_step). */
int or_step_solver(int precision, const or_mesh* mesh, or_state* state,
                   const or_material* materials, uint32_t lanes,
                   const or_settings* settings, const double gravity[3], double dt,
                   or_report* report, or_solver* solver);

int or_step(int precision, const or_mesh* mesh, or_state* state,
            const or_material* materials, uint32_t lanes,
            const or_settings* settings, const double gravity[3], double dt,
            or_report* report);

/* Element laws, one tet (material.cc).  deformed/rest: [12]; rest_inverse: [9];
 * committed_plastic: [10]; outputs: force [12], rotation [9], plastic [10],
 * tangent [144] (row-major 12x12 d(force)/d(x) sign convention of
 * TetStiffness blocks, i.e. +K), scalars [4] = energy, plastic work,
 * yielding, loading. */
int or_tet_point_trial(int precision, const double* deformed, const double* rest,
                       const double* rest_inverse, double volume,
                       const or_material* material, const double* committed_plastic,
                       double margin, int rotation_mode, int return_mapping,
                       double* force, double* rotation, double* plastic,
                       double* tangent, double* scalars);

/* Corotated elastic trial (material.cc:236-265): force [12], rotation [9],
 * energy [1]. */
int or_tet_trial(int precision, const double* deformed, const double* rest,
                 const double* rest_inverse, double volume,
                 const or_material* material, int rotation_mode,
                 double* force, double* rotation, double* energy);

/* Stable neo-Hookean tet (P from neohookean.cc:183-184 at one point):
 * force [12], energy [1], hessian_blocks [144] (Gauss-Newton blocks
 * mu (g_a.g_b) I + (lambda+mu) b_a b_b^T, neohookean.cc:189-192). */
int or_snh_tet(int precision, const double* deformed, const double* rest,
               const double* rest_inverse, double volume,
               const or_material* material, double* force, double* energy,
               double* hessian_blocks);

/* polarRotation (material.cc:168-197) and the Invertible rotation
 * (material.cc:24-64). gradient/out: [9] row-major. */
/* Stiffness damping operator of one tet (factor.cc:780-853): out = D(direction),
 * the elastic stiffness rotated by `rotation` between two removals of the
 * rigid motion fitted to `corners`.  corners, direction, out: [12]. */
int or_damping_apply(int precision, const double* corners, const double* rotation, const double* rest_inverse,
                     double volume, const or_material* material, const double* direction, double* out);

int or_rotation(int precision, const double* gradient, int rotation_mode,
                double* out);

/* plasticflow.cc:96-150 returnMap of one point: elastic [9] row-major F_e,
 * shear modulus, yield stress.  Returns 1 and writes the returned elastic
 * map [9], strain = (q - yield) / (3 shear) and trial = q when the point is
 * past its yield surface, else 0. */
int or_hencky_return(const double* elastic, double shear, double yield_stress, double* returned, double* strain,
                     double* trial);

/* plasticflow.cc:96-108 vonMises: sqrt(3/2) 2 shear |dev log V_e|. */
double or_hencky_von_mises(const double* elastic, double shear);

/* plasticflow.cc:184-247 flowLattice for one point: deformation [9] F,
 * plastic [9] P = Fp^-1 and *hardening updated in place; shear and bulk
 * moduli; the material's yield stress, hardening modulus, crush stress and
 * limit and plastic cap.  Returns 1 when P changed. */
int or_hencky_flow(const double* deformation, double* plastic, double* hardening, double shear, double bulk,
                   const or_material* material);

#ifdef __cplusplus
}
#endif
