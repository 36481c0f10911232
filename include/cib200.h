/*
 * cib200.h -- C ABI of the B200 (sm_100a) material-point and periodic-RVE kernels.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream (passed as
 * `void*`, NULL = legacy default stream).  Nothing here allocates device memory for data:
 * all buffers, including solver work vectors, are passed in by the caller (the one
 * exception is cib_rve_newton_graph_create, which builds and instantiates a CUDA graph).  All calls are
 * asynchronous on the given stream.  The integer return value reports argument and
 * launch errors only (0 = launched); per-point numerical failures are reported through
 * the `first_failure` word, which the caller initialises to CIB_NO_FAILURE and reads
 * back after the stream has drained.
 *
 * Voigt order everywhere is (xx, yy, zz, yz, xz, xy) with engineering shear strains,
 * as in the reference's src/fem/assembly/elasticity.py:160-183.
 *
 * Reference interfaces replaced (paths are relative to the reference project):
 *   cib_j2vp_update_soa_*   J2ViscoplasticMaterial.update -> _update_points
 *                           (src/fem/materials/plasticity.py:110-117, 343-431),
 *                           batched incremental form with stress-carried state
 *   cib_j2vp_update         J2ViscoplasticMaterial.update, reference form: total strains,
 *                           plastic_strain / equivalent_plastic_strain /
 *                           viscoplastic_multiplier state, tangents, free energy,
 *                           dissipation and the per-point diagnostics dict
 *                           (src/fem/materials/plasticity.py:343-431, 526-708)
 *   cib_j2vp_diagnose_point the diagnostics carried by MaterialPointConvergenceError
 *                           (src/fem/materials/plasticity.py:711-904, 1441-1465;
 *                           src/fem/materials/errors.py:15-33)
 *   cib_linear_elastic_update  evaluate_linear_elastic_points
 *                           (src/fem/materials/linear_elastic.py:74-100)
 *   cib_rve_*               solve_rve_microequilibrium and its assembly
 *                           (src/fem/rve/solver.py:62-227, 253-364, 438-461;
 *                           src/fem/assembly/nonlinear_solid.py:113-180, 428-493)
 *   cib_hex8_mass_csr, cib_newmark_*, cib_csr_pcg
 *                           assemble_consistent_mass_matrix and the implicit Newmark step
 *                           (src/fem/assembly/elasticity.py:50-70, 109-140;
 *                           src/fem/dynamics/material.py:300-701)
 */
#ifndef CIB200_H
#define CIB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CIB_NO_FAILURE 0xFFFFFFFFFFFFFFFFull

/* Number of per-point diagnostic rows written by cib_j2vp_update (row-major, CIB_J2_NDIAG x n). */
#define CIB_J2_NDIAG 22

/* Error codes (returned by the entry points). */
#define CIB_OK 0
#define CIB_EINVAL (-1)   /* bad argument (null pointer, negative size, misaligned buffer) */
#define CIB_ECUDA (-2)    /* a CUDA launch failed; cib_last_cuda_error() has the code */
#define CIB_ERANGE (-3)   /* a size exceeds what the entry point supports */

/* Per-point status codes: the `reason` strings of MaterialPointConvergenceError. */
#define CIB_J2_OK 0
#define CIB_J2_NON_FINITE_J2_INVARIANT 1
#define CIB_J2_NEGATIVE_J2_INVARIANT 2
#define CIB_J2_INVALID_YIELD_ACTIVATION_TOLERANCE 3
#define CIB_J2_NON_FINITE_CLOSED_FORM 4
#define CIB_J2_CLOSED_FORM_SOLUTION_OUT_OF_BOUNDS 5
#define CIB_J2_INVALID_ITERATION_LIMIT 6
#define CIB_J2_NON_FINITE_PROBLEM_SCALE 7
#define CIB_J2_INVALID_CORRECTED_OVERSTRESS 8
#define CIB_J2_NON_FINITE_ITERATION_VALUE 9
#define CIB_J2_NON_POSITIVE_DERIVATIVE 10
#define CIB_J2_CONVERGED_SOLUTION_OUT_OF_BOUNDS 11
#define CIB_J2_NON_FINITE_NEWTON_CANDIDATE 12
#define CIB_J2_NEWTON_CANDIDATE_OUT_OF_BOUNDS 13
#define CIB_J2_MAXIMUM_ITERATIONS_EXCEEDED 14
#define CIB_J2_NON_POSITIVE_TANGENT_OVERSTRESS 15

/* J2ViscoplasticMaterial parameters (src/fem/materials/plasticity.py:80-117). */
typedef struct cib_j2vp_material {
  double young_modulus;
  double poisson_ratio;
  double yield_stress;
  double hardening_modulus;
  double time_scale;
  double reference_stress;
  double rate_exponent;
} cib_j2vp_material;

/* MaterialUpdateSettings (src/fem/materials/data.py:17-23). */
typedef struct cib_update_settings {
  int32_t max_iterations;
  int32_t pad_;
  double yield_relative_tolerance;
  double residual_absolute_tolerance;
  double residual_relative_tolerance;
} cib_update_settings;

/* Snapshot of one failed point, the fields of the reference's failure diagnostics
 * (_build_j2_newton_diagnostics, plasticity.py:857-894, and the invariant / activation
 * payloads at plasticity.py:548-563, 1441-1465). Written by cib_j2vp_diagnose_point. */
typedef struct cib_j2vp_failure {
  int32_t reason;
  int32_t iteration;
  int32_t max_iterations;
  int32_t algorithm; /* 0 local Newton, 1 equivalent stress, 2 yield activation, 3 tangent */
  double time_step;
  double shear_modulus;
  double hardening_slope;
  double trial_yield;
  double physical_upper_bound;
  double plastic_multiplier;
  double corrected_overstress;
  double residual;
  double residual_tolerance;
  double derivative;
  double newton_candidate;
  double radicand;
  double yield_scale;
  double yield_activation_threshold;
  double trial_equivalent_stress;
  double yield_radius;
  double equivalent_plastic_strain;
  double trial_stress[6];
  double deviatoric_stress[6];
  int32_t has_residual;
  int32_t has_derivative;
  int32_t has_newton_candidate;
  int32_t pad_;
} cib_j2vp_failure;

/* --- Return map, batched incremental form (structure of arrays) ------------------------
 * State carried per point: stress (6), plastic strain (6), equivalent plastic strain (1).
 * Input strain increment dstrain (6).  All 6-component arrays are SoA with leading
 * dimension ld >= n: component c of point p is at [c * ld + p]; tangent has 36 rows
 * [(6 * i + j) * ld + p] (NULL skips it); the equivalent plastic strain is a plain
 * array [p].  The trial stress is stress_n + C dstrain, which is the reference's
 * C (strain - plastic_strain) with strain = C^-1 stress_n + plastic_strain_n + dstrain.
 * The vectorised path needs 16-byte aligned buffers and ld a multiple of 4; the rest is
 * handled by a scalar path.  Inputs and outputs must not alias.  The f32 variant keeps
 * the equivalent plastic strain history in double. */
int cib_j2vp_update_soa_f64(const cib_j2vp_material* material, const cib_update_settings* settings,
                            int64_t n, int64_t ld, double time_step, const double* dstrain, const double* stress_n,
                            const double* plastic_strain_n, const double* eqps_n, double* stress,
                            double* plastic_strain, double* eqps, double* tangent,
                            unsigned long long* first_failure, void* stream);

int cib_j2vp_update_soa_f32(const cib_j2vp_material* material, const cib_update_settings* settings,
                            int64_t n, int64_t ld, double time_step, const float* dstrain, const float* stress_n,
                            const float* plastic_strain_n, const double* eqps_n, float* stress,
                            float* plastic_strain, double* eqps, float* tangent,
                            unsigned long long* first_failure, void* stream);

/* The same update with the consistent tangent in compact form: tangent8 has 8 rows
 * [r * ld + p]: the flow direction n (6), f and c, such that
 *   C = K 1 (x) 1 + f P + c n (x) n
 * with K the bulk modulus and P the deviatoric projector in engineering-shear Voigt form
 * (P_ij = delta_ij - 1/3 for i, j < 3, P_ii = 1/2 for i >= 3, else 0) -- the factored form
 * of the reference's _j2_viscoplastic_consistent_tangent (plasticity.py:929-963).  An
 * elastic point has n = 0, f = 2G, c = 0.  8 instead of 36 tangent values per point. */
int cib_j2vp_update_soa_compact_f64(const cib_j2vp_material* material, const cib_update_settings* settings,
                                    int64_t n, int64_t ld, double time_step, const double* dstrain,
                                    const double* stress_n, const double* plastic_strain_n, const double* eqps_n,
                                    double* stress, double* plastic_strain, double* eqps, double* tangent8,
                                    unsigned long long* first_failure, void* stream);

int cib_j2vp_update_soa_compact_f32(const cib_j2vp_material* material, const cib_update_settings* settings,
                                    int64_t n, int64_t ld, double time_step, const float* dstrain,
                                    const float* stress_n, const float* plastic_strain_n, const double* eqps_n,
                                    float* stress, float* plastic_strain, double* eqps, float* tangent8,
                                    unsigned long long* first_failure, void* stream);

/* --- Return map, reference form (array of structures, float64) -------------------------
 * strain (n,6), optional strain_rate (n,6) (NULL = None), state plastic_strain (n,6),
 * equivalent_plastic_strain (n), viscoplastic_multiplier (n).  Outputs: stress (n,6),
 * new state, optional tangent (n,6,6), free_energy (n), dissipation (n), and optional
 * diagnostics (CIB_J2_NDIAG rows of n, in the order given by cib_j2_diagnostic_name).
 * active_count (device uint64, may be NULL) receives the number of viscoplastic points
 * (added to its current value). */
int cib_j2vp_update(const cib_j2vp_material* material, const cib_update_settings* settings, int64_t n,
                    double time_step, const double* strain, const double* strain_rate,
                    const double* plastic_strain_n, const double* eqps_n, const double* vpm_n,
                    double* stress, double* plastic_strain, double* eqps, double* vpm, double* tangent,
                    double* free_energy, double* dissipation, double* diagnostics,
                    unsigned long long* active_count, unsigned long long* first_failure, void* stream);

/* Re-run the return map of one point of a cib_j2vp_update call and write its failure
 * snapshot to `record` (device memory, one struct). */
int cib_j2vp_diagnose_point(const cib_j2vp_material* material, const cib_update_settings* settings,
                            int64_t n, double time_step, const double* strain, const double* strain_rate,
                            const double* plastic_strain_n, const double* eqps_n, int64_t point,
                            cib_j2vp_failure* record, void* stream);

/* Linear elasticity, reference form: stress (n,6) = strain (n,6) C^T; optional tangent
 * (n,6,6), free_energy (n), dissipation (n, zeros), and, when strain_rate is given, the
 * elastic-phase diagnostics of phased.py:172-191 (incremental_work_density,
 * equivalent_stress_increment) as 2 rows of n. */
int cib_linear_elastic_update(double young_modulus, double poisson_ratio, int64_t n, double time_step,
                              const double* strain, const double* strain_rate, double* stress,
                              double* tangent, double* free_energy, double* dissipation,
                              double* increment_diagnostics, void* stream);

/* --- General Hex8 assembly (arbitrary nodes and connectivity) ---------------------------
 * nodes (N,3) float64, elements (E,8) int64 in the lexicographic node order of the
 * reference (src/fem/elements/lagrange.py:50-76), 2x2x2 Gauss rule.  Replaces the loops of
 * src/fem/assembly/nonlinear_solid.py:391-493. */

/* dN/dx per (element, Gauss point, node): grads (E*8*8*3), J*w (E*8); bad_count (device
 * uint64) is incremented for every point with det J <= 0. */
int cib_hex8_geometry(int64_t nelem, const double* nodes, const int64_t* elements, double* grads, double* jw,
                      unsigned long long* bad_count, void* stream);

/* strain (8E,6) = B u_e and, when rate is not NULL, rate (8E,6) = B (u_e - u_prev,e) / dt. */
int cib_hex8_strains(int64_t nelem, const int64_t* elements, const double* grads, const double* u,
                     const double* u_prev, double time_step, double* strain, double* rate, void* stream);

/* Internal force (3N) = sum_e sum_q w B^T sigma: element nodal forces into fe (E*8*3,
 * scratch), then a fixed-order gather per node over node_list[node_ptr[n] .. node_ptr[n+1])
 * (entries 8 e + a). */
int cib_hex8_internal_force(int64_t nelem, int64_t nnode, const double* grads, const double* jw, const double* stress,
                            const int64_t* node_ptr, const int64_t* node_list, double* fe, double* force,
                            void* stream);

/* Tangent in CSR: element matrices into ke (E*24*24, scratch) from tangents (8E,6,6), then
 * values[k] = sum of ke[csr_list[csr_ptr[k] .. csr_ptr[k+1])] in a fixed order. */
int cib_hex8_tangent_csr(int64_t nelem, const double* grads, const double* jw, const double* tangent, int64_t nnz,
                         const int64_t* csr_ptr, const int64_t* csr_list, double* ke, double* values, void* stream);

/* dst[k] = sum of src[list[ptr[k] .. ptr[k+1])] in a fixed order, k < nnz: the values of a
 * matrix whose entries are sums of another's, e.g. the reduced periodic tangent T^T K T of a
 * general RVE mesh from the CSR tangent K (src/fem/rve/solver.py:143, 438-461). */
int cib_csr_gather(int64_t nnz, const int64_t* ptr, const int64_t* list, const double* src, double* dst,
                   void* stream);

/* --- Periodic structured Hex8 RVE batch ------------------------------------------------
 * A batch holds R structured periodic RVEs (unit-cell boxes of nx*ny*nz Hex8 elements).
 * RVE r owns elements [elem_offset, elem_offset + nx*ny*nz), the RVEs one after the other
 * (elem_offset ascending, RVE 0 at 0, the last ending at nelem); its periodic node (class)
 * c = i + nx*(j + ny*k) is batch node elem_offset + c; class 0 is the eliminated
 * reference class (src/fem/rve/periodic.py:20-104).  Periodic vectors (fluctuation w,
 * residual, PCG vectors) are float64 with 3 entries per batch node.  Gauss-point arrays
 * are SoA over the 8*nelem points (point 8*e + q).  The element arithmetic type is
 * float64 or float32 (`precision`); equivalent plastic strain and the viscoplastic
 * multiplier are always float64.  All arrays are device memory except `mats`. */
#define CIB_RVE_MAX_PHASES 8
#define CIB_RVE_NOUT 130
#define CIB_PHASE_LINEAR_ELASTIC 0
#define CIB_PHASE_J2_VISCOPLASTIC 1

typedef struct cib_rve_desc {
  int32_t nx, ny, nz, pad_;
  int64_t elem_offset;
  double hx, hy, hz; /* element edge lengths */
} cib_rve_desc;

typedef struct cib_phase_material {
  int32_t kind; /* CIB_PHASE_* */
  int32_t pad_;
  cib_j2vp_material params; /* young_modulus / poisson_ratio used by both kinds */
} cib_phase_material;

typedef struct cib_rve_batch {
  int32_t nrve;
  int32_t nphase;
  int64_t nelem;             /* total elements = total periodic nodes */
  int32_t precision;         /* 64 or 32 */
  int32_t max_nxy;           /* max nx*ny over the batch (PCG shared memory) */
  const cib_rve_desc* desc;  /* device, nrve */
  const uint8_t* phase;      /* device, nelem: phase id per element */
  cib_phase_material mats[CIB_RVE_MAX_PHASES];
  cib_update_settings settings;
  /* committed Gauss-point state */
  const void* plastic_strain_n; /* T, 6 x 8*nelem */
  const double* eqps_n;         /* 8*nelem */
  const double* vpm_n;          /* 8*nelem */
  /* trial Gauss-point state and tangent data (written by cib_rve_residual) */
  void* plastic_strain;         /* T, 6 x 8*nelem */
  double* eqps;
  double* vpm;
  void* stress;                 /* T, 6 x 8*nelem */
  void* tparam;                 /* T, 8 x 8*nelem: flow direction (6), f, c */
  uint8_t* tflag;               /* 8*nelem: 1 where the consistent tangent is viscoplastic */
  /* element work arrays (caller-provided scratch) */
  double* fe;                   /* 24 * nelem: element nodal forces */
  double* de;                   /* 24 * nelem: element tangent diagonals */
  /* SoA stride of the Gauss-point arrays; 0 = 8 * nelem.  A view of the first nrve RVEs of
   * a larger batch (kernels launched over those RVEs only) keeps the larger batch's stride. */
  int64_t point_stride;
} cib_rve_batch;

/* Fused residual pass (nonlinear_solid.py:428-493 + solver.py:88-100): for every Gauss
 * point, strain = macro + B (w + alpha dw) on the periodic mesh, return map from the
 * committed state, trial state, stress, tangent data, element nodal forces w B^T sigma and
 * element tangent diagonals.  time_step and macro: 1 and 6 per RVE; dw and alpha (per RVE) may be NULL;
 * inactive RVEs (active[r] == 0) are skipped.  fail: one word per RVE, lowest failing
 * local point index (initialised to CIB_NO_FAILURE by the caller). */
int cib_rve_residual(const cib_rve_batch* batch, const double* time_step, const double* macro, const double* w,
                     const double* dw, const double* alpha, const int32_t* active, unsigned long long* fail,
                     void* stream);

/* Periodic gather of the last residual pass: reduced residual r = T^T f_int (class 0
 * removed, solver.py:97-100), inverse Jacobi diagonal, ||r||^2, ||w + alpha dw||^2 and the
 * largest class force (class 0 included) per RVE; optional w_out = w + alpha dw. */
int cib_rve_gather(const cib_rve_batch* batch, const double* w, const double* dw, const double* alpha,
                   const int32_t* active, double* residual, double* dinv, double* rnorm2, double* wnorm2,
                   double* class_max, double* w_out, void* stream);

/* Jacobi-preconditioned CG on the reduced periodic tangent of the last residual pass
 * (replaces the reference's Tt K T + spsolve, solver.py:143-144), one system per CTA:
 * system s belongs to RVE sys_rve[s] and its vectors start at sys_off[s] (doubles) in b,
 * x, r, p and Ap.  Stops when ||r|| <= rtol ||b|| or after maxit iterations; status 0
 * converged, 1 iteration limit, 2 breakdown. */
int cib_rve_pcg(const cib_rve_batch* batch, int32_t nsys, const int32_t* sys_rve, const int64_t* sys_off,
                const int32_t* active, const double* b, const double* dinv, double* x, double* r, double* p,
                double* Ap, double rtol, int32_t maxit, int32_t* status, int32_t* iterations,
                double* rel_residual, double* xnorm, void* stream);

/* cib_rve_pcg with `cluster` (1, 2, 4 or 8) CTAs of one thread-block cluster per system:
 * each CTA owns a slab of z node layers, slab boundaries are exchanged and the dot
 * products combined through distributed shared memory (fixed rank order, so results are
 * reproducible for a given cluster size).  Every RVE needs nz >= cluster (else that
 * system's status is 3); cluster 1 is cib_rve_pcg.  Bits 4-7 of `cluster` select the launch
 * shape of the cluster kernel (threads per CTA / CTAs per SM, which caps the registers):
 * 0 the default (256 / 2 in FP32, 256 / 1 in FP64), 1 (128 / 4 FP32, 128 / 2 FP64),
 * 2 (512 / 1), 3 (256 / 1 FP32, 256 / 2 FP64); results do not depend on the shape beyond
 * rounding of the CTA sums.  Same reference interface as cib_rve_pcg (Tᵀ K T + spsolve,
 * src/fem/rve/solver.py:143-144). */
int cib_rve_pcg_cluster(const cib_rve_batch* batch, int32_t nsys, const int32_t* sys_rve, const int64_t* sys_off,
                        const int32_t* active, const double* b, const double* dinv, double* x, double* r, double* p,
                        double* Ap, double rtol, int32_t maxit, int32_t cluster, int32_t* status,
                        int32_t* iterations, double* rel_residual, double* xnorm, void* stream);
/* The solve of cib_rve_pcg for callers that cannot allocate device memory -- code running
 * inside an allocator's or memory pool's own hooks, or under a host framework that forbids
 * device allocations after start-up.  No counterpart in the reference (which has no GPU
 * path).  The work vectors r, p and Ap live in one array compiled into the library:
 * 3 x CIB_PCG_NOALLOC_MAX_VEC doubles (1.5 MiB), held by every GPU that loads the library
 * until the process exits; nothing is allocated by the call.  vec_len is the length of b
 * and x (doubles) and every system's vectors must lie inside it, as for cib_rve_pcg;
 * vec_len > CIB_PCG_NOALLOC_MAX_VEC returns CIB_ERANGE without launching, and a system
 * whose vectors (sys_off .. sys_off + 3 E) would leave [0, vec_len) is skipped on the
 * device with status 3, so a wrong offset never writes outside the array.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress) and should come
 * before any stream capture; the address is looked up again when the device's context has
 * changed (after cudaDeviceReset).  All calls on a device share the array: calls that
 * overlap on the GPU race and must not be issued; no content is carried from one call to
 * the next.  Outputs and other status codes are those of cib_rve_pcg. */
#define CIB_PCG_NOALLOC_MAX_VEC 65536
int cib_rve_pcg_noalloc(const cib_rve_batch* batch, int32_t nsys, const int32_t* sys_rve, const int64_t* sys_off,
                        const int32_t* active, int64_t vec_len, const double* b, const double* dinv, double* x,
                        double rtol, int32_t maxit, int32_t* status, int32_t* iterations, double* rel_residual,
                        double* xnorm, void* stream);

/* Effective tangent (solver.py:438-461): right-hand sides K_we = T^T K A (6 columns per
 * RVE, layout [18*elem_offset + j*3*E_r + 3*c + d]) and K_ee = A^T K A (36 per RVE);
 * fe6 is scratch of 6*24*nelem doubles.  Then C = (K_ee - K_we^T S) / V from the PCG
 * solutions S (same layout). */
int cib_rve_tangent_rhs(const cib_rve_batch* batch, const int32_t* active, double* fe6, double* rhs, double* kee,
                        void* stream);
int cib_rve_tangent_finish(const cib_rve_batch* batch, const int32_t* active, const double* rhs, const double* sol,
                           const double* kee, double* ceff, void* stream);

/* Homogenisation and diagnostics of a converged state (solver.py:253-364, 464-494):
 * CIB_RVE_NOUT doubles per RVE (sums of stress, energy, work, activity and phase
 * quantities, virtual-work and reaction sums, periodicity mismatch, activation-margin
 * extrema); optional per-point outputs: point_out (14 x 8*nelem: strain 6, strain rate 6,
 * free energy, dissipation) and diagnostics (CIB_J2_NDIAG x 8*nelem). */
int cib_rve_response(const cib_rve_batch* batch, const double* time_step, const double* macro, const double* macro_n,
                     const double* w, const double* w_n, const int32_t* active, double* sums, double* point_out,
                     double* diagnostics, void* stream);

/* Device-controlled batched Newton solve of every RVE of a batch from its committed state
 * (solver.py:62-227 without the Armijo search): the residual and increment tests, the
 * per-RVE convergence and live masks, the Eisenstat-Walker forcing of the PCG tolerance
 * (inexact != 0: eta = 0.9 (max live ||r_k|| / ||r_k-1||)^2 with its safeguard, at most
 * 0.1, at least pcg_rtol) and the update w += -dw run on the device.  The whole solve is
 * one CUDA graph: w = w_n, then a conditional WHILE node whose body is residual, gather,
 * convergence check, PCG, increment check and update, repeated until every live RVE has
 * converged or an error stopped it -- no host round trip inside a step.  Afterwards the
 * trial state of every RVE is its converged state and active = live_mask.
 * Outputs in iwork / dwork (sizes from cib_rve_newton_workspace; layout below):
 *   iwork[0] iterations run, [1] error (0 none, 1 material point failure, 2 non-finite
 *   increment, 3 maximum iterations), [2] failing RVE, [3] failing local point or PCG
 *   status, [16 + r] Newton iterations of RVE r, [16 + R + r] PCG iterations of RVE r;
 *   dwork[16 + r] residual norm, [16 + R + r] residual tolerance, [16 + 2R + r] increment
 *   norm, [16 + 3R + r] increment tolerance (at the last check).
 * All pointers are device memory of the batch's buffers (the same meaning as in
 * cib_rve_residual, cib_rve_gather and cib_rve_pcg_cluster). */
typedef struct cib_rve_newton {
  int32_t max_iterations;
  int32_t inexact;
  double residual_absolute_tolerance;
  double residual_relative_tolerance;
  double increment_absolute_tolerance;
  double increment_relative_tolerance;
  double pcg_rtol;
  int32_t pcg_maxit;
  int32_t cluster; /* PCG CTAs per system (1, 2, 4, 8) and launch shape, as in cib_rve_pcg_cluster */
  const double* time_step;
  const double* macro;
  const double* w_n;
  double* w;
  double* w_out;
  double* x;
  double* r;
  double* p;
  double* Ap;
  double* residual;
  double* dinv;
  double* rnorm2;
  double* wnorm2;
  double* class_max;
  double* alpha;
  int32_t* active;
  const int32_t* live_mask; /* RVEs to solve; the others keep w = w_n and stay inactive */
  unsigned long long* fail;
  const int32_t* sys_rve;
  const int64_t* sys_off;
  int32_t* pcg_status;
  int32_t* pcg_iterations;
  double* pcg_rel_residual;
  double* pcg_xnorm;
  int32_t* iwork;
  double* dwork;
} cib_rve_newton;
void cib_rve_newton_workspace(int32_t nrve, int64_t* n_int, int64_t* n_double);
/* Build the graph (captured on a private stream; the batch struct and the settings are
 * baked in, so a change of either needs a new graph).  *graph receives an opaque handle. */
int cib_rve_newton_graph_create(const cib_rve_batch* batch, const cib_rve_newton* newton, void** graph);
int cib_rve_newton_graph_launch(void* graph, void* stream);
int cib_rve_newton_graph_destroy(void* graph);

/* --- Tensor-core MLP GEMM (recurrent material surrogate) --------------------------------
 * C[M x N] = A[M x K] . B[N x K]^T, A and B bf16 row-major (leading dimensions lda, ldb,
 * multiples of 8; 16-byte aligned), fp32 accumulation in tensor memory (tcgen05.mma).
 * N in {16, 32, ..., 128}, K a multiple of 16.  B must hold N rows.  Epilogues:
 *   0 C = acc (fp32)                      1 C = acc + bias (fp32)
 *   2 Z = acc + bias (fp32; Z may be NULL), H = gelu(Z) (bf16), optional
 *     Ht[n * ldht + row_offset + m] = H
 *   3 H = acc * gelu'(Z) (bf16), optional Ht as above
 *   4 fp32 partial sums per K slice into C[(slice * M + m) * ldc + n] (splits > 1), reduced
 *     by cib_splitk_reduce in a fixed order.
 * err (device uint32) becomes 1 if a tensor-core completion wait exceeds 2 s (the CTA then
 * returns after releasing its tensor memory).  No reference counterpart: the reference
 * runs its surrogate through torch.nn.Linear (src/concrete_impact/nn/models/rve_rno.py:63-93). */
#define CIB_EPI_F32 0
#define CIB_EPI_BIAS_F32 1
#define CIB_EPI_BIAS_GELU 2
#define CIB_EPI_GELU_BWD 3
#define CIB_EPI_PARTIAL 4
int cib_mlp_gemm(int32_t epilogue, int32_t M, int32_t N, int32_t K, const void* A, int32_t lda, const void* B,
                 int32_t ldb, int32_t splits, const float* bias, float* C, int32_t ldc, float* Z, int32_t ldz, void* H,
                 int32_t ldh, void* Ht, int32_t ldht, int32_t row_offset, unsigned int* err, void* stream);
int cib_splitk_reduce(int32_t M, int32_t N, int32_t splits, const float* partial, int32_t ldc, float* out, int32_t ldo,
                      void* stream);

/* --- Recurrent surrogate (RNO) elementwise kernels ------------------------------------
 * Per time step for B paths: x = [strain 6, strain rate 6, latent 6, zeros 14] (bf16,
 * B x 32, optional transpose Xt[c * ldxt + row_offset + p]); output Y (B x 16 fp32):
 * normalised stress (0..5) and latent rate (6..11); z' = z + coef * Y[:, 6:12] (the
 * forward-Euler latent step of src/concrete_impact/nn/models/rve_rno.py:383-387);
 * gY = loss_scale * 2 (Y[:, 0:6] - target); loss_part[block] = sum of squared errors
 * (256 paths per block). */
int cib_rno_input(int32_t B, const float* strain, const float* rate, const float* z, void* X, void* Xt, int32_t ldxt,
                  int32_t row_offset, void* stream);
int cib_rno_forward_tail(int32_t B, const float* Y, const float* target, const float* coef, const float* z,
                         float* z_next, float* gY, float loss_scale, double* loss_part, void* stream);
/* dY = [gY, coef * dz_next, 0] (bf16, B x 16) and its transpose; dz = dz_next + dX[:, 12:18]. */
int cib_rno_backward_head(int32_t B, const float* gY, const float* coef, const float* dz_next, void* dY, void* dYt,
                          int32_t lddyt, int32_t row_offset, void* stream);
int cib_rno_backward_tail(int32_t B, const float* dz_next, const float* dX, float* dz, void* stream);
/* out[n] = sum over r < R of X[n * ld + r] (bf16 rows; bias gradients). */
int cib_row_sum_bf16(int32_t rows, int32_t R, const void* X, int32_t ld, float* out, void* stream);
/* Adam with bias correction on fp32 weights (rows x cols), refreshing the bf16 copy Wb and
 * its transpose Wt when given (NULL skips).  The step number is read from device memory
 * (so a captured graph can replay it); cib_counter_increment adds one to it. */
int cib_adam_step(int32_t rows, int32_t cols, float* w, const float* g, float* m, float* v, float lr, float beta1,
                  float beta2, float eps, const int32_t* step, void* Wb, int32_t ldb, void* Wt, int32_t ldt,
                  void* stream);
int cib_counter_increment(int32_t* counter, void* stream);

/* --- Fused recurrent window (one CTA per 128 paths for all T steps) -------------------
 * Forward over a window of T steps for B paths with hidden width 128, in normalised units:
 * x = [strain, rate, z] (bf16), three bias+GELU layers, output layer Y (16);
 * s = Y[0:6] + skip (strain - z) (skip: 6x6 row-major, NULL for none), z' = z + coef Y[6:12]
 * (forward-Euler latent step, src/concrete_impact/nn/models/rve_rno.py:383-387).
 * Layout: strain, rate, target, stress, gS (T, B, 6); coef (T, B); z (T + 1, B, 6) with
 * z[0] read and z[1..T] written; W[l] bf16 row-major (out x in_pad) = 128x32, 128x128,
 * 128x128, 16x128 and Wt[l] their transposes; bias[l] fp32; Z[l] (T, B, 128) fp32
 * pre-activations; Xt (32, ldt), Ht[l] (128, ldt), dYt (16, ldt), dZt[l] (128, ldt) bf16
 * transposes with column t B + p.  Optional outputs may be NULL in the forward (Z, Xt, Ht,
 * stress, target/gS/loss_part); the backward needs Wt, Z, gS, dYt and dZt.
 * loss_part (T, ceil(B / 128)): row 0 holds each CTA's sum of squared errors over the
 * window, the other rows zero.  gS = loss_scale * 2 (s - target).  The backward runs the
 * window in reverse with dz(T) = 0 and writes dY^T, dZ^T for the weight-gradient GEMMs.
 * err (device uint32) becomes 1 when a tensor-core wait exceeds 2 s.  No reference
 * counterpart (the reference runs torch.nn layers per step). */
typedef struct cib_rno_window {
  int32_t B;
  int32_t T;
  int32_t hidden;
  float loss_scale;
  int64_t ldt; /* leading dimension of Xt, Ht, dYt, dZt (>= T B; 0 means T B) */
  const float* strain;
  const float* rate;
  const float* coef;
  const float* target;
  float* z;
  const void* W[4];
  const void* Wt[4];
  const float* bias[4];
  const float* skip;
  float* Z[3];
  void* Xt;
  void* Ht[3];
  float* stress;
  float* gS;
  double* loss_part;
  void* dYt;
  void* dZt[3];
  unsigned int* err;
} cib_rno_window;
int cib_rno_window_forward(const cib_rno_window* w, void* stream);
int cib_rno_window_backward(const cib_rno_window* w, void* stream);

/* --- Explicit macro dynamics (FE^2)---------------------------------------------------
 * Velocity-Verlet step of src/fem/dynamics/material.py:164-219 with a lumped mass and
 * homogeneous Dirichlet DOFs (fixed[i] != 0): predictor u' = u + dt v + dt^2/2 a, then
 * corrector a' = (load_scale f_unit - f_int) / m, v' = v + dt/2 (a + a'). */
int cib_verlet_predict(int64_t n, const double* u, const double* v, const double* a, const uint8_t* fixed, double dt,
                       double* u_next, void* stream);
int cib_verlet_correct(int64_t n, const double* f_unit, double load_scale, const double* f_int, const double* mass,
                       const uint8_t* fixed, double dt, const double* a, const double* v, double* a_next,
                       double* v_next, void* stream);

/* --- Implicit macro dynamics (Newmark) -------------------------------------------------
 * Device side of src/fem/dynamics/material.py:300-701 (solve_material_implicit_newmark,
 * _solve_implicit_step, _evaluate_implicit_trial) on the CSR pattern of the Hex8 tangent
 * (indptr/indices of n = 3N rows, int64).  free_mask[i] != 0 marks a free DOF; the
 * homogeneous Dirichlet DOFs are the others. */

/* Consistent mass (src/fem/assembly/elasticity.py:50-70, 109-140) in the CSR pattern and
 * gather lists of cib_hex8_tangent_csr: element matrices into me (E*24*24, scratch), then the
 * fixed-order gather into values (nnz). */
int cib_hex8_mass_csr(int64_t nelem, const double* jw, double density, int64_t nnz, const int64_t* csr_ptr,
                      const int64_t* csr_list, double* me, double* values, void* stream);

/* a = (u - u_pred) / beta_dt2 and v = v_pred + gamma_dt * a (material.py:687-688). */
int cib_newmark_kinematics(int64_t n, const double* u, const double* u_pred, const double* v_pred, double beta_dt2,
                           double gamma_dt, double* a, double* v, void* stream);

/* r = (M a + f_int) - f_ext on free rows, 0 on fixed rows (material.py:699). */
int cib_newmark_residual(int64_t n, const int64_t* indptr, const int64_t* indices, const double* mass, const double* a,
                         const double* f_int, const double* f_ext, const uint8_t* free_mask, double* r, void* stream);

/* out = k_values + m_values / beta_dt2 (material.py:540; k_values may be NULL) and the Jacobi
 * inverse diagonal dinv (1 / diag on free rows, 1 where diag <= 0, 0 on fixed rows). */
int cib_newmark_effective_tangent(int64_t n, const int64_t* indptr, const int64_t* indices, const double* k_values,
                                  const double* m_values, double beta_dt2, const uint8_t* free_mask, double* out,
                                  double* dinv, void* stream);

/* y = A x for a CSR matrix of n rows. */
int cib_csr_spmv(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values, const double* x,
                 double* y, void* stream);

/* Jacobi-preconditioned CG for A x = b on the free rows (x = 0 on fixed rows), replacing the
 * sparse direct solve of material.py:541-544 (src/fem/solvers/linear.py:15).  r, z, p, q are
 * n-vectors of scratch, work CIB_CSR_PCG_WORK_DOUBLES doubles (device).  Stops when
 * ||r|| <= rtol ||b|| or after maxit iterations; the host reads the device status every
 * check_every iterations.  Host outputs: status 0 converged, 1 iteration limit, 2 breakdown
 * (p.Ap <= 0 or a non-finite value); iterations; relative_residual ||r|| / ||b||.  The dot
 * products are reduced in a fixed order: bitwise repeatable.  Returns CIB_ERANGE when n
 * needs more than CIB_CSR_PCG_MAX_GRID blocks of partials. */
#define CIB_CSR_PCG_MAX_GRID 1024
#define CIB_CSR_PCG_WORK_DOUBLES (3 * CIB_CSR_PCG_MAX_GRID + 8)
int cib_csr_pcg(int64_t n, const int64_t* indptr, const int64_t* indices, const double* values,
                const uint8_t* free_mask, const double* dinv, const double* b, double* x, double* r, double* z,
                double* p, double* q, double* work, double rtol, int32_t maxit, int32_t check_every, int32_t* status,
                int32_t* iterations, double* relative_residual, void* stream);

/* --- Energy-based RVE-RNO (the reference's surrogate family) ------------------------------
 * FP32 update of src/concrete_impact/nn/models/rve_rno.py:334-418 (EnergyDissipationRVERNO,
 * direct_rate evolution) with the input gradients of ScalarMLP.value_and_input_gradient
 * (:110-129).  Three SiLU networks of `layers` hidden layers of width `hidden` (<= 128):
 * equilibrium potential (6 inputs), non-equilibrium potential (6 + latent inputs), state
 * evolution (6 + latent -> latent).  `params` packs, network after network in that order,
 * for every hidden layer l: W [hidden][in_l] (torch Linear layout), its transpose
 * Wt [in_l][hidden], bias [hidden]; then the output weights [out][hidden] and output bias
 * [out] (zeros for the two potentials).  integrator 1 = current_state_stress_forward_euler
 * (stress from the forward-Euler candidate state), 0 = cs_semi_implicit_forward_euler
 * (stress from the previous state).  latent <= 8. */
typedef struct cib_energy_rno {
  int32_t hidden;
  int32_t layers;
  int32_t latent;
  int32_t integrator;
  double reference_time_scale;
  const float* params;       /* cib_energy_rno_param_count floats (device) */
  const float* strain_scale; /* 6 floats (device): network strain = strain / scale */
} cib_energy_rno;

/* Length of `params` for a model shape (-1 for an invalid shape); host only. */
int64_t cib_energy_rno_param_count(int32_t hidden, int32_t layers, int32_t latent);

/* Zero-state energy anchors (prepare_energy_anchors, rve_rno.py:227-247) into 14 floats:
 * equilibrium value, its strain gradient (6), non-equilibrium value, its strain gradient (6). */
int cib_energy_rno_anchors(const cib_energy_rno* model, float* anchors, void* stream);

/* One update of n points (update_batch without tangent, rve_rno.py:249-313): strain (n,6),
 * latent (n,latent), time_step (n), anchors (14, NULL = zeros) -> stress (n,6), latent_out,
 * state_rate and dimensionless_rate (n,latent), scalars (4 rows of n: dissipation, free
 * energy, thermodynamic violation, non-equilibrium energy increment).  All FP32, device. */
int cib_energy_rno_update(const cib_energy_rno* model, int64_t n, const float* strain, const float* latent,
                          const float* time_step, const float* anchors, float* stress, float* latent_out,
                          float* state_rate, float* dimensionless_rate, float* scalars, void* stream);

/* Algorithmic tangent d stress / d strain of the update above, (n, 6, 6) FP32 row-major
 * [i][j] = d stress_i / d strain_j -- the rows the reference obtains by autograd
 * (rve_rno.py:283-297): second derivatives of the two potentials by forward-over-reverse
 * passes through the networks, through the candidate latent state (strain Jacobian of the
 * evolution network) for the current-state integrator.  2 to 4 hidden layers of up to 128
 * (CIB_ERANGE beyond what fits in shared memory). */
int cib_energy_rno_tangent(const cib_energy_rno* model, int64_t n, const float* strain, const float* latent,
                           const float* time_step, float* tangent, void* stream);

/* Error gate of the surrogate at n macro points (no reference counterpart; the reference's
 * deployment adapter, src/concrete_impact/nn/deployment.py:68-165, has no input gate).
 * prepare: strain_n = strain / strain_scale, rate_n = rate / rate_scale (fp32, n x 6),
 * coef_out[i] = coef, and fresh[i] = 1 for each point not yet `flagged` whose strain or rate
 * component exceeds limits[0..5] / limits[6..11] (normalised units) or is not finite;
 * finish: stress = stress_n * stress_scale (double) and fresh[i] = 1 also where the
 * surrogate's answer is not finite.  Both add the number of newly set `fresh` points to
 * the device counter `count`. */
int cib_rno_gate_prepare(int64_t n, const double* strain, const double* rate, double strain_scale, double rate_scale,
                         const double* limits, double coef, const uint8_t* flagged, float* strain_n, float* rate_n,
                         float* coef_out, uint8_t* fresh, unsigned int* count, void* stream);
int cib_rno_gate_finish(int64_t n, const float* stress_n, double stress_scale, const uint8_t* flagged, uint8_t* fresh,
                        unsigned int* count, double* stress, void* stream);

/* Strided host<->device copy of `rows` rows of `row_bytes` bytes (one cudaMemcpy2DAsync);
 * kind 1 = host to device, 2 = device to host, 3 = device to device. */
int cib_copy_rows_async(void* dst, int64_t dst_pitch, const void* src, int64_t src_pitch, int64_t row_bytes,
                        int64_t rows, int kind, void* stream);

/* Name of diagnostic row `row` of cib_j2vp_update, NULL when out of range. */
const char* cib_j2_diagnostic_name(int row);
/* The reference's reason string for a per-point status code. */
const char* cib_j2_reason(int code);
/* The last CUDA error recorded by a failed launch in this thread (cudaError_t value). */
int cib_last_cuda_error(void);
/* Library version string. */
const char* cib_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CIB200_H */
