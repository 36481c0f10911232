/*
 * cib200.h -- C ABI of the B200 (sm_100a) material-point and periodic-RVE kernels.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream (passed as
 * `void*`, NULL = legacy default stream).  Nothing here allocates device memory: all
 * buffers, including solver work vectors, are passed in by the caller.  All calls are
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
