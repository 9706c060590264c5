/*
 * gpop_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU FP64 restatement of the OpenGPOP propagation + closest-approach path. It is the checker for
 * the CUDA product: only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 * The product (libgpop.so) never links, calls or reads anything in this directory.
 *
 * Every function follows the reference file and line cited beside it (paths are relative to the
 * reference project root). Parity of this restatement is pinned against the reference's own golden
 * vectors and known-answer tests (ported in tests/test_oracle_golden.py).
 */
#pragma once
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t year, month, day, hour, min;
    double sec;
} or_time; /* lib/common/types/types/Parameters.hpp:19-22 (TimeData) */

/* ---- data sets (lib/force_model/src/utility/dataset_loaders.cu:30-299) ---- */
void* or_data_load(const char* data_dir, int32_t degree); /* degree <= 0: gfc header max_degree */
void or_data_free(void* d);
int32_t or_data_degree(const void* d);
double or_data_gm(const void* d);
double or_data_radius(const void* d);
int64_t or_data_eop_count(const void* d);
int64_t or_data_leap_count(const void* d);
int64_t or_data_nut_count(const void* d, int32_t which); /* 0 lon j0, 1 lon j1, 2 obl j0, 3 obl j1 */
void or_data_eop_record(const void* d, double mjd_utc, double out4[4]); /* mjd, xp, yp, ut1-utc */
double or_data_leap_seconds(const void* d, double mjd_utc);
/* C and S coefficient of degree n, order m as loaded */
void or_data_coef(const void* d, int32_t n, int32_t m, double* c, double* s);

/* ---- reference-system pieces (lib/force_model/src/utility/ref_sys_trans.cu:24-376) ---- */
double or_calendar_to_mjd(int32_t y, int32_t mon, int32_t day, int32_t h, int32_t min, double sec);
void or_ftable(double t, double F[14]);
void or_precession(double t, double out4[4]); /* eps_A, gamma_bar, phi_bar, psi_bar */
void or_nutation(const void* d, double mjd_tt, double out2[2]); /* delta_psi, delta_eps */
double or_gast(double mjd_ut1, double mjd_tt, double delta_psi, double eps_A, const double F[14]);
double or_ntp_to_mjd(int64_t ntp_seconds);
void or_rot(int32_t axis, double angle, double out9[9]);

/* Per-epoch ITRS->GCRS matrices, column-major 3x3 per epoch
 * (lib/force_model/src/time_points.cu:26-71,160-201). */
void or_frame_matrices(const void* d, const or_time* start, double h, int32_t count,
    int32_t use_midpoints, int32_t before_epoch, double* m_out, double* mjd_out);

/* ---- gravity (lib/force_model/src/acceleration/gravity_source*.cu) ----
 * r_gcrs: n x 3, m9: ITRS->GCRS column-major (NULL = identity), a_out: n x 3 GCRS. */
void or_gravity(const void* d, int64_t n, const double* r_gcrs, const double* m9, double* a_out);

/* ---- force kinds ---- */
enum {
    OR_FORCE_GRAVITY = 0,
    OR_FORCE_ZERO = 1, /* unit_tests/include/gpu_test_helpers.cuh NoAcceleration */
    OR_FORCE_CONST = 2, /* AccelerationFunction (1,2,3) */
    OR_FORCE_POLY7 = 3,
    OR_FORCE_POLY8 = 4,
    OR_FORCE_POLY9 = 5,
    OR_FORCE_EXP = 6,
    OR_FORCE_DAMPED = 7,
};

/* Flags: bit 0 set = fix the backward-RK8 frame epoch (reference quirk Q1 reproduced when clear). */
enum { OR_FLAG_FIX_Q1 = 1, OR_FLAG_FIX_Q3 = 2 };

/* ---- integrator (lib/gpu_startup, lib/gpu_integrator, lib/gpu_propagator) ---- */
/* RK8 +-4 steps only: r27/v27 = 9 columns x 3 (column 4 = epoch). */
void or_rk8(const void* d, int32_t kind, const or_time* start, double h, const double r0[3],
    const double v0[3], uint32_t flags, double* r27, double* v27);
/* Full startup (RK8 + ncorr mid-corrector passes). */
void or_startup(const void* d, int32_t kind, const or_time* start, double h, int32_t ncorr,
    const double r0[3], const double v0[3], uint32_t flags, double* r27, double* v27, double* a27,
    double* s27, double* S27);
/* Corrector unit pieces on given matrices with an analytic force (gpu_startup.cu:170-294).
 * op 0: constructor only (acceleration matrix), 1: + CalculateS0, 2: + one Correct(). */
void or_corrector_unit(int32_t kind, double h, int32_t op, double* r27, double* v27, double* a27,
    double* s27, double* S27);
/* Predictor unit (prediction.cu:49-74) with analytic force: in place on r3, v3, a27, s3, S3. */
void or_predict_unit(int32_t kind, double h, int32_t step, double* r3, double* v3, double* a27,
    double* s3, double* S3);
/* FinalizeCorrectionKernel (gpu_propagator/src/device/dev_functions.cu:52-69), in place. */
void or_finalize_correction_unit(double h, double* r3, double* v3, const double* a27,
    const double* s3, const double* S3);

/* Propagate n objects for `steps` steps. Per-step outputs (steps x n x 3) may be NULL.
 * a_steps receives the acceleration the reference exports after each Step() (column 8 of the
 * history). Returns 0 on success. */
int32_t or_propagate(const void* d, int32_t kind, const or_time* start, double h, int32_t steps,
    int32_t ncorr, int64_t n, const double* r0, const double* v0, uint32_t flags, double* r_steps,
    double* v_steps, double* a_steps, double* r_final, double* v_final, int32_t threads);

/* ---- closest approach (lib/closest_approach) ---- */
/* Partition parameters (partition_parameters.cuh:94-135). Returns 0 if the set ids are invalid.
 * set_offsets/num_higher/map_offsets must hold n entries. */
int32_t or_partition(const uint32_t* set_ids, int64_t n, uint32_t* num_sets, uint64_t* num_pairs,
    uint32_t* set_offsets, uint32_t* num_higher, uint64_t* map_offsets);
int64_t or_partition_map_idx(const uint32_t* set_ids, uint32_t num_sets, const uint32_t* set_offsets,
    const uint32_t* num_higher, const uint64_t* map_offsets, uint32_t a, uint32_t b);
int32_t or_partition_map_pair(uint32_t num_sets, const uint32_t* set_offsets,
    const uint32_t* num_higher, const uint64_t* map_offsets, uint64_t idx, uint32_t* a, uint32_t* b);

/* Hermite polynomial (interpolation.cuh:27-98): coeffs9 out, value/derivative at t. */
void or_hermite_coeffs(const double nodes9[9], double dt, double coeffs9[9]);
double or_hermite_eval(const double coeffs9[9], double dt, double t);
double or_hermite_deriv(const double coeffs9[9], double dt, double t);
/* Secant root of the approach function of two interpolated objects (interpolation.cuh:106-152).
 * nodesA/nodesB: 3 axes x 9 nodes (before p,v,a; closest p,v,a; after p,v,a). */
double or_approach_func(const double* nodesA27, const double* nodesB27, double dt, double t);
double or_find_root_approach(const double* nodesA27, const double* nodesB27, double dt, double x0,
    double x1, double tol, int32_t max_iter);
/* Secant on the test functions of closest_approach_utils_test.cu (0: 3x-6, 1: x^2-9, 2: x^2). */
double or_find_root_test(int32_t fn, double x0, double x1, double tol, int32_t max_iter);

/* Screen a trajectory (steps x n x 3 for r, v, a; step k is the state after propagation step k+1)
 * with the reference's per-pair running minimum (device.cu:56-91), then refine every pair
 * (device.cu:93-173). Outputs are indexed by the reference's pair index.
 * step_offset: number of steps already screened in earlier phases (0 for a single phase).
 * State arrays (min_dist, closest_step, before/closest/after nodes, last_*) carry across phases:
 * pass init=1 on the first phase. */
typedef struct {
    double* min_dist; /* P */
    uint32_t* closest_step; /* P */
    double* nodes; /* P x 2 objects x 3 nodes x 9 (p,v,a xyz) */
    double* last; /* n x 9 (p,v,a of the previous screened step) */
} or_ca_state;
void or_ca_screen(int64_t n, int32_t steps, const double* r, const double* v, const double* a,
    const uint32_t* set_ids, uint32_t step_offset, int32_t init, or_ca_state* st, int32_t threads);
void or_ca_refine(int64_t n, const uint32_t* set_ids, double h, uint32_t total_steps,
    const or_ca_state* st, double* dist_out, double* time_out, double* posA_out, double* posB_out,
    int32_t threads);

/* Finite-difference side of the adjoint checks, in x87 extended precision (long double) so that the
 * difference quotient is not swamped by rounding noise at small steps. For each pair (objects A and
 * B with initial states rA, vA, rB, vB [n_pairs][3]) propagates both objects with gravity over
 * `steps` steps, screens the pair (running minimum of the sampled distance, or_ca_screen's rules)
 * and refines the miss distance and TCA (or_ca_refine's Hermite and secant); then does the same
 * with each of the 12 initial-state components moved by +-dr (positions, m) or +-dv (velocities,
 * m/s), the moves applied in long double. Outputs per pair: miss, tca, and grad[12] = central
 * differences d miss / d(r0_A, v0_A, r0_B, v0_B). Returns 0 on success. */
int32_t or_miss_fd_ld(const void* data, const or_time* start, double h, int32_t steps, int32_t ncorr,
    int64_t n_pairs, const double* rA, const double* vA, const double* rB, const double* vB, double dr,
    double dv, double* miss, double* tca, double* grad, int32_t threads);
/* The same in double precision (the CPU baseline of the miss-gradient workload). */
int32_t or_miss_fd(const void* data, const or_time* start, double h, int32_t steps, int32_t ncorr,
    int64_t n_pairs, const double* rA, const double* vA, const double* rB, const double* vB, double dr,
    double dv, double* miss, double* tca, double* grad, int32_t threads);

#ifdef __cplusplus
}
#endif
