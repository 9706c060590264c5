/*
 * gpop.h -- C ABI of the B200 propagation + closest-approach library (libgpop.so).
 *
 * Plain C types only: host or device pointers, sizes, status codes. Every entry point names the
 * reference interface it replaces (file:line relative to the reference project root). Device
 * pointers are caller-owned; the context owns all scratch memory. Errors are returned as status
 * codes (the reference calls exit()); gpop_last_error() gives the message. A context is used from
 * one host thread at a time; distinct contexts are independent.
 */
#ifndef GPOP_H
#define GPOP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef struct gpop_ctx gpop_ctx;
typedef struct gpop_propagator gpop_propagator;
typedef struct gpop_ca gpop_ca;

typedef enum {
    GPOP_OK = 0,
    GPOP_ERR_INVALID_ARG = 1,
    GPOP_ERR_CUDA = 2,
    GPOP_ERR_DATA = 3, /* a model data file is missing or malformed */
    GPOP_ERR_NOMEM = 4,
    GPOP_ERR_TIMEOUT = 5, /* a bounded device wait gave up */
    GPOP_ERR_UNSUPPORTED = 6,
    GPOP_ERR_STATE = 7, /* call out of order (e.g. find before propagate) */
} gpop_status;

/* TimeData (lib/common/types/types/Parameters.hpp:19-22) */
typedef struct {
    int32_t year, month, day, hour, min;
    double sec;
} gpop_time;

typedef enum { GPOP_FP64 = 0, GPOP_MIXED = 1 } gpop_precision;

/* Reference quirks (kept by default so results match the reference build; a set bit fixes it). */
enum {
    GPOP_FIX_BACKWARD_RK8_EPOCH = 1u << 0, /* Q1: force_model.cu:69-71 uses (-i + c_k) h */
    GPOP_FIX_STARTUP_EXPORT_ACC = 1u << 1, /* Q3: gpu_propagator.cu:48-53,68-72 exports column 8 */
    GPOP_FIX_PHASE_EPOCH = 1u << 2, /* closest_approach.cu:134: each phase restarts the epoch */
};
/* No counterpart in the reference. Mixed precision only: the FP32 sums of the degree > 8 terms are
 * compensated (TwoSum per added term) instead of summed in two levels; the propagation then walks
 * one or two objects per thread (no lane split). Slower; for error studies. */
enum { GPOP_MIXED_COMPENSATED = 1u << 3 };

/* Analytic force models of the reference's test suite (unit_tests/include/gpu_test_helpers.cuh) */
typedef enum {
    GPOP_FORCE_GRAVITY = 0,
    GPOP_FORCE_ZERO = 1,
    GPOP_FORCE_CONST = 2,
    GPOP_FORCE_POLY7 = 3,
    GPOP_FORCE_POLY8 = 4,
    GPOP_FORCE_POLY9 = 5,
    GPOP_FORCE_EXP = 6,
    GPOP_FORCE_DAMPED = 7,
} gpop_force_kind;

typedef struct {
    const char* data_dir; /* directory with JGM3.gfc, nutation, EOP and leap-second files */
    int32_t device; /* CUDA device ordinal (the reference hard-wires 0: force_model.cu:25) */
    int32_t gravity_degree; /* <= 0: max_degree of the gfc header (dataset_loaders.cu:245-248) */
    int32_t n_corrections; /* corrector passes; the reference uses 7 (exec/runner.cu:36) */
    int32_t precision; /* gpop_precision */
    uint32_t flags; /* GPOP_FIX_* */
} gpop_config;

/* ---- context ---- */
void gpop_config_default(gpop_config* cfg);
/* Replaces ForceModel(...) + PreInitialize (force_model.cuh:30-40, force_model.cu:23-45):
 * loads the data sets once and uploads the gravity table. */
gpop_status gpop_create(const gpop_config* cfg, gpop_ctx** out);
void gpop_destroy(gpop_ctx* ctx);
const char* gpop_last_error(const gpop_ctx* ctx);
const char* gpop_status_string(int32_t status);
int32_t gpop_gravity_degree(const gpop_ctx* ctx);
/* Number of device kernels this context has launched (monotonic). */
int64_t gpop_kernel_launches(const gpop_ctx* ctx);

/* ---- propagation ---- */
/* Input states: where the reference exits (gpu_utils.cuh:28-48) or propagates bad values into
 * NaNs, these calls return GPOP_ERR_INVALID_ARG for a state with a non-finite component or a
 * position at the origin. Host inputs are checked before any work; device inputs by the startup
 * kernel, which still propagates the other objects and writes their results. */
/* exec propagate (exec/runner.cu:11-70) / GpuPropagator::Step x steps + CopyStateToHost
 * (gpu_propagator.cu:28-84): host AoS buffers [n][3] in metres and m/s (GCRS). */
gpop_status gpop_propagate(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps, int64_t n,
    const double* r_in, const double* v_in, double* r_out, double* v_out);
/* Device-pointer variant: r_dev/v_dev ([n][3] AoS) are updated in place, like the caller-owned
 * buffers of GpuPropagator (gpu_propagator.cu:128-129). stream may be NULL (legacy default). */
gpop_status gpop_propagate_device(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps,
    int64_t n, double* r_dev, double* v_dev, void* stream);
/* Same, also writing the per-step trajectory (device, [steps][3][n] SoA each; any may be NULL):
 * positions, velocities and the acceleration the reference exports after each Step()
 * (MoveColumnToVectorKernel, gpu_propagator/src/device/dev_functions.cu:71-82). */
gpop_status gpop_propagate_trajectory(gpop_ctx* ctx, const gpop_time* start, double h,
    int32_t steps, int64_t n, double* r_dev, double* v_dev, double* traj_r, double* traj_v,
    double* traj_a, void* stream);
/* GpuPropagator (lib/gpu_propagator/include/gpu_propagator/gpu_propagator.cuh:26-59): binds the
 * caller-owned device buffers r_dev/v_dev ([n][3] AoS, updated in place after every step call);
 * max_steps sizes the epoch table like the reference's maxSteps argument. */
gpop_status gpop_propagator_create(gpop_ctx* ctx, const gpop_time* start, double h,
    int32_t max_steps, int64_t n, double* r_dev, double* v_dev, gpop_propagator** out);
/* GpuPropagator::Step (gpu_propagator.cu:28-77) called `steps` times: the first call runs the
 * startup. traj_* ([steps][3][n] SoA, may be NULL) are indexed from this call's first step. */
gpop_status gpop_propagator_step(gpop_propagator* p, int32_t steps, double* traj_r, double* traj_v,
    double* traj_a, void* stream);
/* Steps taken so far. */
int32_t gpop_propagator_steps_done(const gpop_propagator* p);
/* No counterpart in the reference. The gravity walk the propagation calls take for n objects on a
 * GPU of num_sms SMs at the given precision: 1 = one object per thread, 2 = two objects per
 * thread, 3 = lanes per object, 4 = lanes per group of two objects (*lanes_out = the lanes for 3
 * and 4, else 1); -1 for invalid arguments. Host arithmetic only, no CUDA call. */
int32_t gpop_walk_policy(int64_t n, int32_t num_sms, int32_t precision, int32_t* lanes_out);
/* No counterpart in the reference. Where the walk is two objects per thread: the owner warps of
 * the split block it launches (8 warps per SM, of which the owners carry the objects and the
 * others walk the low gravity columns of the owners' objects), 5 to 7 when each SM carries 5 to 7
 * sets of 64 objects and the degree is above 8; 0 for the plain block. -1 for invalid arguments.
 * Host arithmetic only. */
int32_t gpop_split_block(int64_t n, int32_t num_sms, int32_t degree);
void gpop_propagator_destroy(gpop_propagator* p);
/* No counterpart in the reference. gpop_propagate_device for callers that may not allocate device
 * memory while running (services that reserve their memory budget at start-up and forbid later
 * allocation; hosts whose device memory is held by another allocator's pool). The scratch lives in
 * one fixed device array of the library (about 4.5 MB on every GPU that loads it, until exit), so
 * calls are limited to GPOP_NOALLOC_MAX_OBJECTS objects and GPOP_NOALLOC_MAX_STEPS steps; larger
 * requests return GPOP_ERR_INVALID_ARG. All calls share that array: calls that overlap on the GPU
 * race. Every call looks the array's device address up (cudaGetSymbolAddress, which allocates
 * nothing), so calls stay correct across a cudaDeviceReset; the first call on a device also loads
 * the library's device code and should come before any stream capture. The call waits for its
 * own work to finish before it returns. Same walk, tables and results as gpop_propagate_device. */
#define GPOP_NOALLOC_MAX_OBJECTS 4096
#define GPOP_NOALLOC_MAX_STEPS 20160
gpop_status gpop_propagate_device_noalloc(gpop_ctx* ctx, const gpop_time* start, double h,
    int32_t steps, int64_t n, double* r_dev, double* v_dev, void* stream);
/* Analytic test forces through the same integrator kernels (MockForceModel,
 * unit_tests/include/mock_force_model.cuh:46-112). Times follow the mock: (idx - 4) h. */
gpop_status gpop_propagate_analytic(gpop_ctx* ctx, int32_t kind, double h, int32_t steps,
    int32_t n_corrections, int64_t n, double* r_dev, double* v_dev, double* traj_r, double* traj_v,
    double* traj_a, void* stream);

/* ---- batched propagation ---- */
/* One propagation request of a batch: the arguments of exec propagate (exec/runner.cu:11-70)
 * for one input, with its own step size, step count and gravity degree. Host buffers [n][3]. */
typedef struct {
    gpop_time start;
    double h;
    int32_t steps;
    int32_t degree; /* <= 0 or > the context's degree: the context's degree */
    int64_t n;
    const double* r_in;
    const double* v_in;
    double* r_out;
    double* v_out;
} gpop_request;

/* Propagates many independent requests (uneven object counts, durations, step sizes, degrees) in
 * one persistent launch: the reference runs one GpuPropagator per request (gpu_propagator.cu:
 * 121-136), i.e. one exec propagate call each. Results equal those of gpop_propagate per request
 * to rounding. The launch sequence is captured in a CUDA graph and replayed when the next batch
 * has the same shape. A request that cannot run (invalid arguments; an object whose position or
 * velocity is not finite, or whose position is the origin) is refused alone: the others are
 * propagated and written, its outputs are left untouched, and the call returns
 * GPOP_ERR_INVALID_ARG naming the first refused request. */
gpop_status gpop_propagate_batch(gpop_ctx* ctx, const gpop_request* reqs, int32_t n_req);
/* No counterpart in the reference (which exits on bad input, gpu_utils.cuh:28-48).
 * gpop_propagate_batch with one status per request in status[n_req] (NULL: none): GPOP_OK for
 * the propagated requests, GPOP_ERR_INVALID_ARG for the refused ones; when the batch itself fails,
 * its status for every request that was to run. */
gpop_status gpop_propagate_batch_status(gpop_ctx* ctx, const gpop_request* reqs, int32_t n_req,
    int32_t* status);
/* The batch plan: lanes per object chosen for each request and the estimated makespan (s). The
 * planner also picks the block shape of the persistent grid (4 or 8 warps per SM), the one with the
 * shorter simulated makespan; gpop_batch_warps_per_sm gives the last planned batch's. */
gpop_status gpop_batch_plan(gpop_ctx* ctx, const gpop_request* reqs, int32_t n_req,
    int32_t* lanes_per_object, double* est_seconds);
/* No counterpart in the reference. Warps per SM (the block shape) of the last planned batch. */
int32_t gpop_batch_warps_per_sm(const gpop_ctx* ctx);
/* Device time (s, CUDA events) of the last gpop_propagate_batch launch: frames, startup and the
 * persistent GJ8 kernel, without the host copies. */
double gpop_batch_device_seconds(const gpop_ctx* ctx);
/* Autotuner: measures the throughput of the batched GJ8 kernel for each block shape (4 and 8 warps
 * per SM), gravity degree in {8, 20, 36, 70} (up to the context's) and 1..32 lanes per object (the
 * item tile: 32/P objects, 64 with one lane), which the batch planner then uses. cache_path (may
 * be NULL) is read if it exists and written otherwise. */
gpop_status gpop_tune(gpop_ctx* ctx, const char* cache_path);

/* ---- variational equations and adjoint (FP64; the reference has no counterpart) ----
 * Derivatives of the discrete propagation map of gpop_propagate in FP64 (RK8 startup + GJ8 with
 * the context's corrector passes, gravity at every iterate), with respect to the initial GCRS
 * state x0 = (r0, v0). Host buffers. */
/* Gravity acceleration (a_dev may be NULL) and its Jacobian jac_dev [n][3][3] = d a_i / d r_j at
 * GCRS positions r_dev [n][3] with frame matrix frame9_dev (as gpop_gravity; NULL = identity).
 * FP64, device buffers. */
gpop_status gpop_gravity_jacobian(gpop_ctx* ctx, int64_t n, const double* r_dev,
    const double* frame9_dev, double* a_dev, double* jac_dev, void* stream);
/* 6x6 state transition matrices by the forward variational equations: stm_out [n][6][6],
 * stm[i][j] = d x_N,i / d x0_j with x = (r, v); r_out, v_out (may be NULL) = the final state. */
gpop_status gpop_stm(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps, int64_t n,
    const double* r_in, const double* v_in, double* r_out, double* v_out, double* stm_out);
/* Vector-Jacobian product by the adjoint (reverse) sweep, GJ8 state checkpointed every 64
 * steps: grad_r0, grad_v0 [n][3] = d(sum r_bar . r_N + v_bar . v_N) / d(r0, v0). r_bar or v_bar
 * may be NULL (zero). */
gpop_status gpop_propagate_vjp(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps,
    int64_t n, const double* r_in, const double* v_in, const double* r_bar, const double* v_bar,
    double* grad_r0, double* grad_v0);
/* Closest approach of listed pairs (pairs [n_pairs][2] object indices, a != b) over `steps` steps
 * with the reference's running minimum, Hermite interpolation and secant TCA
 * (closest_approach/src/device.cu:56-173), and the adjoint gradient of each miss distance:
 * tca, miss [n_pairs]; grad [n_pairs][12] = d miss / d(r0_a, v0_a, r0_b, v0_b). */
gpop_status gpop_miss_gradient(gpop_ctx* ctx, const gpop_time* start, double h, int32_t steps,
    int64_t n, const double* r_in, const double* v_in, int64_t n_pairs, const int32_t* pairs,
    double* tca, double* miss, double* grad);

/* ---- Monte Carlo ensembles ---- */
/* PerturbationGenerator::generatePerturbedSatellites (perturbation_generator.cu:21-79): n
 * samples of one object, r = r_nominal + sigma_r z, v = v_nominal + sigma_v z', z and z' standard
 * normal (the reference perturbs the velocity only: sigma_r = 0). Philox4x32-10 counter-based
 * generator keyed by seed, Box-Muller; sample i depends only on (seed, i). Not the reference's
 * curand sequence. r_nominal, v_nominal: host [3]; r_dev, v_dev: device [n][3]. */
gpop_status gpop_sample_states(gpop_ctx* ctx, const double* r_nominal, const double* v_nominal,
    double sigma_r, double sigma_v, uint64_t seed, int64_t n, double* r_dev, double* v_dev, void* stream);

/* ---- startup and integrator pieces (device buffers, one object each) ---- */
/* GpuStartup::Startup (gpu_startup.cu:55-68). Outputs 9 columns x 3 (column 4 = epoch):
 * r27, v27, a27, s27, S27 (device). n_corrections = 0 returns the RK8 guess only. */
gpop_status gpop_startup(gpop_ctx* ctx, int32_t kind, const gpop_time* start, double h,
    int32_t n_corrections, const double* r0_dev, const double* v0_dev, double* r27, double* v27,
    double* a27, double* s27, double* S27, void* stream);
/* StartupCorrector on given matrices (gpu_startup.cu:170-294): op 0 = acceleration matrix only,
 * 1 = + CalculateS0, 2 = + one Correct(). In place on device buffers. */
gpop_status gpop_corrector_unit(gpop_ctx* ctx, int32_t kind, double h, int32_t op, double* r27,
    double* v27, double* a27, double* s27, double* S27, void* stream);
/* Predictor::Predict (prediction.cu:49-74) at `step`, in place. */
gpop_status gpop_predict_unit(gpop_ctx* ctx, int32_t kind, double h, int32_t step, double* r3,
    double* v3, double* a27, double* s3, double* S3, void* stream);
/* FinalizeCorrectionKernel (gpu_propagator/src/device/dev_functions.cu:52-69), in place. */
gpop_status gpop_finalize_correction_unit(gpop_ctx* ctx, double h, double* r3, double* v3,
    const double* a27, const double* s3, const double* S3, void* stream);

/* ---- integrator pieces between force evaluations (n objects, caller-supplied accelerations) ----
 * The path of the reference's GpuStartup, Predictor and GpuPropagator with an arbitrary
 * IForceModel: the caller evaluates the model's hooks between these calls. Buffers are device
 * AoS in the reference's layouts: x, v, r, s3, S3, prev3, sum1, sum2 [n][3]; R27, V27, A27, s27,
 * S27 [n][9][3]; Kx30, Kv30 [n][10][3]. None of them allocates. ctx may be NULL (the current
 * device; no error text). */
/* RK8::step stage k of startup step `step` (+-1..4) (gpu_startup.cu:108-135): writes the stage
 * state to x_dev, v_dev and the stage velocity to Kx30 slot k; stages 1..9 read Kx30 and Kv30
 * slots 0..k-1 (Kv30: the generation accelerations the hook wrote). */
gpop_status gpop_rk8_stage(gpop_ctx* ctx, int64_t n, double h, int32_t step, int32_t k,
    const double* R27, const double* V27, double* Kx30, const double* Kv30, double* x_dev,
    double* v_dev, void* stream);
/* RK8::step end (gpu_startup.cu:136-144): column 4 + step of R27, V27 from the ten stages. */
gpop_status gpop_rk8_finish(gpop_ctx* ctx, int64_t n, double h, int32_t step, double* R27,
    double* V27, const double* Kx30, const double* Kv30, void* stream);
/* GpuStartup before its predictor (gpu_startup.cu:55-60): column 4 of R27, V27 = r, v; the rest
 * of R27, V27 and all of A27, s27, S27 (each may be NULL) zeroed. */
gpop_status gpop_startup_init(gpop_ctx* ctx, int64_t n, const double* r_dev, const double* v_dev,
    double* R27, double* V27, double* A27, double* s27, double* S27, void* stream);
/* StartupCorrector::Correct without its force evaluations (gpu_startup.cu:247-290): s27, S27
 * from A27, then the state columns other than the epoch's. */
gpop_status gpop_startup_correct(gpop_ctx* ctx, int64_t n, double h, double* R27, double* V27,
    const double* A27, double* s27, double* S27, void* stream);
/* Predictor::Predict without its force evaluation (prediction.cu:49-70): r, v predicted, S3
 * advanced, A27 shifted one column (column 8 is then the hook's), and prev3 = s3 and the corrector
 * sums sum1, sum2 of GpuPropagator::Correct (gpu_propagator.cu:86-100). */
gpop_status gpop_gj8_predict(gpop_ctx* ctx, int64_t n, double h, double* r_dev, double* v_dev,
    double* A27, const double* s3, double* S3, double* prev3, double* sum1, double* sum2, void* stream);
/* One pass of GpuPropagator::Correct after its force evaluation wrote A27 column 8
 * (gpu_propagator.cu:101-117): s3, v, r. */
gpop_status gpop_gj8_correct(gpop_ctx* ctx, int64_t n, double h, double* r_dev, double* v_dev,
    const double* A27, double* s3, const double* S3, const double* prev3, const double* sum1,
    const double* sum2, void* stream);
/* Column col of an [n][cols][3] matrix copied to the [n][3] vector v3_dev (to_matrix = 0) or
 * from it (CopyStartupStateKernel, MoveColumnToVectorKernel, CopySKernel). */
gpop_status gpop_matrix_column(gpop_ctx* ctx, int64_t n, double* m_dev, int32_t cols, int32_t col,
    double* v3_dev, int32_t to_matrix, void* stream);
/* The Gauss-Jackson (a90) and summed-Adams (b90) ordinate tables in the layout of the reference's
 * devA / devB (gpu_constants::createCoefficients): entry 10 k + c is the coefficient of history
 * column k in row c. Either may be NULL. */
gpop_status gpop_gj8_coefficients(gpop_ctx* ctx, double* a90_dev, double* b90_dev, void* stream);

/* ---- force model ---- */
/* GravitySource::ComputeAcceleration (gravity_source.cu:168-211): r_dev, a_dev [n][3] GCRS;
 * frame9_dev = ITRS->GCRS column-major 3x3 (NULL = identity). precision: gpop_precision. */
gpop_status gpop_gravity(gpop_ctx* ctx, int64_t n, const double* r_dev, const double* frame9_dev,
    double* a_dev, int32_t precision, void* stream);
/* FMTimePoints::CalculateParameters (time_points.cu:126-201): count ITRS->GCRS matrices
 * (column-major, 9 each) and UTC MJDs for epochs start - before_epoch h + i h (or the RK8
 * midpoints when use_midpoints). Device outputs; mjd_dev may be NULL. */
gpop_status gpop_frame_matrices(gpop_ctx* ctx, const gpop_time* start, double h, int32_t count,
    int32_t use_midpoints, int32_t before_epoch, double* m_dev, double* mjd_dev, void* stream);

/* ---- closest approach (lib/closest_approach) ---- */
/* One record per cross-set pair i < j (exec/runner.cu:96-106, ClosestApproachData::Get). */
typedef struct {
    uint32_t object_index1, object_index2;
    double distance; /* m */
    double time; /* s from the start of the first phase */
    double position_a[3], position_b[3];
} gpop_ca_record;

/* ClosestApproach::Initialize (closest_approach.cu:47-127). set_ids: start at 0, non-decreasing by
 * at most 1, at least two sets. Host buffers. */
gpop_status gpop_ca_create(gpop_ctx* ctx, const gpop_time* start, double h, int64_t n,
    const double* r_in, const double* v_in, const uint32_t* set_ids, gpop_ca** out);
/* ClosestApproach constructed over a MockForceModel (unit_tests/include/mock_force_model.cuh:46-112,
 * used by unit_tests/closest_approach_test.cu): same screen and refinement, analytic force kind. */
gpop_status gpop_ca_create_analytic(gpop_ctx* ctx, int32_t kind, double h, int64_t n,
    const double* r_in, const double* v_in, const uint32_t* set_ids, gpop_ca** out);
/* ClosestApproach over an arbitrary IForceModel (closest_approach.cu:47-157 with a force model
 * that is not the library's): the same partition, screen and refinement, with the trajectory
 * supplied by the caller through gpop_ca_append (r_in, v_in: host epoch state, kept for
 * gpop_ca_trajectory). gpop_ca_propagate is refused on such an object. */
gpop_status gpop_ca_create_external(gpop_ctx* ctx, double h, int64_t n, const double* r_in,
    const double* v_in, const uint32_t* set_ids, gpop_ca** out);
/* The next `steps` propagated steps of an external object: device AoS [steps][n][3] positions,
 * velocities and the steps' exported accelerations (GpuPropagator::Step's devAccelerationVector);
 * runs the screen over them (UpdateClosestApproachKernel, closest_approach.cu:138-146). */
gpop_status gpop_ca_append(gpop_ca* ca, int32_t steps, const double* r_dev, const double* v_dev,
    const double* a_dev);
/* No counterpart in the reference. Sizes the trajectory store for total_steps steps in all, so
 * that later gpop_ca_propagate / gpop_ca_append calls up to that many steps neither reallocate
 * nor copy it (without it, appends grow the store by doubling). */
gpop_status gpop_ca_reserve(gpop_ca* ca, int32_t total_steps);
/* ClosestApproach::Propagate (closest_approach.cu:129-157): steps more steps; running minima
 * persist across calls. */
gpop_status gpop_ca_propagate(gpop_ca* ca, int32_t steps);
/* ClosestApproach::FindClosest (closest_approach.cu:159-209) + the runner's record loop. Writes
 * the records whose distance < threshold_m (threshold_m < 0: every pair, reference semantics),
 * sorted by (object_index1, object_index2). out may be NULL to query the count. */
gpop_status gpop_ca_find(gpop_ca* ca, double threshold_m, gpop_ca_record* out, int64_t capacity,
    int64_t* n_out);
/* Per-pair results in the reference's pair order (PartitionParameters map), host buffers of
 * num_pairs entries (any may be NULL): refined distance, time, positions, closest step. */
gpop_status gpop_ca_pairs(gpop_ca* ca, double* dist, double* time, double* pos_a, double* pos_b,
    uint32_t* closest_step);
int64_t gpop_ca_num_pairs(const gpop_ca* ca);
/* No counterpart in the reference (one process per GPU for the screen). Narrows this object to
 * the pairs whose first object lies in rows [row_begin, row_end): the screen, the refinement,
 * gpop_ca_find and gpop_ca_pairs then cover only those pairs, a contiguous range of the pair
 * order, and gpop_ca_pairs fills only that range of its num_pairs-long arrays. begin and end are
 * multiples of 64 (the screen's tile) or n. Only before the first propagate or append. */
gpop_status gpop_ca_set_rows(gpop_ca* ca, int64_t row_begin, int64_t row_end);
/* [pair_begin, pair_end): the pair indices this object screens (all pairs by default). */
gpop_status gpop_ca_pair_range(const gpop_ca* ca, int64_t* pair_begin, int64_t* pair_end);
/* Device trajectory of the propagated phases ([steps][3][n] SoA), for inspection and tests. */
gpop_status gpop_ca_trajectory(gpop_ca* ca, double* r_host, double* v_host, double* a_host,
    int32_t* steps_out);
/* Cumulative device time (s, CUDA events) of this object's propagation, screen and TCA refinement:
 * out3 = {propagation, screen, refinement}. No counterpart in the reference. */
gpop_status gpop_ca_device_seconds(const gpop_ca* ca, double* out3);
void gpop_ca_destroy(gpop_ca* ca);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* GPOP_H */
