/*
 * cgmli_backend.h - C ABI of the B200 sliding-window backend solver.
 *
 * This is the device boundary that sits behind the reference's
 * `estimator_parameters.backend_visual_batch: schur` switch.  The reference
 * crosses it through the C++ classes `VisualCudaBatch` and
 * `MarginalCudaWorkspace` (src/backend/VisualCudaBatch.hpp:44-104); this
 * header exports the same operations with plain pointers and sizes so that a
 * C++ backend (or a ctypes / cgo / JNI binding) can call them without any
 * C++ or torch types in the signatures.
 *
 * Conventions (identical to the reference, src/backend/README.md:44-47,
 * src/backend/LeftSE3Manifold.hpp:151-156):
 *   - pose ambient      [p_WB(3), qx, qy, qz, qw], tangent [rho(3), theta(3)],
 *                       Plus(T, d) = Exp(d) * T (left SE(3));
 *   - speed/bias        [v_W(3), b_g(3), b_a(3)], Euclidean;
 *   - rig extrinsic     T_BR, same chart as a pose;
 *   - landmark          one inverse distance rho along a fixed anchor bearing;
 *   - camera pose       T_WC = T_WB * T_BR[e(c)] * T_RC[c].
 * Tangent columns of a window: keyframe k owns [15k, 15k+6) (pose) and
 * [15k+6, 15k+15) (speed/bias); then 6 columns per estimated extrinsic
 * block; then one column for an estimated time offset.  N_r is their total.
 *
 * Every entry point returns 0 on success or one of the CGMLI_E_* codes;
 * cgmli_last_error() returns a thread-local message for the last failure.
 * There is no CPU fallback behind any entry point: a failure is reported to
 * the caller, which decides what to do (the reference falls back to Ceres,
 * src/backend/BackendOptimizer.cpp:964-989).
 */
#ifndef CGMLI_BACKEND_H
#define CGMLI_BACKEND_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CGMLI_OK = 0,
    CGMLI_E_INVALID = 1,      /* malformed input (sizes, indices, layout) */
    CGMLI_E_NONFINITE = 2,    /* a factor or state evaluated to NaN/Inf */
    CGMLI_E_NOMEM = 3,        /* device or pinned allocation failed */
    CGMLI_E_CUDA = 4,         /* CUDA runtime error (see cgmli_last_error) */
    CGMLI_E_NOT_PD = 5,       /* damped reduced system is not positive definite */
    CGMLI_E_INDEFINITE = 6,   /* marginal information significantly negative */
    CGMLI_E_UNSUPPORTED = 7,  /* layout outside what the kernels implement */
    CGMLI_E_NO_STEP = 8,      /* LM found no acceptable step */
    CGMLI_E_LIMIT = 9,        /* size beyond a documented maximum */
    CGMLI_E_COST_MISMATCH = 10,/* relinearized cost disagrees with accepted trial */
    CGMLI_E_PENDING = 11       /* served request not complete yet */
};

enum { CGMLI_PRECISION_FP64 = 0, CGMLI_PRECISION_MIXED = 1 };
enum { CGMLI_PRIOR_POSE = 0, CGMLI_PRIOR_SPEED_BIAS = 1, CGMLI_PRIOR_EXTRINSIC = 2, CGMLI_PRIOR_TIME_OFFSET = 3 };
enum { CGMLI_MARGIN_OLD = 0, CGMLI_MARGIN_SECOND_NEW = 1, CGMLI_MARGIN_SECOND_NEW_IMU_MERGE = 2 };
/* Solve-time charts of cgmli_window (kf_fixed bits, ext_chart values). */
enum { CGMLI_FIX_POSE = 1, CGMLI_FIX_VELOCITY = 2, CGMLI_FIX_BIAS = 4 };
enum { CGMLI_CHART_FULL = 0, CGMLI_CHART_ROTATION_ONLY = 1, CGMLI_CHART_FIXED = 2 };
/* Outcome of the IMU merge of a CGMLI_MARGIN_SECOND_NEW_IMU_MERGE marginalization. */
enum { CGMLI_IMU_MERGE_NONE = 0,         /* no victim, or another policy */
       CGMLI_IMU_MERGE_REINTEGRATED = 1, /* the two edges became one re-integrated factor */
       CGMLI_IMU_MERGE_BRIDGE = 2,       /* conditions not met: the edges entered the Schur step */
       CGMLI_IMU_MERGE_SUPPRESSED = 3 }; /* interval above the maximum: both edges dropped */

/* Frozen IMU preintegration of one keyframe interval.  Same fields and
 * storage order as the reference's FrozenImuData
 * (src/backend/GpuRetainedFactors.hpp:7-13): 3x3 matrices and the 15x15
 * whitening are column-major, quaternions are [x, y, z, w]. */
typedef struct cgmli_frozen_imu {
    double duration, gravity;
    double sensor_position[3], sensor_quaternion[4], gyros[6];
    double delta_quaternion[4], delta_velocity[3], delta_position[3], reference_bias[6];
    double rotation_gyro[9], velocity_gyro[9], position_gyro[9], velocity_accel[9], position_accel[9];
    double whitening[225];
} cgmli_frozen_imu;

/* One sliding window in structure-of-arrays form.  Observations are
 * landmark-major: the observations of landmark l are
 * [lm_obs_begin[l], lm_obs_begin[l+1]).  The anchor observation of a
 * landmark has no residual and is not listed (src/backend/README.md:62-64).
 * State arrays are read by cgmli_solver_set_windows and written back by
 * cgmli_solver_read_states. */
typedef struct cgmli_window {
    int num_keyframes;          /* K */
    int num_cameras;            /* C fixed rig cameras */
    int num_extrinsics;         /* E >= 1 T_BR blocks; camera c uses cam_ext[c] */
    int estimate_extrinsics;    /* 1: extrinsic blocks are free variables */
    int estimate_td;            /* 1: the time offset is a free scalar */
    int num_landmarks;          /* L */
    int num_observations;       /* F visual factors */
    int num_imu;                /* frozen IMU factors */
    int prior_rank;             /* rows of the square-root prior (0: none) */
    int prior_num_blocks;       /* blocks in the prior's column order */
    double huber_scale;         /* whitened Huber delta, <= 0 disables */
    double min_inverse_distance;/* lower bound of every rho */
    double *poses;              /* K*7 */
    double *speed_bias;         /* K*9 */
    double *extrinsics;         /* E*7 */
    double *td;                 /* 1, or NULL: td equals each anchor's reference time */
    double *rho;                /* L */
    const double *cam_R;        /* C*9 row-major R_RC */
    const double *cam_t;        /* C*3 t_RC */
    const int *cam_ext;         /* C, extrinsic block of each camera */
    const int *lm_anchor_kf;    /* L */
    const int *lm_anchor_cam;   /* L */
    const int *lm_obs_begin;    /* L+1 */
    const double *lm_anchor_bearing;  /* L*3 */
    const double *lm_anchor_velocity; /* L*3 bearing velocity, or NULL */
    const double *lm_anchor_time;     /* L reference time offset, or NULL (0) */
    const int *obs_kf;          /* F observer keyframe */
    const int *obs_cam;         /* F observer camera */
    const double *obs_bearing;  /* F*3 measured unit bearing */
    const double *obs_P;        /* F*6 sqrtInfo * basis^T, 2x3 row-major */
    const double *obs_velocity; /* F*3 or NULL */
    const double *obs_time;     /* F or NULL */
    const cgmli_frozen_imu *imu;/* num_imu */
    const int *imu_kf;          /* num_imu: factor links keyframe imu_kf[i] -> imu_kf[i]+1 */
    const int *prior_block_kind;  /* prior_num_blocks, CGMLI_PRIOR_* */
    const int *prior_block_index; /* prior_num_blocks */
    const double *prior_ref;    /* concatenated ambient references (7, 9, 7 or 1 per block) */
    const double *prior_A;      /* prior_rank x (sum of tangent sizes, at most 1024: CGMLI_E_LIMIT), row-major */
    const double *prior_r0;     /* prior_rank */
    /* Solve-time charts: blocks held constant and restricted tangents for the LM
     * solve only, as the reference sets them on its Ceres problem for one solve
     * (constant blocks are not variables, BackendOptimizer.cpp:44-66; the
     * bias-frozen speed/bias SubsetManifold and the rotation-only rig chart,
     * :83-91,783-795).  NULL: every block free with its full chart.  The
     * marginalization, the gate and the calibration information keep the full
     * charts (the reference's graph, marginalizer and prior do too). */
    const unsigned char *kf_fixed;  /* K or NULL: CGMLI_FIX_POSE | _VELOCITY | _BIAS (gyro and accel bias) bits */
    const unsigned char *ext_chart; /* E or NULL (estimate_extrinsics = 1): CGMLI_CHART_FULL, _ROTATION_ONLY
                                       (the translation stays; Plus(T, theta) = (Exp(theta) R, p)) or _FIXED */
    const unsigned char *lm_fixed;  /* L or NULL: 1 holds the inverse distance constant (no Schur elimination) */
} cgmli_window;

typedef struct cgmli_solver_options {
    int precision;           /* CGMLI_PRECISION_FP64 (default) or _MIXED: the LM linearization
                                rounds the bearing factors' Jacobian blocks over the pose,
                                extrinsic and td columns and their robust weights to FP32
                                once formed, and stages the weighted rows of the J^T J pass
                                in FP32; residuals, the depth derivative, costs, gradients,
                                the landmark sums, the reduced system, its Cholesky and every
                                marginalization stay FP64 */
    int refinement_steps;    /* iterative refinement after the FP64 Cholesky (0..2) */
    double initial_lambda;   /* reference: 1e-4 */
    int min_iterations;      /* iterations a window always runs before the time budget may stop it
                                (the reference's minIterations, BackendOptimizer.cpp:177,242) */
    double time_budget_s;    /* <= 0: none.  Otherwise each window's solve stops, as the reference's
                                realtime limit does (realtime_time_limit 0.04 s in its robot
                                configuration): before iteration i >= max(min_iterations, 1) once the
                                budget has elapsed, and after a step solved at i >= min_iterations once
                                it has elapsed and a step was accepted (that step's trial is dropped).
                                Elapsed time is device time since the solve's first kernel. */
} cgmli_solver_options;

typedef struct cgmli_solve_report {
    double initial_cost, final_cost, lambda, predicted_reduction, max_increment;
    int iterations, accepted_steps, converged, status;
} cgmli_solve_report;

typedef struct cgmli_solver cgmli_solver;

/* Message of the last failed call on this thread (never NULL). */
const char *cgmli_last_error(void);

void cgmli_default_options(cgmli_solver_options *options);

/* Host-only check of a batch: builds the device layout of the windows on up to
 * `threads` host threads (0: all) without touching a CUDA device, and verifies
 * its invariants (the landmark order is a permutation of each window's
 * landmarks, observation ranges and slots match the caller's data, the key
 * order of the J^T J pass is sorted, every work unit stays in its window and
 * covers each landmark / observation once).  Returns the windows' validation
 * code, or CGMLI_E_INVALID naming the failed invariant; *seconds (may be NULL)
 * receives the build time.  A diagnostic of this library for callers that
 * prepare windows on machines without a GPU; it has no counterpart in the
 * reference. */
int cgmli_topology_check(const cgmli_window *windows, int count, int threads, double *seconds);

/* Work decomposition of a batch and the kernel shapes it is launched with: the
 * work units the host planner cuts, and the compiled variants of the landmark
 * and trial passes (warps per CTA, and the CTAs per SM their register budget is
 * compiled for). */
typedef struct cgmli_tuning {
    int run_landmarks;  /* landmarks per warp run of the linearization and trial passes;
                           0: from the batch size (enough runs to fill the GPU) */
    int pair_chunk;     /* key-ordered observations per warp of the J^T J pass, 8..1024 (0: 32) */
    int schur_rows;     /* landmarks per chunk of the Schur pass, 8..128 (0: 128) */
    int lin_shape;      /* landmark pass: 0: 6 warps x 2 CTAs per SM (168 registers), 1: 8 x 1 (255),
                           2: 4 x 3 (168), 3: 6 x 1 (255) */
    int trial_shape;    /* trial pass: 0: 8 warps x 2 CTAs per SM (128 registers), 1: 8 x 1 (255), 2: 4 x 4 (128) */
    int deterministic;  /* 0: the J^T J and Schur passes add their work units into each window's
                           sums with FP64 atomics (order of additions set by scheduling);
                           1: each window's pair chunks and Schur chunks are split into
                           contiguous units (about 256 observations, 2 Schur chunks; at most
                           128 of each), every unit sums into a slot of its own and
                           one reduction adds a window's slots in unit order, so that a window's
                           result is bitwise the same alone, in any batch, and eager or as a
                           graph (the reference sums with FP64 atomics,
                           src/backend/VisualCudaBatch.cu:85-93).  The autotuner keeps it. */
    double ms;          /* cgmli_solver_autotune: device time of the timed solve */
} cgmli_tuning;
/* cgmli_topology_check with a given work decomposition (NULL: the default). */
int cgmli_topology_check_tuned(const cgmli_window *windows, int count, int threads, const cgmli_tuning *tuning,
                               double *seconds);
/* 64-bit FNV-1a digest of the device layout the host builds for the batch (every
 * index, work-unit and staged array, in upload order), built on up to `threads`
 * host threads without touching a CUDA device.  The layout does not depend on the
 * thread count: the digest is the same for any `threads`.  A diagnostic with no
 * counterpart in the reference. */
int cgmli_topology_digest(const cgmli_window *windows, int count, int threads, const cgmli_tuning *tuning,
                          unsigned long long *digest);

/* Replaces VisualCudaWorkspace construction (src/backend/BackendOptimizer.cpp:334-341). */
int cgmli_solver_create(int device, const cgmli_solver_options *options, cgmli_solver **out);
void cgmli_solver_destroy(cgmli_solver *solver);

/* Topology + upload of a batch of windows (VisualCudaBatch::linearizeSchur with
 * newTopology=true, configureRetained and configureResident;
 * src/backend/VisualCudaBatch.cu:433-511,606-624,673-691).  All later calls
 * operate on these windows, in this order. */
/* Work decomposition used by the next cgmli_solver_set_windows (validated:
 * CGMLI_E_INVALID outside the ranges of cgmli_tuning) and the one in use. */
int cgmli_solver_set_tuning(cgmli_solver *solver, const cgmli_tuning *tuning);
int cgmli_solver_get_tuning(cgmli_solver *solver, cgmli_tuning *tuning);
/* Autotuner: builds the batch with candidate work decompositions and kernel
 * shapes (coordinate search over run_landmarks, pair_chunk and schur_rows from
 * the current ones, then every lin_shape and trial_shape), times `iterations` LM
 * iterations of each from the windows' states on the device, keeps the fastest
 * for later set_windows calls and leaves the batch set with it (states as
 * given).  *best (may be NULL) receives it. */
int cgmli_solver_autotune(cgmli_solver *solver, const cgmli_window *windows, int count, int iterations, cgmli_tuning *best);
int cgmli_solver_set_windows(cgmli_solver *solver, const cgmli_window *windows, int count);
/* Upload new state values only (same topology). */
int cgmli_solver_upload_states(cgmli_solver *solver, const cgmli_window *windows, int count);

/* Device-resident damped LM over every window (the native loop of
 * solveVisualSchur, src/backend/BackendOptimizer.cpp:167-307, with the
 * lambda schedule evaluated on the device).  Asynchronous on the solver's
 * stream; no host round trip between iterations. */
int cgmli_solver_solve(cgmli_solver *solver, int max_iterations);
int cgmli_solver_synchronize(cgmli_solver *solver);
/* VisualCudaBatch::readResident (src/backend/VisualCudaBatch.cu:704-713). */
int cgmli_solver_read_states(cgmli_solver *solver, cgmli_window *windows, int count);
int cgmli_solver_read_reports(cgmli_solver *solver, cgmli_solve_report *reports, int count);

/* One damped step at fixed lambda from the current states, without moving
 * them: linearizeSchur + linearizeRetained + solveOnline
 * (src/backend/VisualCudaBatch.cu:530-604).  Writes, for window w, the
 * increment (N_r state tangents then L inverse distances), the linearized
 * cost, the predicted reduction, the trial cost and whether it is valid. */
int cgmli_solver_step(cgmli_solver *solver, double lambda);
int cgmli_solver_read_step(cgmli_solver *solver, int window, double *increment, double *cost,
                           double *predicted, double *trial_cost, int *trial_valid);
/* Reduced system of the last cgmli_solver_step of window w: S (N_r x N_r
 * row-major, damped at that lambda) and its right-hand side, as factored: with
 * solve-time charts, restricted to the free directions (a rotation-only
 * extrinsic's theta columns hold M^T S M, M = [[p]x; I]) with identity rows and
 * zero right-hand side at the fixed and folded columns. */
int cgmli_solver_read_reduced(cgmli_solver *solver, int window, double *S, double *rhs);
/* Sizes: N_r of window w. */
int cgmli_solver_window_dims(cgmli_solver *solver, int window, int *retained, int *landmarks);

/* Elapsed device milliseconds of the last cgmli_solver_solve / _step measured
 * with CUDA events on the solver's stream, and the number of kernel launches. */
int cgmli_solver_last_timing(cgmli_solver *solver, double *milliseconds, int *launches);
/* Device bytes the solver's grow-only arrays hold (they stay allocated until
 * cgmli_solver_destroy).  A diagnostic of this library; no counterpart in the
 * reference. */
int cgmli_solver_device_bytes(cgmli_solver *solver, long long *bytes);

/* Per-factor evaluation of every bearing factor of the batch at the accepted
 * states (VisualCudaBatch::evaluate, src/backend/VisualCudaBatch.cu:404-431):
 * the whitened residual, the validity and, with derivatives, the tangent
 * Jacobian before the robust loss.  The reference returns ambient 2x7 blocks
 * that its caller lifts by the PlusJacobian; these are the lifted (left SE(3)
 * tangent) blocks directly.  cgmli_solver_read_factors copies window w's
 * num_observations factors in the caller's observation order: residuals 2 per
 * factor, valid 1 per factor, jacobians CGMLI_FACTOR_JACOBIAN per factor (NULL:
 * skipped; needs derivatives), row-major 2 x 26 over the columns anchor pose
 * [0, 6), observer pose [6, 12), anchor camera extrinsic [12, 18), observer
 * camera extrinsic [18, 24), time offset 24, inverse distance 25.  A factor whose
 * two cameras share one extrinsic block carries that block's whole derivative in
 * [12, 18) and zeros in [18, 24); a same-epoch factor has zero pose columns, and
 * with a shared extrinsic zero extrinsic columns too (the reference requires
 * them to cancel exactly).  Extrinsic and time-offset columns are filled only
 * for windows that estimate them.  Asynchronous; the read waits. */
#define CGMLI_FACTOR_JACOBIAN 52
int cgmli_solver_evaluate(cgmli_solver *solver, int derivatives);
int cgmli_solver_read_factors(cgmli_solver *solver, int window, double *residuals, int *valid, double *jacobians);

/* ---- Caller-evaluated factors --------------------------------------------------
 * The reference keeps factors its device path does not support on the CPU and
 * hands their normal equations to each solveOnline call (retainedH, retainedG;
 * src/backend/VisualCudaBatch.hpp:61, evaluated at src/backend/BackendOptimizer.cpp:
 * 210-221 and added to the trial cost at :276-279).  cgmli_solver_solve_host runs
 * the same damped LM as cgmli_solver_solve with such factors: at every new
 * linearization point of a window it calls fn with trial = 0, the window's
 * accepted states (poses K*7, speed/bias K*9, extrinsics E*7, td 1) and zeroed
 * H (N_r x N_r row-major, the window's retained tangent columns) and g (N_r);
 * fn writes the factors' Gauss-Newton H = J^T J and gradient g = J^T r and their
 * cost 0.5 |r|^2, which are added to the window's retained system and cost.
 * Before each acceptance test it calls fn with trial = 1, the candidate states
 * and H = g = NULL for the cost alone.  Windows with has_host[w] = 0 (or
 * has_host NULL: every window) are not called.  fn returns 0, or nonzero to fail
 * the window with CGMLI_E_NONFINITE.  Unlike cgmli_solver_solve the host takes
 * part in every iteration: after each linearization and after each trial the
 * library waits for the device and copies the states of the called windows,
 * as the reference's non-resident loop does; fn runs on the calling thread. */
typedef int (*cgmli_host_factor_fn)(void *ctx, int window, int trial, const double *poses, const double *speed_bias,
                                    const double *extrinsics, const double *td, double *H, double *g, double *cost);
int cgmli_solver_solve_host(cgmli_solver *solver, int max_iterations, const unsigned char *has_host, cgmli_host_factor_fn fn,
                            void *ctx);

/* Device-side snapshot of the accepted states and its restore: the numeric
 * checkpoint / rollback of a backend transaction
 * (src/backend/BackendOptimizer.cpp:609-641, FixedLagBackend.cpp:171-179). */
int cgmli_solver_checkpoint(cgmli_solver *solver);
int cgmli_solver_rollback(cgmli_solver *solver);

/* Per-kernel CUDA-event timing.  enable=1 starts recording events around every
 * launch (and clears the totals); ms[k] / calls[k] return the accumulated time
 * and launch count of kernel kind k since then, for k in
 * CGMLI_KERNEL_* (ms and calls hold CGMLI_KERNEL_KINDS entries). */
enum { CGMLI_KERNEL_ZERO = 0, CGMLI_KERNEL_LINEARIZE, CGMLI_KERNEL_RETAINED, CGMLI_KERNEL_FACTOR, CGMLI_KERNEL_CANDIDATE,
       CGMLI_KERNEL_BACKSUB_TRIAL, CGMLI_KERNEL_RETAINED_TRIAL, CGMLI_KERNEL_LM_UPDATE, CGMLI_KERNEL_ACCEPT,
       CGMLI_KERNEL_LIN_PAIRS, CGMLI_KERNEL_LIN_SCHUR, CGMLI_KERNEL_KINDS };
/* CGMLI_KERNEL_LINEARIZE is the per-landmark pass of the linearization (factor
 * evaluation, cross vectors); _LIN_PAIRS the J^T J / J^T r pass; _LIN_SCHUR the
 * lambda-dependent Schur term. */
int cgmli_solver_kernel_times(cgmli_solver *solver, int enable, double *ms, int *calls);

/* Schur marginalization of one keyframe per window at the current states
 * (Marginalizer::compute, src/backend/Marginalizer.cpp:284-474, with the
 * elimination set of SlidingWindowManager::marginalize,
 * src/backend/SlidingWindowManager.cpp:627-652).  victim_kf[w] is the
 * keyframe removed from window w; policy is CGMLI_MARGIN_OLD or
 * CGMLI_MARGIN_SECOND_NEW. */
int cgmli_solver_marginalize(cgmli_solver *solver, const int *victim_kf, int policy);
/* CGMLI_MARGIN_SECOND_NEW_IMU_MERGE is SECOND_NEW as the reference runs it in
 * production (SlidingWindowManager::prepareEviction, src/backend/
 * SlidingWindowManager.cpp:263-310, mergeBodyImuRecords, src/factor/
 * BodyImuFactor.cpp:306-388): when the victim has exactly two IMU edges
 * (left -> victim -> right), its speed/bias is not in the prior and the batch's
 * samples are on the device (cgmli_solver_set_imu_samples, the two edges' ranges
 * contiguous in one stream), the edges leave the problem instead of entering the
 * Schur step and are replaced by one factor re-integrated over [t_left, t_right]
 * at the left keyframe's accepted bias, computed on the device with the prior.
 * An interval longer than the maximum duration drops both edges without a
 * replacement (the reference's suppressed factor); otherwise the merged interval
 * may hold at most the maximum number of samples (CGMLI_E_LIMIT).  Windows that
 * do not meet the conditions keep the Schur bridge of CGMLI_MARGIN_SECOND_NEW.
 * Limits default to the reference's maxImuIntervalSeconds = 10 and
 * maxImuSamplesPerEpoch = 10000.  cgmli_solver_read_merged_imu gives window w's
 * outcome (CGMLI_IMU_MERGE_*) and, when reintegrated, the new factor; a failed
 * re-integration returns its CGMLI_E_* code. */
int cgmli_solver_set_imu_merge_limits(cgmli_solver *solver, double max_interval_s, int max_samples);

/* Conditional information of the calibration blocks given every other state of
 * each window at its accepted states (BackendOptimizer::calibrationInformation,
 * src/backend/BackendOptimizer.cpp:1084-1170): the visual factors (Huber-weighted,
 * with the derivatives of every extrinsic and the time offset whether estimated
 * or not), every IMU factor and, with include_prior, the square-root prior are
 * linearized; every landmark range is eliminated by its scalar Schur complement
 * (ranges with information at or below max(1e-12, 1e-9 max) skipped); the poses
 * and speed/biases are removed by the eigen-based PSD solve with the cutoff
 * max(1e-12, 1e-9 lambda_max) (significantly negative eigenvalues:
 * CGMLI_E_INDEFINITE).  A window without calibration Jacobians reports
 * CGMLI_E_INVALID.  The result is laid out per block: each extrinsic as
 * [theta(3), p(3)] (the physical translation, dp = rho - [p]x dtheta), the time
 * offset as one entry; symmetrized, with negative round-off eigenvalues clamped
 * to 0.  The reference lays out one camera extrinsic and the time offset (its
 * first 7 entries); with several extrinsic blocks each gets its 6.  Results
 * replace a previous marginalization's (read_prior then fails until the next
 * cgmli_solver_marginalize). */
int cgmli_solver_calibration_information(cgmli_solver *solver, int include_prior);
/* size = calibration entries, blocks as CGMLI_PRIOR_EXTRINSIC / _TIME_OFFSET
 * (kind, index); conditional size x size row-major; eigenvalues ascending. */
int cgmli_solver_read_calibration_information(cgmli_solver *solver, int window, int *size, int *num_blocks, int *block_kind,
                                              int *block_index, double *conditional, double *eigenvalues);
int cgmli_solver_read_merged_imu(cgmli_solver *solver, int window, int *state, cgmli_frozen_imu *imu);
/* Result of window w: rank and separator width, then (when the buffers are
 * not NULL) the separator blocks, their ambient references, A
 * (rank x cols, row-major) and r0.  Call once with NULL buffers for sizes. */
int cgmli_solver_read_prior(cgmli_solver *solver, int window, int *rank, int *cols, int *num_blocks,
                            int *block_kind, int *block_index, double *reference, double *A, double *r0,
                            double *formation /* 4: robust cost, linearized |r|^2, eliminated reduction, cutoff */);

/* Dense FP64 marginalization helpers with the semantics of
 * MarginalCudaWorkspace (src/backend/VisualCudaBatch.cu:911-957).
 * Matrices are column-major, host memory in and out. */
int cgmli_marg_eigen(const double *H, int n, double *eigenvalues, double *eigenvectors);
int cgmli_marg_psd_solve(const double *H, const double *rhs, int n, int columns,
                         double absolute_cutoff, double relative_cutoff, double *solution);
int cgmli_marg_subtract(const double *coupling, const double *solution, int eliminated, int retained,
                        double *H, double *g);

/* Allocation-free form of cgmli_marg_eigen, for callers that must not
 * allocate device memory: a process whose GPU also runs latency-critical work
 * (cudaFree synchronizes the whole device), or whose device memory is owned by
 * another allocator.  This entry point has no counterpart in the reference.
 * H (n x n, column-major, lower triangle read), eigenvalues (n, ascending) and
 * eigenvectors (n x n, column-major) are DEVICE pointers owned by the caller;
 * stream is a cudaStream_t (NULL: the default stream).  Every call waits for
 * the stream before it returns (it copies the solver's status word to the host
 * and synchronizes), so it cannot be called while that stream, or any stream,
 * is being captured into a CUDA graph.  The solver's work arrays live in one
 * fixed device array of about 1 MiB that every GPU loading the library holds
 * until the process exits, so n is limited to CGMLI_MARG_EIGEN_NOALLOC_MAX_N
 * (larger n: CGMLI_E_LIMIT).  The first call on a device looks the array's
 * address up (set-up).  All calls share the array: calls that overlap on the
 * GPU (other host threads or streams) race and must be serialized by the
 * caller. */
#define CGMLI_MARG_EIGEN_NOALLOC_MAX_N 256
int cgmli_marg_eigen_noalloc(const double *H, int n, double *eigenvalues, double *eigenvectors, void *stream);

/* ---- Outlier gate and refits ---------------------------------------------------
 * cgmli_solver_solve_gated is cgmli_solver_solve with the reference's whitened
 * pre-loss NIS gate and outlier refits (BackendOptimizer::statisticalGate and
 * the gates and refit loop of optimizeImpl, src/backend/BackendOptimizer.cpp:
 * 394-472,669-686,1030-1079): with pre_gate, the gate first runs at the initial
 * states (the reference's pre-NIS, skipped by its skipPreNis); after each pass
 * every visual factor of the window still in the
 * problem is evaluated at the accepted state without the robust loss; those with
 * |r|^2 above nis_threshold (the reference's visualNisThreshold, 9.21) are
 * rejected for good; a window that rejected factors, has refits left (at most
 * max_refits, the reference's maxOutlierRefits = 3) and iteration budget left
 * is solved again from its state with the initial lambda.  All passes share
 * max_iterations, each charged at least one iteration.  The factors rejected by
 * the last gate stay rejected without a further refit.  IMU factors and the
 * prior are not gated (infinite thresholds in the reference).  Everything runs
 * on the device; a rejection persists until the next cgmli_solver_set_windows
 * (checkpoint / rollback restore states only).
 * cgmli_solver_read_gate reports window w's gate and, when rejected is not
 * NULL, marks each of its num_observations factors (caller order) 1 if rejected. */
typedef struct cgmli_gate_report {
    int passes;          /* LM passes run: 1 + outlier refits */
    int rejected_pre;    /* rejected by the gate before the first solve */
    int evaluated;       /* visual factors evaluated by the last gate */
    int rejected_last;   /* of them, rejected by the last gate (no refit followed) */
    int rejected_total;  /* visual factors rejected since cgmli_solver_set_windows */
    double nis_sum, nis_max; /* whitened pre-loss |r|^2 of the last gate's evaluated factors */
} cgmli_gate_report;
int cgmli_solver_solve_gated(cgmli_solver *solver, int max_iterations, double nis_threshold, int max_refits, int pre_gate);
int cgmli_solver_read_gate(cgmli_solver *solver, int window, cgmli_gate_report *report, unsigned char *rejected);

/* ---- IMU preintegration ------------------------------------------------------
 * Batched construction of frozen IMU factors, the device form of what the
 * reference does on the host per factor when it builds or refreshes a
 * BodyImuCost (src/factor/BodyImuFactor.cpp:136-166, called on bias drift by
 * src/backend/FixedLagBackend.cpp:395-411):
 *   - the sample checks of validImuInterval (src/factor/BodyImuFactor.cpp:10-28);
 *   - ImuError::redoPreintegration (src/factor/ImuError.cpp:254-462) at the
 *     interval's linearization bias: rotation, velocity and position deltas,
 *     their bias Jacobians, the noise covariance propagated through the 15x15
 *     transition, and the whitening W = diag(1/sqrt(lambda)) U^T of
 *     PseudoInverse::symmSqrtU (src/factor/PseudoInverse.hpp:117-145);
 *   - the gyro readings at both ends (gyroAt, src/factor/BodyImuFactor.cpp:29-38)
 *     and the sensor pose T_BS.
 * Times are integer nanoseconds, as the reference's cgmli::Time; a difference
 * converts to seconds as Duration::toSec does (whole seconds + 1e-9 * nsec). */
typedef struct cgmli_imu_parameters {
    double sigma_g_c, sigma_a_c;     /* gyro / accelerometer noise densities */
    double sigma_gw_c, sigma_aw_c;   /* gyro / accelerometer bias random-walk densities */
    double g_max, a_max;             /* saturation: a reading above it inflates that noise */
    double g;                        /* gravity magnitude, copied to frozen.gravity */
    double max_sample_gap;           /* seconds; a longer gap inside an interval is invalid */
    double sensor_position[3], sensor_quaternion[4]; /* T_BS, quaternion [x, y, z, w] */
} cgmli_imu_parameters;

/* Preintegrates count intervals.  Sample j has time sample_time_ns[j] and
 * readings sample_readings[6j..6j+5] = [gyro (rad/s), accelerometer (m/s^2)].
 * Interval i integrates the samples [range[2i], range[2i+1]) (strictly
 * increasing times, first <= t0_ns[i] < t1_ns[i] <= last; ranges may overlap)
 * at the bias bias[6i..6i+5] = [b_g, b_a] and writes every field of frozen[i].
 * CGMLI_E_INVALID names the first malformed interval in cgmli_last_error();
 * CGMLI_E_NONFINITE reports an interval whose result is not finite. */
int cgmli_imu_preintegrate(const cgmli_imu_parameters *params, const long long *sample_time_ns, const double *sample_readings,
                           int num_samples, const int *range, const long long *t0_ns, const long long *t1_ns,
                           const double *bias, int count, cgmli_frozen_imu *frozen);
/* Device time (CUDA events around the kernel) of the last successful
 * cgmli_imu_preintegrate call in this process. */
int cgmli_imu_last_timing(double *kernel_ms);

/* Resident refresh of a solver's IMU factors.  cgmli_solver_set_imu_samples
 * keeps on the device the samples of the current batch's IMU factors: factor q
 * (windows in order, each window's imu[] in order) integrates samples
 * [range[2q], range[2q+1]) from t0_ns[q] to t1_ns[q] with params (those the
 * factors were built with).  The next cgmli_solver_set_windows drops them.
 * cgmli_solver_refresh_imu then re-preintegrates, on the solver's stream at
 * the accepted states, every factor whose first keyframe's bias moved from the
 * factor's reference bias by more than gyro_threshold in |d b_g| or
 * accel_threshold in |d b_a| (bodyImuNeedsRefresh + makeBodyImuFactor before
 * each optimization, src/backend/FixedLagBackend.cpp:395-411, thresholds 0.0003
 * and 0.02 there), replacing it in place for the next solve or marginalization;
 * states and checkpoints are untouched.  With refreshed == NULL the call only
 * enqueues the work (no host round trip); otherwise it waits, stores the number
 * of replaced factors and returns CGMLI_E_INVALID / _E_NONFINITE for a factor
 * whose samples or result were bad (such a factor keeps its previous value).
 * A factor whose range is empty (range[2q] == range[2q+1]) has no samples: the
 * refresh keeps it as given (the served mode uses this for windows that bring no
 * samples).
 * cgmli_solver_read_imu copies window w's current factors (num_imu) to the host. */
int cgmli_solver_set_imu_samples(cgmli_solver *solver, const cgmli_imu_parameters *params, const long long *sample_time_ns,
                                 const double *sample_readings, int num_samples, const int *range, const long long *t0_ns,
                                 const long long *t1_ns);
int cgmli_solver_refresh_imu(cgmli_solver *solver, double gyro_threshold, double accel_threshold, int *refreshed);
int cgmli_solver_read_imu(cgmli_solver *solver, int window, cgmli_frozen_imu *imu);

/* ---- Served mode: continuous batching of window solves ---------------------
 * Windows from many rigs arrive as independent requests.  A request is one
 * window (its arrays are the caller's and must stay valid and unmodified until
 * the request completes; the solved states are written back into them),
 * solved with options.iterations damped LM iterations and, when victim_kf >= 0,
 * marginalized (options.policy).  A scheduler thread admits queued requests in
 * arrival order into the next batch while the batch stays within
 * max_batch_windows windows and its estimated device footprint within
 * memory_budget_bytes; the host build and upload of one batch overlap the
 * device work of the previous one (two solvers on two streams), so requests
 * that arrive while the GPU is busy join the next batch.  Every window of a
 * batch is solved exactly as alone (same arithmetic up to the order of FP64
 * reductions).  The reference solves one window per backend step and has no
 * served mode; this is the batched form of its solveVisualSchur +
 * Marginalizer::compute. */
typedef struct cgmli_server_options {
    int device;
    int max_batch_windows;          /* 0: 512 */
    long long memory_budget_bytes;  /* 0: 40 GiB; device bytes of both solvers together (see
                                       cgmli_server_device_bytes) */
    int iterations;                 /* LM iterations per request, >= 1 */
    int policy;                     /* CGMLI_MARGIN_OLD, _SECOND_NEW or _SECOND_NEW_IMU_MERGE for requests
                                       with a victim (the merge needs the request's IMU samples; default
                                       limits of cgmli_solver_set_imu_merge_limits) */
    double nis_threshold;           /* > 0: solve with the NIS gate and outlier refits
                                       (cgmli_solver_solve_gated); 0: plain solve */
    int max_refits;                 /* refits of the gated solve (reference: 3) */
    int pre_gate;                   /* gated solve: gate at the submitted states first */
    int precision;                  /* CGMLI_PRECISION_FP64 or _MIXED (cgmli_solver_options) */
    /* requests with IMU samples (cgmli_server_submit_request): the model of the
       samples and the drift thresholds of the refresh before the solve
       (cgmli_solver_refresh_imu; the reference's FixedLagBackend uses 3e-4 and 0.02) */
    cgmli_imu_parameters imu_params;
    double imu_gyro_threshold, imu_accel_threshold;
    int calibration_include_prior;  /* requests for the calibration information: include the prior */
    int deterministic;              /* 1: the solvers sum with cgmli_tuning.deterministic = 1, so a request's
                                       solved states and report are bitwise those of its window solved
                                       alone that way, whatever batch it joins (the marginal prior stays
                                       at rounding level: the marginalization adds with atomics) */
} cgmli_server_options;

/* A served request with the optional parts of a backend step around the solve:
 * the IMU samples of the window's IMU factors, so that factors whose bias drifted
 * are re-preintegrated on the device before the solve (the resident refresh of
 * FixedLagBackend.cpp:395-411; layout as cgmli_solver_set_imu_samples for this
 * window's factors, ranges into this request's samples), and the conditional
 * calibration information at the solved states (cgmli_solver_calibration_information;
 * BackendOptimizer::calibrationInformation, BackendOptimizer.cpp:1084-1170).
 * The arrays are the caller's and stay valid until the request completes. */
typedef struct cgmli_server_request {
    cgmli_window *window;
    int victim_kf;                      /* -1: no marginalization */
    const long long *imu_sample_time_ns;
    const double *imu_sample_readings;  /* 6 per sample: gyro, accelerometer */
    int num_imu_samples;                /* 0: no samples (the factors are used as given) */
    const int *imu_range;               /* 2 per IMU factor of the window */
    const long long *imu_t0_ns, *imu_t1_ns;
    int calibration_information;        /* 1: compute it for this request */
} cgmli_server_request;
typedef struct cgmli_server cgmli_server;

int cgmli_server_create(const cgmli_server_options *options, cgmli_server **out);
/* Completes every submitted request, then releases the server. */
void cgmli_server_destroy(cgmli_server *server);
/* Queues a request; the window is validated here (CGMLI_E_INVALID / _LIMIT). */
int cgmli_server_submit(cgmli_server *server, cgmli_window *window, int victim_kf, long long *ticket);
/* CGMLI_OK with the report (status of the solve, or of the marginalization when
 * that failed) and the submit-to-completion latency once the request is
 * complete; CGMLI_E_PENDING while it is not and wait == 0.  wait != 0 blocks. */
int cgmli_server_poll(cgmli_server *server, long long ticket, int wait, cgmli_solve_report *report, double *latency_ms);
/* cgmli_server_submit with the optional IMU samples and calibration request. */
int cgmli_server_submit_request(cgmli_server *server, const cgmli_server_request *request, long long *ticket);
/* The IMU factors (num_imu) of a completed request with samples, after the refresh;
 * refreshed = how many were re-preintegrated. */
int cgmli_server_read_imu(cgmli_server *server, long long ticket, cgmli_frozen_imu *imu, int *refreshed);
/* The calibration information of a completed request that asked for it, laid out
 * as cgmli_solver_read_calibration_information (sizes first with NULL buffers);
 * the calibration call's status when it failed for this window. */
int cgmli_server_read_calibration_information(cgmli_server *server, long long ticket, int *size, int *num_blocks, int *block_kind,
                                              int *block_index, double *conditional, double *eigenvalues);
/* Outcome of a completed request's IMU merge (server policy
 * CGMLI_MARGIN_SECOND_NEW_IMU_MERGE, request with a victim), as
 * cgmli_solver_read_merged_imu: *state is CGMLI_IMU_MERGE_*, and imu (may be NULL)
 * receives the merged factor when it was re-integrated. */
int cgmli_server_read_merged_imu(cgmli_server *server, long long ticket, int *state, cgmli_frozen_imu *imu);
/* Prior of a completed request with a victim, laid out as cgmli_solver_read_prior
 * (sizes first with NULL buffers). */
int cgmli_server_read_prior(cgmli_server *server, long long ticket, int *rank, int *cols, int *num_blocks, int *block_kind,
                            int *block_index, double *reference, double *A, double *r0);
/* Gate report and rejected factors (num_observations flags, or NULL) of a
 * completed request of a server with nis_threshold > 0. */
int cgmli_server_read_gate(cgmli_server *server, long long ticket, cgmli_gate_report *report, unsigned char *rejected);
/* Frees a completed request's record. */
int cgmli_server_release(cgmli_server *server, long long ticket);
/* Device bytes both solvers of the server hold (each keeps its grow-only arrays
 * between batches).  Admission keeps this within memory_budget_bytes: a batch
 * may use at most half of the budget, counting the arrays' growth headroom (a
 * window that alone exceeds that half still runs, alone in its batch, and can
 * take the total above the budget).
 * A diagnostic of this library; no counterpart in the reference. */
int cgmli_server_device_bytes(cgmli_server *server, long long *bytes);
/* Replays a request trace from a host thread (load testing): request i submits
 * windows[i] with victims[i] at arrival_s[i] seconds (non-decreasing) after the
 * call starts; latency_ms[i] is measured from that scheduled arrival to the
 * completion, so queueing delay is included; status[i] is the request's solve
 * status; span_s the time from the start to the last completion.  A window
 * listed again is resubmitted only after its earlier request completed.
 * Returns after every submitted request completed. */
int cgmli_server_replay(cgmli_server *server, cgmli_window *const *windows, const int *victims, const double *arrival_s,
                        int count, double *latency_ms, int *status, double *span_s);

#ifdef __cplusplus
}
#endif
#endif
