/* hzlb.h -- C ABI of the B200 ensemble forecast/analysis path.
 *
 * This library replaces, for the reference pvasbob/HZL-stochasticFlowInference, the
 * GPU solver and the per-member loops of its ensemble, particle-filter and EnKF drivers:
 *
 *   reference interface (include/hzl/...)              replaced by
 *   CudaSolver(n, Parameters, initial)                 hzlb_ensemble_create + hzlb_set_state
 *     (cuda_solver.hpp:9, cuda_solver.cu:126-171)
 *   CudaSolver::step(dt) / step(dt, forcing)           hzlb_set_forcing + hzlb_step
 *     (cuda_solver.hpp:13-14, cuda_solver.cu:173-218)
 *   CudaSolver::coefficients()                         hzlb_get_state
 *     (cuda_solver.hpp:16, cuda_solver.cu:222-235)
 *   Solver::diagnostics() per member                   hzlb_diagnostics
 *     (solver.hpp:85, solver.cpp:381-397)
 *   Solver::physical_vorticity() per member            hzlb_physical / hzlb_observe
 *     (solver.hpp:86, solver.cpp:398-402)
 *   hzl::ensemble(n, p, dt, steps, count, ...)         hzlb_ensemble_create + hzlb_step +
 *     (inference.hpp:85-86, inference.cpp:555-590)     hzlb_diagnostics
 *   (averaged_)particle_log_likelihood                hzlb_particle_log_likelihood
 *     (filter.hpp:19-24, filter.cpp:141-165)
 *   bootstrap_filter weights / resampling             hzlb_pf_weights, hzlb_systematic_resample,
 *     (filter.hpp:17-18, filter.cpp:66-120)            hzlb_gather_members
 *   ensemble_kalman_filter analysis                    hzlb_enkf_analysis
 *     (filter.hpp:52-54, filter.cpp:237-321)
 *   fit_pod / PODBasis                                 hzlb_fit_pod
 *     (reduced.hpp:6-17, reduced.cpp:8-136)
 *   GalerkinModel (rhs, step)                          hzlb_galerkin_create / _rhs / _step
 *     (reduced.hpp:19-30, reduced.cpp:137-209)
 *
 * Conventions.  Every function returns HZLB_OK (0) or a negative HZLB_E* code; the message
 * of the last failure on the calling thread is hzlb_last_error().  HZLB_EINVAL corresponds
 * to the reference's std::invalid_argument, HZLB_ERUNTIME to std::runtime_error (CFL limit,
 * nonfinite state), HZLB_ECUDA to CUDA failures (std::runtime_error("<op>: <cuda msg>") in
 * the reference).  The caller owns host buffers; the library owns device memory.  Each
 * ensemble handle owns one CUDA stream; calls on one handle are not thread-safe, separate
 * handles are independent.
 *
 * Field layout at this boundary: complex spectra as interleaved (re, im) doubles, n*n
 * entries per member in the reference layout (index y*n + x, Fourier coefficients
 * normalised by 1/n^2 on the forward transform: include/hzl/fft.hpp:7-9).  Members are
 * consecutive.
 */
#ifndef HZLB_H
#define HZLB_H
#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define HZLB_API __attribute__((visibility("default")))
#else
#define HZLB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define HZLB_OK 0
#define HZLB_EINVAL (-1)
#define HZLB_ERUNTIME (-2)
#define HZLB_ECUDA (-3)
#define HZLB_ETIMEOUT (-4)

/* Device status bits returned by hzlb_status. */
#define HZLB_STATUS_CFL 1u       /* dt * max(|u|+|v|) n / 2pi > 0.5 (solver.cpp:213) */
#define HZLB_STATUS_NONFINITE 2u /* nonfinite coefficient after a step (solver.cpp:247-250) */
#define HZLB_STATUS_TIMEOUT 4u

typedef struct hzlb_ensemble hzlb_ensemble;

typedef struct {
    int n;                     /* grid size, power of two in [8, 512] */
    int members;               /* ensemble members held by this handle */
    int precision;             /* 4: complex64 spectra (FP32 path), 8: complex128 (FP64 path) */
    double nu, alpha;          /* viscosity, linear friction (hzl::Parameters, solver.hpp:16-17) */
    int forcing_kmax;          /* forcing stored for columns kx <= forcing_kmax; -1: no forcing */
    int forcing_per_member;    /* 0: one forcing field shared by all members; 1: one per member */
    double noise_sigma;        /* Euler-Maruyama noise amplitude after each step; 0: off */
    int noise_kmax;            /* noise on modes with 1 <= |k|^2 <= noise_kmax^2; needs
                                  3 noise_kmax < n and noise_kmax <= 15 */
    uint64_t seed;             /* Philox key for the noise */
    uint32_t member_base;      /* global index of member 0 (Philox key; sharding offset) */
    int device;                /* CUDA device ordinal */
} hzlb_config;

HZLB_API const char *hzlb_last_error(void);
/* Library version string. */
HZLB_API const char *hzlb_version(void);

HZLB_API int hzlb_ensemble_create(const hzlb_config *config, hzlb_ensemble **out);
HZLB_API void hzlb_ensemble_destroy(hzlb_ensemble *h);

/* Spectral state of members [first, first+count), reference layout (see above).  set_state
 * keeps only the retained 2/3-rule modes, as CudaSolver's constructor and Solver::project do
 * (cuda_solver.cu:158-167, solver.cpp:140-144); nonfinite input is HZLB_EINVAL. */
HZLB_API int hzlb_set_state(hzlb_ensemble *h, const double *spectra, int first, int count);
HZLB_API int hzlb_get_state(hzlb_ensemble *h, double *spectra, int first, int count);
/* The same in the handle's compact device layout ([member][kx 0..K][j 0..2K], K=(n-1)/3,
 * ky = j for j <= K else j - 2K - 1), in the handle's precision (float or double pairs).
 * No layout conversion; used for bulk transfers. */
HZLB_API int hzlb_set_state_compact(hzlb_ensemble *h, const void *compact, int first, int count);
HZLB_API int hzlb_get_state_compact(hzlb_ensemble *h, void *compact, int first, int count);
HZLB_API size_t hzlb_compact_size(const hzlb_ensemble *h); /* complex entries per member */

/* Forcing spectra held constant over each step (the midpoint forcing of the reference's
 * RK4 step, solver.cpp:217-234; CudaSolver::step(dt, forcing), cuda_solver.cu:184-202).
 * Shared forcing: count must be 1.  Must be conjugate-symmetric to 1e-12 and vanish outside
 * columns |kx| <= forcing_kmax (HZLB_EINVAL otherwise). */
HZLB_API int hzlb_set_forcing(hzlb_ensemble *h, const double *spectra, int first, int count);

/* Ornstein-Uhlenbeck shell forcing on the device (the reference's ShellForcing,
 * solver.cpp:67-119, with Philox draws instead of its host mt19937_64 streams: parity is
 * statistical).  Needs forcing_per_member = 1 and forcing_kmax >= kmax.  Every later step is
 * the reference's midpoint scheme: a transition of dt/2, the RK4 stages with that forcing, a
 * transition of dt/2; the modes kmin^2 <= |k|^2 <= kmax^2 of the forcing are owned by the
 * process (others keep what hzlb_set_forcing put there).  initialize != 0 draws the stationary
 * start sigma sqrt(tau/4) (xi1 + i xi2) (initialize_ou, solver.cpp:84-92).  No counterpart
 * entry point in the reference. */
HZLB_API int hzlb_enable_ou(hzlb_ensemble *h, double sigma, double tau, int kmin, int kmax,
                            int initialize);
/* Forcing of members [first, first+count) in the compact forcing layout (forcing_kmax + 1
 * columns of 2K+1 entries) as interleaved doubles. */
HZLB_API int hzlb_get_forcing_compact(hzlb_ensemble *h, double *out, int first, int count);

/* Advance every member by nsteps RK4 steps of size dt (asynchronous on the handle's stream).
 * HZLB_EINVAL for a nonpositive/nonfinite dt or dt * (2 nu K^2 + alpha) > 2.5
 * (cuda_solver.cu:205-208). */
HZLB_API int hzlb_step(hzlb_ensemble *h, double dt, uint64_t nsteps);
/* One RK4 step with CudaSolver::advance's failure semantics (cuda_solver.cu:106-117,
 * 203-215): when the stage-1 velocities of some member violate dt max(|u|+|v|) n/2pi <= 0.5,
 * the state, forcing, clock and step counter are left as they were before the call and
 * HZLB_ERUNTIME ("GPU CFL limit exceeded") is returned.  Synchronous. */
HZLB_API int hzlb_step_checked(hzlb_ensemble *h, double dt);
/* No counterpart in the reference.  How hzlb_step's graphs run the members: 0, one row and one
 * column pass per RK stage over the whole ensemble; 1, the members in two parts, each with its
 * own passes on its own stream, side by side; 2, as 1 with the second part one row pass behind
 * the first, so that one part's row passes (bound by arithmetic) overlap the other's column
 * passes (bound by memory).  Parts need at least 256 members and no device OU forcing (else
 * schedule 0 runs).  Default 1.  Results are identical bit for bit under every schedule. */
HZLB_API int hzlb_set_step_schedule(hzlb_ensemble *h, int schedule);
HZLB_API int hzlb_step_schedule(hzlb_ensemble *h, int *schedule);
/* No counterpart in the reference (its CudaSolver copies each member's state in and out around
 * every step, cuda_solver.cu:173-235).  The ensemble state lives on the host: state_in is read
 * and state_out written (both all members, the compact layout of the configured precision, as
 * hzlb_set_state_compact; they may be the same buffer), nsteps steps in between.  The members
 * go in chunks of about chunk_members (0: a sixteenth of the ensemble, at least 32 members),
 * each chunk's copies overlapping the stepping of the others; pinned host buffers are needed
 * for the overlap.
 * Results equal hzlb_set_state_compact + hzlb_step + hzlb_get_state_compact bit for bit.
 * Asynchronous on the handle's stream; device OU forcing is not supported here. */
HZLB_API int hzlb_step_host(hzlb_ensemble *h, const void *state_in, void *state_out, double dt,
                            uint64_t nsteps, int chunk_members);
/* Waits for the handle's stream; returns the accumulated status bits and clears them. */
HZLB_API int hzlb_status(hzlb_ensemble *h, uint32_t *status);
/* Test hook, no counterpart in the reference: the next row pass of h leaves the first tile
 * copy of one block unissued, so that block's bounded wait (one second of the device's global
 * timer) runs out with no copy in flight; the block records HZLB_STATUS_TIMEOUT and returns,
 * the step's result is not valid, and the context stays usable.  Tests the failure path of
 * the device waits without faulting or hanging the GPU. */
HZLB_API int hzlb_test_inject_wait_timeout(hzlb_ensemble *h);
HZLB_API int hzlb_synchronize(hzlb_ensemble *h);
/* The handle's CUDA stream (a cudaStream_t), for callers that order their own work or
 * record events against the library's kernels. */
HZLB_API void *hzlb_stream(hzlb_ensemble *h);
/* Profiling variant of hzlb_step: runs nsteps steps with individual launches (no graph) and
 * CUDA events around every launch; returns the mean duration in milliseconds of the row-pass
 * and column-pass launches.  Same results as hzlb_step. */
HZLB_API int hzlb_step_profiled(hzlb_ensemble *h, double dt, uint64_t nsteps, double *row_ms,
                                double *column_ms);
/* Simulated time and the noise step counter. */
HZLB_API int hzlb_time(hzlb_ensemble *h, double *time, uint64_t *step_index);
HZLB_API int hzlb_set_time(hzlb_ensemble *h, double time, uint64_t step_index);

/* Per member {time, energy, enstrophy, dissipation, injection, cfl_rate} (hzl::Diagnostics,
 * solver.hpp:24-26); out has 6*members doubles. */
HZLB_API int hzlb_diagnostics(hzlb_ensemble *h, double *out);
/* Physical vorticity of every member, members*n*n doubles indexed [m][y][x]. */
HZLB_API int hzlb_physical(hzlb_ensemble *h, double *out);
/* Physical vorticity at p grid points (x[o], y[o]) of every member: out[m*p + o]. */
HZLB_API int hzlb_observe(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y, size_t p, double *out);

/* ---- particle filter (filter.cpp:65-120) ------------------------------------------- */
/* Every step below runs on the device in FP64, in the reference's order of operations. */
/* Adds the Gaussian observation log-likelihood of every member to log_weights[m] (the
 * residual (field - value)/sd with the log sd + log(2 pi)/2 constants, filter.cpp:66-75);
 * log_weights is a host array of members doubles, read and written. */
HZLB_API int hzlb_pf_loglik(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y, const double *values,
                   const double *sd, size_t p, double *log_weights);
/* Log-sum-exp increment, normalised weights, ESS = 1/sum w^2, max weight of `count` host
 * log-weights (filter.cpp:76-92), computed on h's device.  HZLB_ERUNTIME if the largest
 * log-weight is not finite. */
HZLB_API int hzlb_pf_weights(hzlb_ensemble *h, const double *log_weights, size_t count, double *weights,
                    double *increment, double *ess, double *max_weight);
/* Systematic resampling on h's device: start = u/M, positions start + i/M walked against the
 * sequential cumulative sum of the weights (filter.cpp:102-112).  Bit-exact with the
 * reference given identical weights and u.  h must not be NULL. */
HZLB_API int hzlb_systematic_resample(hzlb_ensemble *h, const double *weights, size_t count, double u,
                             uint32_t *ancestors);

/* Outcome of one observation time of one particle filter (filter.cpp:76-101). */
typedef struct {
    double increment;   /* log-likelihood increment: max + log sum_j exp(l_j - max) */
    double ess;         /* effective sample size 1 / sum_j w_j^2 */
    double max_weight;  /* largest normalised weight */
    int32_t resampled;  /* 1: systematic resampling ran and the members were replaced */
    int32_t collapsed;  /* 1: the largest log-weight was not finite; nothing was changed */
} hzlb_pf_record;
/* The ensemble as members / particles independent bootstrap filters (segments) of
 * `particles` consecutive members each, their weights on the device reset to 1/particles
 * (bootstrap_filter's initial weights, filter.cpp:52).  members must be a multiple of
 * particles, particles >= 2.  Until the first call the whole ensemble is one segment. */
HZLB_API int hzlb_pf_reset(hzlb_ensemble *h, int particles);
/* One observation time of every segment's bootstrap filter, weights resident on the device
 * (filter.cpp:65-120): the observation operator, log w_j = log(w_j) - sum_o [0.5 r^2 + log sd_o
 * + log(2 pi)/2], the increment, normalised weights, ESS and max weight; then, for a segment
 * whose ESS is below particles/2 and whose u[s] lies in [0, 1), systematic resampling with
 * start u[s]/particles, the members replaced by their ancestors (and their forcing when it is
 * per member) and the weights reset to 1/particles -- all without a host round trip.
 *   u:       segments uniforms, or NULL; u[s] < 0 forbids resampling of segment s (the
 *            reference's last observation time).  The reference draws the uniform only when
 *            it resamples, so a caller that draws its u[s] ahead and reuses it until a call
 *            reports the segment resampled consumes the reference's sequence of uniforms.
 *   active:  segments flags, or NULL for all; a segment with flag 0 is left untouched.
 *   records: segments hzlb_pf_record (out).
 *   ancestors:     members entries (out, may be NULL): member i's ancestor (i if unchanged).
 *   weighted_mean: segments x hzlb_compact_size complex entries as interleaved doubles (out,
 *            may be NULL): sum over the segment's members of w_j x_j with the normalised
 *            weights of this time, before any resampling (filter.cpp:113-120). */
HZLB_API int hzlb_pf_assimilate(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y,
                                const double *values, const double *sd, size_t p, const double *u,
                                const uint8_t *active, hzlb_pf_record *records,
                                uint32_t *ancestors, double *weighted_mean);
/* The device weights of hzlb_pf_reset / hzlb_pf_assimilate (members doubles). */
HZLB_API int hzlb_pf_get_weights(hzlb_ensemble *h, double *weights);
/* Replace member i's state with member ancestors[i]'s (and its forcing if per member). */
HZLB_API int hzlb_gather_members(hzlb_ensemble *h, const uint32_t *ancestors);

/* ---- EnKF (filter.cpp:237-321) ------------------------------------------------------ */
/* Multiplicative anomaly inflation of the spectral state about the ensemble mean
 * (filter.cpp:237-253 for the vorticity part). */
HZLB_API int hzlb_inflate(hzlb_ensemble *h, double inflation);
/* Perturbed-observation EnKF analysis of all p observations at once:
 *   X_a = X + A (HA)^T (HA HA^T/(M-1) + R)^{-1} (y + sd*eps - HX) / (M-1)
 * with the p x p innovation system factorised by an FP64 Cholesky on the device.
 * perturbations: M x p standard normals (row m = member).  With p = 1 this equals the
 * reference's serial scalar update (filter.cpp:265-321, no localisation). */
HZLB_API int hzlb_enkf_analysis(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y,
                       const double *values, const double *sd, size_t p,
                       const double *perturbations);
/* No counterpart in the reference (it defines no innovation-consistency test).  The same
 * analysis, returning the normalised innovation statistic of the forecast ensemble,
 *   nis = dbar^T (HA HA^T/(M-1) + R)^{-1} dbar / p,   dbar = y - mean(HX),
 * which is 1 in expectation for a consistent forecast.  With nis_limit > 0 and nis above it
 * the state is left unchanged and *applied = 0 (the caller falls back to another forecast);
 * otherwise the update is applied and *applied = 1.  perturbations: as above, or NULL to draw
 * them on the device from the Philox stream keyed by (perturbation_seed, member_base + m)
 * with counter (cycle, observation pair). */
HZLB_API int hzlb_enkf_analysis_nis(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y,
                                    const double *values, const double *sd, size_t p,
                                    const double *perturbations, uint64_t perturbation_seed,
                                    uint64_t cycle, double nis_limit, double *nis, int *applied);
/* No counterpart entry point in the reference (it runs one process): the ensemble-space
 * weights of the perturbed-observation EnKF (filter.cpp:265-321, batched) for `members`
 * members whose predicted observations were gathered from several ranks,
 *   W = HA^T (HA HA^T/(M-1) + R)^{-1} (y + sd eps - HX) / (M-1)
 * (M x M, row-major, rows: contributing member, columns: updated member), with the FP64
 * innovation system factorised and solved on h's device (the solve of hzlb_enkf_analysis).
 * hx, eps: device arrays, members x p (row m = member); values, sd: host arrays of p;
 * W: device array members x members (out); nis (may be NULL) receives dbar^T S^{-1} dbar / p.
 * Synchronous on h's stream; the caller orders its own writes of hx and eps before the call. */
HZLB_API int hzlb_enkf_weights(hzlb_ensemble *h, const double *hx, const double *values,
                               const double *sd, const double *eps, int members, size_t p,
                               double *W, double *nis);
/* FP64 product on the device's FP64 tensor cores (the analysis's mma.sync kernel):
 *   C[m][n] = alpha sum_k A(m,k) B(k,n) + beta C[m][n],
 *   A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn], C row-major with leading dimension ldc.
 * Device pointers; C must not overlap A or B.  Asynchronous on `stream` (a cudaStream_t or
 * NULL).  No counterpart in the reference. */
HZLB_API int hzlb_dgemm(int M, int N, int K, double alpha, const double *A, long long sam,
                        long long sak, const double *B, long long sbk, long long sbn, double beta,
                        double *C, long long ldc, void *stream);
/* No counterpart in the reference.  Device address of the compact state (members x
 * hzlb_compact_size complex entries of the configured precision, member-major), for device
 * code that reads or modifies the ensemble in place (the learned reduced forecast).  Valid
 * until the handle is destroyed; call it again before each modification so the next step
 * does not reuse velocities cached from the old state. */
HZLB_API int hzlb_state_device(hzlb_ensemble *h, void **state);
/* Ensemble mean in the compact layout as interleaved doubles (hzlb_compact_size complex
 * entries), summed in member order as the reference's filters do (filter.cpp:238-243). */
HZLB_API int hzlb_ensemble_mean(hzlb_ensemble *h, double *mean);
/* Weighted member sum sum_m w[m] x_m in the compact layout as interleaved doubles, in member
 * order (the bootstrap filter's weighted mean, filter.cpp:113-120); w: members doubles. */
HZLB_API int hzlb_weighted_mean(hzlb_ensemble *h, const double *weights, double *mean);
/* The member mean of the compact state into a device array of hzlb_compact_size complex
 * entries in the handle's precision (summed in FP64 over member slices). */
HZLB_API int hzlb_ensemble_mean_device(hzlb_ensemble *h, void *mean);

/* ---- drop-in drivers for the reference's ensemble entry points ---------------------- */
/* hzl::Parameters (include/hzl/solver.hpp:15-23). */
typedef struct {
    double viscosity, friction, forcing_sigma, forcing_tau;
    int forcing_min, forcing_max;
} hzlb_parameters;
/* hzl::Observation (include/hzl/inference.hpp:33-36). */
typedef struct {
    uint64_t step;
    uint32_t x, y;
    double value, standard_deviation;
} hzlb_observation;
/* hzl::Dataset (include/hzl/inference.hpp:37-46). */
typedef struct {
    int n;
    double dt;
    int stochastic, forcing_min, forcing_max;
    size_t count;
    const hzlb_observation *observations;
} hzlb_dataset;
/* Dataset files.  hzlb_dataset_save writes HZL_OBSERVATIONS_V2 text, byte for byte as
 * hzl::Dataset::save (include/hzl/inference.hpp:43-45, src/inference.cpp:214-226);
 * hzlb_dataset_load reads V1 or V2 files as hzl::Dataset::load (src/inference.cpp:227-257).
 * Both validate as hzl::Dataset::validate (src/inference.cpp:197-213): HZLB_EINVAL for an
 * invalid dataset, HZLB_ERUNTIME for a malformed or unwritable file.  load: *count receives
 * the number of observations; with observations NULL only the header is filled (a first call
 * to size the buffer), else capacity must hold *count entries and header->observations points
 * at them. */
HZLB_API int hzlb_dataset_save(const hzlb_dataset *data, const char *path);
HZLB_API int hzlb_dataset_load(const char *path, hzlb_dataset *header,
                               hzlb_observation *observations, size_t capacity, size_t *count);
/* hzl::Dataset::validate (src/inference.cpp:197-213) alone. */
HZLB_API int hzlb_dataset_validate(const hzlb_dataset *data);
/* hzl::FilterRecord without the field (include/hzl/filter.hpp:5-9). */
typedef struct {
    uint64_t step;
    double log_likelihood_increment, effective_particles, maximum_weight;
} hzlb_filter_record;
/* hzl::EnKFOptions (include/hzl/filter.hpp:43-50). */
typedef struct {
    double inflation, localization_radius;
    uint64_t forecast_steps, forecast_every;
} hzlb_enkf_options;
/* hzl::EnsembleFilterRecord without the field (include/hzl/filter.hpp:37-42). */
typedef struct {
    uint64_t step;
    double forecast_sensor_rmse, posterior_spread;
    int is_forecast;
} hzlb_enkf_record;

/* hzl::ensemble(n, p, dt, steps, count, workers, seed) (include/hzl/inference.hpp:85-86,
 * src/inference.cpp:555-590): member i starts from "zero" with OU forcing seeded by
 * stream_seed(seed, i); out receives count x {time, energy, enstrophy, dissipation,
 * injection, cfl_rate} in member order.  All members advance together on the device. */
HZLB_API int hzlb_run_ensemble(int n, const hzlb_parameters *params, double dt, uint64_t steps,
                               uint64_t count, uint64_t seed, int precision, int device,
                               double *out);
/* hzl::Solver::linearized_drift(state, direction) and Solver::adjoint_drift(state, cotangent)
 * (include/hzl/solver.hpp:70-71, src/solver.cpp:264-324) for `count` pairs at once, FP64 on
 * the device: states, directions / cotangents and out are count x n*n complex spectra in the
 * reference's Field layout (y outer, x inner).  The Hermitian part of each input on the active
 * (dealiased) modes is used, which is what the reference reads of the projected fields it
 * passes (its physical fields keep their real part only); out is zero off the active modes.
 * params: the solver's parameters (viscosity and friction enter; the forcing shell is
 * validated as the Solver constructor does). */
HZLB_API int hzlb_linearized_drift(int n, const hzlb_parameters *params, const double *states,
                                   const double *directions, uint64_t count, int device,
                                   double *out);
HZLB_API int hzlb_adjoint_drift(int n, const hzlb_parameters *params, const double *states,
                                const double *cotangents, uint64_t count, int device,
                                double *out);
/* hzl::AdjointEvaluation (include/hzl/inference.hpp:55-58). */
typedef struct {
    double value, gradient[2];
    uint64_t checkpoint_fields, peak_block_fields, replayed_steps;
} hzlb_adjoint_evaluation;
/* hzl::likelihood_adjoint(data, log_parameters, checkpoint_stride) (include/hzl/inference.hpp:
 * 59-60, src/adjoint.cpp:43-161) for `count` parameter vectors at once (log_parameters: count x
 * {log nu, log alpha}): the deterministic "multimode" run with checkpoints every
 * checkpoint_stride steps, the Gaussian objective of the observations and its gradient by the
 * discrete adjoint of RK4, FP64 on the device.  A vector outside [-12, 0]^2 or past the
 * explicit diffusion bound gets value +inf as in the reference; the others advance together.
 * HZLB_EINVAL for stochastic data or a zero stride (the reference's std::invalid_argument). */
HZLB_API int hzlb_likelihood_adjoint(const hzlb_dataset *data, const double *log_parameters,
                                     uint64_t count, uint64_t checkpoint_stride, int device,
                                     hzlb_adjoint_evaluation *out);
/* A set of hzl::Solver instances advanced together on the device, with HZL_CHECKPOINT_V1
 * files for each (include/hzl/solver.hpp:61-99, src/solver.cpp:120-138, 204-254, 434-491; RK4, the
 * reference's default integrator).
 * create: solver i is Solver(n, p, seeds[i]) after initialize(initial), initial one of
 * "taylor-green", "multimode", "zero" (hzl::ensemble's members use seeds[i] =
 * stream_seed(seed, i); the simulate command one solver with the seed itself).
 * load: Solver::load of each file, with its checks and messages (HZLB_ERUNTIME for a malformed
 * or inconsistent file); the files of one set must share grid, parameters and time.
 * step: Solver::step(dt) `steps` times for every solver; the diffusion bound is checked first
 * and the advective (CFL) bound after the steps (the reference checks it before each step).
 * diagnostics: count x {time, energy, enstrophy, dissipation, injection, cfl_rate}.
 * coefficients: count x n*n complex omega and/or latent forcing (either may be NULL).
 * save: Solver::save of one solver; the random stream and forcing lines are the reference's
 * exactly, omega equals the reference's to FP64 roundoff. */
typedef struct hzlb_solvers hzlb_solvers;
HZLB_API int hzlb_solvers_create(int n, const hzlb_parameters *params, const uint64_t *seeds,
                                 uint64_t count, const char *initial, int precision, int device,
                                 hzlb_solvers **out);
HZLB_API int hzlb_solvers_load(const char *const *paths, uint64_t count, int precision,
                               int device, hzlb_solvers **out);
HZLB_API void hzlb_solvers_destroy(hzlb_solvers *h);
HZLB_API int hzlb_solvers_step(hzlb_solvers *h, double dt, uint64_t steps);
HZLB_API int hzlb_solvers_diagnostics(hzlb_solvers *h, double *out);
HZLB_API int hzlb_solvers_coefficients(hzlb_solvers *h, double *omega, double *forcing);
HZLB_API int hzlb_solvers_save(hzlb_solvers *h, uint64_t member, const char *path);
/* Grid size and number of solvers of a set (no counterpart in the reference). */
HZLB_API int hzlb_solvers_shape(hzlb_solvers *h, int *n, uint64_t *count);
/* hzl::synthetic_observations(n, dt, steps, every, truth, noise, seed, truth_fields)
 * (include/hzl/inference.hpp:47-49, src/inference.cpp:258-288): the truth run on the device.
 * *count receives 8 x (steps / every); with observations NULL only *count and the header are
 * filled and nothing runs, else capacity must hold *count entries.  truth_fields (optional):
 * (steps / every) x n x n doubles, the physical vorticity at each observation time (the real
 * part of the reference's truth fields).  Observation values equal the reference's to
 * roundoff in FP64 (precision 8); the noise draws are the reference's exactly. */
HZLB_API int hzlb_synthetic_observations(int n, const hzlb_parameters *truth, double dt,
                                         uint64_t steps, uint64_t every, double noise,
                                         uint64_t seed, int precision, int device,
                                         hzlb_dataset *header, hzlb_observation *observations,
                                         size_t capacity, size_t *count, double *truth_fields);
/* hzl::bootstrap_filter(data, p, particles, seed, retain_states) (include/hzl/filter.hpp:17-18,
 * src/filter.cpp:38-126).  mean_vorticity (optional): capacity x n*n complex, the weighted
 * mean physical vorticity per record. */
HZLB_API int hzlb_bootstrap_filter(const hzlb_dataset *data, const hzlb_parameters *params,
                                   uint64_t particles, uint64_t seed, int retain_states,
                                   int precision, int device, double *log_likelihood,
                                   uint64_t *resampling_events, hzlb_filter_record *records,
                                   size_t capacity, size_t *nrecords, double *mean_vorticity);
/* hzl::particle_log_likelihood(data, q, particles, seed) (averaged = 0) and
 * hzl::averaged_particle_log_likelihood(data, q, particles, replicates, seed) (averaged = 1)
 * (include/hzl/filter.hpp:19-24, src/filter.cpp:141-165).  log_parameters = {log nu, log alpha,
 * log sigma, log tau}; *out = -inf outside the prior's support or past the explicit diffusion
 * bound, else the (log-mean-exp over replicates of the) bootstrap filter log-likelihood.  All
 * replicates x particles members advance as one ensemble; replicate r reproduces
 * bootstrap_filter(data, decode(q), particles, stream_seed(seed, r)) (seed itself when
 * averaged = 0).  replicates is ignored when averaged = 0. */
HZLB_API int hzlb_particle_log_likelihood(const hzlb_dataset *data, const double *log_parameters,
                                          uint64_t particles, uint64_t replicates, uint64_t seed,
                                          int averaged, int precision, int device, double *out);
/* hzl::ensemble_kalman_filter(data, p, members, seed, options) (include/hzl/filter.hpp:52-54,
 * src/filter.cpp:204-356): serial perturbed-observation updates of the joint (vorticity,
 * forcing) state.  mean_vorticity (optional): capacity x n*n complex per record. */
HZLB_API int hzlb_ensemble_kalman_filter(const hzlb_dataset *data, const hzlb_parameters *params,
                                         uint64_t members, uint64_t seed,
                                         const hzlb_enkf_options *options, int precision,
                                         int device, hzlb_enkf_record *records, size_t capacity,
                                         size_t *nrecords, double *mean_vorticity);

/* ---- tensor-core contractions ------------------------------------------------------ */
/* C[M x N] = alpha * opA * opB^T + beta * C on the tcgen05 tensor cores with FP32 accumulation
 * (device pointers, asynchronous on `stream`).  dtype 2: A and B are BF16; dtype 4: A and B are
 * FP32 read as TF32.  opA is M x K: A[m*lda + k] when a_kcontig, else A[k*lda + m]; opB is
 * N x K likewise.  Used by the learned forecast and the ensemble-space analysis products; no
 * counterpart in the reference (whose filter updates are per-scalar loops). */
HZLB_API int hzlb_gemm(int M, int N, int K, int dtype, const void *A, long long lda, int a_kcontig,
                       const void *B, long long ldb, int b_kcontig, float *C, long long ldc,
                       float alpha, float beta, void *stream);

/* ---- stepping without device allocation ------------------------------------------- */
/* No counterpart in the reference.  For callers that may not allocate GPU memory while they
 * run (device memory owned and budgeted by the application's own pool, or a hot loop where an
 * allocation and its possible failure are not acceptable): the same RK4 step as hzlb_step,
 * with every scratch buffer taken from one device array of HZLB_NOALLOC_SCRATCH_BYTES built
 * into the library (held on every GPU that loads the library's device code until exit).
 * state: device pointer, members x hzlb_compact_size() complex entries in the compact layout
 * of the configured precision, advanced in place by nsteps steps of dt; forcing: device
 * pointer in the compact forcing layout (columns kx <= forcing_kmax, one field or one per
 * member) or NULL; first_step: noise counter of the first step; stream: a cudaStream_t or
 * NULL; status: if non-NULL, the call waits for the stream and stores the HZLB_STATUS_* bits;
 * with status NULL the call does not wait and the step's CFL, nonfinite and timeout bits are
 * lost (the next call clears them), so a caller that captures the call into a graph has no
 * error report from it.  Sizes whose scratch exceeds the limit are HZLB_EINVAL (for example
 * at most 31 members at 256^2 FP32, 15 in FP64).  The first call on a device, and the first
 * for each (precision, n) on it, resolves the array's device address, configures the kernels
 * and writes that grid's twiddle table into the array; make those calls before any stream
 * capture.  Calls share the array, so calls that overlap on the GPU race: serialise them. */
#define HZLB_NOALLOC_SCRATCH_BYTES (32u << 20)
HZLB_API int hzlb_step_noalloc(const hzlb_config *config, double dt, uint64_t nsteps,
                               uint64_t first_step, void *state, const void *forcing, void *stream,
                               uint32_t *status);

/* ---- learned reduced forecast (no counterpart in the reference, which has no learned model;
 * its reduced forecast is the Galerkin ROM of reduced.cpp:137-209) ----------------------
 * A multilayer perceptron advancing r POD coefficients over one forecast window:
 *   y = a + s_out * (W3 gelu(W2 gelu(W1 (x / s_in) + b1) + b2) + b3),   x = (a, xi)
 * x: r coefficients a followed by q noise-mode amplitudes xi; hidden width H (multiple of 16);
 * gelu is the tanh form.  Weights and activations are BF16 with FP32 accumulation on the
 * tcgen05 tensor cores; FP32 master parameters with Adam (beta1 0.9, beta2 0.999, eps 1e-8).
 * Parameter vector (FP32): W1 [H][r+q], W2 [H][H], W3 [r][H], b1 [H], b2 [H], b3 [r];
 * creation initialises W1, W2 ~ N(0, 1.96/fan_in), W3 ~ N(0, 0.01/fan_in), biases 0, scales 1
 * from `seed`.  Batches are row-major [batch][features] device arrays of FP32. */
typedef struct hzlb_mlp hzlb_mlp;
HZLB_API int hzlb_mlp_create(int r, int q, int hidden, int max_batch, int device, uint64_t seed,
                             hzlb_mlp **out);
HZLB_API void hzlb_mlp_destroy(hzlb_mlp *h);
HZLB_API size_t hzlb_mlp_param_count(const hzlb_mlp *h);
/* r, q, hidden width and maximum batch of the network */
HZLB_API int hzlb_mlp_shape(const hzlb_mlp *h, int *r, int *q, int *hidden, int *max_batch);
/* host arrays of hzlb_mlp_param_count floats; grads (may be NULL) receives the gradient of the
 * last training step */
HZLB_API int hzlb_mlp_set_params(hzlb_mlp *h, const float *params);
HZLB_API int hzlb_mlp_get_params(hzlb_mlp *h, float *params, float *grads);
/* host arrays: s_in [r+q], s_out [r] */
HZLB_API int hzlb_mlp_set_scales(hzlb_mlp *h, const float *s_in, const float *s_out);
/* y [batch][r] = forward(x [batch][r+q]); device pointers.  stream NULL: the handle's stream,
 * waited for; otherwise enqueued on `stream` without waiting. */
HZLB_API int hzlb_mlp_forward(hzlb_mlp *h, const float *x, int batch, float *y, void *stream);
/* One Adam step on the mean squared error of forward(x) against target [batch][r] (device
 * pointers); *loss = that error before the update.  lr = 0 computes the gradient only. */
HZLB_API int hzlb_mlp_train_step(hzlb_mlp *h, const float *x, const float *target, int batch,
                                 float lr, double *loss);

/* ---- proper orthogonal decomposition (reduced.cpp:36-136) ---------------------------- */
/* PODBasis fit_pod(snapshots, maximum_rank, variance_fraction) (reduced.hpp:16-17) on the
 * GPU: m (2..512) snapshots of `dimension` complex entries (interleaved doubles), mean,
 * Gram matrix of the centred snapshots (Re sum conj(a) b) in FP64 on the device, the
 * reference's cyclic Jacobi eigensolver and truncation rules, modes X^T v / sqrt(lambda)
 * orthonormalised as by its two Gram-Schmidt passes.  Outputs: *rank modes (modes: max_rank
 * x dimension complex), mean (dimension complex), singular_values (max_rank), *captured.
 * Errors as the reference: HZLB_EINVAL for its invalid_argument cases, HZLB_ERUNTIME for
 * non-convergence, degenerate modes or no resolved mode. */
HZLB_API int hzlb_fit_pod(size_t m, size_t dimension, const double *snapshots, size_t max_rank,
                          double fraction, int device, size_t *rank, double *mean, double *modes,
                          double *singular_values, double *captured);

/* GalerkinModel(PODBasis, Solver&) (reduced.hpp:19-30, reduced.cpp:137-209): the quadratic
 * reduced model da/dt = c + A a + Q(a,a) of the deterministic drift in the coefficients of a
 * POD basis (mean and `rank` modes in the reference layout, e.g. from hzlb_fit_pod).  The
 * drifts it needs are evaluated by the batched FP64 spectral kernels in one launch sequence.
 * HZLB_EINVAL for forcing_sigma != 0, as the reference. */
typedef struct hzlb_galerkin hzlb_galerkin;
HZLB_API int hzlb_galerkin_create(int n, const hzlb_parameters *p, const double *mean,
                                  const double *modes, size_t rank, int device,
                                  hzlb_galerkin **out);
HZLB_API void hzlb_galerkin_destroy(hzlb_galerkin *h);
/* c (rank), A (rank x rank, [i][j]), Q (rank^3, [i][j][k]); any may be NULL */
HZLB_API int hzlb_galerkin_coefficients(hzlb_galerkin *h, double *constant, double *linear,
                                        double *quadratic);
/* GalerkinModel::rhs for `count` coefficient vectors (host arrays, count x rank) */
HZLB_API int hzlb_galerkin_rhs(hzlb_galerkin *h, const double *coefficients, size_t count,
                               double *out);
/* GalerkinModel::step: nsteps RK4 steps of dt for `count` coefficient vectors in place;
 * HZLB_ERUNTIME "unstable Galerkin trajectory" on a nonfinite result */
HZLB_API int hzlb_galerkin_step(hzlb_galerkin *h, double *coefficients, size_t count, double dt,
                                uint64_t nsteps);

/* No counterpart in the reference (its fit is capped at 512 snapshots).  POD of `snapshots`
 * FP32 fields of an n x n ensemble in the compact layout (device pointer, snapshots x
 * hzlb_compact_size complex floats), with the reference's inner product (spectral_inner over
 * the full spectrum of the real fields).  Gram matrix by 3xTF32 tensor-core products; the
 * leading `rank` eigenpairs by subspace iteration on rank + oversample vectors (`iterations`
 * sweeps, random start from `seed`) and a Rayleigh-Ritz step, or by Jacobi on the whole Gram
 * matrix when snapshots <= 256.  The handle keeps the mean and modes for hzlb_pod_project and
 * hzlb_learned_forecast. */
typedef struct hzlb_pod hzlb_pod;
HZLB_API int hzlb_pod_fit(int n, int snapshots, const void *data, int rank, int oversample,
                          int iterations, uint64_t seed, int device, hzlb_pod **out);
HZLB_API void hzlb_pod_destroy(hzlb_pod *h);
/* rank, eigenvalues (rank doubles), captured variance fraction, and the largest relative
 * eigen-residual |G v - lambda v| / lambda of the returned pairs */
HZLB_API int hzlb_pod_info(hzlb_pod *h, int *rank, double *eigenvalues, double *captured,
                           double *residual);
/* host copies: modes (rank x compact complex floats, orthonormal under spectral_inner) and
 * the mean (compact complex floats); either may be NULL */
HZLB_API int hzlb_pod_modes(hzlb_pod *h, float *modes, float *mean);
/* coefficients[i][j] (row stride ldc) = spectral_inner(mode j, state i - mean), the
 * reference's PODBasis::project (reduced.cpp:16-26), for `count` compact FP32 states (device
 * pointers).  stream NULL: the handle's stream, waited for. */
HZLB_API int hzlb_pod_project(hzlb_pod *h, const void *states, int count, float *coefficients,
                              long long ldc, void *stream);
/* Noise-mode amplitudes of a forecast window for `count` members of an ensemble configured by
 * `config`: for (kx, ky) = (1,0), (0,1), (1,1), (1,-1), the sum over steps [first_step,
 * first_step + steps) of the noise increments hzlb_step adds to that mode, re and im:
 * out[m][0..7] (device, row stride ldo).  stream NULL: waited for. */
HZLB_API int hzlb_noise_amplitudes(const hzlb_config *config, double dt, uint64_t first_step,
                                   uint64_t steps, int count, float *out, long long ldo,
                                   void *stream);
/* Adds to `count` compact FP32 states (device) the noise of a window: on every mode of the
 * noise shell, the sum of the increments hzlb_step adds over steps [first_step, first_step +
 * steps) (same Philox draws).  stream NULL: waited for. */
HZLB_API int hzlb_add_window_noise(const hzlb_config *config, double dt, uint64_t first_step,
                                   uint64_t steps, int count, void *state, void *stream);
/* One window of the learned reduced forecast on an FP32 ensemble, in place of `steps`
 * steps of hzlb_step: a = project(state), x = (a, noise amplitudes of the window),
 * state += modes (mlp(x) - a), then the window's noise increments (hzlb_add_window_noise).
 * The network predicts the coefficients at the end of the window less the projection of the
 * window's noise; outside the POD space the state changes by the noise alone.  Advances the
 * ensemble's time and step counter by `steps`.  The network must have r = the POD rank, q = 8
 * and max_batch >= members.  mean_increment: NULL, or a device array (compact FP32 field)
 * added to every member after the network's change: with centre != 0 the change of the
 * ensemble mean over the window from another forecast of the mean (the spectral step of a
 * one-member ensemble holding hzlb_ensemble_mean_device), the network then moving the members
 * only about their mean (its coefficient changes are centred over the ensemble); with
 * centre == 0 an increment the network cannot carry (e.g. the motion outside the POD space),
 * the network's changes kept whole. */
HZLB_API int hzlb_learned_forecast(hzlb_ensemble *h, hzlb_pod *pod, hzlb_mlp *mlp, double dt,
                                   uint64_t steps, const void *mean_increment, int centre);

/* ---- mixed-resolution batches (no counterpart in the reference) -----------------------
 * Ensembles of different grid sizes (and precisions) on one device advanced together: one CUDA
 * graph per batch of steps holds every resolution's launches, either as concurrent branches
 * (each resolution's persistent kernels capped to a share of the GPU) or one after another.
 * hzlb_mixed_group returns the handle of resolution `group` (owned by the batch: set states,
 * forcing, read diagnostics through it; do not destroy it).  dt: one time step per group. */
typedef struct hzlb_mixed hzlb_mixed;
HZLB_API int hzlb_mixed_create(const hzlb_config *configs, int count, hzlb_mixed **out);
HZLB_API void hzlb_mixed_destroy(hzlb_mixed *h);
HZLB_API hzlb_ensemble *hzlb_mixed_group(hzlb_mixed *h, int group);
HZLB_API int hzlb_mixed_step(hzlb_mixed *h, const double *dt, uint64_t nsteps);
/* Autotuner: times the serial schedule and the concurrent one with each group's grid cap
 * chosen by coordinate descent over fractions of its resident blocks (`repeats` graph
 * launches of 8 steps per candidate) and keeps the fastest; *ms_per_step = its step time.
 * The ensembles' states, clocks and status are restored afterwards. */
HZLB_API int hzlb_mixed_tune(hzlb_mixed *h, const double *dt, int repeats, double *ms_per_step);
/* The schedule in effect: serial flag and per-group grid caps (blocks) of the column and row
 * kernels; set_schedule overrides it (caps 0 or NULL: every resident block). */
HZLB_API int hzlb_mixed_schedule(hzlb_mixed *h, int *serial, int *col_caps, int *row_caps);
HZLB_API int hzlb_mixed_set_schedule(hzlb_mixed *h, int serial, const int *col_caps,
                                     const int *row_caps);
/* Schedule modes: 0 serial, 1 concurrent (each resolution's kernels on its own graph branch,
 * grids capped by col_caps / row_caps, 0 = every resident block), 2 fused (one persistent row
 * kernel and one column kernel per RK stage over the whole mixed work list: FP32, resolutions
 * among 64, 128, 256 and 512 with one ensemble each, no device OU forcing), 3 fused with the
 * 512^2 ensemble's own kernels on a concurrent branch (its caps apply).  hzlb_mixed_tune
 * measures every mode that applies and keeps the fastest; hzlb_mixed_mode reports the mode in
 * effect and the tuner's best ms per step of modes 0..3 (tuned_ms: 4 doubles, 0 where not
 * measured; may be NULL). */
HZLB_API int hzlb_mixed_set_mode(hzlb_mixed *h, int mode, const int *col_caps, const int *row_caps);
HZLB_API int hzlb_mixed_mode(hzlb_mixed *h, int *mode, double *tuned_ms);
/* Row-kernel block shape per group in the serial and concurrent modes (and the 512^2 branch of
 * mode 3): 64 or 128 threads, both compiled for every resolution (a block of 64 holds half the
 * rows of one of 128).  hzlb_mixed_row_threads reports the shapes in effect (one int per group);
 * set_row_threads sets them (0: the resolution's default); hzlb_mixed_tune chooses them after
 * the grid caps; set_mode and set_schedule return them to the defaults.  The shape changes no
 * result bit. */
HZLB_API int hzlb_mixed_row_threads(hzlb_mixed *h, int *threads);
HZLB_API int hzlb_mixed_set_row_threads(hzlb_mixed *h, const int *threads);

/* ---- seeded synthetic inputs (no counterpart in the reference, which has only built-in
 * analytic initial fields, solver.cpp:145-161) -------------------------------------- */
/* Gaussian random vorticity spectrum, E(k) ~ k^4 exp(-(k/6)^2), unit enstrophy, retained modes
 * only; Philox4x32-10 normals keyed by (seed, member).  out: n*n complex, reference layout. */
HZLB_API int hzlb_grf_spectrum(int n, uint64_t seed, uint32_t member, double *out);
/* amplitude * sin(wavenumber * y) as spectral coefficients, reference layout. */
HZLB_API int hzlb_kolmogorov_forcing(int n, double amplitude, int wavenumber, double *out);

#ifdef __cplusplus
}
#endif
#endif
