/* TEST INFRASTRUCTURE ONLY -- CPU oracle for the ensemble forecast/analysis path.
 *
 * A plain-C restatement of the reference algorithm (pvasbob/HZL-stochasticFlowInference):
 * the radix-2 Fourier transform, the pseudo-spectral RK4 vorticity step with OU shell
 * forcing, diagnostics, the particle-filter weight/resample step, the serial EnKF update,
 * and the snapshot POD, plus the seeded-synthetic extensions used by the benchmark
 * workloads (Philox4x32-10 noise, Gaussian-random-field initial vorticity, Kolmogorov
 * forcing).  Each function cites the reference file:line it restates.  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU baseline call it; the product never does.
 *
 * Parity status: pinned.  The restatement is checked against the reference's own CPU
 * library (oracle/_ref/libhzlref.so, built from the reference sources by oracle/Makefile)
 * and against the golden vectors in tests/golden/ generated from that library.
 *
 * Layout: complex fields are interleaved (re, im) doubles, n*n entries, index y*n + x
 * (include/hzl/fft.hpp:7-8 of the reference).  Return codes: 0 ok, -1 invalid argument,
 * -2 runtime failure (CFL/nonfinite); ho_last_error() holds the message. */
#ifndef HZL_ORACLE_H
#define HZL_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

const char *ho_last_error(void);

/* ---- random numbers -------------------------------------------------------------- */
uint64_t ho_stream_seed(uint64_t base, uint64_t index);
typedef struct {
    uint64_t mt[312];
    int mti;
    int has_spare;
    double spare;
} ho_normal_stream;
void ho_normal_init(ho_normal_stream *s, uint64_t seed);
uint64_t ho_mt_next(ho_normal_stream *s);
double ho_normal_next(ho_normal_stream *s);
void ho_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* Two standard normals for (seed, member, step, mode code); see ho_philox_normals in .c */
void ho_philox_normal_pair(uint64_t seed, uint32_t member, uint64_t step, uint32_t mode_code,
                           double *xi1, double *xi2);
uint32_t ho_mode_code(int kx, int ky);

/* ---- transform ------------------------------------------------------------------- */
int ho_fft(int n, double *data, int inverse);

/* ---- solver ---------------------------------------------------------------------- */
typedef struct ho_solver ho_solver;
/* p6 = {nu, alpha, sigma, tau, kmin, kmax} as in hzl::Parameters (solver.hpp:15-23). */
int ho_solver_create(int n, const double *p6, uint64_t seed, ho_solver **out);
void ho_solver_destroy(ho_solver *s);
int ho_solver_initialize(ho_solver *s, const char *name);
int ho_solver_initialize_physical(ho_solver *s, const double *field);
int ho_solver_set_state(ho_solver *s, const double *omega, const double *forcing);
int ho_solver_get_state(const ho_solver *s, double *omega, double *forcing);
int ho_solver_midpoint_forcing(const ho_solver *s, double *out);
/* Reference step (solver.cpp:217-254): validate, OU(dt/2), RK4 with frozen forcing,
 * finite check, project, OU(dt/2). */
int ho_solver_step(ho_solver *s, double dt);
/* RK4 step with caller-supplied forcing held over the step (cuda_solver.cu:184-218 semantics;
 * forcing may be NULL for zero); no OU transition, no validate. */
int ho_solver_step_forced(ho_solver *s, double dt, const double *forcing);
int ho_solver_diagnostics(ho_solver *s, double *out6);
int ho_solver_physical_vorticity(ho_solver *s, double *out);
int ho_solver_update_latent_state(ho_solver *s, const double *omega, const double *forcing);
double ho_solver_time(const ho_solver *s);
void ho_solver_reseed_future(ho_solver *s, uint64_t seed);

/* ---- seeded synthetic workload (Kolmogorov + EM noise + GRF) ------------------------ */
/* Gaussian random field, E(k) ~ k^4 exp(-(k/6)^2), unit enstrophy, active modes only;
 * writes the spectral coefficients (n*n complex). */
int ho_grf_spectrum(int n, uint64_t seed, uint32_t member, double *omega_hat);
/* Kolmogorov forcing amplitude*sin(4y) as spectral coefficients (n*n complex). */
int ho_kolmogorov_forcing(int n, double amplitude, int wavenumber, double *forcing_hat);
/* Adds the Euler-Maruyama increment sigma*sqrt(dt)*(xi1 + i xi2)/sqrt(2) on 1<=|k|<=kmax
 * (active modes; conjugate partner mirrored) for (seed, member, step). */
int ho_add_noise(int n, double *omega_hat, double sigma, double dt, int kmax, uint64_t seed,
                 uint32_t member, uint64_t step);
/* One seeded-synthetic step: RK4 with the given frozen forcing, project, then noise. */
int ho_synthetic_step(ho_solver *s, double dt, const double *forcing, double sigma,
                      int noise_kmax, uint64_t seed, uint32_t member, uint64_t step);

/* ---- particle filter ------------------------------------------------------------- */
/* filter.cpp:66-92: log-weights -> increment, normalised weights, ESS, max weight. */
int ho_pf_weights(int count, const double *log_weights, double *weights, double *increment,
                  double *ess, double *max_weight);
/* filter.cpp:102-116: systematic resampling from normalised weights and a uniform u. */
int ho_systematic_resample(int count, const double *weights, double u, uint32_t *ancestors);
double ho_resampling_uniform(uint64_t raw);

/* ---- EnKF ------------------------------------------------------------------------ */
/* One serial scalar-observation update (filter.cpp:265-321) without localisation, applied to
 * the members' (omega, forcing) latent states given their predicted observations and the
 * perturbation draws, ending in update_latent_state for every member. */
int ho_enkf_scalar_update(int members, ho_solver **s, const double *predictions, double value,
                          double sd, const double *perturbations);

/* ---- POD ------------------------------------------------------------------------- */
int ho_fit_pod(int m, int64_t dimension, const double *snapshots, int max_rank, double fraction,
               int *rank, double *mean, double *modes, double *singular_values, double *captured);

#ifdef __cplusplus
}
#endif
#endif
