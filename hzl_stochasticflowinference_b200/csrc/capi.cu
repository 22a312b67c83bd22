// extern "C" boundary (include/hzlb.h): exception -> status code mapping around the engine.
#include "engine.h"
#include "dense64.cuh"

#include <cmath>
#include <exception>
#include <string>
#include <vector>


namespace {
thread_local std::string last_error;

template <class F> int guarded(F &&f) {
    try {
        f();
        return HZLB_OK;
    } catch (const hzlb::Error &e) {
        last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        last_error = "host allocation failed";
        return HZLB_ERUNTIME;
    } catch (const std::exception &e) {
        last_error = e.what();
        return HZLB_ERUNTIME;
    } catch (...) {
        last_error = "unknown failure";
        return HZLB_ERUNTIME;
    }
}
hzlb::Engine &engine(hzlb_ensemble *h) {
    if (!h || !h->engine)
        hzlb::raise(HZLB_EINVAL, "null ensemble handle");
    ++h->engine->api_calls;
    return *h->engine;
}
void need(const void *p, const char *what) {
    if (!p)
        hzlb::raise(HZLB_EINVAL, std::string("null pointer: ") + what);
}
} // namespace

void hzlb::set_last_error(const std::string &message) { last_error = message; }

extern "C" {

const char *hzlb_last_error(void) { return last_error.c_str(); }
const char *hzlb_version(void) { return "hzlb 0.1 (sm_100a)"; }

int hzlb_ensemble_create(const hzlb_config *config, hzlb_ensemble **out) {
    return guarded([&] {
        need(config, "config");
        need(out, "out");
        *out = nullptr;
        auto h = std::make_unique<hzlb_ensemble>();
        h->engine = hzlb::make_engine(*config);
        *out = h.release();
    });
}
void hzlb_ensemble_destroy(hzlb_ensemble *h) { delete h; }

int hzlb_set_state(hzlb_ensemble *h, const double *spectra, int first, int count) {
    return guarded([&] {
        need(spectra, "spectra");
        engine(h).set_state(spectra, first, count);
    });
}
int hzlb_get_state(hzlb_ensemble *h, double *spectra, int first, int count) {
    return guarded([&] {
        need(spectra, "spectra");
        engine(h).get_state(spectra, first, count);
    });
}
int hzlb_set_state_compact(hzlb_ensemble *h, const void *compact, int first, int count) {
    return guarded([&] {
        need(compact, "compact");
        engine(h).set_state_compact(compact, first, count);
    });
}
int hzlb_get_state_compact(hzlb_ensemble *h, void *compact, int first, int count) {
    return guarded([&] {
        need(compact, "compact");
        engine(h).get_state_compact(compact, first, count);
    });
}
size_t hzlb_compact_size(const hzlb_ensemble *h) {
    return h && h->engine ? h->engine->compact_size() : 0;
}
int hzlb_set_forcing(hzlb_ensemble *h, const double *spectra, int first, int count) {
    return guarded([&] {
        need(spectra, "spectra");
        engine(h).set_forcing(spectra, first, count);
    });
}
int hzlb_step(hzlb_ensemble *h, double dt, uint64_t nsteps) {
    return guarded([&] { engine(h).step(dt, nsteps); });
}
int hzlb_test_inject_wait_timeout(hzlb_ensemble *h) {
    return guarded([&] { engine(h).inject_wait_timeout(); });
}
int hzlb_step_checked(hzlb_ensemble *h, double dt) {
    return guarded([&] { engine(h).step_checked(dt); });
}
int hzlb_set_step_schedule(hzlb_ensemble *h, int schedule) {
    return guarded([&] { engine(h).set_step_schedule(schedule); });
}
int hzlb_step_schedule(hzlb_ensemble *h, int *schedule) {
    return guarded([&] {
        need(schedule, "schedule");
        *schedule = engine(h).step_schedule();
    });
}
int hzlb_step_host(hzlb_ensemble *h, const void *state_in, void *state_out, double dt,
                   uint64_t nsteps, int chunk_members) {
    return guarded([&] { engine(h).step_host(state_in, state_out, dt, nsteps, chunk_members); });
}
void *hzlb_stream(hzlb_ensemble *h) {
    if (!h || !h->engine)
        return nullptr;
    ++h->engine->api_calls;   // the caller may order its own work on the stream
    return h->engine->stream();
}
int hzlb_step_profiled(hzlb_ensemble *h, double dt, uint64_t nsteps, double *row_ms,
                       double *column_ms) {
    return guarded([&] {
        need(row_ms, "row_ms");
        need(column_ms, "column_ms");
        engine(h).step_profiled(dt, nsteps, row_ms, column_ms);
    });
}
int hzlb_status(hzlb_ensemble *h, uint32_t *status) {
    return guarded([&] {
        need(status, "status");
        *status = engine(h).status();
    });
}
int hzlb_synchronize(hzlb_ensemble *h) {
    return guarded([&] { engine(h).synchronize(); });
}
int hzlb_time(hzlb_ensemble *h, double *time, uint64_t *step_index) {
    return guarded([&] {
        auto &e = engine(h);
        if (time)
            *time = e.time;
        if (step_index)
            *step_index = e.step_index;
    });
}
int hzlb_set_time(hzlb_ensemble *h, double time, uint64_t step_index) {
    return guarded([&] {
        if (!std::isfinite(time) || time < 0)
            hzlb::raise(HZLB_EINVAL, "invalid time");
        engine(h).set_time(time, step_index);
    });
}
int hzlb_diagnostics(hzlb_ensemble *h, double *out) {
    return guarded([&] {
        need(out, "out");
        engine(h).diagnostics(out);
    });
}
int hzlb_physical(hzlb_ensemble *h, double *out) {
    return guarded([&] {
        need(out, "out");
        engine(h).physical(out);
    });
}
int hzlb_observe(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y, size_t p, double *out) {
    return guarded([&] {
        if (p) {
            need(x, "x");
            need(y, "y");
            need(out, "out");
        }
        engine(h).observe(x, y, p, out);
    });
}

int hzlb_pf_loglik(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y, const double *values,
                   const double *sd, size_t p, double *log_weights) {
    return guarded([&] {
        need(log_weights, "log_weights");
        if (p == 0)
            return;
        need(x, "x");
        need(y, "y");
        need(values, "values");
        need(sd, "sd");
        engine(h).pf_loglik(x, y, values, sd, p, log_weights);
    });
}
int hzlb_pf_weights(hzlb_ensemble *h, const double *log_weights, size_t count, double *weights,
                    double *increment, double *ess, double *max_weight) {
    return guarded([&] {
        need(log_weights, "log_weights");
        need(weights, "weights");
        need(increment, "increment");
        need(ess, "ess");
        need(max_weight, "max_weight");
        engine(h).pf_weights(log_weights, count, weights, increment, ess, max_weight);
    });
}
int hzlb_systematic_resample(hzlb_ensemble *h, const double *weights, size_t count, double u,
                             uint32_t *ancestors) {
    return guarded([&] {
        need(weights, "weights");
        need(ancestors, "ancestors");
        if (count == 0)
            hzlb::raise(HZLB_EINVAL, "resampling needs at least one weight");
        if (!std::isfinite(u) || u < 0 || u >= 1)
            hzlb::raise(HZLB_EINVAL, "resampling uniform must lie in [0, 1)");
        engine(h).resample(weights, count, u, ancestors);
    });
}
int hzlb_pf_reset(hzlb_ensemble *h, int particles) {
    return guarded([&] { engine(h).pf_reset(particles); });
}
int hzlb_pf_assimilate(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y, const double *values,
                       const double *sd, size_t p, const double *u, const uint8_t *active,
                       hzlb_pf_record *records, uint32_t *ancestors, double *weighted_mean) {
    return guarded([&] {
        need(records, "records");
        if (p) {
            need(x, "x");
            need(y, "y");
            need(values, "values");
            need(sd, "sd");
        }
        engine(h).pf_assimilate(x, y, values, sd, p, u, active, records, ancestors, weighted_mean);
    });
}
int hzlb_pf_get_weights(hzlb_ensemble *h, double *weights) {
    return guarded([&] {
        need(weights, "weights");
        engine(h).pf_get_weights(weights);
    });
}
int hzlb_gather_members(hzlb_ensemble *h, const uint32_t *ancestors) {
    return guarded([&] {
        need(ancestors, "ancestors");
        engine(h).gather(ancestors);
    });
}
int hzlb_inflate(hzlb_ensemble *h, double inflation) {
    return guarded([&] { engine(h).inflate(inflation); });
}
int hzlb_enkf_analysis(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y,
                       const double *values, const double *sd, size_t p,
                       const double *perturbations) {
    return guarded([&] {
        if (p) {
            need(x, "x");
            need(y, "y");
            need(values, "values");
            need(sd, "sd");
            need(perturbations, "perturbations");
        }
        engine(h).enkf(hzlb::EnkfRequest{x, y, values, sd, p, perturbations, 0, 0, 0.0});
    });
}
int hzlb_enkf_analysis_nis(hzlb_ensemble *h, const uint32_t *x, const uint32_t *y,
                           const double *values, const double *sd, size_t p,
                           const double *perturbations, uint64_t perturbation_seed,
                           uint64_t cycle, double nis_limit, double *nis, int *applied) {
    return guarded([&] {
        if (p) {
            need(x, "x");
            need(y, "y");
            need(values, "values");
            need(sd, "sd");
        }
        if (!std::isfinite(nis_limit))
            hzlb::raise(HZLB_EINVAL, "innovation statistic limit must be finite");
        const hzlb::EnkfResult r = engine(h).enkf(hzlb::EnkfRequest{
            x, y, values, sd, p, perturbations, perturbation_seed, cycle, nis_limit});
        if (nis)
            *nis = r.nis;
        if (applied)
            *applied = r.applied;
    });
}
int hzlb_enkf_weights(hzlb_ensemble *h, const double *hx, const double *values, const double *sd,
                      const double *eps, int members, size_t p, double *W, double *nis) {
    return guarded([&] {
        need(hx, "hx");
        need(values, "values");
        need(sd, "sd");
        need(eps, "eps");
        need(W, "W");
        if (members < 2 || members > (1 << 16))
            hzlb::raise(HZLB_EINVAL, "EnKF weights need between 2 and 65536 members");
        const double v = engine(h).enkf_weights(hx, values, sd, eps, members, p, W);
        if (nis)
            *nis = v;
    });
}
int hzlb_dgemm(int M, int N, int K, double alpha, const double *A, long long sam, long long sak,
               const double *B, long long sbk, long long sbn, double beta, double *C, long long ldc,
               void *stream) {
    return guarded([&] {
        if (M < 0 || N < 0 || K < 0)
            hzlb::raise(HZLB_EINVAL, "GEMM sizes must be nonnegative");
        if (M > 0 && N > 0) {
            need(C, "C");
            if (K > 0) {
                need(A, "A");
                need(B, "B");
            }
            if (ldc < N)
                hzlb::raise(HZLB_EINVAL, "ldc must be at least N");
        }
        hzlb::cuda_check(hzlb::d64::gemm(hzlb::d64::GemmArgs{M, N, K, alpha, beta, A, sam, sak, B,
                                                             sbk, sbn, C, ldc},
                                         static_cast<cudaStream_t>(stream)),
                         "launch FP64 GEMM");
    });
}
int hzlb_learned_forecast(hzlb_ensemble *h, hzlb_pod *pod, hzlb_mlp *mlp, double dt,
                          uint64_t steps, const void *mean_increment, int centre) {
    int rc = HZLB_OK;
    const int outer = guarded([&] {
        auto &e = engine(h);
        rc = hzlb::learned_forecast(e, e.config(), pod, mlp, 8, dt, steps, mean_increment,
                                    centre != 0);
    });
    return outer != HZLB_OK ? outer : rc;
}
int hzlb_weighted_mean(hzlb_ensemble *h, const double *weights, double *mean) {
    return guarded([&] {
        need(weights, "weights");
        need(mean, "mean");
        engine(h).member_sum(weights, 0.0, mean);
    });
}
int hzlb_ensemble_mean_device(hzlb_ensemble *h, void *mean) {
    return guarded([&] {
        need(mean, "mean");
        engine(h).mean_device(mean);
    });
}
int hzlb_ensemble_mean(hzlb_ensemble *h, double *mean) {
    return guarded([&] {
        need(mean, "mean");
        auto &e = engine(h);
        e.member_sum(nullptr, static_cast<double>(e.members()), mean);
    });
}
int hzlb_enable_ou(hzlb_ensemble *h, double sigma, double tau, int kmin, int kmax,
                   int initialize) {
    return guarded([&] { engine(h).enable_ou(sigma, tau, kmin, kmax, initialize != 0); });
}
int hzlb_get_forcing_compact(hzlb_ensemble *h, double *out, int first, int count) {
    return guarded([&] {
        need(out, "out");
        engine(h).get_forcing_compact(out, first, count);
    });
}
int hzlb_state_device(hzlb_ensemble *h, void **state) {
    return guarded([&] {
        need(state, "state");
        *state = engine(h).state_device();
    });
}

} // extern "C"
