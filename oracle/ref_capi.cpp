// TEST INFRASTRUCTURE ONLY: a C wrapper over the reference's own C++ API.
//
// This file is compiled together with the reference sources (src/fft.cpp, src/solver.cpp,
// src/inference.cpp, src/adjoint.cpp, src/filter.cpp, src/reduced.cpp of the reference tree,
// which stay where they lie) into oracle/_ref/libhzlref.so by oracle/Makefile.  The library
// is the checker for the CUDA path and the "reference" CPU baseline; nothing in the product
// links it.  Every function returns 0 on success and a negative code after catching a C++
// exception, whose message is kept for ref_last_error().
//
// Complex fields cross this boundary as interleaved (re, im) doubles, n*n entries in the
// reference layout (index y*n + x, include/hzl/fft.hpp:7-8).
#include "hzl/filter.hpp"
#include "hzl/inference.hpp"
#include "hzl/reduced.hpp"
#include "hzl/solver.hpp"

#include <atomic>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

extern "C" {
#include "hzl_oracle.h"
}

namespace {
thread_local std::string last_error;

template <class F> int guarded(F &&f) {
    try {
        f();
        return 0;
    } catch (const std::invalid_argument &e) {
        last_error = e.what();
        return -1;
    } catch (const std::exception &e) {
        last_error = e.what();
        return -2;
    } catch (...) {
        last_error = "unknown exception";
        return -3;
    }
}

hzl::Field to_field(const double *v, std::size_t count) {
    hzl::Field f(count);
    for (std::size_t i = 0; i < count; ++i)
        f[i] = {v[2 * i], v[2 * i + 1]};
    return f;
}

void from_field(const hzl::Field &f, double *out) {
    for (std::size_t i = 0; i < f.size(); ++i) {
        out[2 * i] = f[i].real();
        out[2 * i + 1] = f[i].imag();
    }
}

hzl::Parameters params(const double *p6) {
    hzl::Parameters p;
    p.viscosity = p6[0];
    p.friction = p6[1];
    p.forcing_sigma = p6[2];
    p.forcing_tau = p6[3];
    p.forcing_min = static_cast<int>(p6[4]);
    p.forcing_max = static_cast<int>(p6[5]);
    return p;
}

hzl::Dataset dataset(std::size_t n, double dt, int stochastic, int fmin, int fmax,
                     std::size_t count, const unsigned long long *steps, const unsigned *xs,
                     const unsigned *ys, const double *values, const double *sds) {
    hzl::Dataset d;
    d.n = n;
    d.dt = dt;
    d.stochastic = stochastic != 0;
    d.forcing_min = fmin;
    d.forcing_max = fmax;
    d.observations.resize(count);
    for (std::size_t i = 0; i < count; ++i)
        d.observations[i] = {static_cast<std::size_t>(steps[i]), xs[i], ys[i], values[i], sds[i]};
    return d;
}
} // namespace

extern "C" {
const char *ref_last_error(void) { return last_error.c_str(); }

unsigned long long ref_stream_seed(unsigned long long base, unsigned long long index) {
    return hzl::stream_seed(base, index);
}

int ref_fft(int n, double *data, int inverse) {
    return guarded([&] {
        hzl::Fourier2D f(static_cast<std::size_t>(n));
        auto field = to_field(data, static_cast<std::size_t>(n) * n);
        if (inverse)
            f.inverse(field);
        else
            f.forward(field);
        from_field(field, data);
    });
}

// ---- hzl::Solver ------------------------------------------------------------------------
int ref_solver_create(int n, const double *p6, unsigned long long seed, void **out) {
    return guarded([&] { *out = new hzl::Solver(static_cast<std::size_t>(n), params(p6), seed); });
}
void ref_solver_destroy(void *h) { delete static_cast<hzl::Solver *>(h); }
int ref_solver_initialize(void *h, const char *name) {
    return guarded([&] { static_cast<hzl::Solver *>(h)->initialize(name); });
}
int ref_solver_initialize_physical(void *h, const double *field) {
    return guarded([&] {
        auto *s = static_cast<hzl::Solver *>(h);
        s->initialize_physical(to_field(field, s->size() * s->size()));
    });
}
int ref_solver_step(void *h, double dt, int steps) {
    return guarded([&] {
        for (int i = 0; i < steps; ++i)
            static_cast<hzl::Solver *>(h)->step(dt);
    });
}
int ref_solver_coefficients(void *h, double *out) {
    return guarded([&] { from_field(static_cast<hzl::Solver *>(h)->coefficients(), out); });
}
int ref_solver_forcing(void *h, double *out) {
    return guarded([&] { from_field(static_cast<hzl::Solver *>(h)->forcing(), out); });
}
int ref_solver_midpoint_forcing(void *h, double *out) {
    return guarded([&] { from_field(static_cast<hzl::Solver *>(h)->midpoint_forcing(), out); });
}
int ref_solver_update_latent_state(void *h, const double *w, const double *f) {
    return guarded([&] {
        auto *s = static_cast<hzl::Solver *>(h);
        const auto c = s->size() * s->size();
        s->update_latent_state(to_field(w, c), to_field(f, c));
    });
}
int ref_solver_diagnostics(void *h, double *out6) {
    return guarded([&] {
        const auto d = static_cast<hzl::Solver *>(h)->diagnostics();
        out6[0] = d.time;
        out6[1] = d.energy;
        out6[2] = d.enstrophy;
        out6[3] = d.dissipation;
        out6[4] = d.injection;
        out6[5] = d.cfl_rate;
    });
}
int ref_solver_physical_vorticity(void *h, double *out) {
    return guarded([&] { from_field(static_cast<hzl::Solver *>(h)->physical_vorticity(), out); });
}
int ref_solver_drift(void *h, const double *state, double *out) {
    return guarded([&] {
        auto *s = static_cast<hzl::Solver *>(h);
        from_field(s->drift(to_field(state, s->size() * s->size())), out);
    });
}
int ref_solver_linearized_drift(void *h, const double *state, const double *direction,
                                double *out) {
    return guarded([&] {
        auto *s = static_cast<hzl::Solver *>(h);
        const auto c = s->size() * s->size();
        from_field(s->linearized_drift(to_field(state, c), to_field(direction, c)), out);
    });
}
int ref_solver_adjoint_drift(void *h, const double *state, const double *cotangent,
                             double *out) {
    return guarded([&] {
        auto *s = static_cast<hzl::Solver *>(h);
        const auto c = s->size() * s->size();
        from_field(s->adjoint_drift(to_field(state, c), to_field(cotangent, c)), out);
    });
}
int ref_solver_save(void *h, const char *path) {
    return guarded([&] { static_cast<hzl::Solver *>(h)->save(path); });
}
int ref_solver_load(const char *path, void **out) {
    return guarded([&] { *out = new hzl::Solver(hzl::Solver::load(path)); });
}
int ref_solver_size(void *h) { return static_cast<int>(static_cast<hzl::Solver *>(h)->size()); }
int ref_solver_reseed_future(void *h, unsigned long long seed) {
    return guarded([&] { static_cast<hzl::Solver *>(h)->reseed_future(seed); });
}

// ---- hzl::ShellForcing ------------------------------------------------------------------
int ref_shell_forcing_create(int n, const double *p6, unsigned long long seed, void **out) {
    return guarded(
        [&] { *out = new hzl::ShellForcing(static_cast<std::size_t>(n), params(p6), seed); });
}
void ref_shell_forcing_destroy(void *h) { delete static_cast<hzl::ShellForcing *>(h); }
int ref_shell_forcing_midpoint_step(void *h, double dt, double *midpoint_out) {
    return guarded(
        [&] { from_field(static_cast<hzl::ShellForcing *>(h)->midpoint_step(dt), midpoint_out); });
}
int ref_shell_forcing_coefficients(void *h, double *out) {
    return guarded([&] { from_field(static_cast<hzl::ShellForcing *>(h)->coefficients(), out); });
}

// ---- hzl::ensemble ----------------------------------------------------------------------
int ref_ensemble(int n, const double *p6, double dt, unsigned long long steps,
                 unsigned long long count, unsigned long long workers, unsigned long long seed,
                 double *out6xcount) {
    return guarded([&] {
        const auto r = hzl::ensemble(static_cast<std::size_t>(n), params(p6), dt, steps, count,
                                     workers, seed);
        for (std::size_t i = 0; i < r.size(); ++i) {
            out6xcount[6 * i + 0] = r[i].time;
            out6xcount[6 * i + 1] = r[i].energy;
            out6xcount[6 * i + 2] = r[i].enstrophy;
            out6xcount[6 * i + 3] = r[i].dissipation;
            out6xcount[6 * i + 4] = r[i].injection;
            out6xcount[6 * i + 5] = r[i].cfl_rate;
        }
    });
}

// ---- the seeded-synthetic workload through the reference's public API ---------------------
// `count` members of the benchmark physics, each a reference hzl::Solver: OU forcing switched
// off (sigma 0, tau 1e300: the transition's decay is exactly 1 and its scale 0, so the latent
// forcing stays as installed, src/solver.cpp:93-105), the Kolmogorov forcing and the member's
// random initial field installed by Solver::update_latent_state, then per step Solver::step(dt)
// (RK4 with its validate_step) and the Euler-Maruyama noise of that step (the oracle's Philox
// draws, keyed by (seed, member)) added through update_latent_state.  Members are shared out
// over `workers` threads as hzl::ensemble does (src/inference.cpp:555-590).  final_out (may be
// null) receives the members' final spectra, n*n interleaved complex each.
int ref_synthetic_ensemble(int n, double nu, double dt, unsigned long long steps,
                           unsigned long long count, unsigned long long workers,
                           unsigned long long seed, double sigma, int noise_kmax,
                           double *final_out) {
    return guarded([&] {
        if (n < 16 || count == 0 || workers == 0)
            throw std::invalid_argument("invalid synthetic ensemble");
        const std::size_t nn = static_cast<std::size_t>(n) * n;
        hzl::Parameters p;
        p.viscosity = nu;
        p.friction = 0.0;
        p.forcing_sigma = 0.0;
        p.forcing_tau = 1e300;
        p.forcing_min = 4;
        p.forcing_max = 4;
        std::vector<double> kolm(2 * nn);
        if (ho_kolmogorov_forcing(n, 0.1, 4, kolm.data()) != 0)
            throw std::runtime_error("Kolmogorov forcing");
        const hzl::Field forcing = to_field(kolm.data(), nn);
        std::atomic<unsigned long long> next{0};
        std::vector<std::string> errors(workers);
        auto work = [&](std::size_t w) {
            try {
                std::vector<double> buf(2 * nn);
                for (unsigned long long m = next++; m < count; m = next++) {
                    hzl::Solver s(static_cast<std::size_t>(n), p, 0);
                    if (ho_grf_spectrum(n, seed, static_cast<uint32_t>(m), buf.data()) != 0)
                        throw std::runtime_error("random field");
                    s.update_latent_state(to_field(buf.data(), nn), forcing);
                    for (unsigned long long i = 0; i < steps; ++i) {
                        s.step(dt);
                        from_field(s.coefficients(), buf.data());
                        ho_add_noise(n, buf.data(), sigma, dt, noise_kmax, seed,
                                     static_cast<uint32_t>(m), i);
                        // a copy: update_latent_state must not read the forcing it rewrites
                        const hzl::Field f = s.forcing();
                        s.update_latent_state(to_field(buf.data(), nn), f);
                    }
                    if (final_out)
                        from_field(s.coefficients(), final_out + 2 * nn * m);
                }
            } catch (const std::exception &e) {
                errors[w] = e.what();
            }
        };
        {
            std::vector<std::jthread> pool;
            for (std::size_t w = 0; w < workers; ++w)
                pool.emplace_back(work, w);
        }
        for (const auto &e : errors)
            if (!e.empty())
                throw std::runtime_error(e);
    });
}

// ---- observations -----------------------------------------------------------------------
// Writes at most `capacity` observations; *count receives the number produced.
int ref_synthetic_observations(int n, double dt, unsigned long long steps, unsigned long long every,
                               const double *p6, double noise, unsigned long long seed,
                               unsigned long long capacity, unsigned long long *count,
                               unsigned long long *out_steps, unsigned *out_x, unsigned *out_y,
                               double *out_values, double *out_sd) {
    return guarded([&] {
        const auto d = hzl::synthetic_observations(static_cast<std::size_t>(n), dt, steps, every,
                                                   params(p6), noise, seed);
        if (d.observations.size() > capacity)
            throw std::invalid_argument("observation buffer too small");
        *count = d.observations.size();
        for (std::size_t i = 0; i < d.observations.size(); ++i) {
            const auto &o = d.observations[i];
            out_steps[i] = o.step;
            out_x[i] = static_cast<unsigned>(o.x);
            out_y[i] = static_cast<unsigned>(o.y);
            out_values[i] = o.value;
            out_sd[i] = o.standard_deviation;
        }
    });
}

// ---- filters ----------------------------------------------------------------------------
// History arrays: per observation group, (step, increment, ess, max weight) and optionally
// the mean physical vorticity (n*n complex interleaved).
int ref_bootstrap_filter(int n, double dt, int stochastic, int fmin, int fmax,
                         unsigned long long nobs, const unsigned long long *steps,
                         const unsigned *xs, const unsigned *ys, const double *values,
                         const double *sds, const double *p6, unsigned long long particles,
                         unsigned long long seed, int retain, double *loglik,
                         unsigned long long *resampling_events, unsigned long long capacity,
                         unsigned long long *groups, double *record4, double *means) {
    return guarded([&] {
        const auto d = dataset(static_cast<std::size_t>(n), dt, stochastic, fmin, fmax, nobs, steps,
                               xs, ys, values, sds);
        const auto r = hzl::bootstrap_filter(d, params(p6), particles, seed, retain != 0);
        if (r.history.size() > capacity)
            throw std::invalid_argument("history buffer too small");
        *loglik = r.log_likelihood;
        *resampling_events = r.resampling_events;
        *groups = r.history.size();
        for (std::size_t g = 0; g < r.history.size(); ++g) {
            const auto &h = r.history[g];
            record4[4 * g + 0] = static_cast<double>(h.step);
            record4[4 * g + 1] = h.log_likelihood_increment;
            record4[4 * g + 2] = h.effective_particles;
            record4[4 * g + 3] = h.maximum_weight;
            if (retain && means)
                from_field(h.mean_vorticity, means + 2 * g * static_cast<std::size_t>(n) * n);
        }
    });
}

// likelihood_adjoint: value, gradient[2], counters[3]
int ref_likelihood_adjoint(int n, double dt, int stochastic, int fmin, int fmax,
                           unsigned long long nobs, const unsigned long long *steps,
                           const unsigned *xs, const unsigned *ys, const double *values,
                           const double *sds, const double *q2, unsigned long long stride,
                           double *value, double *gradient, unsigned long long *counters) {
    return guarded([&] {
        const auto d = dataset(static_cast<std::size_t>(n), dt, stochastic, fmin, fmax, nobs, steps,
                               xs, ys, values, sds);
        const auto r = hzl::likelihood_adjoint(d, hzl::Vector(q2, q2 + 2), stride);
        *value = r.objective.value;
        gradient[0] = r.objective.gradient.size() > 0 ? r.objective.gradient[0] : 0;
        gradient[1] = r.objective.gradient.size() > 1 ? r.objective.gradient[1] : 0;
        counters[0] = r.checkpoint_fields;
        counters[1] = r.peak_block_fields;
        counters[2] = r.replayed_steps;
    });
}

// Dataset::save / Dataset::load
int ref_dataset_save(int n, double dt, int stochastic, int fmin, int fmax, unsigned long long nobs,
                     const unsigned long long *steps, const unsigned *xs, const unsigned *ys,
                     const double *values, const double *sds, const char *path) {
    return guarded([&] {
        hzl::Dataset d;
        d.n = static_cast<std::size_t>(n);
        d.dt = dt;
        d.stochastic = stochastic != 0;
        d.forcing_min = fmin;
        d.forcing_max = fmax;
        for (unsigned long long i = 0; i < nobs; ++i)
            d.observations.push_back({steps[i], xs[i], ys[i], values[i], sds[i]});
        d.save(path);
    });
}
int ref_dataset_load(const char *path, unsigned long long capacity, int *n, double *dt,
                     int *stochastic, int *fmin, int *fmax, unsigned long long *count,
                     unsigned long long *steps, unsigned *xs, unsigned *ys, double *values,
                     double *sds) {
    return guarded([&] {
        const auto d = hzl::Dataset::load(path);
        if (d.observations.size() > capacity)
            throw std::invalid_argument("observation buffer too small");
        *n = static_cast<int>(d.n);
        *dt = d.dt;
        *stochastic = d.stochastic ? 1 : 0;
        *fmin = d.forcing_min;
        *fmax = d.forcing_max;
        *count = d.observations.size();
        for (std::size_t i = 0; i < d.observations.size(); ++i) {
            const auto &o = d.observations[i];
            steps[i] = o.step;
            xs[i] = static_cast<unsigned>(o.x);
            ys[i] = static_cast<unsigned>(o.y);
            values[i] = o.value;
            sds[i] = o.standard_deviation;
        }
    });
}

// particle_log_likelihood (averaged = 0) / averaged_particle_log_likelihood (averaged = 1)
int ref_particle_log_likelihood(int n, double dt, int stochastic, int fmin, int fmax,
                                unsigned long long nobs, const unsigned long long *steps,
                                const unsigned *xs, const unsigned *ys, const double *values,
                                const double *sds, const double *q4, unsigned long long particles,
                                unsigned long long replicates, unsigned long long seed,
                                int averaged, double *out) {
    return guarded([&] {
        const auto d = dataset(static_cast<std::size_t>(n), dt, stochastic, fmin, fmax, nobs, steps,
                               xs, ys, values, sds);
        const hzl::Vector q(q4, q4 + 4);
        *out = averaged ? hzl::averaged_particle_log_likelihood(d, q, particles, replicates, seed)
                        : hzl::particle_log_likelihood(d, q, particles, seed);
    });
}

int ref_enkf(int n, double dt, int stochastic, int fmin, int fmax, unsigned long long nobs,
             const unsigned long long *steps, const unsigned *xs, const unsigned *ys,
             const double *values, const double *sds, const double *p6, unsigned long long members,
             unsigned long long seed, double inflation, double localization,
             unsigned long long forecast_steps, unsigned long long forecast_every,
             unsigned long long capacity, unsigned long long *records, double *record4,
             double *means) {
    return guarded([&] {
        const auto d = dataset(static_cast<std::size_t>(n), dt, stochastic, fmin, fmax, nobs, steps,
                               xs, ys, values, sds);
        const auto r = hzl::ensemble_kalman_filter(
            d, params(p6), members, seed, {inflation, localization, forecast_steps, forecast_every});
        if (r.size() > capacity)
            throw std::invalid_argument("history buffer too small");
        *records = r.size();
        for (std::size_t g = 0; g < r.size(); ++g) {
            record4[4 * g + 0] = static_cast<double>(r[g].step);
            record4[4 * g + 1] = r[g].forecast_sensor_rmse;
            record4[4 * g + 2] = r[g].posterior_spread;
            record4[4 * g + 3] = r[g].is_forecast ? 1.0 : 0.0;
            if (means)
                from_field(r[g].mean_vorticity, means + 2 * g * static_cast<std::size_t>(n) * n);
        }
    });
}

// ---- POD --------------------------------------------------------------------------------
// snapshots: m fields of `dimension` complex entries; outputs up to max_rank modes.
int ref_fit_pod(unsigned long long m, unsigned long long dimension, const double *snapshots,
                unsigned long long max_rank, double fraction, unsigned long long *rank,
                double *mean, double *modes, double *singular_values, double *captured) {
    return guarded([&] {
        std::vector<hzl::Field> s(m);
        for (std::size_t i = 0; i < m; ++i)
            s[i] = to_field(snapshots + 2 * i * dimension, dimension);
        const auto b = hzl::fit_pod(s, max_rank, fraction);
        *rank = b.modes.size();
        from_field(b.mean, mean);
        for (std::size_t j = 0; j < b.modes.size(); ++j) {
            from_field(b.modes[j], modes + 2 * j * dimension);
            singular_values[j] = b.singular_values[j];
        }
        *captured = b.captured_variance;
    });
}
// hzl::GalerkinModel over a POD basis given as mean + modes (reference layout): its rhs at
// `count` coefficient vectors, and `steps` RK4 steps of dt from them (in place).
int ref_galerkin(int n, const double *p6, unsigned long long rank, const double *mean,
                 const double *modes, unsigned long long count, const double *a, double *rhs,
                 double *stepped, double dt, unsigned long long steps) {
    return guarded([&] {
        const std::size_t dim = static_cast<std::size_t>(n) * n;
        hzl::PODBasis basis;
        basis.mean = to_field(mean, dim);
        for (std::size_t j = 0; j < rank; ++j)
            basis.modes.push_back(to_field(modes + 2 * j * dim, dim));
        basis.singular_values.assign(rank, 1.0);
        hzl::Solver solver(static_cast<std::size_t>(n), params(p6), 0);
        hzl::GalerkinModel model(basis, solver);
        for (std::size_t s = 0; s < count; ++s) {
            hzl::Vector v(a + s * rank, a + (s + 1) * rank);
            const auto r = model.rhs(v);
            std::copy(r.begin(), r.end(), rhs + s * rank);
            for (std::size_t t = 0; t < steps; ++t)
                model.step(v, dt);
            std::copy(v.begin(), v.end(), stepped + s * rank);
        }
    });
}
} // extern "C"
