/* TEST INFRASTRUCTURE ONLY -- CPU oracle; see hzl_oracle.h for scope and parity status.
 *
 * Arithmetic is written in the same operation order as the reference C++ (std::complex
 * products as (ac - bd, ad + bc), complex/real division component-wise), so that with the
 * same compiler flags the restatement reproduces the reference library bit for bit on the
 * FFT and the deterministic step; tests/test_oracle.py checks that. */
#define _GNU_SOURCE
#include "hzl_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define HO_PI 3.141592653589793238462643383279502884
static _Thread_local char last_error[256];
const char *ho_last_error(void) { return last_error; }
static int fail(int code, const char *message) {
    snprintf(last_error, sizeof last_error, "%s", message);
    return code;
}

/* ---- complex helpers (std::complex<double> semantics) ----------------------------- */
typedef struct {
    double re, im;
} cplx;
static inline cplx cmul(cplx a, cplx b) {
    cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
    return r;
}
static inline cplx cadd(cplx a, cplx b) {
    cplx r = {a.re + b.re, a.im + b.im};
    return r;
}
static inline cplx csub(cplx a, cplx b) {
    cplx r = {a.re - b.re, a.im - b.im};
    return r;
}
static inline cplx cscale(double s, cplx a) {
    cplx r = {s * a.re, s * a.im};
    return r;
}
static inline cplx cconj(cplx a) {
    cplx r = {a.re, -a.im};
    return r;
}
static inline double cnorm(cplx a) { return a.re * a.re + a.im * a.im; }
static inline int cfinite(cplx a) { return isfinite(a.re) && isfinite(a.im); }

/* ---- random numbers --------------------------------------------------------------- */
/* stream_seed: SplitMix64 mix of (base, index), solver.cpp:61-66. */
uint64_t ho_stream_seed(uint64_t base, uint64_t index) {
    uint64_t x = base + 0x9e3779b97f4a7c15ULL * (index + 1);
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

/* MT19937-64 (Matsumoto & Nishimura 2000), the engine behind std::mt19937_64 with its
 * standard seeding; NormalStream wraps it (solver.hpp:27-38). */
void ho_normal_init(ho_normal_stream *s, uint64_t seed) {
    s->mt[0] = seed;
    for (int i = 1; i < 312; ++i)
        s->mt[i] = 6364136223846793005ULL * (s->mt[i - 1] ^ (s->mt[i - 1] >> 62)) + (uint64_t)i;
    s->mti = 312;
    s->has_spare = 0;
    s->spare = 0;
}
uint64_t ho_mt_next(ho_normal_stream *s) {
    static const uint64_t mag[2] = {0ULL, 0xB5026F5AA96619E9ULL};
    const uint64_t um = 0xFFFFFFFF80000000ULL, lm = 0x7FFFFFFFULL;
    if (s->mti >= 312) {
        int i;
        uint64_t x;
        for (i = 0; i < 312 - 156; ++i) {
            x = (s->mt[i] & um) | (s->mt[i + 1] & lm);
            s->mt[i] = s->mt[i + 156] ^ (x >> 1) ^ mag[x & 1ULL];
        }
        for (; i < 311; ++i) {
            x = (s->mt[i] & um) | (s->mt[i + 1] & lm);
            s->mt[i] = s->mt[i + (156 - 312)] ^ (x >> 1) ^ mag[x & 1ULL];
        }
        x = (s->mt[311] & um) | (s->mt[0] & lm);
        s->mt[311] = s->mt[155] ^ (x >> 1) ^ mag[x & 1ULL];
        s->mti = 0;
    }
    uint64_t y = s->mt[s->mti++];
    y ^= (y >> 29) & 0x5555555555555555ULL;
    y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
    y ^= (y << 37) & 0xFFF7EEE000000000ULL;
    y ^= (y >> 43);
    return y;
}
/* NormalStream::operator(), solver.cpp:41-53: Box-Muller with a cached spare. */
double ho_normal_next(ho_normal_stream *s) {
    if (s->has_spare) {
        s->has_spare = 0;
        return s->spare;
    }
    const double u1 = ((double)(ho_mt_next(s) >> 11) + 0.5) * 0x1.0p-53;
    const double r = sqrt(-2 * log(u1));
    const double u2 = ((double)(ho_mt_next(s) >> 11) + 0.5) * 0x1.0p-53;
    const double angle = 2 * HO_PI * u2;
    s->spare = r * sin(angle);
    s->has_spare = 1;
    return r * cos(angle);
}

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of the 4x32 S-box with
 * multipliers 0xD2511F53 / 0xCD9E8D57 and Weyl key increments 0x9E3779B9 / 0xBB67AE85. */
void ho_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0;
        c1 = n1;
        c2 = n2;
        c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}
/* Mode code: (kx, ky) as two signed 16-bit fields, kx in the low half. */
uint32_t ho_mode_code(int kx, int ky) {
    return ((uint32_t)kx & 0xFFFFu) | (((uint32_t)ky & 0xFFFFu) << 16);
}
/* The seeded-synthetic noise convention.  Key = (low 32 bits of seed, member); counter =
 * (mode code, step low, step high, high 32 bits of seed); step 2^64-1 is reserved for the
 * initial field.  Two 53-bit uniforms in (0,1) from the output words (x1:x0) and (x3:x2),
 * then Box-Muller: xi1 = r cos(2 pi u2), xi2 = r sin(2 pi u2), r = sqrt(-2 log u1). */
void ho_philox_normal_pair(uint64_t seed, uint32_t member, uint64_t step, uint32_t mode_code,
                           double *xi1, double *xi2) {
    const uint32_t key[2] = {(uint32_t)seed, member};
    const uint32_t ctr[4] = {mode_code, (uint32_t)step, (uint32_t)(step >> 32),
                             (uint32_t)(seed >> 32)};
    uint32_t x[4];
    ho_philox4x32_10(ctr, key, x);
    const uint64_t a = ((uint64_t)x[1] << 32) | x[0], b = ((uint64_t)x[3] << 32) | x[2];
    const double u1 = ((double)(a >> 11) + 0.5) * 0x1.0p-53;
    const double u2 = ((double)(b >> 11) + 0.5) * 0x1.0p-53;
    const double r = sqrt(-2.0 * log(u1)), angle = 2.0 * HO_PI * u2;
    *xi1 = r * cos(angle);
    *xi2 = r * sin(angle);
}

/* ---- Fourier2D, fft.cpp:9-69 ------------------------------------------------------ */
static int wave_number(int index, int n) { return index < n / 2 ? index : index - n; }
static int valid_grid(int n) { return n >= 8 && n <= 4096 && (n & (n - 1)) == 0; }

typedef struct {
    int n;
    int *reversed;
    cplx *roots, *scratch;
} fourier2d;
static int fourier_init(fourier2d *f, int n) {
    if (!valid_grid(n))
        return fail(-1, "grid must be a power of two between 8 and 4096");
    f->n = n;
    f->reversed = malloc(sizeof(int) * (size_t)n);
    f->roots = malloc(sizeof(cplx) * (size_t)(n / 2));
    f->scratch = malloc(sizeof(cplx) * (size_t)n);
    int bits = 0;
    while ((1 << bits) < n)
        ++bits;
    for (int i = 0; i < n; ++i) {
        int x = i, r = 0;
        for (int b = 0; b < bits; ++b) {
            r = (r << 1) | (x & 1);
            x >>= 1;
        }
        f->reversed[i] = r;
    }
    for (int i = 0; i < n / 2; ++i) {
        const double theta = -2.0 * HO_PI * (double)i / (double)n;
        f->roots[i].re = cos(theta);
        f->roots[i].im = sin(theta);
    }
    return 0;
}
static void fourier_free(fourier2d *f) {
    free(f->reversed);
    free(f->roots);
    free(f->scratch);
}
/* Iterative radix-2 DIT on the scratch line, fft.cpp:29-43. */
static void fourier_line(fourier2d *f, int inverse) {
    const int n = f->n;
    cplx *s = f->scratch;
    for (int i = 0; i < n; ++i)
        if (i < f->reversed[i]) {
            cplx t = s[i];
            s[i] = s[f->reversed[i]];
            s[f->reversed[i]] = t;
        }
    for (int length = 2; length <= n; length *= 2) {
        const int half = length / 2, stride = n / length;
        for (int start = 0; start < n; start += length)
            for (int j = 0; j < half; ++j) {
                const cplx root = inverse ? cconj(f->roots[j * stride]) : f->roots[j * stride];
                const cplx a = s[start + j], b = cmul(root, s[start + j + half]);
                s[start + j] = cadd(a, b);
                s[start + j + half] = csub(a, b);
            }
    }
}
/* Rows, then columns through the scratch line; forward scaled by 1/n^2, fft.cpp:44-62. */
static void fourier_transform(fourier2d *f, cplx *data, int inverse) {
    const int n = f->n;
    for (int y = 0; y < n; ++y) {
        memcpy(f->scratch, data + (size_t)y * n, sizeof(cplx) * (size_t)n);
        fourier_line(f, inverse);
        memcpy(data + (size_t)y * n, f->scratch, sizeof(cplx) * (size_t)n);
    }
    for (int x = 0; x < n; ++x) {
        for (int y = 0; y < n; ++y)
            f->scratch[y] = data[(size_t)y * n + x];
        fourier_line(f, inverse);
        for (int y = 0; y < n; ++y)
            data[(size_t)y * n + x] = f->scratch[y];
    }
    if (!inverse) {
        const double scale = (double)((size_t)n * n);
        for (size_t i = 0; i < (size_t)n * n; ++i) {
            data[i].re /= scale;
            data[i].im /= scale;
        }
    }
}
int ho_fft(int n, double *data, int inverse) {
    fourier2d f;
    int rc = fourier_init(&f, n);
    if (rc)
        return rc;
    fourier_transform(&f, (cplx *)data, inverse);
    fourier_free(&f);
    return 0;
}

/* ---- Solver, solver.cpp:31-254, 381-425 ----------------------------------------- */
typedef struct {
    int i, j;
} mode_pair;
struct ho_solver {
    int n;
    double nu, alpha, sigma, tau;
    int kmin, kmax;
    fourier2d fft;
    ho_normal_stream random;
    double time;
    cplx *omega, *forcing, *midpoint, *u, *v, *wx, *wy, *nonlinear, *temporary, *k1, *k2, *k3,
        *k4;
    double *kx, *ky, *ksq;
    unsigned char *active;
    mode_pair *pairs;
    int npairs;
};

/* Parameters::validate, solver.cpp:31-40. */
static int validate_parameters(int n, const double *p6) {
    const double nu = p6[0], alpha = p6[1], sigma = p6[2], tau = p6[3];
    const int kmin = (int)p6[4], kmax = (int)p6[5];
    if (!isfinite(nu) || nu < 0 || !isfinite(alpha) || alpha < 0 || !isfinite(sigma) ||
        sigma < 0 || !isfinite(tau) || tau <= 0)
        return fail(-1, "nu, alpha, sigma must be finite and nonnegative; tau must be positive");
    if (kmin < 1 || kmax < kmin || 3LL * kmax >= (long long)n)
        return fail(-1, "forcing shell must lie strictly inside the dealiased grid");
    return 0;
}

int ho_solver_create(int n, const double *p6, uint64_t seed, ho_solver **out) {
    if (!valid_grid(n))
        return fail(-1, "grid must be a power of two between 8 and 4096");
    int rc = validate_parameters(n, p6);
    if (rc)
        return rc;
    ho_solver *s = calloc(1, sizeof *s);
    s->n = n;
    s->nu = p6[0];
    s->alpha = p6[1];
    s->sigma = p6[2];
    s->tau = p6[3];
    s->kmin = (int)p6[4];
    s->kmax = (int)p6[5];
    fourier_init(&s->fft, n);
    ho_normal_init(&s->random, seed);
    const size_t c = (size_t)n * n;
    cplx **fields[] = {&s->omega, &s->forcing, &s->midpoint, &s->u,         &s->v,
                       &s->wx,    &s->wy,      &s->nonlinear, &s->temporary, &s->k1,
                       &s->k2,    &s->k3,      &s->k4};
    for (size_t f = 0; f < sizeof fields / sizeof fields[0]; ++f)
        *fields[f] = calloc(c, sizeof(cplx));
    s->kx = malloc(c * sizeof(double));
    s->ky = malloc(c * sizeof(double));
    s->ksq = malloc(c * sizeof(double));
    s->active = malloc(c);
    s->pairs = malloc(c * sizeof(mode_pair));
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const size_t i = (size_t)y * n + x;
            const int a = wave_number(x, n), b = wave_number(y, n);
            s->kx[i] = a;
            s->ky[i] = b;
            s->ksq[i] = a * a + b * b;
            s->active[i] = 3 * abs(a) < n && 3 * abs(b) < n && i != 0;
        }
    /* forcing_pairs, solver.cpp:67-83 */
    s->npairs = 0;
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const int a = wave_number(x, n), b = wave_number(y, n);
            const int i = y * n + x, partner = ((n - y) % n) * n + (n - x) % n;
            const int k2 = a * a + b * b;
            if (3 * abs(a) < n && 3 * abs(b) < n && i < partner && k2 >= s->kmin * s->kmin &&
                k2 <= s->kmax * s->kmax) {
                s->pairs[s->npairs].i = i;
                s->pairs[s->npairs].j = partner;
                ++s->npairs;
            }
        }
    if (s->npairs == 0) {
        ho_solver_destroy(s);
        return fail(-1, "empty forcing shell");
    }
    /* initialize_ou, solver.cpp:84-92: stationary OU draw */
    const double scale = s->sigma * sqrt(s->tau / 4);
    for (int p = 0; p < s->npairs; ++p) {
        const double re = ho_normal_next(&s->random), im = ho_normal_next(&s->random);
        const cplx z = {re, im};
        s->forcing[s->pairs[p].i] = cscale(scale, z);
        s->forcing[s->pairs[p].j] = cconj(s->forcing[s->pairs[p].i]);
    }
    *out = s;
    return 0;
}
void ho_solver_destroy(ho_solver *s) {
    if (!s)
        return;
    cplx *fields[] = {s->omega, s->forcing, s->midpoint,  s->u,  s->v,  s->wx, s->wy,
                      s->nonlinear, s->temporary, s->k1, s->k2, s->k3, s->k4};
    for (size_t f = 0; f < sizeof fields / sizeof fields[0]; ++f)
        free(fields[f]);
    free(s->kx);
    free(s->ky);
    free(s->ksq);
    free(s->active);
    free(s->pairs);
    fourier_free(&s->fft);
    free(s);
}
static void project(const ho_solver *s, cplx *field) {
    const size_t c = (size_t)s->n * s->n;
    for (size_t i = 0; i < c; ++i)
        if (!s->active[i])
            field[i].re = field[i].im = 0;
}
/* transition_ou, solver.cpp:93-105 */
static int transition_ou(ho_solver *s, double dt) {
    if (!isfinite(dt) || dt <= 0)
        return fail(-1, "invalid OU transition interval");
    const double decay = exp(-dt / s->tau),
                 scale = s->sigma * sqrt(-s->tau * expm1(-2 * dt / s->tau) / 4);
    for (int p = 0; p < s->npairs; ++p) {
        const double re = ho_normal_next(&s->random), im = ho_normal_next(&s->random);
        const cplx z = {re, im};
        cplx *f = &s->forcing[s->pairs[p].i];
        *f = cadd(cscale(decay, *f), cscale(scale, z));
        s->forcing[s->pairs[p].j] = cconj(*f);
    }
    return 0;
}
/* Solver::initialize, solver.cpp:145-161 */
int ho_solver_initialize(ho_solver *s, const char *name) {
    const int tg = strcmp(name, "taylor-green") == 0, mm = strcmp(name, "multimode") == 0,
              zero = strcmp(name, "zero") == 0;
    if (!tg && !mm && !zero)
        return fail(-1, "unknown initial condition");
    if (s->time != 0)
        return fail(-2, "cannot reinitialize an evolved solver");
    const int n = s->n;
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const double a = 2 * HO_PI * (double)x / (double)n,
                         b = 2 * HO_PI * (double)y / (double)n;
            cplx *w = &s->omega[(size_t)y * n + x];
            w->re = zero ? 0.0 : 2 * cos(a) * cos(b);
            w->im = 0;
            if (mm)
                w->re += 0.6 * sin(2 * a + b) + 0.4 * cos(a - 3 * b) + 0.3 * sin(3 * a + 2 * b);
        }
    fourier_transform(&s->fft, s->omega, 0);
    project(s, s->omega);
    return 0;
}
/* Solver::initialize_physical, solver.cpp:162-173 */
int ho_solver_initialize_physical(ho_solver *s, const double *field) {
    if (s->time != 0)
        return fail(-2, "cannot reinitialize an evolved solver");
    const size_t c = (size_t)s->n * s->n;
    const cplx *f = (const cplx *)field;
    for (size_t i = 0; i < c; ++i)
        if (!cfinite(f[i]) || f[i].im != 0)
            return fail(-1, "physical initial vorticity must be finite and real");
    memcpy(s->omega, f, c * sizeof(cplx));
    fourier_transform(&s->fft, s->omega, 0);
    project(s, s->omega);
    return 0;
}
int ho_solver_set_state(ho_solver *s, const double *omega, const double *forcing) {
    const size_t c = (size_t)s->n * s->n;
    if (omega)
        memcpy(s->omega, omega, c * sizeof(cplx));
    if (forcing)
        memcpy(s->forcing, forcing, c * sizeof(cplx));
    return 0;
}
int ho_solver_get_state(const ho_solver *s, double *omega, double *forcing) {
    const size_t c = (size_t)s->n * s->n;
    if (omega)
        memcpy(omega, s->omega, c * sizeof(cplx));
    if (forcing)
        memcpy(forcing, s->forcing, c * sizeof(cplx));
    return 0;
}
int ho_solver_midpoint_forcing(const ho_solver *s, double *out) {
    memcpy(out, s->midpoint, (size_t)s->n * s->n * sizeof(cplx));
    return 0;
}
double ho_solver_time(const ho_solver *s) { return s->time; }
void ho_solver_reseed_future(ho_solver *s, uint64_t seed) { ho_normal_init(&s->random, seed); }

/* Solver::velocity, solver.cpp:177-185: Poisson solve then u = i ky psi, v = -i kx psi. */
static void velocity(ho_solver *s, const cplx *w) {
    const size_t c = (size_t)s->n * s->n;
    const cplx imaginary = {0, 1}, minus_imaginary = {-0.0, -1.0};
    for (size_t i = 0; i < c; ++i) {
        cplx psi = {0, 0};
        if (s->ksq[i] > 0) {
            psi.re = w[i].re / s->ksq[i];
            psi.im = w[i].im / s->ksq[i];
        }
        s->u[i] = cmul(cscale(s->ky[i], imaginary), psi);
        s->v[i] = cmul(cscale(s->kx[i], minus_imaginary), psi);
    }
    fourier_transform(&s->fft, s->u, 1);
    fourier_transform(&s->fft, s->v, 1);
}
/* Solver::rhs, solver.cpp:186-203, with the forcing field passed explicitly. */
static void rhs(ho_solver *s, const cplx *state, const cplx *forcing, cplx *result) {
    const size_t c = (size_t)s->n * s->n;
    const cplx imaginary = {0, 1};
    velocity(s, state);
    for (size_t i = 0; i < c; ++i) {
        s->wx[i] = cmul(cscale(s->kx[i], imaginary), state[i]);
        s->wy[i] = cmul(cscale(s->ky[i], imaginary), state[i]);
    }
    fourier_transform(&s->fft, s->wx, 1);
    fourier_transform(&s->fft, s->wy, 1);
    for (size_t i = 0; i < c; ++i) {
        s->nonlinear[i].re = s->u[i].re * s->wx[i].re + s->v[i].re * s->wy[i].re;
        s->nonlinear[i].im = 0;
    }
    fourier_transform(&s->fft, s->nonlinear, 0);
    for (size_t i = 0; i < c; ++i) {
        if (s->active[i]) {
            const cplx minus_nl = {-s->nonlinear[i].re, -s->nonlinear[i].im};
            cplx r = csub(minus_nl, cscale(s->nu * s->ksq[i] + s->alpha, state[i]));
            if (forcing)
                r = cadd(r, forcing[i]);
            result[i] = r;
        } else {
            result[i].re = result[i].im = 0;
        }
    }
}
/* Solver::diagnostics, solver.cpp:381-397 */
int ho_solver_diagnostics(ho_solver *s, double *out6) {
    const size_t c = (size_t)s->n * s->n;
    const double area = 4 * HO_PI * HO_PI;
    double energy = 0, enstrophy = 0, injection = 0, cfl = 0;
    for (size_t i = 1; i < c; ++i) {
        const double norm = cnorm(s->omega[i]);
        energy += area / 2 * norm / s->ksq[i];
        enstrophy += area / 2 * norm;
        injection += area * cmul(cconj(s->omega[i]), s->forcing[i]).re / s->ksq[i];
    }
    velocity(s, s->omega);
    for (size_t i = 0; i < c; ++i) {
        const double rate = (fabs(s->u[i].re) + fabs(s->v[i].re)) * (double)s->n / (2 * HO_PI);
        cfl = rate > cfl ? rate : cfl;
    }
    out6[0] = s->time;
    out6[1] = energy;
    out6[2] = enstrophy;
    out6[3] = 2 * s->nu * enstrophy;
    out6[4] = injection;
    out6[5] = cfl;
    return 0;
}
/* Solver::validate_step, solver.cpp:204-216 */
static int validate_step(ho_solver *s, double dt) {
    if (!isfinite(dt) || dt <= 0 || !isfinite(s->time + dt) || s->time + dt == s->time)
        return fail(-1, "invalid time step");
    double d[6];
    ho_solver_diagnostics(s, d);
    double max_linear = 0;
    const size_t c = (size_t)s->n * s->n;
    for (size_t i = 0; i < c; ++i)
        if (s->active[i]) {
            const double l = s->nu * s->ksq[i] + s->alpha;
            max_linear = l > max_linear ? l : max_linear;
        }
    if (dt * d[5] > 0.5 || dt * max_linear > 2.5)
        return fail(-2, "time step exceeds conservative explicit stability limits; reduce dt");
    return 0;
}
/* The RK4 branch of Solver::step, solver.cpp:222-234, then the finite check and projection
 * (:247-251). */
static int rk4(ho_solver *s, double dt, const cplx *forcing) {
    const size_t c = (size_t)s->n * s->n;
    rhs(s, s->omega, forcing, s->k1);
    for (size_t i = 0; i < c; ++i)
        s->temporary[i] = cadd(s->omega[i], cscale(dt / 2, s->k1[i]));
    rhs(s, s->temporary, forcing, s->k2);
    for (size_t i = 0; i < c; ++i)
        s->temporary[i] = cadd(s->omega[i], cscale(dt / 2, s->k2[i]));
    rhs(s, s->temporary, forcing, s->k3);
    for (size_t i = 0; i < c; ++i)
        s->temporary[i] = cadd(s->omega[i], cscale(dt, s->k3[i]));
    rhs(s, s->temporary, forcing, s->k4);
    for (size_t i = 0; i < c; ++i) {
        const cplx sum = cadd(cadd(cadd(s->k1[i], cscale(2.0, s->k2[i])), cscale(2.0, s->k3[i])),
                              s->k4[i]);
        s->omega[i] = cadd(s->omega[i], cscale(dt / 6, sum));
    }
    for (size_t i = 0; i < c; ++i)
        if (!cfinite(s->omega[i]))
            return fail(-2, "nonfinite flow state");
    project(s, s->omega);
    return 0;
}
/* Solver::step (RK4), solver.cpp:217-254 */
int ho_solver_step(ho_solver *s, double dt) {
    int rc = validate_step(s, dt);
    if (rc)
        return rc;
    if ((rc = transition_ou(s, dt / 2)))
        return rc;
    if (s->sigma > 0)
        memcpy(s->midpoint, s->forcing, (size_t)s->n * s->n * sizeof(cplx));
    if ((rc = rk4(s, dt, s->forcing)))
        return rc;
    if ((rc = transition_ou(s, dt / 2)))
        return rc;
    s->time += dt;
    return 0;
}
int ho_solver_step_forced(ho_solver *s, double dt, const double *forcing) {
    if (!isfinite(dt) || dt <= 0)
        return fail(-1, "invalid time step");
    int rc = rk4(s, dt, (const cplx *)forcing);
    if (rc)
        return rc;
    s->time += dt;
    return 0;
}
int ho_solver_physical_vorticity(ho_solver *s, double *out) {
    memcpy(out, s->omega, (size_t)s->n * s->n * sizeof(cplx));
    fourier_transform(&s->fft, (cplx *)out, 1);
    return 0;
}
/* Solver::update_latent_state, solver.cpp:403-425 */
int ho_solver_update_latent_state(ho_solver *s, const double *omega, const double *forcing) {
    const int n = s->n;
    const size_t c = (size_t)n * n;
    const cplx *w = (const cplx *)omega, *f = (const cplx *)forcing;
    for (size_t i = 0; i < c; ++i)
        if (!cfinite(w[i]) || !cfinite(f[i]))
            return fail(-1, "nonfinite assimilation state");
    memmove(s->omega, w, c * sizeof(cplx));
    project(s, s->omega);
    cplx *copy = malloc(c * sizeof(cplx));
    memcpy(copy, f, c * sizeof(cplx));
    memset(s->forcing, 0, c * sizeof(cplx));
    for (int p = 0; p < s->npairs; ++p) {
        const int i = s->pairs[p].i, j = s->pairs[p].j;
        s->forcing[i] = cscale(0.5, cadd(copy[i], cconj(copy[j])));
        s->forcing[j] = cconj(s->forcing[i]);
    }
    free(copy);
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const size_t i = (size_t)y * n + x, j = (size_t)((n - y) % n) * n + (n - x) % n;
            if (i < j) {
                s->omega[i] = cscale(0.5, cadd(s->omega[i], cconj(s->omega[j])));
                s->omega[j] = cconj(s->omega[i]);
            }
        }
    return 0;
}

/* ---- seeded-synthetic workload ------------------------------------------------------ */
/* Gaussian random field: per representative active mode (kx > 0, or kx == 0 and ky > 0)
 * omega_hat = sqrt(v(k)/2) (xi1 + i xi2) with v(k) = k^5 exp(-k^2/36), the per-mode variance
 * that gives a shell energy spectrum E(k) ~ k^4 exp(-(k/6)^2) under E = A/2 sum |w|^2/k^2;
 * partner = conjugate; then scaled to enstrophy A/2 sum |w|^2 = 1. */
int ho_grf_spectrum(int n, uint64_t seed, uint32_t member, double *omega_hat) {
    if (!valid_grid(n))
        return fail(-1, "grid must be a power of two between 8 and 4096");
    cplx *w = (cplx *)omega_hat;
    const size_t c = (size_t)n * n;
    memset(w, 0, c * sizeof(cplx));
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const int kx = wave_number(x, n), ky = wave_number(y, n);
            if (!(3 * abs(kx) < n && 3 * abs(ky) < n) || (kx == 0 && ky == 0))
                continue;
            if (!(kx > 0 || (kx == 0 && ky > 0)))
                continue;
            const double k2 = (double)(kx * kx + ky * ky), k = sqrt(k2);
            const double variance = k2 * k2 * k * exp(-k2 / 36.0);
            double xi1, xi2;
            ho_philox_normal_pair(seed, member, UINT64_MAX, ho_mode_code(kx, ky), &xi1, &xi2);
            const double amp = sqrt(variance / 2.0);
            const size_t i = (size_t)y * n + x;
            const size_t j = (size_t)((n - y) % n) * n + (n - x) % n;
            w[i].re = amp * xi1;
            w[i].im = amp * xi2;
            w[j] = cconj(w[i]);
        }
    const double area = 4 * HO_PI * HO_PI;
    double z = 0;
    for (size_t i = 0; i < c; ++i)
        z += area / 2 * cnorm(w[i]);
    if (!(z > 0))
        return fail(-1, "empty random field");
    const double scale = 1.0 / sqrt(z);
    for (size_t i = 0; i < c; ++i)
        w[i] = cscale(scale, w[i]);
    return 0;
}
/* amplitude*sin(k y) = amplitude (e^{iky} - e^{-iky})/(2i): coefficient -i amplitude/2 at
 * (0, k) and +i amplitude/2 at (0, -k). */
int ho_kolmogorov_forcing(int n, double amplitude, int wavenumber, double *forcing_hat) {
    if (!valid_grid(n) || wavenumber <= 0 || 3 * wavenumber >= n)
        return fail(-1, "Kolmogorov wavenumber must lie inside the dealiased grid");
    cplx *f = (cplx *)forcing_hat;
    memset(f, 0, (size_t)n * n * sizeof(cplx));
    f[(size_t)wavenumber * n].im = -amplitude / 2;
    f[(size_t)(n - wavenumber) * n].im = amplitude / 2;
    return 0;
}
int ho_add_noise(int n, double *omega_hat, double sigma, double dt, int kmax, uint64_t seed,
                 uint32_t member, uint64_t step) {
    cplx *w = (cplx *)omega_hat;
    const double scale = sigma * sqrt(dt) / sqrt(2.0);
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const int kx = wave_number(x, n), ky = wave_number(y, n);
            const int k2 = kx * kx + ky * ky;
            if (!(3 * abs(kx) < n && 3 * abs(ky) < n) || k2 < 1 || k2 > kmax * kmax)
                continue;
            if (!(kx > 0 || (kx == 0 && ky > 0)))
                continue;
            double xi1, xi2;
            ho_philox_normal_pair(seed, member, step, ho_mode_code(kx, ky), &xi1, &xi2);
            const size_t i = (size_t)y * n + x;
            const size_t j = (size_t)((n - y) % n) * n + (n - x) % n;
            w[i].re += scale * xi1;
            w[i].im += scale * xi2;
            w[j].re += scale * xi1;
            w[j].im -= scale * xi2;
        }
    return 0;
}
int ho_synthetic_step(ho_solver *s, double dt, const double *forcing, double sigma,
                      int noise_kmax, uint64_t seed, uint32_t member, uint64_t step) {
    int rc = ho_solver_step_forced(s, dt, forcing);
    if (rc)
        return rc;
    if (sigma > 0)
        ho_add_noise(s->n, (double *)s->omega, sigma, dt, noise_kmax, seed, member, step);
    return 0;
}

/* ---- particle filter, filter.cpp:76-120 -------------------------------------------- */
int ho_pf_weights(int count, const double *logs, double *weights, double *increment, double *ess,
                  double *max_weight) {
    /* std::max_element semantics: first largest element */
    double maximum = logs[0];
    for (int i = 1; i < count; ++i)
        if (maximum < logs[i])
            maximum = logs[i];
    if (!isfinite(maximum))
        return fail(-2, "particle likelihood collapsed numerically");
    double total = 0;
    for (int i = 0; i < count; ++i)
        total += exp(logs[i] - maximum);
    const double inc = maximum + log(total);
    double squared = 0, mw = 0;
    for (int i = 0; i < count; ++i) {
        weights[i] = exp(logs[i] - inc);
        squared += weights[i] * weights[i];
        mw = weights[i] > mw ? weights[i] : mw;
    }
    *increment = inc;
    *ess = 1 / squared;
    *max_weight = mw;
    return 0;
}
double ho_resampling_uniform(uint64_t raw) { return (double)(raw >> 11) * 0x1.0p-53; }
int ho_systematic_resample(int count, const double *weights, double u, uint32_t *ancestors) {
    int ancestor = 0;
    double cumulative = weights[0];
    const double start = u / (double)count;
    for (int i = 0; i < count; ++i) {
        const double position = start + (double)i / (double)count;
        while (position > cumulative && ancestor + 1 < count)
            cumulative += weights[++ancestor];
        ancestors[i] = (uint32_t)ancestor;
    }
    return 0;
}

/* ---- EnKF serial scalar update, filter.cpp:265-321 (no localisation) --------------- */
int ho_enkf_scalar_update(int count, ho_solver **s, const double *predictions, double value,
                          double sd, const double *perturbations) {
    if (count < 2)
        return fail(-1, "EnKF requires at least two ensemble members");
    const size_t dim = (size_t)s[0]->n * s[0]->n;
    cplx *mean_state = calloc(dim, sizeof(cplx)), *mean_forcing = calloc(dim, sizeof(cplx));
    cplx *sc = calloc(dim, sizeof(cplx)), *fc = calloc(dim, sizeof(cplx));
    cplx *state = malloc(dim * sizeof(cplx)), *forcing = malloc(dim * sizeof(cplx));
    const double dc = (double)count;
    double mean_prediction = 0;
    for (int i = 0; i < count; ++i) {
        mean_prediction += predictions[i] / dc;
        for (size_t j = 0; j < dim; ++j) {
            mean_state[j] = cadd(mean_state[j], (cplx){s[i]->omega[j].re / dc, s[i]->omega[j].im / dc});
            mean_forcing[j] =
                cadd(mean_forcing[j], (cplx){s[i]->forcing[j].re / dc, s[i]->forcing[j].im / dc});
        }
    }
    double variance = 0;
    for (int i = 0; i < count; ++i) {
        const double delta = predictions[i] - mean_prediction;
        variance += delta * delta / (double)(count - 1);
        const double w = delta / (double)(count - 1);
        for (size_t j = 0; j < dim; ++j) {
            sc[j] = cadd(sc[j], cscale(w, csub(s[i]->omega[j], mean_state[j])));
            fc[j] = cadd(fc[j], cscale(w, csub(s[i]->forcing[j], mean_forcing[j])));
        }
    }
    const double denominator = variance + sd * sd;
    int rc = 0;
    for (int i = 0; i < count && !rc; ++i) {
        const double innovation = (value + sd * perturbations[i] - predictions[i]) / denominator;
        for (size_t j = 0; j < dim; ++j) {
            state[j] = cadd(s[i]->omega[j], cscale(innovation, sc[j]));
            forcing[j] = cadd(s[i]->forcing[j], cscale(innovation, fc[j]));
        }
        rc = ho_solver_update_latent_state(s[i], (double *)state, (double *)forcing);
    }
    free(mean_state);
    free(mean_forcing);
    free(sc);
    free(fc);
    free(state);
    free(forcing);
    return rc;
}

/* ---- POD, reduced.cpp:8-136 -------------------------------------------------------- */
static double spectral_inner(const cplx *a, const cplx *b, int64_t dim) {
    double value = 0;
    for (int64_t i = 0; i < dim; ++i)
        value += cmul(cconj(a[i]), b[i]).re;
    return value;
}
typedef struct {
    const double *diag;
    int m;
} order_ctx;
static _Thread_local order_ctx sort_ctx;
static int by_eigenvalue_desc(const void *a, const void *b) {
    const int i = *(const int *)a, j = *(const int *)b;
    const double di = sort_ctx.diag[(size_t)i * sort_ctx.m + i],
                 dj = sort_ctx.diag[(size_t)j * sort_ctx.m + j];
    return di > dj ? -1 : (di < dj ? 1 : (i < j ? -1 : 1));
}
int ho_fit_pod(int m, int64_t dimension, const double *snapshots, int max_rank, double fraction,
               int *rank, double *mean_out, double *modes_out, double *singular_values,
               double *captured) {
    if (m < 2 || m > 512 || dimension <= 0 || max_rank <= 0 || !isfinite(fraction) ||
        fraction <= 0 || fraction > 1)
        return fail(-1,
                    "POD requires 2..512 snapshots, positive rank, and variance fraction in (0,1]");
    const cplx *snap = (const cplx *)snapshots;
    cplx *mean = (cplx *)mean_out;
    memset(mean, 0, (size_t)dimension * sizeof(cplx));
    for (int s = 0; s < m; ++s)
        for (int64_t i = 0; i < dimension; ++i) {
            const cplx z = snap[(size_t)s * dimension + i];
            if (!cfinite(z))
                return fail(-1, "nonfinite snapshot");
            mean[i].re += z.re / (double)m;
            mean[i].im += z.im / (double)m;
        }
    cplx *centered = malloc((size_t)m * dimension * sizeof(cplx));
    for (int s = 0; s < m; ++s)
        for (int64_t i = 0; i < dimension; ++i)
            centered[(size_t)s * dimension + i] = csub(snap[(size_t)s * dimension + i], mean[i]);
    double *cov = calloc((size_t)m * m, sizeof(double)), *vec = calloc((size_t)m * m, sizeof(double));
    double trace = 0;
    for (int i = 0; i < m; ++i) {
        vec[(size_t)i * m + i] = 1;
        for (int j = 0; j <= i; ++j)
            cov[(size_t)i * m + j] = cov[(size_t)j * m + i] =
                spectral_inner(centered + (size_t)i * dimension, centered + (size_t)j * dimension,
                               dimension);
        trace += cov[(size_t)i * m + i];
    }
    int rc = 0;
    if (trace <= 0 || !isfinite(trace)) {
        rc = fail(-1, "snapshots have no finite variance");
        goto done;
    }
    int converged = 0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double maximum = 0;
        for (int p = 0; p < m; ++p)
            for (int q = p + 1; q < m; ++q) {
                const double off = cov[(size_t)p * m + q];
                maximum = fabs(off) > maximum ? fabs(off) : maximum;
                if (fabs(off) < 1e-14 * trace)
                    continue;
                const double tau = (cov[(size_t)q * m + q] - cov[(size_t)p * m + p]) / (2 * off);
                const double t = copysign(1.0, tau) / (fabs(tau) + hypot(1.0, tau)),
                             c = 1 / sqrt(1 + t * t), sn = t * c;
                const double pp = cov[(size_t)p * m + p], qq = cov[(size_t)q * m + q];
                cov[(size_t)p * m + p] = pp - t * off;
                cov[(size_t)q * m + q] = qq + t * off;
                cov[(size_t)p * m + q] = cov[(size_t)q * m + p] = 0;
                for (int k = 0; k < m; ++k) {
                    if (k != p && k != q) {
                        const double a = cov[(size_t)k * m + p], b = cov[(size_t)k * m + q];
                        cov[(size_t)k * m + p] = cov[(size_t)p * m + k] = c * a - sn * b;
                        cov[(size_t)k * m + q] = cov[(size_t)q * m + k] = sn * a + c * b;
                    }
                    const double a = vec[(size_t)k * m + p], b = vec[(size_t)k * m + q];
                    vec[(size_t)k * m + p] = c * a - sn * b;
                    vec[(size_t)k * m + q] = sn * a + c * b;
                }
            }
        if (maximum < 1e-12 * trace) {
            converged = 1;
            break;
        }
    }
    if (!converged) {
        rc = fail(-2, "snapshot Jacobi eigensolver failed to converge");
        goto done;
    }
    int *order = malloc((size_t)m * sizeof(int));
    for (int i = 0; i < m; ++i)
        order[i] = i;
    sort_ctx.diag = cov;
    sort_ctx.m = m;
    qsort(order, (size_t)m, sizeof(int), by_eigenvalue_desc);
    double retained = 0;
    int r = 0;
    cplx *modes = (cplx *)modes_out;
    for (int o = 0; o < m; ++o) {
        const int column = order[o];
        const double eigenvalue = cov[(size_t)column * m + column];
        if (eigenvalue <= 1e-12 * trace || r >= max_rank)
            break;
        cplx *mode = modes + (size_t)r * dimension;
        memset(mode, 0, (size_t)dimension * sizeof(cplx));
        for (int j = 0; j < m; ++j) {
            const double w = vec[(size_t)j * m + column] / sqrt(eigenvalue);
            for (int64_t i = 0; i < dimension; ++i)
                mode[i] = cadd(mode[i], cscale(w, centered[(size_t)j * dimension + i]));
        }
        for (int pass = 0; pass < 2; ++pass)
            for (int prev = 0; prev < r; ++prev) {
                const cplx *pm = modes + (size_t)prev * dimension;
                const double overlap = spectral_inner(pm, mode, dimension);
                for (int64_t i = 0; i < dimension; ++i)
                    mode[i] = csub(mode[i], cscale(overlap, pm[i]));
            }
        const double norm = sqrt(spectral_inner(mode, mode, dimension));
        if (norm < 1e-8) {
            free(order);
            rc = fail(-2, "numerically degenerate POD mode");
            goto done;
        }
        for (int64_t i = 0; i < dimension; ++i) {
            mode[i].re /= norm;
            mode[i].im /= norm;
        }
        singular_values[r] = sqrt(eigenvalue);
        ++r;
        retained += eigenvalue;
        if (retained / trace >= fraction)
            break;
    }
    free(order);
    if (r == 0) {
        rc = fail(-2, "no resolved POD modes");
        goto done;
    }
    *rank = r;
    *captured = retained / trace;
done:
    free(centered);
    free(cov);
    free(vec);
    return rc;
}
