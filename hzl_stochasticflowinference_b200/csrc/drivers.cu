// Drop-in drivers for the reference's ensemble entry points, on the batched B200 engine:
//   hzl::ensemble               (src/inference.cpp:555-590)
//   hzl::bootstrap_filter       (src/filter.cpp:38-126)
//   hzl::ensemble_kalman_filter (src/filter.cpp:204-356)
// They keep the reference's semantics exactly: member i's OU forcing draws from
// NormalStream(stream_seed(seed, i)) (mt19937_64 + Box-Muller), forcing is frozen at the
// midpoint over the RK4 step (solver.cpp:217-254), the particle filter resamples with
// mt19937_64(stream_seed(seed, 2^64-1)) and reseeds clones with stream_seed(seed, (g+1)M+i),
// and the EnKF assimilates scalar observations serially with perturbations from
// NormalStream(stream_seed(seed, M)).  The OU forcing is a few shell modes per member, so it
// lives on the host (one batched upload per step); the flow state lives on the device.
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <limits>
#include <random>
#include <sstream>
#include <string>

namespace hzlb {
namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;
using cd = std::complex<double>;

int wave(int i, int n) { return i < n / 2 ? i : i - n; }

// SplitMix64 mix of (base, index): the reference's logical stream identities.
uint64_t stream_seed(uint64_t base, uint64_t index) {
    uint64_t x = base + 0x9e3779b97f4a7c15ULL * (index + 1);
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
    return x ^ (x >> 31);
}

// mt19937_64 uniforms ((x >> 11) + 1/2) 2^-53 and Box-Muller with a cached spare.
class NormalStream {
  public:
    explicit NormalStream(uint64_t seed = 0) : engine_(seed) {}
    double operator()() {
        if (has_spare_) {
            has_spare_ = false;
            return spare_;
        }
        const double u1 = (static_cast<double>(engine_() >> 11) + 0.5) * 0x1.0p-53;
        const double r = std::sqrt(-2 * std::log(u1));
        const double u2 = (static_cast<double>(engine_() >> 11) + 0.5) * 0x1.0p-53;
        const double angle = 2 * kPi * u2;
        spare_ = r * std::sin(angle);
        has_spare_ = true;
        return r * std::cos(angle);
    }
    // checkpoint text of the stream (solver.cpp:54-60): the engine's standard textual state,
    // then the cached second normal
    void write(std::ostream &out) const { out << engine_ << '\n' << has_spare_ << ' ' << spare_ << '\n'; }
    void read(std::istream &in) {
        if (!(in >> engine_ >> has_spare_ >> spare_) || !std::isfinite(spare_))
            raise(HZLB_ERUNTIME, "invalid checkpoint random stream");
    }

  private:
    std::mt19937_64 engine_;
    bool has_spare_ = false;
    double spare_ = 0;
};

struct Params {
    double nu, alpha, sigma, tau;
    int kmin, kmax;
};
void validate_params(int n, const Params &p) {
    if (!std::isfinite(p.nu) || p.nu < 0 || !std::isfinite(p.alpha) || p.alpha < 0 ||
        !std::isfinite(p.sigma) || p.sigma < 0 || !std::isfinite(p.tau) || p.tau <= 0)
        raise(HZLB_EINVAL, "nu, alpha, sigma must be finite and nonnegative; tau must be positive");
    if (p.kmin < 1 || p.kmax < p.kmin || 3LL * p.kmax >= static_cast<long long>(n))
        raise(HZLB_EINVAL, "forcing shell must lie strictly inside the dealiased grid");
}

// Per-member OU shell forcing: the pairs (i < partner) of retained modes with
// kmin^2 <= |k|^2 <= kmax^2 in the reference's enumeration order (y outer, x inner).
class OuBank {
  public:
    OuBank(int n, const Params &p, int members, uint64_t seed)
        : OuBank(n, p, member_seeds(members, seed)) {}
    // member m draws from NormalStream(stream_seeds[m])
    static std::vector<uint64_t> member_seeds(int members, uint64_t seed) {
        std::vector<uint64_t> v(members);
        for (int m = 0; m < members; ++m)
            v[m] = stream_seed(seed, static_cast<uint64_t>(m));
        return v;
    }
    OuBank(int n, const Params &p, const std::vector<uint64_t> &stream_seeds)
        : n_(n), p_(p), M_(static_cast<int>(stream_seeds.size())) {
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                const int a = wave(x, n), b = wave(y, n);
                const int i = y * n + x, partner = ((n - y) % n) * n + (n - x) % n;
                const int k2 = a * a + b * b;
                if (3 * std::abs(a) < n && 3 * std::abs(b) < n && i < partner &&
                    k2 >= p.kmin * p.kmin && k2 <= p.kmax * p.kmax)
                    modes_.push_back({a, b});
            }
        if (modes_.empty())
            raise(HZLB_EINVAL, "empty forcing shell");
        const size_t P = modes_.size();
        value_.assign(static_cast<size_t>(M_) * P, cd(0, 0));
        midpoint_.assign(value_.size(), cd(0, 0));
        streams_.reserve(M_);
        const double scale = p.sigma * std::sqrt(p.tau / 4);   // stationary draw
        for (int m = 0; m < M_; ++m) {
            streams_.emplace_back(stream_seeds[m]);
            for (size_t k = 0; k < P; ++k) {
                const double re = streams_[m](), im = streams_[m]();
                value_[m * P + k] = scale * cd(re, im);
            }
        }
    }
    size_t pairs() const { return modes_.size(); }
    void transition(double h) {
        const double decay = std::exp(-h / p_.tau),
                     scale = p_.sigma * std::sqrt(-p_.tau * std::expm1(-2 * h / p_.tau) / 4);
        const size_t P = modes_.size();
        for (int m = 0; m < M_; ++m)
            for (size_t k = 0; k < P; ++k) {
                const double re = streams_[m](), im = streams_[m]();
                value_[m * P + k] = decay * value_[m * P + k] + scale * cd(re, im);
            }
    }
    // OU(dt/2), keep the midpoint, OU(dt/2): Solver::step's forcing schedule.
    void midpoint_step(double dt) {
        if (!std::isfinite(dt) || dt <= 0)
            raise(HZLB_EINVAL, "invalid OU transition interval");
        transition(dt / 2);
        midpoint_ = value_;
        transition(dt / 2);
    }
    // Compact forcing (columns kx <= kmax) of `which` (midpoint or current), interleaved.
    void compact(bool midpoint, int cols, std::vector<double> &out) const {
        const int K = (n_ - 1) / 3, LD = 2 * K + 1;
        const size_t block = static_cast<size_t>(cols) * LD, P = modes_.size();
        out.assign(2 * block * M_, 0.0);
        const auto &src = midpoint ? midpoint_ : value_;
        for (int m = 0; m < M_; ++m)
            for (size_t k = 0; k < P; ++k) {
                int kx = modes_[k].first, ky = modes_[k].second;
                cd v = src[m * P + k];
                if (kx < 0 || (kx == 0 && ky < 0)) {   // store the kx >= 0 member of the pair
                    kx = -kx;
                    ky = -ky;
                    v = std::conj(v);
                }
                auto put = [&](int kxx, int kyy, cd z) {
                    const int j = kyy >= 0 ? kyy : kyy + LD;
                    const size_t at = m * block + static_cast<size_t>(kxx) * LD + j;
                    out[2 * at] = z.real();
                    out[2 * at + 1] = z.imag();
                };
                put(kx, ky, v);
                if (kx == 0)
                    put(0, -ky, std::conj(v));
            }
    }
    void gather(const std::vector<uint32_t> &anc) {
        const size_t P = modes_.size();
        std::vector<cd> v(value_.size()), mid(midpoint_.size());
        for (int i = 0; i < M_; ++i)
            for (size_t k = 0; k < P; ++k) {
                v[i * P + k] = value_[anc[i] * P + k];
                mid[i * P + k] = midpoint_[anc[i] * P + k];
            }
        value_.swap(v);
        midpoint_.swap(mid);
    }
    void reseed(int m, uint64_t seed) { streams_[m] = NormalStream(seed); }
    NormalStream &stream(int m) { return streams_[m]; }
    std::vector<cd> &values() { return value_; }
    const std::vector<std::pair<int, int>> &modes() const { return modes_; }

  private:
    int n_;
    Params p_;
    int M_;
    std::vector<std::pair<int, int>> modes_;   // (kx, ky) of the pair's first index
    std::vector<cd> value_, midpoint_;         // [member][pair]
    std::vector<NormalStream> streams_;
};

// 2-D transform in the reference convention (forward scaled by 1/n^2), radix-2 with
// precomputed roots; used on single fields (ensemble means, covariances).
void host_fft2(int n, std::vector<cd> &a, bool inverse) {
    std::vector<cd> roots(n / 2), line(n);
    for (int i = 0; i < n / 2; ++i)
        roots[i] = std::polar(1.0, (inverse ? 2.0 : -2.0) * kPi * i / n);
    int bits = 0;
    while ((1 << bits) < n)
        ++bits;
    auto transform = [&](cd *base, int stride) {
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int b = 0; b < bits; ++b)
                r |= ((i >> b) & 1) << (bits - 1 - b);
            line[r] = base[static_cast<size_t>(i) * stride];
        }
        for (int len = 2; len <= n; len <<= 1)
            for (int s = 0; s < n; s += len)
                for (int j = 0; j < len / 2; ++j) {
                    const cd u = line[s + j], t = roots[j * (n / len)] * line[s + j + len / 2];
                    line[s + j] = u + t;
                    line[s + j + len / 2] = u - t;
                }
        for (int i = 0; i < n; ++i)
            base[static_cast<size_t>(i) * stride] = line[i];
    };
    for (int y = 0; y < n; ++y)
        transform(&a[static_cast<size_t>(y) * n], 1);
    for (int x = 0; x < n; ++x)
        transform(&a[x], n);
    if (!inverse)
        for (auto &z : a)
            z /= static_cast<double>(n) * n;
}

// compact interleaved (kx 0..K, j) -> full n*n reference layout with conjugate partners
std::vector<cd> compact_to_full(int n, const std::vector<double> &c) {
    const int K = (n - 1) / 3, LD = 2 * K + 1;
    std::vector<cd> f(static_cast<size_t>(n) * n, cd(0, 0));
    for (int kx = 0; kx <= K; ++kx)
        for (int j = 0; j < LD; ++j) {
            const int ypos = j <= K ? j : n - LD + j;
            const size_t at = static_cast<size_t>(kx) * LD + j;
            const cd z(c[2 * at], c[2 * at + 1]);
            f[static_cast<size_t>(ypos) * n + kx] = z;
            if (kx > 0)
                f[static_cast<size_t>((n - ypos) % n) * n + (n - kx)] = std::conj(z);
        }
    return f;
}
std::vector<double> full_to_compact(int n, const std::vector<cd> &f) {
    const int K = (n - 1) / 3, LD = 2 * K + 1;
    std::vector<double> c(2 * static_cast<size_t>(K + 1) * LD);
    for (int kx = 0; kx <= K; ++kx)
        for (int j = 0; j < LD; ++j) {
            const int ypos = j <= K ? j : n - LD + j;
            const cd z = f[static_cast<size_t>(ypos) * n + kx];
            const size_t at = static_cast<size_t>(kx) * LD + j;
            c[2 * at] = z.real();
            c[2 * at + 1] = z.imag();
        }
    c[0] = c[1] = 0;
    return c;
}

// The reference's "multimode" initial vorticity (solver.cpp:145-161) as coefficients.
std::vector<cd> initial_field(int n, const char *name) {
    std::vector<cd> w(static_cast<size_t>(n) * n);
    const bool zero = std::strcmp(name, "zero") == 0, mm = std::strcmp(name, "multimode") == 0;
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const double a = 2 * kPi * x / n, b = 2 * kPi * y / n;
            double v = zero ? 0.0 : 2 * std::cos(a) * std::cos(b);
            if (mm)
                v += 0.6 * std::sin(2 * a + b) + 0.4 * std::cos(a - 3 * b) + 0.3 * std::sin(3 * a + 2 * b);
            w[static_cast<size_t>(y) * n + x] = v;
        }
    host_fft2(n, w, false);
    return w;
}

struct Dataset {
    int n;
    double dt;
    int fmin, fmax;
    std::vector<hzlb_observation> obs;
};
Dataset load_dataset(const hzlb_dataset *d) {
    if (!d || (d->count && !d->observations))
        raise(HZLB_EINVAL, "invalid observation dataset");
    Dataset ds{d->n, d->dt, d->forcing_min, d->forcing_max, {}};
    if (d->n < 16 || d->n > 512 || (d->n & (d->n - 1)) || !std::isfinite(d->dt) || d->dt <= 0 ||
        d->count == 0)
        raise(HZLB_EINVAL, "invalid observation dataset");
    Params p{0.01, 0.1, 0.2, 0.5, d->forcing_min, d->forcing_max};
    validate_params(d->n, p);
    ds.obs.assign(d->observations, d->observations + d->count);
    uint64_t previous = 0;
    for (const auto &o : ds.obs) {
        if (o.step < previous || o.x >= static_cast<uint32_t>(d->n) ||
            o.y >= static_cast<uint32_t>(d->n) || !std::isfinite(o.value) ||
            !std::isfinite(o.standard_deviation) || o.standard_deviation <= 0)
            raise(HZLB_EINVAL, "observations must be time ordered, finite, in bounds, and have "
                               "positive uncertainty");
        previous = o.step;
    }
    return ds;
}

// An ensemble of reference-physics members on the engine plus their host OU forcing.
struct RefEnsemble {
    int n, M;
    Params p;
    std::unique_ptr<Engine> engine;
    OuBank bank;
    int precision_;
    std::vector<double> fbuf;
    RefEnsemble(int n_, const Params &p_, int members, uint64_t seed, int precision, int device)
        : RefEnsemble(n_, p_, OuBank::member_seeds(members, seed), precision, device) {}
    RefEnsemble(int n_, const Params &p_, const std::vector<uint64_t> &stream_seeds, int precision,
                int device)
        : n(n_), M(static_cast<int>(stream_seeds.size())), p(p_), bank(n_, p_, stream_seeds),
          precision_(precision) {
        hzlb_config c{};
        c.n = n;
        c.members = M;
        c.precision = precision;
        c.nu = p.nu;
        c.alpha = p.alpha;
        c.forcing_kmax = p.kmax;
        c.forcing_per_member = 1;
        c.device = device;
        engine = make_engine(c);
    }
    void set_initial(const char *name) {
        const auto w = initial_field(n, name);
        const auto c = full_to_compact(n, w);
        std::vector<double> all(c.size() * M);
        for (int m = 0; m < M; ++m)
            std::copy(c.begin(), c.end(), all.begin() + m * c.size());
        if (engine->compact_size() * 2 != c.size())
            raise(HZLB_ERUNTIME, "compact layout mismatch");
        upload_compact(all);
    }
    void upload_compact(const std::vector<double> &all) {
        // the engine's compact upload takes its own precision
        const size_t elems = all.size() / 2;
        if (precision() == 8) {
            engine->set_state_compact(all.data(), 0, M);
            engine->synchronize();
        } else {
            std::vector<float> f(2 * elems);
            for (size_t i = 0; i < 2 * elems; ++i)
                f[i] = static_cast<float>(all[i]);
            engine->set_state_compact(f.data(), 0, M);
            engine->synchronize();
        }
    }
    int precision() const { return precision_; }
    void step(double dt) {
        bank.midpoint_step(dt);
        bank.compact(true, engine->forcing_columns(), fbuf);
        engine->set_forcing_compact(fbuf.data(), 0, M);
        engine->step(dt, 1);
    }
    void check_status() {
        const uint32_t s = engine->status();
        if (s & HZLB_STATUS_NONFINITE)
            raise(HZLB_ERUNTIME, "nonfinite flow state");
        if (s & HZLB_STATUS_CFL)
            raise(HZLB_ERUNTIME, "time step exceeds conservative explicit stability limits; reduce dt");
    }
    void upload_current_forcing() {
        bank.compact(false, engine->forcing_columns(), fbuf);
        engine->set_forcing_compact(fbuf.data(), 0, M);
    }
    std::vector<double> mean() {   // sum of coefficient / M in member order
        std::vector<double> out(2 * engine->compact_size());
        engine->member_sum(nullptr, static_cast<double>(M), out.data());
        return out;
    }
};

void validate_dt(int n, const Params &p, double dt) {
    const int largest = (n - 1) / 3;
    if (!std::isfinite(dt) || dt <= 0 || dt * (2 * p.nu * largest * largest + p.alpha) > 2.5)
        raise(HZLB_EINVAL, "invalid time step or diffusion stability limit exceeded");
}

// ---- HZL_CHECKPOINT_V1 (Solver::save / Solver::load, src/solver.cpp:434-491) ----------------
// One member as the reference's Solver would hold it: n, time, parameters, its OU stream,
// then omega and the latent forcing over the whole n x n spectrum (y outer, x inner).
struct Checkpoint {
    int n = 0;
    double time = 0;
    Params p{};
    NormalStream stream;
    std::vector<cd> omega, forcing;
};

void write_checkpoint(const std::string &path, const Checkpoint &c) {
    std::ofstream out(path);
    if (!out)
        raise(HZLB_ERUNTIME, "cannot open checkpoint for writing");
    out << std::setprecision(std::numeric_limits<double>::max_digits10);
    out << "HZL_CHECKPOINT_V1\n"
        << c.n << ' ' << c.time << '\n'
        << c.p.nu << ' ' << c.p.alpha << ' ' << c.p.sigma << ' ' << c.p.tau << ' ' << c.p.kmin
        << ' ' << c.p.kmax << '\n';
    c.stream.write(out);
    for (size_t i = 0; i < c.omega.size(); ++i)
        out << c.omega[i].real() << ' ' << c.omega[i].imag() << ' ' << c.forcing[i].real() << ' '
            << c.forcing[i].imag() << '\n';
    if (!out)
        raise(HZLB_ERUNTIME, "checkpoint write failed");
}

bool active_mode(int n, int x, int y) {
    const int a = wave(x, n), b = wave(y, n);
    return 3 * std::abs(a) < n && 3 * std::abs(b) < n && (x != 0 || y != 0);
}

// Solver::load's parse and checks, in its order and with its messages.  The device grid is
// limited to 512.
Checkpoint read_checkpoint(const std::string &path) {
    std::ifstream in(path);
    std::string magic;
    size_t n = 0;
    Checkpoint c;
    double nu = 0, alpha = 0, sigma = 0, tau = 0;
    int kmin = 0, kmax = 0;
    if (!(in >> magic >> n >> c.time >> nu >> alpha >> sigma >> tau >> kmin >> kmax) ||
        magic != "HZL_CHECKPOINT_V1" || !std::isfinite(c.time) || c.time < 0)
        raise(HZLB_ERUNTIME, "invalid checkpoint header");
    if (n < 8 || n > 4096 || (n & (n - 1)))
        raise(HZLB_EINVAL, "grid must be a power of two between 8 and 4096");
    c.n = static_cast<int>(n);
    c.p = Params{nu, alpha, sigma, tau, kmin, kmax};
    validate_params(c.n, c.p);
    if (n > 512)
        raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
    OuBank shell(c.n, c.p, std::vector<uint64_t>{0});   // the forced pairs ("empty forcing shell")
    c.stream.read(in);
    const size_t nn = n * n;
    c.omega.assign(nn, cd(0, 0));
    c.forcing.assign(nn, cd(0, 0));
    for (size_t i = 0; i < nn; ++i) {
        double a = 0, b = 0, f = 0, g = 0;
        if (!(in >> a >> b >> f >> g) || !std::isfinite(a) || !std::isfinite(b) ||
            !std::isfinite(f) || !std::isfinite(g))
            raise(HZLB_ERUNTIME, "invalid checkpoint field");
        c.omega[i] = cd(a, b);
        c.forcing[i] = cd(f, g);
    }
    std::vector<bool> forced(nn, false);
    for (const auto &[a, b] : shell.modes()) {
        const int x = (a + c.n) % c.n, y = (b + c.n) % c.n;
        forced[static_cast<size_t>(y) * n + x] = true;
        forced[static_cast<size_t>((c.n - y) % c.n) * n + (c.n - x) % c.n] = true;
    }
    for (int y = 0; y < c.n; ++y)
        for (int x = 0; x < c.n; ++x) {
            const size_t i = static_cast<size_t>(y) * n + x,
                         partner = static_cast<size_t>((c.n - y) % c.n) * n + (c.n - x) % c.n;
            if ((!active_mode(c.n, x, y) && c.omega[i] != cd(0, 0)) ||
                (!forced[i] && c.forcing[i] != cd(0, 0)) ||
                std::abs(c.omega[i] - std::conj(c.omega[partner])) >
                    1e-10 * (1 + std::abs(c.omega[i])) ||
                c.forcing[i] != std::conj(c.forcing[partner]))
                raise(HZLB_ERUNTIME, "checkpoint violates spectral constraints");
        }
    std::string trailing;
    if (in >> trailing)
        raise(HZLB_ERUNTIME, "unexpected checkpoint data");
    return c;
}

} // namespace
} // namespace hzlb

using namespace hzlb;

namespace {
thread_local std::string driver_error;
template <class F> int guarded_driver(F &&f) {
    try {
        f();
        return HZLB_OK;
    } catch (const Error &e) {
        driver_error = e.what();
        set_last_error(driver_error);
        return e.code;
    } catch (const std::exception &e) {
        driver_error = e.what();
        set_last_error(driver_error);
        return HZLB_ERUNTIME;
    }
}
Params to_params(const hzlb_parameters *p) {
    if (!p)
        raise(HZLB_EINVAL, "null parameters");
    return Params{p->viscosity, p->friction, p->forcing_sigma, p->forcing_tau, p->forcing_min,
                  p->forcing_max};
}
} // namespace

// A set of reference Solvers (one OU stream each) advanced together on the device, with the
// time each of them would hold (the sum of its steps' dt, as Solver::step accumulates it).
struct hzlb_solvers {
    std::unique_ptr<RefEnsemble> e;
    double time = 0;
};

namespace {
void check_grid(int n) {
    if (n < 8 || n > 512 || (n & (n - 1)))
        raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
}
hzlb_solvers &solvers(hzlb_solvers *h) {
    if (!h || !h->e)
        raise(HZLB_EINVAL, "null solver handle");
    return *h;
}
// latent forcing of member m over the whole spectrum (the pair's first index, its conjugate at
// the partner)
std::vector<cd> full_forcing(RefEnsemble &e, int m) {
    const int n = e.n;
    std::vector<cd> f(static_cast<size_t>(n) * n, cd(0, 0));
    const auto &modes = e.bank.modes();
    const size_t P = modes.size();
    for (size_t k = 0; k < P; ++k) {
        const int x = (modes[k].first + n) % n, y = (modes[k].second + n) % n;
        const cd v = e.bank.values()[static_cast<size_t>(m) * P + k];
        f[static_cast<size_t>(y) * n + x] = v;
        f[static_cast<size_t>((n - y) % n) * n + (n - x) % n] = std::conj(v);
    }
    return f;
}
} // namespace

extern "C" {

HZLB_API int hzlb_solvers_create(int n, const hzlb_parameters *params, const uint64_t *seeds,
                                 uint64_t count, const char *initial, int precision, int device,
                                 hzlb_solvers **out) {
    return guarded_driver([&] {
        if (!out || !seeds)
            raise(HZLB_EINVAL, "null argument");
        *out = nullptr;
        if (count == 0 || count > static_cast<uint64_t>(std::numeric_limits<int>::max()))
            raise(HZLB_EINVAL, "solver count must be positive");
        const Params p = to_params(params);
        check_grid(n);
        validate_params(n, p);
        const std::string name = initial ? initial : "";
        if (name != "taylor-green" && name != "multimode" && name != "zero")
            raise(HZLB_EINVAL, "unknown initial condition");
        auto h = std::make_unique<hzlb_solvers>();
        h->e = std::make_unique<RefEnsemble>(n, p, std::vector<uint64_t>(seeds, seeds + count),
                                             precision, device);
        h->e->set_initial(name.c_str());
        *out = h.release();
    });
}

HZLB_API int hzlb_solvers_load(const char *const *paths, uint64_t count, int precision,
                               int device, hzlb_solvers **out) {
    return guarded_driver([&] {
        if (!out || !paths)
            raise(HZLB_EINVAL, "null argument");
        *out = nullptr;
        if (count == 0 || count > static_cast<uint64_t>(std::numeric_limits<int>::max()))
            raise(HZLB_EINVAL, "solver count must be positive");
        std::vector<Checkpoint> cps;
        cps.reserve(count);
        for (uint64_t i = 0; i < count; ++i) {
            if (!paths[i])
                raise(HZLB_EINVAL, "null path");
            cps.push_back(read_checkpoint(paths[i]));
            const Checkpoint &a = cps.front(), &b = cps.back();
            if (b.n != a.n || b.time != a.time || b.p.nu != a.p.nu || b.p.alpha != a.p.alpha ||
                b.p.sigma != a.p.sigma || b.p.tau != a.p.tau || b.p.kmin != a.p.kmin ||
                b.p.kmax != a.p.kmax)
                raise(HZLB_EINVAL, "checkpoints of one ensemble must share grid, parameters and time");
        }
        const int n = cps[0].n, M = static_cast<int>(count);
        const size_t nn = static_cast<size_t>(n) * n;
        auto h = std::make_unique<hzlb_solvers>();
        h->e = std::make_unique<RefEnsemble>(n, cps[0].p, std::vector<uint64_t>(count, 0),
                                             precision, device);
        RefEnsemble &e = *h->e;
        std::vector<double> spectra(2 * nn * count);
        for (int m = 0; m < M; ++m)
            std::memcpy(spectra.data() + 2 * nn * m, cps[m].omega.data(), sizeof(cd) * nn);
        e.engine->set_state(spectra.data(), 0, M);
        const auto &modes = e.bank.modes();
        const size_t P = modes.size();
        for (int m = 0; m < M; ++m) {
            for (size_t k = 0; k < P; ++k) {
                const int x = (modes[k].first + n) % n, y = (modes[k].second + n) % n;
                e.bank.values()[static_cast<size_t>(m) * P + k] = cps[m].forcing[static_cast<size_t>(y) * n + x];
            }
            e.bank.stream(m) = cps[m].stream;
        }
        h->time = cps[0].time;
        e.engine->set_time(h->time, 0);
        *out = h.release();
    });
}

HZLB_API void hzlb_solvers_destroy(hzlb_solvers *h) { delete h; }

HZLB_API int hzlb_solvers_step(hzlb_solvers *h, double dt, uint64_t steps) {
    return guarded_driver([&] {
        hzlb_solvers &s = solvers(h);
        validate_dt(s.e->n, s.e->p, dt);
        for (uint64_t i = 0; i < steps; ++i) {
            s.e->step(dt);
            s.time += dt;
        }
        s.e->check_status();
    });
}

HZLB_API int hzlb_solvers_diagnostics(hzlb_solvers *h, double *out) {
    return guarded_driver([&] {
        hzlb_solvers &s = solvers(h);
        if (!out)
            raise(HZLB_EINVAL, "null output");
        s.e->upload_current_forcing();
        s.e->engine->diagnostics(out);
    });
}

HZLB_API int hzlb_solvers_coefficients(hzlb_solvers *h, double *omega, double *forcing) {
    return guarded_driver([&] {
        hzlb_solvers &s = solvers(h);
        const size_t nn = static_cast<size_t>(s.e->n) * s.e->n;
        if (omega)
            s.e->engine->get_state(omega, 0, s.e->M);
        if (forcing)
            for (int m = 0; m < s.e->M; ++m) {
                const auto f = full_forcing(*s.e, m);
                std::memcpy(forcing + 2 * nn * m, f.data(), sizeof(cd) * nn);
            }
    });
}

HZLB_API int hzlb_solvers_shape(hzlb_solvers *h, int *n, uint64_t *count) {
    return guarded_driver([&] {
        hzlb_solvers &s = solvers(h);
        if (!n || !count)
            raise(HZLB_EINVAL, "null output");
        *n = s.e->n;
        *count = static_cast<uint64_t>(s.e->M);
    });
}

HZLB_API int hzlb_solvers_save(hzlb_solvers *h, uint64_t member, const char *path) {
    return guarded_driver([&] {
        hzlb_solvers &s = solvers(h);
        if (!path)
            raise(HZLB_EINVAL, "null path");
        if (member >= static_cast<uint64_t>(s.e->M))
            raise(HZLB_EINVAL, "member out of range");
        const int n = s.e->n, m = static_cast<int>(member);
        const size_t nn = static_cast<size_t>(n) * n;
        Checkpoint c;
        c.n = n;
        c.time = s.time;
        c.p = s.e->p;
        c.stream = s.e->bank.stream(m);
        c.omega.resize(nn);
        s.e->engine->get_state(reinterpret_cast<double *>(c.omega.data()), m, 1);
        for (int y = 0; y < n; ++y)   // inactive modes are exactly zero in a Solver
            for (int x = 0; x < n; ++x)
                if (!active_mode(n, x, y))
                    c.omega[static_cast<size_t>(y) * n + x] = cd(0, 0);
        c.forcing = full_forcing(*s.e, m);
        write_checkpoint(path, c);
    });
}

HZLB_API int hzlb_run_ensemble(int n, const hzlb_parameters *params, double dt, uint64_t steps,
                               uint64_t count, uint64_t seed, int precision, int device,
                               double *out) {
    return guarded_driver([&] {
        if (count == 0)
            raise(HZLB_EINVAL, "ensemble count and workers must be positive");
        if (!out)
            raise(HZLB_EINVAL, "null output");
        const Params p = to_params(params);
        if (n < 8 || n > 512 || (n & (n - 1)))
            raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
        validate_params(n, p);
        if (steps)
            validate_dt(n, p, dt);
        RefEnsemble e(n, p, static_cast<int>(count), seed, precision, device);
        e.set_initial("zero");
        for (uint64_t s = 0; s < steps; ++s)
            e.step(dt);
        e.check_status();
        e.upload_current_forcing();
        e.engine->diagnostics(out);
    });
}

// hzl::synthetic_observations(n, dt, steps, every, truth, noise, seed, truth_fields)
// (src/inference.cpp:258-288): one truth member from "multimode" with OU forcing from
// stream_seed(seed, 0), advanced on the device; every `every` steps, 8 point observations at
// x = (j n/8 + 1) mod n, y = (j^2 + 3j + 2) mod n of the physical vorticity plus noise x
// NormalStream(stream_seed(seed, 1)).  With observations NULL only *count and the header are
// filled (a sizing call; nothing runs).
HZLB_API int hzlb_synthetic_observations(int n, const hzlb_parameters *truth, double dt,
                                         uint64_t steps, uint64_t every, double noise,
                                         uint64_t seed, int precision, int device,
                                         hzlb_dataset *header, hzlb_observation *observations,
                                         size_t capacity, size_t *count, double *truth_fields) {
    return guarded_driver([&] {
        if (!header || !count)
            raise(HZLB_EINVAL, "null output");
        if (every == 0 || steps < every || !std::isfinite(noise) || noise <= 0)
            raise(HZLB_EINVAL, "observation experiment requires steps >= every and positive noise");
        const Params p = to_params(truth);
        if (n < 8 || n > 512 || (n & (n - 1)))
            raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
        validate_params(n, p);
        validate_dt(n, p, dt);
        if (n < 16)   // the reference's closing Dataset::validate
            raise(HZLB_EINVAL, "invalid observation dataset");
        const uint64_t groups = steps / every;
        const size_t total = static_cast<size_t>(groups) * 8;
        *count = total;
        if (observations && capacity < total)
            raise(HZLB_EINVAL, "observation buffer too small");
        header->n = n;
        header->dt = dt;
        header->stochastic = p.sigma > 0 ? 1 : 0;
        header->forcing_min = p.kmin;
        header->forcing_max = p.kmax;
        header->count = observations ? total : 0;
        header->observations = observations;
        if (!observations)
            return;
        RefEnsemble e(n, p, std::vector<uint64_t>{stream_seed(seed, 0)}, precision, device);
        e.set_initial("multimode");
        NormalStream random(stream_seed(seed, 1));
        uint32_t xs[8], ys[8];
        for (uint32_t j = 0; j < 8; ++j) {
            xs[j] = static_cast<uint32_t>((j * static_cast<uint32_t>(n) / 8 + 1) % n);
            ys[j] = static_cast<uint32_t>((j * j + 3 * j + 2) % static_cast<uint32_t>(n));
        }
        const size_t nn = static_cast<size_t>(n) * n;
        size_t k = 0, g = 0;
        for (uint64_t step = 1; step <= steps; ++step) {
            e.step(dt);
            if (step % every == 0) {
                e.check_status();
                double values[8];
                e.engine->observe(xs, ys, 8, values);
                if (truth_fields)
                    e.engine->physical(truth_fields + g * nn);
                for (int j = 0; j < 8; ++j)
                    observations[k++] = {step, xs[j], ys[j], values[j] + noise * random(), noise};
                ++g;
            }
        }
        e.check_status();
    });
}

HZLB_API int hzlb_bootstrap_filter(const hzlb_dataset *data, const hzlb_parameters *params,
                                   uint64_t count, uint64_t seed, int retain_states, int precision,
                                   int device, double *log_likelihood, uint64_t *resampling_events,
                                   hzlb_filter_record *records, size_t capacity, size_t *nrecords,
                                   double *mean_vorticity) {
    return guarded_driver([&] {
        if (!log_likelihood || !resampling_events || !nrecords || (capacity && !records))
            raise(HZLB_EINVAL, "null output");
        const Dataset ds = load_dataset(data);
        Params p = to_params(params);
        p.kmin = ds.fmin;
        p.kmax = ds.fmax;
        validate_params(ds.n, p);
        if (count < 2)
            raise(HZLB_EINVAL, "particle filter needs at least two particles");
        validate_dt(ds.n, p, ds.dt);
        const int M = static_cast<int>(count), n = ds.n;
        RefEnsemble e(n, p, M, seed, precision, device);
        e.set_initial("multimode");
        // weights live on the device (uniform 1/M); the resampling uniform is drawn ahead
        // and kept until a resampling consumes it, so the engine's sequence is the reference's
        e.engine->pf_reset(M);
        std::mt19937_64 resampling(stream_seed(seed, std::numeric_limits<uint64_t>::max()));
        bool pending = false;
        double next_u = 0;
        double ll = 0;
        uint64_t events = 0;
        size_t nrec = 0, current = 0, begin = 0, group = 0;
        const size_t nn = static_cast<size_t>(n) * n;
        std::vector<uint32_t> anc(M);
        std::vector<double> mean;
        while (begin < ds.obs.size()) {
            const uint64_t target = ds.obs[begin].step;
            size_t end = begin;
            while (end < ds.obs.size() && ds.obs[end].step == target)
                ++end;
            for (uint64_t s = current; s < target; ++s)
                e.step(ds.dt);
            e.check_status();
            // log-weights, normalisation and (when the ESS falls below M/2 before the last
            // observation time) resampling and the member gather, on the device
            // (filter.cpp:65-112)
            const size_t p_count = end - begin;
            std::vector<uint32_t> xs(p_count), ys(p_count);
            std::vector<double> vals(p_count), sds(p_count);
            for (size_t o = 0; o < p_count; ++o) {
                const auto &ob = ds.obs[begin + o];
                xs[o] = ob.x;
                ys[o] = ob.y;
                vals[o] = ob.value;
                sds[o] = ob.standard_deviation;
            }
            double u = -1;
            if (end < ds.obs.size()) {
                if (!pending) {
                    next_u = static_cast<double>(resampling() >> 11) * 0x1.0p-53;
                    pending = true;
                }
                u = next_u;
            }
            const bool want_mean = retain_states && mean_vorticity && nrec < capacity;
            if (want_mean)
                mean.resize(2 * e.engine->compact_size());
            hzlb_pf_record rec{};
            e.engine->pf_assimilate(xs.data(), ys.data(), vals.data(), sds.data(), p_count, &u,
                                    nullptr, &rec, anc.data(), want_mean ? mean.data() : nullptr);
            if (rec.collapsed) {
                ll = -std::numeric_limits<double>::infinity();
                break;
            }
            ll += rec.increment;
            if (nrec < capacity) {
                records[nrec] = {target, rec.increment, rec.ess, rec.max_weight};
                if (want_mean) {
                    auto full = compact_to_full(n, mean);
                    host_fft2(n, full, true);
                    std::memcpy(mean_vorticity + 2 * nrec * nn, full.data(), sizeof(cd) * nn);
                }
            }
            ++nrec;
            if (rec.resampled) {
                pending = false;
                e.bank.gather(anc);
                for (int i = 0; i < M; ++i)
                    e.bank.reseed(i, stream_seed(seed, (group + 1) * count + i));
                ++events;
            }
            current = target;
            begin = end;
            ++group;
        }
        *log_likelihood = ll;
        *resampling_events = events;
        *nrecords = std::min(nrec, capacity);
    });
}

// particle_log_likelihood / averaged_particle_log_likelihood (filter.cpp:141-165): the prior
// (stochastic_log_prior, :127-140) and stability checks, then `replicates` bootstrap filters
// (one for the plain likelihood) run as one batched ensemble: replicate r is the reference's
// bootstrap_filter(data, decode(q), particles, seed_r) with seed_r = stream_seed(seed, r) for
// the averaged likelihood (seed itself for the plain one) — its members draw their OU forcing
// from stream_seed(seed_r, j), its resampling uniforms from mt19937_64(stream_seed(seed_r,
// 2^64-1)) and its clones are reseeded with stream_seed(seed_r, (g+1) particles + j) — while
// every step and observation of all replicates' members is one launch sequence.
HZLB_API int hzlb_particle_log_likelihood(const hzlb_dataset *data, const double *log_parameters,
                                          uint64_t particles, uint64_t replicates, uint64_t seed,
                                          int averaged, int precision, int device, double *out) {
    return guarded_driver([&] {
        if (!data || !log_parameters || !out)
            raise(HZLB_EINVAL, "null argument");
        if (averaged && replicates == 0)
            raise(HZLB_EINVAL, "averaged particle likelihood needs at least one replicate");
        const double ninf = -std::numeric_limits<double>::infinity();
        // stochastic_log_prior: only its finiteness matters here
        for (int i = 0; i < 4; ++i) {
            const double q = log_parameters[i];
            if (!std::isfinite(q) || q < -10 || q > (i < 2 ? 0 : 2)) {
                *out = ninf;
                return;
            }
        }
        // decode, then the explicit diffusion bound, both before the dataset is validated
        Params p{std::exp(log_parameters[0]), std::exp(log_parameters[1]),
                 std::exp(log_parameters[2]), std::exp(log_parameters[3]), data->forcing_min,
                 data->forcing_max};
        if (data->n < 0)
            raise(HZLB_EINVAL, "invalid observation dataset");
        const double largest = static_cast<double>((static_cast<uint64_t>(data->n) - 1) / 3);
        if (data->dt * (2 * p.nu * largest * largest + p.alpha) > 2.5) {
            *out = ninf;
            return;
        }
        const Dataset ds = load_dataset(data);
        validate_params(ds.n, p);
        if (particles < 2)
            raise(HZLB_EINVAL, "particle filter needs at least two particles");
        if (particles > (1u << 20) || (averaged && replicates > (1u << 16)) ||
            (averaged ? replicates : 1) * particles > (1u << 22))
            raise(HZLB_EINVAL, "particle count times replicates exceeds the batch limit");
        const int R = averaged ? static_cast<int>(replicates) : 1;
        const int P = static_cast<int>(particles), M = R * P, n = ds.n;
        std::vector<uint64_t> rseed(R), member_seed(M);
        for (int r = 0; r < R; ++r) {
            rseed[r] = averaged ? stream_seed(seed, static_cast<uint64_t>(r)) : seed;
            for (int j = 0; j < P; ++j)
                member_seed[r * P + j] = stream_seed(rseed[r], static_cast<uint64_t>(j));
        }
        RefEnsemble e(n, p, member_seed, precision, device);
        e.set_initial("multimode");
        // R segments of P particles, weights on the device; each replicate's resampling
        // uniform is drawn ahead and kept until its segment resamples
        e.engine->pf_reset(P);
        std::vector<double> ll(R, 0.0), u(R, -1.0), next_u(R, 0.0);
        std::vector<uint8_t> active(R, 1), pending(R, 0);
        std::vector<hzlb_pf_record> recs(R);
        std::vector<uint32_t> anc(M);
        std::vector<std::mt19937_64> resampling;
        for (int r = 0; r < R; ++r)
            resampling.emplace_back(stream_seed(rseed[r], std::numeric_limits<uint64_t>::max()));
        size_t current = 0, begin = 0, group = 0;
        while (begin < ds.obs.size()) {
            const uint64_t target = ds.obs[begin].step;
            size_t end = begin;
            while (end < ds.obs.size() && ds.obs[end].step == target)
                ++end;
            for (uint64_t s = current; s < target; ++s)
                e.step(ds.dt);
            e.check_status();
            const size_t pc = end - begin;
            std::vector<uint32_t> xs(pc), ys(pc);
            std::vector<double> vals(pc), sds(pc);
            for (size_t o = 0; o < pc; ++o) {
                const auto &ob = ds.obs[begin + o];
                xs[o] = ob.x;
                ys[o] = ob.y;
                vals[o] = ob.value;
                sds[o] = ob.standard_deviation;
            }
            const bool may_resample = end < ds.obs.size();
            for (int r = 0; r < R; ++r) {
                u[r] = -1;
                if (active[r] && may_resample) {
                    if (!pending[r]) {
                        next_u[r] = static_cast<double>(resampling[r]() >> 11) * 0x1.0p-53;
                        pending[r] = 1;
                    }
                    u[r] = next_u[r];
                }
            }
            e.engine->pf_assimilate(xs.data(), ys.data(), vals.data(), sds.data(), pc, u.data(),
                                    active.data(), recs.data(), anc.data(), nullptr);
            std::vector<int> resampled_replicates, retired;
            for (int r = 0; r < R; ++r) {
                if (!active[r])
                    continue;
                if (recs[r].collapsed) {
                    ll[r] = ninf;
                    active[r] = 0;
                    retired.push_back(r);
                    continue;
                }
                ll[r] += recs[r].increment;
                if (recs[r].resampled) {
                    pending[r] = 0;
                    resampled_replicates.push_back(r);
                }
            }
            const auto live = std::find(active.begin(), active.end(), 1);
            if (live == active.end())
                break;
            // a replicate that has ended stops being weighted; its members are overwritten by
            // a copy of a live member so that they stay finite while the others advance
            // (the resampled segments were gathered on the device already)
            if (!retired.empty()) {
                const uint32_t source = static_cast<uint32_t>((live - active.begin()) * P);
                std::vector<uint32_t> patch(M);
                for (int i = 0; i < M; ++i)
                    patch[i] = static_cast<uint32_t>(i);
                for (int r : retired)
                    for (int j = 0; j < P; ++j)
                        anc[r * P + j] = patch[r * P + j] = source;
                e.engine->gather(patch.data());
            }
            if (!resampled_replicates.empty() || !retired.empty()) {
                e.bank.gather(anc);
                for (int r : resampled_replicates)
                    for (int j = 0; j < P; ++j)
                        e.bank.reseed(r * P + j,
                                      stream_seed(rseed[r], (group + 1) * particles + static_cast<uint64_t>(j)));
            }
            current = target;
            begin = end;
            ++group;
        }
        if (!averaged) {
            *out = ll[0];
            return;
        }
        const double maximum = *std::max_element(ll.begin(), ll.end());
        if (!std::isfinite(maximum)) {
            *out = ninf;
            return;
        }
        double total = 0;
        for (double v : ll)
            total += std::exp(v - maximum);
        *out = maximum + std::log(total / static_cast<double>(R));
    });
}

HZLB_API int hzlb_ensemble_kalman_filter(const hzlb_dataset *data, const hzlb_parameters *params,
                                         uint64_t count, uint64_t seed,
                                         const hzlb_enkf_options *options, int precision,
                                         int device, hzlb_enkf_record *records, size_t capacity,
                                         size_t *nrecords, double *mean_vorticity) {
    return guarded_driver([&] {
        if (!nrecords || (capacity && !records))
            raise(HZLB_EINVAL, "null output");
        const Dataset ds = load_dataset(data);
        const hzlb_enkf_options opt = options ? *options : hzlb_enkf_options{1.0, 0.0, 0, 1};
        if (count < 2)
            raise(HZLB_EINVAL, "EnKF requires at least two ensemble members");
        if (!std::isfinite(opt.inflation) || opt.inflation < 1 ||
            !std::isfinite(opt.localization_radius) || opt.localization_radius < 0)
            raise(HZLB_EINVAL, "EnKF inflation must be >= 1 and localization radius nonnegative");
        if (opt.forecast_every == 0)
            raise(HZLB_EINVAL, "EnKF forecast output interval must be positive");
        Params p = to_params(params);
        p.kmin = ds.fmin;
        p.kmax = ds.fmax;
        validate_params(ds.n, p);
        validate_dt(ds.n, p, ds.dt);
        const int M = static_cast<int>(count), n = ds.n;
        const size_t nn = static_cast<size_t>(n) * n;
        RefEnsemble e(n, p, M, seed, precision, device);
        e.set_initial("multimode");
        NormalStream perturbations(stream_seed(seed, count));
        size_t nrec = 0;
        auto emit = [&](uint64_t step, double rmse, double spread, bool forecast) {
            if (nrec < capacity) {
                records[nrec] = {step, rmse, spread, forecast ? 1 : 0};
                if (mean_vorticity) {
                    auto full = compact_to_full(n, e.mean());
                    host_fft2(n, full, true);
                    std::memcpy(mean_vorticity + 2 * nrec * nn, full.data(), sizeof(cd) * nn);
                }
            }
            ++nrec;
        };
        auto spread = [&]() {
            const auto mean = e.mean();
            return std::sqrt(e.engine->spread(mean.data()) / static_cast<double>(M - 1));
        };
        auto& vals = e.bank.values();
        const size_t P = e.bank.pairs();
        uint64_t step = 0;
        size_t begin = 0;
        while (begin < ds.obs.size()) {
            const uint64_t target = ds.obs[begin].step;
            size_t end = begin;
            while (end < ds.obs.size() && ds.obs[end].step == target)
                ++end;
            for (uint64_t s = step; s < target; ++s)
                e.step(ds.dt);
            e.check_status();
            if (opt.inflation > 1) {   // filter.cpp:237-253
                e.engine->inflate(opt.inflation);
                e.engine->symmetrize();
                for (size_t k = 0; k < P; ++k) {
                    cd mean(0, 0);
                    for (int m = 0; m < M; ++m)
                        mean += vals[m * P + k] / static_cast<double>(M);
                    for (int m = 0; m < M; ++m)
                        vals[m * P + k] = mean + opt.inflation * (vals[m * P + k] - mean);
                }
            }
            // forecast sensor RMSE from the mean state, before any update (filter.cpp:254-264)
            double forecast_error = 0;
            {
                auto full = compact_to_full(n, e.mean());
                host_fft2(n, full, true);
                for (size_t o = begin; o < end; ++o) {
                    const double d = full[static_cast<size_t>(ds.obs[o].y) * n + ds.obs[o].x].real() -
                                     ds.obs[o].value;
                    forecast_error += d * d;
                }
            }
            for (size_t o = begin; o < end; ++o) {   // serial scalar updates (filter.cpp:265-321)
                const auto &ob = ds.obs[o];
                std::vector<double> pred(M);
                e.engine->observe(&ob.x, &ob.y, 1, pred.data());
                double mean_prediction = 0;
                for (int i = 0; i < M; ++i)
                    mean_prediction += pred[i] / static_cast<double>(M);
                double variance = 0;
                std::vector<double> d(M);
                for (int i = 0; i < M; ++i) {
                    const double delta = pred[i] - mean_prediction;
                    variance += delta * delta / static_cast<double>(M - 1);
                    d[i] = delta / static_cast<double>(M - 1);
                }
                // forcing cross-covariance on the host (shell pairs only)
                std::vector<cd> fcov(P, cd(0, 0));
                for (size_t k = 0; k < P; ++k) {
                    cd mean(0, 0);
                    for (int m = 0; m < M; ++m)
                        mean += vals[m * P + k] / static_cast<double>(M);
                    for (int m = 0; m < M; ++m)
                        fcov[k] += (vals[m * P + k] - mean) * d[m];
                }
                std::vector<double> cov;
                if (opt.localization_radius > 0) {
                    cov.resize(2 * e.engine->compact_size());
                    e.engine->covariance(d.data(), cov.data());
                    // Gaspari-Cohn taper in physical space (filter.cpp:25-36, 290-308)
                    auto full = compact_to_full(n, cov);
                    host_fft2(n, full, true);
                    std::vector<cd> ffull(nn, cd(0, 0));
                    for (size_t k = 0; k < P; ++k) {
                        const auto [kx, ky] = e.bank.modes()[k];
                        const int x = (kx + n) % n, y = (ky + n) % n;
                        ffull[static_cast<size_t>(y) * n + x] = fcov[k];
                        ffull[static_cast<size_t>((n - y) % n) * n + (n - x) % n] = std::conj(fcov[k]);
                    }
                    host_fft2(n, ffull, true);
                    const double radius = opt.localization_radius;
                    auto gc = [&](double dist) {
                        const double x = dist / radius;
                        if (x >= 2)
                            return 0.0;
                        if (x <= 1)
                            return 1 - 5.0 / 3 * x * x + 5.0 / 8 * x * x * x + 0.5 * std::pow(x, 4) -
                                   0.25 * std::pow(x, 5);
                        return 4 - 5 * x + 5.0 / 3 * x * x + 5.0 / 8 * x * x * x - 0.5 * std::pow(x, 4) +
                               std::pow(x, 5) / 12 - 2.0 / (3 * x);
                    };
                    for (int y = 0; y < n; ++y)
                        for (int x = 0; x < n; ++x) {
                            const int ax = std::abs(x - static_cast<int>(ob.x)),
                                      ay = std::abs(y - static_cast<int>(ob.y));
                            const double dx = std::min(ax, n - ax), dy = std::min(ay, n - ay);
                            const double taper = gc(std::hypot(dx, dy));
                            full[static_cast<size_t>(y) * n + x] *= taper;
                            ffull[static_cast<size_t>(y) * n + x] *= taper;
                        }
                    host_fft2(n, full, false);
                    host_fft2(n, ffull, false);
                    // update_latent_state averages each pair with its conjugate partner
                    for (int y = 0; y < n; ++y)
                        for (int x = 1; x < n / 2; ++x) {
                            const size_t i = static_cast<size_t>(y) * n + x,
                                         j = static_cast<size_t>((n - y) % n) * n + (n - x);
                            full[i] = 0.5 * (full[i] + std::conj(full[j]));
                        }
                    cov = full_to_compact(n, full);
                    // forcing: restricted to the shell pairs and symmetrised by update_latent_state
                    for (size_t k = 0; k < P; ++k) {
                        const auto [kx, ky] = e.bank.modes()[k];
                        const int x = (kx + n) % n, y = (ky + n) % n;
                        const cd a = ffull[static_cast<size_t>(y) * n + x],
                                 b = ffull[static_cast<size_t>((n - y) % n) * n + (n - x) % n];
                        fcov[k] = 0.5 * (a + std::conj(b));
                    }
                } else {
                    e.engine->covariance(d.data(), nullptr);
                }
                const double denominator = variance + ob.standard_deviation * ob.standard_deviation;
                std::vector<double> innov(M);
                for (int i = 0; i < M; ++i)
                    innov[i] = (ob.value + ob.standard_deviation * perturbations() - pred[i]) / denominator;
                e.engine->rank1(cov.empty() ? nullptr : cov.data(), innov.data());
                e.engine->symmetrize();
                // forcing update, then update_latent_state's pair symmetrisation
                for (int m = 0; m < M; ++m)
                    for (size_t k = 0; k < P; ++k)
                        vals[m * P + k] += fcov[k] * innov[m];
            }
            emit(target, std::sqrt(forecast_error / static_cast<double>(end - begin)), spread(), false);
            step = target;
            begin = end;
        }
        for (uint64_t h = 1; h <= opt.forecast_steps; ++h) {   // filter.cpp:337-354
            e.step(ds.dt);
            if (h % opt.forecast_every != 0 && h != opt.forecast_steps)
                continue;
            e.check_status();
            emit(step + h, std::numeric_limits<double>::quiet_NaN(), spread(), true);
        }
        *nrecords = std::min(nrec, capacity);
    });
}

} // extern "C"
