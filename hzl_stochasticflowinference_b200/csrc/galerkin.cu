// The reference's Galerkin reduced model (GalerkinModel, src/reduced.cpp:137-209) built on the
// device: da/dt = c + A a + Q(a, a) in the coefficients of a POD basis, with
//   c_i    = <m_i, D(mean)>,
//   A_ij   = <m_i, D'(mean) m_j>,
//   Q_ijj  = <m_i, D(m_j) + (nu k^2 + alpha) m_j>,
//   Q_ijk  = Q_ikj = <m_i, (D(m_j + m_k) - D(m_j) - D(m_k)) / 2>   (k < j),
// D the full model's deterministic drift -N - (nu k^2 + alpha) w (Solver::drift, which leaves
// the forcing out), <.,.> the reference's spectral_inner.  Every drift is evaluated by the
// batched spectral kernels in one FP64 ensemble whose members are the needed fields (the
// stage-1 derivative of the RK step); the tangent D'(mean) m_j is the symmetric difference
// (D(mean + m_j) - D(mean - m_j)) / 2, exact for the quadratic drift.  The projections are one
// FP64 device product.  The reduced RHS and its RK4 step run in FP64, one block per state,
// summing in the reference's order.
#include "dense64.cuh"
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

namespace hzlb {
namespace {

// out[s][i] = c_i + sum_j (A_ij a_j + sum_k Q_ijk a_j a_k) for state s (reduced.cpp:182-192)
__global__ void galerkin_rhs(const double *c, const double *A, const double *Q, int r,
                             const double *a, int count, double *out) {
    extern __shared__ double sa[];
    for (int s = blockIdx.x; s < count; s += gridDim.x) {
        __syncthreads();
        for (int j = threadIdx.x; j < r; j += blockDim.x)
            sa[j] = a[static_cast<long long>(s) * r + j];
        __syncthreads();
        for (int i = threadIdx.x; i < r; i += blockDim.x) {
            double v = c[i];
            for (int j = 0; j < r; ++j) {
                v += A[i * r + j] * sa[j];
                const double *q = Q + (static_cast<long long>(i) * r + j) * r;
                for (int k = 0; k < r; ++k)
                    v += q[k] * sa[j] * sa[k];
            }
            out[static_cast<long long>(s) * r + i] = v;
        }
    }
}
// y = a + h k (elementwise)
__global__ void axpy_states(const double *a, const double *k, double h, long long n, double *y) {
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        y[i] = a[i] + h * k[i];
}
// a += dt/6 (k1 + 2 k2 + 2 k3 + k4), flagging nonfinite results (reduced.cpp:193-209)
__global__ void rk4_finish(double *a, const double *k1, const double *k2, const double *k3,
                           const double *k4, double dt, long long n, int *bad) {
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double v = a[i] + dt / 6 * (k1[i] + 2 * k2[i] + 2 * k3[i] + k4[i]);
        a[i] = v;
        if (!isfinite(v))
            *bad = 1;
    }
}

} // namespace

class Galerkin {
  public:
    Galerkin(int n, const hzlb_parameters &p, const double *mean, const double *modes, int r,
             int device)
        : n_(n), r_(r), device_(device) {
        if (r < 1 || !mean || !modes)
            raise(HZLB_EINVAL, "invalid Galerkin basis");
        if (p.forcing_sigma != 0)
            raise(HZLB_EINVAL, "Galerkin prototype currently models deterministic drift only");
        if (n < 8 || n > 512 || (n & (n - 1)))
            raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
        const int K = (n - 1) / 3, C = K + 1, LD = 2 * K + 1;
        const size_t E = static_cast<size_t>(C) * LD;   // complex entries per compact field
        // compact copies of the mean and the modes (the basis is of real fields: the
        // kx < 0 half of the full spectrum is the conjugate of the stored half)
        auto compact = [&](const double *full, double *out) {
            for (int kx = 0; kx < C; ++kx)
                for (int j = 0; j < LD; ++j) {
                    const int y = j <= K ? j : n - LD + j;
                    const double *z = full + 2 * (static_cast<size_t>(y) * n + kx);
                    out[2 * (static_cast<size_t>(kx) * LD + j)] = z[0];
                    out[2 * (static_cast<size_t>(kx) * LD + j) + 1] = z[1];
                }
            out[0] = out[1] = 0;   // the mean mode is outside the retained set
        };
        std::vector<double> m(2 * E), U(2 * E * r);
        compact(mean, m.data());
        for (int j = 0; j < r; ++j)
            compact(modes + 2 * static_cast<size_t>(j) * n * n, U.data() + 2 * E * j);
        // fields whose drift is needed: mean, m_j, mean + m_j, mean - m_j, m_j + m_k (k < j)
        const int F = 1 + 3 * r + r * (r - 1) / 2;
        std::vector<double> fields(2 * E * static_cast<size_t>(F));
        auto put = [&](int f, const double *x, double ax, const double *y, double ay) {
            double *o = fields.data() + 2 * E * f;
            for (size_t e = 0; e < 2 * E; ++e)
                o[e] = ax * x[e] + (y ? ay * y[e] : 0.0);
        };
        auto mode = [&](int j) { return U.data() + 2 * E * j; };
        put(0, m.data(), 1, nullptr, 0);
        for (int j = 0; j < r; ++j) {
            put(1 + j, mode(j), 1, nullptr, 0);
            put(1 + r + j, m.data(), 1, mode(j), 1);
            put(1 + 2 * r + j, m.data(), 1, mode(j), -1);
        }
        std::vector<int> pair_index(static_cast<size_t>(r) * r, -1);
        int f = 1 + 3 * r;
        for (int j = 0; j < r; ++j)
            for (int k = 0; k < j; ++k) {
                put(f, mode(j), 1, mode(k), 1);
                pair_index[static_cast<size_t>(j) * r + k] = f++;
            }
        // drifts of all fields in one FP64 ensemble without forcing or noise
        hzlb_config cfg{};
        cfg.n = n;
        cfg.members = F;
        cfg.precision = 8;
        cfg.nu = p.viscosity;
        cfg.alpha = p.friction;
        cfg.forcing_kmax = -1;
        cfg.noise_sigma = 0;
        cfg.noise_kmax = 1;
        cfg.device = device;
        auto engine = make_engine(cfg);
        engine->set_state_compact(fields.data(), 0, F);
        DeviceBuffer drifts, wm, proj;
        drifts.ensure(sizeof(double) * 2 * E * F, "allocate drifts");
        engine->drift(drifts.ptr);
        engine.reset();
        // P[i][f] = <m_i, D(field f)>: the reference's spectral_inner over the full spectrum,
        // which for real fields weighs the kx > 0 columns twice
        std::vector<double> w(2 * E * r);
        for (int j = 0; j < r; ++j)
            for (size_t e = 0; e < 2 * E; ++e)
                w[2 * E * j + e] = mode(j)[e] * ((e / 2) / LD > 0 ? 2.0 : 1.0);
        cuda_check(cudaSetDevice(device), "select CUDA device");
        wm.ensure(sizeof(double) * w.size(), "allocate weighted modes");
        cuda_check(cudaMemcpy(wm.ptr, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice),
                   "upload modes");
        proj.ensure(sizeof(double) * static_cast<size_t>(r) * F, "allocate projections");
        const long long D = static_cast<long long>(2 * E);
        cuda_check(d64::gemm(d64::GemmArgs{r, F, static_cast<int>(D), 1.0, 0.0, wm.as<double>(), D, 1,
                                           drifts.as<double>(), 1, D, proj.as<double>(), F},
                             nullptr),
                   "launch Galerkin projections");
        std::vector<double> P(static_cast<size_t>(r) * F);
        cuda_check(cudaMemcpy(P.data(), proj.ptr, sizeof(double) * P.size(), cudaMemcpyDeviceToHost),
                   "download projections");
        auto at = [&](int i, int fi) { return P[static_cast<size_t>(i) * F + fi]; };
        // <m_i, (nu k^2 + alpha) m_j> for the diagonal quadratic terms
        std::vector<double> damp(static_cast<size_t>(r) * r, 0.0);
        for (int kx = 0; kx < C; ++kx)
            for (int jj = 0; jj < LD; ++jj) {
                const int ky = jj <= K ? jj : jj - LD;
                const double rate = p.viscosity * (kx * kx + ky * ky) + p.friction;
                const double weight = (kx > 0 ? 2.0 : 1.0) * rate;
                const size_t e = 2 * (static_cast<size_t>(kx) * LD + jj);
                for (int i = 0; i < r; ++i)
                    for (int j = 0; j < r; ++j)
                        damp[static_cast<size_t>(i) * r + j] +=
                            weight * (mode(i)[e] * mode(j)[e] + mode(i)[e + 1] * mode(j)[e + 1]);
            }
        c_.assign(r, 0.0);
        A_.assign(static_cast<size_t>(r) * r, 0.0);
        Q_.assign(static_cast<size_t>(r) * r * r, 0.0);
        for (int i = 0; i < r; ++i) {
            c_[i] = at(i, 0);
            for (int j = 0; j < r; ++j) {
                A_[static_cast<size_t>(i) * r + j] = 0.5 * (at(i, 1 + r + j) - at(i, 1 + 2 * r + j));
                Q_[(static_cast<size_t>(i) * r + j) * r + j] = at(i, 1 + j) + damp[static_cast<size_t>(i) * r + j];
                for (int k = 0; k < j; ++k) {
                    const double v =
                        0.5 * (at(i, pair_index[static_cast<size_t>(j) * r + k]) - at(i, 1 + j) - at(i, 1 + k));
                    Q_[(static_cast<size_t>(i) * r + j) * r + k] = v;
                    Q_[(static_cast<size_t>(i) * r + k) * r + j] = v;
                }
            }
        }
        coef_.ensure(sizeof(double) * (c_.size() + A_.size() + Q_.size()), "allocate Galerkin tensors");
        double *d = coef_.as<double>();
        cuda_check(cudaMemcpy(d, c_.data(), sizeof(double) * r, cudaMemcpyHostToDevice), "upload c");
        cuda_check(cudaMemcpy(d + r, A_.data(), sizeof(double) * A_.size(), cudaMemcpyHostToDevice),
                   "upload A");
        cuda_check(cudaMemcpy(d + r + A_.size(), Q_.data(), sizeof(double) * Q_.size(),
                              cudaMemcpyHostToDevice),
                   "upload Q");
    }
    int rank() const { return r_; }
    void coefficients(double *c, double *A, double *Q) const {
        if (c)
            std::memcpy(c, c_.data(), sizeof(double) * c_.size());
        if (A)
            std::memcpy(A, A_.data(), sizeof(double) * A_.size());
        if (Q)
            std::memcpy(Q, Q_.data(), sizeof(double) * Q_.size());
    }
    // host arrays: a, out are count x r
    void rhs(const double *a, size_t count, double *out) {
        prepare(count);
        cuda_check(cudaMemcpy(work_.as<double>(), a, sizeof(double) * count * r_, cudaMemcpyHostToDevice),
                   "upload coefficients");
        launch_rhs(work_.as<double>(), count, work_.as<double>() + count * r_);
        cuda_check(cudaMemcpy(out, work_.as<double>() + count * r_, sizeof(double) * count * r_,
                              cudaMemcpyDeviceToHost),
                   "download right-hand sides");
    }
    void step(double *a, size_t count, double dt, uint64_t nsteps) {
        if (!std::isfinite(dt) || dt <= 0)
            raise(HZLB_EINVAL, "invalid Galerkin time step");
        prepare(count);
        const size_t n = count * r_;
        double *x = work_.as<double>(), *y = x + n, *k1 = y + n, *k2 = k1 + n, *k3 = k2 + n,
               *k4 = k3 + n;
        int *bad = reinterpret_cast<int *>(k4 + n);
        cuda_check(cudaMemcpy(x, a, sizeof(double) * n, cudaMemcpyHostToDevice), "upload coefficients");
        cuda_check(cudaMemset(bad, 0, sizeof(int)), "clear flag");
        const int blocks = static_cast<int>(std::min<size_t>((n + 255) / 256, 1024));
        for (uint64_t s = 0; s < nsteps; ++s) {
            launch_rhs(x, count, k1);
            axpy_states<<<blocks, 256>>>(x, k1, dt / 2, static_cast<long long>(n), y);
            launch_rhs(y, count, k2);
            axpy_states<<<blocks, 256>>>(x, k2, dt / 2, static_cast<long long>(n), y);
            launch_rhs(y, count, k3);
            axpy_states<<<blocks, 256>>>(x, k3, dt, static_cast<long long>(n), y);
            launch_rhs(y, count, k4);
            rk4_finish<<<blocks, 256>>>(x, k1, k2, k3, k4, dt, static_cast<long long>(n), bad);
        }
        cuda_check(cudaGetLastError(), "launch Galerkin steps");
        int host_bad = 0;
        cuda_check(cudaMemcpy(&host_bad, bad, sizeof(int), cudaMemcpyDeviceToHost), "read flag");
        cuda_check(cudaMemcpy(a, x, sizeof(double) * n, cudaMemcpyDeviceToHost), "download coefficients");
        if (host_bad)
            raise(HZLB_ERUNTIME, "unstable Galerkin trajectory");
    }

  private:
    void prepare(size_t count) {
        if (count == 0)
            raise(HZLB_EINVAL, "no states");
        cuda_check(cudaSetDevice(device_), "select CUDA device");
        work_.ensure(sizeof(double) * 6 * count * r_ + 16, "allocate Galerkin workspace");
    }
    void launch_rhs(const double *a, size_t count, double *out) {
        const double *d = coef_.as<double>();
        const int threads = std::min(256, std::max(32, (r_ + 31) / 32 * 32));
        const int blocks = static_cast<int>(std::min<size_t>(count, 4096));
        galerkin_rhs<<<blocks, threads, sizeof(double) * r_>>>(d, d + r_, d + r_ + static_cast<size_t>(r_) * r_,
                                                             r_, a, static_cast<int>(count), out);
        cuda_check(cudaGetLastError(), "launch Galerkin right-hand side");
    }

    int n_, r_, device_;
    std::vector<double> c_, A_, Q_;
    DeviceBuffer coef_, work_;
};

} // namespace hzlb

struct hzlb_galerkin {
    std::unique_ptr<hzlb::Galerkin> g;
};

namespace {
template <class F> int guarded_galerkin(F &&f) {
    try {
        f();
        return HZLB_OK;
    } catch (const hzlb::Error &e) {
        hzlb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception &e) {
        hzlb::set_last_error(e.what());
        return HZLB_ERUNTIME;
    }
}
hzlb::Galerkin &galerkin(hzlb_galerkin *h) {
    if (!h || !h->g)
        hzlb::raise(HZLB_EINVAL, "null Galerkin handle");
    return *h->g;
}
} // namespace

extern "C" {
HZLB_API int hzlb_galerkin_create(int n, const hzlb_parameters *p, const double *mean,
                                  const double *modes, size_t rank, int device,
                                  hzlb_galerkin **out) {
    return guarded_galerkin([&] {
        if (!p || !out)
            hzlb::raise(HZLB_EINVAL, "null argument");
        auto h = std::make_unique<hzlb_galerkin>();
        h->g = std::make_unique<hzlb::Galerkin>(n, *p, mean, modes, static_cast<int>(rank), device);
        *out = h.release();
    });
}
HZLB_API void hzlb_galerkin_destroy(hzlb_galerkin *h) { delete h; }
HZLB_API int hzlb_galerkin_coefficients(hzlb_galerkin *h, double *constant, double *linear,
                                        double *quadratic) {
    return guarded_galerkin([&] { galerkin(h).coefficients(constant, linear, quadratic); });
}
HZLB_API int hzlb_galerkin_rhs(hzlb_galerkin *h, const double *coefficients, size_t count,
                               double *out) {
    return guarded_galerkin([&] {
        if (!coefficients || !out)
            hzlb::raise(HZLB_EINVAL, "null argument");
        galerkin(h).rhs(coefficients, count, out);
    });
}
HZLB_API int hzlb_galerkin_step(hzlb_galerkin *h, double *coefficients, size_t count, double dt,
                                uint64_t nsteps) {
    return guarded_galerkin([&] {
        if (!coefficients)
            hzlb::raise(HZLB_EINVAL, "null argument");
        galerkin(h).step(coefficients, count, dt, nsteps);
    });
}
} // extern "C"
