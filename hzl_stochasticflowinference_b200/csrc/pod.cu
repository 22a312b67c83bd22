// Proper orthogonal decomposition of vorticity snapshots on the device, and the learned
// reduced forecast built on it.
//
// Two fits share one eigensolver (a cyclic Jacobi restated from the reference's fit_pod,
// reduced.cpp:66-101, so that eigenvectors come out with the same signs):
//
// * hzlb_fit_pod: the reference's fit_pod (reduced.cpp:36-136) on full complex spectra in
//   FP64: snapshot mean, Gram matrix Re sum conj(a) b of the centred snapshots (FP64 GEMM on
//   the device), Jacobi eigenpairs, modes X^T v / sqrt(lambda) (device), and the reference's
//   two Gram-Schmidt passes and normalisation, done here as two Cholesky QR passes (the same
//   orthonormal factor), with its degenerate-mode check and truncation rules.
//
// * hzlb_pod_fit: snapshots of an FP32 ensemble in the compact dealiased layout, beyond the
//   reference's 512-snapshot cap.  The inner product is the reference's spectral_inner over
//   the full spectrum, which for real fields weighs the kx > 0 columns twice; the snapshots
//   are centred and scaled by w = sqrt(2) on those columns so it becomes a plain dot product.
//   The Gram matrix is a 3xTF32 product on the tcgen05 tensor cores; its leading eigenpairs
//   come from subspace iteration (FP64 device GEMMs, Cholesky QR with host factorisations)
//   and a Rayleigh-Ritz step through the Jacobi solver; modes as above.  The handle then
//   projects ensemble states onto the modes and adds mode combinations back (split-K and
//   plain 3xTF32 tensor-core products), which is what the learned forecast needs.
#include "dense64.cuh"
#include "engine.h"
#include "umma_gemm.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <numeric>
#include <random>
#include <string>
#include <vector>

namespace hzlb {
namespace {

constexpr double kSqrt2 = 1.4142135623730950488;

// ---- host dense helpers ------------------------------------------------------------------
// Cyclic Jacobi on the symmetric m x m matrix a (row-major): sweeps over p < q, rotations
// skipped below 1e-14 * scale, converged when every off-diagonal entry of a sweep is below
// 1e-12 * scale (the reference's rules, reduced.cpp:66-101).  On return a's diagonal holds
// the eigenvalues and column c of v the eigenvector of a[c][c].
bool jacobi(std::vector<double> &a, std::vector<double> &v, size_t m, double scale) {
    v.assign(m * m, 0.0);
    for (size_t i = 0; i < m; ++i)
        v[i * m + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double largest = 0;
        for (size_t p = 0; p < m; ++p)
            for (size_t q = p + 1; q < m; ++q) {
                const double apq = a[p * m + q];
                largest = std::max(largest, std::abs(apq));
                if (std::abs(apq) < 1e-14 * scale)
                    continue;
                const double theta = (a[q * m + q] - a[p * m + p]) / (2 * apq);
                const double t = std::copysign(1.0, theta) / (std::abs(theta) + std::hypot(1.0, theta));
                const double c = 1 / std::sqrt(1 + t * t), s = t * c;
                const double app = a[p * m + p], aqq = a[q * m + q];
                a[p * m + p] = app - t * apq;
                a[q * m + q] = aqq + t * apq;
                a[p * m + q] = a[q * m + p] = 0;
                for (size_t k = 0; k < m; ++k) {
                    if (k != p && k != q) {
                        const double x = a[k * m + p], y = a[k * m + q];
                        a[k * m + p] = a[p * m + k] = c * x - s * y;
                        a[k * m + q] = a[q * m + k] = s * x + c * y;
                    }
                    const double x = v[k * m + p], y = v[k * m + q];
                    v[k * m + p] = c * x - s * y;
                    v[k * m + q] = s * x + c * y;
                }
            }
        if (largest < 1e-12 * scale)
            return true;
    }
    return false;
}
// Eigenvalue order, largest first.
std::vector<size_t> descending(const std::vector<double> &a, size_t m) {
    std::vector<size_t> order(m);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](size_t i, size_t j) { return a[i * m + i] > a[j * m + j]; });
    return order;
}
// In-place lower Cholesky of the k x k matrix b; returns the smallest pivot (<= 0 on failure).
double cholesky_host(std::vector<double> &b, size_t k) {
    double smallest = INFINITY;
    for (size_t j = 0; j < k; ++j) {
        double d = b[j * k + j];
        for (size_t l = 0; l < j; ++l)
            d -= b[j * k + l] * b[j * k + l];
        if (!(d > 0))
            return d == d ? d : -1.0;   // nonpositive (or NaN) pivot
        const double piv = std::sqrt(d);
        smallest = std::min(smallest, piv);
        b[j * k + j] = piv;
        for (size_t i = j + 1; i < k; ++i) {
            double s = b[i * k + j];
            for (size_t l = 0; l < j; ++l)
                s -= b[i * k + l] * b[j * k + l];
            b[i * k + j] = s / piv;
        }
        for (size_t l = j + 1; l < k; ++l)
            b[j * k + l] = 0;
    }
    return smallest;
}
// Orthonormalise the k columns of the m x k row-major matrix y in place (two Gram-Schmidt
// passes per column); a column that loses almost all of its norm is replaced by a random one.
void gram_schmidt_host(std::vector<double> &y, size_t m, size_t k, std::mt19937_64 &rng) {
    std::normal_distribution<double> nd;
    auto col_norm = [&](size_t j) {
        double s = 0;
        for (size_t i = 0; i < m; ++i)
            s += y[i * k + j] * y[i * k + j];
        return std::sqrt(s);
    };
    for (size_t j = 0; j < k; ++j) {
        for (int attempt = 0; attempt < 8; ++attempt) {
            const double before = col_norm(j);
            for (int pass = 0; pass < 2; ++pass)
                for (size_t l = 0; l < j; ++l) {
                    double d = 0;
                    for (size_t i = 0; i < m; ++i)
                        d += y[i * k + l] * y[i * k + j];
                    for (size_t i = 0; i < m; ++i)
                        y[i * k + j] -= d * y[i * k + l];
                }
            const double after = col_norm(j);
            if (after > 1e-10 * before && after > 0) {
                for (size_t i = 0; i < m; ++i)
                    y[i * k + j] /= after;
                break;
            }
            for (size_t i = 0; i < m; ++i)
                y[i * k + j] = nd(rng);
        }
    }
}
// Inverse of a lower-triangular k x k matrix.
std::vector<double> lower_inverse(const std::vector<double> &L, size_t k) {
    std::vector<double> X(k * k, 0.0);
    for (size_t c = 0; c < k; ++c) {
        X[c * k + c] = 1 / L[c * k + c];
        for (size_t i = c + 1; i < k; ++i) {
            double s = 0;
            for (size_t l = c; l < i; ++l)
                s += L[i * k + l] * X[l * k + c];
            X[i * k + c] = -s / L[i * k + i];
        }
    }
    return X;
}

// ---- device kernels ----------------------------------------------------------------------
template <typename T>
__global__ void column_mean(const T *x, long long n, int rows, T *out) {
    __shared__ double part[8][33];
    const long long e = static_cast<long long>(blockIdx.x) * 32 + threadIdx.x;
    double s = 0;
    if (e < n)
        for (int m = threadIdx.y; m < rows; m += 8)
            s += static_cast<double>(x[static_cast<long long>(m) * n + e]);
    part[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && e < n) {
        double t = 0;
        for (int w = 0; w < 8; ++w)
            t += part[w][threadIdx.x];
        out[e] = static_cast<T>(t / rows);
    }
}
__device__ __forceinline__ float tf32_round(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
// Weight of real entry e of a compact member: sqrt(2) on the columns kx > 0, i.e. from
// complex index ld on.
__device__ __forceinline__ double column_weight(long long e, int ld) {
    return (e >> 1) >= ld ? kSqrt2 : 1.0;
}
// c = w (x - mean) for rows x D reals of the compact layout; FP64 copy (optional) and 3xTF32
// split into hi / lo.  Grid: x over the entries of a row, y over rows.
__global__ void center_weight(const float *x, const float *mean, int rows, int D, int ld,
                              double *xd, float *hi, float *lo) {
    for (int row = blockIdx.y; row < rows; row += gridDim.y)
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < D; e += gridDim.x * blockDim.x) {
            const long long i = static_cast<long long>(row) * D + e;
            const double c = column_weight(e, ld) * (static_cast<double>(x[i]) - static_cast<double>(mean[e]));
            if (xd)
                xd[i] = c;
            const float f = static_cast<float>(c), h = tf32_round(f);
            hi[i] = h;
            lo[i] = f - h;
        }
}
dim3 center_grid(int rows, long long D) {
    return dim3(static_cast<unsigned>((D + 255) / 256), static_cast<unsigned>(std::min(rows, 65535)));
}
__global__ void center_double(const double *x, const double *mean, long long rows, long long D,
                              double *out) {
    const long long total = rows * D;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = x[i] - mean[i % D];
}
__global__ void symmetric_to_double(const float *g, int m, double *out) {
    const long long total = static_cast<long long>(m) * m;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long r = i / m, c = i % m;
        out[i] = 0.5 * (static_cast<double>(g[i]) + static_cast<double>(g[c * m + r]));
    }
}
// From the weighted orthonormal modes U (r x D, FP64): the 3xTF32 split of U (projection),
// the unweighted modes U / w as FP32 (r x D), and for the update the transposed unweighted
// modes with the three split terms side by side along K: ut3[e] = (hi[0..r), lo[0..r),
// hi[0..r)), so one product with K = 3r sums hi*hi + hi*lo + lo*hi.
__global__ void mode_tables(const double *U, int r, long long D, int ld, float *uw_hi, float *uw_lo,
                            float *modes, float *ut3) {
    const long long total = static_cast<long long>(r) * D;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long j = i / D, e = i % D;
        const float f = static_cast<float>(U[i]), h = tf32_round(f);
        uw_hi[i] = h;
        uw_lo[i] = f - h;
        const float u = static_cast<float>(U[i] / column_weight(e, ld)), uh = tf32_round(u);
        modes[i] = u;
        ut3[e * 3 * r + j] = uh;
        ut3[e * 3 * r + r + j] = u - uh;
        ut3[e * 3 * r + 2 * r + j] = uh;
    }
}
// C[i][j] (leading dimension ldc) = sum over slices z of partial[z][i][j]
__global__ void sum_slices(const float *partial, int slices, int M, int N, float *C, long long ldc) {
    const long long total = static_cast<long long>(M) * N;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        float s = 0;
        for (int z = 0; z < slices; ++z)
            s += partial[z * total + i];
        C[(i / N) * ldc + i % N] = s;
    }
}
// mean[j] = sum_m (y[m][j] - x[m][j]) / rows: the ensemble mean of the coefficient change
__global__ void delta_mean(const float *y, const float *x, long long ldx, int rows, int r,
                           float *mean) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= r)
        return;
    double s = 0;
    for (int m = 0; m < rows; ++m)
        s += static_cast<double>(y[static_cast<long long>(m) * r + j]) - x[m * ldx + j];
    mean[j] = static_cast<float>(s / rows);
}
// x[m][e] += inc[e] for every member
__global__ void add_to_members(float *x, const float *inc, int rows, long long D) {
    const long long total = rows * D;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        x[i] += inc[i % D];
}
// delta = y - x[:, :r] (x row stride ldx), less center[j] if given, split for 3xTF32 into
// d3[m] = (hi[0..r), hi[0..r), lo[0..r)) to pair with ut3 of mode_tables.
__global__ void delta_split(const float *y, const float *x, long long ldx, int rows, int r,
                            const float *center, float *d3) {
    const long long total = static_cast<long long>(rows) * r;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / r;
        const int j = static_cast<int>(i % r);
        const float d = y[i] - x[m * ldx + j] - (center ? center[j] : 0.0f);
        const float h = tf32_round(d);
        d3[m * 3 * r + j] = h;
        d3[m * 3 * r + r + j] = h;
        d3[m * 3 * r + 2 * r + j] = d - h;
    }
}
// Noise-mode amplitudes of a forecast window: for the four lowest modes (kx, ky) = (1,0),
// (0,1), (1,1), (1,-1) the sum over the window's steps of the Euler-Maruyama increments the
// spectral step adds there (same Philox keys), re then im: out[m][8] (row stride ldo).
__global__ void noise_window(uint64_t seed, uint32_t member_base, int members, uint64_t first_step,
                             uint64_t steps, double scale, int kmax2, float *out, long long ldo) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= members)
        return;
    const int kx[4] = {1, 0, 1, 1}, ky[4] = {0, 1, 1, -1};
    for (int q = 0; q < 4; ++q) {
        double sr = 0, si = 0;
        if (kx[q] * kx[q] + ky[q] * ky[q] <= kmax2)
            for (uint64_t s = 0; s < steps; ++s) {
                double xi1, xi2;
                philox_normal_pair(seed, member_base + m, first_step + s, mode_code(kx[q], ky[q]), xi1,
                                   xi2);
                sr += scale * xi1;
                si += scale * xi2;
            }
        out[m * ldo + 2 * q] = static_cast<float>(sr);
        out[m * ldo + 2 * q + 1] = static_cast<float>(si);
    }
}

// Adds to every member's compact FP32 state the window's noise: on every mode of the noise
// shell, the sum over steps [first_step, first_step + steps) of the increments the spectral
// step adds there (same Philox draws, same conjugate handling of the kx = 0 column).  One block
// per member, one thread per (kx, ky) candidate with 0 <= kx, |ky| <= kmax.
__global__ void add_window_noise(float2 *x, int C, int LD, int K, uint64_t seed, uint32_t member_base,
                                 uint64_t first_step, uint64_t steps, double scale, int kmax) {
    const int m = blockIdx.x;
    const int side = 2 * kmax + 1;
    for (int t = threadIdx.x; t < (kmax + 1) * side; t += blockDim.x) {
        const int kx = t / side, ky = t % side - kmax;
        const int k2 = kx * kx + ky * ky;
        if (k2 < 1 || k2 > kmax * kmax || kx >= C || ky > K || -ky > K)
            continue;
        const bool rep = kx > 0 || ky > 0;
        const uint32_t code = mode_code(kx, rep ? ky : -ky);
        double sr = 0, si = 0;
        for (uint64_t s = 0; s < steps; ++s) {
            double xi1, xi2;
            philox_normal_pair(seed, member_base + m, first_step + s, code, xi1, xi2);
            sr += scale * xi1;
            si += rep ? scale * xi2 : -(scale * xi2);
        }
        const int j = ky >= 0 ? ky : ky + LD;
        float2 &v = x[(static_cast<long long>(m) * C + kx) * LD + j];
        v.x += static_cast<float>(sr);
        v.y += static_cast<float>(si);
    }
}

int blocks_for(long long n) {
    return static_cast<int>(std::min<long long>((n + 255) / 256, 8192));
}

void d64_check(cudaError_t e, const char *what) { cuda_check(e, what); }

// ---- host helpers on device data ---------------------------------------------------------
template <typename T> void upload(DeviceBuffer &b, const std::vector<T> &v, cudaStream_t s) {
    b.ensure(v.size() * sizeof(T), "allocate POD workspace");
    cuda_check(cudaMemcpyAsync(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, s),
               "upload POD data");
}
template <typename T> std::vector<T> download(const T *d, size_t count, cudaStream_t s) {
    std::vector<T> v(count);
    cuda_check(cudaMemcpyAsync(v.data(), d, count * sizeof(T), cudaMemcpyDeviceToHost, s),
               "download POD data");
    cuda_check(cudaStreamSynchronize(s), "POD download");
    return v;
}

// Orthonormalise the rows of U (r x D, device, in place through `tmp`) by two Cholesky QR
// passes: U <- L^{-1} U with U U^T = L L^T.  Equals Gram-Schmidt on the rows in order followed
// by normalisation.  Returns the diagonal of the first pass's L: the norm of each row after
// removing its components along the earlier rows.
std::vector<double> cholesky_qr_rows(double *U, double *tmp, int r, long long D, DeviceBuffer &gram,
                                     DeviceBuffer &linv, cudaStream_t s) {
    std::vector<double> first;
    gram.ensure(sizeof(double) * r * r, "allocate POD Gram");
    for (int pass = 0; pass < 2; ++pass) {
        d64_check(d64::gemm(d64::GemmArgs{r, r, static_cast<int>(D), 1.0, 0.0, U, D, 1, U, 1, D,
                                          gram.as<double>(), r},
                            s),
                  "launch mode Gram");
        std::vector<double> b = download(gram.as<double>(), static_cast<size_t>(r) * r, s);
        std::vector<double> diag(r);
        const double smallest = cholesky_host(b, r);
        for (int j = 0; j < r; ++j)
            diag[j] = b[static_cast<size_t>(j) * r + j];
        if (pass == 0)
            first = diag;
        if (!(smallest > 0))
            raise(HZLB_ERUNTIME, "numerically degenerate POD mode");
        upload(linv, lower_inverse(b, r), s);
        d64_check(d64::gemm(d64::GemmArgs{r, static_cast<int>(D), r, 1.0, 0.0, linv.as<double>(), r, 1,
                                          U, D, 1, tmp, D},
                            s),
                  "launch mode orthonormalisation");
        cuda_check(cudaMemcpyAsync(U, tmp, sizeof(double) * r * D, cudaMemcpyDeviceToDevice, s),
                   "copy modes");
    }
    return first;
}

} // namespace

// ---- compact FP32 basis (handle) -----------------------------------------------------------
class PodBasis {
  public:
    int n, K, C, LD, r, device;
    long long D;   // reals per member
    std::vector<double> eigenvalues;
    double captured = 0, residual = 0;

    PodBasis(int n_, int device_) : n(n_), device(device_) {
        K = (n - 1) / 3;
        C = K + 1;
        LD = 2 * K + 1;
        D = 2LL * C * LD;
        cuda_check(cudaSetDevice(device), "select CUDA device");
        cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "create stream");
    }
    ~PodBasis() {
        if (stream_)
            cudaStreamDestroy(stream_);
    }

    void fit(const float *snaps, int m, int rank, int oversample, int iterations, uint64_t seed) {
        if (m < 2 || rank < 1 || rank >= m || oversample < 0 || iterations < 1)
            raise(HZLB_EINVAL, "POD needs 2 <= rank + 1 <= snapshots, oversample >= 0, iterations >= 1");
        cudaStream_t s = stream_;
        r = rank;
        mean_.ensure(sizeof(float) * D, "allocate POD mean");
        column_mean<float><<<static_cast<unsigned>((D + 31) / 32), dim3(32, 8), 0, s>>>(snaps, D, m,
                                                                                     mean_.as<float>());
        DeviceBuffer xd, hl, gram32, gram;
        xd.ensure(sizeof(double) * m * D, "allocate centred snapshots");
        hl.ensure(sizeof(float) * 2 * m * D, "allocate snapshot split");
        float *hi = hl.as<float>(), *lo = hi + static_cast<long long>(m) * D;
        center_weight<<<center_grid(m, D), 256, 0, s>>>(snaps, mean_.as<float>(), m, static_cast<int>(D),
                                                         LD, xd.as<double>(), hi, lo);
        cuda_check(cudaGetLastError(), "launch snapshot centring");
        // Gram matrix on the tensor cores: hi hi^T + hi lo^T + lo hi^T
        gram32.ensure(sizeof(float) * m * m, "allocate snapshot Gram");
        const float *pa[3] = {hi, hi, lo}, *pb[3] = {hi, lo, hi};
        for (int i = 0; i < 3; ++i) {
            tc::GemmArgs g{};
            g.M = m;
            g.N = m;
            g.K = static_cast<int>(D);
            g.A = pa[i];
            g.lda = D;
            g.a_kcontig = 1;
            g.B = pb[i];
            g.ldb = D;
            g.b_kcontig = 1;
            g.C = gram32.as<float>();
            g.ldc = m;
            g.alpha = 1.0f;
            g.beta = i ? 1.0f : 0.0f;
            g.status = status_ptr();
            cuda_check(gemm(g, 4, s), "launch snapshot Gram");
        }
        gram.ensure(sizeof(double) * m * m, "allocate snapshot Gram");
        double *G = gram.as<double>();
        symmetric_to_double<<<blocks_for(static_cast<long long>(m) * m), 256, 0, s>>>(gram32.as<float>(),
                                                                                    m, G);
        std::vector<double> Gh = download(G, static_cast<size_t>(m) * m, s);
        double trace = 0;
        for (int i = 0; i < m; ++i)
            trace += Gh[static_cast<size_t>(i) * m + i];
        if (!(trace > 0) || !std::isfinite(trace))
            raise(HZLB_EINVAL, "snapshots have no finite variance");

        const int k = std::min(m, rank + oversample);
        std::vector<double> V;   // m x r leading eigenvectors (host)
        eigenvalues.assign(r, 0.0);
        if (k >= m || m <= 256) {
            std::vector<double> a = Gh, vec;
            if (!jacobi(a, vec, m, trace))
                raise(HZLB_ERUNTIME, "snapshot Jacobi eigensolver failed to converge");
            const auto order = descending(a, m);
            V.assign(static_cast<size_t>(m) * r, 0.0);
            for (int j = 0; j < r; ++j) {
                eigenvalues[j] = a[order[j] * m + order[j]];
                for (int i = 0; i < m; ++i)
                    V[static_cast<size_t>(i) * r + j] = vec[static_cast<size_t>(i) * m + order[j]];
            }
        } else {
            subspace(G, m, k, iterations, seed, trace, V);
        }
        for (int j = 0; j < r; ++j)
            if (!(eigenvalues[j] > 1e-12 * trace))
                raise(HZLB_ERUNTIME, "fewer resolved POD modes than the requested rank");
        double kept = 0;
        for (int j = 0; j < r; ++j)
            kept += eigenvalues[j];
        captured = kept / trace;
        // residuals |G v - lambda v| / lambda of the returned pairs
        {
            DeviceBuffer vd, yd;
            upload(vd, V, s);
            yd.ensure(sizeof(double) * m * r, "allocate residual");
            d64_check(d64::gemm(d64::GemmArgs{m, r, m, 1.0, 0.0, G, m, 1, vd.as<double>(), r, 1,
                                              yd.as<double>(), r},
                                s),
                      "launch residual");
            std::vector<double> Y = download(yd.as<double>(), static_cast<size_t>(m) * r, s);
            residual = 0;
            for (int j = 0; j < r; ++j) {
                double e2 = 0;
                for (int i = 0; i < m; ++i) {
                    const double d = Y[static_cast<size_t>(i) * r + j] - eigenvalues[j] * V[static_cast<size_t>(i) * r + j];
                    e2 += d * d;
                }
                residual = std::max(residual, std::sqrt(e2) / eigenvalues[j]);
            }
        }
        // modes U = (V / sqrt(lambda))^T Xc in the weighted space, then orthonormalised
        std::vector<double> wt(static_cast<size_t>(r) * m);
        for (int j = 0; j < r; ++j)
            for (int i = 0; i < m; ++i)
                wt[static_cast<size_t>(j) * m + i] = V[static_cast<size_t>(i) * r + j] / std::sqrt(eigenvalues[j]);
        DeviceBuffer wd, ud, tmp, g2, li;
        upload(wd, wt, s);
        ud.ensure(sizeof(double) * r * D, "allocate modes");
        tmp.ensure(sizeof(double) * r * D, "allocate modes");
        d64_check(d64::gemm(d64::GemmArgs{r, static_cast<int>(D), m, 1.0, 0.0, wd.as<double>(), m, 1,
                                          xd.as<double>(), D, 1, ud.as<double>(), D},
                            s),
                  "launch mode synthesis");
        const std::vector<double> norms = cholesky_qr_rows(ud.as<double>(), tmp.as<double>(), r, D, g2, li, s);
        for (double v : norms)
            if (v < 1e-8)
                raise(HZLB_ERUNTIME, "numerically degenerate POD mode");
        tables_.ensure(sizeof(float) * 6 * r * D, "allocate mode tables");
        float *t = tables_.as<float>();
        mode_tables<<<blocks_for(r * D), 256, 0, s>>>(ud.as<double>(), r, D, LD, t, t + r * D,
                                                       t + 2 * r * D, t + 3 * r * D);
        cuda_check(cudaGetLastError(), "launch mode tables");
        check_status(s);
    }

    // a[count][r] (row stride ldc) = projections of compact FP32 states (count x D) on the modes
    void project(const float *x, int count, float *a, long long ldc, cudaStream_t s) {
        ensure_fitted();
        const long long cd = static_cast<long long>(count) * D;
        work_.ensure(sizeof(float) * 2 * cd, "allocate projection workspace");
        float *hi = work_.as<float>(), *lo = hi + cd;
        center_weight<<<center_grid(count, D), 256, 0, s>>>(x, mean_.as<float>(), count,
                                                             static_cast<int>(D), LD, nullptr, hi, lo);
        cuda_check(cudaGetLastError(), "launch state centring");
        // split-K: each of the three products over K = D in chunks of kchunk
        const int eps = tc::SLAB / 4;
        int splits = std::max(1, std::min(32, 148 * 2 / std::max(1, (count + 127) / 128)));
        int kchunk = static_cast<int>(((D + splits - 1) / splits + eps - 1) / eps * eps);
        splits = static_cast<int>((D + kchunk - 1) / kchunk);
        const long long slice = static_cast<long long>(count) * r;
        partial_.ensure(sizeof(float) * 3 * splits * slice, "allocate split-K workspace");
        const float *uw_hi = tables_.as<float>(), *uw_lo = uw_hi + r * D;
        const float *pa[3] = {hi, hi, lo}, *pb[3] = {uw_hi, uw_lo, uw_hi};
        for (int i = 0; i < 3; ++i) {
            tc::GemmArgs g{};
            g.M = count;
            g.N = r;
            g.K = static_cast<int>(D);
            g.A = pa[i];
            g.lda = D;
            g.a_kcontig = 1;
            g.B = pb[i];
            g.ldb = D;
            g.b_kcontig = 1;
            g.alpha = 1.0f;
            g.splits = splits;
            g.kchunk = kchunk;
            g.partial = partial_.as<float>() + i * splits * slice;
            g.status = status_ptr();
            cuda_check(gemm(g, 4, s), "launch projection");
        }
        sum_slices<<<blocks_for(slice), 256, 0, s>>>(partial_.as<float>(), 3 * splits, count, r, a, ldc);
        cuda_check(cudaGetLastError(), "launch split-K sum");
    }
    // x[count][D] += delta[count][r] (unweighted) modes: one 3xTF32 product with the split
    // terms side by side along K (d3 from delta_split, ut3 from mode_tables), so the ensemble
    // state is read and written once
    void update(float *x, int count, const float *d3, cudaStream_t s) {
        ensure_fitted();
        tc::GemmArgs g{};
        g.M = count;
        g.N = static_cast<int>(D);
        g.K = 3 * r;
        g.A = d3;
        g.lda = 3 * r;
        g.a_kcontig = 1;
        g.B = tables_.as<float>() + 3 * r * D;
        g.ldb = 3 * r;
        g.b_kcontig = 1;
        g.C = x;
        g.ldc = D;
        g.alpha = 1.0f;
        g.beta = 1.0f;
        g.status = status_ptr();
        cuda_check(gemm(g, 4, s), "launch mode update");
    }
    // One window of the learned forecast on an ensemble held by `e`: project, add the window's
    // noise amplitudes, run the network (which predicts the coefficients without the direct
    // contribution of the window's noise), add the change of the coefficients back, then add
    // the window's noise increments themselves on every noise mode.
    //
    // With mean_increment (device, D floats) that field is added to every member after the
    // network's change.  With centre it is the change of the ensemble mean over the window from
    // another forecast (e.g. the spectral solver run on the mean) and the network only moves
    // the members about their mean: the members' coefficient changes are centred over the
    // ensemble.  Without centre the network's changes are kept whole and the increment carries
    // what the network cannot (e.g. the motion outside the POD space).
    void learned_window(Engine &e, const hzlb_config &cfg, hzlb_mlp *mlp, int q, double dt,
                        uint64_t steps, const float *mean_increment, bool centre) {
        ensure_fitted();
        const int M = e.members();
        cudaStream_t s = static_cast<cudaStream_t>(e.stream());
        const int in = r + q;
        io_.ensure(sizeof(float) * (static_cast<size_t>(M) * (in + 4 * r) + r), "allocate forecast buffers");
        float *xin = io_.as<float>(), *y = xin + static_cast<size_t>(M) * in, *d3 = y + static_cast<size_t>(M) * r,
              *dmean = d3 + static_cast<size_t>(M) * 3 * r;
        float *state = static_cast<float *>(e.state_device());
        project(state, M, xin, in, s);
        const double scale = cfg.noise_sigma > 0 ? cfg.noise_sigma * std::sqrt(dt) / kSqrt2 : 0.0;
        noise_window<<<(M + 127) / 128, 128, 0, s>>>(cfg.seed, cfg.member_base, M, e.step_index, steps,
                                                     scale, cfg.noise_kmax * cfg.noise_kmax, xin + r, in);
        cuda_check(cudaGetLastError(), "launch noise amplitudes");
        if (int rc = hzlb_mlp_forward(mlp, xin, M, y, s))
            raise(rc, std::string("learned forecast network: ") + hzlb_last_error());
        const bool centred = mean_increment && centre;
        if (centred)
            delta_mean<<<(r + 63) / 64, 64, 0, s>>>(y, xin, in, M, r, dmean);
        delta_split<<<blocks_for(static_cast<long long>(M) * r), 256, 0, s>>>(
            y, xin, in, M, r, centred ? dmean : nullptr, d3);
        cuda_check(cudaGetLastError(), "launch coefficient change");
        update(state, M, d3, s);
        if (mean_increment) {
            add_to_members<<<blocks_for(M * D), 256, 0, s>>>(state, mean_increment, M, D);
            cuda_check(cudaGetLastError(), "launch mean increment");
        }
        if (scale > 0) {
            add_window_noise<<<M, 64, 0, s>>>(reinterpret_cast<float2 *>(state), C, LD, K, cfg.seed,
                                              cfg.member_base, e.step_index, steps, scale,
                                              cfg.noise_kmax);
            cuda_check(cudaGetLastError(), "launch window noise");
        }
        e.set_time(e.time + static_cast<double>(steps) * dt, e.step_index + steps);
    }
    void modes(float *modes_host, float *mean_host) {
        ensure_fitted();
        if (modes_host)
            cuda_check(cudaMemcpyAsync(modes_host, tables_.as<float>() + 2 * r * D, sizeof(float) * r * D,
                                       cudaMemcpyDeviceToHost, stream_),
                       "download modes");
        if (mean_host)
            cuda_check(cudaMemcpyAsync(mean_host, mean_.ptr, sizeof(float) * D, cudaMemcpyDeviceToHost,
                                       stream_),
                       "download mean");
        cuda_check(cudaStreamSynchronize(stream_), "download modes");
    }
    void check_status(cudaStream_t s) {
        uint32_t st = 0;
        cuda_check(cudaMemcpyAsync(&st, status_ptr(), sizeof(st), cudaMemcpyDeviceToHost, s),
                   "read POD status");
        cuda_check(cudaStreamSynchronize(s), "POD");
        if (st)
            raise(HZLB_ERUNTIME, "tensor-core GEMM wait expired in the POD");
    }
    cudaStream_t stream() const { return stream_; }

  private:
    uint32_t *status_ptr() {
        if (!status_.ptr) {
            status_.ensure(sizeof(uint32_t), "allocate status");
            cuda_check(cudaMemset(status_.ptr, 0, sizeof(uint32_t)), "clear status");
        }
        return status_.as<uint32_t>();
    }
    void ensure_fitted() const {
        if (!tables_.ptr)
            raise(HZLB_EINVAL, "POD basis has not been fitted");
    }
    // Leading r eigenpairs of the m x m device matrix G by subspace iteration with k columns.
    void subspace(const double *G, int m, int k, int iterations, uint64_t seed, double trace,
                  std::vector<double> &V) {
        cudaStream_t s = stream_;
        std::mt19937_64 rng(seed);
        std::normal_distribution<double> nd;
        std::vector<double> q(static_cast<size_t>(m) * k);
        for (double &v : q)
            v = nd(rng);
        DeviceBuffer qd, yd, bd, rd;
        upload(qd, q, s);
        yd.ensure(sizeof(double) * m * k, "allocate subspace");
        bd.ensure(sizeof(double) * k * k, "allocate subspace");
        // Q <- orthonormal basis of span(Y) by Cholesky QR twice (columns scaled to unit norm
        // first); pass 0 writes Q from Y, pass 1 writes Y from Q (the product is never in place)
        auto orthonormalise = [&](double *Y, double *Q) {
            for (int pass = 0; pass < 2; ++pass) {
                const double *src = pass == 0 ? Y : Q;
                double *dst = pass == 0 ? Q : Y;
                d64_check(d64::gemm(d64::GemmArgs{k, k, m, 1.0, 0.0, src, 1, k, src, k, 1, bd.as<double>(), k},
                                    s),
                          "launch subspace Gram");
                std::vector<double> b = download(bd.as<double>(), static_cast<size_t>(k) * k, s);
                std::vector<double> dsc(k);
                for (int j = 0; j < k; ++j)
                    dsc[j] = 1 / std::sqrt(std::max(b[static_cast<size_t>(j) * k + j], 1e-300));
                for (int i = 0; i < k; ++i)
                    for (int j = 0; j < k; ++j)
                        b[static_cast<size_t>(i) * k + j] *= dsc[i] * dsc[j];
                if (!(cholesky_host(b, k) > 1e-7)) {
                    // (numerically) dependent columns: Gram-Schmidt on the host, replacing
                    // each dependent column by a fresh random direction
                    std::vector<double> y = download(src, static_cast<size_t>(m) * k, s);
                    gram_schmidt_host(y, m, k, rng);
                    upload(rd, y, s);
                    cuda_check(cudaMemcpyAsync(Q, rd.ptr, sizeof(double) * m * k, cudaMemcpyDeviceToDevice, s),
                               "copy subspace basis");
                    cuda_check(cudaMemcpyAsync(Y, rd.ptr, sizeof(double) * m * k, cudaMemcpyDeviceToDevice, s),
                               "copy subspace basis");
                    return;
                }
                const std::vector<double> li = lower_inverse(b, k);
                // Q = Y D L^{-T}:  rhs[l][j] = dsc[l] li[j][l]
                std::vector<double> rhs(static_cast<size_t>(k) * k);
                for (int l = 0; l < k; ++l)
                    for (int j = 0; j < k; ++j)
                        rhs[static_cast<size_t>(l) * k + j] = dsc[l] * li[static_cast<size_t>(j) * k + l];
                upload(rd, rhs, s);
                d64_check(d64::gemm(d64::GemmArgs{m, k, k, 1.0, 0.0, src, k, 1, rd.as<double>(), k, 1, dst, k},
                                    s),
                          "launch subspace basis");
            }
            cuda_check(cudaMemcpyAsync(Q, Y, sizeof(double) * m * k, cudaMemcpyDeviceToDevice, s),
                       "copy subspace basis");
        };
        // the random start is made orthonormal through the same routine
        cuda_check(cudaMemcpyAsync(yd.ptr, qd.ptr, sizeof(double) * m * k, cudaMemcpyDeviceToDevice, s),
                   "copy subspace");
        orthonormalise(yd.as<double>(), qd.as<double>());
        for (int it = 0; it < iterations; ++it) {
            d64_check(d64::gemm(d64::GemmArgs{m, k, m, 1.0, 0.0, G, m, 1, qd.as<double>(), k, 1,
                                              yd.as<double>(), k},
                                s),
                      "launch subspace product");
            orthonormalise(yd.as<double>(), qd.as<double>());
        }
        // Rayleigh-Ritz: T = Q^T G Q, eigenpairs by Jacobi, V = Q S
        d64_check(d64::gemm(d64::GemmArgs{m, k, m, 1.0, 0.0, G, m, 1, qd.as<double>(), k, 1,
                                          yd.as<double>(), k},
                            s),
                  "launch Ritz product");
        d64_check(d64::gemm(d64::GemmArgs{k, k, m, 1.0, 0.0, qd.as<double>(), 1, k, yd.as<double>(), k, 1,
                                          bd.as<double>(), k},
                            s),
                  "launch Ritz matrix");
        std::vector<double> T = download(bd.as<double>(), static_cast<size_t>(k) * k, s);
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < i; ++j)
                T[static_cast<size_t>(i) * k + j] = T[static_cast<size_t>(j) * k + i] =
                    0.5 * (T[static_cast<size_t>(i) * k + j] + T[static_cast<size_t>(j) * k + i]);
        std::vector<double> S;
        if (!jacobi(T, S, k, trace))
            raise(HZLB_ERUNTIME, "Ritz Jacobi eigensolver failed to converge");
        const auto order = descending(T, k);
        const std::vector<double> Q = download(qd.as<double>(), static_cast<size_t>(m) * k, s);
        V.assign(static_cast<size_t>(m) * r, 0.0);
        for (int j = 0; j < r; ++j) {
            eigenvalues[j] = T[order[j] * k + order[j]];
            for (int i = 0; i < m; ++i) {
                double v = 0;
                for (int l = 0; l < k; ++l)
                    v += Q[static_cast<size_t>(i) * k + l] * S[static_cast<size_t>(l) * k + order[j]];
                V[static_cast<size_t>(i) * r + j] = v;
            }
        }
    }

    cudaStream_t stream_ = nullptr;
    DeviceBuffer mean_, tables_, work_, partial_, io_, status_;
};

} // namespace hzlb

struct hzlb_pod {
    std::unique_ptr<hzlb::PodBasis> basis;
};

namespace {
template <class F> int guarded_pod(F &&f) {
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
hzlb::PodBasis &basis(hzlb_pod *h) {
    if (!h || !h->basis)
        hzlb::raise(HZLB_EINVAL, "null POD handle");
    return *h->basis;
}
} // namespace

extern "C" {

HZLB_API int hzlb_fit_pod(size_t m, size_t dimension, const double *snapshots, size_t max_rank,
                          double fraction, int device, size_t *rank, double *mean, double *modes,
                          double *singular_values, double *captured) {
    using namespace hzlb;
    return guarded_pod([&] {
        if (m < 2 || m > 512 || dimension == 0 || max_rank == 0 || !std::isfinite(fraction) ||
            fraction <= 0 || fraction > 1)
            raise(HZLB_EINVAL,
                  "POD requires 2..512 snapshots, positive rank, and variance fraction in (0,1]");
        if (!snapshots || !rank || !mean || !modes || !singular_values || !captured)
            raise(HZLB_EINVAL, "null argument");
        for (size_t i = 0; i < 2 * m * dimension; ++i)
            if (!std::isfinite(snapshots[i]))
                raise(HZLB_EINVAL, "nonfinite snapshot");
        cuda_check(cudaSetDevice(device), "select CUDA device");
        cudaStream_t s = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "create stream");
        struct StreamGuard {
            cudaStream_t s;
            ~StreamGuard() { cudaStreamDestroy(s); }
        } guard{s};
        const int mi = static_cast<int>(m);
        const long long D = 2LL * static_cast<long long>(dimension);
        DeviceBuffer xs, xc, mn, gram;
        xs.ensure(sizeof(double) * m * D, "allocate snapshots");
        xc.ensure(sizeof(double) * m * D, "allocate snapshots");
        mn.ensure(sizeof(double) * D, "allocate mean");
        cuda_check(cudaMemcpyAsync(xs.ptr, snapshots, sizeof(double) * m * D, cudaMemcpyHostToDevice, s),
                   "upload snapshots");
        column_mean<double><<<static_cast<unsigned>((D + 31) / 32), dim3(32, 8), 0, s>>>(
            xs.as<double>(), D, mi, mn.as<double>());
        center_double<<<blocks_for(mi * D), 256, 0, s>>>(xs.as<double>(), mn.as<double>(), mi, D,
                                                         xc.as<double>());
        cuda_check(cudaGetLastError(), "launch snapshot centring");
        gram.ensure(sizeof(double) * m * m, "allocate Gram");
        d64_check(d64::gemm(d64::GemmArgs{mi, mi, static_cast<int>(D), 1.0, 0.0, xc.as<double>(), D, 1,
                                          xc.as<double>(), 1, D, gram.as<double>(), mi},
                            s),
                  "launch snapshot Gram");
        std::vector<double> a = download(gram.as<double>(), m * m, s);
        for (size_t i = 0; i < m; ++i)   // exact symmetry, as the reference fills both halves
            for (size_t j = 0; j < i; ++j)
                a[j * m + i] = a[i * m + j];
        double trace = 0;
        for (size_t i = 0; i < m; ++i)
            trace += a[i * m + i];
        if (trace <= 0 || !std::isfinite(trace))
            raise(HZLB_EINVAL, "snapshots have no finite variance");
        std::vector<double> vec;
        if (!jacobi(a, vec, m, trace))
            raise(HZLB_ERUNTIME, "snapshot Jacobi eigensolver failed to converge");
        const auto order = descending(a, m);
        // the reference's truncation (reduced.cpp:106-131)
        std::vector<size_t> cols;
        double retained = 0;
        for (size_t column : order) {
            const double ev = a[column * m + column];
            if (ev <= 1e-12 * trace || cols.size() >= max_rank)
                break;
            cols.push_back(column);
            retained += ev;
            if (retained / trace >= fraction)
                break;
        }
        if (cols.empty())
            raise(HZLB_ERUNTIME, "no resolved POD modes");
        const int r = static_cast<int>(cols.size());
        std::vector<double> wt(static_cast<size_t>(r) * m);
        for (int j = 0; j < r; ++j) {
            const double ev = a[cols[j] * m + cols[j]];
            for (size_t i = 0; i < m; ++i)
                wt[j * m + i] = vec[i * m + cols[j]] / std::sqrt(ev);
            singular_values[j] = std::sqrt(ev);
        }
        DeviceBuffer wd, ud, tmp, g2, li;
        upload(wd, wt, s);
        ud.ensure(sizeof(double) * r * D, "allocate modes");
        tmp.ensure(sizeof(double) * r * D, "allocate modes");
        d64_check(d64::gemm(d64::GemmArgs{r, static_cast<int>(D), mi, 1.0, 0.0, wd.as<double>(), mi, 1,
                                          xc.as<double>(), D, 1, ud.as<double>(), D},
                            s),
                  "launch mode synthesis");
        const std::vector<double> norms = cholesky_qr_rows(ud.as<double>(), tmp.as<double>(), r, D, g2, li, s);
        for (double v : norms)
            if (v < 1e-8)
                raise(HZLB_ERUNTIME, "numerically degenerate POD mode");
        cuda_check(cudaMemcpyAsync(modes, ud.ptr, sizeof(double) * r * D, cudaMemcpyDeviceToHost, s),
                   "download modes");
        cuda_check(cudaMemcpyAsync(mean, mn.ptr, sizeof(double) * D, cudaMemcpyDeviceToHost, s),
                   "download mean");
        cuda_check(cudaStreamSynchronize(s), "fit POD");
        *rank = static_cast<size_t>(r);
        *captured = retained / trace;
    });
}

HZLB_API int hzlb_pod_fit(int n, int snapshots, const void *data, int rank, int oversample,
                          int iterations, uint64_t seed, int device, hzlb_pod **out) {
    using namespace hzlb;
    return guarded_pod([&] {
        if (!out || !data)
            raise(HZLB_EINVAL, "null argument");
        if (n < 8 || n > 512 || (n & (n - 1)))
            raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
        auto h = std::make_unique<hzlb_pod>();
        h->basis = std::make_unique<PodBasis>(n, device);
        h->basis->fit(static_cast<const float *>(data), snapshots, rank, oversample, iterations, seed);
        *out = h.release();
    });
}
HZLB_API void hzlb_pod_destroy(hzlb_pod *h) { delete h; }
HZLB_API int hzlb_pod_info(hzlb_pod *h, int *rank, double *eigenvalues, double *captured,
                           double *residual) {
    return guarded_pod([&] {
        auto &b = basis(h);
        if (rank)
            *rank = b.r;
        if (eigenvalues)
            std::memcpy(eigenvalues, b.eigenvalues.data(), sizeof(double) * b.r);
        if (captured)
            *captured = b.captured;
        if (residual)
            *residual = b.residual;
    });
}
HZLB_API int hzlb_pod_modes(hzlb_pod *h, float *modes, float *mean) {
    return guarded_pod([&] { basis(h).modes(modes, mean); });
}
HZLB_API int hzlb_pod_project(hzlb_pod *h, const void *states, int count, float *coefficients,
                              long long ldc, void *stream) {
    return guarded_pod([&] {
        auto &b = basis(h);
        if (!states || !coefficients || count < 1 || ldc < b.r)
            hzlb::raise(HZLB_EINVAL, "invalid projection arguments");
        cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : b.stream();
        b.project(static_cast<const float *>(states), count, coefficients, ldc, s);
        if (!stream)
            b.check_status(s);
    });
}
HZLB_API int hzlb_add_window_noise(const hzlb_config *config, double dt, uint64_t first_step,
                                   uint64_t steps, int count, void *state, void *stream) {
    using namespace hzlb;
    return guarded_pod([&] {
        if (!config || !state || count < 1 || !(dt > 0))
            raise(HZLB_EINVAL, "invalid window noise arguments");
        const hzlb_config &c = *config;
        if (c.precision != 4)
            raise(HZLB_EINVAL, "window noise is added to FP32 states");
        const int K = (c.n - 1) / 3, C = K + 1, LD = 2 * K + 1;
        if (!(c.noise_sigma > 0) || c.noise_kmax < 1)
            return;
        const double scale = c.noise_sigma * std::sqrt(dt) / kSqrt2;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        add_window_noise<<<count, 64, 0, s>>>(static_cast<float2 *>(state), C, LD, K, c.seed,
                                              c.member_base, first_step, steps, scale, c.noise_kmax);
        cuda_check(cudaGetLastError(), "launch window noise");
        if (!stream)
            cuda_check(cudaStreamSynchronize(s), "window noise");
    });
}
HZLB_API int hzlb_noise_amplitudes(const hzlb_config *config, double dt, uint64_t first_step,
                                   uint64_t steps, int count, float *out, long long ldo, void *stream) {
    using namespace hzlb;
    return guarded_pod([&] {
        if (!config || !out || count < 1 || ldo < 8 || !(dt > 0))
            raise(HZLB_EINVAL, "invalid noise amplitude arguments");
        const hzlb_config &c = *config;
        const double scale = c.noise_sigma > 0 ? c.noise_sigma * std::sqrt(dt) / kSqrt2 : 0.0;
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        noise_window<<<(count + 127) / 128, 128, 0, s>>>(c.seed, c.member_base, count, first_step, steps,
                                                         scale, c.noise_kmax * c.noise_kmax, out, ldo);
        cuda_check(cudaGetLastError(), "launch noise amplitudes");
        if (!stream)
            cuda_check(cudaStreamSynchronize(s), "noise amplitudes");
    });
}

} // extern "C"

namespace hzlb {
// Defined here so the learned forecast can reach both the engine and the basis.
int learned_forecast(Engine &e, const hzlb_config &cfg, hzlb_pod *pod, hzlb_mlp *mlp, int q,
                     double dt, uint64_t steps, const void *mean_increment, bool centre) {
    return guarded_pod([&] {
        if (!mlp || q != 8 || !(dt > 0) || steps == 0)
            raise(HZLB_EINVAL, "learned forecast needs a network with 8 noise inputs, dt > 0, steps > 0");
        if (cfg.precision != 4)
            raise(HZLB_EINVAL, "learned forecast runs on FP32 ensembles");
        auto &b = basis(pod);
        if (b.n != cfg.n)
            raise(HZLB_EINVAL, "POD basis and ensemble grid differ");
        int nr = 0, nq = 0, hidden = 0, batch = 0;
        if (int rc = hzlb_mlp_shape(mlp, &nr, &nq, &hidden, &batch))
            raise(rc, hzlb_last_error());
        if (nr != b.r || nq != q || batch < e.members())
            raise(HZLB_EINVAL, "network shape does not match the POD rank, 8 noise inputs and the "
                               "ensemble size");
        b.learned_window(e, cfg, mlp, q, dt, steps, static_cast<const float *>(mean_increment),
                         centre);
        b.check_status(static_cast<cudaStream_t>(e.stream()));
    });
}
} // namespace hzlb
