// Batched tangent and adjoint drifts of the reference Solver, FP64 on the device:
//   Solver::linearized_drift(state, direction)  (src/solver.cpp:264-292)
//     = -F[u_d . grad(w) + u . grad(d)] - (nu k^2 + alpha) d
//   Solver::adjoint_drift(state, cotangent)     (src/solver.cpp:293-324)
//     = F[u . grad(L)] + i ky/k^2 F[L w_x] - i kx/k^2 F[L w_y] - (nu k^2 + alpha) l
// with u = (i ky psi, -i kx psi), psi = w/k^2 the velocity of the state w (u_d that of the
// direction d), L the physical cotangent l, F the forward transform normalised by 1/N^2 and the
// inverse unnormalised (the reference's Fourier2D), results on the active modes only.
//
// `count` (state, second field) pairs are processed as one batch: the spectral operators of
// both fields are formed in the compact half-spectrum, every physical field of the batch comes
// from the step's inverse column/row transforms, the reference's pointwise products are formed
// on the grid, and the product spectra return through forward row/column transforms.  Inputs
// are full n x n spectra (the reference's Field layout) of real fields; their Hermitian part on
// the retained modes is used, which is all the reference reads of a projected state (it keeps
// only the real part of every physical field).
#include "engine.h"
#include "launch.h"
#include "physical.cuh"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>
#include <vector>

namespace hzlb {
namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

enum FieldOp : int { OP_U = 0, OP_V = 1, OP_DX = 2, OP_DY = 3, OP_ID = 4 };
struct OpTable {
    int op[8], src[8], count;
};

// out[f][m][kx][j] = op_f applied to field src_f (a or b) in the compact half-spectrum
__global__ void spectral_ops(const cx<double> *a, const cx<double> *b, long long members, int C,
                             int LD, int K, OpTable t, cx<double> *out) {
    const long long per = static_cast<long long>(C) * LD, total = per * members;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int kx = static_cast<int>((i % per) / LD), j = static_cast<int>(i % LD);
        const int ky = j <= K ? j : j - LD;
        const double k2 = static_cast<double>(kx * kx + ky * ky);
        const double fx = static_cast<double>(kx), fy = static_cast<double>(ky);
        for (int f = 0; f < t.count; ++f) {
            const cx<double> w = (t.src[f] ? b : a)[i];
            const cx<double> psi = k2 > 0 ? mk(w.x / k2, w.y / k2) : mk(0.0, 0.0);
            cx<double> r;
            switch (t.op[f]) {
            case OP_U: r = mk(-fy * psi.y, fy * psi.x); break;    // i ky psi
            case OP_V: r = mk(fx * psi.y, -fx * psi.x); break;    // -i kx psi
            case OP_DX: r = mk(-fx * w.y, fx * w.x); break;       // i kx w
            case OP_DY: r = mk(-fy * w.y, fy * w.x); break;       // i ky w
            default: r = w;
            }
            out[f * total + i] = r;
        }
    }
}

// The reference's grid products (without fused multiply-adds, as its CPU build evaluates them).
// PRODUCT_TANGENT: fields {u_d, v_d, w_x, w_y, u, v, d_x, d_y} -> {u_d w_x + v_d w_y + u d_x + v d_y}
// PRODUCT_ADJOINT: fields {u, v, w_x, w_y, L, L_x, L_y}       -> {u L_x + v L_y, L w_x, L w_y}
// PRODUCT_DRIFT:   fields {u, v, w_x, w_y}                    -> {u w_x + v w_y}
enum ProductMode : int { PRODUCT_TANGENT = 0, PRODUCT_ADJOINT = 1, PRODUCT_DRIFT = 2 };
__global__ void grid_products(const double *phys, long long cells, int mode, double *out) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < cells;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double *f = phys + i;
        auto at = [&](int k) { return f[k * cells]; };
        if (mode == PRODUCT_DRIFT) {
            out[i] = __dadd_rn(__dmul_rn(at(0), at(2)), __dmul_rn(at(1), at(3)));
        } else if (mode == PRODUCT_TANGENT) {
            double s = __dadd_rn(__dmul_rn(at(0), at(2)), __dmul_rn(at(1), at(3)));
            s = __dadd_rn(s, __dadd_rn(__dmul_rn(at(4), at(6)), __dmul_rn(at(5), at(7))));
            out[i] = s;
        } else {
            out[i] = __dadd_rn(__dmul_rn(at(0), at(5)), __dmul_rn(at(1), at(6)));
            out[cells + i] = __dmul_rn(at(4), at(2));
            out[2 * cells + i] = __dmul_rn(at(4), at(3));
        }
    }
}

// max over the grid of (|u| + |v|) n / (2 pi) per member (the reference's cfl_rate,
// src/solver.cpp:392-395) from the physical velocity fields u = phys[0], v = phys[1], kept as a
// running maximum (bit pattern of a nonnegative double, monotone as an unsigned integer).
__global__ void cfl_rate_max(const double *phys, long long cells, long long nn, int n,
                             unsigned long long *bits) {
    const double scale = static_cast<double>(n) / (2 * kPi);
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < cells;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double r = (fabs(phys[i]) + fabs(phys[cells + i])) * scale;
        atomicMax(bits + i / nn, static_cast<unsigned long long>(__double_as_longlong(r)));
    }
}

// Forward row transforms of real fields, two rows packed as a + i b: x-spectra kx = 0..K of
// both rows into cols[m][kx][y].
template <int N>
__global__ void __launch_bounds__(Cfg<double, N>::ROW_THREADS)
    field_row_forward(const double *phys, cx<double> *cols, const cx<double> *tw_g) {
    using G = Cfg<double, N>;
    constexpr int E = G::E, T = G::T, C = G::C, K = G::K, TY = G::TY;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<double> *tw = reinterpret_cast<cx<double> *>(smem_raw);
    cx<double> *lines = tw + G::TWE;
    load_pass_twiddles<N, E, double>(tw, tw_g);
    __syncthreads();
    const int g = threadIdx.x / T, t = threadIdx.x % T, m = blockIdx.x;
    const bool active = g < TY / 2;
    const int ya = blockIdx.y * TY + (active ? 2 * g : 0);
    const double *ra = phys + (static_cast<size_t>(m) * N + ya) * N, *rb = ra + N;
    cx<double> *sm = lines + g * G::BUF;
    cx<double> z[E];
#pragma unroll
    for (int r = 0; r < E; ++r)
        z[r] = mk(ra[t + r * T], rb[t + r * T]);
    fft_line<N, E, -1, double>(z, sm, tw, t);
#pragma unroll
    for (int r = 0; r < E; ++r)
        sm[pad<E>(t + r * T)] = z[r];
    __syncwarp();
    if (active) {
        cx<double> *dst = cols + static_cast<size_t>(m) * C * N;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int p = t + r * T;
            if (p <= K) {
                const cx<double> zk = z[r], zc = conj(sm[pad<E>((N - p) & (N - 1))]);
                const cx<double> sa = zk + zc, sb = zk - zc;
                dst[static_cast<size_t>(p) * N + ya] = mk(sa.x / 2, sa.y / 2);
                dst[static_cast<size_t>(p) * N + ya + 1] = mk(sb.y / 2, -sb.x / 2);
            }
        }
    }
}

// Forward column transforms of cols[m][kx][y], retained ky only, normalised by 1/N^2:
// out[m][kx][j] in the compact layout.
template <int N>
__global__ void __launch_bounds__(Cfg<double, N>::COL_THREADS)
    field_column_forward(const cx<double> *cols, cx<double> *out, const cx<double> *tw_g) {
    using G = Cfg<double, N>;
    constexpr int E = G::E, T = G::T, C = G::C, LD = G::LD;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<double> *tw = reinterpret_cast<cx<double> *>(smem_raw);
    cx<double> *lines = tw + G::TWE;
    load_pass_twiddles<N, E, double>(tw, tw_g);
    __syncthreads();
    const int line = threadIdx.x / T, t = threadIdx.x % T;
    const int kx = blockIdx.y * G::LPB + line, m = blockIdx.x;
    const bool valid = kx < C;
    const int kxc = valid ? kx : 0;
    const cx<double> *src = cols + (static_cast<size_t>(m) * C + kxc) * N;
    cx<double> v[E];
#pragma unroll
    for (int r = 0; r < E; ++r)
        v[r] = src[t + r * T];
    fft_line<N, E, -1, double>(v, lines + line * G::BUF, tw, t);
    if (valid) {
        constexpr double nn = static_cast<double>(N) * N;
        cx<double> *dst = out + (static_cast<size_t>(m) * C + kxc) * LD;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int j = compact_j<N>(t + r * T);
            if (j >= 0)
                dst[j] = mk(v[r].x / nn, v[r].y / nn);
        }
    }
}

// The drift from the product spectra s[F'][m][kx][j] and the second field b (direction or
// cotangent); (0, 0) is not an active mode.
__global__ void combine(const cx<double> *s, const cx<double> *b, long long members, int C,
                        int LD, int K, const double *nu, const double *alpha, int adjoint,
                        cx<double> *out) {
    const long long per = static_cast<long long>(C) * LD, total = per * members;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int kx = static_cast<int>((i % per) / LD), j = static_cast<int>(i % LD);
        const int ky = j <= K ? j : j - LD;
        const int k2i = kx * kx + ky * ky;
        if (k2i == 0) {
            out[i] = mk(0.0, 0.0);
            continue;
        }
        const long long m = i / per;
        const double k2 = static_cast<double>(k2i), rate = nu[m] * k2 + alpha[m];
        const cx<double> d = b[i];
        if (!adjoint) {
            const cx<double> nl = s[i];
            out[i] = mk(-nl.x - rate * d.x, -nl.y - rate * d.y);
        } else {
            const cx<double> nl = s[i], p = s[total + i], q = s[2 * total + i];
            const double cy = static_cast<double>(ky) / k2, cxk = static_cast<double>(kx) / k2;
            // nl + (i ky/k^2) p - (i kx/k^2) q - rate l
            const double re = nl.x - cy * p.y + cxk * q.y - rate * d.x;
            const double im = nl.y + cy * p.x - cxk * q.x - rate * d.y;
            out[i] = mk(re, im);
        }
    }
}

template <int N> struct Forward {
    static cudaError_t run(const double *phys, cx<double> *cols, cx<double> *out,
                           const cx<double> *tw, int members, cudaStream_t s) {
        using G = Cfg<double, N>;
        const size_t row_smem = sizeof(cx<double>) * (G::TWE + G::GROUPS * G::BUF);
        const size_t col_smem = sizeof(cx<double>) * (G::TWE + G::LPB * G::BUF);
        field_row_forward<N><<<dim3(members, N / G::TY), G::ROW_THREADS, row_smem, s>>>(phys, cols, tw);
        field_column_forward<N><<<dim3(members, (G::C + G::LPB - 1) / G::LPB), G::COL_THREADS,
                                  col_smem, s>>>(cols, out, tw);
        return cudaGetLastError();
    }
};

cudaError_t launch_forward(int n, const double *phys, cx<double> *cols, cx<double> *out,
                           const cx<double> *tw, int members, cudaStream_t s) {
    switch (n) {
    case 8: return Forward<8>::run(phys, cols, out, tw, members, s);
    case 16: return Forward<16>::run(phys, cols, out, tw, members, s);
    case 32: return Forward<32>::run(phys, cols, out, tw, members, s);
    case 64: return Forward<64>::run(phys, cols, out, tw, members, s);
    case 128: return Forward<128>::run(phys, cols, out, tw, members, s);
    case 256: return Forward<256>::run(phys, cols, out, tw, members, s);
    case 512: return Forward<512>::run(phys, cols, out, tw, members, s);
    default: return cudaErrorInvalidValue;
    }
}

// Hermitian part of a full spectrum on the retained modes, compact layout [kx][j]
void to_compact(int n, const double *full, std::vector<cx<double>> &out, size_t at) {
    const int K = (n - 1) / 3, LD = 2 * K + 1;
    for (int kx = 0; kx <= K; ++kx)
        for (int j = 0; j < LD; ++j) {
            const int ky = j <= K ? j : j - LD;
            const size_t i = static_cast<size_t>((ky + n) % n) * n + kx;
            const size_t p = static_cast<size_t>((n - ky) % n) * n + (n - kx) % n;
            const std::complex<double> a(full[2 * i], full[2 * i + 1]), b(full[2 * p], full[2 * p + 1]);
            const std::complex<double> h = (kx == 0 && ky == 0) ? 0.0 : 0.5 * (a + std::conj(b));
            out[at + static_cast<size_t>(kx) * LD + j] = mk(h.real(), h.imag());
        }
}

void to_full(int n, const cx<double> *c, double *full) {
    const int K = (n - 1) / 3, LD = 2 * K + 1;
    std::fill(full, full + 2 * static_cast<size_t>(n) * n, 0.0);
    for (int kx = 0; kx <= K; ++kx)
        for (int j = 0; j < LD; ++j) {
            const int ky = j <= K ? j : j - LD;
            const cx<double> z = c[static_cast<size_t>(kx) * LD + j];
            const size_t i = static_cast<size_t>((ky + n) % n) * n + kx;
            full[2 * i] = z.x;
            full[2 * i + 1] = z.y;
            if (kx > 0) {
                const size_t p = static_cast<size_t>((n - ky) % n) * n + (n - kx);
                full[2 * p] = z.x;
                full[2 * p + 1] = -z.y;
            }
        }
}

void check_inputs(int n, const hzlb_parameters *p) {
    if (n < 8 || n > 512 || (n & (n - 1)))
        raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
    if (!p)
        raise(HZLB_EINVAL, "null parameters");
    if (!std::isfinite(p->viscosity) || p->viscosity < 0 || !std::isfinite(p->friction) ||
        p->friction < 0 || !std::isfinite(p->forcing_sigma) || p->forcing_sigma < 0 ||
        !std::isfinite(p->forcing_tau) || p->forcing_tau <= 0)
        raise(HZLB_EINVAL, "nu, alpha, sigma must be finite and nonnegative; tau must be positive");
    if (p->forcing_min < 1 || p->forcing_max < p->forcing_min ||
        3 * static_cast<long long>(p->forcing_max) >= static_cast<long long>(n))
        raise(HZLB_EINVAL, "forcing shell must lie strictly inside the dealiased grid");
}

// Restores the calling thread's current device when the call that selected another ends.
struct DeviceRestore {
    int previous = -1;
    DeviceRestore() {
        if (cudaGetDevice(&previous) != cudaSuccess)
            previous = -1;
    }
    ~DeviceRestore() {
        if (previous >= 0)
            cudaSetDevice(previous);
    }
};

// Device scratch for batched drifts of up to `capacity` members on an n x n grid, one stream.
// Every operation takes per-member viscosity and friction (device arrays).
class Workspace {
  public:
    Workspace(int n, int capacity, int device) : n_(n), cap_(capacity) {
        K_ = (n - 1) / 3;
        C_ = K_ + 1;
        LD_ = 2 * K_ + 1;
        per_ = static_cast<size_t>(C_) * LD_;
        nn_ = static_cast<size_t>(n) * n;
        cuda_check(cudaSetDevice(device), "select CUDA device");
        cuda_check(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking), "create stream");
        const size_t M = static_cast<size_t>(capacity);
        fields_.ensure(sizeof(cx<double>) * per_ * 8 * M, "allocate spectral fields");
        cols_.ensure(sizeof(cx<double>) * C_ * static_cast<size_t>(n) * 8 * M, "allocate columns");
        phys_.ensure(sizeof(double) * nn_ * 8 * M, "allocate physical fields");
        prod_.ensure(sizeof(double) * nn_ * 3 * M, "allocate products");
        spec_.ensure(sizeof(cx<double>) * per_ * 3 * M, "allocate product spectra");
        tw_.ensure(sizeof(cx<double>) * n, "allocate twiddles");
        std::vector<cx<double>> tw(n);
        for (int k = 0; k < n; ++k) {   // W_N^k, the construction of the reference's roots (fft.cpp:25-27)
            const double theta = -2.0 * kPi * static_cast<double>(k) / static_cast<double>(n);
            tw[k] = mk(std::cos(theta), std::sin(theta));
        }
        cuda_check(cudaMemcpyAsync(tw_.ptr, tw.data(), sizeof(cx<double>) * n, cudaMemcpyHostToDevice, s_),
                   "upload twiddles");
        cuda_check(cudaStreamSynchronize(s_), "upload twiddles");
    }
    ~Workspace() {
        if (s_) {
            cudaStreamSynchronize(s_);
            cudaStreamDestroy(s_);
        }
    }
    Workspace(const Workspace &) = delete;
    Workspace &operator=(const Workspace &) = delete;

    cudaStream_t stream() const { return s_; }
    size_t per() const { return per_; }
    size_t nn() const { return nn_; }
    int C() const { return C_; }
    int LD() const { return LD_; }
    int K() const { return K_; }
    const cx<double> *tw() const { return tw_.as<cx<double>>(); }
    int blocks(long long work) const {
        return static_cast<int>(std::max<long long>(1, std::min<long long>(148 * 8, (work + 255) / 256)));
    }

    // out = drift(x) = -F[u . grad x] - (nu k^2 + alpha) x, the reference's Solver::drift with no
    // forcing; with cfl_bits non-NULL the running CFL-rate maximum of each member is updated
    void drift(const cx<double> *x, int M, const double *nu, const double *alpha, cx<double> *out,
               unsigned long long *cfl_bits = nullptr) {
        OpTable t{};
        const int ops[4] = {OP_U, OP_V, OP_DX, OP_DY};
        std::copy(ops, ops + 4, t.op);
        t.count = 4;
        run(x, x, M, t, PRODUCT_DRIFT, 1, nu, alpha, 0, x, out, cfl_bits);
    }
    // Solver::linearized_drift(w, d)
    void tangent(const cx<double> *w, const cx<double> *d, int M, const double *nu,
                 const double *alpha, cx<double> *out) {
        OpTable t{};
        const int ops[8] = {OP_U, OP_V, OP_DX, OP_DY, OP_U, OP_V, OP_DX, OP_DY};
        const int src[8] = {1, 1, 0, 0, 0, 0, 1, 1};
        std::copy(ops, ops + 8, t.op);
        std::copy(src, src + 8, t.src);
        t.count = 8;
        run(w, d, M, t, PRODUCT_TANGENT, 1, nu, alpha, 0, d, out, nullptr);
    }
    // Solver::adjoint_drift(w, l)
    void adjoint(const cx<double> *w, const cx<double> *l, int M, const double *nu,
                 const double *alpha, cx<double> *out) {
        OpTable t{};
        const int ops[7] = {OP_U, OP_V, OP_DX, OP_DY, OP_ID, OP_DX, OP_DY};
        const int src[7] = {0, 0, 0, 0, 1, 1, 1};
        std::copy(ops, ops + 7, t.op);
        std::copy(src, src + 7, t.src);
        t.count = 7;
        run(w, l, M, t, PRODUCT_ADJOINT, 3, nu, alpha, 1, l, out, nullptr);
    }
    // physical field of x (the reference's physical_vorticity, real part): phys[m][y][x]
    const double *physical(const cx<double> *x, int M) {
        cuda_check(launch_physical<double>(n_, x, static_cast<long long>(per_), cols_.as<cx<double>>(),
                                           phys_.as<double>(), tw(), M, s_),
                   "launch inverse transforms");
        return phys_.as<double>();
    }

  private:
    void run(const cx<double> *a, const cx<double> *b, int M, const OpTable &t, int mode, int fout,
             const double *nu, const double *alpha, int adjoint, const cx<double> *second,
             cx<double> *out, unsigned long long *cfl_bits) {
        if (M > cap_)
            raise(HZLB_ERUNTIME, "drift batch exceeds the workspace");
        spectral_ops<<<blocks(static_cast<long long>(per_) * M), 256, 0, s_>>>(
            a, b, M, C_, LD_, K_, t, fields_.as<cx<double>>());
        cuda_check(cudaGetLastError(), "launch spectral operators");
        cuda_check(launch_physical<double>(n_, fields_.as<cx<double>>(), static_cast<long long>(per_),
                                           cols_.as<cx<double>>(), phys_.as<double>(), tw(),
                                           t.count * M, s_),
                   "launch inverse transforms");
        const long long cells = static_cast<long long>(nn_) * M;
        if (cfl_bits) {   // fields 0 and 1 are the velocity of the state
            cfl_rate_max<<<blocks(cells), 256, 0, s_>>>(phys_.as<double>(), cells,
                                                        static_cast<long long>(nn_), n_, cfl_bits);
            cuda_check(cudaGetLastError(), "launch CFL rate");
        }
        grid_products<<<blocks(cells), 256, 0, s_>>>(phys_.as<double>(), cells, mode, prod_.as<double>());
        cuda_check(cudaGetLastError(), "launch grid products");
        cuda_check(launch_forward(n_, prod_.as<double>(), cols_.as<cx<double>>(),
                                  spec_.as<cx<double>>(), tw(), fout * M, s_),
                   "launch forward transforms");
        combine<<<blocks(static_cast<long long>(per_) * M), 256, 0, s_>>>(
            spec_.as<cx<double>>(), second, M, C_, LD_, K_, nu, alpha, adjoint, out);
        cuda_check(cudaGetLastError(), "launch drift combination");
    }

    int n_, cap_, K_ = 0, C_ = 0, LD_ = 0;
    size_t per_ = 0, nn_ = 0;
    cudaStream_t s_ = nullptr;
    DeviceBuffer fields_, cols_, phys_, prod_, spec_, tw_;
};

// The pairs of the drop-in drift calls, in batches bounded by about 2 GB of device scratch.
void drift_batch(int n, const hzlb_parameters &p, const double *a_full, const double *b_full,
                 int count, bool adjoint, double *out_full, int device) {
    const size_t nn = static_cast<size_t>(n) * n;
    for (size_t i = 0; i < 2 * nn * count; ++i)
        if (!std::isfinite(a_full[i]) || !std::isfinite(b_full[i]))
            raise(HZLB_EINVAL, "nonfinite drift input");
    const int K = (n - 1) / 3, C = K + 1;
    const size_t per = static_cast<size_t>(C) * (2 * K + 1);
    const size_t bytes_per = sizeof(cx<double>) * per * 15 + sizeof(cx<double>) * C * n * 8 +
                             sizeof(double) * nn * 11;
    const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(count, (size_t{2} << 30) / bytes_per)));
    Workspace ws(n, chunk, device);
    DeviceBuffer dab, dres, dpar;
    dab.ensure(sizeof(cx<double>) * per * 2 * chunk, "allocate drift inputs");
    dres.ensure(sizeof(cx<double>) * per * chunk, "allocate drift");
    dpar.ensure(sizeof(double) * 2 * chunk, "allocate parameters");
    std::vector<double> par(2 * chunk);
    std::fill(par.begin(), par.begin() + chunk, p.viscosity);
    std::fill(par.begin() + chunk, par.end(), p.friction);
    cuda_check(cudaMemcpyAsync(dpar.ptr, par.data(), sizeof(double) * 2 * chunk, cudaMemcpyHostToDevice,
                               ws.stream()),
               "upload parameters");
    const double *nu = dpar.as<double>(), *alpha = nu + chunk;
    std::vector<cx<double>> host(per * 2 * chunk), res(per * chunk);
    for (int first = 0; first < count; first += chunk) {
        const int m = std::min(chunk, count - first);
        for (int i = 0; i < m; ++i) {
            to_compact(n, a_full + 2 * nn * (first + i), host, per * i);
            to_compact(n, b_full + 2 * nn * (first + i), host, per * (m + i));
        }
        cuda_check(cudaMemcpyAsync(dab.ptr, host.data(), sizeof(cx<double>) * per * 2 * m,
                                   cudaMemcpyHostToDevice, ws.stream()),
                   "upload drift inputs");
        const cx<double> *da = dab.as<cx<double>>(), *db = da + per * m;
        if (adjoint)
            ws.adjoint(da, db, m, nu, alpha, dres.as<cx<double>>());
        else
            ws.tangent(da, db, m, nu, alpha, dres.as<cx<double>>());
        cuda_check(cudaMemcpyAsync(res.data(), dres.ptr, sizeof(cx<double>) * per * m,
                                   cudaMemcpyDeviceToHost, ws.stream()),
                   "download drift");
        cuda_check(cudaStreamSynchronize(ws.stream()), "drift");
        for (int i = 0; i < m; ++i)
            to_full(n, res.data() + per * i, out_full + 2 * nn * (first + i));
    }
}

// ---- likelihood_adjoint (src/adjoint.cpp:43-161), batched over parameter vectors ---------
// Elementwise complex updates in the reference's association, each product and sum rounded
// separately as its CPU build evaluates them.
__device__ __forceinline__ cx<double> axpy(cx<double> x, double h, cx<double> k) {
    return mk(__dadd_rn(x.x, __dmul_rn(h, k.x)), __dadd_rn(x.y, __dmul_rn(h, k.y)));
}
// out = x + h k
__global__ void stage_input(const cx<double> *x, const cx<double> *k, double h, long long total,
                            cx<double> *out) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = axpy(x[i], h, k[i]);
}
// out = x + dt/6 (k1 + 2 k2 + 2 k3 + k4), with a nonfinite flag
__global__ void rk4_next(const cx<double> *x, const cx<double> *k1, const cx<double> *k2,
                         const cx<double> *k3, const cx<double> *k4, double dt, long long total,
                         cx<double> *out, int *nonfinite) {
    const double h = dt / 6;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        auto part = [&](double a, double b, double c, double d) {
            return __dadd_rn(__dadd_rn(__dadd_rn(a, __dmul_rn(2.0, b)), __dmul_rn(2.0, c)), d);
        };
        const cx<double> s = mk(part(k1[i].x, k2[i].x, k3[i].x, k4[i].x),
                                part(k1[i].y, k2[i].y, k3[i].y, k4[i].y));
        const cx<double> r = axpy(x[i], h, s);
        if (!(isfinite(r.x) && isfinite(r.y)))
            *nonfinite = 1;
        out[i] = r;
    }
}
// out = s x
__global__ void scale_field(const cx<double> *x, double s, long long total, cx<double> *out) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = mk(__dmul_rn(s, x[i].x), __dmul_rn(s, x[i].y));
}
// dst += s x
__global__ void add_field(cx<double> *dst, const cx<double> *x, double s, long long total) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        dst[i] = axpy(dst[i], s, x[i]);
}
// dst[m] = src for every member
__global__ void broadcast(const cx<double> *src, long long per, long long total, cx<double> *dst) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        dst[i] = src[i % per];
}
// The observations [o0, o1) of one step, in order, for every member: residual r = (field -
// value) / sd, objective += r^2 / 2, weight[o][m] = r / sd.
__global__ void observe_residuals(const double *phys, int M, long long nn, int n, const int *ox,
                                  const int *oy, const double *ov, const double *osd, int o0,
                                  int o1, double *objective, double *weight) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M)
        return;
    double acc = objective[m];
    for (int o = o0; o < o1; ++o) {
        const double field = phys[m * nn + static_cast<long long>(oy[o]) * n + ox[o]];
        const double r = __ddiv_rn(__dadd_rn(field, -ov[o]), osd[o]);
        acc = __dadd_rn(acc, __dmul_rn(__dmul_rn(0.5, r), r));
        weight[static_cast<long long>(o) * M + m] = __ddiv_rn(r, osd[o]);
    }
    objective[m] = acc;
}
// cotangent += the spectrum of the observation adjoint of one step on the active modes: the
// forward transform of sum_o weight_o n^2 delta(x_o, y_o), i.e. sum_o weight_o W_N^(kx x + ky y)
__global__ void inject_observations(cx<double> *cot, int M, int C, int LD, int K, int n,
                                    const int *ox, const int *oy, const double *weight, int o0,
                                    int o1, const cx<double> *tw) {
    const long long per = static_cast<long long>(C) * LD, total = per * M;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long m = i / per;
        const int kx = static_cast<int>((i % per) / LD), j = static_cast<int>(i % LD);
        const int ky = j <= K ? j : j - LD;
        if (kx == 0 && ky == 0)
            continue;
        cx<double> s = mk(0.0, 0.0);
        for (int o = o1 - 1; o >= o0; --o) {
            const int idx = ((kx * ox[o] + ky * oy[o]) % n + n) % n;
            const double w = weight[static_cast<long long>(o) * M + m];
            s = mk(s.x + w * tw[idx].x, s.y + w * tw[idx].y);
        }
        cot[i] = mk(cot[i].x + s.x, cot[i].y + s.y);
    }
}
// gradient[m] -= {nu sum k^2 Re(conj(w) s), alpha sum Re(conj(w) s)} over the whole spectrum
// (a kx > 0 entry stands for itself and its conjugate partner); one block per member
__global__ void parameter_contribution(const cx<double> *state, const cx<double> *weight, int C,
                                       int LD, int K, const double *nu, const double *alpha,
                                       double *gradient) {
    const int m = blockIdx.x;
    const long long per = static_cast<long long>(C) * LD;
    double s0 = 0, s1 = 0;
    for (long long i = threadIdx.x; i < per; i += blockDim.x) {
        const int kx = static_cast<int>(i / LD), j = static_cast<int>(i % LD);
        const int ky = j <= K ? j : j - LD;
        const cx<double> a = state[m * per + i], w = weight[m * per + i];
        const double inner = (kx > 0 ? 2.0 : 1.0) * (w.x * a.x + w.y * a.y);
        s0 += static_cast<double>(kx * kx + ky * ky) * inner;
        s1 += inner;
    }
    __shared__ double r0[256], r1[256];
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (static_cast<int>(threadIdx.x) < h) {
            r0[threadIdx.x] += r0[threadIdx.x + h];
            r1[threadIdx.x] += r1[threadIdx.x + h];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        gradient[2 * m] -= nu[m] * r0[0];
        gradient[2 * m + 1] -= alpha[m] * r1[0];
    }
}

// The reference's likelihood_adjoint for the parameter vectors `q` (count x 2: log nu, log
// alpha) that pass its range and stability checks, all advanced in lockstep (they share the
// dataset, so the steps, checkpoints and observation times are the same for all of them).
void likelihood_adjoint_batch(const hzlb_dataset *data, const double *q, int count, size_t stride,
                              int device, hzlb_adjoint_evaluation *out) {
    if (int rc = hzlb_dataset_validate(data))
        raise(rc, hzlb_last_error());
    if (data->stochastic || stride == 0)
        raise(HZLB_EINVAL,
              "adjoint requires deterministic data, two parameters, and positive checkpoint stride");
    const int n = data->n;
    if (n > 512)
        raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
    const double dt = data->dt;
    const hzlb_observation *obs = data->observations;
    const int nobs = static_cast<int>(data->count);
    std::vector<int> active;
    std::vector<double> nu_h, alpha_h;
    for (int i = 0; i < count; ++i) {
        out[i] = hzlb_adjoint_evaluation{};
        const double q0 = q[2 * i], q1 = q[2 * i + 1];
        bool inside = true;
        for (double v : {q0, q1})
            if (!std::isfinite(v) || v < -12 || v > 0)
                inside = false;
        if (!inside) {
            out[i].value = std::numeric_limits<double>::infinity();
            continue;
        }
        const double nu = std::exp(q0), alpha = std::exp(q1);
        const double largest = static_cast<double>((static_cast<size_t>(n) - 1) / 3);
        if (dt * (2 * nu * largest * largest + alpha) > 2.5) {
            out[i].value = std::numeric_limits<double>::infinity();
            continue;
        }
        active.push_back(i);
        nu_h.push_back(nu);
        alpha_h.push_back(alpha);
    }
    if (active.empty())
        return;
    const int M = static_cast<int>(active.size());

    // checkpoint steps and the block structure of the reverse pass
    const uint64_t last = obs[nobs - 1].step;
    std::vector<uint64_t> csteps{0};
    for (uint64_t st = 1; st <= last; ++st)
        if (st % stride == 0 || st == last)
            csteps.push_back(st);
    const size_t ncheck = csteps.size();
    size_t peak = 0, replayed = 0, longest = 0;
    for (size_t b = ncheck; b > 1; --b) {
        const size_t len = csteps[b - 1] - csteps[b - 2];
        replayed += 2 * len;
        peak = std::max(peak, len + 1);
        longest = std::max(longest, len);
    }

    Workspace ws(n, M, device);
    const cudaStream_t st = ws.stream();
    const size_t per = ws.per(), nn = ws.nn();
    const long long total = static_cast<long long>(per) * M;
    const int C = ws.C(), LD = ws.LD(), K = ws.K();
    const double storage = static_cast<double>(sizeof(cx<double>)) * per * M * (ncheck + longest + 1 + 18);
    if (storage > 64e9)
        raise(HZLB_EINVAL, "checkpoint storage exceeds the device budget; use a larger stride");
    const size_t fb = sizeof(cx<double>) * per * M;
    DeviceBuffer dpar, dfields, dstates, dchecks, dobs_i, dobs_d, dweights, dobj, dgrad, dcfl, dflag, dinit;
    dpar.ensure(sizeof(double) * 2 * M, "allocate parameters");
    enum { X, XN, Y, K1, K2, K3, K4, S2, S3, S4, COT, PREV, A1, A2, A3, A4, B, NF };
    dfields.ensure(fb * NF, "allocate adjoint fields");
    dstates.ensure(fb * (longest + 1), "allocate replayed states");
    dchecks.ensure(fb * ncheck, "allocate checkpoints");
    dobs_i.ensure(sizeof(int) * 2 * nobs, "allocate observation sites");
    dobs_d.ensure(sizeof(double) * 2 * nobs, "allocate observation values");
    dweights.ensure(sizeof(double) * static_cast<size_t>(nobs) * M, "allocate residual weights");
    dobj.ensure(sizeof(double) * M, "allocate objective");
    dgrad.ensure(sizeof(double) * 2 * M, "allocate gradient");
    dcfl.ensure(sizeof(unsigned long long) * M, "allocate CFL rates");
    dflag.ensure(sizeof(int), "allocate flag");
    dinit.ensure(sizeof(double) * nn + sizeof(cx<double>) * (static_cast<size_t>(C) * n + per),
                 "allocate initial field");
    auto field = [&](int f) { return dfields.as<cx<double>>() + static_cast<size_t>(f) * per * M; };
    auto state = [&](size_t s) { return dstates.as<cx<double>>() + s * per * M; };
    auto check = [&](size_t c) { return dchecks.as<cx<double>>() + c * per * M; };

    std::vector<double> par(2 * M);
    std::copy(nu_h.begin(), nu_h.end(), par.begin());
    std::copy(alpha_h.begin(), alpha_h.end(), par.begin() + M);
    std::vector<int> oi(2 * nobs);
    std::vector<double> od(2 * nobs);
    for (int o = 0; o < nobs; ++o) {
        oi[o] = static_cast<int>(obs[o].x);
        oi[nobs + o] = static_cast<int>(obs[o].y);
        od[o] = obs[o].value;
        od[nobs + o] = obs[o].standard_deviation;
    }
    cuda_check(cudaMemcpyAsync(dpar.ptr, par.data(), sizeof(double) * 2 * M, cudaMemcpyHostToDevice, st), "upload parameters");
    cuda_check(cudaMemcpyAsync(dobs_i.ptr, oi.data(), sizeof(int) * 2 * nobs, cudaMemcpyHostToDevice, st), "upload observations");
    cuda_check(cudaMemcpyAsync(dobs_d.ptr, od.data(), sizeof(double) * 2 * nobs, cudaMemcpyHostToDevice, st), "upload observations");
    cuda_check(cudaMemsetAsync(dobj.ptr, 0, sizeof(double) * M, st), "clear objective");
    cuda_check(cudaMemsetAsync(dgrad.ptr, 0, sizeof(double) * 2 * M, st), "clear gradient");
    cuda_check(cudaMemsetAsync(dcfl.ptr, 0, sizeof(unsigned long long) * M, st), "clear CFL rates");
    cuda_check(cudaMemsetAsync(dflag.ptr, 0, sizeof(int), st), "clear flag");
    const double *nu = dpar.as<double>(), *alpha = nu + M;
    const int *ox = dobs_i.as<int>(), *oy = ox + nobs;
    const double *ov = dobs_d.as<double>(), *osd = ov + nobs;
    int *flag = dflag.as<int>();
    const int eb = ws.blocks(total);

    // the initial "multimode" field (Solver::initialize, src/solver.cpp:145-160), projected
    {
        std::vector<double> w(nn);
        for (int y = 0; y < n; ++y)
            for (int x = 0; x < n; ++x) {
                const double a = 2 * kPi * static_cast<double>(x) / static_cast<double>(n),
                             b = 2 * kPi * static_cast<double>(y) / static_cast<double>(n);
                w[static_cast<size_t>(y) * n + x] = 2 * std::cos(a) * std::cos(b) +
                                                    0.6 * std::sin(2 * a + b) +
                                                    0.4 * std::cos(a - 3 * b) +
                                                    0.3 * std::sin(3 * a + 2 * b);
            }
        double *dphys = dinit.as<double>();
        cx<double> *dcols = reinterpret_cast<cx<double> *>(dphys + nn);
        cx<double> *dspec = dcols + static_cast<size_t>(C) * n;
        cuda_check(cudaMemcpyAsync(dphys, w.data(), sizeof(double) * nn, cudaMemcpyHostToDevice, st), "upload initial field");
        cuda_check(launch_forward(n, dphys, dcols, dspec, ws.tw(), 1, st), "transform initial field");
        cuda_check(cudaMemsetAsync(dspec, 0, sizeof(cx<double>), st), "project initial field");
        broadcast<<<eb, 256, 0, st>>>(dspec, static_cast<long long>(per), total, field(X));
        cuda_check(cudaGetLastError(), "launch broadcast");
    }
    auto copy = [&](cx<double> *dst, const cx<double> *src) {
        cuda_check(cudaMemcpyAsync(dst, src, fb, cudaMemcpyDeviceToDevice, st), "copy fields");
    };
    // rk4_stages (src/adjoint.cpp:12-32): stage inputs s2, s3, s4 and, with next, the new state
    auto stages = [&](const cx<double> *x, cx<double> *next, unsigned long long *cfl) {
        ws.drift(x, M, nu, alpha, field(K1), cfl);
        stage_input<<<eb, 256, 0, st>>>(x, field(K1), dt / 2, total, field(S2));
        ws.drift(field(S2), M, nu, alpha, field(K2));
        stage_input<<<eb, 256, 0, st>>>(x, field(K2), dt / 2, total, field(S3));
        ws.drift(field(S3), M, nu, alpha, field(K3));
        stage_input<<<eb, 256, 0, st>>>(x, field(K3), dt, total, field(S4));
        if (next) {
            ws.drift(field(S4), M, nu, alpha, field(K4));
            rk4_next<<<eb, 256, 0, st>>>(x, field(K1), field(K2), field(K3), field(K4), dt, total,
                                         next, flag);
        }
        cuda_check(cudaGetLastError(), "launch RK4 stages");
    };

    // forward pass: checkpoints and residuals (Solver::step checks the CFL rate of each state)
    copy(check(0), field(X));
    size_t ci = 1;
    int ob = 0;
    for (uint64_t step = 0; step <= last; ++step) {
        if (step > 0) {
            stages(field(X), field(XN), dcfl.as<unsigned long long>());
            copy(field(X), field(XN));
            if (step % stride == 0 || step == last)
                copy(check(ci++), field(X));
        }
        if (ob < nobs && obs[ob].step == step) {
            const int o0 = ob;
            while (ob < nobs && obs[ob].step == step)
                ++ob;
            const double *phys = ws.physical(field(X), M);
            observe_residuals<<<(M + 127) / 128, 128, 0, st>>>(phys, M, static_cast<long long>(nn), n,
                                                               ox, oy, ov, osd, o0, ob,
                                                               dobj.as<double>(), dweights.as<double>());
            cuda_check(cudaGetLastError(), "launch residuals");
        }
    }

    // reverse pass (src/adjoint.cpp:120-158)
    cuda_check(cudaMemsetAsync(field(COT), 0, fb, st), "clear cotangent");
    ob = nobs;
    for (size_t b = ncheck; b > 1; --b) {
        const uint64_t begin = csteps[b - 2], end = csteps[b - 1];
        copy(state(0), check(b - 2));
        for (uint64_t s2 = begin; s2 < end; ++s2)
            stages(state(s2 - begin), state(s2 - begin + 1), nullptr);
        for (uint64_t step = end; step > begin; --step) {
            if (ob > 0 && obs[ob - 1].step == step) {
                const int o1 = ob;
                while (ob > 0 && obs[ob - 1].step == step)
                    --ob;
                inject_observations<<<eb, 256, 0, st>>>(field(COT), M, C, LD, K, n, ox, oy,
                                                        dweights.as<double>(), ob, o1, ws.tw());
                cuda_check(cudaGetLastError(), "launch observation adjoint");
            }
            const cx<double> *x = state(step - begin - 1);
            stages(x, nullptr, nullptr);
            copy(field(PREV), field(COT));
            scale_field<<<eb, 256, 0, st>>>(field(COT), dt / 6, total, field(A1));
            scale_field<<<eb, 256, 0, st>>>(field(COT), dt / 3, total, field(A2));
            scale_field<<<eb, 256, 0, st>>>(field(COT), dt / 3, total, field(A3));
            scale_field<<<eb, 256, 0, st>>>(field(COT), dt / 6, total, field(A4));
            const cx<double> *stage_of[4] = {x, field(S2), field(S3), field(S4)};
            const int weight_of[4] = {A1, A2, A3, A4};
            for (int k = 3; k >= 0; --k) {   // fourth, third, second, first stage
                parameter_contribution<<<M, 256, 0, st>>>(stage_of[k], field(weight_of[k]), C, LD, K,
                                                          nu, alpha, dgrad.as<double>());
                ws.adjoint(stage_of[k], field(weight_of[k]), M, nu, alpha, field(B));
                add_field<<<eb, 256, 0, st>>>(field(PREV), field(B), 1.0, total);
                if (k > 0)
                    add_field<<<eb, 256, 0, st>>>(field(weight_of[k - 1]), field(B),
                                                  k == 3 ? dt : dt / 2, total);
                cuda_check(cudaGetLastError(), "launch adjoint stage");
            }
            copy(field(COT), field(PREV));
        }
    }

    std::vector<double> obj(M), grad(2 * M);
    std::vector<unsigned long long> cfl(M);
    int nonfinite = 0;
    cuda_check(cudaMemcpyAsync(obj.data(), dobj.ptr, sizeof(double) * M, cudaMemcpyDeviceToHost, st), "download objective");
    cuda_check(cudaMemcpyAsync(grad.data(), dgrad.ptr, sizeof(double) * 2 * M, cudaMemcpyDeviceToHost, st), "download gradient");
    cuda_check(cudaMemcpyAsync(cfl.data(), dcfl.ptr, sizeof(unsigned long long) * M, cudaMemcpyDeviceToHost, st), "download CFL rates");
    cuda_check(cudaMemcpyAsync(&nonfinite, dflag.ptr, sizeof(int), cudaMemcpyDeviceToHost, st), "download flag");
    cuda_check(cudaStreamSynchronize(st), "likelihood adjoint");
    for (int i = 0; i < M; ++i) {
        double rate;
        std::memcpy(&rate, &cfl[i], sizeof rate);
        if (dt * rate > 0.5)
            raise(HZLB_ERUNTIME, "time step exceeds conservative explicit stability limits; reduce dt");
    }
    if (nonfinite)
        raise(HZLB_ERUNTIME, "nonfinite flow state");
    for (int i = 0; i < M; ++i) {
        hzlb_adjoint_evaluation &r = out[active[i]];
        r.value = obj[i];
        r.gradient[0] = grad[2 * i];
        r.gradient[1] = grad[2 * i + 1];
        r.checkpoint_fields = ncheck;
        r.peak_block_fields = peak;
        r.replayed_steps = replayed;
    }
}

thread_local std::string tangent_error;
template <class F> int guarded(F &&f) {
    try {
        f();
        return HZLB_OK;
    } catch (const Error &e) {
        tangent_error = e.what();
        set_last_error(tangent_error);
        return e.code;
    } catch (const std::exception &e) {
        tangent_error = e.what();
        set_last_error(tangent_error);
        return HZLB_ERUNTIME;
    }
}

} // namespace
} // namespace hzlb

using namespace hzlb;

extern "C" {

HZLB_API int hzlb_linearized_drift(int n, const hzlb_parameters *params, const double *states,
                                   const double *directions, uint64_t count, int device,
                                   double *out) {
    return guarded([&] {
        check_inputs(n, params);
        if (count == 0)
            return;
        if (!states || !directions || !out)
            raise(HZLB_EINVAL, "null argument");
        if (count > (1u << 24))
            raise(HZLB_EINVAL, "too many drift pairs");
        DeviceRestore restore;
        drift_batch(n, *params, states, directions, static_cast<int>(count), false, out, device);
    });
}

HZLB_API int hzlb_likelihood_adjoint(const hzlb_dataset *data, const double *log_parameters,
                                     uint64_t count, uint64_t checkpoint_stride, int device,
                                     hzlb_adjoint_evaluation *out) {
    return guarded([&] {
        if (!data || (count && (!log_parameters || !out)))
            raise(HZLB_EINVAL, "null argument");
        if (count > (1u << 20))
            raise(HZLB_EINVAL, "too many parameter vectors");
        if (count == 0)
            return;
        DeviceRestore restore;
        likelihood_adjoint_batch(data, log_parameters, static_cast<int>(count),
                                 static_cast<size_t>(checkpoint_stride), device, out);
    });
}

HZLB_API int hzlb_adjoint_drift(int n, const hzlb_parameters *params, const double *states,
                                const double *cotangents, uint64_t count, int device,
                                double *out) {
    return guarded([&] {
        check_inputs(n, params);
        if (count == 0)
            return;
        if (!states || !cotangents || !out)
            raise(HZLB_EINVAL, "null argument");
        if (count > (1u << 24))
            raise(HZLB_EINVAL, "too many drift pairs");
        DeviceRestore restore;
        drift_batch(n, *params, states, cotangents, static_cast<int>(count), true, out, device);
    });
}

} // extern "C"
