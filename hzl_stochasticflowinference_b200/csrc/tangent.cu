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
// tangent: fields {u_d, v_d, w_x, w_y, u, v, d_x, d_y} -> {u_d w_x + v_d w_y + u d_x + v d_y}
// adjoint: fields {u, v, w_x, w_y, L, L_x, L_y}       -> {u L_x + v L_y, L w_x, L w_y}
__global__ void grid_products(const double *phys, long long cells, int adjoint, double *out) {
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < cells;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double *f = phys + i;
        auto at = [&](int k) { return f[k * cells]; };
        if (!adjoint) {
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
                        int LD, int K, double nu, double alpha, int adjoint, cx<double> *out) {
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
        const double k2 = static_cast<double>(k2i), rate = nu * k2 + alpha;
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

struct StreamGuard {
    cudaStream_t s = nullptr;
    ~StreamGuard() {
        if (s)
            cudaStreamDestroy(s);
    }
};

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

// One batch of pairs on the device: spectral operators -> physical fields -> products ->
// forward transforms -> drift.
void drift_batch(int n, const hzlb_parameters &p, const double *a_full, const double *b_full,
                 int count, bool adjoint, double *out_full, int device) {
    const int K = (n - 1) / 3, C = K + 1, LD = 2 * K + 1;
    const size_t per = static_cast<size_t>(C) * LD, nn = static_cast<size_t>(n) * n;
    for (size_t i = 0; i < 2 * nn * count; ++i)
        if (!std::isfinite(a_full[i]) || !std::isfinite(b_full[i]))
            raise(HZLB_EINVAL, "nonfinite drift input");
    cuda_check(cudaSetDevice(device), "select CUDA device");
    OpTable t{};
    int fout;
    if (!adjoint) {   // {u_d, v_d, w_x, w_y, u, v, d_x, d_y}
        const int ops[8] = {OP_U, OP_V, OP_DX, OP_DY, OP_U, OP_V, OP_DX, OP_DY};
        const int src[8] = {1, 1, 0, 0, 0, 0, 1, 1};
        std::copy(ops, ops + 8, t.op);
        std::copy(src, src + 8, t.src);
        t.count = 8;
        fout = 1;
    } else {          // {u, v, w_x, w_y, L, L_x, L_y}
        const int ops[7] = {OP_U, OP_V, OP_DX, OP_DY, OP_ID, OP_DX, OP_DY};
        const int src[7] = {0, 0, 0, 0, 1, 1, 1};
        std::copy(ops, ops + 7, t.op);
        std::copy(src, src + 7, t.src);
        t.count = 7;
        fout = 3;
    }
    // batch size bounded by about 2 GB of device scratch
    const size_t bytes_per = sizeof(cx<double>) * per * (2 + t.count + fout + 1) +
                             sizeof(cx<double>) * C * static_cast<size_t>(n) * t.count +
                             sizeof(double) * nn * (t.count + fout);
    const int chunk = static_cast<int>(std::max<size_t>(1, std::min<size_t>(count, (size_t{2} << 30) / bytes_per)));
    StreamGuard sg;
    cuda_check(cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking), "create stream");
    DeviceBuffer dab, dfields, dcols, dphys, dprod, dspec, dres, dtw;
    dab.ensure(sizeof(cx<double>) * per * 2 * chunk, "allocate drift inputs");
    dfields.ensure(sizeof(cx<double>) * per * t.count * chunk, "allocate spectral fields");
    dcols.ensure(sizeof(cx<double>) * C * static_cast<size_t>(n) * t.count * chunk, "allocate columns");
    dphys.ensure(sizeof(double) * nn * t.count * chunk, "allocate physical fields");
    dprod.ensure(sizeof(double) * nn * fout * chunk, "allocate products");
    dspec.ensure(sizeof(cx<double>) * per * fout * chunk, "allocate product spectra");
    dres.ensure(sizeof(cx<double>) * per * chunk, "allocate drift");
    dtw.ensure(sizeof(cx<double>) * n, "allocate twiddles");
    std::vector<cx<double>> tw(n);
    for (int k = 0; k < n; ++k) {   // W_N^k, the construction of the reference's roots (fft.cpp:25-27)
        const double theta = -2.0 * kPi * static_cast<double>(k) / static_cast<double>(n);
        tw[k] = mk(std::cos(theta), std::sin(theta));
    }
    cuda_check(cudaMemcpyAsync(dtw.ptr, tw.data(), sizeof(cx<double>) * n, cudaMemcpyHostToDevice, sg.s),
               "upload twiddles");
    std::vector<cx<double>> host(per * 2 * chunk), res(per * chunk);
    for (int first = 0; first < count; first += chunk) {
        const int m = std::min(chunk, count - first);
        for (int i = 0; i < m; ++i) {
            to_compact(n, a_full + 2 * nn * (first + i), host, per * i);
            to_compact(n, b_full + 2 * nn * (first + i), host, per * (m + i));
        }
        cuda_check(cudaMemcpyAsync(dab.ptr, host.data(), sizeof(cx<double>) * per * 2 * m,
                                   cudaMemcpyHostToDevice, sg.s),
                   "upload drift inputs");
        const cx<double> *da = dab.as<cx<double>>(), *db = da + per * m;
        const int threads = 256;
        const int blocks = static_cast<int>(std::min<long long>(148 * 8, (static_cast<long long>(per) * m + threads - 1) / threads));
        spectral_ops<<<blocks, threads, 0, sg.s>>>(da, db, m, C, LD, K, t, dfields.as<cx<double>>());
        cuda_check(cudaGetLastError(), "launch spectral operators");
        cuda_check(launch_physical<double>(n, dfields.as<cx<double>>(), static_cast<long long>(per),
                                           dcols.as<cx<double>>(), dphys.as<double>(),
                                           dtw.as<cx<double>>(), t.count * m, sg.s),
                   "launch inverse transforms");
        const long long cells = static_cast<long long>(nn) * m;
        const int pblocks = static_cast<int>(std::min<long long>(148 * 8, (cells + threads - 1) / threads));
        grid_products<<<pblocks, threads, 0, sg.s>>>(dphys.as<double>(), cells, adjoint ? 1 : 0,
                                                     dprod.as<double>());
        cuda_check(cudaGetLastError(), "launch grid products");
        cuda_check(launch_forward(n, dprod.as<double>(), dcols.as<cx<double>>(),
                                  dspec.as<cx<double>>(), dtw.as<cx<double>>(), fout * m, sg.s),
                   "launch forward transforms");
        combine<<<blocks, threads, 0, sg.s>>>(dspec.as<cx<double>>(), db, m, C, LD, K,
                                              p.viscosity, p.friction, adjoint ? 1 : 0,
                                              dres.as<cx<double>>());
        cuda_check(cudaGetLastError(), "launch drift combination");
        cuda_check(cudaMemcpyAsync(res.data(), dres.ptr, sizeof(cx<double>) * per * m,
                                   cudaMemcpyDeviceToHost, sg.s),
                   "download drift");
        cuda_check(cudaStreamSynchronize(sg.s), "drift");
        for (int i = 0; i < m; ++i)
            to_full(n, res.data() + per * i, out_full + 2 * nn * (first + i));
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
        drift_batch(n, *params, states, directions, static_cast<int>(count), false, out, device);
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
        drift_batch(n, *params, states, cotangents, static_cast<int>(count), true, out, device);
    });
}

} // extern "C"
