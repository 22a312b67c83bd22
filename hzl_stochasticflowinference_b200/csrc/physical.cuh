// Spectral -> physical transforms and per-member reductions that sit beside the step:
// the observation operator (physical vorticity, reference Solver::physical_vorticity,
// src/solver.cpp:398-402), the CFL rate and the integral diagnostics (src/solver.cpp:381-397).
#pragma once
#include "spectral_step.cuh"

namespace hzlb {

// Inverse column FFT of one compact spectral field per (member, kx): out[m][kx][y].
template <typename R, int N>
__global__ void __launch_bounds__(Cfg<R, N>::COL_THREADS)
    field_column_inverse(const cx<R> *field, long long member_stride, cx<R> *out,
                         const cx<R> *tw_g) {
    using G = Cfg<R, N>;
    constexpr int E = G::E, T = G::T, C = G::C, LD = G::LD;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<R> *tw = reinterpret_cast<cx<R> *>(smem_raw);
    cx<R> *lines = tw + G::TWE;
    load_pass_twiddles<N, G::E, R>(tw, tw_g);
    __syncthreads();
    const int line = threadIdx.x / T, t = threadIdx.x % T;
    const int kx = blockIdx.y * G::LPB + line, m = blockIdx.x;
    const bool valid = kx < C;
    const int kxc = valid ? kx : 0;
    const cx<R> *src = field + static_cast<size_t>(m) * member_stride + static_cast<size_t>(kxc) * LD;
    cx<R> v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int j = compact_j<N>(t + r * T);
        v[r] = (valid && j >= 0) ? src[j] : mk<R>(0, 0);
    }
    fft_line<N, E, +1, R>(v, lines + line * G::BUF, tw, t);
    if (valid) {
        cx<R> *dst = out + (static_cast<size_t>(m) * C + kxc) * N;
#pragma unroll
        for (int r = 0; r < E; ++r)
            dst[t + r * T] = v[r];
    }
}

// Inverse row transforms of the column-pass output: rows (2g, 2g+1) packed into one complex
// transform; writes the real physical field phys[m][y][x].
template <typename R, int N>
__global__ void __launch_bounds__(Cfg<R, N>::ROW_THREADS)
    field_row_inverse(const cx<R> *cols, R *phys, const cx<R> *tw_g) {
    using G = Cfg<R, N>;
    constexpr int E = G::E, T = G::T, C = G::C, K = G::K, TY = G::TY;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<R> *tw = reinterpret_cast<cx<R> *>(smem_raw);
    cx<R> *lines = tw + G::TWE;
    load_pass_twiddles<N, G::E, R>(tw, tw_g);
    __syncthreads();
    const int g = threadIdx.x / T, t = threadIdx.x % T, m = blockIdx.x;
    const bool active = g < TY / 2;
    const int ya = blockIdx.y * TY + (active ? 2 * g : 0);
    const cx<R> *src = cols + static_cast<size_t>(m) * C * N;
    cx<R> z[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int p = t + r * T;
        cx<R> za = mk<R>(0, 0), zb = mk<R>(0, 0);
        if (p <= K) {
            za = src[static_cast<size_t>(p) * N + ya];
            zb = src[static_cast<size_t>(p) * N + ya + 1];
            if (p == 0) {
                za.y = 0;
                zb.y = 0;
            }
        } else if (p >= N - K) {
            za = conj(src[static_cast<size_t>(N - p) * N + ya]);
            zb = conj(src[static_cast<size_t>(N - p) * N + ya + 1]);
        }
        z[r] = mk<R>(za.x - zb.y, za.y + zb.x);
    }
    fft_line<N, E, +1, R>(z, lines + g * G::BUF, tw, t);
    if (active) {
        R *da = phys + (static_cast<size_t>(m) * N + ya) * N;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            da[t + r * T] = z[r].x;
            da[N + t + r * T] = z[r].y;
        }
    }
}

// max over the grid of |u| + |v| per member from the velocity rows W ([m][y][field][kx]),
// written as the bit pattern of a nonnegative double (monotone as an unsigned integer).
template <typename R, int N>
__global__ void __launch_bounds__(Cfg<R, N>::ROW_THREADS)
    velocity_max(const cx<R> *w, unsigned long long *vmax_bits, const cx<R> *tw_g) {
    using G = Cfg<R, N>;
    constexpr int E = G::E, T = G::T, K = G::K, TY = G::TY;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<R> *tw = reinterpret_cast<cx<R> *>(smem_raw);
    cx<R> *lines = tw + G::TWE;
    load_pass_twiddles<N, G::E, R>(tw, tw_g);
    __syncthreads();
    const int g = threadIdx.x / T, t = threadIdx.x % T, m = blockIdx.x;
    const bool active = g < TY / 2;
    const cx<R> *wm = w + static_cast<size_t>(m) * N * 2 * G::CW;   // rows [y][field][kx]
    double best = 0;
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
        const int y = blockIdx.y * TY + (active ? 2 * g + h : 0);
        const cx<R> *u = wm + static_cast<size_t>(y) * 2 * G::CW, *v = u + G::CW;
        cx<R> z[E];
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int p = t + r * T;
            cx<R> za = mk<R>(0, 0), zb = mk<R>(0, 0);
            if (p <= K) {
                za = u[p];
                zb = v[p];
                if (p == 0) {
                    za.y = 0;
                    zb.y = 0;
                }
            } else if (p >= N - K) {
                za = conj(u[N - p]);
                zb = conj(v[N - p]);
            }
            z[r] = mk<R>(za.x - zb.y, za.y + zb.x);
        }
        fft_line<N, E, +1, R>(z, lines + g * G::BUF, tw, t);
#pragma unroll
        for (int r = 0; r < E; ++r)
            best = fmax(best, static_cast<double>(fabs(z[r].x)) + static_cast<double>(fabs(z[r].y)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        best = fmax(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0)
        atomicMax(vmax_bits + m, static_cast<unsigned long long>(__double_as_longlong(best)));
}

// Energy, enstrophy and forcing injection per member (solver.cpp:384-391) from the compact
// half-spectrum: the kx = 0 column holds both +ky and -ky; every kx > 0 entry stands for
// itself and its conjugate partner, so it counts twice.  out[m] = {E, Z, I}.
template <typename R>
__global__ void integral_diagnostics(const cx<R> *omega, const cx<R> *forcing,
                                     long long forcing_stride, int forcing_cols, int n,
                                     double *out) {
    const int K = (n - 1) / 3, C = K + 1, LD = 2 * K + 1, m = blockIdx.x;
    const double area = 4.0 * 3.141592653589793238462643383279502884 * 3.141592653589793238462643383279502884;
    double e = 0, z = 0, inj = 0;
    const cx<R> *w = omega + static_cast<size_t>(m) * C * LD;
    for (int i = threadIdx.x; i < C * LD; i += blockDim.x) {
        const int kx = i / LD, j = i % LD, ky = j <= K ? j : j - LD;
        const double k2 = static_cast<double>(kx * kx + ky * ky);
        if (k2 == 0)
            continue;
        const double mult = kx == 0 ? 1.0 : 2.0;
        const double wr = w[i].x, wi = w[i].y, norm = wr * wr + wi * wi;
        e += mult * (area / 2 * norm / k2);
        z += mult * (area / 2 * norm);
        if (forcing && kx < forcing_cols) {
            const cx<R> f = forcing[static_cast<size_t>(m) * forcing_stride + i];
            inj += mult * (area * (wr * static_cast<double>(f.x) + wi * static_cast<double>(f.y)) / k2);
        }
    }
    __shared__ double red[3][32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        z += __shfl_xor_sync(0xffffffffu, z, o);
        inj += __shfl_xor_sync(0xffffffffu, inj, o);
    }
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) {
        red[0][warp] = e;
        red[1][warp] = z;
        red[2][warp] = inj;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0, s1 = 0, s2 = 0;
        for (int i = 0; i < static_cast<int>(blockDim.x / 32); ++i) {
            s0 += red[0][i];
            s1 += red[1][i];
            s2 += red[2][i];
        }
        out[3 * m + 0] = s0;
        out[3 * m + 1] = s1;
        out[3 * m + 2] = s2;
    }
}

// Inverse row transforms of the listed row pairs only (rows 2 q_i and 2 q_i + 1 for each
// entry q_i of pairs, the pairs that observation rows lie in), packed two rows per complex
// transform exactly as field_row_inverse packs them, so every value equals the full
// transform's: out[m][2 i + h][x], h = 0, 1.
template <typename R, int N>
__global__ void __launch_bounds__(Cfg<R, N>::ROW_THREADS)
    field_row_pairs_inverse(const cx<R> *cols, const int *pairs, int npairs, R *out,
                            const cx<R> *tw_g) {
    using G = Cfg<R, N>;
    constexpr int E = G::E, T = G::T, C = G::C, K = G::K, TY = G::TY;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    cx<R> *tw = reinterpret_cast<cx<R> *>(smem_raw);
    cx<R> *lines = tw + G::TWE;
    load_pass_twiddles<N, G::E, R>(tw, tw_g);
    __syncthreads();
    const int g = threadIdx.x / T, t = threadIdx.x % T, m = blockIdx.x;
    const int q = blockIdx.y * (TY / 2) + g;
    const bool active = g < TY / 2 && q < npairs;
    const int ya = active ? 2 * pairs[q] : 0;
    const cx<R> *src = cols + static_cast<size_t>(m) * C * N;
    cx<R> z[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int pos = t + r * T;
        cx<R> za = mk<R>(0, 0), zb = mk<R>(0, 0);
        if (pos <= K) {
            za = src[static_cast<size_t>(pos) * N + ya];
            zb = src[static_cast<size_t>(pos) * N + ya + 1];
            if (pos == 0) {
                za.y = 0;
                zb.y = 0;
            }
        } else if (pos >= N - K) {
            za = conj(src[static_cast<size_t>(N - pos) * N + ya]);
            zb = conj(src[static_cast<size_t>(N - pos) * N + ya + 1]);
        }
        z[r] = mk<R>(za.x - zb.y, za.y + zb.x);
    }
    fft_line<N, E, +1, R>(z, lines + g * G::BUF, tw, t);
    if (active) {
        R *da = out + (static_cast<size_t>(m) * npairs + q) * 2 * N;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            da[t + r * T] = z[r].x;
            da[N + t + r * T] = z[r].y;
        }
    }
}

// Sample rows of physical fields at p points: out[m][o] = rows[m][slot_o][x_o].
template <typename R>
__global__ void gather_rows(const R *rows, int nrows, int n, const unsigned *xs,
                            const unsigned *slots, int p, int members, double *out) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(members) * p)
        return;
    const int m = static_cast<int>(i / p), o = static_cast<int>(i % p);
    out[i] = rows[(static_cast<size_t>(m) * nrows + slots[o]) * n + xs[o]];
}

// Sample the physical fields at p points: out[m][o] = phys[m][y_o][x_o].
template <typename R>
__global__ void gather_points(const R *phys, int n, const unsigned *xs, const unsigned *ys, int p,
                              int members, double *out) {
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<long long>(members) * p)
        return;
    const int m = static_cast<int>(i / p), o = static_cast<int>(i % p);
    out[i] = phys[(static_cast<size_t>(m) * n + ys[o]) * n + xs[o]];
}

} // namespace hzlb
