// Batched pseudo-spectral RK4 step for the 2-D periodic vorticity equation
//   d(w)/dt = -u.grad(w) + nu lap(w) - alpha w + f,   lap(psi) = -w,  u = psi_y, v = -psi_x
// restating the math of the reference's Solver::rhs/step (src/solver.cpp:177-254) and
// CudaSolver (src/cuda_solver.cu:26-84, 203-218) for thousands of members at once.
//
// The advection term is evaluated in Basdevant's form for 2-D incompressible flow,
//   u.grad(w) = d2/dxdy (v^2 - u^2) + (d2/dx2 - d2/dy2)(u v),
// i.e. A^(k) = -kx ky F[v^2 - u^2] - (kx^2 - ky^2) F[u v].  With the strict 2/3 truncation the
// products are alias-free on the retained modes, so this equals the reference's
// F[u wx + v wy] there (to roundoff) while needing four real transforms per stage instead of
// five: inverse u, v (one packed complex transform per row) and forward v^2 - u^2, u v (one
// packed complex transform per row).
//
// One RK stage is two kernels:
//   column kernel  (per member x kx column): forward column FFTs of the two product spectra,
//                  RK stage epilogue (dealias mask, viscosity/friction, forcing, accumulator,
//                  noise on the last stage), then u^ = i ky psi^, v^ = -i kx psi^ of the next
//                  stage input and their inverse column FFTs;
//   row kernel     (per member x tile of y rows): inverse row FFT of u + i v, the products
//                  v^2 - u^2 and u v, the CFL check on stage 1, and the forward row FFT of
//                  (v^2 - u^2) + i (u v), keeping kx = 0..K of each.
// HBM layouts (complex R):
//   state / stage input / accumulator  [m][kx][j]          (K+1) x (2K+1) per member
//   velocity columns W                 [m][field][kx][y]   2 x (K+1) x N   (u^, v^)
//   product rows NL                    [m][field][kx][y]   2 x (K+1) x N   (v^2-u^2, u v)
#pragma once
#include "fft.cuh"

namespace hzlb {

// E (elements per thread) keeps a line inside one warp; FP64 uses fewer registers per thread.
template <typename R, int N> struct Cfg {
    static constexpr int E = sizeof(R) == 4 ? (N < 16 ? N : 16) : (N <= 256 ? (N < 8 ? N : 8) : 16);
    static constexpr int T = N / E;
    static constexpr int K = (N - 1) / 3;
    static constexpr int C = K + 1;          // retained kx columns
    static constexpr int LD = 2 * K + 1;     // compact column length
    static constexpr int LPB = T >= 64 ? 1 : 64 / T;  // column lines per block
    static constexpr int COL_THREADS = LPB * T;
    static constexpr int TY_RAW = 128 / T;   // rows per row-kernel block, one row per group
    static constexpr int TY = TY_RAW > N ? N : (TY_RAW < 2 ? 2 : TY_RAW);
    static constexpr int GROUPS = TY * T >= 32 ? TY : 32 / T;
    static constexpr int ROW_THREADS = GROUPS * T;
    static constexpr int SC = C | 1;         // odd row stride of the W tile (bank spread)
    static constexpr int BUF = N + N / E;
};

struct StepControl {
    unsigned long long step;   // index of the step being taken (noise counter)
    unsigned int arrivals;     // column-kernel block arrivals on the final stage
    unsigned int status;       // STATUS_* bits
};

template <typename R> struct ColumnArgs {
    const cx<R> *nl;        // [M][2][C][N]
    cx<R> *w;               // [M][2][C][N]
    cx<R> *omega;           // [M][C][LD]
    cx<R> *ystage;          // [M][C][LD]
    cx<R> *acc;             // [M][C][LD]
    const cx<R> *forcing;   // [.][fcols][LD]
    long long forcing_stride;  // elements between members (0: shared)
    int forcing_cols;       // forcing present for kx < forcing_cols
    const cx<R> *tw;        // N twiddles
    double nu, alpha, dt;
    int stage;              // 0 start, 1..3 intermediate, 4 final
    int emit;               // write W (derivative columns) for the next stage input
    double noise_scale;     // sigma sqrt(dt)/sqrt(2); 0 disables
    int noise_kmax2;
    unsigned long long seed;
    unsigned int member_base;
    StepControl *ctl;
    int members;
};

template <typename R> struct RowArgs {
    const cx<R> *w;       // [M][2][C][N]
    cx<R> *nl;            // [M][2][C][N]
    const cx<R> *tw;
    double cfl_scale;     // dt * N / (2 pi); > 0 enables the stage-1 CFL check
    StepControl *ctl;
    int members;
};

// Compact index j of FFT position p in a column (or -1 if p is outside the retained band).
template <int N> __device__ __forceinline__ int compact_j(int p) {
    constexpr int K = (N - 1) / 3, LD = 2 * K + 1;
    return p <= K ? p : (p >= N - K ? p - (N - LD) : -1);
}

template <typename R, int N>
__global__ void __launch_bounds__(Cfg<R, N>::COL_THREADS)
    column_kernel(const ColumnArgs<R> a) {
    using G = Cfg<R, N>;
    constexpr int E = G::E, T = G::T, C = G::C, LD = G::LD, K = G::K;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R> *tw = reinterpret_cast<cx<R> *>(smem_raw);
    cx<R> *lines = tw + N;
    for (int i = threadIdx.x; i < N; i += blockDim.x)
        tw[i] = a.tw[i];
    __shared__ unsigned long long step_sh;
    if (threadIdx.x == 0)
        step_sh = a.ctl->step;
    __syncthreads();

    const int line = threadIdx.x / T, t = threadIdx.x % T;
    const int kx = blockIdx.y * G::LPB + line;
    const int m = blockIdx.x;
    const bool valid = kx < C;
    const int kxc = valid ? kx : 0;
    cx<R> *sm = lines + line * G::BUF;
    const size_t cbase = (static_cast<size_t>(m) * C + kxc) * LD;
    const R kxr = static_cast<R>(kxc);

    cx<R> y[E];   // next stage input at this thread's positions (zero outside the band)
    cx<R> v[E];
    if (a.stage == 0) {
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int j = compact_j<N>(t + r * T);
            y[r] = (valid && j >= 0) ? a.omega[cbase + j] : mk<R>(0, 0);
        }
    } else {
        // forward column FFTs of the product spectra (unnormalised; 1/N^2 below):
        // A^ = -kx ky P^ - (kx^2 - ky^2) Q^ with P = v^2 - u^2, Q = u v
        const cx<R> *src = a.nl + (static_cast<size_t>(m) * 2 * C + kxc) * N;
        cx<R> adv[E];
#pragma unroll
        for (int r = 0; r < E; ++r)
            v[r] = valid ? src[t + r * T] : mk<R>(0, 0);
        fft_line<N, E, -1, R>(v, sm, tw, t);
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int j = compact_j<N>(t + r * T);
            const int ky = j <= K ? j : j - LD;
            adv[r] = scale(static_cast<R>(-kxc * ky), v[r]);
        }
#pragma unroll
        for (int r = 0; r < E; ++r)
            v[r] = valid ? src[static_cast<size_t>(C) * N + t + r * T] : mk<R>(0, 0);
        fft_line<N, E, -1, R>(v, sm, tw, t);
        const R inv_n2 = static_cast<R>(1.0 / (static_cast<double>(N) * N));
        const R nu = static_cast<R>(a.nu), alpha = static_cast<R>(a.alpha),
                dt = static_cast<R>(a.dt);
        bool bad = false;
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int j = compact_j<N>(t + r * T);
            y[r] = mk<R>(0, 0);
            if (!valid || j < 0)
                continue;
            const int ky = j <= K ? j : j - LD;
            const R k2 = static_cast<R>(kxc * kxc + ky * ky);
            const size_t idx = cbase + j;
            const cx<R> wn = a.omega[idx];
            const cx<R> ys = a.stage == 1 ? wn : a.ystage[idx];
            // rhs: active ? -A^ - (nu k^2 + alpha) w + f : 0   (solver.cpp:197-202)
            cx<R> k = mk<R>(0, 0);
            if (!(kxc == 0 && j == 0)) {
                const cx<R> nl = scale(inv_n2, adv[r] - scale(static_cast<R>(kxc * kxc - ky * ky), v[r]));
                const R rate = nu * k2 + alpha;
                k = mk<R>(-nl.x, -nl.y) - scale(rate, ys);
                if (kxc < a.forcing_cols)
                    k = k + a.forcing[static_cast<size_t>(m) * a.forcing_stride +
                                      static_cast<size_t>(kxc) * LD + j];
            }
            if (a.stage == 1) {
                a.acc[idx] = k;
                y[r] = wn + scale(dt / 2, k);
                a.ystage[idx] = y[r];
            } else if (a.stage == 2) {
                a.acc[idx] = a.acc[idx] + scale(static_cast<R>(2.0), k);
                y[r] = wn + scale(dt / 2, k);
                a.ystage[idx] = y[r];
            } else if (a.stage == 3) {
                a.acc[idx] = a.acc[idx] + scale(static_cast<R>(2.0), k);
                y[r] = wn + scale(dt, k);
                a.ystage[idx] = y[r];
            } else {
                // w += dt/6 (k1 + 2 k2 + 2 k3 + k4)   (solver.cpp:233-234)
                cx<R> w1 = wn + scale(dt / 6, a.acc[idx] + k);
                if (a.noise_scale > 0 && kxc * kxc + ky * ky >= 1 &&
                    kxc * kxc + ky * ky <= a.noise_kmax2) {
                    double xi1, xi2;
                    const bool rep = kxc > 0 || ky > 0;
                    philox_normal_pair(a.seed, a.member_base + m, step_sh,
                                       mode_code(kxc, rep ? ky : -ky), xi1, xi2);
                    const double s = a.noise_scale;
                    w1 = w1 + mk<R>(static_cast<R>(s * xi1),
                                    static_cast<R>(rep ? s * xi2 : -(s * xi2)));
                }
                bad |= !(isfinite(w1.x) && isfinite(w1.y));
                a.omega[idx] = w1;
                y[r] = w1;
            }
        }
        if (bad)
            atomicOr(&a.ctl->status, STATUS_NONFINITE);
    }

    if (a.emit) {
        // velocity of the next stage input (solver.cpp:177-185): u^ = i ky psi^,
        // v^ = -i kx psi^ with psi^ = w^/k^2, then inverse column FFTs
        cx<R> *dst = a.w + (static_cast<size_t>(m) * 2 * C + kxc) * N;
#pragma unroll 1
        for (int f = 0; f < 2; ++f) {
#pragma unroll
            for (int r = 0; r < E; ++r) {
                const int j = compact_j<N>(t + r * T);
                cx<R> z = mk<R>(0, 0);
                if (j >= 0) {
                    const int ky = j <= K ? j : j - LD;
                    const R kyr = static_cast<R>(ky);
                    const R k2 = static_cast<R>(kxc * kxc + ky * ky);
                    const cx<R> psi = k2 > 0 ? mk<R>(y[r].x / k2, y[r].y / k2) : mk<R>(0, 0);
                    z = f == 0 ? mk<R>(-kyr * psi.y, kyr * psi.x) : mk<R>(kxr * psi.y, -kxr * psi.x);
                }
                v[r] = z;
            }
            fft_line<N, E, +1, R>(v, sm, tw, t);
            if (valid) {
#pragma unroll
                for (int r = 0; r < E; ++r)
                    dst[static_cast<size_t>(f) * C * N + t + r * T] = v[r];
            }
        }
    }

    if (a.stage == 4) {
        // the last block to finish advances the device step counter (every block read it
        // before arriving, so no block sees the new value)
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            const unsigned total = gridDim.x * gridDim.y;
            const unsigned prev = atomicAdd(&a.ctl->arrivals, 1u);
            if (prev == total - 1) {
                a.ctl->arrivals = 0;
                a.ctl->step = step_sh + 1;
                __threadfence();
            }
        }
    }
}

// Inverse row transform of two real fields packed as a + i b.  A and B hold the x-spectra of
// the row for kx = 0..K (column-pass output); negative kx follow from the fields being real
// (A(-kx) = conj A(kx)), and the kx = 0 entries are real (imaginary roundoff dropped, as the
// reference keeps only the real part of its inverse transforms).  On exit z = a + i b at
// the thread's x positions.
template <int N, int E, typename R>
__device__ __forceinline__ void packed_row_inverse(cx<R> (&z)[E], const cx<R> *A, const cx<R> *B,
                                                   cx<R> *sm, const cx<R> *tw, int t) {
    constexpr int T = N / E, K = (N - 1) / 3;
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const int p = t + r * T;
        cx<R> za = mk<R>(0, 0), zb = mk<R>(0, 0);
        if (p <= K) {
            za = A[p];
            zb = B[p];
            if (p == 0) {
                za.y = 0;
                zb.y = 0;
            }
        } else if (p >= N - K) {
            za = conj(A[N - p]);
            zb = conj(B[N - p]);
        }
        z[r] = mk<R>(za.x - zb.y, za.y + zb.x);
    }
    fft_line<N, E, +1, R>(z, sm, tw, t);
}

template <typename R, int N>
__global__ void __launch_bounds__(Cfg<R, N>::ROW_THREADS) row_kernel(const RowArgs<R> a) {
    using G = Cfg<R, N>;
    constexpr int E = G::E, T = G::T, C = G::C, K = G::K, TY = G::TY, SC = G::SC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<R> *tw = reinterpret_cast<cx<R> *>(smem_raw);
    cx<R> *wt = tw + N;                      // [2][TY][SC]
    cx<R> *nlt = wt + 2 * TY * SC;           // [2][C][TY+1]
    cx<R> *lines = nlt + 2 * C * (TY + 1);   // [GROUPS][BUF]
    const int m = blockIdx.x, y0 = blockIdx.y * TY;
    for (int i = threadIdx.x; i < N; i += blockDim.x)
        tw[i] = a.tw[i];
    // load the velocity tile: for each (field, kx) a run of TY consecutive rows
    const cx<R> *src = a.w + static_cast<size_t>(m) * 2 * C * N;
    for (int i = threadIdx.x; i < 2 * C * TY; i += blockDim.x) {
        const int ty = i % TY, fk = i / TY, f = fk / C, kx = fk % C;
        wt[(f * TY + ty) * SC + kx] = src[static_cast<size_t>(fk) * N + y0 + ty];
    }
    __syncthreads();

    const int g = threadIdx.x / T, t = threadIdx.x % T;
    const bool active = g < TY;
    const int ty = active ? g : 0;
    cx<R> *sm = lines + g * G::BUF;
    cx<R> z[E];
    packed_row_inverse<N, E, R>(z, wt + (0 * TY + ty) * SC, wt + (1 * TY + ty) * SC, sm, tw, t);
    R vmax = 0;
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const R u = z[r].x, v = z[r].y;
        vmax = fmax(vmax, fabs(u) + fabs(v));
        z[r] = mk<R>(v * v - u * u, u * v);   // P + i Q
    }
    if (a.cfl_scale > 0) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        if ((threadIdx.x & 31) == 0 && static_cast<double>(vmax) * a.cfl_scale > 0.5)
            atomicOr(&a.ctl->status, STATUS_CFL);
    }
    fft_line<N, E, -1, R>(z, sm, tw, t);
#pragma unroll
    for (int r = 0; r < E; ++r)
        sm[pad<E>(t + r * T)] = z[r];
    __syncwarp();
    if (active) {
#pragma unroll
        for (int r = 0; r < E; ++r) {
            const int p = t + r * T;
            if (p <= K) {
                const cx<R> zk = z[r], zc = conj(sm[pad<E>((N - p) & (N - 1))]);
                const cx<R> sa = zk + zc, sb = zk - zc;
                nlt[p * (TY + 1) + ty] = mk<R>(sa.x / 2, sa.y / 2);                  // P^
                nlt[(C + p) * (TY + 1) + ty] = mk<R>(sb.y / 2, -sb.x / 2);           // Q^
            }
        }
    }
    __syncthreads();
    cx<R> *dst = a.nl + static_cast<size_t>(m) * 2 * C * N;
    for (int i = threadIdx.x; i < 2 * C * TY; i += blockDim.x) {
        const int t2 = i % TY, fk = i / TY;
        dst[static_cast<size_t>(fk) * N + y0 + t2] = nlt[fk * (TY + 1) + t2];
    }
}

template <typename R, int N> constexpr size_t column_smem() {
    using G = Cfg<R, N>;
    return sizeof(cx<R>) * (N + G::LPB * G::BUF);
}
template <typename R, int N> constexpr size_t row_smem() {
    using G = Cfg<R, N>;
    return sizeof(cx<R>) * (N + 2 * G::TY * G::SC + 2 * G::C * (G::TY + 1) + G::GROUPS * G::BUF);
}

} // namespace hzlb
