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
// One RK stage is two persistent kernels, each streaming its inputs into shared memory with
// bulk asynchronous copies (cp.async.bulk + mbarrier) one work item ahead of the compute:
//   column kernel  (work item = member x group of LPB kx columns): forward column FFTs of the
//                  two product spectra, the RK stage epilogue (dealias mask, viscosity and
//                  friction, forcing, accumulator, Euler-Maruyama noise on the last stage),
//                  then u^ = i ky psi^, v^ = -i kx psi^ of the next stage input and their
//                  inverse column FFTs, written out row-major through shared memory;
//   row kernel     (work item = member x tile of TY rows): inverse row FFT of u + i v, the
//                  products v^2 - u^2 and u v, the CFL check on stage 1, and the forward row
//                  FFT of (v^2 - u^2) + i (u v), keeping kx = 0..K of each.
// HBM layouts (complex R):
//   state / stage input / accumulator  [m][kx][j]          (K+1) x (2K+1) per member
//   velocity rows W                    [m][y][field][kx]   N x 2 x CW      (u^, v^ per row;
//                                                                           kx > K zero pad)
//   product columns NL                 [m][field][kx][y]   2 x (K+1) x N   (v^2-u^2, u v)
// so each row tile of W and each column group of NL is one contiguous bulk copy.
#pragma once
#include "async_copy.cuh"
#include "fft.cuh"

#include <cuda.h>
#include <type_traits>

namespace hzlb {

// Row stride of the velocity rows W in complex entries: C rounded up so that every row starts
// on a 32-byte sector boundary and each column group's run of LPB entries covers whole sectors
// (the last group also writes the zero pad entries).  No partially written sector of W then
// waits in L2 for the neighbouring group's stores, which at large ensembles were evicted first
// and cost a read of the sector from DRAM.
template <typename R> __host__ __device__ constexpr int velocity_row_stride(int n) {
    const int e = n < 16 ? n : 16, t = n / e, c = (n - 1) / 3 + 1;
    const int lpb = t >= 64 ? 1 : 64 / t;
    const int per32 = 32 / (2 * static_cast<int>(sizeof(R)));
    const int q = lpb > per32 ? lpb : per32;
    return (c + q - 1) / q * q;
}

// E (elements per thread) keeps a line inside one warp.  16 elements (two radix-16 passes at
// 256) beat 8 (three passes, twice the threads per line) in both precisions: measured at 256^2,
// FP32 0.63 against 1.00 ms per column launch, FP64 252k against 221k member-steps/s.
// RT: threads of a row-pass block (128 for every kernel but the standalone FP32 256^2 row
// kernel, row_kernel_threads below).
template <typename R, int N, int RT = 128> struct Cfg {
    static constexpr int E = N < 16 ? N : 16;
    static constexpr int T = N / E;
    static constexpr int K = (N - 1) / 3;
    static constexpr int C = K + 1;          // retained kx columns
    static constexpr int LD = 2 * K + 1;     // compact column length
    static constexpr int BUF = N + N / E;    // padded FFT line buffer
    // column kernel: LPB lines (columns) per block, 64 threads at least
    static constexpr int LPB = T >= 64 ? 1 : 64 / T;
    static constexpr int COL_THREADS = LPB * T;
    static constexpr int NCG = (C + LPB - 1) / LPB;   // column groups per member
    static constexpr int CW = velocity_row_stride<R>(N);   // row stride of W
    // state window per array: LPB columns plus one entry of 16-byte alignment slack, rounded
    // up to whole 16-byte chunks
    static constexpr int PER16 = 16 / (2 * static_cast<int>(sizeof(R)));
    static constexpr int ST_STRIDE = (LPB * LD + PER16 + PER16 - 1) / PER16 * PER16;
    // per-line stride of the product buffer and of the inverse-transform exchange area: a
    // padded FFT line buffer rounded up to whole 16-byte chunks
    static constexpr int LS = (BUF + PER16 - 1) / PER16 * PER16;
    static constexpr int ST_WORDS = 3 * ST_STRIDE > LPB * (LS + N) ? 3 * ST_STRIDE : LPB * (LS + N);
    // row kernel: TY rows per block, one row per group of T threads, RT threads at least
    static constexpr int TY_RAW = RT / T;
    static constexpr int TY = TY_RAW > N ? N : (TY_RAW < 2 ? 2 : TY_RAW);
    static constexpr int GROUPS = TY * T >= 32 ? TY : 32 / T;
    static constexpr int ROW_THREADS = GROUPS * T;
    static constexpr int TILE = TY * 2 * CW;          // row tile, complex entries
    // The row pass writes a tile's product spectra ([2C] columns x TY rows) with one tiled
    // tensor store when a staged column is one hardware swizzle span (32, 64 or 128 bytes) and
    // the 2C columns fit one box (N = 128, 256 in FP32; 256 in FP64); the staging area then
    // starts on a 1024-byte boundary inside the line buffers.
    static constexpr int ROW_SPAN = TY * static_cast<int>(2 * sizeof(R));
    static constexpr bool ROW_TMA = N >= 128 &&
                                    (ROW_SPAN == 32 || ROW_SPAN == 64 || ROW_SPAN == 128) &&
                                    2 * C <= 256 &&
                                    2 * C * ROW_SPAN + 1024 <= GROUPS * BUF * static_cast<int>(2 * sizeof(R));
    static constexpr int TWE = pass_twiddle_entries<N, E>() > 0 ? pass_twiddle_entries<N, E>() : 1;
};

// XOR swizzle of a [row][S] staging array (S a power of two): entry c of row y is stored at
// y*S + (c ^ swz(y)), which spreads 16 consecutive rows of one column over distinct 8-byte bank
// slots while keeping each row contiguous (a permutation within the row).
template <int S> __device__ __forceinline__ int swz(int y) {
    if constexpr (S <= 16)
        return ((y * S) >> 4) & (S - 1);
    else
        return y & 15;
}

struct StepControl {
    unsigned long long step;   // index of the step being taken (noise counter)
    unsigned int arrivals;     // column-kernel block arrivals on the final stage
    unsigned int status;       // STATUS_* bits
    unsigned int inject;       // test hook (hzlb_test_inject_wait_timeout): nonzero makes the
                               // next row pass leave block 0's first tile copy unissued
};

template <typename R> struct ColumnArgs {
    const cx<R> *nl;        // [M][2][C][N]: 2 P^, 2 Q^ (x-transformed products, doubled)
    cx<R> *w;               // [M][N][2][CW]
    cx<R> *omega;           // [M][C][LD]
    cx<R> *ystage;          // [M][C][LD]
    cx<R> *acc;             // [M][C][LD]
    const cx<R> *forcing;   // [.][fcols][LD]
    long long forcing_stride;  // elements between members (0: shared)
    int forcing_cols;       // forcing present for kx < forcing_cols
    const cx<R> *tw;        // N twiddles
    double nu, alpha, dt;
    int stage;              // 0 start, 1..3 intermediate, 4 final
    int emit;               // write W (velocity rows) for the next stage input
    double noise_scale;     // sigma sqrt(dt)/sqrt(2); 0 disables
    int noise_kmax2;
    unsigned long long seed;
    unsigned int member_base;
    StepControl *ctl;
    int members;
};

template <typename R> struct RowArgs {
    // tensor map of the product spectra as 4-byte words {N * sizeof(cx<R>) / 4, 2C, M}, box
    // {TY * sizeof(cx<R>) / 4, 2C, 1}, swizzle of the row span (filled by launch_row when the
    // resolution stores through it, Cfg::ROW_TMA)
    CUtensorMap nlmap;
    const cx<R> *w;       // [M][N][2][CW]
    cx<R> *nl;            // [M][2][C][N]
    const cx<R> *tw;
    double cfl_scale;     // dt * N / (2 pi); > 0 enables the stage-1 CFL check
    StepControl *ctl;
    int members;
};

// Band of FFT positions p = t + r T (t = 0..T-1) relative to the retained set |k| <= K:
// LOW all p <= K, HIGH all p >= N-K (negative wave numbers), ZERO none retained, else MIXED.
template <int N, int T, int r> struct Band {
    static constexpr int K = (N - 1) / 3, lo = r * T, hi = r * T + T - 1;
    static constexpr bool low = hi <= K;
    static constexpr bool high = lo >= N - K;
    static constexpr bool zero = lo > K && hi < N - K;
    static constexpr bool mixed = !(low || high || zero);
};
template <int I, int E, class F> __device__ __forceinline__ void static_for(F &&f) {
    if constexpr (I < E) {
        f(std::integral_constant<int, I>{});
        static_for<I + 1, E>(f);
    }
}
// Compact index j of FFT position p in a column (or -1 if p is outside the retained band).
template <int N> __device__ __forceinline__ int compact_j(int p) {
    constexpr int K = (N - 1) / 3, LD = 2 * K + 1;
    return p <= K ? p : (p >= N - K ? p - (N - LD) : -1);
}
template <int N, int T, int r> __device__ __forceinline__ int band_j(int p) {
    using B = Band<N, T, r>;
    constexpr int LD = 2 * B::K + 1;
    if constexpr (B::low)
        return p;
    else if constexpr (B::high)
        return p - (N - LD);
    else if constexpr (B::zero)
        return -1;
    else
        return compact_j<N>(p);
}

// Largest radius of the additive noise shell 1 <= |k| <= noise_kmax on grids of 48^2 and up (on
// smaller grids the shell is bounded by the retained band K <= 15 anyway).  With it, only the
// register positions whose ky can lie in |ky| <= 15 carry the noise draw, so the final stage's
// body holds 2 copies of it at 256^2 instead of 16.
constexpr int NOISE_KMAX_CAP = 15;
template <int N, int T, int r> struct NoiseBand {
    static constexpr int lo = r * T, hi = r * T + T - 1;
    static constexpr bool possible = lo <= NOISE_KMAX_CAP || hi >= N - NOISE_KMAX_CAP;
};

// Block-uniform bounded wait: thread 0 polls, the outcome is shared through `flag`, then
// every thread observes the completed phase.  Returns false on every thread on timeout.
__device__ __forceinline__ bool block_wait(uint64_t *bar, uint32_t parity, volatile int *flag) {
    if (threadIdx.x == 0)
        *flag = mbar_wait_bounded(bar, parity) ? 1 : 0;
    __syncthreads();
    const bool ok = *flag != 0;
    if (ok)
        mbar_wait_bounded(bar, parity);
    return ok;
}

// A line transform with the between-pass twiddles in registers (FP32) or read from the
// shared per-pass table (FP64, whose registers the data needs).
template <int N, int E, int SIGN, typename R>
__device__ __forceinline__ void transform_line(cx<R> (&x)[E], cx<R> *xsm, const cx<R> *tw,
                                               const cx<R> (&twr)[thread_twiddles<N, E>()], int t) {
    if constexpr (sizeof(R) == 4)
        fft_line_rt<N, E, SIGN, R>(x, xsm, twr, t);
    else
        fft_line<N, E, SIGN, R>(x, xsm, tw, t);
}

// S is the RK stage (0: velocity of the initial state only, 1..3 intermediate, 4 final), a
// compile-time constant so that each stage's epilogue is straight-line code.
// The column pass over work items first, first + stride, ... < items (member x group of LPB
// kx columns), with `smem_raw` as its dynamic shared memory; column_kernel runs one resolution,
// the mixed kernels run several one after another in one launch.  Every block of the grid
// calls it (also with no items), as the final stage's step counter counts one arrival a block.
template <typename R, int N, int S>
__device__ __forceinline__ void column_pass(const ColumnArgs<R> &a, int items, int first,
                                            int stride, unsigned char *smem_raw) {
    using G = Cfg<R, N>;
    constexpr int E = G::E, T = G::T, C = G::C, LD = G::LD, K = G::K, LPB = G::LPB;
    // product input [2][LPB][LS]: each line's two input columns, padded, double as the
    // exchange buffers of its forward transforms once read; state window [3][ST_STRIDE],
    // reused once the epilogue has consumed it as the exchange buffers [LPB][LS] of the
    // inverse transforms followed by the staging rows [N][LPB] of one output field
    cx<R> *nlbuf = reinterpret_cast<cx<R> *>(smem_raw);
    cx<R> *stbuf = nlbuf + 2 * LPB * G::LS;
    cx<R> *tw = stbuf + G::ST_WORDS;                               // [TWE] per-pass twiddles
    __shared__ __align__(8) uint64_t bars[3];                      // nl, (unused), state
    __shared__ int flags[2];
    __shared__ unsigned long long step_sh;

    constexpr bool forward = S > 0;
    constexpr int nst = S <= 1 ? 1 : 3;   // state arrays read: w_n (and stage input, acc)
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        mbar_init_fence();
        step_sh = a.ctl->step;
    }
    load_pass_twiddles<N, E, R>(tw, a.tw);
    __syncthreads();

    // one bulk copy per product column, issued by the lanes of warp 0 once lane 0 has armed
    // the barrier (every lane of warp 0 calls this)
    auto issue_nl = [&](int it) {
        const int m = it / G::NCG, kx0 = (it % G::NCG) * LPB;
        const int nl = min(LPB, C - kx0);
        constexpr uint32_t bytes = static_cast<uint32_t>(N * sizeof(cx<R>));
        const int lane = threadIdx.x & 31;
        if (lane == 0)
            mbar_arrive_expect(&bars[0], 2 * nl * bytes);
        __syncwarp();
        for (int c = lane; c < 2 * nl; c += 32) {
            const int f = c / nl, l = c % nl;
            bulk_copy_g2s(nlbuf + (f * LPB + l) * G::LS,
                          a.nl + ((static_cast<size_t>(m) * 2 + f) * C + kx0 + l) * N, bytes,
                          &bars[0]);
        }
    };
    // state window of a column group: starts `shift` entries early so that the copy is
    // 16-byte aligned, and covers whole 16-byte chunks
    auto window = [&](int it, int &shift, uint32_t &bytes) -> size_t {
        const int m = it / G::NCG, kx0 = (it % G::NCG) * LPB;
        const int nl = min(LPB, C - kx0);
        const size_t off = (static_cast<size_t>(m) * C + kx0) * LD;
        shift = static_cast<int>(off % G::PER16);
        const int count = (shift + nl * LD + G::PER16 - 1) / G::PER16 * G::PER16;
        bytes = static_cast<uint32_t>(count * sizeof(cx<R>));
        return off - shift;
    };
    auto issue_state = [&](int it) {
        int shift;
        uint32_t bytes;
        const size_t base = window(it, shift, bytes);
        mbar_arrive_expect(&bars[2], nst * bytes);
        bulk_copy_g2s(stbuf, a.omega + base, bytes, &bars[2]);
        if constexpr (nst == 3) {
            bulk_copy_g2s(stbuf + G::ST_STRIDE, a.ystage + base, bytes, &bars[2]);
            bulk_copy_g2s(stbuf + 2 * G::ST_STRIDE, a.acc + base, bytes, &bars[2]);
        }
    };
    // writes the item's columns of one state array from its window region (updated in place)
    // back to HBM: the whole 16-byte chunks as one bulk copy, the at most PER16 - 1 entries
    // before the first and after the last chunk boundary by plain stores (thread 0 alone)
    auto store_window = [&](cx<R> *dst, int region, int it) {
        const int m = it / G::NCG, kx0 = (it % G::NCG) * LPB;
        const int nl = min(LPB, C - kx0);
        const size_t off = (static_cast<size_t>(m) * C + kx0) * LD;
        const size_t end = off + static_cast<size_t>(nl) * LD;
        const cx<R> *src = stbuf + region * G::ST_STRIDE + static_cast<int>(off % G::PER16);
        const size_t a0 = min(end, (off + G::PER16 - 1) / G::PER16 * G::PER16);
        const size_t a1 = max(a0, end / G::PER16 * G::PER16);
        for (size_t e = off; e < a0; ++e)
            dst[e] = src[e - off];
        if (a1 > a0)
            bulk_copy_s2g(dst + a0, src + (a0 - off), static_cast<uint32_t>((a1 - a0) * sizeof(cx<R>)));
        for (size_t e = a1; e < end; ++e)
            dst[e] = src[e - off];
    };

    const int line = threadIdx.x / T, t = threadIdx.x % T;
    // FP32: this thread's between-pass twiddles in registers for every transform it does
    // (FP64 keeps reading the shared table: its registers are spent on the data)
    constexpr bool reg_tw = sizeof(R) == 4;
    cx<R> twr[thread_twiddles<N, E>()];
    if constexpr (reg_tw)
        load_thread_twiddles<N, E, R>(twr, tw, t);
    if (threadIdx.x < 32 && forward && first < items)
        issue_nl(first);
    bool timed_out = false;
    int k = 0;
    for (int it = first; it < items; it += stride, ++k) {
        const int m = it / G::NCG, kx0 = (it % G::NCG) * LPB;
        const int kx = kx0 + line;
        const bool valid = kx < C;
        const int kxc = valid ? kx : 0;
        if (threadIdx.x == 0) {
            fence_proxy_async_shared();
            issue_state(it);
        }
        int shift;
        uint32_t sbytes;
        window(it, shift, sbytes);
        // this line's columns in the window regions, updated in place by the epilogue
        cx<R> *s_w = stbuf + shift + line * LD, *s_y = s_w + G::ST_STRIDE,
              *s_a = s_w + 2 * G::ST_STRIDE;
        const R kxr = static_cast<R>(kxc);

        cx<R> y[E];   // next stage input at this thread's positions (zero outside the band)
        cx<R> v[E];
        if constexpr (!forward) {
            if (!block_wait(&bars[2], k & 1, &flags[1])) {
                timed_out = true;
                break;
            }
            static_for<0, E>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                const int j = band_j<N, T, r>(t + r * T);
                y[r] = (valid && j >= 0) ? s_w[j] : mk<R>(0, 0);
            });
        } else {
            if (!block_wait(&bars[0], k & 1, &flags[0])) {
                timed_out = true;
                break;
            }
            // forward column FFTs of the product spectra (unnormalised; 1/N^2 below):
            // A^ = -kx ky P^ - (kx^2 - ky^2) Q^ with P = v^2 - u^2, Q = u v.  One loop body for
            // both fields keeps a single copy of the transform in the kernel.
            cx<R> adv[E];
#pragma unroll 1
            for (int f = 0; f < 2; ++f) {
                cx<R> *src = nlbuf + (f * LPB + line) * G::LS;
#pragma unroll
                for (int r = 0; r < E; ++r)
                    v[r] = src[t + r * T];
                __syncwarp();   // the line's lanes have read the column it exchanges in
                transform_line<N, E, -1, R>(v, src, tw, twr, t);
                if (f == 0) {
                    static_for<0, E>([&](auto rc) {
                        constexpr int r = decltype(rc)::value;
                        const int p = t + r * T;
                        const int ky = Band<N, T, r>::low ? p : (Band<N, T, r>::high ? p - N : (p <= K ? p : p - N));
                        adv[r] = scale(static_cast<R>(-kxc * ky), v[r]);
                    });
                }
            }
            // every line is done with the product buffer: stream the next item's in
            fence_proxy_async_shared();
            __syncthreads();
            if (threadIdx.x < 32 && it + stride < items)
                issue_nl(it + stride);
            if (!block_wait(&bars[2], k & 1, &flags[1])) {
                timed_out = true;
                break;
            }
            // 1/N^2 of the unnormalised transforms, halved: the row pass stores 2 P^ and 2 Q^
            const R inv_n2 = static_cast<R>(0.5 / (static_cast<double>(N) * N));
            const R nu = static_cast<R>(a.nu), alpha = static_cast<R>(a.alpha),
                    dt = static_cast<R>(a.dt);
            bool bad = false;
            static_for<0, E>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                y[r] = mk<R>(0, 0);
                const int j = band_j<N, T, r>(t + r * T);
                if (valid && j >= 0) {
                    const int ky = j <= K ? j : j - LD;
                    const R k2 = static_cast<R>(kxc * kxc + ky * ky);
                    const cx<R> wn = s_w[j];
                    const cx<R> ys = S == 1 ? wn : s_y[j];
                    // rhs: active ? -A^ - (nu k^2 + alpha) w + f : 0   (solver.cpp:197-202)
                    cx<R> kk = mk<R>(0, 0);
                    if (!(kxc == 0 && j == 0)) {
                        const cx<R> nl =
                            scale(inv_n2, adv[r] - scale(static_cast<R>(kxc * kxc - ky * ky), v[r]));
                        const R rate = nu * k2 + alpha;
                        kk = mk<R>(-nl.x, -nl.y) - scale(rate, ys);
                        if (kxc < a.forcing_cols)
                            kk = kk + a.forcing[static_cast<size_t>(m) * a.forcing_stride +
                                                static_cast<size_t>(kxc) * LD + j];
                    }
                    if constexpr (S == 1) {
                        s_a[j] = kk;
                        y[r] = wn + scale(dt / 2, kk);
                        s_y[j] = y[r];
                    } else if constexpr (S == 2) {
                        s_a[j] = s_a[j] + scale(static_cast<R>(2.0), kk);
                        y[r] = wn + scale(dt / 2, kk);
                        s_y[j] = y[r];
                    } else if constexpr (S == 3) {
                        s_a[j] = s_a[j] + scale(static_cast<R>(2.0), kk);
                        y[r] = wn + scale(dt, kk);
                        s_y[j] = y[r];
                    } else {
                        // w += dt/6 (k1 + 2 k2 + 2 k3 + k4)   (solver.cpp:233-234)
                        cx<R> w1 = wn + scale(dt / 6, s_a[j] + kk);
                        const int kk2 = kxc * kxc + ky * ky;
                        if (NoiseBand<N, T, r>::possible && a.noise_scale > 0 && kk2 >= 1 &&
                            kk2 <= a.noise_kmax2) {
                            double xi1, xi2;
                            const bool rep = kxc > 0 || ky > 0;
                            philox_normal_pair(a.seed, a.member_base + m, step_sh,
                                               mode_code(kxc, rep ? ky : -ky), xi1, xi2);
                            const double s = a.noise_scale;
                            w1 = w1 + mk<R>(static_cast<R>(s * xi1),
                                            static_cast<R>(rep ? s * xi2 : -(s * xi2)));
                        }
                        bad |= !(isfinite(w1.x) && isfinite(w1.y));
                        s_w[j] = w1;
                        y[r] = w1;
                    }
                }
            });
            if (bad)
                atomicOr(&a.ctl->status, STATUS_NONFINITE);
            // the item's new state leaves from the window in bulk; the window is reused below
            // and by the next item's copies once the engine has read it
            fence_proxy_async_shared();
            __syncthreads();
            if (threadIdx.x == 0) {
                if constexpr (S == 4) {
                    store_window(a.omega, 0, it);
                } else {
                    store_window(a.ystage, 1, it);
                    store_window(a.acc, 2, it);
                }
                bulk_commit();
                bulk_wait_read_all();
            }
        }

        if (a.emit) {
            // velocity of the next stage input (solver.cpp:177-185): u^ = i ky psi^,
            // v^ = -i kx psi^ with psi^ = w^/k^2; inverse column FFTs exchanging in the state
            // window, each field staged there as rows [y][line] (swizzled) and written to the
            // rows [y][field][kx] of W in 32-byte runs
            fence_proxy_async_shared();
            __syncthreads();   // every line is done with the state window
            cx<R> *xb = stbuf + line * G::LS;
            // psi^ = w^ / k^2 once per mode (k = 0 gives 0), then u^ and v^ from it
            static_for<0, E>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                const int j = band_j<N, T, r>(t + r * T);
                cx<R> psi = mk<R>(0, 0);
                if (j >= 0) {
                    const int ky = j <= K ? j : j - LD;
                    const int k2 = kxc * kxc + ky * ky;
                    if (k2 > 0) {
                        const R inv = static_cast<R>(1) / static_cast<R>(k2);
                        psi = mk<R>(y[r].x * inv, y[r].y * inv);
                    }
                }
                y[r] = psi;
            });
            cx<R> *wst = stbuf + LPB * G::LS;   // one field's rows [N][LPB]
            const int nl = min(LPB, C - kx0);
            // runs of the group's columns and, in the last group, of the zero pad up to CW
            const int nw = min(LPB, G::CW - kx0);
            cx<R> *dst = a.w + static_cast<size_t>(m) * N * 2 * G::CW + kx0;
#pragma unroll 1
            for (int f = 0; f < 2; ++f) {
                static_for<0, E>([&](auto rc) {
                    constexpr int r = decltype(rc)::value;
                    const int p = t + r * T;
                    const int ky = Band<N, T, r>::low ? p : (Band<N, T, r>::high ? p - N : (p <= K ? p : p - N));
                    const R kyr = static_cast<R>(ky);
                    const cx<R> psi = y[r];
                    v[r] = f == 0 ? mk<R>(-kyr * psi.y, kyr * psi.x) : mk<R>(kxr * psi.y, -kxr * psi.x);
                });
                transform_line<N, E, +1, R>(v, xb, tw, twr, t);
                if (f == 1)
                    __syncthreads();   // field 0 is out of the staging rows
#pragma unroll
                for (int r = 0; r < E; ++r) {
                    const int yy = t + r * T;
                    wst[yy * LPB + (line ^ swz<LPB>(yy))] = v[r];
                }
                __syncthreads();
                for (int i = threadIdx.x; i < N * LPB; i += blockDim.x) {
                    const int l = i % LPB, yy = i / LPB;
                    if (l < nw)
                        dst[(static_cast<size_t>(yy) * 2 + f) * G::CW + l] = wst[yy * LPB + (l ^ swz<LPB>(yy))];
                }
            }
        }
        fence_proxy_async_shared();   // this thread's shared-memory accesses precede the next bulk copies
        __syncthreads();              // buffers of this item are free for the next copies
    }
    if (threadIdx.x == 0)
        bulk_wait_all();   // this block's state stores are complete before it leaves
    if (timed_out) {
        if (threadIdx.x == 0)
            atomicOr(&a.ctl->status, STATUS_TIMEOUT);
        return;   // uniform across the block
    }

    if constexpr (S == 4) {
        // the last block to finish advances the device step counter (every block read it
        // before arriving, so no block sees the new value)
        if (threadIdx.x == 0) {
            __threadfence();
            const unsigned total = gridDim.x;
            const unsigned prev = atomicAdd(&a.ctl->arrivals, 1u);
            if (prev == total - 1) {
                a.ctl->arrivals = 0;
                a.ctl->step = step_sh + 1;
                __threadfence();
            }
        }
    }
}

template <typename R, int N, int S>
__global__ void __launch_bounds__(Cfg<R, N>::COL_THREADS)
    column_kernel(const ColumnArgs<R> a, int items) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    column_pass<R, N, S>(a, items, static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x),
                         smem_raw);
}

// Packs the x-spectra of two real fields as a + i b for the inverse row transform.  A and B
// hold kx = 0..K of the row (column-pass output); negative kx follow from the fields being
// real (A(-kx) = conj A(kx)), and the kx = 0 entries are real (imaginary roundoff dropped, as
// the reference keeps only the real part of its inverse transforms).
template <int N, int E, typename R>
__device__ __forceinline__ void pack_row(cx<R> (&z)[E], const cx<R> *A, const cx<R> *B, int t) {
    constexpr int T = N / E, K = (N - 1) / 3;
    static_for<0, E>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        using Bd = Band<N, T, r>;
        const int p = t + r * T;
        cx<R> za = mk<R>(0, 0), zb = mk<R>(0, 0);
        if constexpr (Bd::low) {
            za = A[p];
            zb = B[p];
            if (r == 0 && p == 0) {
                za.y = 0;
                zb.y = 0;
            }
        } else if constexpr (Bd::high) {
            za = conj(A[N - p]);
            zb = conj(B[N - p]);
        } else if constexpr (Bd::mixed) {
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
        }
        z[r] = mk<R>(za.x - zb.y, za.y + zb.x);
    });
}

// Number of a thread's positions p = t + r T that can hold a retained kx (0 <= p <= K).
template <int N, int E> struct LowSlots {
    static constexpr int T = N / E, K = (N - 1) / 3;
    static constexpr int value = K / T + 1 < E ? K / T + 1 : E;
};

// One row's work between its inputs and its product spectra, by the T lanes that hold the
// row: inverse transform of u + i v, products P = v^2 - u^2, Q = u v (and, with a.cfl_scale > 0,
// the CFL check on |u| + |v|), forward transform of P + i Q, then separation of P^ and Q^ at
// kx = p = t + r T (r < RL) from z(p) and conj z(N - p), both stored doubled (the column pass
// folds the halving into its 1/N^2: power-of-two scalings commute with rounding, so the
// results are those of halving here).  Position N - p of this row is held by
// lane T - t at register E - 1 - r (t > 0), or by this lane at register (E - r) mod E (t = 0):
// two shuffles per value, no trip through shared memory.  Every lane of the warp calls it.
template <typename R, int N>
__device__ __forceinline__ void row_line(cx<R> (&z)[Cfg<R, N>::E], cx<R> *sm, const cx<R> *tw,
                                         const cx<R> (&twr)[thread_twiddles<N, Cfg<R, N>::E>()],
                                         int t, const RowArgs<R> &a,
                                         cx<R> (&ph)[LowSlots<N, Cfg<R, N>::E>::value],
                                         cx<R> (&qh)[LowSlots<N, Cfg<R, N>::E>::value]) {
    using G = Cfg<R, N>;
    constexpr int E = G::E, T = G::T, RL = LowSlots<N, E>::value;
    transform_line<N, E, +1, R>(z, sm, tw, twr, t);
    if (a.cfl_scale > 0) {   // uniform: the stage-1 launch checks the velocities
        R vmax = 0;
#pragma unroll
        for (int r = 0; r < E; ++r)
            vmax = fmax(vmax, fabs(z[r].x) + fabs(z[r].y));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
            vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        if ((threadIdx.x & 31) == 0 && static_cast<double>(vmax) * a.cfl_scale > 0.5)
            atomicOr(&a.ctl->status, STATUS_CFL);
    }
#pragma unroll
    for (int r = 0; r < E; ++r) {
        const R u = z[r].x, v = z[r].y;
        z[r] = mk<R>(v * v - u * u, u * v);   // P + i Q
    }
    transform_line<N, E, -1, R>(z, sm, tw, twr, t);
    const int lane = threadIdx.x & 31;
    const int src = (lane & ~(T - 1)) + ((T - t) & (T - 1));
    static_for<0, RL>([&](auto rc) {
        constexpr int r = decltype(rc)::value;
        constexpr int rs = E - 1 - r, r0 = (E - r) & (E - 1);
        cx<R> zp;
        zp.x = __shfl_sync(0xffffffffu, z[rs].x, src);
        zp.y = __shfl_sync(0xffffffffu, z[rs].y, src);
        if (t == 0)
            zp = z[r0];
        const cx<R> zk = z[r], zc = conj(zp);
        const cx<R> sa = zk + zc, sb = zk - zc;
        ph[r] = sa;                   // 2 P^
        qh[r] = mk<R>(sb.y, -sb.x);   // 2 Q^
    });
}

// The row pass over work items first, first + stride, ... < items (member x tile of TY rows),
// with `smem_raw` as its dynamic shared memory; row_kernel runs one resolution, the mixed
// kernels run several one after another in one launch.
template <typename R, int N, int RT = 128>
__device__ __forceinline__ void row_pass(const RowArgs<R> &a, int items, int first, int stride,
                                         unsigned char *smem_raw) {
    using G = Cfg<R, N, RT>;
    constexpr int E = G::E, T = G::T, C = G::C, K = G::K, TY = G::TY;
    // input tile [TY][2][CW], refilled with the next item's tile as soon as every row has read
    // its entries; FFT line buffers [GROUPS][BUF], reused once every row has finished its
    // transforms as the staging of the product spectra [2C][TY] (swizzled rows)
    cx<R> *tile = reinterpret_cast<cx<R> *>(smem_raw);
    cx<R> *lines = tile + G::TILE;
    cx<R> *tw = lines + G::GROUPS * G::BUF;
    static_assert(2 * C * TY <= G::GROUPS * G::BUF, "product staging fits in the line buffers");
    __shared__ __align__(8) uint64_t bar;
    __shared__ int flag;
    constexpr int tiles_per_member = N / TY;
    constexpr uint32_t tile_bytes = G::TILE * sizeof(cx<R>);
    static_assert(tile_bytes % 16 == 0, "bulk copies move 16-byte multiples");
    constexpr int RL = LowSlots<N, E>::value;

    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    load_pass_twiddles<N, E, R>(tw, a.tw);
    __syncthreads();
    auto issue = [&](int it) {
        const int m = it / tiles_per_member, y0 = (it % tiles_per_member) * TY;
        mbar_arrive_expect(&bar, tile_bytes);
        bulk_copy_g2s(tile, a.w + (static_cast<size_t>(m) * N + y0) * 2 * G::CW, tile_bytes, &bar);
    };
    if (threadIdx.x == 0 && first < items) {
        // test hook: a pending injection (consumed here) leaves this block's first copy
        // unissued, so its bounded wait below runs out with no copy in flight
        const bool skip = blockIdx.x == 0 && *static_cast<volatile unsigned *>(&a.ctl->inject) != 0 &&
                          atomicExch(&a.ctl->inject, 0u) != 0;
        if (!skip)
            issue(first);
    }

    const int g = threadIdx.x / T, t = threadIdx.x % T;
    // FP32: this thread's between-pass twiddles in registers (see column_kernel)
    constexpr bool reg_tw = sizeof(R) == 4;
    cx<R> twr[thread_twiddles<N, E>()];
    if constexpr (reg_tw)
        load_thread_twiddles<N, E, R>(twr, tw, t);
    const bool active = g < TY;
    const int ty = active ? g : 0;
    cx<R> *sm = lines + g * G::BUF;
    int k = 0;
    for (int it = first; it < items; it += stride, ++k) {
        const int m = it / tiles_per_member, y0 = (it % tiles_per_member) * TY;
        if (!block_wait(&bar, k & 1, &flag)) {
            if (threadIdx.x == 0) {
                atomicOr(&a.ctl->status, STATUS_TIMEOUT);
                bulk_wait_all();   // the product stores in flight complete before the block leaves
            }
            return;   // uniform across the block
        }
        const cx<R> *row = tile + ty * 2 * G::CW;
        cx<R> z[E];
        pack_row<N, E, R>(z, row, row + G::CW, t);
        // every row holds its inputs in registers: stream the next item's tile in; the previous
        // item's product store has read the staging area before the transforms write it
        fence_proxy_async_shared();
        if constexpr (G::ROW_TMA)
            if (threadIdx.x == 0)
                bulk_wait_read_all();
        __syncthreads();
        if (threadIdx.x == 0 && it + stride < items)
            issue(it + stride);
        cx<R> ph[RL], qh[RL];
        row_line<R, N>(z, sm, tw, twr, t, a, ph, qh);
        __syncthreads();   // every row is done with its line buffer: stage the products there
        if constexpr (G::ROW_TMA) {
            // staged [2C][TY] in the layout of the tensor map's swizzle (16-byte chunk bits
            // 4.. of an offset XORed with its bits 7..); one tiled store writes the tile's 2C
            // column segments.  The swizzle spreads a row's 16-byte entries (FP64) over every
            // bank; 8-byte entries (FP32) share address bit 3 within a row and reach half the
            // banks per half warp (pairing rows by shuffles into 16-byte chunks removed those
            // conflicts but cost as many instructions as it saved wavefronts: measured equal)
            constexpr unsigned SZ = sizeof(cx<R>), RB = G::ROW_SPAN;
            constexpr unsigned SWM = (RB / 16 - 1) << 4;
            unsigned char *stage = reinterpret_cast<unsigned char *>(lines) +
                                   ((1024u - (smem_u32(lines) & 1023u)) & 1023u);
            if (active) {
                static_for<0, RL>([&](auto rc) {
                    constexpr int r = decltype(rc)::value;
                    const int p = t + r * T;
                    if (Band<N, T, r>::low || p <= K) {
                        unsigned o = static_cast<unsigned>(p) * RB + ty * SZ;
                        *reinterpret_cast<cx<R> *>(stage + (o ^ ((o >> 3) & SWM))) = ph[r];   // P^
                        o = static_cast<unsigned>(C + p) * RB + ty * SZ;
                        *reinterpret_cast<cx<R> *>(stage + (o ^ ((o >> 3) & SWM))) = qh[r];   // Q^
                    }
                });
            }
            fence_proxy_async_shared();
            __syncthreads();
            if (threadIdx.x == 0) {
                tensor_store_3d(&a.nlmap, stage, y0 * static_cast<int>(SZ / 4), 0, m);
                bulk_commit();
            }
            continue;
        }
        cx<R> *nlt = lines;
        if (active) {
            static_for<0, RL>([&](auto rc) {
                constexpr int r = decltype(rc)::value;
                const int p = t + r * T;
                if (Band<N, T, r>::low || p <= K) {
                    nlt[p * TY + (ty ^ swz<TY>(p))] = ph[r];                 // P^
                    nlt[(C + p) * TY + (ty ^ swz<TY>(C + p))] = qh[r];       // Q^
                }
            });
        }
        __syncthreads();
        cx<R> *dst = a.nl + static_cast<size_t>(m) * 2 * C * N;
        // entry (fk, t2) of the staged products goes to column fk, row y0 + t2; the threads
        // cover fk * TY + t2 in order, so each keeps one t2 and steps fk
        static_assert(G::ROW_THREADS % TY == 0, "whole staged columns per pass");
        constexpr int FSTEP = G::ROW_THREADS / TY;
        {
            const int t2 = threadIdx.x % TY;
            cx<R> *row = dst + y0 + t2;
#pragma unroll 4
            for (int fk = threadIdx.x / TY; fk < 2 * C; fk += FSTEP)
                row[static_cast<size_t>(fk) * N] = nlt[fk * TY + (t2 ^ swz<TY>(fk))];
        }
        // the next item's transforms write the line buffers only after its tile barrier and
        // the block barrier that follows it
    }
    if constexpr (G::ROW_TMA)
        if (threadIdx.x == 0)
            bulk_wait_all();   // this block's product stores are complete before it leaves
}

// Threads of a standalone row-kernel block: 64 at 128^2 and 256^2 (FP32 256^2: 4-row tiles,
// 12 blocks per SM; FP64 256^2: 6 blocks), else 128 (the shape the mixed kernels share).
template <typename R, int N> __host__ __device__ constexpr int row_kernel_threads() {
    return N == 256 || (sizeof(R) == 4 && N == 128) ? 64 : 128;
}
// FP32: at most 80 registers, so that 6 blocks of 128 (12 of 64) threads fit an SM (95
// unconstrained: 5 blocks; measured 0.368 against 0.383 ms per launch at 2048 members, 256^2).
// RT: the block shape (64 or 128 threads); both are compiled for every resolution, the
// default is row_kernel_threads and a mixed batch's tuner may choose the other.
template <typename R, int N, int RT>
__global__ void __launch_bounds__(Cfg<R, N, RT>::ROW_THREADS, sizeof(R) == 4 ? (RT == 64 ? 12 : 6) : 1)
    row_kernel(const __grid_constant__ RowArgs<R> a, int items) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    row_pass<R, N, RT>(a, items, static_cast<int>(blockIdx.x), static_cast<int>(gridDim.x), smem_raw);
}

template <typename R, int N> constexpr size_t column_smem() {
    using G = Cfg<R, N>;
    return sizeof(cx<R>) * (2 * G::LPB * G::LS + G::ST_WORDS + G::TWE);
}
template <typename R, int N, int RT = 128> constexpr size_t row_smem() {
    using G = Cfg<R, N, RT>;
    return sizeof(cx<R>) * (G::TILE + G::GROUPS * G::BUF + G::TWE);
}
} // namespace hzlb

namespace hzlb {

// ---- one persistent kernel per RK stage over several resolutions ----------------------
// The work list of a mixed-resolution batch: class c (resolution 64 << c) holds items[c] work
// items of its pass, the global indices [offset[c], offset[c] + items[c]) of one list the
// persistent grid strides over, block b taking the indices congruent to b modulo the grid.
// Each block runs the classes' passes one after another, so the grid stays busy across the
// resolution boundaries instead of draining one resolution's launch before the next begins.
constexpr int MIXED_CLASSES = 4;
template <typename R> struct MixedRowArgs {
    RowArgs<R> cls[MIXED_CLASSES];
    int items[MIXED_CLASSES], offset[MIXED_CLASSES];
};
template <typename R> struct MixedColumnArgs {
    ColumnArgs<R> cls[MIXED_CLASSES];
    int items[MIXED_CLASSES], offset[MIXED_CLASSES];
};
// first local item of this block in a class whose items start at global index `offset`
__device__ __forceinline__ int mixed_first(int offset) {
    const int g = static_cast<int>(gridDim.x);
    const int r = (static_cast<int>(blockIdx.x) - offset) % g;
    return r < 0 ? r + g : r;
}
// between two classes' passes: every thread is done with the shared memory, through both the
// generic and the bulk-copy proxy, before the next pass writes it
__device__ __forceinline__ void mixed_boundary() {
    fence_proxy_async_shared();
    __syncthreads();
}
template <typename R, int... Ns> __host__ __device__ constexpr bool mixed_shapes_agree() {
    return ((Cfg<R, Ns>::ROW_THREADS == 128 && Cfg<R, Ns>::COL_THREADS == 64) && ...);
}
// one class's pass in a mixed kernel; a class without items (a resolution the batch does not
// hold: its arguments are empty) is skipped by every block alike
template <typename R, int N>
__device__ __forceinline__ void mixed_row_class(const MixedRowArgs<R> &a, int c, unsigned char *smem) {
    if (a.items[c] > 0) {
        row_pass<R, N>(a.cls[c], a.items[c], mixed_first(a.offset[c]), static_cast<int>(gridDim.x),
                       smem);
        mixed_boundary();
    }
}
template <typename R, int N, int S>
__device__ __forceinline__ void mixed_column_class(const MixedColumnArgs<R> &a, int c,
                                                   unsigned char *smem) {
    if (a.items[c] > 0) {
        column_pass<R, N, S>(a.cls[c], a.items[c], mixed_first(a.offset[c]),
                             static_cast<int>(gridDim.x), smem);
        mixed_boundary();
    }
}
// class (argument slot) of resolution n
__host__ __device__ constexpr int mixed_class(int n) {
    return n == 64 ? 0 : n == 128 ? 1 : n == 256 ? 2 : 3;
}
// The passes run in the order of the pack, heaviest items first (512^2 .. 64^2), so a block's
// last items are the lightest and the launch ends without a tail of one large item; the host
// numbers the work list in the same order.
template <typename R, int MINB, int... Ns>
__global__ void __launch_bounds__(128, MINB) mixed_row_kernel(const __grid_constant__ MixedRowArgs<R> a) {
    static_assert(mixed_shapes_agree<R, Ns...>(), "one block shape for every resolution");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    (mixed_row_class<R, Ns>(a, mixed_class(Ns), smem_raw), ...);
}
template <typename R, int S, int MINB, int... Ns>
__global__ void __launch_bounds__(64, MINB) mixed_column_kernel(const MixedColumnArgs<R> a) {
    static_assert(mixed_shapes_agree<R, Ns...>(), "one block shape for every resolution");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    (mixed_column_class<R, Ns, S>(a, mixed_class(Ns), smem_raw), ...);
}

} // namespace hzlb
