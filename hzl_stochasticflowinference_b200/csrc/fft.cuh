// Register-resident Stockham FFT for one line of length N, held by T = N/E threads of one
// warp (E elements per thread).  Radix-E passes exchange through a padded shared-memory line
// buffer (warp-synchronous; no block barrier); the last pass may use a smaller radix and
// needs no exchange.  Butterflies are radix-2/4/8/16 DFTs in registers with exact special
// cases for the trivial and sqrt(1/2) twiddles.  Twiddles between passes come from a table
// W_N^k = exp(-2 pi i k / N) built on the host in double precision (the same construction as
// the reference's std::polar roots, src/fft.cpp:25-27), so the FP64 path keeps the
// reference's twiddle accuracy.
#pragma once
#include "common.cuh"

namespace hzlb {

// cos(2 pi k/16) for 0 <= k <= 8, to double precision (sin(2 pi k/16) = cos16(|4 - k|)).
__device__ __forceinline__ double cos16(int k) {
    switch (k) {
    case 0: return 1.0;
    case 1: return 0.92387953251128675613;
    case 2: return 0.70710678118654752440;
    case 3: return 0.38268343236508977173;
    case 4: return 0.0;
    case 5: return -0.38268343236508977173;
    case 6: return -0.70710678118654752440;
    case 7: return -0.92387953251128675613;
    default: return -1.0;
    }
}

// z * exp(SIGN * 2 pi i k / RAD) for 0 <= k < RAD/2 (k is a compile-time constant after
// unrolling, so the branches fold).
template <int RAD, int SIGN, typename R>
__device__ __forceinline__ cx<R> twiddle_const(int k, cx<R> z) {
    if (k == 0)
        return z;
    if (4 * k == RAD)
        return mk<R>(-SIGN * z.y, SIGN * z.x);
    const R h = static_cast<R>(0.70710678118654752440);
    if (8 * k == RAD)
        return mk<R>(h * (z.x - SIGN * z.y), h * (SIGN * z.x + z.y));
    if (8 * k == 3 * RAD)
        return mk<R>(h * (-z.x - SIGN * z.y), h * (SIGN * z.x - z.y));
    const int i = k * (16 / RAD);
    const R c = static_cast<R>(cos16(i)), s = static_cast<R>(SIGN * cos16(i < 4 ? 4 - i : i - 4));
    return mk<R>(z.x * c - z.y * s, z.x * s + z.y * c);
}

// In-place DFT of RAD points in registers, natural-order output.
template <int RAD, int SIGN, typename R> struct Dft {
    static __device__ __forceinline__ void run(cx<R> *a) {
        constexpr int H = RAD / 2;
        cx<R> e[H], o[H];
#pragma unroll
        for (int i = 0; i < H; ++i) {
            e[i] = a[2 * i];
            o[i] = a[2 * i + 1];
        }
        Dft<H, SIGN, R>::run(e);
        Dft<H, SIGN, R>::run(o);
#pragma unroll
        for (int k = 0; k < H; ++k) {
            const cx<R> t = twiddle_const<RAD, SIGN, R>(k, o[k]);
            a[k] = e[k] + t;
            a[k + H] = e[k] - t;
        }
    }
};
template <int SIGN, typename R> struct Dft<1, SIGN, R> {
    static __device__ __forceinline__ void run(cx<R> *) {}
};

template <int E> __device__ __forceinline__ int pad(int i) { return i + i / E; }
template <int N, int E> struct FftShape {
    static constexpr int T = N / E;                // threads per line
    static constexpr int BUF = N + N / E;          // padded line buffer, elements
    static_assert(T >= 1 && T <= 32, "a line must fit in one warp");
};

// One Stockham pass with stride NS; recursion over the remaining passes.
template <int N, int E, int SIGN, typename R, int NS>
__device__ __forceinline__ void fft_pass(cx<R> (&v)[E], cx<R> *sm, const cx<R> *tw, int t) {
    constexpr int T = N / E;
    constexpr int RAD = (E < N / NS) ? E : N / NS;
    constexpr int NB = E / RAD;
    constexpr bool LAST = NS * RAD == N;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int j = t + q * T;
        const int k = j & (NS - 1);
        cx<R> u[RAD];
#pragma unroll
        for (int r = 0; r < RAD; ++r)
            u[r] = v[q + r * NB];
        if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < RAD; ++r) {
                cx<R> w = tw[(k * r) * (N / (NS * RAD))];
                if constexpr (SIGN > 0)
                    w.y = -w.y;
                u[r] = cmul(u[r], w);
            }
        }
        Dft<RAD, SIGN, R>::run(u);
        if constexpr (LAST) {
#pragma unroll
            for (int r = 0; r < RAD; ++r)
                v[q + r * NB] = u[r];
        } else {
            const int base = (j - k) * RAD + k;
#pragma unroll
            for (int r = 0; r < RAD; ++r)
                sm[pad<E>(base + r * NS)] = u[r];
        }
    }
    if constexpr (!LAST) {
        __syncwarp();
#pragma unroll
        for (int r = 0; r < E; ++r)
            v[r] = sm[pad<E>(t + r * T)];
        __syncwarp();
        fft_pass<N, E, SIGN, R, NS * RAD>(v, sm, tw, t);
    }
}

// Unnormalised DFT of one line: X[k] = sum_n x[n] exp(SIGN 2 pi i n k / N).
// Thread t (0 <= t < N/E) holds x[t + r*(N/E)] in v[r] on entry and X[t + r*(N/E)] on exit.
// Every lane of the warp must call this together (warp-synchronous exchanges).
template <int N, int E, int SIGN, typename R>
__device__ __forceinline__ void fft_line(cx<R> (&v)[E], cx<R> *sm, const cx<R> *tw, int t) {
    (void)FftShape<N, E>::T;
    fft_pass<N, E, SIGN, R, 1>(v, sm, tw, t);
}

} // namespace hzlb
