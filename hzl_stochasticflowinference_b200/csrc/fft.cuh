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

// Between-pass twiddles laid out per pass as [q][r-1][t] (t fastest), so the T threads of a
// line read consecutive entries (no bank conflicts, unlike reading W_N^(k r) with stride r).
template <int N, int E, int NS> struct PassTw {
    static constexpr int T = N / E;
    static constexpr int RAD = (E < N / NS) ? E : N / NS;
    static constexpr int NB = E / RAD;
    static constexpr bool LAST = NS * RAD == N;
    static constexpr int own = NS > 1 ? NB * (RAD - 1) * T : 0;   // entries of this pass
    static constexpr int rest() {
        if constexpr (LAST)
            return 0;
        else
            return PassTw<N, E, NS * RAD>::own + PassTw<N, E, NS * RAD>::rest();
    }
    static constexpr int total = own + rest();                     // this and later passes
};
template <int N, int E> __host__ __device__ constexpr int pass_twiddle_entries() { return PassTw<N, E, 1>::total; }

// Fills the per-pass table (cooperatively, all threads of the block) from the base table
// base[k] = W_N^k = exp(-2 pi i k / N).
template <int N, int E, typename R, int NS = 1>
__device__ __forceinline__ void load_pass_twiddles(cx<R> *dst, const cx<R> *base) {
    using P = PassTw<N, E, NS>;
    if constexpr (NS > 1) {
        for (int e = threadIdx.x; e < P::own; e += blockDim.x) {
            const int t = e % P::T, qr = e / P::T, r = qr % (P::RAD - 1) + 1, q = qr / (P::RAD - 1);
            const int j = t + q * P::T, k = j & (NS - 1);
            dst[e] = base[(k * r) * (N / (NS * P::RAD))];
        }
    }
    if constexpr (!P::LAST)
        load_pass_twiddles<N, E, R, NS * P::RAD>(dst + P::own, base);
}

// One Stockham pass with stride NS; recursion over the remaining passes.  tw(i) returns
// entry i of this thread's between-pass twiddles: passes after the first in order, within a
// pass [q][r-1] (the per-pass table's entry i*T + t, or a register copy of it).
template <int N, int E, int SIGN, typename R, int NS, int TI, class Tw>
__device__ __forceinline__ void fft_pass(cx<R> (&v)[E], cx<R> *sm, const Tw &tw, int t) {
    constexpr int T = N / E;
    using P = PassTw<N, E, NS>;
    constexpr int RAD = P::RAD;
    constexpr int NB = P::NB;
    constexpr bool LAST = P::LAST;
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
                cx<R> w = tw(TI + q * (RAD - 1) + (r - 1));
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
        fft_pass<N, E, SIGN, R, NS * RAD, TI + P::own / T>(v, sm, tw, t);
    }
}

// Between-pass twiddles held per thread (a line position t keeps the same entries in every
// transform): registers in place of shared-memory loads.
template <int N, int E> __host__ __device__ constexpr int thread_twiddles() {
    return pass_twiddle_entries<N, E>() / (N / E) > 0 ? pass_twiddle_entries<N, E>() / (N / E) : 1;
}
template <int N, int E, typename R>
__device__ __forceinline__ void load_thread_twiddles(cx<R> (&twr)[thread_twiddles<N, E>()],
                                                     const cx<R> *tw, int t) {
    constexpr int T = N / E;
#pragma unroll
    for (int i = 0; i < thread_twiddles<N, E>(); ++i)
        twr[i] = i * T < pass_twiddle_entries<N, E>() ? tw[i * T + t] : mk<R>(1, 0);
}

// Unnormalised DFT of one line: X[k] = sum_n x[n] exp(SIGN 2 pi i n k / N).
// Thread t (0 <= t < N/E) holds x[t + r*(N/E)] in v[r] on entry and X[t + r*(N/E)] on exit.
// `tw` is the per-pass twiddle table (load_pass_twiddles).  Every lane of the warp must call
// this together (warp-synchronous exchanges).
template <int N, int E, int SIGN, typename R>
__device__ __forceinline__ void fft_line(cx<R> (&v)[E], cx<R> *sm, const cx<R> *tw, int t) {
    (void)FftShape<N, E>::T;
    constexpr int T = N / E;
    const auto get = [&](int i) { return tw[i * T + t]; };
    fft_pass<N, E, SIGN, R, 1, 0>(v, sm, get, t);
}
// The same with this thread's twiddles in registers (load_thread_twiddles).
template <int N, int E, int SIGN, typename R>
__device__ __forceinline__ void fft_line_rt(cx<R> (&v)[E], cx<R> *sm,
                                            const cx<R> (&twr)[thread_twiddles<N, E>()], int t) {
    const auto get = [&](int i) { return twr[i]; };
    fft_pass<N, E, SIGN, R, 1, 0>(v, sm, get, t);
}

} // namespace hzlb
