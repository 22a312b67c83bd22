// FP64 dense linear algebra for the EnKF innovation system (p x p, p up to a few thousand):
// a GEMM with arbitrary operand strides on the FP64 tensor cores (mma.sync m8n8k4 f64 tiles;
// tcgen05 has no FP64 kind), a blocked right-looking Cholesky whose diagonal blocks are
// factored and inverted in shared memory, and blocked forward substitution for many
// right-hand sides built from the same GEMM.  FP64 stays here on purpose: the innovation
// Cholesky and solve are the one place the analysis needs it.
#pragma once
#include "common.cuh"

#include <cstdint>
#include <cuda_runtime.h>

namespace hzlb {
namespace d64 {

constexpr int BM = 64, BN = 64, BK = 16;   // GEMM tile; 4 warps of 32 x 32, 16 MMA tiles each
constexpr int GEMM_THREADS = 128;
constexpr int LDS = BM + 4;                 // shared row pitch: conflict-free fragment loads
constexpr int NB = 64;                      // Cholesky / substitution block

// C[m][n] = alpha sum_k A(m,k) B(k,n) + beta C[m][n],  A(m,k) = A[m*sam + k*sak],
// B(k,n) = B[k*sbk + n*sbn], C row-major with leading dimension ldc.
struct GemmArgs {
    int M, N, K;
    double alpha, beta;
    const double *A;
    long long sam, sak;
    const double *B;
    long long sbk, sbn;
    double *C;
    long long ldc;
};

// D (8 x 8) += A (8 x 4, row) B (4 x 8, col) on the FP64 tensor cores.  Lane l = 4g + t holds
// A[g][t], B[t][g] and D[g][2t], D[g][2t + 1].
__device__ __forceinline__ void dmma_8x8x4(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// One 64 x 64 tile of C per block.  Warp w owns rows 32 (w / 2) .. +32 and columns
// 32 (w % 2) .. +32 as 4 x 4 tiles of 8 x 8.  K advances in slabs of 16 staged through shared
// memory as [k][m] and [k][n] (any operand strides: the loads are coalesced along whichever
// index is contiguous); the next slab is read into registers while the tensor cores work on
// the current one.  Shared rows are LDS = 68 doubles apart, so the fragment loads of a half
// warp (k = t, m = g + 0..3 or 4..7) fall in 16 distinct 8-byte bank pairs.
// LOWER: skip tiles strictly above the diagonal (only C[m][n], n <= m, is wanted).  A block
// reads all of its A rows before it writes C, so C may alias the A rows of its own tile when
// N <= BN (one tile column).
template <bool LOWER> __global__ void __launch_bounds__(GEMM_THREADS) gemm_kernel(const GemmArgs g) {
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    if (LOWER && n0 > m0 + BM - 1)
        return;
    __shared__ double As[2][BK][LDS], Bs[2][BK][LDS];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32, lg = lane >> 2, lt = lane & 3;
    constexpr int PER = BM * BK / GEMM_THREADS;   // staged elements per thread and operand
    double acc[4][4][2] = {};
    const bool a_k = g.sak == 1, b_k = g.sbk == 1;
    double ra[PER], rb[PER];
    auto fetch = [&](int k0) {
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int q = tid + GEMM_THREADS * r;
            const int mk_m = a_k ? q / BK : q % BM, mk_k = a_k ? q % BK : q / BM;
            const int gm = m0 + mk_m, gk = k0 + mk_k;
            ra[r] = (gm < g.M && gk < g.K) ? g.A[gm * g.sam + gk * g.sak] : 0.0;
            const int kn_n = b_k ? q / BK : q % BN, kn_k = b_k ? q % BK : q / BN;
            const int gn = n0 + kn_n, gk2 = k0 + kn_k;
            rb[r] = (gn < g.N && gk2 < g.K) ? g.B[gk2 * g.sbk + gn * g.sbn] : 0.0;
        }
    };
    auto stash = [&](int buf) {
#pragma unroll
        for (int r = 0; r < PER; ++r) {
            const int q = tid + GEMM_THREADS * r;
            const int mk_m = a_k ? q / BK : q % BM, mk_k = a_k ? q % BK : q / BM;
            As[buf][mk_k][mk_m] = ra[r];
            const int kn_n = b_k ? q / BK : q % BN, kn_k = b_k ? q % BK : q / BN;
            Bs[buf][kn_k][kn_n] = rb[r];
        }
    };
    fetch(0);
    stash(0);
    __syncthreads();
    int buf = 0;
    for (int k0 = 0; k0 < g.K; k0 += BK) {
        const bool more = k0 + BK < g.K;
        if (more)
            fetch(k0 + BK);   // global loads in flight during the products below
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                a[i] = As[buf][kk + lt][wm + 8 * i + lg];
                b[i] = Bs[buf][kk + lt][wn + 8 * i + lg];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    dmma_8x8x4(acc[i][j], a[i], b[j]);
        }
        if (more) {
            stash(buf ^ 1);
            __syncthreads();
            buf ^= 1;
        }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int m = m0 + wm + 8 * i + lg;
        if (m >= g.M)
            continue;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int n = n0 + wn + 8 * j + 2 * lt + h;
                if (n >= g.N)
                    continue;
                double *c = g.C + m * g.ldc + n;
                *c = g.beta == 0.0 ? g.alpha * acc[i][j][h] : fma(g.alpha, acc[i][j][h], g.beta * *c);
            }
    }
}

// lower: only C[m][n], n <= m, is wanted.
inline cudaError_t gemm(const GemmArgs &g, cudaStream_t s, bool lower = false) {
    if (g.M <= 0 || g.N <= 0)
        return cudaSuccess;
    const dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM);
    if (lower)
        gemm_kernel<true><<<grid, GEMM_THREADS, 0, s>>>(g);
    else
        gemm_kernel<false><<<grid, GEMM_THREADS, 0, s>>>(g);
    return cudaGetLastError();
}

// Factor the nb x nb diagonal block at (k0, k0) of S (row-major, ld p): S_kk = L L^T, written
// back (lower; upper part of the block zeroed), and L^{-1} (lower) to inv (ld NB).  info[0] =
// first nonpositive pivot + 1 (left at 0 on success).
//
// One block of 64 threads; thread l holds column l in registers.  Elimination without
// scaling: at step j the owner of column j publishes it to shared memory (double-buffered, so
// one barrier a step suffices: a buffer is rewritten only after the next step's barrier, which
// every reader of it has passed) and every thread l > j subtracts A[i][j] A[l][j] / A[j][j]
// from its rows i > j.  A thread's rows shift up one register per step (the multiply-add writes
// row i + 1's result into the slot of row i), so the code of a step indexes registers at
// compile-time positions without unrolling the step loop: a fully unrolled 64 x 64 nest runs
// once, straight through, and measured instruction-fetch bound (161 us a block against 77 us
// for a shared-memory loop).  Afterwards each thread scales its column by 1 / sqrt(A[l][l]).
// The inverse is the same scheme on L x = e_l (one thread per column of L^{-1}) over L staged
// transposed in shared memory, with zero rows past the block so shifted reads stay in bounds.
// A ragged last block (nb < 64) is factored as diag(S_kk, I), whose padding stays the identity
// and is not written back.
constexpr int POTRF_LT = 2 * NB + 1;   // row pitch of the transposed factor (zero-padded rows)
constexpr size_t POTRF_SMEM = sizeof(double) * NB * POTRF_LT;
static __global__ void __launch_bounds__(NB) potrf_block(double *S, int p, int k0, int nb, double *inv,
                                                         int *info) {
    __shared__ double col[2][2 * NB];
    __shared__ double rdiag[NB];
    extern __shared__ double lt[];   // lt[k * POTRF_LT + i] = L[i][k], zero for i >= NB
    const int l = threadIdx.x;
    double a[NB];   // a[q] = row l + q of column l ... shifted: row j + q before step j
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int i = q;   // before the first step a[q] is row q
        if (l < nb && i < nb)
            a[q] = i >= l ? S[static_cast<long long>(k0 + i) * p + k0 + l] : 0.0;
        else
            a[q] = i == l ? 1.0 : 0.0;
    }
    col[0][NB + l] = 0.0;
    col[1][NB + l] = 0.0;
    for (int q = l; q < NB * POTRF_LT; q += NB)
        lt[q] = 0.0;
    __syncthreads();
    // elimination without scaling; thread l is active while l > j (its rows shift up one per
    // step, so a[0] is always the row of the current step) and publishes its column at j = l
#pragma unroll 1
    for (int j = 0; j < NB; ++j) {
        double *c = col[j & 1];
        if (l == j) {
#pragma unroll
            for (int q = 0; q < NB; ++q)
                if (q < NB - j)   // rows j + q of column j (the rest of the buffer stays zero)
                    c[j + q] = a[q];
            if (!(a[0] > 0) && info[0] == 0)
                info[0] = k0 + j + 1;
        }
        __syncthreads();
        if (l > j) {
            const double d = c[j];
            const double t = c[l] * (d > 0 ? 1.0 / d : 1.0);
            const double *cr = c + j + 1;
#pragma unroll
            for (int q = 0; q < NB - 1; ++q)
                a[q] = fma(-cr[q], t, a[q + 1]);
            a[NB - 1] = 0.0;
        }
    }
    // thread l: a[q] = A[l + q][l]; column l of L is a[q] / sqrt(a[0]) below, sqrt(a[0]) on it
    const double piv = a[0] > 0 ? sqrt(a[0]) : 1.0, rp = 1.0 / piv;
    double *lc = lt + l * POTRF_LT;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
        const int i = l + q;
        const double v = q == 0 ? piv : a[q] * rp;
        if (i < NB) {
            lc[i] = v;
            if (i < nb && l < nb)
                S[static_cast<long long>(k0 + i) * p + k0 + l] = v;
        }
    }
    // the block's upper part is zero
    for (int i = 0; i < l && i < nb; ++i)
        if (l < nb)
            S[static_cast<long long>(k0 + i) * p + k0 + l] = 0.0;
    rdiag[l] = rp;
    __syncthreads();
    // column l of L^{-1} by forward substitution L x = e_l, right-looking: b[q] is the residual
    // of row k + q before step k; x_k = b[0] / L[k][k]; the rows below lose L[k+1+q][k] x_k
    double *b = a;
#pragma unroll
    for (int q = 0; q < NB; ++q)
        b[q] = q == l ? 1.0 : 0.0;
#pragma unroll 1
    for (int k = 0; k < NB; ++k) {
        const double x = b[0] * rdiag[k];
        if (k < nb && l < nb)
            inv[k * NB + l] = x;
        else
            inv[k * NB + l] = 0.0;
        const double *lk = lt + k * POTRF_LT + k + 1;
#pragma unroll
        for (int q = 0; q < NB - 1; ++q)
            b[q] = fma(-lk[q], x, b[q + 1]);
        b[NB - 1] = 0.0;
    }
}

// In-place blocked Cholesky S = L L^T (lower triangle of S, row-major p x p); inv receives
// the inverses of the diagonal blocks (ceil(p/NB) blocks of NB x NB).  info must be zeroed.
// Only the lower triangle of S is read.
static inline cudaError_t cholesky(double *S, int p, double *inv, int *info, cudaStream_t s) {
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        const cudaError_t e = cudaFuncSetAttribute(potrf_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   static_cast<int>(POTRF_SMEM));
        if (e != cudaSuccess)
            return e;
        configured[dev] = true;
    }
    for (int k0 = 0; k0 < p; k0 += NB) {
        const int nb = p - k0 < NB ? p - k0 : NB;
        double *ib = inv + static_cast<long long>(k0 / NB) * NB * NB;
        potrf_block<<<1, NB, POTRF_SMEM, s>>>(S, p, k0, nb, ib, info);
        const int pr = p - k0 - nb;
        if (pr > 0) {
            // panel: L_ik = S_ik L_kk^{-T}, in place (one tile column since nb <= BN)
            GemmArgs g{pr, nb, nb, 1.0, 0.0, S + static_cast<long long>(k0 + nb) * p + k0, p, 1,
                       ib, 1, NB, S + static_cast<long long>(k0 + nb) * p + k0, p};
            cudaError_t e = gemm(g, s);
            if (e != cudaSuccess)
                return e;
            // trailing update of the lower triangle: S_rest -= L_panel L_panel^T
            GemmArgs t{pr, pr, nb, -1.0, 1.0, S + static_cast<long long>(k0 + nb) * p + k0, p, 1,
                       S + static_cast<long long>(k0 + nb) * p + k0, 1, p,
                       S + static_cast<long long>(k0 + nb) * p + k0 + nb, p};
            e = gemm(t, s, true);
            if (e != cudaSuccess)
                return e;
        }
    }
    return cudaGetLastError();
}

// Forward substitution L y = d for each of `rows` right-hand sides stored as the rows of D
// (rows x p, row-major): the solutions go to Y (rows x p); D is overwritten on the way.
inline cudaError_t forward_rows(const double *L, int p, const double *inv, double *D, double *Y,
                                int rows, cudaStream_t s) {
    const int nblk = (p + NB - 1) / NB;
    // Y_k = (D_k - sum_{j<k} Y_j L_kj^T) L_kk^{-T}, right-looking on D
    for (int b = 0; b < nblk; ++b) {
        const int k0 = b * NB, nb = p - k0 < NB ? p - k0 : NB, pr = p - k0 - nb;
        const double *ib = inv + static_cast<long long>(b) * NB * NB;
        GemmArgs g{rows, nb, nb, 1.0, 0.0, D + k0, p, 1, ib, 1, NB, Y + k0, p};
        cudaError_t e = gemm(g, s);
        if (e != cudaSuccess)
            return e;
        if (pr > 0) {
            GemmArgs u{rows, pr, nb, -1.0, 1.0, Y + k0, p, 1,
                       L + static_cast<long long>(k0 + nb) * p + k0, 1, p, D + k0 + nb, p};
            e = gemm(u, s);
            if (e != cudaSuccess)
                return e;
        }
    }
    return cudaGetLastError();
}

} // namespace d64
} // namespace hzlb
