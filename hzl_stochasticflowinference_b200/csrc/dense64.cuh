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

// Factor the nb x nb diagonal block at (k0, k0) of S (row-major, ld p) in shared memory:
// S_kk = L L^T, written back (lower; upper part of the block zeroed), and L^{-1} (lower) to
// inv (ld NB).  info[0] = first nonpositive pivot + 1 (left at 0 on success).  L occupies the
// lower triangle of A and L^{-1} the rest, transposed and shifted one column right:
// (L^{-1})[i][c], i >= c, lives at A[c][i + 1].
static __global__ void __launch_bounds__(256) potrf_block(double *S, int p, int k0, int nb, double *inv,
                                                  int *info) {
    __shared__ double A[NB][NB + 1];
    __shared__ double piv[NB];
    const int tid = threadIdx.x;
    for (int q = tid; q < nb * nb; q += blockDim.x) {
        const int i = q / nb, j = q % nb;
        if (j <= i)
            A[i][j] = S[static_cast<long long>(k0 + i) * p + k0 + j];
    }
    __syncthreads();
    // right-looking elimination without scaling (one barrier per column): step j subtracts
    // A[i][j] A[l][j] / A[j][j] from the trailing lower triangle; column j is then final up to
    // the scaling by 1 / sqrt(A[j][j]) applied below
    for (int j = 0; j < nb; ++j) {
        const double d = A[j][j];
        if (tid == 0 && !(d > 0) && info[0] == 0)
            info[0] = k0 + j + 1;
        const double rinv = d > 0 ? 1.0 / d : 1.0;
        for (int i = j + 1 + (tid >> 4); i < nb; i += 16) {
            const double aij = A[i][j] * rinv;
            for (int l = j + 1 + (tid & 15); l <= i; l += 16)
                A[i][l] -= aij * A[l][j];
        }
        __syncthreads();
    }
    if (tid < nb)
        piv[tid] = A[tid][tid] > 0 ? sqrt(A[tid][tid]) : 1.0;
    __syncthreads();
    for (int q = tid; q < nb * nb; q += blockDim.x) {
        const int i = q / nb, j = q % nb;
        if (j < i)
            A[i][j] /= piv[j];
        else if (j == i)
            A[i][i] = piv[i];
    }
    __syncthreads();
    // L^{-1} by rows i, all columns c <= i at once; the four lanes of a column split the sum
    // and only ever exchange values among themselves, so a warp barrier orders them (every
    // lane takes part in the shuffles, so they stay warp-uniform)
    const int c = tid / 4, part = tid % 4;
    for (int i = 0; i < nb; ++i) {
        double s = 0;
        if (c < i)
            for (int l = c + part; l < i; l += 4)
                s += A[i][l] * A[c][l + 1];
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        if (part == 0 && c <= i && c < nb)
            A[c][i + 1] = c == i ? 1.0 / A[i][i] : -s / A[i][i];
        __syncwarp();
    }
    __syncthreads();
    for (int q = tid; q < nb * nb; q += blockDim.x) {
        const int i = q / nb, j = q % nb;
        S[static_cast<long long>(k0 + i) * p + k0 + j] = j <= i ? A[i][j] : 0.0;
        inv[i * NB + j] = j <= i ? A[j][i + 1] : 0.0;
    }
}

// In-place blocked Cholesky S = L L^T (lower triangle of S, row-major p x p); inv receives
// the inverses of the diagonal blocks (ceil(p/NB) blocks of NB x NB).  info must be zeroed.
// Only the lower triangle of S is read.
inline cudaError_t cholesky(double *S, int p, double *inv, int *info, cudaStream_t s) {
    for (int k0 = 0; k0 < p; k0 += NB) {
        const int nb = p - k0 < NB ? p - k0 : NB;
        double *ib = inv + static_cast<long long>(k0 / NB) * NB * NB;
        potrf_block<<<1, 256, 0, s>>>(S, p, k0, nb, ib, info);
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
