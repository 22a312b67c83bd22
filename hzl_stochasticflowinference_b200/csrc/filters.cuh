// Filter analysis kernels: systematic resampling, member gather, ensemble inflation and the
// perturbed-observation EnKF (innovation Gram, FP64 Cholesky and triangular solves, ensemble
// weight matrix, and the anomaly update X_a = X + A W).
#pragma once
#include "common.cuh"

namespace hzlb {

// Systematic resampling (filter.cpp:102-112).  One thread forms the cumulative weights with
// the reference's sequential left-to-right sum (so the rounding is identical); every thread
// then finds, for its positions u/M + i/M, the first ancestor whose cumulative weight is not
// below the position, which is where the reference's walk stops.
__global__ void systematic_resample_kernel(const double *w, double *cum, int count, double u,
                                           unsigned *ancestors) {
    if (threadIdx.x == 0) {
        double c = w[0];
        cum[0] = c;
        for (int a = 1; a < count; ++a) {
            c += w[a];
            cum[a] = c;
        }
    }
    __syncthreads();
    const double start = u / static_cast<double>(count);
    for (int i = threadIdx.x; i < count; i += blockDim.x) {
        const double position = start + static_cast<double>(i) / static_cast<double>(count);
        int lo = 0, hi = count - 1;   // smallest a with cum[a] >= position, capped at count-1
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (position > cum[mid])
                lo = mid + 1;
            else
                hi = mid;
        }
        ancestors[i] = static_cast<unsigned>(lo);
    }
}

// dst[i] = src[ancestor[i]] for member blocks of `block` complex entries.
template <typename R>
__global__ void gather_blocks(const cx<R> *src, cx<R> *dst, const unsigned *anc, long long block) {
    const int i = blockIdx.y;
    const cx<R> *s = src + static_cast<size_t>(anc[i]) * block;
    cx<R> *d = dst + static_cast<size_t>(i) * block;
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x)
        d[e] = s[e];
}

// x_m <- mean + inflation (x_m - mean) for every entry (filter.cpp:238-252).
template <typename R>
__global__ void inflate_kernel(cx<R> *x, long long block, int members, double inflation) {
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        double mr = 0, mi = 0;
        for (int m = 0; m < members; ++m) {
            mr += static_cast<double>(x[static_cast<size_t>(m) * block + e].x) / members;
            mi += static_cast<double>(x[static_cast<size_t>(m) * block + e].y) / members;
        }
        for (int m = 0; m < members; ++m) {
            cx<R> &v = x[static_cast<size_t>(m) * block + e];
            v.x = static_cast<R>(mr + inflation * (static_cast<double>(v.x) - mr));
            v.y = static_cast<R>(mi + inflation * (static_cast<double>(v.y) - mi));
        }
    }
}

// ---- EnKF ---------------------------------------------------------------------------
// HA[m][o] = HX[m][o] - mean_m HX[.][o];  D[m][o] = y_o + sd_o eps[m][o] - HX[m][o].
__global__ void enkf_innovations(const double *hx, const double *y, const double *sd,
                                 const double *eps, int members, int p, double *ha, double *d) {
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= p)
        return;
    double mean = 0;
    for (int m = 0; m < members; ++m)
        mean += hx[static_cast<size_t>(m) * p + o] / members;
    for (int m = 0; m < members; ++m) {
        const size_t i = static_cast<size_t>(m) * p + o;
        ha[i] = hx[i] - mean;
        d[i] = y[o] + sd[o] * eps[i] - hx[i];
    }
}
// P[a][b] = sum_m HA[m][a] HA[m][b] / (M-1) + (a == b) sd_a^2   (FP64, p x p)
__global__ void enkf_gram(const double *ha, const double *sd, int members, int p, double *P) {
    __shared__ double ta[16][17], tb[16][17];
    const int a = blockIdx.y * 16 + threadIdx.y, b = blockIdx.x * 16 + threadIdx.x;
    double s = 0;
    for (int m0 = 0; m0 < members; m0 += 16) {
        const int ma = m0 + threadIdx.x, mb = m0 + threadIdx.y;
        const int ra = blockIdx.y * 16 + threadIdx.y, rb = blockIdx.x * 16 + threadIdx.x;
        ta[threadIdx.y][threadIdx.x] = (ma < members && ra < p) ? ha[static_cast<size_t>(ma) * p + ra] : 0;
        tb[threadIdx.y][threadIdx.x] = (mb < members && rb < p) ? ha[static_cast<size_t>(mb) * p + rb] : 0;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k)
            s += ta[threadIdx.y][k] * tb[k][threadIdx.x];
        __syncthreads();
    }
    if (a < p && b < p)
        P[static_cast<size_t>(a) * p + b] = s / (members - 1) + (a == b ? sd[a] * sd[a] : 0.0);
}
// In-place Cholesky P = L L^T (lower triangle), one block, column by column (right-looking).
// info[0] is set to the first nonpositive pivot + 1 (0 on success).
__global__ void cholesky_kernel(double *P, int p, int *info) {
    __shared__ double pivot;
    if (threadIdx.x == 0)
        info[0] = 0;
    for (int k = 0; k < p; ++k) {
        if (threadIdx.x == 0) {
            const double d = P[static_cast<size_t>(k) * p + k];
            if (!(d > 0) && info[0] == 0)
                info[0] = k + 1;
            pivot = d > 0 ? sqrt(d) : 1.0;
            P[static_cast<size_t>(k) * p + k] = pivot;
        }
        __syncthreads();
        for (int i = k + 1 + threadIdx.x; i < p; i += blockDim.x)
            P[static_cast<size_t>(i) * p + k] /= pivot;
        __syncthreads();
        // trailing update of the lower triangle: P[i][j] -= L[i][k] L[j][k], k < j <= i;
        // one warp per row i, lanes over j
        const int warp = threadIdx.x / 32, lane = threadIdx.x % 32, warps = blockDim.x / 32;
        for (int i = k + 1 + warp; i < p; i += warps) {
            const double lik = P[static_cast<size_t>(i) * p + k];
            for (int j = k + 1 + lane; j <= i; j += 32)
                P[static_cast<size_t>(i) * p + j] -= lik * P[static_cast<size_t>(j) * p + k];
        }
        __syncthreads();
    }
}
// Solve L L^T z = d for every member's innovation vector (row m of D, in place).
__global__ void cholesky_solve(const double *L, int p, double *D, int members) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= members)
        return;
    double *z = D + static_cast<size_t>(m) * p;
    for (int i = 0; i < p; ++i) {
        double s = z[i];
        for (int k = 0; k < i; ++k)
            s -= L[static_cast<size_t>(i) * p + k] * z[k];
        z[i] = s / L[static_cast<size_t>(i) * p + i];
    }
    for (int i = p - 1; i >= 0; --i) {
        double s = z[i];
        for (int k = i + 1; k < p; ++k)
            s -= L[static_cast<size_t>(k) * p + i] * z[k];
        z[i] = s / L[static_cast<size_t>(i) * p + i];
    }
}
// W[a][m] = sum_o HA[a][o] Z[m][o] / (M-1)   (members x members, FP64)
__global__ void enkf_weights(const double *ha, const double *z, int members, int p, double *W) {
    __shared__ double ta[16][17], tb[16][17];
    const int a = blockIdx.y * 16 + threadIdx.y, m = blockIdx.x * 16 + threadIdx.x;
    double s = 0;
    for (int o0 = 0; o0 < p; o0 += 16) {
        const int oa = o0 + threadIdx.x, ob = o0 + threadIdx.y;
        ta[threadIdx.y][threadIdx.x] = (a < members && oa < p) ? ha[static_cast<size_t>(a) * p + oa] : 0;
        const int mb = blockIdx.x * 16 + threadIdx.x;
        tb[threadIdx.y][threadIdx.x] = (mb < members && ob < p) ? z[static_cast<size_t>(mb) * p + ob] : 0;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 16; ++k)
            s += ta[threadIdx.y][k] * tb[k][threadIdx.x];
        __syncthreads();
    }
    if (a < members && m < members)
        W[static_cast<size_t>(a) * members + m] = s / (members - 1);
}
// Column means of the ensemble state: mean[e] = sum_m X[m][e] / M.
template <typename R>
__global__ void ensemble_mean(const cx<R> *x, long long block, int members, cx<R> *mean) {
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        double mr = 0, mi = 0;
        for (int m = 0; m < members; ++m) {
            mr += static_cast<double>(x[static_cast<size_t>(m) * block + e].x) / members;
            mi += static_cast<double>(x[static_cast<size_t>(m) * block + e].y) / members;
        }
        mean[e] = mk<R>(static_cast<R>(mr), static_cast<R>(mi));
    }
}
// X_a[m][e] = X[m][e] + sum_a (X[a][e] - mean[e]) W[a][m]: a (members x 2*block) by
// (members x members) product, tiled 64 entries x 16 members with the W tile in shared memory.
template <typename R>
__global__ void anomaly_update(const cx<R> *x, const cx<R> *mean, const double *W, long long block,
                               int members, cx<R> *out) {
    __shared__ double ws[32][17];
    const long long e = static_cast<long long>(blockIdx.x) * 64 + threadIdx.x;
    const int m0 = blockIdx.y * 16;
    double accr[16], acci[16];
#pragma unroll
    for (int j = 0; j < 16; ++j)
        accr[j] = acci[j] = 0;
    const bool ve = e < block;
    const cx<R> mu = ve ? mean[e] : mk<R>(0, 0);
    for (int a0 = 0; a0 < members; a0 += 32) {
        __syncthreads();
        for (int t = threadIdx.x; t < 32 * 16; t += blockDim.x) {
            const int aa = a0 + t / 16, mm = m0 + t % 16;
            ws[t / 16][t % 16] = (aa < members && mm < members) ? W[static_cast<size_t>(aa) * members + mm] : 0;
        }
        __syncthreads();
        const int amax = min(32, members - a0);
        for (int a = 0; a < amax; ++a) {
            const cx<R> xa = ve ? x[static_cast<size_t>(a0 + a) * block + e] : mk<R>(0, 0);
            const double dr = static_cast<double>(xa.x) - static_cast<double>(mu.x);
            const double di = static_cast<double>(xa.y) - static_cast<double>(mu.y);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                accr[j] += dr * ws[a][j];
                acci[j] += di * ws[a][j];
            }
        }
    }
    if (!ve)
        return;
#pragma unroll
    for (int j = 0; j < 16; ++j) {
        const int m = m0 + j;
        if (m < members) {
            const cx<R> xm = x[static_cast<size_t>(m) * block + e];
            out[static_cast<size_t>(m) * block + e] =
                mk<R>(static_cast<R>(static_cast<double>(xm.x) + accr[j]),
                      static_cast<R>(static_cast<double>(xm.y) + acci[j]));
        }
    }
}

} // namespace hzlb

namespace hzlb {
// Round-to-nearest FP32 -> TF32 (10-bit mantissa), kept in an FP32 container.
__device__ __forceinline__ float to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}
// Split for 3xTF32 products: A = hi + lo with hi exactly representable in TF32; the products
// hi*hi + hi*lo + lo*hi recover FP32-level accuracy on the tensor cores.
// Anomalies a = x - mean of the member-major state (members x n reals).
__global__ void anomaly_split_tf32(const float *x, const float *mean, long long n, int members,
                                   float *hi, float *lo) {
    const long long total = n * members;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float a = x[i] - mean[i % n];
        const float h = to_tf32(a);
        hi[i] = h;
        lo[i] = a - h;
    }
}
__global__ void split_tf32(const double *w, long long count, float *hi, float *lo) {
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float v = static_cast<float>(w[i]);
        const float h = to_tf32(v);
        hi[i] = h;
        lo[i] = v - h;
    }
}
// out[e] = sum over members (in member order) of w[m] x[m][e], or of x[m][e] / divisor when
// divisor > 0 (the reference's mean accumulates coefficient / count, filter.cpp:238-243).
template <typename R>
__global__ void member_sum_kernel(const cx<R> *x, const double *w, double divisor, long long block,
                           int members, double *out) {
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        double sr = 0, si = 0;
        for (int m = 0; m < members; ++m) {
            const cx<R> v = x[static_cast<size_t>(m) * block + e];
            if (divisor > 0) {
                sr += static_cast<double>(v.x) / divisor;
                si += static_cast<double>(v.y) / divisor;
            } else {
                sr += w[m] * static_cast<double>(v.x);
                si += w[m] * static_cast<double>(v.y);
            }
        }
        out[2 * e] = sr;
        out[2 * e + 1] = si;
    }
}
// cov[e] = sum_m (x[m][e] - mean[e]) d[m], mean[e] = sum_m x[m][e] / M (filter.cpp:272-288).
template <typename R>
__global__ void member_covariance_kernel(const cx<R> *x, const double *d, long long block, int members,
                                  double *cov) {
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        double mr = 0, mi = 0;
        for (int m = 0; m < members; ++m) {
            const cx<R> v = x[static_cast<size_t>(m) * block + e];
            mr += static_cast<double>(v.x) / members;
            mi += static_cast<double>(v.y) / members;
        }
        double cr = 0, ci = 0;
        for (int m = 0; m < members; ++m) {
            const cx<R> v = x[static_cast<size_t>(m) * block + e];
            cr += (static_cast<double>(v.x) - mr) * d[m];
            ci += (static_cast<double>(v.y) - mi) * d[m];
        }
        cov[2 * e] = cr;
        cov[2 * e + 1] = ci;
    }
}
// x[m][e] += cov[e] innov[m]   (filter.cpp:314-318)
template <typename R>
__global__ void rank1_update(cx<R> *x, const double *cov, const double *innov, long long block,
                             int members) {
    const int m = blockIdx.y;
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        cx<R> &v = x[static_cast<size_t>(m) * block + e];
        v.x = static_cast<R>(static_cast<double>(v.x) + cov[2 * e] * innov[m]);
        v.y = static_cast<R>(static_cast<double>(v.y) + cov[2 * e + 1] * innov[m]);
    }
}
// Conjugate symmetry of the kx = 0 column (Solver::update_latent_state, solver.cpp:417-424):
// w(0, ky) <- (w(0, ky) + conj w(0, -ky)) / 2 for ky > 0, w(0, -ky) <- conj w(0, ky).
template <typename R> __global__ void symmetrize_column0(cx<R> *x, int n, int members) {
    const int K = (n - 1) / 3, LD = 2 * K + 1;
    const size_t block = static_cast<size_t>(K + 1) * LD;
    const int m = blockIdx.x;
    for (int ky = 1 + threadIdx.x; ky <= K; ky += blockDim.x) {
        cx<R> &a = x[m * block + ky], &b = x[m * block + (LD - ky)];
        const double re = 0.5 * (static_cast<double>(a.x) + static_cast<double>(b.x));
        const double im = 0.5 * (static_cast<double>(a.y) - static_cast<double>(b.y));
        a.x = static_cast<R>(re);
        a.y = static_cast<R>(im);
        b.x = static_cast<R>(re);
        b.y = static_cast<R>(-im);
    }
}
// sum over members and retained modes of |x - mean|^2 with Hermitian multiplicity (kx = 0
// column once, kx > 0 twice): the reference's spread numerator (filter.cpp:326-330).
template <typename R>
__global__ void spread_sum(const cx<R> *x, const double *mean, long long block, int ld, int members,
                           double *out) {
    double s = 0;
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double mult = e < ld ? 1.0 : 2.0;
        for (int m = 0; m < members; ++m) {
            const cx<R> v = x[static_cast<size_t>(m) * block + e];
            const double dr = static_cast<double>(v.x) - mean[2 * e],
                         di = static_cast<double>(v.y) - mean[2 * e + 1];
            s += mult * (dr * dr + di * di);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(out, s);
}
} // namespace hzlb
