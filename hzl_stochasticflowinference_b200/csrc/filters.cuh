// Filter analysis kernels: systematic resampling, member gather, ensemble inflation and the
// element-wise parts of the perturbed-observation EnKF (innovations, perturbations, the
// innovation statistic and the anomaly update X_a = X + A W); its FP64 Gram, Cholesky and
// solves are in dense64.cuh.
#pragma once
#include "common.cuh"

#include <math_constants.h>

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

// ---- particle-filter weights (filter.cpp:65-112) ------------------------------------
// Outcome of one observation time for one segment (an independent filter over `particles`
// consecutive members); the layout of hzlb_pf_record.
struct PfRecord {
    double increment, ess, max_weight;
    int resampled, collapsed;
};

// log w_m of every member (one thread per member): the prior term -- the log of the member's
// normalised weight (minus infinity for a zero weight) when `prior` is set, else the value
// already in logs[m] -- then, observation by observation in the reference's order,
//   value -= 0.5 r^2 + log sd_o + half_log_two_pi,   r = (H x_m - y_o) / sd_o
// (filter.cpp:65-75).  Every product and sum is rounded on its own (no fused multiply-add),
// as the reference's CPU build evaluates them.  hx is members x p (observe_device); members of
// inactive segments are left as they are.
__global__ void pf_loglik_kernel(const double *hx, int p, const double *values, const double *sd,
                                 double half_log_two_pi, const double *prior, double *logs,
                                 int members, int particles, const unsigned char *active) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < members; m += gridDim.x * blockDim.x) {
        if (active && !active[m / particles])
            continue;
        double value;
        if (prior)
            value = prior[m] > 0 ? log(prior[m]) : -CUDART_INF;
        else
            value = logs[m];
        const double *h = hx + static_cast<size_t>(m) * p;
        for (int o = 0; o < p; ++o) {
            const double r = __ddiv_rn(__dsub_rn(h[o], values[o]), sd[o]);
            const double term = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(0.5, r), r), log(sd[o])),
                                          half_log_two_pi);
            value = __dsub_rn(value, term);
        }
        logs[m] = value;
    }
}

template <int TPB> __device__ __forceinline__ double block_max(double v, double *red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    __syncthreads();   // `red` may still be read from an earlier call
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x / 32] = v;
    __syncthreads();
    double r = red[0];
#pragma unroll
    for (int w = 1; w < TPB / 32; ++w)
        r = fmax(r, red[w]);
    return r;
}

// One block per segment s of `particles` members (filter.cpp:76-112), skipped when active[s]
// is 0 (identity ancestors, record untouched):
//  * maximum: the first log-weight, then every larger one (std::max_element: a NaN in first
//    place is the maximum, NaNs elsewhere are passed over); not finite -> collapsed, nothing
//    else changes;
//  * increment = max + log(sum_j exp(l_j - max)), the sum formed left to right by one thread;
//  * w_j = exp(l_j - increment) (written to `weights`), ESS = 1 / sum_j w_j^2 (left to right,
//    each square rounded before the sum), largest weight;
//  * with u[s] in [0, 1) and ESS < particles / 2: systematic resampling -- the cumulative
//    weights left to right by one thread, each position u/P + i/P located by binary search
//    (the first ancestor whose cumulative weight is not below it, as the reference's walk
//    stops), ancestors as member indices.  The weights keep their normalised values (the
//    reset to 1/P follows in pf_reset_resampled, after any weighted mean of this time).
// `scratch` holds `members` doubles.
template <int TPB>
__global__ void __launch_bounds__(TPB)
    pf_normalise_kernel(const double *logs, double *weights, double *scratch, int particles,
                        const double *u, const unsigned char *active, PfRecord *rec,
                        unsigned *anc) {
    __shared__ double red[TPB / 32];
    __shared__ double total_sh;
    const int s = blockIdx.x, tid = threadIdx.x;
    const size_t base = static_cast<size_t>(s) * particles;
    const double *l = logs + base;
    double *w = weights + base, *x = scratch + base;
    unsigned *as = anc + base;
    const auto identity = [&] {
        for (int i = tid; i < particles; i += TPB)
            as[i] = static_cast<unsigned>(base + i);
    };
    if (active && !active[s]) {
        identity();
        return;
    }
    double mx = l[0];
    if (!isnan(mx))
        for (int i = tid; i < particles; i += TPB)
            mx = fmax(mx, l[i]);
    mx = isnan(l[0]) ? l[0] : block_max<TPB>(mx, red);
    if (!isfinite(mx)) {
        identity();
        if (tid == 0)
            rec[s] = PfRecord{-CUDART_INF, 0.0, 0.0, 0, 1};
        return;
    }
    for (int i = tid; i < particles; i += TPB)
        x[i] = exp(__dsub_rn(l[i], mx));
    __syncthreads();
    if (tid == 0) {
        double t = 0;
        for (int i = 0; i < particles; ++i)
            t = __dadd_rn(t, x[i]);
        total_sh = t;
    }
    __syncthreads();
    const double increment = __dadd_rn(mx, log(total_sh));
    double mw = 0;
    for (int i = tid; i < particles; i += TPB) {
        const double wi = exp(__dsub_rn(l[i], increment));
        w[i] = wi;
        x[i] = wi;
        mw = fmax(mw, wi);
    }
    mw = block_max<TPB>(mw, red);
    if (tid == 0) {
        double q = 0;
        for (int i = 0; i < particles; ++i)
            q = __dadd_rn(q, __dmul_rn(x[i], x[i]));
        total_sh = q;
    }
    __syncthreads();
    const double ess = 1.0 / total_sh;
    const bool resample = u && u[s] >= 0.0 && ess < static_cast<double>(particles) / 2;
    if (resample) {
        if (tid == 0) {
            double c = w[0];
            x[0] = c;
            for (int a = 1; a < particles; ++a) {
                c = __dadd_rn(c, w[a]);
                x[a] = c;
            }
        }
        __syncthreads();
        const double start = u[s] / static_cast<double>(particles);
        for (int i = tid; i < particles; i += TPB) {
            const double position = __dadd_rn(start, static_cast<double>(i) / static_cast<double>(particles));
            int lo = 0, hi = particles - 1;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (position > x[mid])
                    lo = mid + 1;
                else
                    hi = mid;
            }
            as[i] = static_cast<unsigned>(base + lo);
        }
    } else {
        identity();
    }
    if (tid == 0)
        rec[s] = PfRecord{increment, ess, mw, resample ? 1 : 0, 0};
}

// out[s][e] = sum over the members j of segment s, in member order, of w_j x_j[e] (the
// bootstrap filter's weighted mean, filter.cpp:113-120), as interleaved doubles; grid.y =
// segments.  Inactive and collapsed segments are written too (their weights as they stand).
template <typename R>
__global__ void segment_weighted_sum(const cx<R> *x, const double *w, long long block, int particles,
                                     double *out) {
    const int s = blockIdx.y;
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x) {
        double sr = 0, si = 0;
        for (int j = 0; j < particles; ++j) {
            const size_t m = static_cast<size_t>(s) * particles + j;
            const cx<R> v = x[m * block + e];
            sr = __dadd_rn(sr, __dmul_rn(w[m], static_cast<double>(v.x)));
            si = __dadd_rn(si, __dmul_rn(w[m], static_cast<double>(v.y)));
        }
        out[2 * (static_cast<size_t>(s) * block + e)] = sr;
        out[2 * (static_cast<size_t>(s) * block + e) + 1] = si;
    }
}

// Weights of the segments that were resampled back to 1/particles (filter.cpp:117).
__global__ void pf_reset_resampled(double *weights, const PfRecord *rec, int members, int particles) {
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < members; m += gridDim.x * blockDim.x)
        if (rec[m / particles].resampled)
            weights[m] = 1.0 / static_cast<double>(particles);
}

// dst[i] = src[anc[i]] for the members of resampled segments only (grid.y = members), then
// pf_commit_resampled copies them back: the members of other segments move nowhere.
template <typename R>
__global__ void pf_gather_resampled(const cx<R> *src, cx<R> *dst, const unsigned *anc,
                                    const PfRecord *rec, int particles, long long block) {
    const int i = blockIdx.y;
    if (!rec[i / particles].resampled)
        return;
    const cx<R> *s = src + static_cast<size_t>(anc[i]) * block;
    cx<R> *d = dst + static_cast<size_t>(i) * block;
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x)
        d[e] = s[e];
}
template <typename R>
__global__ void pf_commit_resampled(const cx<R> *src, cx<R> *dst, const PfRecord *rec, int particles,
                                    long long block) {
    const int i = blockIdx.y;
    if (!rec[i / particles].resampled)
        return;
    const cx<R> *s = src + static_cast<size_t>(i) * block;
    cx<R> *d = dst + static_cast<size_t>(i) * block;
    for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < block;
         e += static_cast<long long>(gridDim.x) * blockDim.x)
        d[e] = s[e];
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

// Member means of a member-major array (members x n values of T): out[e] = sum_m x[m][e] / M.
// Blocks of (32, 8): 32 columns, eight warps over interleaved member slices, FP64 sums
// combined in shared memory.  Grid x = ceil(n / 32).
template <typename T>
__global__ void member_mean(const T *x, long long n, int members, T *out) {
    __shared__ double part[8][33];
    const long long e = static_cast<long long>(blockIdx.x) * 32 + threadIdx.x;
    double s = 0;
    if (e < n)
        for (int m = threadIdx.y; m < members; m += 8)
            s += static_cast<double>(x[static_cast<long long>(m) * n + e]);
    part[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.y == 0 && e < n) {
        double t = 0;
        for (int w = 0; w < 8; ++w)
            t += part[w][threadIdx.x];
        out[e] = static_cast<T>(t / members);
    }
}

// x_m <- mean + inflation (x_m - mean) for every entry (filter.cpp:238-252), with the member
// mean from member_mean; x is viewed as members x n reals.
template <typename R>
__global__ void inflate_kernel(R *x, const R *mean, long long n, int members, double inflation) {
    const long long total = n * members;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double m = static_cast<double>(mean[i % n]);
        x[i] = static_cast<R>(m + inflation * (static_cast<double>(x[i]) - m));
    }
}

// ---- EnKF ---------------------------------------------------------------------------
// Observation perturbation of member m, observation o, analysis `cycle`: a standard normal
// from the Philox stream keyed by (seed, member); the counter's step word carries the cycle
// with a domain tag in its high half so these draws never coincide with forcing noise.
__device__ __forceinline__ double enkf_perturbation(uint64_t seed, uint32_t member, uint64_t cycle,
                                                    int o) {
    double xi1, xi2;
    philox_normal_pair(seed, member, cycle ^ (0x454E4B46ull << 32), static_cast<uint32_t>(o >> 1),
                       xi1, xi2);
    return (o & 1) ? xi2 : xi1;
}
// HA[m][o] = HX[m][o] - mean[o];  D[m][o] = y_o + sd_o eps[m][o] - HX[m][o] for m < M and the
// mean innovation D[M][o] = y_o - mean[o].  eps: host-supplied M x p normals, or (eps == null)
// enkf_perturbation(seed, member_base + m, cycle, o).
__global__ void enkf_innovations(const double *hx, const double *mean, const double *y,
                                 const double *sd, const double *eps, uint64_t seed,
                                 uint32_t member_base, uint64_t cycle, int members, int p,
                                 double *ha, double *d) {
    const long long total = static_cast<long long>(members + 1) * p;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int m = static_cast<int>(i / p), o = static_cast<int>(i % p);
        if (m == members) {
            d[i] = y[o] - mean[o];
            continue;
        }
        const double e = eps ? eps[i] : enkf_perturbation(seed, member_base + m, cycle, o);
        ha[i] = hx[i] - mean[o];
        d[i] = y[o] + sd[o] * e - hx[i];
    }
}
// P[a][a] += sd_a^2 (observation error on the diagonal of the innovation covariance)
__global__ void add_obs_variance(double *P, const double *sd, int p) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < p)
        P[static_cast<size_t>(a) * p + a] += sd[a] * sd[a];
}
// Normalised innovation statistic dbar^T S^{-1} dbar / p = |L^{-1} dbar|^2 / p, given
// w = L^{-1} dbar with S = L L^T (one block).
__global__ void innovation_statistic(const double *w, int p, double *out) {
    __shared__ double part[32];
    double s = 0;
    for (int o = threadIdx.x; o < p; o += blockDim.x)
        s += w[o] * w[o];
    for (int k = 16; k > 0; k >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, k);
    if ((threadIdx.x & 31) == 0)
        part[threadIdx.x / 32] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x / 32); ++w)
            t += part[w];
        *out = t / p;
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
// The operands of the update product X += A W are written transposed, member index
// contiguous, so it is the K dimension of both tensor-core operands; 32 x 32 tiles pass through
// shared memory so reads and writes stay coalesced.  Launch with blockDim (32, 8).
// Anomalies a[m][e] = x[m][e] - mean[e] of the member-major state (members x n reals) ->
// hiT[e][m], loT[e][m].
__global__ void anomaly_split_tf32_t(const float *x, const float *mean, long long n, int members,
                                     float *hiT, float *loT) {
    __shared__ float t[32][33];
    const long long e0 = static_cast<long long>(blockIdx.x) * 32;
    const int m0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int m = m0 + r;
        const long long e = e0 + threadIdx.x;
        t[r][threadIdx.x] = (m < members && e < n) ? x[static_cast<long long>(m) * n + e] - mean[e]
                                                   : 0.0f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const long long e = e0 + r;
        const int m = m0 + threadIdx.x;
        if (e < n && m < members) {
            const float a = t[threadIdx.x][r];
            const float h = to_tf32(a);
            hiT[e * members + m] = h;
            loT[e * members + m] = a - h;
        }
    }
}
// Ensemble weights W[a][m] (members x members, FP64) -> hiT[m][a], loT[m][a].
__global__ void split_tf32_t(const double *w, int members, float *hiT, float *loT) {
    __shared__ float t[32][33];
    const int a0 = blockIdx.x * 32, m0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int a = a0 + r, m = m0 + threadIdx.x;
        t[r][threadIdx.x] = (a < members && m < members)
                                ? static_cast<float>(w[static_cast<long long>(a) * members + m])
                                : 0.0f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int m = m0 + r, a = a0 + threadIdx.x;
        if (a < members && m < members) {
            const float v = t[threadIdx.x][r];
            const float h = to_tf32(v);
            hiT[static_cast<long long>(m) * members + a] = h;
            loT[static_cast<long long>(m) * members + a] = v - h;
        }
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
