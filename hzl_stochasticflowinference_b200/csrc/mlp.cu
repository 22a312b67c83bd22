// Learned reduced forecast: a small MLP that advances POD coefficients by one forecast window,
//   y = a + s_out * L3(gelu(L2(gelu(L1(x / s_in)))))
// with x = (a, xi): r POD coefficients and q noise-mode amplitudes of the window; L1: (r+q) -> H,
// L2: H -> H, L3: H -> r.  Weights and activations are BF16, accumulation FP32, on the tcgen05
// tensor cores (umma_gemm.cuh); FP32 master weights with Adam.  No counterpart in the reference.
#include "engine.h"
#include "umma_gemm.cuh"

#include <cmath>
#include <cuda_bf16.h>
#include <memory>
#include <random>
#include <vector>

namespace hzlb {
namespace {

using bf16 = __nv_bfloat16;

__global__ void scale_to_bf16(const float *x, const float *scale, int rows, int cols, bf16 *out) {
    const long long total = static_cast<long long>(rows) * cols;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = __float2bfloat16(x[i] / scale[i % cols]);
}
// y[b][j] = x[b][j] + s_out[j] r[b][j] for the r coefficient columns of x (row stride in_cols)
__global__ void residual_out(const float *x, int in_cols, const float *r, const float *s_out,
                             int rows, int cols, float *y) {
    const long long total = static_cast<long long>(rows) * cols;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const long long b = i / cols;
        const int j = static_cast<int>(i % cols);
        y[i] = x[b * in_cols + j] + s_out[j] * r[i];
    }
}
// dr = s_out * 2 (y - t) / (rows cols); loss partial sums of (y - t)^2
__global__ void mse_grad(const float *y, const float *t, const float *s_out, int rows, int cols,
                         float *dr, bf16 *dr_bf, double *loss) {
    const long long total = static_cast<long long>(rows) * cols;
    double acc = 0;
    const float inv = 2.0f / static_cast<float>(total);
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float d = y[i] - t[i];
        acc += static_cast<double>(d) * d;
        const float g = s_out[i % cols] * d * inv;
        dr[i] = g;
        dr_bf[i] = __float2bfloat16(g);
    }
    for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0)
        atomicAdd(loss, acc);
}
__device__ __forceinline__ float gelu_grad(float x) {
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    const float u = k0 * (x + k1 * x * x * x);
    const float th = tanhf(u);
    return 0.5f * (1.0f + th) + 0.5f * x * (1.0f - th * th) * k0 * (1.0f + 3.0f * k1 * x * x);
}
// dpre = dh * gelu'(pre), FP32 and BF16 copies
__global__ void gelu_backward(const float *dh, const float *pre, long long total, float *dpre,
                              bf16 *dpre_bf) {
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float g = dh[i] * gelu_grad(pre[i]);
        dpre[i] = g;
        dpre_bf[i] = __float2bfloat16(g);
    }
}
// column sums (bias gradients): out[j] = sum_b d[b][j]
__global__ void column_sum(const float *d, int rows, int cols, float *out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols)
        return;
    float s = 0;
    for (int b = 0; b < rows; ++b)
        s += d[static_cast<long long>(b) * cols + j];
    out[j] = s;
}
// Adam on the FP32 master parameters, refreshing the BF16 copies of the weight matrices.
__global__ void adam_step(float *p, const float *g, float *m, float *v, long long count, float lr,
                          float beta1, float beta2, float eps, float c1, float c2, bf16 *p_bf,
                          long long bf_count) {
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const float gi = g[i];
        const float mi = beta1 * m[i] + (1 - beta1) * gi;
        const float vi = beta2 * v[i] + (1 - beta2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        if (i < bf_count)
            p_bf[i] = __float2bfloat16(pi);
    }
}
__global__ void to_bf16(const float *x, long long count, bf16 *out) {
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x)
        out[i] = __float2bfloat16(x[i]);
}

} // namespace

// Parameter block (FP32, contiguous): W1 [H][I], W2 [H][H], W3 [R][H], b1 [H], b2 [H], b3 [R].
// Weight matrices come first so their BF16 copies are one contiguous prefix.
class Mlp {
  public:
    Mlp(int r, int q, int hidden, int max_batch, int device, uint64_t seed)
        : R_(r), I_(r + q), H_(hidden), B_(max_batch) {
        if (r < 1 || q < 0 || hidden < 16 || hidden % 16 || max_batch < 1)
            raise(HZLB_EINVAL, "invalid MLP shape");
        cuda_check(cudaSetDevice(device), "select CUDA device");
        cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "create stream");
        w1_ = 0;
        w2_ = w1_ + static_cast<size_t>(H_) * I_;
        w3_ = w2_ + static_cast<size_t>(H_) * H_;
        b1_ = w3_ + static_cast<size_t>(R_) * H_;
        b2_ = b1_ + H_;
        b3_ = b2_ + H_;
        count_ = b3_ + R_;
        wcount_ = b1_;
        const size_t P = count_;
        params_.ensure(4 * P * sizeof(float), "allocate MLP parameters");   // p, grad, m, v
        pbf_.ensure(wcount_ * sizeof(bf16), "allocate MLP BF16 weights");
        scales_.ensure((I_ + R_) * sizeof(float), "allocate MLP scales");
        const size_t BI = static_cast<size_t>(B_) * I_, BH = static_cast<size_t>(B_) * H_,
                     BR = static_cast<size_t>(B_) * R_;
        act_.ensure(sizeof(float) * (2 * BH + 2 * BR + 2 * BH + BR) + 64, "allocate activations");
        actbf_.ensure(sizeof(bf16) * (BI + 2 * BH + BR + BH), "allocate BF16 activations");
        loss_.ensure(sizeof(double) + sizeof(uint32_t), "allocate loss and status");
        // He-style initialisation from a fixed seed
        std::vector<float> p(P, 0.0f);
        std::mt19937_64 rng(seed);
        std::normal_distribution<float> nd(0.0f, 1.0f);
        auto fill = [&](size_t off, int rows, int cols, float gain) {
            const float sd = gain / std::sqrt(static_cast<float>(cols));
            for (size_t i = 0; i < static_cast<size_t>(rows) * cols; ++i)
                p[off + i] = sd * nd(rng);
        };
        fill(w1_, H_, I_, 1.4f);
        fill(w2_, H_, H_, 1.4f);
        fill(w3_, R_, H_, 0.1f);
        std::vector<float> ones(I_ + R_, 1.0f);
        cuda_check(cudaMemset(params_.ptr, 0, params_.bytes), "clear MLP state");
        cuda_check(cudaMemset(loss_.ptr, 0, loss_.bytes), "clear MLP status");
        cuda_check(cudaMemcpy(params_.ptr, p.data(), P * sizeof(float), cudaMemcpyHostToDevice),
                   "upload MLP parameters");
        cuda_check(cudaMemcpy(scales_.ptr, ones.data(), ones.size() * sizeof(float),
                              cudaMemcpyHostToDevice),
                   "upload MLP scales");
        refresh_bf16();
        cuda_check(cudaStreamSynchronize(stream_), "initialise MLP");
    }
    ~Mlp() {
        if (stream_)
            cudaStreamDestroy(stream_);
    }
    size_t count() const { return count_; }
    void shape(int *r, int *q, int *hidden, int *max_batch) const {
        if (r)
            *r = R_;
        if (q)
            *q = I_ - R_;
        if (hidden)
            *hidden = H_;
        if (max_batch)
            *max_batch = B_;
    }
    void *stream() const { return stream_; }
    void set_params(const float *host) {
        cuda_check(cudaMemcpyAsync(params_.ptr, host, count_ * sizeof(float), cudaMemcpyHostToDevice,
                                   stream_),
                   "upload MLP parameters");
        refresh_bf16();
        cuda_check(cudaStreamSynchronize(stream_), "set MLP parameters");
    }
    void get_params(float *host, float *grads_host) {
        cuda_check(cudaMemcpyAsync(host, params_.ptr, count_ * sizeof(float), cudaMemcpyDeviceToHost,
                                   stream_),
                   "download MLP parameters");
        if (grads_host)
            cuda_check(cudaMemcpyAsync(grads_host, params_.as<float>() + count_,
                                       count_ * sizeof(float), cudaMemcpyDeviceToHost, stream_),
                       "download MLP gradients");
        cuda_check(cudaStreamSynchronize(stream_), "get MLP parameters");
    }
    void set_scales(const float *s_in, const float *s_out) {
        cuda_check(cudaMemcpyAsync(scales_.ptr, s_in, I_ * sizeof(float), cudaMemcpyHostToDevice,
                                   stream_),
                   "upload input scales");
        cuda_check(cudaMemcpyAsync(scales_.as<float>() + I_, s_out, R_ * sizeof(float),
                                   cudaMemcpyHostToDevice, stream_),
                   "upload output scales");
        cuda_check(cudaStreamSynchronize(stream_), "set MLP scales");
    }
    // y (B x R) = forward(x (B x I)); device pointers; keeps activations for backward
    void forward(const float *x, int B, float *y, cudaStream_t s) {
        check_batch(B);
        const size_t BH = static_cast<size_t>(B_) * H_;
        float *pre1 = act_.as<float>(), *pre2 = pre1 + BH, *r = pre2 + BH;
        bf16 *xbf = actbf_.as<bf16>(), *h1 = xbf + static_cast<size_t>(B_) * I_, *h2 = h1 + BH;
        const float *p = params_.as<float>();
        const bf16 *pb = pbf_.as<bf16>();
        scale_to_bf16<<<256, 256, 0, s>>>(x, scales_.as<float>(), B, I_, xbf);
        cuda_check(cudaGetLastError(), "launch input scaling");
        layer(xbf, pb + w1_, p + b1_, B, H_, I_, nullptr, h1, pre1, tc::EPI_BIAS_GELU, s);
        layer(h1, pb + w2_, p + b2_, B, H_, H_, nullptr, h2, pre2, tc::EPI_BIAS_GELU, s);
        layer(h2, pb + w3_, p + b3_, B, R_, H_, r, nullptr, nullptr, tc::EPI_BIAS, s);
        residual_out<<<256, 256, 0, s>>>(x, I_, r, scales_.as<float>() + I_, B, R_, y);
        cuda_check(cudaGetLastError(), "launch residual output");
    }
    // One training step on (x, target); returns the mean squared error before the update.
    double train_step(const float *x, const float *target, int B, float lr) {
        check_batch(B);
        cudaStream_t s = stream_;
        const size_t BH = static_cast<size_t>(B_) * H_, BR = static_cast<size_t>(B_) * R_;
        float *pre1 = act_.as<float>(), *pre2 = pre1 + BH, *r = pre2 + BH, *y = r + BR,
              *dh = y + BR, *dpre = dh + BH, *dr = dpre + BH;
        bf16 *xbf = actbf_.as<bf16>(), *h1 = xbf + static_cast<size_t>(B_) * I_, *h2 = h1 + BH,
             *drbf = h2 + BH, *dprebf = drbf + BR;
        float *p = params_.as<float>(), *g = p + count_, *m = g + count_, *v = m + count_;
        const bf16 *pb = pbf_.as<bf16>();
        forward(x, B, y, s);
        cuda_check(cudaMemsetAsync(loss_.ptr, 0, sizeof(double), s), "clear loss");
        mse_grad<<<256, 256, 0, s>>>(y, target, scales_.as<float>() + I_, B, R_, dr, drbf,
                                     loss_.as<double>());
        // layer 3: dW3 = dr^T h2, db3 = sum dr, dh2 = dr W3
        wgrad(drbf, h2, B, R_, H_, g + w3_, s);
        column_sum<<<(R_ + 127) / 128, 128, 0, s>>>(dr, B, R_, g + b3_);
        dgrad(drbf, pb + w3_, B, H_, R_, dh, s);
        gelu_backward<<<1024, 256, 0, s>>>(dh, pre2, static_cast<long long>(B) * H_, dpre, dprebf);
        // layer 2
        wgrad(dprebf, h1, B, H_, H_, g + w2_, s);
        column_sum<<<(H_ + 127) / 128, 128, 0, s>>>(dpre, B, H_, g + b2_);
        dgrad(dprebf, pb + w2_, B, H_, H_, dh, s);
        gelu_backward<<<1024, 256, 0, s>>>(dh, pre1, static_cast<long long>(B) * H_, dpre, dprebf);
        // layer 1
        wgrad(dprebf, xbf, B, H_, I_, g + w1_, s);
        column_sum<<<(H_ + 127) / 128, 128, 0, s>>>(dpre, B, H_, g + b1_);
        cuda_check(cudaGetLastError(), "launch MLP backward");
        if (lr > 0) {
            ++t_;
            const float b1 = 0.9f, b2 = 0.999f;
            const float c1 = 1 - std::pow(b1, static_cast<float>(t_)),
                        c2 = 1 - std::pow(b2, static_cast<float>(t_));
            adam_step<<<1024, 256, 0, s>>>(p, g, m, v, static_cast<long long>(count_), lr, b1, b2,
                                           1e-8f, c1, c2, pbf_.as<bf16>(),
                                           static_cast<long long>(wcount_));
            cuda_check(cudaGetLastError(), "launch Adam");
        }
        double loss = 0;
        cuda_check(cudaMemcpyAsync(&loss, loss_.ptr, sizeof(double), cudaMemcpyDeviceToHost, s),
                   "read loss");
        cuda_check(cudaStreamSynchronize(s), "MLP training step");
        check_status(s);
        return loss / (static_cast<double>(B) * R_);
    }

    // GEMM status bits (STATUS_TIMEOUT after an expired mbarrier wait); raises if set
    void check_status(cudaStream_t s) {
        uint32_t st = 0;
        cuda_check(cudaMemcpyAsync(&st, status(), sizeof(st), cudaMemcpyDeviceToHost, s),
                   "read MLP status");
        cuda_check(cudaStreamSynchronize(s), "MLP status");
        if (st)
            raise(HZLB_ERUNTIME, "tensor-core GEMM wait expired in the MLP");
    }

  private:
    uint32_t *status() const {
        return reinterpret_cast<uint32_t *>(static_cast<unsigned char *>(loss_.ptr) + sizeof(double));
    }
    void check_batch(int B) const {
        if (B < 1 || B > B_)
            raise(HZLB_EINVAL, "MLP batch exceeds the configured maximum");
    }
    void refresh_bf16() {
        to_bf16<<<256, 256, 0, stream_>>>(params_.as<float>(), static_cast<long long>(wcount_),
                                          pbf_.as<bf16>());
        cuda_check(cudaGetLastError(), "launch BF16 refresh");
    }
    // out (B x N) = in (B x K) W^T (+ bias, GELU)
    void layer(const bf16 *in, const bf16 *W, const float *bias, int B, int N, int K, float *out,
               bf16 *out_bf, float *pre, int epi, cudaStream_t s) {
        tc::GemmArgs g{};
        g.M = B;
        g.N = N;
        g.K = K;
        g.A = in;
        g.lda = K;
        g.a_kcontig = 1;
        g.B = W;
        g.ldb = K;
        g.b_kcontig = 1;
        g.C = out;
        g.Cbf = out_bf;
        g.ldc = N;
        g.alpha = 1.0f;
        g.beta = 0.0f;
        g.bias = bias;
        g.pre = pre;
        g.epilogue = epi;
        g.status = status();
        cuda_check(gemm(g, 2, s), "launch MLP layer");
    }
    // dW (N x K) = d^T (N x B) in (B x K)
    void wgrad(const bf16 *d, const bf16 *in, int B, int N, int K, float *dW, cudaStream_t s) {
        tc::GemmArgs g{};
        g.M = N;
        g.N = K;
        g.K = B;
        g.A = d;          // opA[n][b] = d[b][n]
        g.lda = N;
        g.a_kcontig = 0;
        g.B = in;         // opB[k][b] = in[b][k]
        g.ldb = K;
        g.b_kcontig = 0;
        g.C = dW;
        g.ldc = K;
        g.alpha = 1.0f;
        g.beta = 0.0f;
        g.epilogue = tc::EPI_NONE;
        g.status = status();
        cuda_check(gemm(g, 2, s), "launch MLP weight gradient");
    }
    // din (B x K) = d (B x N) W (N x K)
    void dgrad(const bf16 *d, const bf16 *W, int B, int K, int N, float *din, cudaStream_t s) {
        tc::GemmArgs g{};
        g.M = B;
        g.N = K;
        g.K = N;
        g.A = d;          // opA[b][n] = d[b][n]
        g.lda = N;
        g.a_kcontig = 1;
        g.B = W;          // opB[k][n] = W[n][k]
        g.ldb = K;
        g.b_kcontig = 0;
        g.C = din;
        g.ldc = K;
        g.alpha = 1.0f;
        g.beta = 0.0f;
        g.epilogue = tc::EPI_NONE;
        g.status = status();
        cuda_check(gemm(g, 2, s), "launch MLP input gradient");
    }

    int R_, I_, H_, B_;
    size_t w1_, w2_, w3_, b1_, b2_, b3_, count_, wcount_;
    cudaStream_t stream_ = nullptr;
    DeviceBuffer params_, pbf_, scales_, act_, actbf_, loss_;
    long long t_ = 0;
};

} // namespace hzlb

struct hzlb_mlp {
    std::unique_ptr<hzlb::Mlp> mlp;
};

namespace {
template <class F> int guarded_mlp(F &&f) {
    try {
        f();
        return HZLB_OK;
    } catch (const hzlb::Error &e) {
        hzlb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception &e) {
        hzlb::set_last_error(e.what());
        return HZLB_ERUNTIME;
    }
}
hzlb::Mlp &get(hzlb_mlp *h) {
    if (!h || !h->mlp)
        hzlb::raise(HZLB_EINVAL, "null MLP handle");
    return *h->mlp;
}
} // namespace

extern "C" {
HZLB_API int hzlb_mlp_create(int r, int q, int hidden, int max_batch, int device, uint64_t seed,
                             hzlb_mlp **out) {
    return guarded_mlp([&] {
        if (!out)
            hzlb::raise(HZLB_EINVAL, "null output");
        auto h = std::make_unique<hzlb_mlp>();
        h->mlp = std::make_unique<hzlb::Mlp>(r, q, hidden, max_batch, device, seed);
        *out = h.release();
    });
}
HZLB_API void hzlb_mlp_destroy(hzlb_mlp *h) { delete h; }
HZLB_API size_t hzlb_mlp_param_count(const hzlb_mlp *h) { return h && h->mlp ? h->mlp->count() : 0; }
HZLB_API int hzlb_mlp_shape(const hzlb_mlp *h, int *r, int *q, int *hidden, int *max_batch) {
    return guarded_mlp([&] {
        if (!h || !h->mlp)
            hzlb::raise(HZLB_EINVAL, "null MLP handle");
        h->mlp->shape(r, q, hidden, max_batch);
    });
}
HZLB_API int hzlb_mlp_set_params(hzlb_mlp *h, const float *params) {
    return guarded_mlp([&] { get(h).set_params(params); });
}
HZLB_API int hzlb_mlp_get_params(hzlb_mlp *h, float *params, float *grads) {
    return guarded_mlp([&] { get(h).get_params(params, grads); });
}
HZLB_API int hzlb_mlp_set_scales(hzlb_mlp *h, const float *s_in, const float *s_out) {
    return guarded_mlp([&] { get(h).set_scales(s_in, s_out); });
}
HZLB_API int hzlb_mlp_forward(hzlb_mlp *h, const float *x, int batch, float *y, void *stream) {
    return guarded_mlp([&] {
        auto &m = get(h);
        m.forward(x, batch, y, stream ? static_cast<cudaStream_t>(stream)
                                      : static_cast<cudaStream_t>(m.stream()));
        if (!stream)
            m.check_status(static_cast<cudaStream_t>(m.stream()));
    });
}
HZLB_API int hzlb_mlp_train_step(hzlb_mlp *h, const float *x, const float *target, int batch,
                                 float lr, double *loss) {
    return guarded_mlp([&] {
        const double l = get(h).train_step(x, target, batch, lr);
        if (loss)
            *loss = l;
    });
}
} // extern "C"
