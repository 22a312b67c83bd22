// Launchers and C ABI of the tcgen05 GEMM (umma_gemm.cuh).
#include "engine.h"
#include "umma_gemm.cuh"

namespace hzlb {
namespace {
template <typename TIn, int BN> cudaError_t launch(const tc::GemmArgs &g, cudaStream_t s) {
    constexpr size_t smem = tc::gemm_smem<TIn, BN>();
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(tc::umma_gemm_kernel<TIn, BN>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess)
            return e;
        configured[dev] = true;
    }
    const dim3 grid((g.N + BN - 1) / BN, (g.M + tc::BM - 1) / tc::BM, g.splits > 1 ? g.splits : 1);
    tc::umma_gemm_kernel<TIn, BN><<<grid, 128, smem, s>>>(g);
    return cudaGetLastError();
}
template <typename TIn> cudaError_t launch_any(const tc::GemmArgs &g, cudaStream_t s) {
    if (g.N >= 128)
        return launch<TIn, 128>(g, s);
    if (g.N > 32)
        return launch<TIn, 64>(g, s);
    return launch<TIn, 32>(g, s);
}
} // namespace

cudaError_t gemm(const tc::GemmArgs &g, int dtype, cudaStream_t s) {
    if (g.M <= 0 || g.N <= 0 || g.K <= 0)
        return cudaSuccess;
    return dtype == 2 ? launch_any<__nv_bfloat16>(g, s) : launch_any<float>(g, s);
}

} // namespace hzlb

extern "C" HZLB_API int hzlb_gemm(int M, int N, int K, int dtype, const void *A, long long lda,
                                  int a_kcontig, const void *B, long long ldb, int b_kcontig,
                                  float *C, long long ldc, float alpha, float beta, void *stream) {
    using namespace hzlb;
    if (M < 0 || N < 0 || K < 0 || (dtype != 2 && dtype != 4) || !A || !B || !C) {
        set_last_error("invalid GEMM arguments");
        return HZLB_EINVAL;
    }
    tc::GemmArgs g{};
    g.M = M;
    g.N = N;
    g.K = K;
    g.A = A;
    g.lda = lda;
    g.a_kcontig = a_kcontig;
    g.B = B;
    g.ldb = ldb;
    g.b_kcontig = b_kcontig;
    g.C = C;
    g.ldc = ldc;
    g.alpha = alpha;
    g.beta = beta;
    g.epilogue = tc::EPI_NONE;
    const cudaError_t e = gemm(g, dtype, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_last_error(std::string("launch GEMM: ") + cudaGetErrorString(e));
        return HZLB_ECUDA;
    }
    return HZLB_OK;
}
