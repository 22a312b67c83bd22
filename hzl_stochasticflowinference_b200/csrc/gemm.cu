// Launchers and C ABI of the tcgen05 GEMM: the TMA-fed kernel (umma_tma.cuh) when both
// operands are K-contiguous with 16-byte aligned rows, the cp.async kernel (umma_gemm.cuh)
// otherwise.
#include "engine.h"
#include "umma_gemm.cuh"
#include "umma_tma.cuh"

#include <mutex>

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
// Tensor map of a K-contiguous operand (rows x K, row stride ld elements): boxes of
// box_rows x 128 bytes, 128-byte swizzle, zero fill out of range.
template <typename TIn>
bool make_map(CUtensorMap *map, const void *ptr, int rows, int K, long long ld, int box_rows) {
    EncodeTiled fn = tensor_map_encoder();
    if (!fn || (reinterpret_cast<uintptr_t>(ptr) & 15) || (ld * sizeof(TIn)) % 16)
        return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(K), static_cast<cuuint64_t>(rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(ld * sizeof(TIn))};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(tc::SLAB / sizeof(TIn)),
                               static_cast<cuuint32_t>(box_rows)};
    const cuuint32_t estr[2] = {1, 1};
    const CUtensorMapDataType dt =
        sizeof(TIn) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    return fn(map, dt, 2, const_cast<void *>(ptr), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}
template <typename TIn, int BN, int ST> cudaError_t launch_tma(const tc::GemmArgs &g, cudaStream_t s,
                                                               bool &used) {
    used = false;
    CUtensorMap ma, mb, ma2, mb2;
    const int kext = g.split3 > 0 ? g.split3 : g.K;
    if (!make_map<TIn>(&ma, g.A, g.M, kext, g.lda, tc::BM) ||
        !make_map<TIn>(&mb, g.B, g.N, kext, g.ldb, BN))
        return cudaSuccess;
    ma2 = ma;
    mb2 = mb;
    if (g.split3 > 0 && (!make_map<TIn>(&ma2, g.A2, g.M, kext, g.lda, tc::BM) ||
                         !make_map<TIn>(&mb2, g.B2, g.N, kext, g.ldb, BN)))
        return cudaSuccess;
    constexpr size_t smem = tc::tma_smem<BN, ST>();
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(tc::umma_tma_kernel<TIn, BN, ST>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess)
            return e;
        configured[dev] = true;
    }
    const dim3 grid((g.N + BN - 1) / BN, (g.M + tc::BM - 1) / tc::BM, g.splits > 1 ? g.splits : 1);
    tc::umma_tma_kernel<TIn, BN, ST><<<grid, 128, smem, s>>>(ma, mb, ma2, mb2, g);
    used = true;
    return cudaGetLastError();
}
template <typename TIn> cudaError_t launch_any(const tc::GemmArgs &g, cudaStream_t s);
// A split3 product whose operands the TMA path cannot map: the three terms one after another.
template <typename TIn> cudaError_t launch_split3_terms(const tc::GemmArgs &g, cudaStream_t s) {
    const void *as[3] = {g.A, g.A, g.A2}, *bs[3] = {g.B, g.B2, g.B};
    for (int i = 0; i < 3; ++i) {
        tc::GemmArgs t = g;
        t.split3 = 0;
        t.K = g.split3;
        t.A = as[i];
        t.B = bs[i];
        if (i > 0)
            t.beta = 1.0f;
        const cudaError_t e = launch_any<TIn>(t, s);
        if (e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}
template <typename TIn> cudaError_t launch_any(const tc::GemmArgs &g, cudaStream_t s) {
    if (g.split3 > 0 && (!g.a_kcontig || !g.b_kcontig || g.splits > 1 || g.epilogue != tc::EPI_NONE))
        return launch_split3_terms<TIn>(g, s);
    if (g.a_kcontig && g.b_kcontig) {
        bool used = false;
        cudaError_t e;
        if (g.N >= 128)
            e = launch_tma<TIn, 128, 3>(g, s, used);
        else if (g.N > 32)
            e = launch_tma<TIn, 64, 4>(g, s, used);
        else
            e = launch_tma<TIn, 32, 4>(g, s, used);
        if (e != cudaSuccess || used)
            return e;
        if (g.split3 > 0)
            return launch_split3_terms<TIn>(g, s);
    }
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
