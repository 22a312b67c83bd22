// Dense contractions on the 5th-generation tensor cores (tcgen05 / UMMA, sm_100a).
//
//   C[M x N] = alpha * opA[M x K] * opB[N x K]^T + beta * C      (FP32 accumulate in TMEM)
//
// opA / opB are BF16 (kind::f16) or FP32 read as TF32 (kind::tf32), each given either
// K-contiguous ([rows][K]) or rows-contiguous ([K][rows]).  One CTA (4 warps) computes a
// 128 x BN tile: all threads stage 128 x 64-byte (A) and BN x 64-byte (B) slabs of K into shared
// memory in the canonical K-major core-matrix layout (8 rows x 16 bytes per core matrix, no
// swizzle); one elected thread issues the MMAs (two per slab, 32 bytes of K each) and commits
// them to an mbarrier; the slabs are double-buffered so staging overlaps the tensor cores.  The
// accumulator lives in TMEM (BN 32-bit columns) and is read back with tcgen05.ld (warp w owns
// lanes 32w..32w+31 = rows) for the epilogue.  Every mbarrier wait is bounded; on expiry the
// CTA records STATUS_TIMEOUT, frees its TMEM and returns.
#pragma once
#include "async_copy.cuh"
#include "common.cuh"

#include <cuda_bf16.h>

namespace hzlb {
namespace tc {

// ---- descriptors ---------------------------------------------------------------------
// Shared-memory matrix descriptor, K-major, no swizzle: start address, leading byte offset
// (between the two core matrices along K of one MMA), stride byte offset (between 8-row
// groups), descriptor version 1.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;
}
// Instruction descriptor: FP32 accumulate, A/B format (1 = BF16, 2 = TF32), both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t instr_desc(uint32_t ab_format, int M, int N) {
    return (1u << 4) | (ab_format << 7) | (ab_format << 10) |
           (static_cast<uint32_t>(N >> 3) << 17) | (static_cast<uint32_t>(M >> 4) << 24);
}

// ---- tcgen05 wrappers ------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}
template <bool TF32>
__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                    uint32_t accumulate) {
    if constexpr (TF32)
        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                     " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
                     "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                     : "memory");
    else
        asm volatile("{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                     " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem_d),
                     "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
                     : "memory");
}
// Arrive on `bar` when all previously issued MMAs of this thread have completed.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
// 32 lanes x 16 consecutive 32-bit columns per warp.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
                 "%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i)
        v[i] = __uint_as_float(r[i]);
}

enum Epilogue : int { EPI_NONE = 0, EPI_BIAS = 1, EPI_BIAS_GELU = 2 };

struct GemmArgs {
    int M, N, K;
    const void *A;
    long long lda;
    int a_kcontig;   // 1: A[m*lda + k], 0: A[k*lda + m]
    const void *B;
    long long ldb;
    int b_kcontig;   // 1: B[n*ldb + k], 0: B[k*ldb + n]
    float *C;        // FP32 output (may be null if only Cbf is wanted)
    long long ldc;
    __nv_bfloat16 *Cbf;   // optional BF16 copy of the output
    float alpha, beta;
    const float *bias;    // per-column bias (EPI_BIAS*)
    float *pre;           // optional pre-activation output (EPI_BIAS_GELU), ldc
    int epilogue;
    unsigned int *status;
};

constexpr int BM = 128;
constexpr int SLAB = 64;   // bytes of K per staged slab (2 MMAs of 32 bytes)

template <typename TIn> __device__ __forceinline__ float to_f(TIn v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) {
    return __bfloat162float(v);
}

// Stages rows [row0, row0 + ROWS) x K-bytes [kb0, kb0 + SLAB) of an operand into the
// core-matrix layout: chunk c (16 bytes) of row r at ((r/8) * 4 + c) * 128 + (r%8) * 16.
template <typename TIn, int ROWS>
__device__ __forceinline__ void stage_slab(unsigned char *dst, const TIn *src, long long ld,
                                           bool kcontig, int rows, int K, int row0, int k0) {
    constexpr int EPC = 16 / sizeof(TIn);   // elements per 16-byte chunk
    for (int q = threadIdx.x; q < ROWS * 4; q += blockDim.x) {
        const int r = q % ROWS, c = q / ROWS;
        const int gr = row0 + r, gk = k0 + c * EPC;
        alignas(16) TIn vals[EPC];
        if (kcontig && gr < rows && gk + EPC <= K &&
            (reinterpret_cast<uintptr_t>(src + gr * ld + gk) & 15) == 0) {
            const uint4 raw = *reinterpret_cast<const uint4 *>(src + gr * ld + gk);
            *reinterpret_cast<uint4 *>(vals) = raw;
        } else {
#pragma unroll
            for (int e = 0; e < EPC; ++e) {
                const int kk = gk + e;
                TIn v;
                if (gr < rows && kk < K)
                    v = kcontig ? src[gr * ld + kk] : src[static_cast<long long>(kk) * ld + gr];
                else
                    v = TIn(0.0f);
                vals[e] = v;
            }
        }
        *reinterpret_cast<uint4 *>(dst + ((r / 8) * 4 + c) * 128 + (r % 8) * 16) =
            *reinterpret_cast<const uint4 *>(vals);
    }
}

__device__ __forceinline__ float gelu(float x) {
    // tanh approximation of GELU (Hendrycks & Gimpel)
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    return 0.5f * x * (1.0f + tanhf(k0 * (x + k1 * x * x * x)));
}

template <typename TIn, int BN>
__global__ void __launch_bounds__(128) umma_gemm_kernel(const GemmArgs g) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M = 128");
    constexpr bool TF32 = sizeof(TIn) == 4;
    constexpr int EPS = SLAB / sizeof(TIn);   // K elements per slab
    constexpr uint32_t A_BYTES = BM * SLAB, B_BYTES = BN * SLAB;
    constexpr uint32_t IDESC = instr_desc(TF32 ? 2u : 1u, BM, BN);
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sa = smem;                          // [2][A_BYTES]
    unsigned char *sb = smem + 2 * A_BYTES;            // [2][B_BYTES]
    __shared__ __align__(8) uint64_t bars[3];          // slab 0, slab 1 consumed; final
    __shared__ uint32_t tmem_base;
    __shared__ int ok_sh;

    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const TIn *A = static_cast<const TIn *>(g.A);
    const TIn *B = static_cast<const TIn *>(g.B);
    const int warp = threadIdx.x / 32;
    constexpr uint32_t NCOLS = BN < 32 ? 32 : (BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256)));
    if (warp == 0)
        tmem_alloc(&tmem_base, NCOLS);
    if (threadIdx.x == 0) {
        mbar_init(&bars[0], 1);
        mbar_init(&bars[1], 1);
        mbar_init(&bars[2], 1);
        mbar_init_fence();
        ok_sh = 1;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    const int slabs = (g.K + EPS - 1) / EPS;
    uint32_t uses[2] = {0, 0};
    bool ok = true;
    for (int s = 0; s < slabs; ++s) {
        const int b = s & 1;
        // the MMAs that read this buffer two slabs ago must be done before it is refilled
        if (s >= 2) {
            if (threadIdx.x == 0)
                ok_sh = mbar_wait_bounded(&bars[b], (uses[b] - 1) & 1) ? ok_sh : 0;
            __syncthreads();
            if (!ok_sh) {
                ok = false;
                break;
            }
        }
        stage_slab<TIn, BM>(sa + b * A_BYTES, A, g.lda, g.a_kcontig, g.M, g.K, m0, s * EPS);
        stage_slab<TIn, BN>(sb + b * B_BYTES, B, g.ldb, g.b_kcontig, g.N, g.K, n0, s * EPS);
        fence_proxy_async_shared();   // generic-proxy stores -> visible to the tensor cores
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sa + b * A_BYTES), b0 = smem_u32(sb + b * B_BYTES);
#pragma unroll
            for (int h = 0; h < 2; ++h)   // two 32-byte K steps: core matrices 2h, 2h+1
                mma<TF32>(tmem, smem_desc(a0 + h * 256, 128, 512), smem_desc(b0 + h * 256, 128, 512),
                          IDESC, (s > 0 || h > 0) ? 1u : 0u);
            mma_commit(&bars[b]);
        }
        ++uses[b];
    }
    // all issued MMAs complete (or, after a failed wait, a bounded wait for them) before the
    // accumulator is read or freed
    if (threadIdx.x == 0) {
        mma_commit(&bars[2]);
        const bool done = mbar_wait_bounded(&bars[2], 0);
        ok_sh = (ok && done) ? 1 : 0;
    }
    __syncthreads();
    ok = ok_sh != 0;
    if (ok) {
        tc_fence_after();
        // epilogue: warp w reads rows 32w..32w+31 (TMEM lanes), 16 columns at a time
        const int row = m0 + warp * 32 + (threadIdx.x % 32);
        for (int c0 = 0; c0 < BN; c0 += 16) {
            float v[16];
            tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
            if (row < g.M) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int col = n0 + c0 + i;
                    if (col >= g.N)
                        continue;
                    float x = g.alpha * v[i];
                    const long long at = static_cast<long long>(row) * g.ldc + col;
                    if (g.beta != 0.0f && g.C)
                        x += g.beta * g.C[at];
                    if (g.epilogue >= EPI_BIAS)
                        x += g.bias[col];
                    if (g.epilogue == EPI_BIAS_GELU) {
                        if (g.pre)
                            g.pre[at] = x;
                        x = gelu(x);
                    }
                    if (g.C)
                        g.C[at] = x;
                    if (g.Cbf)
                        g.Cbf[at] = __float2bfloat16(x);
                }
            }
        }
    } else if (threadIdx.x == 0 && g.status) {
        atomicOr(g.status, STATUS_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        tmem_dealloc(tmem, NCOLS);
}

template <typename TIn, int BN> constexpr size_t gemm_smem() {
    return 2 * (BM * SLAB + BN * SLAB);
}

} // namespace tc
} // namespace hzlb
