// Dense contractions on the 5th-generation tensor cores (tcgen05 / UMMA, sm_100a).
//
//   C[M x N] = alpha * opA[M x K] * opB[N x K]^T + beta * C      (FP32 accumulate in TMEM)
//
// opA / opB are BF16 (kind::f16) or FP32 read as TF32 (kind::tf32), each given either
// K-contiguous ([rows][K]) or rows-contiguous ([K][rows]).  One CTA (4 warps) computes a
// 128 x BN tile.  K advances in slabs of 128 bytes per row held in a STAGES-deep ring of shared
// memory buffers in the canonical K-major core-matrix layout (8 rows x 16 bytes per core matrix,
// no swizzle).  K-contiguous, 16-byte aligned operands are copied with cp.async (16-byte chunks,
// zero-filled past the matrix edges), STAGES - 1 slabs ahead of the tensor cores; other layouts
// are staged by plain loads.  One elected thread issues the MMAs (four per slab, 32 bytes of K
// each) and commits them to the slab buffer's mbarrier, which gates the buffer's refill.  The
// accumulator lives in TMEM (BN 32-bit columns) and is read back with tcgen05.ld (warp w owns
// lanes 32w..32w+31 = rows) for the epilogue.  Every mbarrier wait is bounded; on expiry the
// CTA records STATUS_TIMEOUT, drains its copies, frees its TMEM and returns.
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
    // split-K: with splits > 1, blockIdx.z takes K elements [z kchunk, (z+1) kchunk) (kchunk a
    // multiple of the slab width, every split nonempty) and writes alpha * its partial product
    // to partial[z][M][N] (no beta, bias or activation); the caller sums the slices.
    int splits;
    int kchunk;
    float *partial;
    // 3xTF32 in one product (TMA path): with split3 > 0, K = 3 split3 and the K range is three
    // segments of split3 elements whose A operands are (A, A, A2) and B operands (B, B2, B),
    // so one accumulator sums A B + A B2 + A2 B -- hi hi + hi lo + lo hi of split operands --
    // and C is read and written once.  A2 and B2 have the layouts of A and B.
    const void *A2, *B2;
    int split3;
};

constexpr int BM = 128;
constexpr int SLAB = 128;   // bytes of K per staged slab (4 MMAs of 32 bytes)
constexpr int CPR = SLAB / 16;   // 16-byte chunks per row of a slab
constexpr int STAGES = 3;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <typename TIn> __device__ __forceinline__ float to_f(TIn v);
template <> __device__ __forceinline__ float to_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) {
    return __bfloat162float(v);
}

// Stages rows [row0, row0 + ROWS) x K-elements [k0, k0 + SLAB / sizeof(TIn)) of an operand
// into the core-matrix layout: chunk c (16 bytes) of row r at ((r/8) * CPR + c) * 128 + (r%8) * 16.
// Lane l of each warp takes row 8g + l%8 and chunk 4h + l/8, so a warp writes 512 contiguous
// bytes of shared memory and reads 64 contiguous bytes of each of 8 rows.  `fast`: K-contiguous
// with 16-byte aligned rows, copied by cp.async (the caller commits and waits); otherwise plain
// loads and stores.
template <typename TIn, int ROWS>
__device__ __forceinline__ void stage_slab(unsigned char *dst, const TIn *src, long long ld,
                                           bool kcontig, bool fast, int rows, int K, int row0,
                                           int k0) {
    constexpr int EPC = 16 / sizeof(TIn);   // elements per 16-byte chunk
    for (int q = threadIdx.x; q < ROWS * CPR; q += blockDim.x) {
        const int l = q % 32, wq = q / 32;
        const int r = (wq / (CPR / 4)) * 8 + l % 8, c = (wq % (CPR / 4)) * 4 + l / 8;
        const int gr = row0 + r, gk = k0 + c * EPC;
        unsigned char *d = dst + ((r / 8) * CPR + c) * 128 + (r % 8) * 16;
        if (fast) {
            const int left = gr < rows ? (K - gk) * static_cast<int>(sizeof(TIn)) : 0;
            const int bytes = left < 0 ? 0 : (left > 16 ? 16 : left);
            const TIn *from = bytes > 0 ? src + static_cast<long long>(gr) * ld + gk : src;
            cp_async16(smem_u32(d), from, bytes);
            continue;
        }
        alignas(16) TIn vals[EPC];
#pragma unroll
        for (int e = 0; e < EPC; ++e) {
            const int kk = gk + e;
            TIn v;
            if (gr < rows && kk < K)
                v = kcontig ? src[static_cast<long long>(gr) * ld + kk]
                            : src[static_cast<long long>(kk) * ld + gr];
            else
                v = TIn(0.0f);
            vals[e] = v;
        }
        *reinterpret_cast<uint4 *>(d) = *reinterpret_cast<const uint4 *>(vals);
    }
}

__device__ __forceinline__ float gelu(float x) {
    // tanh approximation of GELU (Hendrycks & Gimpel)
    const float k0 = 0.7978845608028654f, k1 = 0.044715f;
    return 0.5f * x * (1.0f + tanhf(k0 * (x + k1 * x * x * x)));
}

// Warps 2 and 3 are idle while thread 0 feeds and thread 32 issues the MMAs: when the epilogue
// will read C back (beta != 0, no split-K partials), they bring the tile's rows of C into L2
// (one prefetch per 128-byte line), so that read overlaps the main loop instead of following it.
template <int BN>
__device__ __forceinline__ void prefetch_c_tile(const GemmArgs &g, int m0, int n0) {
    if (threadIdx.x < 64 || g.splits > 1 || g.beta == 0.0f || !g.C)
        return;
    constexpr int LINES = BN / 32;   // 128-byte lines of a tile row
    for (int i = static_cast<int>(threadIdx.x) - 64; i < BM * LINES; i += 64) {
        const int row = m0 + i / LINES, col = n0 + (i % LINES) * 32;
        if (row < g.M && col < g.N)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(g.C + static_cast<long long>(row) * g.ldc + col));
    }
}

// Epilogue of a 128 x BN accumulator tile: each warp copies its 32 TMEM lanes (rows) to the
// shared-memory tile `stage` (row stride BN + 1 floats, conflict-free), then writes its rows
// back with lanes along the columns, so every global read and write is a contiguous 128-byte
// row segment.  `stage` must hold 128 x (BN + 1) floats and be free (all copies landed, all
// MMAs complete).
template <int BN>
__device__ __forceinline__ void store_tile(const GemmArgs &g, uint32_t tmem, float *stage, int m0,
                                           int n0) {
    constexpr int TS = BN + 1;
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    float *mine = stage + warp * 32 * TS;
    for (int c0 = 0; c0 < BN; c0 += 16) {
        float v[16];
        tmem_ld16(tmem + (static_cast<uint32_t>(warp * 32) << 16) + c0, v);
#pragma unroll
        for (int i = 0; i < 16; ++i)
            mine[lane * TS + c0 + i] = v[i];
    }
    __syncwarp();
    static_assert(BN % 32 == 0, "store_tile: BN multiple of 32");
    constexpr int CPL = BN / 32;   // columns per lane
    constexpr int RB = 8;          // rows per batch: their C reads are all issued first
    const bool split = g.splits > 1;
    const bool read_c = !split && g.beta != 0.0f && g.C;
    for (int r0 = 0; r0 < 32; r0 += RB) {
        float cin[RB][CPL];
#pragma unroll
        for (int rr = 0; rr < RB; ++rr)
#pragma unroll
            for (int j = 0; j < CPL; ++j) {
                const int row = m0 + warp * 32 + r0 + rr, col = n0 + lane + 32 * j;
                cin[rr][j] = (read_c && row < g.M && col < g.N)
                                 ? g.C[static_cast<long long>(row) * g.ldc + col]
                                 : 0.0f;
            }
#pragma unroll
        for (int rr = 0; rr < RB; ++rr) {
            const int row = m0 + warp * 32 + r0 + rr;
            if (row >= g.M)
                break;
#pragma unroll
            for (int j = 0; j < CPL; ++j) {
                const int c = lane + 32 * j, col = n0 + c;
                if (col >= g.N)
                    continue;
                float x = g.alpha * mine[(r0 + rr) * TS + c];
                if (split) {
                    g.partial[(static_cast<long long>(blockIdx.z) * g.M + row) * g.N + col] = x;
                    continue;
                }
                const long long at = static_cast<long long>(row) * g.ldc + col;
                if (read_c)
                    x += g.beta * cin[rr][j];
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
}

template <typename TIn, int BN>
__global__ void __launch_bounds__(128) umma_gemm_kernel(const GemmArgs g) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M = 128");
    constexpr bool TF32 = sizeof(TIn) == 4;
    constexpr int EPS = SLAB / sizeof(TIn);   // K elements per slab
    constexpr uint32_t A_BYTES = BM * SLAB, B_BYTES = BN * SLAB;
    constexpr uint32_t IDESC = instr_desc(TF32 ? 2u : 1u, BM, BN);
    constexpr uint32_t SBO = CPR * 128;       // byte distance between 8-row core-matrix groups
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *sa = smem;                          // [STAGES][A_BYTES]
    unsigned char *sb = smem + STAGES * A_BYTES;       // [STAGES][B_BYTES]
    __shared__ __align__(8) uint64_t bars[STAGES + 1];   // per-buffer MMA completion; final
    __shared__ uint32_t tmem_base;
    __shared__ int ok_sh;

    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const TIn *A = static_cast<const TIn *>(g.A);
    const TIn *B = static_cast<const TIn *>(g.B);
    int K = g.K;
    if (g.splits > 1) {
        const int kb = blockIdx.z * g.kchunk;
        K = g.K - kb < g.kchunk ? g.K - kb : g.kchunk;
        A += g.a_kcontig ? static_cast<long long>(kb) : static_cast<long long>(kb) * g.lda;
        B += g.b_kcontig ? static_cast<long long>(kb) : static_cast<long long>(kb) * g.ldb;
    }
    const bool a_fast = g.a_kcontig && (reinterpret_cast<uintptr_t>(A) & 15) == 0 &&
                        (g.lda * static_cast<long long>(sizeof(TIn))) % 16 == 0;
    const bool b_fast = g.b_kcontig && (reinterpret_cast<uintptr_t>(B) & 15) == 0 &&
                        (g.ldb * static_cast<long long>(sizeof(TIn))) % 16 == 0;
    const int warp = threadIdx.x / 32;
    constexpr uint32_t NCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    if (warp == 0)
        tmem_alloc(&tmem_base, NCOLS);
    if (threadIdx.x == 0) {
        for (int i = 0; i <= STAGES; ++i)
            mbar_init(&bars[i], 1);
        mbar_init_fence();
        ok_sh = 1;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    const int slabs = (K + EPS - 1) / EPS;
    auto load = [&](int s) {
        const int b = s % STAGES;
        stage_slab<TIn, BM>(sa + b * A_BYTES, A, g.lda, g.a_kcontig, a_fast, g.M, K, m0, s * EPS);
        stage_slab<TIn, BN>(sb + b * B_BYTES, B, g.ldb, g.b_kcontig, b_fast, g.N, K, n0, s * EPS);
    };
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < slabs)
            load(s);
        cp_async_commit();
    }
    bool ok = true;
    for (int s = 0; s < slabs; ++s) {
        const int b = s % STAGES;
        // slab s has landed: its copy group (and every earlier one) is complete
        cp_async_wait<STAGES - 2>();
        fence_proxy_async_shared();   // generic/async-copy writes -> visible to the tensor cores
        __syncthreads();
        if (threadIdx.x == 0) {
            tc_fence_after();
            const uint32_t a0 = smem_u32(sa + b * A_BYTES), b0 = smem_u32(sb + b * B_BYTES);
#pragma unroll
            for (int h = 0; h < SLAB / 32; ++h)   // 32-byte K steps: core matrices 2h, 2h+1
                mma<TF32>(tmem, smem_desc(a0 + h * 256, 128, SBO), smem_desc(b0 + h * 256, 128, SBO),
                          IDESC, (s > 0 || h > 0) ? 1u : 0u);
            mma_commit(&bars[b]);
        }
        // refill the buffer of slab s - 1 with slab s + STAGES - 1 once its MMAs are done
        const int sn = s + STAGES - 1;
        if (sn < slabs && s >= 1) {
            if (threadIdx.x == 0)
                ok_sh = mbar_wait_bounded(&bars[(s - 1) % STAGES], ((s - 1) / STAGES) & 1) ? ok_sh : 0;
            __syncthreads();
            if (!ok_sh) {
                ok = false;
                break;
            }
        }
        if (sn < slabs)
            load(sn);
        cp_async_commit();
    }
    cp_async_wait<0>();
    // all issued MMAs complete (or, after a failed wait, a bounded wait for them) before the
    // accumulator is read or freed
    if (threadIdx.x == 0) {
        mma_commit(&bars[STAGES]);
        const bool done = mbar_wait_bounded(&bars[STAGES], 0);
        ok_sh = (ok && done) ? 1 : 0;
    }
    __syncthreads();
    ok = ok_sh != 0;
    if (ok) {
        tc_fence_after();
        store_tile<BN>(g, tmem, reinterpret_cast<float *>(smem), m0, n0);
    } else if (threadIdx.x == 0 && g.status) {
        atomicOr(g.status, STATUS_TIMEOUT);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        tmem_dealloc(tmem, NCOLS);
}

template <typename TIn, int BN> constexpr size_t gemm_smem() {
    // the ring, which the epilogue reuses for the 128 x (BN + 1) float tile
    return STAGES * (BM * SLAB + BN * SLAB) > BM * (BN + 1) * 4 ? STAGES * (BM * SLAB + BN * SLAB)
                                                                : BM * (BN + 1) * 4;
}

} // namespace tc
} // namespace hzlb
