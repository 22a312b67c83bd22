// TMA-fed variant of the tcgen05 GEMM (umma_gemm.cuh) for K-contiguous operands.
//
// Both operands arrive by tensor-map bulk copies (cp.async.bulk.tensor, no multicast) into a
// ring of ST shared-memory stages, each stage a [rows][128 bytes of K] box written with the
// 128-byte swizzle, which is the canonical K-major SWIZZLE_128B operand layout of the MMA
// (8-row x 128-byte atoms, SBO = 1024 bytes).  Roles inside the 4-warp CTA: thread 0 is the
// producer (waits for a stage to be released, arms its "full" barrier with the expected bytes,
// issues the two copies), thread 32 issues the MMAs (waits for "full", four 32-byte K steps per
// stage, commits the stage's "empty" barrier so the producer may refill it), and all four
// warps run the epilogue once the final commit lands and every copy has landed (store_tile:
// TMEM lanes to a shared-memory tile in the freed ring, then coalesced row writes).
// Out-of-range rows and K are zero-filled by the copy engine.  Every wait is bounded; on
// expiry the CTA records STATUS_TIMEOUT, waits (bounded) for what it issued, frees its TMEM
// and returns.
#pragma once
#include "umma_gemm.cuh"

#include <cuda.h>

namespace hzlb {
namespace tc {

// K-major, 128-byte swizzle: start address, LBO 16 bytes (unused for this layout), SBO 1024
// bytes between 8-row atoms, descriptor version 1, layout type 2 (SWIZZLE_128B).
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>(16 >> 4) << 16;
    d |= static_cast<uint64_t>(1024 >> 4) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    d |= static_cast<uint64_t>(2) << 61;
    return d;
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y,
                                            uint64_t *bar) {
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
                 : "memory");
}

template <int BN, int ST> constexpr size_t tma_smem() {
    // the ring (reused by the epilogue's 128 x (BN + 1) float tile) + alignment slack
    static_assert(static_cast<size_t>(ST) * (BM + BN) * SLAB >= static_cast<size_t>(BM) * (BN + 1) * 4,
                  "epilogue tile must fit in the ring");
    return static_cast<size_t>(ST) * (BM + BN) * SLAB + 1024;
}

// ta2 / tb2 map g.A2 / g.B2 when g.split3 > 0 (otherwise they repeat ta / tb, unused).
template <typename TIn, int BN, int ST>
__global__ void __launch_bounds__(128) umma_tma_kernel(const __grid_constant__ CUtensorMap ta,
                                                       const __grid_constant__ CUtensorMap tb,
                                                       const __grid_constant__ CUtensorMap ta2,
                                                       const __grid_constant__ CUtensorMap tb2,
                                                       const GemmArgs g) {
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "UMMA N for M = 128");
    constexpr bool TF32 = sizeof(TIn) == 4;
    constexpr int EPS = SLAB / sizeof(TIn);   // K elements per stage (128 bytes)
    constexpr uint32_t A_BYTES = BM * SLAB, B_BYTES = BN * SLAB;
    constexpr uint32_t IDESC = instr_desc(TF32 ? 2u : 1u, BM, BN);
    constexpr uint32_t NCOLS = BN <= 32 ? 32 : (BN <= 64 ? 64 : (BN <= 128 ? 128 : 256));
    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    unsigned char *sa = smem, *sb = smem + ST * A_BYTES;
    __shared__ __align__(8) uint64_t full[ST], empty[ST], done;
    __shared__ uint32_t tmem_base;
    __shared__ int err, issued_sh;

    const int warp = threadIdx.x / 32;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    int kb = 0, K = g.K;
    if (g.splits > 1) {
        kb = blockIdx.z * g.kchunk;
        K = g.K - kb < g.kchunk ? g.K - kb : g.kchunk;
    }
    // split3: slabs per K segment (each segment's tail is zero-filled by its map's extent)
    const int sps = g.split3 > 0 ? (g.split3 + EPS - 1) / EPS : 0;
    const int slabs = g.split3 > 0 ? 3 * sps : (K + EPS - 1) / EPS;
    if (warp == 0)
        tmem_alloc(&tmem_base, NCOLS);
    if (threadIdx.x == 32) {
        for (int i = 0; i < ST; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(&done, 1);
        mbar_init_fence();
        err = 0;
        issued_sh = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;
    prefetch_c_tile<BN>(g, m0, n0);

    if (threadIdx.x == 0) {
        // producer
        int issued = 0;
        for (int s = 0; s < slabs; ++s) {
            const int b = s % ST, u = s / ST;
            if (u > 0 && !mbar_wait_bounded(&empty[b], (u - 1) & 1)) {
                atomicExch(&err, 1);
                break;
            }
            const CUtensorMap *mapa = &ta, *mapb = &tb;
            int kk = kb + s * EPS;
            if (sps > 0) {
                const int seg = s / sps;
                kk = (s - seg * sps) * EPS;
                if (seg == 2)
                    mapa = &ta2;
                if (seg == 1)
                    mapb = &tb2;
            }
            mbar_arrive_expect(&full[b], A_BYTES + B_BYTES);
            tma_load_2d(sa + b * A_BYTES, mapa, kk, m0, &full[b]);
            tma_load_2d(sb + b * B_BYTES, mapb, kk, n0, &full[b]);
            issued = s + 1;
        }
        issued_sh = issued;
    } else if (threadIdx.x == 32) {
        // MMA issuer
        for (int s = 0; s < slabs; ++s) {
            const int b = s % ST, u = s / ST;
            if (!mbar_wait_bounded(&full[b], u & 1)) {
                atomicExch(&err, 1);
                break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(sa + b * A_BYTES), b0 = smem_u32(sb + b * B_BYTES);
#pragma unroll
            for (int h = 0; h < SLAB / 32; ++h)
                mma<TF32>(tmem, smem_desc_sw128(a0 + h * 32), smem_desc_sw128(b0 + h * 32), IDESC,
                          (s > 0 || h > 0) ? 1u : 0u);
            mma_commit(&empty[b]);
        }
        mma_commit(&done);   // arrives once every MMA issued above has completed
    }
    __syncthreads();
    __shared__ int ok_sh;
    if (threadIdx.x == 0) {
        bool ok = mbar_wait_bounded(&done, 0) && !err;
        // every copy issued must have landed before the CTA's shared memory is released
        const int issued = issued_sh;
        for (int s = issued > ST ? issued - ST : 0; s < issued; ++s)
            ok = mbar_wait_bounded(&full[s % ST], (s / ST) & 1) && ok;
        ok_sh = ok ? 1 : 0;
    }
    __syncthreads();
    if (ok_sh) {
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

} // namespace tc
} // namespace hzlb
