// Shared device helpers for the B200 ensemble spectral path.
//
// Complex values are (x = re, y = im) pairs of float or double.  Spectral state lives in the
// compact dealiased half-spectrum layout: for grid N the retained wave numbers are
// |k| <= K = (N-1)/3 (strict 2/3 rule 3|k| < N of the reference, src/solver.cpp:133-134);
// columns kx = 0..K, and in each column 2K+1 entries j, ky = j for j <= K and
// ky = j - (2K+1) above (FFT order).  Member m's state is the contiguous block
// [m][kx][j].  Negative kx are implied by Hermitian symmetry.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace hzlb {

// Interleaved complex value, aligned to its size (as float2 / double2) so that one load or
// store moves both parts; device buffers of cx<R> must be aligned to sizeof(cx<R>).
template <typename R> struct alignas(2 * sizeof(R)) cx {
    R x, y;
};
template <typename R> __host__ __device__ __forceinline__ cx<R> mk(R a, R b) {
    cx<R> r;
    r.x = a;
    r.y = b;
    return r;
}
template <typename R> __device__ __forceinline__ cx<R> operator+(cx<R> a, cx<R> b) {
    return mk(a.x + b.x, a.y + b.y);
}
template <typename R> __device__ __forceinline__ cx<R> operator-(cx<R> a, cx<R> b) {
    return mk(a.x - b.x, a.y - b.y);
}
template <typename R> __device__ __forceinline__ cx<R> cmul(cx<R> a, cx<R> b) {
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R> __device__ __forceinline__ cx<R> scale(R s, cx<R> a) {
    return mk(s * a.x, s * a.y);
}
// FP32: the real and imaginary halves go through one packed sm_100 instruction (add.f32x2,
// mul.f32x2, fma.f32x2), half the issue slots of two scalar ones with the same rounding; a - b
// is a + (-1) b as one fused multiply-add, whose product is exact, so it rounds as a subtraction.
__device__ __forceinline__ float2 f2(cx<float> a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ cx<float> c2(float2 a) { return mk(a.x, a.y); }
template <> __device__ __forceinline__ cx<float> operator+(cx<float> a, cx<float> b) {
    return c2(__fadd2_rn(f2(a), f2(b)));
}
template <> __device__ __forceinline__ cx<float> operator-(cx<float> a, cx<float> b) {
    return c2(__ffma2_rn(f2(b), make_float2(-1.0f, -1.0f), f2(a)));
}
template <> __device__ __forceinline__ cx<float> scale(float s, cx<float> a) {
    return c2(__fmul2_rn(make_float2(s, s), f2(a)));
}
template <typename R> __device__ __forceinline__ cx<R> conj(cx<R> a) { return mk(a.x, -a.y); }

// Device status word bits (read by the host after a batch of steps).
enum : uint32_t {
    STATUS_CFL = 1u,       // dt * max(|u|+|v|) N / 2pi > 0.5 on some member
    STATUS_NONFINITE = 2u, // a nonfinite coefficient after a step
    STATUS_TIMEOUT = 4u,   // a bounded device wait gave up
};

__host__ __device__ __forceinline__ int retained_k(int n) { return (n - 1) / 3; }

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        const uint64_t p0 = static_cast<uint64_t>(0xD2511F53u) * c[0];
        const uint64_t p1 = static_cast<uint64_t>(0xCD9E8D57u) * c[2];
        const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
        const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
        const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}
__host__ __device__ __forceinline__ uint32_t mode_code(int kx, int ky) {
    return (static_cast<uint32_t>(kx) & 0xFFFFu) | ((static_cast<uint32_t>(ky) & 0xFFFFu) << 16);
}
// Two standard normals for (seed, member, step, mode): key (seed lo, member), counter
// (mode code, step lo, step hi, seed hi); 53-bit uniforms in (0,1) then Box-Muller.
__device__ __forceinline__ void philox_normal_pair(uint64_t seed, uint32_t member, uint64_t step,
                                                   uint32_t code, double &xi1, double &xi2) {
    uint32_t c[4] = {code, static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32),
                     static_cast<uint32_t>(seed >> 32)};
    philox4x32_10(c, static_cast<uint32_t>(seed), member);
    const uint64_t a = (static_cast<uint64_t>(c[1]) << 32) | c[0];
    const uint64_t b = (static_cast<uint64_t>(c[3]) << 32) | c[2];
    const double u1 = (static_cast<double>(a >> 11) + 0.5) * 0x1.0p-53;
    const double u2 = (static_cast<double>(b >> 11) + 0.5) * 0x1.0p-53;
    const double r = sqrt(-2.0 * log(u1));
    double s, co;
    sincos(2.0 * 3.141592653589793238462643383279502884 * u2, &s, &co);
    xi1 = r * co;
    xi2 = r * s;
}

} // namespace hzlb
