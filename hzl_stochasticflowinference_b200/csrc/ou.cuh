// Ornstein-Uhlenbeck shell forcing advanced on the device (the reference's ShellForcing,
// src/solver.cpp:67-119, with Philox draws in place of its host mt19937_64 streams, so the
// forcing needs no per-step upload; parity with the reference is statistical).
//
// Each retained mode with kmin^2 <= |k|^2 <= kmax^2 is one complex OU process f (its
// conjugate partner follows): over an interval h, f <- e^{-h/tau} f + s (xi1 + i xi2) with
// s = sigma sqrt(-tau expm1(-2h/tau) / 4) (transition_ou, src/solver.cpp:93-105); the stationary
// start has f = sigma sqrt(tau / 4) (xi1 + i xi2) (initialize_ou, :84-92).  A step of dt is the
// reference's midpoint_step: a transition of dt/2 before the RK4 stages (which see that
// midpoint value) and one of dt/2 after.
//
// Draws: key (seed lo, member), counter (mode code, u lo, u hi ^ tag, seed hi) with
// u = 2 step + half (half 0 before the stages, 1 after) from the device step counter, and the
// stationary start at u = 2^64 - 1; the tag keeps these apart from the additive noise's draws.
#pragma once
#include "common.cuh"
#include "spectral_step.cuh"

namespace hzlb {

constexpr uint64_t kOuTag = 0x4F55ull << 48;

// representative (kx, ky) modes of the shell in the compact layout: kx > 0 every ky; kx = 0
// only ky > 0 (its partner (0, -ky) is stored too and set to the conjugate)
template <typename R>
__global__ void ou_transition(cx<R> *forcing, int fcols, int ld, int K, int kmin2, int kmax, double decay,
                              double scale, uint64_t seed, uint32_t member_base,
                              const StepControl *ctl, int half, int stationary) {
    const int m = blockIdx.x;
    const int side = 2 * kmax + 1;
    uint64_t u;
    if (stationary)
        u = ~0ull;
    else {
        const uint64_t step = ctl->step;   // after the step's last stage it counts one more
        u = half ? 2 * (step - 1) + 1 : 2 * step;
    }
    for (int t = threadIdx.x; t < (kmax + 1) * side; t += blockDim.x) {
        const int kx = t / side, ky = t % side - kmax;
        const int k2 = kx * kx + ky * ky;
        if (k2 < kmin2 || k2 > kmax * kmax || kx >= fcols || ky > K || -ky > K)
            continue;
        if (kx == 0 && ky <= 0)
            continue;
        double xi1, xi2;
        philox_normal_pair(seed, member_base + m, u ^ kOuTag, mode_code(kx, ky), xi1, xi2);
        const int j = ky >= 0 ? ky : ky + ld;
        cx<R> &f = forcing[(static_cast<long long>(m) * fcols + kx) * ld + j];
        const double re = decay * static_cast<double>(f.x) + scale * xi1;
        const double im = decay * static_cast<double>(f.y) + scale * xi2;
        f = mk<R>(static_cast<R>(re), static_cast<R>(im));
        if (kx == 0)
            forcing[static_cast<long long>(m) * fcols * ld + (ld - ky)] =
                mk<R>(static_cast<R>(re), static_cast<R>(-im));
    }
}

} // namespace hzlb
