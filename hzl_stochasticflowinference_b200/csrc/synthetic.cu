// Seeded synthetic inputs of the benchmark workloads, generated on the host in FP64 so that the
// FP32 and FP64 device paths (and any CPU checker) start from identical fields:
//   * a Gaussian random vorticity field with shell energy spectrum E(k) ~ k^4 exp(-(k/6)^2),
//     normalised to unit enstrophy Z = A/2 sum |w_k|^2 (the reference's enstrophy,
//     src/solver.cpp:388);
//   * Kolmogorov forcing amplitude * sin(k y) as Fourier coefficients.
#include "engine.h"

#include <cmath>
#include <cstring>

namespace {
constexpr double kPi = 3.141592653589793238462643383279502884;
int wave(int i, int n) { return i < n / 2 ? i : i - n; }
bool valid_grid(int n) { return n >= 8 && n <= 4096 && (n & (n - 1)) == 0; }

// Two standard normals for (seed, member, step, mode) from Philox4x32-10; the same
// convention as the device noise (common.cuh philox_normal_pair).
void normal_pair(uint64_t seed, uint32_t member, uint64_t step, uint32_t code, double &a,
                 double &b) {
    uint32_t c[4] = {code, static_cast<uint32_t>(step), static_cast<uint32_t>(step >> 32),
                     static_cast<uint32_t>(seed >> 32)};
    hzlb::philox4x32_10(c, static_cast<uint32_t>(seed), member);
    const uint64_t x = (static_cast<uint64_t>(c[1]) << 32) | c[0];
    const uint64_t y = (static_cast<uint64_t>(c[3]) << 32) | c[2];
    const double u1 = (static_cast<double>(x >> 11) + 0.5) * 0x1.0p-53;
    const double u2 = (static_cast<double>(y >> 11) + 0.5) * 0x1.0p-53;
    const double r = std::sqrt(-2.0 * std::log(u1)), angle = 2.0 * kPi * u2;
    a = r * std::cos(angle);
    b = r * std::sin(angle);
}
} // namespace

extern "C" {
// Per representative retained mode (kx > 0, or kx = 0 and ky > 0): w = sqrt(v(k)/2)(xi1 + i xi2)
// with v(k) = k^5 exp(-k^2/36) (mode variance giving E(k) ~ k^4 exp(-(k/6)^2) under
// E = A/2 sum |w|^2/k^2), the conjugate partner mirrored, then scaled to unit enstrophy.
// Normals from Philox key (seed, member) at the reserved step 2^64-1.
HZLB_API int hzlb_grf_spectrum(int n, uint64_t seed, uint32_t member, double *out) {
    if (!valid_grid(n) || !out)
        return HZLB_EINVAL;
    const size_t nn = static_cast<size_t>(n) * n;
    std::memset(out, 0, sizeof(double) * 2 * nn);
    for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
            const int kx = wave(x, n), ky = wave(y, n);
            if (!(3 * std::abs(kx) < n && 3 * std::abs(ky) < n) || (kx == 0 && ky == 0))
                continue;
            if (!(kx > 0 || (kx == 0 && ky > 0)))
                continue;
            const double k2 = static_cast<double>(kx * kx + ky * ky), k = std::sqrt(k2);
            const double variance = k2 * k2 * k * std::exp(-k2 / 36.0);
            double a, b;
            normal_pair(seed, member, UINT64_MAX, hzlb::mode_code(kx, ky), a, b);
            const double amp = std::sqrt(variance / 2.0);
            const size_t i = static_cast<size_t>(y) * n + x;
            const size_t j = static_cast<size_t>((n - y) % n) * n + (n - x) % n;
            out[2 * i] = amp * a;
            out[2 * i + 1] = amp * b;
            out[2 * j] = amp * a;
            out[2 * j + 1] = -(amp * b);
        }
    const double area = 4 * kPi * kPi;
    double z = 0;
    for (size_t i = 0; i < nn; ++i)
        z += area / 2 * (out[2 * i] * out[2 * i] + out[2 * i + 1] * out[2 * i + 1]);
    if (!(z > 0))
        return HZLB_EINVAL;
    const double scale = 1.0 / std::sqrt(z);
    for (size_t i = 0; i < 2 * nn; ++i)
        out[i] *= scale;
    return HZLB_OK;
}

// amplitude * sin(k y): coefficient -i amplitude/2 at (0, k), +i amplitude/2 at (0, -k).
HZLB_API int hzlb_kolmogorov_forcing(int n, double amplitude, int wavenumber, double *out) {
    if (!valid_grid(n) || !out || wavenumber <= 0 || 3 * wavenumber >= n)
        return HZLB_EINVAL;
    const size_t nn = static_cast<size_t>(n) * n;
    std::memset(out, 0, sizeof(double) * 2 * nn);
    out[2 * (static_cast<size_t>(wavenumber) * n) + 1] = -amplitude / 2;
    out[2 * (static_cast<size_t>(n - wavenumber) * n) + 1] = amplitude / 2;
    return HZLB_OK;
}
} // extern "C"
