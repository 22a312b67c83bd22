// hzl::CudaSolver on the B200 engine: a drop-in replacement for the reference's
// src/cuda_solver.cu behind its unchanged header include/hzl/cuda_solver.hpp.  Build it in
// place of src/cuda_solver.cu and link libhzlb.so; every other reference file stays as it is.
//
// Semantics kept from the reference (src/cuda_solver.cu):
//  * constructor: validates the grid (Fourier2D), the parameters and the initial field size,
//    rejects nonfinite coefficients, keeps only the 2/3-rule modes (:126-171);
//  * step(dt): sigma must be 0 (:173-183); step(dt, forcing): forcing of size n*n, finite and
//    conjugate-symmetric to 1e-12 (:184-202); RK4 with the forcing held over the step;
//  * std::invalid_argument for bad input and for a time step beyond the diffusion bound
//    (:205-208); std::runtime_error for CUDA failures;
//  * a step whose stage-1 velocities violate the CFL limit throws "GPU CFL limit exceeded"
//    and leaves the state as it was (:106-117); a nonfinite state makes that rate nonfinite,
//    so every step after a nonfinite result throws the same way;
//  * nonfinite coefficients throw "nonfinite GPU result" on download (:222-235).
// The flow state stays on the device between calls; one member per instance.
#include "hzl/cuda_solver.hpp"
#include "hzlb.h"

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

namespace hzl {
namespace {
void throw_on(int rc) {
    if (rc == HZLB_OK)
        return;
    const std::string message = hzlb_last_error();
    if (rc == HZLB_EINVAL)
        throw std::invalid_argument(message);
    throw std::runtime_error(message);
}
} // namespace

struct CudaSolver::Implementation {
    hzlb_ensemble *handle = nullptr;
    std::size_t n = 0;
    Parameters p;
    bool external_forcing = false;
    bool nonfinite = false;   // the last step left a nonfinite coefficient
    ~Implementation() {
        if (handle)
            hzlb_ensemble_destroy(handle);
    }
};

CudaSolver::CudaSolver(std::size_t n, Parameters p, const Field &initial)
    : implementation_(std::make_unique<Implementation>()) {
    Fourier2D validate_grid(n);
    p.validate(n);
    if (initial.size() != n * n)
        throw std::invalid_argument("CUDA initial coefficient size mismatch");
    for (const auto &z : initial)
        if (!std::isfinite(z.real()) || !std::isfinite(z.imag()))
            throw std::invalid_argument("nonfinite initial GPU state");
    auto &s = *implementation_;
    s.n = n;
    s.p = p;
    hzlb_config c{};
    c.n = static_cast<int>(n);
    c.members = 1;
    c.precision = 8;
    c.nu = p.viscosity;
    c.alpha = p.friction;
    c.forcing_kmax = static_cast<int>((n - 1) / 3);   // any retained forcing mode
    c.forcing_per_member = 0;
    c.device = 0;
    throw_on(hzlb_ensemble_create(&c, &s.handle));
    throw_on(hzlb_set_state(s.handle, reinterpret_cast<const double *>(initial.data()), 0, 1));
}

CudaSolver::~CudaSolver() = default;

void CudaSolver::step(double dt) {
    auto &s = *implementation_;
    if (s.p.forcing_sigma != 0)
        throw std::invalid_argument("stochastic GPU step requires midpoint forcing coefficients");
    if (s.external_forcing) {
        const Field zero(s.n * s.n);
        throw_on(hzlb_set_forcing(s.handle, reinterpret_cast<const double *>(zero.data()), 0, 1));
        s.external_forcing = false;
    }
    advance(dt);
}

void CudaSolver::step(double dt, const Field &forcing) {
    auto &s = *implementation_;
    if (forcing.size() != s.n * s.n)
        throw std::invalid_argument("GPU forcing size mismatch");
    throw_on(hzlb_set_forcing(s.handle, reinterpret_cast<const double *>(forcing.data()), 0, 1));
    s.external_forcing = true;
    advance(dt);
}

void CudaSolver::advance(double dt) {
    auto &s = *implementation_;
    if (s.nonfinite)   // the reference's stage-1 rate of a nonfinite state is not finite
        throw std::runtime_error("GPU CFL limit exceeded");
    throw_on(hzlb_step_checked(s.handle, dt));
    uint32_t status = 0;
    throw_on(hzlb_status(s.handle, &status));
    if (status & HZLB_STATUS_NONFINITE)
        s.nonfinite = true;
}

void CudaSolver::synchronize() { throw_on(hzlb_synchronize(implementation_->handle)); }

Field CudaSolver::coefficients() const {
    const auto &s = *implementation_;
    Field result(s.n * s.n);
    throw_on(hzlb_get_state(s.handle, reinterpret_cast<double *>(result.data()), 0, 1));
    for (const auto &z : result)
        if (!std::isfinite(z.real()) || !std::isfinite(z.imag()))
            throw std::runtime_error("nonfinite GPU result");
    return result;
}

} // namespace hzl
