// hzlb_step_noalloc: the ensemble RK4 step for callers that cannot allocate device memory.
//
// Some callers are not allowed to allocate GPU memory once they are running: an application
// whose device memory is owned and budgeted by its own pool, or an assimilation loop on a hot
// path where an allocation (and its possible failure) is not acceptable.  hzlb_ensemble_create
// allocates the stage buffers with cudaMalloc, so those callers use this entry point instead.
// It runs the same row and column kernels as hzlb_step, but every scratch buffer they need
// (the stage input, the RK accumulator, the velocity rows, the product columns, the step
// control word, the twiddle tables and a padded working copy of the state) is carved out of
// one file-scope device array of HZLB_NOALLOC_SCRATCH_BYTES.  The caller passes the state
// (in/out) and the forcing; nothing here calls cudaMalloc, cudaFree or any allocating routine.
//
// The array belongs to this library: every GPU that loads the library's device code holds
// it until the process exits.  All calls share it and it keeps what the previous call left;
// this file clears what must start at zero (the step control word) on every call.  Calls
// whose work overlaps on the GPU (different streams, or different host threads on the same
// device) race on the array, so serialise them.
//
// The first call on each device, and the first for each (precision, grid) on it, does a
// one-time set-up with that device current: it resolves the array's device address with
// cudaGetSymbolAddress (in host code the array's name is only a host-side stand-in, not a
// device address), configures the kernels, and writes the twiddle table of that grid -- the
// host FP64 table hzlb_ensemble_create builds, so both entry points give identical results --
// into a region of the array reserved for it.  Make those first calls before any stream
// capture on the device.
//
// Array layout: [twiddle tables of every grid 8..512, FP32 then FP64 | step control word |
// state copy | stage input | RK accumulator | velocity rows | product columns], each piece
// rounded up to 256 bytes (layout() below).
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

namespace hzlb {
namespace {

__device__ __align__(256) static unsigned char g_scratch[HZLB_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
struct DeviceSetup {
    unsigned char *scratch = nullptr;   // device address of g_scratch
    uint32_t prepared = 0;              // bit (precision index * 8 + log2 n)
};
std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

__global__ void noalloc_init(StepControl *ctl, unsigned long long first_step) {
    ctl->step = first_step;
    ctl->arrivals = 0;
    ctl->status = 0;
    ctl->inject = 0;
}

size_t align256(size_t b) { return (b + 255) / 256 * 256; }

// Twiddle tables of every grid 8, 16, .., 512, one after another: FP32 ones (8 bytes an entry)
// from offset 0, FP64 ones (16 bytes) from kTwDouble.
constexpr size_t kTwEntries = 8 + 16 + 32 + 64 + 128 + 256 + 512;
constexpr size_t kTwDouble = (kTwEntries * 8 + 255) / 256 * 256;
constexpr size_t kTwRegion = kTwDouble + (kTwEntries * 16 + 255) / 256 * 256;
template <typename R> size_t twiddle_offset(int n) {
    return (sizeof(R) == 4 ? 0 : kTwDouble) + sizeof(cx<R>) * static_cast<size_t>(n - 8);
}

struct Layout {
    size_t ctl, omega, ystage, acc, w, nl, total;
};
template <typename R> Layout layout(int n, int members) {
    const size_t K = (n - 1) / 3, C = K + 1, LD = 2 * K + 1, cb = sizeof(cx<R>);
    const size_t state = align256(cb * C * LD * members + 16);   // +16: bulk-copy slack
    Layout l{};
    l.ctl = kTwRegion;
    l.omega = l.ctl + align256(sizeof(StepControl));
    l.ystage = l.omega + state;
    l.acc = l.ystage + state;
    l.w = l.acc + state;
    l.nl = l.w + align256(cb * 2 * n * velocity_row_stride<R>(n) * members);
    l.total = l.nl + align256(cb * 2 * n * C * members);
    return l;
}

// One-time set-up of `device` (current while this runs): the scratch array's device address,
// and for (precision, n) the kernel configuration and the twiddle table.
template <typename R> unsigned char *setup_device(int device, int n) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup &d = g_setup[device];
    if (!d.scratch) {
        void *p = nullptr;
        cuda_check(cudaGetSymbolAddress(&p, g_scratch), "resolve no-alloc scratch address");
        d.scratch = static_cast<unsigned char *>(p);
    }
    int lg = 0;
    while ((1 << lg) < n)
        ++lg;
    const uint32_t bit = 1u << ((sizeof(R) == 4 ? 0 : 8) + lg);
    if (!(d.prepared & bit)) {
        cuda_check(prepare_kernels<R>(n), "configure kernels");
        const std::vector<cx<R>> tw = host_twiddles<R>(n);
        cuda_check(cudaMemcpy(d.scratch + twiddle_offset<R>(n), tw.data(), sizeof(cx<R>) * n,
                              cudaMemcpyHostToDevice),
                   "write no-alloc twiddle table");
        d.prepared |= bit;
    }
    return d.scratch;
}

template <typename R>
void step_noalloc(const hzlb_config &c, double dt, uint64_t nsteps, uint64_t first_step,
                  void *state, const void *forcing, cudaStream_t stream, uint32_t *status) {
    const int n = c.n, M = c.members;
    const Layout l = layout<R>(n, M);
    if (l.total > HZLB_NOALLOC_SCRATCH_BYTES)
        raise(HZLB_EINVAL, std::to_string(M) + " members at " + std::to_string(n) + "^2 need " +
                               std::to_string(l.total) + " bytes of scratch; the no-alloc limit is " +
                               std::to_string(static_cast<size_t>(HZLB_NOALLOC_SCRATCH_BYTES)) +
                               " bytes");
    unsigned char *base = setup_device<R>(c.device, n);
    const int K = (n - 1) / 3, C = K + 1, LD = 2 * K + 1;
    const size_t state_bytes = sizeof(cx<R>) * static_cast<size_t>(C) * LD * M;
    StepControl *ctl = reinterpret_cast<StepControl *>(base + l.ctl);
    const cx<R> *tw = reinterpret_cast<const cx<R> *>(base + twiddle_offset<R>(n));
    cx<R> *omega = reinterpret_cast<cx<R> *>(base + l.omega);

    noalloc_init<<<1, 1, 0, stream>>>(ctl, first_step);
    cuda_check(cudaGetLastError(), "launch no-alloc set-up");
    cuda_check(cudaMemcpyAsync(omega, state, state_bytes, cudaMemcpyDeviceToDevice, stream),
               "copy state into scratch");

    ColumnArgs<R> a{};
    a.nl = reinterpret_cast<cx<R> *>(base + l.nl);
    a.w = reinterpret_cast<cx<R> *>(base + l.w);
    a.omega = omega;
    a.ystage = reinterpret_cast<cx<R> *>(base + l.ystage);
    a.acc = reinterpret_cast<cx<R> *>(base + l.acc);
    const int fcols = c.forcing_kmax < 0 ? 0 : std::min(c.forcing_kmax + 1, C);
    a.forcing = forcing ? static_cast<const cx<R> *>(forcing) : nullptr;
    a.forcing_cols = forcing ? fcols : 0;
    a.forcing_stride = c.forcing_per_member ? static_cast<long long>(fcols) * LD : 0;
    a.tw = tw;
    a.nu = c.nu;
    a.alpha = c.alpha;
    a.dt = dt;
    a.noise_scale = c.noise_sigma > 0 ? c.noise_sigma * std::sqrt(dt) / std::sqrt(2.0) : 0.0;
    a.noise_kmax2 = c.noise_kmax * c.noise_kmax;
    a.seed = c.seed;
    a.member_base = c.member_base;
    a.ctl = ctl;
    a.members = M;
    RowArgs<R> r{};
    r.w = a.w;
    r.nl = reinterpret_cast<cx<R> *>(base + l.nl);
    r.tw = tw;
    r.ctl = ctl;
    r.members = M;

    a.stage = 0;
    a.emit = 1;
    cuda_check(launch_column<R>(n, a, stream), "launch column pass");
    for (uint64_t i = 0; i < nsteps; ++i)
        for (int s = 1; s <= 4; ++s) {
            r.cfl_scale = s == 1 ? dt * n / (2 * 3.141592653589793238462643383279502884) : 0.0;
            cuda_check(launch_row<R>(n, r, stream), "launch row pass");
            a.stage = s;
            a.emit = s < 4 || i + 1 < nsteps;
            cuda_check(launch_column<R>(n, a, stream), "launch column pass");
        }
    cuda_check(cudaMemcpyAsync(state, omega, state_bytes, cudaMemcpyDeviceToDevice, stream),
               "copy state out of scratch");
    if (status) {
        cuda_check(cudaMemcpyAsync(status, &ctl->status, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                   stream),
                   "read status");
        cuda_check(cudaStreamSynchronize(stream), "no-alloc step");
    }
}

} // namespace
} // namespace hzlb

extern "C" HZLB_API int hzlb_step_noalloc(const hzlb_config *config, double dt, uint64_t nsteps,
                                          uint64_t first_step, void *state, const void *forcing,
                                          void *stream, uint32_t *status) {
    using namespace hzlb;
    int previous = -1;
    try {
        if (!config || !state)
            raise(HZLB_EINVAL, "null config or state");
        const hzlb_config &c = *config;
        if (c.n < 8 || c.n > 512 || (c.n & (c.n - 1)))
            raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
        if (c.members < 1)
            raise(HZLB_EINVAL, "ensemble needs at least one member");
        if (c.precision != 4 && c.precision != 8)
            raise(HZLB_EINVAL, "precision must be 4 (FP32) or 8 (FP64)");
        if (!std::isfinite(c.nu) || c.nu < 0 || !std::isfinite(c.alpha) || c.alpha < 0 ||
            !std::isfinite(c.noise_sigma) || c.noise_sigma < 0)
            raise(HZLB_EINVAL, "nu, alpha and noise sigma must be finite and nonnegative");
        if (c.noise_sigma > 0 && (c.noise_kmax < 1 || 3 * c.noise_kmax >= c.n ||
                                  c.noise_kmax > NOISE_KMAX_CAP))
            raise(HZLB_EINVAL, "noise shell must lie strictly inside the dealiased grid, radius <= 15");
        const int largest = (c.n - 1) / 3;
        if (!std::isfinite(dt) || dt <= 0 || dt * (2 * c.nu * largest * largest + c.alpha) > 2.5)
            raise(HZLB_EINVAL, "invalid GPU time step or diffusion stability limit exceeded");
        int devices = 0;
        cuda_check(cudaGetDeviceCount(&devices), "query CUDA devices");
        if (c.device < 0 || c.device >= std::min(devices, kMaxDevices))
            raise(HZLB_EINVAL, "invalid CUDA device ordinal");
        cuda_check(cudaGetDevice(&previous), "query current device");
        cuda_check(cudaSetDevice(c.device), "select CUDA device");
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (c.precision == 4)
            step_noalloc<float>(c, dt, nsteps, first_step, state, forcing, s, status);
        else
            step_noalloc<double>(c, dt, nsteps, first_step, state, forcing, s, status);
        cudaSetDevice(previous);
        return HZLB_OK;
    } catch (const Error &e) {
        if (previous >= 0)
            cudaSetDevice(previous);
        set_last_error(e.what());
        return e.code;
    } catch (const std::exception &e) {
        if (previous >= 0)
            cudaSetDevice(previous);
        set_last_error(e.what());
        return HZLB_ERUNTIME;
    }
}
