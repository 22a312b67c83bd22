// C++ host runtime of one ensemble handle: device buffers, the RK4 stage schedule (replayed
// from captured CUDA graphs), state/forcing I/O in the reference layout, diagnostics, the
// observation operator and the filter analysis steps.
#pragma once
#include "../../include/hzlb.h"
#include "launch.h"

#include <cuda_runtime.h>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace hzlb {

// Exceptions carry the C-ABI code they map to.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] inline void raise(int code, const std::string &message) { throw Error(code, message); }
inline void cuda_check(cudaError_t e, const char *operation) {
    if (e != cudaSuccess)
        raise(HZLB_ECUDA, std::string(operation) + ": " + cudaGetErrorString(e));
}

// Device allocation owned by RAII.
struct DeviceBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    DeviceBuffer() = default;
    DeviceBuffer(const DeviceBuffer &) = delete;
    DeviceBuffer &operator=(const DeviceBuffer &) = delete;
    ~DeviceBuffer() { release(); }
    void release() {
        if (ptr)
            cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    void ensure(size_t b, const char *what) {
        if (b <= bytes)
            return;
        release();
        cuda_check(cudaMalloc(&ptr, b), what);
        bytes = b;
    }
    template <typename T> T *as() const { return static_cast<T *>(ptr); }
};
struct PinnedBuffer {
    void *ptr = nullptr;
    size_t bytes = 0;
    ~PinnedBuffer() {
        if (ptr)
            cudaFreeHost(ptr);
    }
    void ensure(size_t b) {
        if (b <= bytes)
            return;
        if (ptr)
            cudaFreeHost(ptr);
        ptr = nullptr;
        cuda_check(cudaMallocHost(&ptr, b), "allocate pinned staging buffer");
        bytes = b;
    }
    template <typename T> T *as() const { return static_cast<T *>(ptr); }
};

// One perturbed-observation EnKF analysis of p point observations.
struct EnkfRequest {
    const uint32_t *x, *y;          // grid indices of the observations
    const double *values, *sd;      // observed values and their standard deviations
    size_t p;
    const double *perturbations;    // host members x p standard normals, or null: device Philox
    uint64_t perturbation_seed;     // Philox key when perturbations is null
    uint64_t cycle;                 // Philox counter when perturbations is null
    double nis_limit;               // > 0: leave the state unchanged when the statistic exceeds it
};
struct EnkfResult {
    double nis;                     // dbar^T S^{-1} dbar / p of the forecast ensemble
    int applied;                    // 1 if the state was updated
};

class Engine {
  public:
    virtual ~Engine() = default;
    // calls that reach this ensemble through the C ABI (or a mixed batch); a host-pipelined
    // step chains to the previous one only when nothing else came in between
    uint64_t api_calls = 0;
    virtual void set_state(const double *spectra, int first, int count) = 0;
    virtual void get_state(double *spectra, int first, int count) = 0;
    virtual void set_state_compact(const void *data, int first, int count) = 0;
    virtual void get_state_compact(void *data, int first, int count) = 0;
    virtual void set_forcing(const double *spectra, int first, int count) = 0;
    virtual void step(double dt, uint64_t nsteps) = 0;
    // one step, undone (state, forcing, clock, counter) when its stage-1 CFL check fails
    virtual void step_checked(double dt) = 0;
    // how the step graphs run the members (hzlb_set_step_schedule)
    virtual void set_step_schedule(int schedule) = 0;
    virtual int step_schedule() const = 0;
    // nsteps steps of a host-resident state (compact layout): copied in, stepped and copied
    // out in member chunks that overlap copies with stepping
    virtual void step_host(const void *in, void *out, double dt, uint64_t nsteps, int chunk) = 0;
    virtual uint32_t status() = 0;
    // test hook: the next row pass leaves one block's first tile copy unissued (its bounded
    // wait runs out and the step reports STATUS_TIMEOUT)
    virtual void inject_wait_timeout() = 0;
    virtual void synchronize() = 0;
    virtual void diagnostics(double *out) = 0;
    virtual void physical(double *out) = 0;
    virtual void observe(const uint32_t *x, const uint32_t *y, size_t p, double *out) = 0;
    virtual void resample(const double *w, size_t count, double u, uint32_t *anc) = 0;
    // particle filter on the device (filter.cpp:65-120); see hzlb_pf_* in hzlb.h
    virtual void pf_reset(int particles) = 0;
    virtual void pf_get_weights(double *out) = 0;
    virtual void pf_loglik(const uint32_t *x, const uint32_t *y, const double *values,
                           const double *sd, size_t p, double *log_weights) = 0;
    virtual void pf_weights(const double *logs, size_t count, double *w, double *inc, double *ess,
                            double *mw) = 0;
    virtual void pf_assimilate(const uint32_t *x, const uint32_t *y, const double *values,
                               const double *sd, size_t p, const double *u, const uint8_t *active,
                               hzlb_pf_record *records, uint32_t *ancestors,
                               double *weighted_mean) = 0;
    virtual void gather(const uint32_t *ancestors) = 0;
    virtual void inflate(double inflation) = 0;
    virtual EnkfResult enkf(const EnkfRequest &request) = 0;
    // ensemble-space weights W (M x M, device out) of the perturbed-observation analysis of
    // `members` members with predicted observations hx and perturbations eps (device,
    // members x p); returns the innovation statistic
    virtual double enkf_weights(const double *hx, const double *values, const double *sd,
                                const double *eps, int members, size_t p, double *W) = 0;
    // device address of the compact state (members x compact_size complex entries); the
    // caller may modify it until its next call on this ensemble
    virtual void *state_device() = 0;
    virtual const hzlb_config &config() const = 0;
    // OU shell forcing on the device (ou.cuh): per-member forcing, transitions inside the step
    virtual void enable_ou(double sigma, double tau, int kmin, int kmax, bool initialize) = 0;
    virtual void get_forcing_compact(double *out, int first, int count) = 0;
    // drift of every member's state, -N - (nu k^2 + alpha) w + f (the RK stage-1 derivative),
    // into `out` (device or host, members x compact_size entries of the handle's precision);
    // the state is unchanged
    virtual void drift(void *out) = 0;
    // ---- stepping inside a caller's graph (mixed-resolution batches, mixed.cu) ------------
    // validate dt and run the start pass if the velocity columns are stale (waits for it)
    virtual void prepare_steps(double dt) = 0;
    // enqueue `steps` RK4 steps on stream s, persistent grids capped at col_cap / row_cap
    // blocks (0: every resident block), row kernel blocks of row_threads threads (64 or 128;
    // 0: the resolution's default); allowed during stream capture
    virtual void enqueue_steps_on(double dt, int steps, cudaStream_t s, int col_cap, int row_cap,
                                  int row_threads) = 0;
    // the stage kernels' arguments of this handle (ColumnArgs<R> / RowArgs<R> of its
    // precision, stage and CFL scale unset) for a caller that launches the passes itself (the
    // mixed-resolution kernels); OU forcing transitions are not part of them
    virtual void stage_args(double dt, void *column_args, void *row_args) const = 0;
    virtual bool ou_enabled() const = 0;
    // account for nsteps steps enqueued that way (clock, step counter, cached velocities)
    virtual void finish_steps(double dt, uint64_t nsteps) = 0;
    // member mean of the compact state into `out` (device, compact_size entries, own precision)
    virtual void mean_device(void *out) = 0;
    virtual size_t compact_size() const = 0;
    virtual int members() const = 0;
    virtual void *stream() const = 0;
    // building blocks of the reference-order filter drivers (drivers.cu); compact fields cross
    // as interleaved doubles
    virtual void member_sum(const double *w, double divisor, double *out) = 0;
    virtual void covariance(const double *d, double *cov_out) = 0;
    virtual void rank1(const double *cov, const double *innov) = 0;
    virtual void symmetrize() = 0;
    virtual double spread(const double *mean) = 0;
    virtual void set_forcing_compact(const double *compact, int first, int count) = 0;
    virtual int forcing_columns() const = 0;
    virtual void step_profiled(double dt, uint64_t nsteps, double *row_ms, double *col_ms) = 0;

    double time = 0;
    uint64_t step_index = 0;
    virtual void set_time(double t, uint64_t s) = 0;
};

std::unique_ptr<Engine> make_engine(const hzlb_config &c);
} // namespace hzlb

// The opaque handle of include/hzlb.h.
struct hzlb_ensemble {
    std::unique_ptr<hzlb::Engine> engine;
};

namespace hzlb {

// Tensor-core GEMM launcher (gemm.cu); dtype 2 = BF16 operands, 4 = FP32 read as TF32.
namespace tc {
struct GemmArgs;
}
cudaError_t gemm(const tc::GemmArgs &g, int dtype, cudaStream_t s);

// One window of the learned reduced forecast (pod.cu) on an FP32 ensemble.
int learned_forecast(Engine &e, const hzlb_config &cfg, hzlb_pod *pod, hzlb_mlp *mlp, int q,
                     double dt, uint64_t steps, const void *mean_increment, bool centre);

// Message returned by hzlb_last_error() on this thread.
void set_last_error(const std::string &message);

} // namespace hzlb
