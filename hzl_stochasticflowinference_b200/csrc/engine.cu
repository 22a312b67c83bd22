// Ensemble engine: owns the device state of one handle and schedules the kernels.
#include "engine.h"
#include "dense64.cuh"
#include "filters.cuh"
#include "ou.cuh"
#include "umma_gemm.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace hzlb {
namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

bool valid_grid(int n) { return n >= 8 && n <= 512 && (n & (n - 1)) == 0; }
int wave(int i, int n) { return i < n / 2 ? i : i - n; }

// The step counter and status of an ensemble after chunks of it were stepped with their own
// control words: every chunk ends at the same step; status bits accumulate.
__global__ void merge_chunk_control(StepControl *main, const StepControl *chunks, int count,
                                    unsigned long long step) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        unsigned status = 0;
        for (int i = 0; i < count; ++i)
            status |= chunks[i].status;
        main->status |= status;
        main->step = step;
        main->arrivals = 0;
    }
}

// Before the parts of a split step graph run on their own streams: one control word per part,
// each at the ensemble's step with cleared status and arrivals; a pending test injection goes
// to part 0 (its first row pass consumes it).
__global__ void split_control(StepControl *main, StepControl *parts, int count) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        for (int i = 0; i < count; ++i)
            parts[i] = StepControl{main->step, 0u, 0u, i == 0 ? main->inject : 0u};
        main->inject = 0;
    }
}
// After them: status bits accumulate, the step is the parts' (equal) step, and an injection
// no part consumed stays pending.
__global__ void join_control(StepControl *main, const StepControl *parts, int count) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        unsigned status = 0, inject = 0;
        for (int i = 0; i < count; ++i) {
            status |= parts[i].status;
            inject |= parts[i].inject;
        }
        main->status |= status;
        main->step = parts[0].step;
        main->arrivals = 0;
        main->inject = inject;
    }
}

template <typename R> class EngineT final : public Engine {
  public:
    explicit EngineT(const hzlb_config &c) : cfg_(c) {
        if (!valid_grid(c.n))
            raise(HZLB_EINVAL, "grid must be a power of two between 8 and 512");
        if (c.members < 1)
            raise(HZLB_EINVAL, "ensemble needs at least one member");
        if (!std::isfinite(c.nu) || c.nu < 0 || !std::isfinite(c.alpha) || c.alpha < 0)
            raise(HZLB_EINVAL, "nu and alpha must be finite and nonnegative");
        if (!std::isfinite(c.noise_sigma) || c.noise_sigma < 0)
            raise(HZLB_EINVAL, "noise sigma must be finite and nonnegative");
        n_ = c.n;
        M_ = c.members;
        K_ = (n_ - 1) / 3;
        C_ = K_ + 1;
        LD_ = 2 * K_ + 1;
        compact_ = static_cast<size_t>(C_) * LD_;
        fcols_ = c.forcing_kmax < 0 ? 0 : std::min(c.forcing_kmax + 1, C_);
        fcount_ = fcols_ == 0 ? 0 : (c.forcing_per_member ? M_ : 1);
        if (c.noise_sigma > 0 && (c.noise_kmax < 1 || 3 * c.noise_kmax >= n_ ||
                                  c.noise_kmax > NOISE_KMAX_CAP))
            raise(HZLB_EINVAL, "noise shell must lie strictly inside the dealiased grid, radius <= 15");
        int devices = 0;
        cuda_check(cudaGetDeviceCount(&devices), "query CUDA devices");
        if (c.device < 0 || c.device >= devices)
            raise(HZLB_EINVAL, "invalid CUDA device ordinal");
        cuda_check(cudaSetDevice(c.device), "select CUDA device");
        cuda_check(prepare_kernels<R>(n_), "configure kernels");
        cuda_check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking), "create stream");
        const size_t cb = sizeof(cx<R>);
        // +16 bytes: the column pass copies whole 16-byte chunks and may read one entry past
        // the last member
        omega_.ensure(cb * compact_ * M_ + 16, "allocate GPU state");
        ystage_.ensure(cb * compact_ * M_ + 16, "allocate GPU stage input");
        acc_.ensure(cb * compact_ * M_ + 16, "allocate GPU RK accumulator");
        w_.ensure(cb * 2 * velocity_row_stride<R>(n_) * static_cast<size_t>(n_) * M_,
                  "allocate GPU velocity rows");
        nl_.ensure(cb * 2 * C_ * static_cast<size_t>(n_) * M_, "allocate GPU product rows");
        if (fcount_)
            forcing_.ensure(cb * static_cast<size_t>(fcols_) * LD_ * fcount_, "allocate GPU forcing");
        ctl_.ensure(sizeof(StepControl), "allocate step control");
        tw_.ensure(cb * n_, "allocate twiddles");
        cuda_check(cudaMemsetAsync(omega_.ptr, 0, omega_.bytes, stream_), "clear GPU state");
        if (fcount_)
            cuda_check(cudaMemsetAsync(forcing_.ptr, 0, forcing_.bytes, stream_), "clear forcing");
        cuda_check(cudaMemsetAsync(ctl_.ptr, 0, sizeof(StepControl), stream_), "clear control");
        const std::vector<cx<R>> tw = host_twiddles<R>(n_);
        cuda_check(cudaMemcpyAsync(tw_.ptr, tw.data(), cb * n_, cudaMemcpyHostToDevice, stream_),
                   "upload twiddles");
        cuda_check(cudaStreamSynchronize(stream_), "initialise ensemble");
    }
    ~EngineT() override {
        drop_graphs();
        for (auto &e : fevent_)
            if (e)
                cudaEventDestroy(e);
        for (auto &e : pipe_events_)
            cudaEventDestroy(e);
        for (auto &e : d2h_events_)
            cudaEventDestroy(e);
        for (auto &e : split_events_)
            if (e)
                cudaEventDestroy(e);
        for (cudaStream_t t : {copy_in_, copy_out_, compute2_})
            if (t)
                cudaStreamDestroy(t);
        if (stream_)
            cudaStreamDestroy(stream_);
    }

    size_t compact_size() const override { return compact_; }
    int members() const override { return M_; }
    void *stream() const override { return stream_; }
    int forcing_columns() const override { return fcols_; }

    // ---- reference-order filter building blocks -----------------------------------
    int grid_for(size_t elems) const {
        return static_cast<int>(std::min<size_t>((elems + 255) / 256, 2048));
    }
    void member_sum(const double *w, double divisor, double *out) override {
        aux_.ensure(sizeof(double) * (2 * compact_ + M_), "allocate member sum");
        double *dout = aux_.as<double>(), *dw = dout + 2 * compact_;
        if (divisor <= 0)
            cuda_check(cudaMemcpyAsync(dw, w, sizeof(double) * M_, cudaMemcpyHostToDevice, stream_),
                       "upload weights");
        member_sum_kernel<R><<<grid_for(compact_), 256, 0, stream_>>>(
            omega_.as<cx<R>>(), dw, divisor, static_cast<long long>(compact_), M_, dout);
        cuda_check(cudaGetLastError(), "launch member sum");
        cuda_check(cudaMemcpyAsync(out, dout, sizeof(double) * 2 * compact_, cudaMemcpyDeviceToHost,
                                   stream_),
                   "download member sum");
        cuda_check(cudaStreamSynchronize(stream_), "member sum");
    }
    void covariance(const double *d, double *cov_out) override {
        aux_.ensure(sizeof(double) * (2 * compact_ + M_), "allocate covariance");
        double *dcov = aux_.as<double>(), *dd = dcov + 2 * compact_;
        cuda_check(cudaMemcpyAsync(dd, d, sizeof(double) * M_, cudaMemcpyHostToDevice, stream_),
                   "upload covariance weights");
        member_covariance_kernel<R><<<grid_for(compact_), 256, 0, stream_>>>(
            omega_.as<cx<R>>(), dd, static_cast<long long>(compact_), M_, dcov);
        cuda_check(cudaGetLastError(), "launch covariance");
        if (cov_out) {
            cuda_check(cudaMemcpyAsync(cov_out, dcov, sizeof(double) * 2 * compact_,
                                       cudaMemcpyDeviceToHost, stream_),
                       "download covariance");
            cuda_check(cudaStreamSynchronize(stream_), "covariance");
        }
    }
    void rank1(const double *cov, const double *innov) override {
        aux_.ensure(sizeof(double) * (2 * compact_ + M_), "allocate covariance");
        double *dcov = aux_.as<double>(), *dinn = dcov + 2 * compact_;
        if (cov)
            cuda_check(cudaMemcpyAsync(dcov, cov, sizeof(double) * 2 * compact_,
                                       cudaMemcpyHostToDevice, stream_),
                       "upload covariance");
        cuda_check(cudaMemcpyAsync(dinn, innov, sizeof(double) * M_, cudaMemcpyHostToDevice, stream_),
                   "upload innovations");
        const dim3 grid(std::max(1, std::min(grid_for(compact_), 64)), M_);
        rank1_update<R><<<grid, 256, 0, stream_>>>(omega_.as<cx<R>>(), dcov, dinn,
                                                  static_cast<long long>(compact_), M_);
        cuda_check(cudaGetLastError(), "launch rank-1 update");
        cuda_check(cudaStreamSynchronize(stream_), "rank-1 update");
        w_valid_ = false;
    }
    void symmetrize() override {
        symmetrize_column0<R><<<M_, 64, 0, stream_>>>(omega_.as<cx<R>>(), n_, M_);
        cuda_check(cudaGetLastError(), "launch symmetrisation");
        w_valid_ = false;
    }
    double spread(const double *mean) override {
        aux_.ensure(sizeof(double) * (2 * compact_ + 1), "allocate spread");
        double *dmean = aux_.as<double>(), *dout = dmean + 2 * compact_;
        cuda_check(cudaMemcpyAsync(dmean, mean, sizeof(double) * 2 * compact_, cudaMemcpyHostToDevice,
                                   stream_),
                   "upload mean");
        cuda_check(cudaMemsetAsync(dout, 0, sizeof(double), stream_), "clear spread");
        spread_sum<R><<<grid_for(compact_), 256, 0, stream_>>>(
            omega_.as<cx<R>>(), dmean, static_cast<long long>(compact_), LD_, M_, dout);
        cuda_check(cudaGetLastError(), "launch spread");
        double v = 0;
        cuda_check(cudaMemcpyAsync(&v, dout, sizeof(double), cudaMemcpyDeviceToHost, stream_),
                   "download spread");
        cuda_check(cudaStreamSynchronize(stream_), "spread");
        return v;
    }
    // Double-buffered pinned upload of per-member forcing in the compact layout (columns
    // kx < forcing_columns); the host may prepare the next step's forcing while this one runs.
    void set_forcing_compact(const double *compact, int first, int count) override {
        if (fcount_ == 0)
            raise(HZLB_EINVAL, "ensemble was created without forcing");
        if (first < 0 || count < 0 || first + count > fcount_)
            raise(HZLB_EINVAL, "forcing member range out of bounds");
        const size_t block = static_cast<size_t>(fcols_) * LD_, elems = block * count;
        const int b = fbuf_next_;
        fbuf_next_ ^= 1;
        if (!fevent_[b])
            cuda_check(cudaEventCreateWithFlags(&fevent_[b], cudaEventDisableTiming), "create event");
        else
            cuda_check(cudaEventSynchronize(fevent_[b]), "wait for forcing staging");
        fstage_[b].ensure(sizeof(cx<R>) * elems);
        cx<R> *st = fstage_[b].as<cx<R>>();
        for (size_t i = 0; i < elems; ++i)
            st[i] = mk<R>(static_cast<R>(compact[2 * i]), static_cast<R>(compact[2 * i + 1]));
        cuda_check(cudaMemcpyAsync(forcing_.as<cx<R>>() + static_cast<size_t>(first) * block, st,
                                   sizeof(cx<R>) * elems, cudaMemcpyHostToDevice, stream_),
                   "midpoint forcing upload");
        cuda_check(cudaEventRecord(fevent_[b], stream_), "record forcing upload");
    }

    // ---- state I/O ----------------------------------------------------------------
    void check_range(int first, int count) const {
        if (first < 0 || count < 0 || first + count > M_)
            raise(HZLB_EINVAL, "member range out of bounds");
    }
    void set_state(const double *s, int first, int count) override {
        check_range(first, count);
        const size_t nn = static_cast<size_t>(n_) * n_;
        for (size_t i = 0; i < 2 * nn * count; ++i)
            if (!std::isfinite(s[i]))
                raise(HZLB_EINVAL, "nonfinite initial GPU state");
        staging_.ensure(sizeof(cx<R>) * compact_ * count);
        cx<R> *out = staging_.as<cx<R>>();
        for (int m = 0; m < count; ++m)
            for (int kx = 0; kx < C_; ++kx)
                for (int j = 0; j < LD_; ++j) {
                    const int ypos = j <= K_ ? j : n_ - LD_ + j;
                    const double *z = s + 2 * (m * nn + static_cast<size_t>(ypos) * n_ + kx);
                    const bool zero_mode = kx == 0 && j == 0;
                    out[(static_cast<size_t>(m) * C_ + kx) * LD_ + j] =
                        zero_mode ? mk<R>(0, 0) : mk<R>(static_cast<R>(z[0]), static_cast<R>(z[1]));
                }
        cuda_check(cudaMemcpyAsync(omega_.as<cx<R>>() + static_cast<size_t>(first) * compact_, out,
                                   sizeof(cx<R>) * compact_ * count, cudaMemcpyHostToDevice, stream_),
                   "initial state upload");
        cuda_check(cudaStreamSynchronize(stream_), "initial state upload");
        w_valid_ = false;
    }
    void get_state(double *s, int first, int count) override {
        check_range(first, count);
        staging_.ensure(sizeof(cx<R>) * compact_ * count);
        cx<R> *in = staging_.as<cx<R>>();
        cuda_check(cudaMemcpyAsync(in, omega_.as<cx<R>>() + static_cast<size_t>(first) * compact_,
                                   sizeof(cx<R>) * compact_ * count, cudaMemcpyDeviceToHost, stream_),
                   "final state download");
        cuda_check(cudaStreamSynchronize(stream_), "final state download");
        const size_t nn = static_cast<size_t>(n_) * n_;
        std::memset(s, 0, sizeof(double) * 2 * nn * count);
        for (int m = 0; m < count; ++m)
            for (int kx = 0; kx < C_; ++kx)
                for (int j = 0; j < LD_; ++j) {
                    const cx<R> z = in[(static_cast<size_t>(m) * C_ + kx) * LD_ + j];
                    const int ypos = j <= K_ ? j : n_ - LD_ + j;
                    double *d = s + 2 * (m * nn + static_cast<size_t>(ypos) * n_ + kx);
                    d[0] = z.x;
                    d[1] = z.y;
                    if (kx > 0) {   // conjugate partner (-kx, -ky)
                        double *e = s + 2 * (m * nn + static_cast<size_t>((n_ - ypos) % n_) * n_ +
                                             (n_ - kx));
                        e[0] = z.x;
                        e[1] = -static_cast<double>(z.y);
                    }
                }
        for (size_t i = 0; i < 2 * nn * count; ++i)
            if (!std::isfinite(s[i]))
                raise(HZLB_ERUNTIME, "nonfinite GPU result");
    }
    void set_state_compact(const void *d, int first, int count) override {
        check_range(first, count);
        cuda_check(cudaMemcpyAsync(omega_.as<cx<R>>() + static_cast<size_t>(first) * compact_, d,
                                   sizeof(cx<R>) * compact_ * count, cudaMemcpyDefault, stream_),
                   "compact state upload");
        w_valid_ = false;
    }
    void get_state_compact(void *d, int first, int count) override {
        check_range(first, count);
        cuda_check(cudaMemcpyAsync(d, omega_.as<cx<R>>() + static_cast<size_t>(first) * compact_,
                                   sizeof(cx<R>) * compact_ * count, cudaMemcpyDefault, stream_),
                   "compact state download");
        cuda_check(cudaStreamSynchronize(stream_), "compact state download");
    }
    void set_forcing(const double *s, int first, int count) override {
        if (fcount_ == 0)
            raise(HZLB_EINVAL, "ensemble was created without forcing");
        if (first < 0 || count < 0 || first + count > fcount_)
            raise(HZLB_EINVAL, "forcing member range out of bounds");
        const size_t nn = static_cast<size_t>(n_) * n_;
        const size_t block = static_cast<size_t>(fcols_) * LD_;
        staging_.ensure(sizeof(cx<R>) * block * count);
        cx<R> *out = staging_.as<cx<R>>();
        for (int m = 0; m < count; ++m) {
            const double *f = s + 2 * m * nn;
            for (int y = 0; y < n_; ++y)
                for (int x = 0; x < n_; ++x) {
                    const size_t i = static_cast<size_t>(y) * n_ + x,
                                 partner = static_cast<size_t>((n_ - y) % n_) * n_ + (n_ - x) % n_;
                    const double re = f[2 * i], im = f[2 * i + 1];
                    if (!std::isfinite(re) || !std::isfinite(im))
                        raise(HZLB_EINVAL, "nonfinite GPU forcing");
                    // conjugate symmetry to 1e-12 (cuda_solver.cu:191-194)
                    const double dr = re - f[2 * partner], di = im + f[2 * partner + 1];
                    if (std::hypot(dr, di) > 1e-12 * (1 + std::hypot(re, im)))
                        raise(HZLB_EINVAL, "GPU forcing must preserve conjugate symmetry");
                    const int kx = wave(x, n_), ky = wave(y, n_);
                    const bool retained = 3 * std::abs(kx) < n_ && 3 * std::abs(ky) < n_;
                    if (retained && std::abs(kx) >= fcols_ && (re != 0 || im != 0))
                        raise(HZLB_EINVAL, "forcing outside the configured columns");
                }
            for (int kx = 0; kx < fcols_; ++kx)
                for (int j = 0; j < LD_; ++j) {
                    const int ypos = j <= K_ ? j : n_ - LD_ + j;
                    const double *z = f + 2 * (static_cast<size_t>(ypos) * n_ + kx);
                    out[static_cast<size_t>(m) * block + static_cast<size_t>(kx) * LD_ + j] =
                        mk<R>(static_cast<R>(z[0]), static_cast<R>(z[1]));
                }
        }
        cuda_check(cudaMemcpyAsync(forcing_.as<cx<R>>() + static_cast<size_t>(first) * block, out,
                                   sizeof(cx<R>) * block * count, cudaMemcpyHostToDevice, stream_),
                   "midpoint forcing upload");
        cuda_check(cudaStreamSynchronize(stream_), "midpoint forcing upload");
    }

    // ---- stepping -----------------------------------------------------------------
    ColumnArgs<R> column_args(double dt) const {
        ColumnArgs<R> a{};
        a.nl = nl_.as<cx<R>>();
        a.w = w_.as<cx<R>>();
        a.omega = omega_.as<cx<R>>();
        a.ystage = ystage_.as<cx<R>>();
        a.acc = acc_.as<cx<R>>();
        a.forcing = fcount_ ? forcing_.as<cx<R>>() : nullptr;
        a.forcing_stride = cfg_.forcing_per_member ? static_cast<long long>(fcols_) * LD_ : 0;
        a.forcing_cols = fcols_;
        a.tw = tw_.as<cx<R>>();
        a.nu = cfg_.nu;
        a.alpha = cfg_.alpha;
        a.dt = dt;
        a.stage = 0;
        a.emit = 1;
        a.noise_scale = cfg_.noise_sigma > 0 ? cfg_.noise_sigma * std::sqrt(dt) / std::sqrt(2.0) : 0.0;
        a.noise_kmax2 = cfg_.noise_kmax * cfg_.noise_kmax;
        a.seed = cfg_.seed;
        a.member_base = cfg_.member_base;
        a.ctl = ctl_.as<StepControl>();
        a.members = M_;
        return a;
    }
    RowArgs<R> row_args() const {
        RowArgs<R> r{};
        r.w = w_.as<cx<R>>();
        r.nl = nl_.as<cx<R>>();
        r.tw = tw_.as<cx<R>>();
        r.cfl_scale = 0;
        r.ctl = ctl_.as<StepControl>();
        r.members = M_;
        return r;
    }
    void launch_start() {
        ColumnArgs<R> a = column_args(1.0);
        a.stage = 0;
        cuda_check(launch_column<R>(n_, a, stream_), "launch start column pass");
    }
    // The eight launches of one RK4 step; the final column pass also emits the derivative
    // columns of the new state, so consecutive steps chain without a separate start pass.
    void enqueue_step(double dt) { enqueue_steps_on(dt, 1, stream_, 0, 0, 0); }
    // the OU half-step transition (ou.cuh) before (half 0) or after (half 1) a step's stages
    void enqueue_ou(double dt, int half, cudaStream_t s) {
        const double h = dt / 2;
        const double decay = std::exp(-h / ou_tau_);
        const double scale = ou_sigma_ * std::sqrt(-ou_tau_ * std::expm1(-2 * h / ou_tau_) / 4);
        ou_transition<R><<<M_, 64, 0, s>>>(forcing_.as<cx<R>>(), fcols_, LD_, K_, ou_kmin_ * ou_kmin_,
                                           ou_kmax_, decay, scale, cfg_.seed, cfg_.member_base,
                                           ctl_.as<StepControl>(), half, 0);
        cuda_check(cudaGetLastError(), "launch OU transition");
    }
    void enable_ou(double sigma, double tau, int kmin, int kmax, bool initialize) override {
        if (!cfg_.forcing_per_member || fcount_ == 0)
            raise(HZLB_EINVAL, "device OU forcing needs per-member forcing storage");
        if (!std::isfinite(sigma) || sigma < 0 || !std::isfinite(tau) || tau <= 0 || kmin < 1 ||
            kmax < kmin || 3 * kmax >= n_)
            raise(HZLB_EINVAL, "invalid OU forcing parameters");
        if (kmax >= fcols_)
            raise(HZLB_EINVAL, "forcing storage must cover the OU shell (forcing_kmax >= kmax)");
        ou_ = true;
        ou_sigma_ = sigma;
        ou_tau_ = tau;
        ou_kmin_ = kmin;
        ou_kmax_ = kmax;
        drop_graphs();
        if (initialize) {
            ou_transition<R><<<M_, 64, 0, stream_>>>(forcing_.as<cx<R>>(), fcols_, LD_, K_, kmin * kmin,
                                                     kmax, 0.0, sigma * std::sqrt(tau / 4), cfg_.seed,
                                                     cfg_.member_base, ctl_.as<StepControl>(), 0, 1);
            cuda_check(cudaGetLastError(), "launch OU initialisation");
            cuda_check(cudaStreamSynchronize(stream_), "OU initialisation");
        }
    }
    void drift(void *out) override {
        if (!w_valid_)
            launch_start();
        w_valid_ = true;   // the stage-1 column pass below does not emit velocities
        RowArgs<R> r = row_args();
        r.cfl_scale = 0.0;
        cuda_check(launch_row<R>(n_, r, stream_), "launch row pass");
        ColumnArgs<R> a = column_args(1.0);
        a.stage = 1;
        a.emit = 0;
        cuda_check(launch_column<R>(n_, a, stream_), "launch column pass");
        cuda_check(cudaMemcpyAsync(out, acc_.ptr, sizeof(cx<R>) * compact_ * M_, cudaMemcpyDefault,
                                   stream_),
                   "copy drift");
        cuda_check(cudaStreamSynchronize(stream_), "drift");
    }
    void get_forcing_compact(double *out, int first, int count) override {
        if (fcount_ == 0)
            raise(HZLB_EINVAL, "this ensemble holds no forcing");
        if (first < 0 || count < 0 || first + count > fcount_)
            raise(HZLB_EINVAL, "forcing range out of bounds");
        const size_t block = static_cast<size_t>(fcols_) * LD_;
        std::vector<cx<R>> tmp(block * count);
        cuda_check(cudaMemcpyAsync(tmp.data(), forcing_.as<cx<R>>() + first * block,
                                   sizeof(cx<R>) * tmp.size(), cudaMemcpyDeviceToHost, stream_),
                   "download forcing");
        cuda_check(cudaStreamSynchronize(stream_), "download forcing");
        for (size_t i = 0; i < tmp.size(); ++i) {
            out[2 * i] = static_cast<double>(tmp[i].x);
            out[2 * i + 1] = static_cast<double>(tmp[i].y);
        }
    }
    void drop_graphs() {
        for (auto &g : graphs_)
            if (g.exec)
                cudaGraphExecDestroy(g.exec);
        graphs_.clear();
    }
    cudaGraphExec_t graph_for(double dt, int steps) {
        for (auto &g : graphs_)
            if (g.dt == dt && g.steps == steps)
                return g.exec;
        cudaGraph_t graph = nullptr;
        if (split_members() > 0)
            prepare_split();
        cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal),
                   "begin step capture");
        try {
            if (split_members() > 0)
                enqueue_split_steps(dt, steps, split_members());
            else
                for (int i = 0; i < steps; ++i)
                    enqueue_step(dt);
        } catch (...) {
            cudaStreamEndCapture(stream_, &graph);
            if (graph)
                cudaGraphDestroy(graph);
            throw;
        }
        cuda_check(cudaStreamEndCapture(stream_, &graph), "end step capture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        cuda_check(e, "instantiate step graph");
        graphs_.push_back({dt, steps, exec});
        return exec;
    }
    // Members of the first part when the step graph runs the ensemble as two parts on two
    // streams (schedule 1: side by side; 2: the second part one row pass behind the first, so
    // one part's row passes, bound by arithmetic, overlap the other's column passes, bound by
    // memory), else 0.  Each part keeps whole 16-byte runs of every per-member array and at
    // least 128 members; device OU forcing keeps the single pass.
    int split_members() const {
        if (schedule_ == 0 || ou_ || M_ < 256)
            return 0;
        const size_t bytes_per = sizeof(cx<R>) * compact_;
        int q = 1;
        while ((static_cast<size_t>(q) * bytes_per) % 16 != 0)
            ++q;
        return (M_ / 2 + q - 1) / q * q;
    }
    // the second stream, events and part control words of a split step graph (before capture)
    void prepare_split() {
        if (!compute2_)
            cuda_check(cudaStreamCreateWithFlags(&compute2_, cudaStreamNonBlocking), "create stream");
        for (auto &e : split_events_)
            if (!e)
                cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "create event");
        split_ctl_.ensure(sizeof(StepControl) * 2, "allocate part control");
    }
    void enqueue_split_steps(double dt, int steps, int first_part) {
        StepControl *parts = split_ctl_.as<StepControl>();
        split_control<<<1, 32, 0, stream_>>>(ctl_.as<StepControl>(), parts, 2);
        cuda_check(cudaGetLastError(), "split step control");
        cuda_check(cudaEventRecord(split_events_[0], stream_), "fork step parts");
        cuda_check(cudaStreamWaitEvent(compute2_, split_events_[0], 0), "fork step parts");
        for (int p = 0; p < 2; ++p) {
            const int f = p == 0 ? 0 : first_part, k = p == 0 ? first_part : M_ - first_part;
            const cudaStream_t s = p == 0 ? stream_ : compute2_;
            const size_t off = static_cast<size_t>(f) * compact_;
            ColumnArgs<R> a = column_args(dt);
            RowArgs<R> r = row_args();
            a.omega += off;
            a.ystage += off;
            a.acc += off;
            a.w += static_cast<size_t>(f) * n_ * 2 * velocity_row_stride<R>(n_);
            a.nl += static_cast<size_t>(f) * 2 * C_ * n_;
            if (a.forcing && a.forcing_stride)
                a.forcing += static_cast<size_t>(f) * a.forcing_stride;
            a.member_base += static_cast<unsigned>(f);
            a.members = k;
            a.ctl = parts + p;
            r.w = a.w;
            r.nl = nl_.as<cx<R>>() + static_cast<size_t>(f) * 2 * C_ * n_;
            r.members = k;
            r.ctl = parts + p;
            if (p == 1 && schedule_ == 2)
                cuda_check(cudaStreamWaitEvent(s, split_events_[1], 0), "offset second part");
            for (int i = 0; i < steps; ++i)
                for (int st = 1; st <= 4; ++st) {
                    r.cfl_scale = st == 1 ? dt * n_ / (2 * kPi) : 0.0;
                    cuda_check(launch_row<R>(n_, r, s), "launch row pass");
                    if (p == 0 && i == 0 && st == 1)
                        cuda_check(cudaEventRecord(split_events_[1], s), "record first row pass");
                    a.stage = st;
                    cuda_check(launch_column<R>(n_, a, s), "launch column pass");
                }
        }
        cuda_check(cudaEventRecord(split_events_[2], compute2_), "join step parts");
        cuda_check(cudaStreamWaitEvent(stream_, split_events_[2], 0), "join step parts");
        join_control<<<1, 32, 0, stream_>>>(ctl_.as<StepControl>(), parts, 2);
        cuda_check(cudaGetLastError(), "join step control");
    }
    void set_step_schedule(int schedule) override {
        if (schedule < 0 || schedule > 2)
            raise(HZLB_EINVAL, "step schedule must be 0, 1 or 2");
        if (schedule != schedule_)
            drop_graphs();
        schedule_ = schedule;
    }
    int step_schedule() const override { return schedule_; }
    void prepare_steps(double dt) override {
        ++api_calls;   // a mixed batch steps this ensemble: no host-pipelined call chains across it
        const int largest = (n_ - 1) / 3;
        if (!std::isfinite(dt) || dt <= 0 ||
            dt * (2 * cfg_.nu * largest * largest + cfg_.alpha) > 2.5)
            raise(HZLB_EINVAL, "invalid GPU time step or diffusion stability limit exceeded");
        if (!w_valid_) {
            launch_start();
            cuda_check(cudaStreamSynchronize(stream_), "start pass");
            w_valid_ = true;
        }
    }
    void enqueue_steps_on(double dt, int steps, cudaStream_t s, int col_cap, int row_cap,
                          int row_threads) override {
        ColumnArgs<R> a = column_args(dt);
        RowArgs<R> r = row_args();
        for (int i = 0; i < steps; ++i) {
            if (ou_)
                enqueue_ou(dt, 0, s);
            for (int st = 1; st <= 4; ++st) {
                r.cfl_scale = st == 1 ? dt * n_ / (2 * kPi) : 0.0;
                cuda_check(launch_row<R>(n_, r, s, row_cap, row_threads), "launch row pass");
                a.stage = st;
                cuda_check(launch_column<R>(n_, a, s, col_cap), "launch column pass");
            }
            if (ou_)
                enqueue_ou(dt, 1, s);
        }
    }
    void stage_args(double dt, void *col_out, void *row_out) const override {
        *static_cast<ColumnArgs<R> *>(col_out) = column_args(dt);
        *static_cast<RowArgs<R> *>(row_out) = row_args();
    }
    bool ou_enabled() const override { return ou_; }
    void finish_steps(double dt, uint64_t nsteps) override {
        w_valid_ = true;
        time += dt * static_cast<double>(nsteps);
        step_index += nsteps;
    }
    void step(double dt, uint64_t nsteps) override {
        const int largest = (n_ - 1) / 3;
        if (!std::isfinite(dt) || dt <= 0 ||
            dt * (2 * cfg_.nu * largest * largest + cfg_.alpha) > 2.5)
            raise(HZLB_EINVAL, "invalid GPU time step or diffusion stability limit exceeded");
        if (nsteps == 0)
            return;
        if (!w_valid_)
            launch_start();
        constexpr int kBatch = 8;
        uint64_t left = nsteps;
        while (left >= kBatch) {
            cuda_check(cudaGraphLaunch(graph_for(dt, kBatch), stream_), "launch step graph");
            left -= kBatch;
        }
        for (; left > 0; --left)
            cuda_check(cudaGraphLaunch(graph_for(dt, 1), stream_), "launch step graph");
        w_valid_ = true;
        time += dt * static_cast<double>(nsteps);
        step_index += nsteps;
    }
    // One step with the reference CudaSolver's failure semantics (cuda_solver.cu:106-117,
    // 203-215): its stage-1 CFL check throws before the state changes.  Here the step runs
    // and, when its stage-1 row pass flagged the CFL limit, the state, forcing, control word,
    // clock and step counter are put back from a device copy taken before it.
    void step_checked(double dt) override {
        const size_t sb = sizeof(cx<R>) * compact_ * M_;
        const size_t fb = fcount_ ? sizeof(cx<R>) * static_cast<size_t>(fcols_) * LD_ * fcount_ : 0;
        backup_.ensure(sb + fb + sizeof(StepControl) + 64, "allocate step backup");
        unsigned char *bk = backup_.as<unsigned char>();
        cuda_check(cudaMemcpyAsync(bk, omega_.ptr, sb, cudaMemcpyDeviceToDevice, stream_), "back up state");
        if (fb)
            cuda_check(cudaMemcpyAsync(bk + sb, forcing_.ptr, fb, cudaMemcpyDeviceToDevice, stream_),
                       "back up forcing");
        cuda_check(cudaMemcpyAsync(bk + sb + fb, ctl_.ptr, sizeof(StepControl),
                                   cudaMemcpyDeviceToDevice, stream_),
                   "back up step control");
        const double t0 = time;
        const uint64_t s0 = step_index;
        step(dt, 1);
        StepControl c{};
        cuda_check(cudaMemcpyAsync(&c, ctl_.ptr, sizeof c, cudaMemcpyDeviceToHost, stream_),
                   "read status");
        cuda_check(cudaStreamSynchronize(stream_), "checked step");
        if (!(c.status & STATUS_CFL))
            return;
        cuda_check(cudaMemcpyAsync(omega_.ptr, bk, sb, cudaMemcpyDeviceToDevice, stream_), "restore state");
        if (fb)
            cuda_check(cudaMemcpyAsync(forcing_.ptr, bk + sb, fb, cudaMemcpyDeviceToDevice, stream_),
                       "restore forcing");
        cuda_check(cudaMemcpyAsync(ctl_.ptr, bk + sb + fb, sizeof(StepControl),
                                   cudaMemcpyDeviceToDevice, stream_),
                   "restore step control");
        cuda_check(cudaStreamSynchronize(stream_), "restore state");
        time = t0;
        step_index = s0;
        w_valid_ = false;
        raise(HZLB_ERUNTIME, "GPU CFL limit exceeded");
    }
    // Steps the ensemble whose state lives on the host: members [f, f+k) of each chunk are
    // copied in, stepped and copied out, the copies of one chunk overlapping the stepping of
    // the others (copy-in stream -> one of two compute streams -> copy-out stream, ordered by
    // events).
    // Each chunk runs with its own step-control word, started at the current step; the
    // ensemble's counter and status are merged afterwards.  Chunk boundaries keep every
    // chunk's state 16-byte aligned for the bulk copies.
    void step_host(const void *in, void *out, double dt, uint64_t nsteps, int chunk) override {
        const int largest = (n_ - 1) / 3;
        if (!std::isfinite(dt) || dt <= 0 ||
            dt * (2 * cfg_.nu * largest * largest + cfg_.alpha) > 2.5)
            raise(HZLB_EINVAL, "invalid GPU time step or diffusion stability limit exceeded");
        if (!in || !out)
            raise(HZLB_EINVAL, "null host state");
        if (ou_)
            raise(HZLB_EINVAL, "host-pipelined stepping does not advance device OU forcing");
        const size_t bytes_per = sizeof(cx<R>) * compact_;
        int q = 1;   // members per 16 bytes of alignment
        while ((static_cast<size_t>(q) * bytes_per) % 16 != 0)
            ++q;
        // default: sixteen chunks (shorter pipeline fill and drain than eight: 362k against
        // 352k member-steps/s at 2048 members, 256^2 FP32), at least 32 members each
        if (chunk <= 0)
            chunk = std::max((M_ + 15) / 16, 32);
        chunk = std::min(M_, (chunk + q - 1) / q * q);
        const int chunks = (M_ + chunk - 1) / chunk;
        for (cudaStream_t *t : {&copy_in_, &copy_out_, &compute2_})
            if (!*t)
                cuda_check(cudaStreamCreateWithFlags(t, cudaStreamNonBlocking), "create stream");
        while (pipe_events_.size() < static_cast<size_t>(2 * chunks + 3)) {
            cudaEvent_t e;
            cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "create event");
            pipe_events_.push_back(e);
        }
        chunk_ctl_.ensure(sizeof(StepControl) * chunks, "allocate chunk control");
        std::vector<StepControl> init(chunks);
        for (auto &c : init)
            c = StepControl{step_index, 0u, 0u, 0u};
        cuda_check(cudaMemcpyAsync(chunk_ctl_.ptr, init.data(), sizeof(StepControl) * chunks,
                                   cudaMemcpyHostToDevice, stream_),
                   "initialise chunk control");
        cudaEvent_t start = pipe_events_[2 * chunks], end = pipe_events_[2 * chunks + 1],
                    side = pipe_events_[2 * chunks + 2];
        // A call that directly follows another with the same chunks (no other call on this
        // handle in between) lets each chunk's upload wait only for the previous call's
        // download of the same chunk, so the uploads overlap the previous call's last
        // downloads; its steps and downloads still follow the whole previous call.
        const bool chained = pipe_mark_ != 0 && api_calls == pipe_mark_ + 1 && chunks == pipe_chunks_;
        while (d2h_events_.size() < static_cast<size_t>(chunks)) {
            cudaEvent_t e;
            cuda_check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "create event");
            d2h_events_.push_back(e);
        }
        cuda_check(cudaEventRecord(start, stream_), "record event");
        if (!chained)
            cuda_check(cudaStreamWaitEvent(copy_in_, start, 0), "order copy stream");
        cuda_check(cudaStreamWaitEvent(compute2_, start, 0), "order compute stream");
        const auto *src = static_cast<const unsigned char *>(in);
        auto *dst = static_cast<unsigned char *>(out);
        StepControl *ctl = chunk_ctl_.as<StepControl>();
        for (int i = 0; i < chunks; ++i) {
            const int f = i * chunk, k = std::min(chunk, M_ - f);
            const size_t off = static_cast<size_t>(f) * compact_, bytes = bytes_per * k;
            if (chained)
                cuda_check(cudaStreamWaitEvent(copy_in_, d2h_events_[i], 0), "order upload");
            cuda_check(cudaMemcpyAsync(omega_.as<cx<R>>() + off, src + bytes_per * f, bytes,
                                       cudaMemcpyHostToDevice, copy_in_),
                       "host state upload");
            cuda_check(cudaEventRecord(pipe_events_[2 * i], copy_in_), "record event");
            // consecutive chunks alternate between two compute streams, so that one chunk's
            // kernels fill the SMs left idle by the last work items of the other's
            const cudaStream_t cs = (i & 1) ? compute2_ : stream_;
            cuda_check(cudaStreamWaitEvent(cs, pipe_events_[2 * i], 0), "order step");
            ColumnArgs<R> a = column_args(dt);
            RowArgs<R> r = row_args();
            a.omega += off;
            a.ystage += off;
            a.acc += off;
            a.w += static_cast<size_t>(f) * n_ * 2 * velocity_row_stride<R>(n_);
            a.nl += static_cast<size_t>(f) * 2 * C_ * n_;
            if (a.forcing && a.forcing_stride)
                a.forcing += static_cast<size_t>(f) * a.forcing_stride;
            a.member_base += static_cast<unsigned>(f);
            a.members = k;
            a.ctl = ctl + i;
            r.w = a.w;
            r.nl = nl_.as<cx<R>>() + static_cast<size_t>(f) * 2 * C_ * n_;
            r.members = k;
            r.ctl = ctl + i;
            a.stage = 0;
            cuda_check(launch_column<R>(n_, a, cs), "launch start column pass");
            for (uint64_t st = 0; st < nsteps; ++st)
                for (int stage = 1; stage <= 4; ++stage) {
                    r.cfl_scale = stage == 1 ? dt * n_ / (2 * kPi) : 0.0;
                    cuda_check(launch_row<R>(n_, r, cs), "launch row pass");
                    a.stage = stage;
                    cuda_check(launch_column<R>(n_, a, cs), "launch column pass");
                }
            cuda_check(cudaEventRecord(pipe_events_[2 * i + 1], cs), "record event");
            cuda_check(cudaStreamWaitEvent(copy_out_, pipe_events_[2 * i + 1], 0), "order download");
            cuda_check(cudaMemcpyAsync(dst + bytes_per * f, omega_.as<cx<R>>() + off, bytes,
                                       cudaMemcpyDeviceToHost, copy_out_),
                       "host state download");
            cuda_check(cudaEventRecord(d2h_events_[i], copy_out_), "record event");
        }
        cuda_check(cudaEventRecord(side, compute2_), "record event");
        cuda_check(cudaStreamWaitEvent(stream_, side, 0), "join compute streams");
        merge_chunk_control<<<1, 32, 0, stream_>>>(ctl_.as<StepControl>(), ctl, chunks,
                                                    step_index + nsteps);
        cuda_check(cudaGetLastError(), "merge chunk control");
        cuda_check(cudaEventRecord(end, copy_out_), "record event");
        cuda_check(cudaStreamWaitEvent(stream_, end, 0), "order library stream");
        w_valid_ = true;
        time += dt * static_cast<double>(nsteps);
        step_index += nsteps;
        pipe_mark_ = api_calls;
        pipe_chunks_ = chunks;
    }
    void step_profiled(double dt, uint64_t nsteps, double *row_ms, double *col_ms) override {
        const int largest = (n_ - 1) / 3;
        if (!std::isfinite(dt) || dt <= 0 ||
            dt * (2 * cfg_.nu * largest * largest + cfg_.alpha) > 2.5)
            raise(HZLB_EINVAL, "invalid GPU time step or diffusion stability limit exceeded");
        *row_ms = *col_ms = 0;
        if (ou_)
            raise(HZLB_EINVAL, "profiled stepping times the spectral kernels only; it does not "
                               "advance device OU forcing");
        if (nsteps == 0)
            return;
        if (!w_valid_)
            launch_start();
        std::vector<cudaEvent_t> ev(8 * nsteps + 1);
        for (auto &e : ev)
            cuda_check(cudaEventCreate(&e), "create profiling event");
        ColumnArgs<R> a = column_args(dt);
        RowArgs<R> r = row_args();
        size_t k = 0;
        cuda_check(cudaEventRecord(ev[k++], stream_), "record event");
        (void)k;
        for (uint64_t i = 0; i < nsteps; ++i)
            for (int s = 1; s <= 4; ++s) {
                r.cfl_scale = s == 1 ? dt * n_ / (2 * kPi) : 0.0;
                cuda_check(launch_row<R>(n_, r, stream_), "launch row pass");
                cuda_check(cudaEventRecord(ev[k++], stream_), "record event");
                a.stage = s;
                cuda_check(launch_column<R>(n_, a, stream_), "launch column pass");
                cuda_check(cudaEventRecord(ev[k++], stream_), "record event");
            }
        cuda_check(cudaStreamSynchronize(stream_), "profiled steps");
        double rsum = 0, csum = 0;
        // events: ev[0] before the first launch, then one after every launch
        for (size_t i = 0; i < 4 * nsteps; ++i) {
            float t1 = 0, t2 = 0;
            cuda_check(cudaEventElapsedTime(&t1, ev[2 * i], ev[2 * i + 1]), "event time");
            cuda_check(cudaEventElapsedTime(&t2, ev[2 * i + 1], ev[2 * i + 2]), "event time");
            rsum += t1;
            csum += t2;
        }
        for (auto &e : ev)
            cudaEventDestroy(e);
        *row_ms = rsum / (4.0 * nsteps);
        *col_ms = csum / (4.0 * nsteps);
        w_valid_ = true;
        time += dt * static_cast<double>(nsteps);
        step_index += nsteps;
    }
    void set_time(double t, uint64_t s) override {
        time = t;
        step_index = s;
        StepControl c{};
        c.step = s;
        cuda_check(cudaMemcpyAsync(ctl_.ptr, &c, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                   stream_),
                   "set step counter");
        cuda_check(cudaStreamSynchronize(stream_), "set step counter");
    }
    void inject_wait_timeout() override {
        const unsigned one = 1;
        cuda_check(cudaMemcpyAsync(&ctl_.as<StepControl>()->inject, &one, sizeof one,
                                   cudaMemcpyHostToDevice, stream_),
                   "arm wait-timeout test hook");
        cuda_check(cudaStreamSynchronize(stream_), "arm wait-timeout test hook");
        w_valid_ = false;
    }
    uint32_t status() override {
        StepControl c{};
        cuda_check(cudaMemcpyAsync(&c, ctl_.ptr, sizeof c, cudaMemcpyDeviceToHost, stream_),
                   "read status");
        cuda_check(cudaStreamSynchronize(stream_), "read status");
        if (c.status) {
            const unsigned zero = 0;
            cuda_check(cudaMemcpyAsync(&ctl_.as<StepControl>()->status, &zero, sizeof zero,
                                       cudaMemcpyHostToDevice, stream_),
                       "clear status");
            cuda_check(cudaStreamSynchronize(stream_), "clear status");
        }
        return c.status;
    }
    void synchronize() override { cuda_check(cudaStreamSynchronize(stream_), "synchronize GPU"); }

    // ---- diagnostics and observations ---------------------------------------------
    void diagnostics(double *out) override {
        scratch_d_.ensure(sizeof(double) * 3 * M_, "allocate diagnostics");
        vbits_.ensure(sizeof(unsigned long long) * M_, "allocate CFL reduction");
        cuda_check(launch_diagnostics<R>(n_, omega_.as<cx<R>>(), fcount_ ? forcing_.as<cx<R>>() : nullptr,
                                         cfg_.forcing_per_member ? static_cast<long long>(fcols_) * LD_ : 0,
                                         fcols_, M_, scratch_d_.as<double>(), stream_),
                   "launch diagnostics");
        launch_start();
        w_valid_ = true;
        cuda_check(cudaMemsetAsync(vbits_.ptr, 0, sizeof(unsigned long long) * M_, stream_),
                   "reset CFL reduction");
        cuda_check(launch_velocity_max<R>(n_, w_.as<cx<R>>(), vbits_.as<unsigned long long>(),
                                          tw_.as<cx<R>>(), M_, stream_),
                   "launch CFL reduction");
        std::vector<double> sums(3 * M_);
        std::vector<unsigned long long> bits(M_);
        cuda_check(cudaMemcpyAsync(sums.data(), scratch_d_.ptr, sizeof(double) * 3 * M_,
                                   cudaMemcpyDeviceToHost, stream_),
                   "diagnostics download");
        cuda_check(cudaMemcpyAsync(bits.data(), vbits_.ptr, sizeof(unsigned long long) * M_,
                                   cudaMemcpyDeviceToHost, stream_),
                   "CFL scalar transfer");
        cuda_check(cudaStreamSynchronize(stream_), "diagnostics");
        for (int m = 0; m < M_; ++m) {
            double vmax;
            std::memcpy(&vmax, &bits[m], sizeof vmax);
            out[6 * m + 0] = time;
            out[6 * m + 1] = sums[3 * m];
            out[6 * m + 2] = sums[3 * m + 1];
            out[6 * m + 3] = 2 * cfg_.nu * sums[3 * m + 1];
            out[6 * m + 4] = sums[3 * m + 2];
            out[6 * m + 5] = vmax * static_cast<double>(n_) / (2 * kPi);
        }
    }
    // physical fields into phys_ (device), via the Jacobian-row buffer as column scratch
    void physical_device() {
        phys_.ensure(sizeof(R) * static_cast<size_t>(n_) * n_ * M_, "allocate physical fields");
        cuda_check(launch_physical<R>(n_, omega_.as<cx<R>>(), static_cast<long long>(compact_),
                                      nl_.as<cx<R>>(), phys_.as<R>(), tw_.as<cx<R>>(), M_, stream_),
                   "launch physical transform");
    }
    void physical(double *out) override {
        physical_device();
        const size_t count = static_cast<size_t>(n_) * n_ * M_;
        staging_.ensure(sizeof(R) * count);
        cuda_check(cudaMemcpyAsync(staging_.ptr, phys_.ptr, sizeof(R) * count,
                                   cudaMemcpyDeviceToHost, stream_),
                   "physical field download");
        cuda_check(cudaStreamSynchronize(stream_), "physical field download");
        const R *p = staging_.as<R>();
        for (size_t i = 0; i < count; ++i)
            out[i] = p[i];
    }
    void observe_device(const uint32_t *x, const uint32_t *y, size_t p) {
        for (size_t o = 0; o < p; ++o)
            if (x[o] >= static_cast<uint32_t>(n_) || y[o] >= static_cast<uint32_t>(n_))
                raise(HZLB_EINVAL, "observation location out of bounds");
        obs_.ensure(sizeof(double) * std::max<size_t>(p, 1) * M_, "allocate observations");
        // the row pairs (2q, 2q+1) the observation rows lie in; when they are fewer than all
        // the rows, only those are transformed (the same values, see field_row_pairs_inverse)
        std::vector<int> pairs;
        for (size_t o = 0; o < p; ++o)
            pairs.push_back(static_cast<int>(y[o] >> 1));
        std::sort(pairs.begin(), pairs.end());
        pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
        if (p > 0 && 2 * pairs.size() < static_cast<size_t>(n_)) {
            const size_t np = pairs.size();
            std::vector<uint32_t> host(2 * p + np);
            for (size_t o = 0; o < p; ++o) {
                host[o] = x[o];
                const size_t q = std::lower_bound(pairs.begin(), pairs.end(), static_cast<int>(y[o] >> 1)) -
                                 pairs.begin();
                host[p + o] = static_cast<uint32_t>(2 * q + (y[o] & 1));
            }
            for (size_t q = 0; q < np; ++q)
                host[2 * p + q] = static_cast<uint32_t>(pairs[q]);
            obs_xy_.ensure(sizeof(uint32_t) * host.size(), "allocate observation points");
            cuda_check(cudaMemcpyAsync(obs_xy_.ptr, host.data(), sizeof(uint32_t) * host.size(),
                                       cudaMemcpyHostToDevice, stream_),
                       "upload observation points");
            phys_.ensure(sizeof(R) * static_cast<size_t>(n_) * n_ * M_, "allocate physical fields");
            const unsigned *dx = obs_xy_.as<unsigned>();
            cuda_check(launch_observe_rows<R>(n_, omega_.as<cx<R>>(), static_cast<long long>(compact_),
                                              nl_.as<cx<R>>(), phys_.as<R>(),
                                              reinterpret_cast<const int *>(dx + 2 * p),
                                              static_cast<int>(np), dx, dx + p, static_cast<int>(p),
                                              tw_.as<cx<R>>(), M_, obs_.as<double>(), stream_),
                       "launch observation operator");
            return;
        }
        physical_device();
        obs_xy_.ensure(sizeof(uint32_t) * 2 * std::max<size_t>(p, 1), "allocate observation points");
        cuda_check(cudaMemcpyAsync(obs_xy_.ptr, x, sizeof(uint32_t) * p, cudaMemcpyHostToDevice, stream_),
                   "upload observation points");
        cuda_check(cudaMemcpyAsync(obs_xy_.as<uint32_t>() + p, y, sizeof(uint32_t) * p,
                                   cudaMemcpyHostToDevice, stream_),
                   "upload observation points");
        cuda_check(launch_gather<R>(phys_.as<R>(), n_, obs_xy_.as<unsigned>(),
                                    obs_xy_.as<unsigned>() + p, static_cast<int>(p), M_,
                                    obs_.as<double>(), stream_),
                   "launch observation gather");
    }
    void observe(const uint32_t *x, const uint32_t *y, size_t p, double *out) override {
        observe_device(x, y, p);
        cuda_check(cudaMemcpyAsync(out, obs_.ptr, sizeof(double) * p * M_, cudaMemcpyDeviceToHost,
                                   stream_),
                   "observation download");
        cuda_check(cudaStreamSynchronize(stream_), "observation download");
    }

    // ---- particle filter on the device (filter.cpp:65-120) -----------------------------
    static constexpr int kPfThreads = 256;
    double half_log_two_pi() const { return 0.5 * std::log(2 * kPi); }
    void pf_ensure() {
        if (pf_particles_ == 0)
            pf_reset(M_);
    }
    void pf_reset(int particles) override {
        if (particles < 2)
            raise(HZLB_EINVAL, "particle filter needs at least two particles");
        if (M_ % particles != 0)
            raise(HZLB_EINVAL, "ensemble members must be a multiple of the particle count");
        const int segments = M_ / particles;
        pfw_.ensure(sizeof(double) * 3 * static_cast<size_t>(M_), "allocate particle weights");
        pfrec_.ensure(sizeof(PfRecord) * segments, "allocate particle records");
        pfctl_.ensure(sizeof(double) * segments + segments + 16, "allocate particle controls");
        anc_.ensure(sizeof(unsigned) * M_, "allocate ancestors");
        std::vector<double> w(M_, 1 / static_cast<double>(particles));
        cuda_check(cudaMemcpyAsync(pfw_.ptr, w.data(), sizeof(double) * M_, cudaMemcpyHostToDevice,
                                   stream_),
                   "reset particle weights");
        cuda_check(cudaStreamSynchronize(stream_), "reset particle weights");
        pf_particles_ = particles;
    }
    void pf_get_weights(double *out) override {
        pf_ensure();
        cuda_check(cudaMemcpyAsync(out, pfw_.ptr, sizeof(double) * M_, cudaMemcpyDeviceToHost, stream_),
                   "download particle weights");
        cuda_check(cudaStreamSynchronize(stream_), "download particle weights");
    }
    // observed values and uncertainties of p observations into a device buffer (2p doubles)
    const double *pf_upload_obs(const double *values, const double *sd, size_t p) {
        for (size_t o = 0; o < p; ++o)
            if (!std::isfinite(values[o]) || !std::isfinite(sd[o]) || sd[o] <= 0)
                raise(HZLB_EINVAL, "observations must be finite and have positive uncertainty");
        pfobs_.ensure(sizeof(double) * 2 * std::max<size_t>(p, 1), "allocate observations");
        cuda_check(cudaMemcpyAsync(pfobs_.ptr, values, sizeof(double) * p, cudaMemcpyHostToDevice,
                                   stream_),
                   "upload observations");
        cuda_check(cudaMemcpyAsync(pfobs_.as<double>() + p, sd, sizeof(double) * p,
                                   cudaMemcpyHostToDevice, stream_),
                   "upload observation errors");
        return pfobs_.as<double>();
    }
    void pf_loglik(const uint32_t *x, const uint32_t *y, const double *values, const double *sd,
                   size_t p, double *log_weights) override {
        pf_ensure();
        const double *ob = pf_upload_obs(values, sd, p);
        observe_device(x, y, p);
        double *logs = pfw_.as<double>() + M_;
        cuda_check(cudaMemcpyAsync(logs, log_weights, sizeof(double) * M_, cudaMemcpyHostToDevice,
                                   stream_),
                   "upload log-weights");
        pf_loglik_kernel<<<(M_ + 127) / 128, 128, 0, stream_>>>(
            obs_.as<double>(), static_cast<int>(p), ob, ob + p, half_log_two_pi(), nullptr, logs, M_,
            M_, nullptr);
        cuda_check(cudaGetLastError(), "launch particle log-likelihood");
        cuda_check(cudaMemcpyAsync(log_weights, logs, sizeof(double) * M_, cudaMemcpyDeviceToHost,
                                   stream_),
                   "download log-weights");
        cuda_check(cudaStreamSynchronize(stream_), "particle log-likelihood");
    }
    void pf_weights(const double *logs, size_t count, double *w, double *inc, double *ess,
                    double *mw) override {
        if (count < 2)
            raise(HZLB_EINVAL, "particle filter needs at least two particles");
        if (count > (1u << 24))
            raise(HZLB_EINVAL, "too many particle weights");
        // logs, weights, scratch, then the record and ancestors
        const size_t bytes = sizeof(double) * 3 * count + sizeof(PfRecord) + sizeof(unsigned) * count;
        pfone_.ensure(bytes + 64, "allocate particle weights");
        double *dl = pfone_.as<double>(), *dw = dl + count, *dx = dw + count;
        PfRecord *rec = reinterpret_cast<PfRecord *>(dx + count);
        unsigned *anc = reinterpret_cast<unsigned *>(rec + 1);
        cuda_check(cudaMemcpyAsync(dl, logs, sizeof(double) * count, cudaMemcpyHostToDevice, stream_),
                   "upload log-weights");
        pf_normalise_kernel<kPfThreads><<<1, kPfThreads, 0, stream_>>>(
            dl, dw, dx, static_cast<int>(count), nullptr, nullptr, rec, anc);
        cuda_check(cudaGetLastError(), "launch particle weights");
        PfRecord r{};
        cuda_check(cudaMemcpyAsync(&r, rec, sizeof r, cudaMemcpyDeviceToHost, stream_),
                   "download particle record");
        cuda_check(cudaMemcpyAsync(w, dw, sizeof(double) * count, cudaMemcpyDeviceToHost, stream_),
                   "download particle weights");
        cuda_check(cudaStreamSynchronize(stream_), "particle weights");
        if (r.collapsed)
            raise(HZLB_ERUNTIME, "particle likelihood collapsed numerically");
        *inc = r.increment;
        *ess = r.ess;
        *mw = r.max_weight;
    }
    void pf_assimilate(const uint32_t *x, const uint32_t *y, const double *values, const double *sd,
                       size_t p, const double *u, const uint8_t *active, hzlb_pf_record *records,
                       uint32_t *ancestors, double *weighted_mean) override {
        static_assert(sizeof(PfRecord) == sizeof(hzlb_pf_record), "record layouts agree");
        pf_ensure();
        const int P = pf_particles_, S = M_ / P;
        const double *ob = pf_upload_obs(values, sd, p);
        if (u)
            for (int s = 0; s < S; ++s)
                if (!(u[s] < 1) || std::isnan(u[s]))
                    raise(HZLB_EINVAL, "resampling uniform must lie in [0, 1) (negative: none)");
        double *du = pfctl_.as<double>();
        unsigned char *dact = reinterpret_cast<unsigned char *>(du + S);
        if (u)
            cuda_check(cudaMemcpyAsync(du, u, sizeof(double) * S, cudaMemcpyHostToDevice, stream_),
                       "upload resampling uniforms");
        if (active)
            cuda_check(cudaMemcpyAsync(dact, active, S, cudaMemcpyHostToDevice, stream_),
                       "upload segment flags");
        double *w = pfw_.as<double>(), *logs = w + M_, *scratch = logs + M_;
        PfRecord *rec = pfrec_.as<PfRecord>();
        unsigned *anc = anc_.as<unsigned>();
        if (p > 0) {
            observe_device(x, y, p);
        } else {
            obs_.ensure(sizeof(double) * M_, "allocate observations");
        }
        // records of inactive segments stay zero (nothing resampled there)
        cuda_check(cudaMemsetAsync(rec, 0, sizeof(PfRecord) * S, stream_), "clear particle records");
        pf_loglik_kernel<<<(M_ + 127) / 128, 128, 0, stream_>>>(
            obs_.as<double>(), static_cast<int>(p), ob, ob + p, half_log_two_pi(), w, logs, M_, P,
            active ? dact : nullptr);
        pf_normalise_kernel<kPfThreads><<<S, kPfThreads, 0, stream_>>>(
            logs, w, scratch, P, u ? du : nullptr, active ? dact : nullptr, rec, anc);
        cuda_check(cudaGetLastError(), "launch particle weights");
        if (weighted_mean) {
            aux_.ensure(sizeof(double) * 2 * compact_ * S + sizeof(double) * M_, "allocate weighted mean");
            const dim3 g(static_cast<unsigned>(std::min<size_t>((compact_ + 255) / 256, 2048)), S);
            segment_weighted_sum<R><<<g, 256, 0, stream_>>>(omega_.as<cx<R>>(), w,
                                                            static_cast<long long>(compact_), P,
                                                            aux_.as<double>());
            cuda_check(cudaGetLastError(), "launch weighted mean");
            cuda_check(cudaMemcpyAsync(weighted_mean, aux_.ptr, sizeof(double) * 2 * compact_ * S,
                                       cudaMemcpyDeviceToHost, stream_),
                       "download weighted mean");
        }
        if (u) {
            pf_reset_resampled<<<(M_ + 255) / 256, 256, 0, stream_>>>(w, rec, M_, P);
            const dim3 gg(std::max<int>(1, static_cast<int>(std::min<size_t>((compact_ + 255) / 256, 64))), M_);
            pf_gather_resampled<R><<<gg, 256, 0, stream_>>>(omega_.as<cx<R>>(), ystage_.as<cx<R>>(),
                                                            anc, rec, P, static_cast<long long>(compact_));
            pf_commit_resampled<R><<<gg, 256, 0, stream_>>>(ystage_.as<cx<R>>(), omega_.as<cx<R>>(),
                                                            rec, P, static_cast<long long>(compact_));
            if (fcount_ > 1) {
                const long long fb = static_cast<long long>(fcols_) * LD_;
                const dim3 fg(std::max<int>(1, static_cast<int>(std::min<long long>((fb + 255) / 256, 64))), M_);
                pf_gather_resampled<R><<<fg, 256, 0, stream_>>>(forcing_.as<cx<R>>(), ystage_.as<cx<R>>(),
                                                                anc, rec, P, fb);
                pf_commit_resampled<R><<<fg, 256, 0, stream_>>>(ystage_.as<cx<R>>(), forcing_.as<cx<R>>(),
                                                                rec, P, fb);
            }
            cuda_check(cudaGetLastError(), "launch resampled gather");
        }
        std::vector<PfRecord> host(S);
        cuda_check(cudaMemcpyAsync(host.data(), rec, sizeof(PfRecord) * S, cudaMemcpyDeviceToHost,
                                   stream_),
                   "download particle records");
        if (ancestors)
            cuda_check(cudaMemcpyAsync(ancestors, anc, sizeof(unsigned) * M_, cudaMemcpyDeviceToHost,
                                       stream_),
                       "download ancestors");
        cuda_check(cudaStreamSynchronize(stream_), "particle filter update");
        for (int s = 0; s < S; ++s)
            if (!active || active[s])
                std::memcpy(&records[s], &host[s], sizeof(PfRecord));
        for (int s = 0; s < S; ++s)
            if (host[s].resampled && (!active || active[s])) {
                w_valid_ = false;
                break;
            }
    }

    // ---- filters --------------------------------------------------------------------
    void resample(const double *w, size_t count, double u, uint32_t *anc) override {
        scratch_d_.ensure(sizeof(double) * 2 * count, "allocate resampling weights");
        anc_.ensure(sizeof(unsigned) * count, "allocate ancestors");
        cuda_check(cudaMemcpyAsync(scratch_d_.ptr, w, sizeof(double) * count, cudaMemcpyHostToDevice,
                                   stream_),
                   "upload weights");
        systematic_resample_kernel<<<1, 1024, 0, stream_>>>(
            scratch_d_.as<double>(), scratch_d_.as<double>() + count, static_cast<int>(count), u,
            anc_.as<unsigned>());
        cuda_check(cudaGetLastError(), "launch resampling");
        cuda_check(cudaMemcpyAsync(anc, anc_.ptr, sizeof(unsigned) * count, cudaMemcpyDeviceToHost,
                                   stream_),
                   "download ancestors");
        cuda_check(cudaStreamSynchronize(stream_), "resampling");
    }
    void gather(const uint32_t *ancestors) override {
        for (int i = 0; i < M_; ++i)
            if (ancestors[i] >= static_cast<uint32_t>(M_))
                raise(HZLB_EINVAL, "ancestor index out of range");
        anc_.ensure(sizeof(unsigned) * M_, "allocate ancestors");
        cuda_check(cudaMemcpyAsync(anc_.ptr, ancestors, sizeof(unsigned) * M_, cudaMemcpyHostToDevice,
                                   stream_),
                   "upload ancestors");
        const dim3 grid(std::max<int>(1, static_cast<int>((compact_ + 255) / 256)), M_);
        gather_blocks<R><<<grid, 256, 0, stream_>>>(omega_.as<cx<R>>(), ystage_.as<cx<R>>(),
                                                    anc_.as<unsigned>(), static_cast<long long>(compact_));
        cuda_check(cudaGetLastError(), "launch member gather");
        cuda_check(cudaMemcpyAsync(omega_.ptr, ystage_.ptr, sizeof(cx<R>) * compact_ * M_,
                                   cudaMemcpyDeviceToDevice, stream_),
                   "commit member gather");
        if (fcount_ > 1) {
            const long long fb = static_cast<long long>(fcols_) * LD_;
            const dim3 fg(std::max<int>(1, static_cast<int>((fb + 255) / 256)), M_);
            gather_blocks<R><<<fg, 256, 0, stream_>>>(forcing_.as<cx<R>>(), ystage_.as<cx<R>>(),
                                                      anc_.as<unsigned>(), fb);
            cuda_check(cudaGetLastError(), "launch forcing gather");
            cuda_check(cudaMemcpyAsync(forcing_.ptr, ystage_.ptr, sizeof(cx<R>) * fb * M_,
                                       cudaMemcpyDeviceToDevice, stream_),
                       "commit forcing gather");
        }
        cuda_check(cudaStreamSynchronize(stream_), "member gather");
        w_valid_ = false;
    }
    void inflate(double inflation) override {
        if (!std::isfinite(inflation) || inflation < 1)
            raise(HZLB_EINVAL, "EnKF inflation must be >= 1");
        if (inflation == 1)
            return;
        const long long nr = 2 * static_cast<long long>(compact_);
        R *mean = acc_.as<R>();   // free between steps
        member_mean<R><<<static_cast<unsigned>((nr + 31) / 32), dim3(32, 8), 0, stream_>>>(
            reinterpret_cast<const R *>(omega_.ptr), nr, M_, mean);
        inflate_kernel<R><<<2048, 256, 0, stream_>>>(reinterpret_cast<R *>(omega_.ptr), mean, nr, M_,
                                                     inflation);
        cuda_check(cudaGetLastError(), "launch inflation");
        w_valid_ = false;
    }
    const hzlb_config &config() const override { return cfg_; }
    void mean_device(void *out) override {
        const long long nr = 2 * static_cast<long long>(compact_);
        member_mean<R><<<static_cast<unsigned>((nr + 31) / 32), dim3(32, 8), 0, stream_>>>(
            reinterpret_cast<const R *>(omega_.ptr), nr, M_, static_cast<R *>(out));
        cuda_check(cudaGetLastError(), "launch ensemble mean");
        cuda_check(cudaStreamSynchronize(stream_), "ensemble mean");
    }
    void *state_device() override {
        w_valid_ = false;
        return omega_.ptr;
    }
    // The FP64 ensemble-space solve of the perturbed-observation analysis for M members whose
    // predicted observations hx (device, M x p, row m = member) are given: innovations and
    // anomalies, S = HA^T HA/(M-1) + R, its Cholesky, the forward substitution of [HA; D; dbar],
    // the innovation statistic and -- unless nis_limit > 0 and the statistic exceeds it --
    // W = (L^-1 HA)^T-rows (L^-1 D)-rows / (M-1) (M x M, rows: contributing member) in the
    // workspace, *W_dev pointing at it.  eps: M x p standard normals on the host
    // (eps_on_device false), on the device (true), or null for the Philox draws keyed by
    // (seed, member_base + m) with counter `cycle`.
    EnkfResult solve_weights(const double *hx, int M, size_t p, const double *values,
                             const double *sd, const double *eps, bool eps_on_device,
                             uint64_t seed, uint64_t cycle, uint32_t member_base,
                             double nis_limit, double **W_dev) {
        if (M < 2)
            raise(HZLB_EINVAL, "EnKF requires at least two ensemble members");
        for (size_t o = 0; o < p; ++o)
            if (!std::isfinite(values[o]) || !std::isfinite(sd[o]) || sd[o] <= 0)
                raise(HZLB_EINVAL, "observations must be finite and have positive uncertainty");
        if (p > (1u << 20))
            raise(HZLB_EINVAL, "too many observations for one analysis");
        const int pi = static_cast<int>(p);
        const size_t mp = static_cast<size_t>(M) * p, m1p = mp + p;
        const size_t nblk = (p + d64::NB - 1) / d64::NB;
        const size_t eps_n = (eps && !eps_on_device) ? mp : 0;
        // ha (M rows) and d (M + 1 rows) are adjacent: one forward substitution covers both
        const size_t doubles = 3 * p + eps_n + mp + m1p + (mp + m1p) + p * p +
                               nblk * d64::NB * d64::NB + static_cast<size_t>(M) * M + 1;
        enkf_.ensure(sizeof(double) * doubles + 64, "allocate EnKF workspace");
        double *ybuf = enkf_.as<double>(), *sdbuf = ybuf + p, *hmean = sdbuf + p,
               *eps_d = hmean + p, *ha = eps_d + eps_n, *d = ha + mp, *yw = d + m1p,
               *P = yw + mp + m1p, *inv = P + p * p, *W = inv + nblk * d64::NB * d64::NB,
               *nis_d = W + static_cast<size_t>(M) * M;
        int *info = reinterpret_cast<int *>(nis_d + 1);
        cuda_check(cudaMemcpyAsync(ybuf, values, sizeof(double) * p, cudaMemcpyHostToDevice,
                                   stream_),
                   "upload observations");
        cuda_check(cudaMemcpyAsync(sdbuf, sd, sizeof(double) * p, cudaMemcpyHostToDevice, stream_),
                   "upload observation errors");
        const double *eps_used = nullptr;
        if (eps && !eps_on_device) {
            cuda_check(cudaMemcpyAsync(eps_d, eps, sizeof(double) * mp, cudaMemcpyHostToDevice,
                                       stream_),
                       "upload perturbations");
            eps_used = eps_d;
        } else if (eps) {
            eps_used = eps;
        }
        cuda_check(cudaMemsetAsync(info, 0, sizeof(int), stream_), "clear Cholesky status");
        member_mean<double><<<(pi + 31) / 32, dim3(32, 8), 0, stream_>>>(hx, pi, M, hmean);
        enkf_innovations<<<1024, 256, 0, stream_>>>(hx, hmean, ybuf, sdbuf, eps_used, seed,
                                                    member_base, cycle, M, pi, ha, d);
        cuda_check(cudaGetLastError(), "launch EnKF innovations");
        // S = HA^T HA / (M-1) + R (lower triangle), FP64
        cuda_check(d64::gemm(d64::GemmArgs{pi, pi, M, 1.0 / (M - 1), 0.0, ha, 1, pi, ha, pi, 1,
                                           P, pi},
                             stream_, true),
                   "launch innovation covariance");
        add_obs_variance<<<(pi + 127) / 128, 128, 0, stream_>>>(P, sdbuf, pi);
        cuda_check(d64::cholesky(P, pi, inv, info, stream_), "launch innovation Cholesky");
        // L^{-1} applied to the anomalies HA, the M perturbed innovations and the mean
        // innovation at once (rows of [HA; D], written to yw): with S = L L^T,
        // W = (L^{-1} HA)^T-rows . (L^{-1} D)-rows / (M-1) and NIS = |L^{-1} dbar|^2 / p
        cuda_check(d64::forward_rows(P, pi, inv, ha, yw, 2 * M + 1, stream_),
                   "launch innovation solve");
        const double *yha = yw, *yd = yw + mp;
        innovation_statistic<<<1, 256, 0, stream_>>>(yd + mp, pi, nis_d);
        cuda_check(cudaGetLastError(), "launch innovation statistic");
        double nis = 0;
        int host_info = 0;
        cuda_check(cudaMemcpyAsync(&nis, nis_d, sizeof(double), cudaMemcpyDeviceToHost, stream_),
                   "read innovation statistic");
        cuda_check(cudaMemcpyAsync(&host_info, info, sizeof(int), cudaMemcpyDeviceToHost, stream_),
                   "read Cholesky status");
        cuda_check(cudaStreamSynchronize(stream_), "EnKF innovation solve");
        if (host_info != 0)
            raise(HZLB_ERUNTIME, "EnKF innovation covariance is not positive definite");
        *W_dev = W;
        if (nis_limit > 0 && !(nis <= nis_limit))
            return EnkfResult{nis, 0};
        // W[a][m] = sum_o (L^{-1} HA)[a][o] (L^{-1} D)[m][o] / (M-1)
        cuda_check(d64::gemm(d64::GemmArgs{M, M, pi, 1.0 / (M - 1), 0.0, yha, pi, 1, yd, 1, pi,
                                           W, M},
                             stream_),
                   "launch ensemble weights");
        return EnkfResult{nis, 1};
    }
    double enkf_weights(const double *hx, const double *values, const double *sd,
                        const double *eps, int members, size_t p, double *W_out) override {
        if (p == 0)
            raise(HZLB_EINVAL, "EnKF weights need at least one observation");
        double *W = nullptr;
        const EnkfResult r = solve_weights(hx, members, p, values, sd, eps, true, 0, 0, 0, 0.0, &W);
        cuda_check(cudaMemcpyAsync(W_out, W, sizeof(double) * members * members,
                                   cudaMemcpyDeviceToDevice, stream_),
                   "copy ensemble weights");
        cuda_check(cudaStreamSynchronize(stream_), "EnKF weights");
        return r.nis;
    }
    EnkfResult enkf(const EnkfRequest &q) override {
        if (M_ < 2)
            raise(HZLB_EINVAL, "EnKF requires at least two ensemble members");
        const size_t p = q.p;
        if (p == 0)
            return EnkfResult{0.0, 0};
        for (size_t o = 0; o < p; ++o)
            if (!std::isfinite(q.values[o]) || !std::isfinite(q.sd[o]) || q.sd[o] <= 0)
                raise(HZLB_EINVAL, "observations must be finite and have positive uncertainty");
        observe_device(q.x, q.y, p);
        double *W = nullptr;
        const EnkfResult solved = solve_weights(
            obs_.as<double>(), M_, p, q.values, q.sd, q.perturbations, false, q.perturbation_seed,
            q.cycle, static_cast<uint32_t>(cfg_.member_base), q.nis_limit, &W);
        if (!solved.applied)
            return solved;
        const double nis = solved.nis;
        cx<R> *mean = acc_.as<cx<R>>();   // free between steps
        member_mean<R><<<static_cast<unsigned>((2 * compact_ + 31) / 32), dim3(32, 8), 0, stream_>>>(
            reinterpret_cast<const R *>(omega_.ptr), static_cast<long long>(2 * compact_), M_,
            reinterpret_cast<R *>(mean));
        if constexpr (sizeof(R) == 4) {
            // X_a = X + A W on the tensor cores: A = X - mean and W split for 3xTF32
            // (hi*hi + hi*lo + lo*hi), accumulated into X in place
            const long long n = 2 * static_cast<long long>(compact_);
            float *x = reinterpret_cast<float *>(omega_.ptr);
            float *ahi = reinterpret_cast<float *>(ystage_.ptr);
            float *alo = reinterpret_cast<float *>(w_.ptr);   // velocity rows: free between steps
            float *mf = reinterpret_cast<float *>(nl_.ptr);
            cuda_check(cudaMemcpyAsync(mf, mean, sizeof(float) * n, cudaMemcpyDeviceToDevice, stream_),
                       "stage ensemble mean");
            split_.ensure(sizeof(float) * 2 * static_cast<size_t>(M_) * M_, "allocate weight split");
            float *whi = split_.as<float>(), *wlo = whi + static_cast<size_t>(M_) * M_;
            const dim3 tb(32, 8);
            anomaly_split_tf32_t<<<dim3(static_cast<unsigned>((n + 31) / 32), (M_ + 31) / 32), tb, 0,
                                   stream_>>>(x, mf, n, M_, ahi, alo);
            split_tf32_t<<<dim3((M_ + 31) / 32, (M_ + 31) / 32), tb, 0, stream_>>>(W, M_, whi, wlo);
            cuda_check(cudaGetLastError(), "launch 3xTF32 split");
            // one product with K = 3M: (whi, whi, wlo) against (ahi, alo, ahi)
            tc::GemmArgs g{};
            g.M = M_;
            g.N = static_cast<int>(n);
            g.K = 3 * M_;
            g.split3 = M_;
            g.A = whi;             // opA[m][a] = W[a][m], stored transposed
            g.A2 = wlo;
            g.lda = M_;
            g.a_kcontig = 1;
            g.B = ahi;             // opB[e][a] = A[a][e], stored transposed
            g.B2 = alo;
            g.ldb = M_;
            g.b_kcontig = 1;
            g.C = x;
            g.ldc = n;
            g.alpha = 1.0f;
            g.beta = 1.0f;
            g.epilogue = tc::EPI_NONE;
            g.status = &ctl_.as<StepControl>()->status;
            cuda_check(gemm(g, 4, stream_), "launch tensor-core EnKF update");
        } else {
            // FP64 path: X_a = X + (X - mean) W with FP64 accumulation
            const dim3 ug(static_cast<unsigned>((compact_ + 63) / 64), (M_ + 15) / 16);
            anomaly_update<R><<<ug, 64, 0, stream_>>>(omega_.as<cx<R>>(), mean, W,
                                                      static_cast<long long>(compact_), M_,
                                                      ystage_.as<cx<R>>());
            cuda_check(cudaGetLastError(), "launch EnKF update");
            cuda_check(cudaMemcpyAsync(omega_.ptr, ystage_.ptr, sizeof(cx<R>) * compact_ * M_,
                                       cudaMemcpyDeviceToDevice, stream_),
                       "commit EnKF update");
        }
        cuda_check(cudaStreamSynchronize(stream_), "EnKF analysis");
        w_valid_ = false;
        return EnkfResult{nis, 1};
    }

  private:
    struct Graph {
        double dt;
        int steps;
        cudaGraphExec_t exec;
    };
    hzlb_config cfg_;
    int n_ = 0, M_ = 0, K_ = 0, C_ = 0, LD_ = 0, fcols_ = 0, fcount_ = 0;
    bool ou_ = false;
    double ou_sigma_ = 0, ou_tau_ = 1;
    int ou_kmin_ = 0, ou_kmax_ = 0;
    size_t compact_ = 0;
    cudaStream_t stream_ = nullptr;
    DeviceBuffer omega_, ystage_, acc_, w_, nl_, forcing_, ctl_, tw_, phys_, scratch_d_, vbits_,
        obs_xy_, obs_, anc_, enkf_, aux_, split_, pfw_, pfrec_, pfctl_, pfobs_, pfone_, backup_;
    int pf_particles_ = 0;
    PinnedBuffer staging_, fstage_[2];
    cudaEvent_t fevent_[2] = {nullptr, nullptr};
    int fbuf_next_ = 0;
    std::vector<Graph> graphs_;
    bool w_valid_ = false;
    cudaStream_t copy_in_ = nullptr, copy_out_ = nullptr, compute2_ = nullptr;
    std::vector<cudaEvent_t> pipe_events_;
    DeviceBuffer chunk_ctl_;
    // host-pipelined stepping: per-chunk download events of the last call, the handle's call
    // count at its end (0: none yet) and its chunk count
    std::vector<cudaEvent_t> d2h_events_;
    uint64_t pipe_mark_ = 0;
    int pipe_chunks_ = 0;
    // step graphs in two parts (split_members); two parts side by side measured 285k against
    // 274k member-steps/s in FP64 and 614k against 606k in FP32 (2048 members, 256^2, graphs
    // of 8 steps), the offset parts 283k and 610k
    int schedule_ = 1;
    cudaEvent_t split_events_[3] = {nullptr, nullptr, nullptr};
    DeviceBuffer split_ctl_;
};

} // namespace

std::unique_ptr<Engine> make_engine(const hzlb_config &c) {
    if (c.precision == 4)
        return std::make_unique<EngineT<float>>(c);
    if (c.precision == 8)
        return std::make_unique<EngineT<double>>(c);
    raise(HZLB_EINVAL, "precision must be 4 (FP32) or 8 (FP64)");
}

} // namespace hzlb
