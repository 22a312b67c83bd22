// Mixed-resolution ensembles advanced together: one CUDA graph per batch of steps holds every
// resolution's RK4 launches.  In the concurrent schedule the graph forks one branch per
// resolution (each branch on its own stream during capture, so the kernels of different
// resolutions share the SMs), and joins at the end; in the serial schedule the resolutions
// follow each other on one stream, each with the whole device.  The persistent row/column
// kernels of each resolution take a cap on their grid (blocks), so concurrent branches can be
// given shares of the GPU.
//
// The autotuner (hzlb_mixed_tune) measures the batch step time of candidate schedules on the
// actual ensembles — the serial schedule, and the concurrent schedule with each resolution's
// grid cap chosen by coordinate descent over fractions of its resident block count (largest
// work first, two passes) and then each resolution's row-kernel block shape (64 or 128
// threads) — and keeps the fastest.  Each candidate is captured as a graph and
// timed with CUDA events after a warm-up launch.  The ensembles' states and clocks are saved
// on the device before tuning and restored after it, so tuning leaves them as they were.
//
// No counterpart in the reference (it steps one solver at a time).
#include "engine.h"
#include "launch.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

namespace hzlb {

struct GroupCaps {
    int col = 0, row = 0;   // 0: every resident block
    int row_threads = 0;    // row kernel block shape, 64 or 128 threads (0: the default)
};

// How a batch's steps are laid out in its graph: each resolution's own kernels one after
// another (serial) or on concurrent branches with capped grids (concurrent); or one persistent
// row kernel and one column kernel per RK stage over the whole mixed work list (fused); or the
// fused kernels over 64^2..256^2 with the 512^2 resolution's kernels on a concurrent branch
// (fused_branch: the 512^2 column pass needs 232 registers, which would cap every resolution's
// residency in one kernel).
enum class Mode : int { Serial = 0, Concurrent = 1, Fused = 2, FusedBranch = 3 };

class Mixed {
  public:
    Mixed(const hzlb_config *cfgs, int count) {
        if (!cfgs || count < 1 || count > 16)
            raise(HZLB_EINVAL, "mixed batch needs 1..16 ensemble configurations");
        device_ = cfgs[0].device;
        for (int g = 0; g < count; ++g) {
            if (cfgs[g].device != device_)
                raise(HZLB_EINVAL, "all resolutions of a mixed batch must be on one device");
            auto h = std::make_unique<hzlb_ensemble>();
            h->engine = make_engine(cfgs[g]);
            groups_.push_back(std::move(h));
        }
        cuda_check(cudaSetDevice(device_), "select CUDA device");
        cuda_check(cudaStreamCreateWithFlags(&main_, cudaStreamNonBlocking), "create stream");
        branch_.resize(count);
        join_.resize(count);
        for (int g = 0; g < count; ++g) {
            cuda_check(cudaStreamCreateWithFlags(&branch_[g], cudaStreamNonBlocking), "create stream");
            cuda_check(cudaEventCreateWithFlags(&join_[g], cudaEventDisableTiming), "create event");
        }
        cuda_check(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "create event");
        caps_.assign(count, GroupCaps{});
        resident_.resize(count);
        for (int g = 0; g < count; ++g) {
            const hzlb_config &c = cfgs[g];
            cudaError_t e = c.precision == 4
                                ? resident_blocks<float>(c.n, &resident_[g].col, &resident_[g].row)
                                : resident_blocks<double>(c.n, &resident_[g].col, &resident_[g].row);
            cuda_check(e, "query resident blocks");
        }
    }
    ~Mixed() {
        drop();
        for (auto s : branch_)
            if (s)
                cudaStreamDestroy(s);
        for (auto e : join_)
            if (e)
                cudaEventDestroy(e);
        if (fork_)
            cudaEventDestroy(fork_);
        if (main_)
            cudaStreamDestroy(main_);
    }
    int count() const { return static_cast<int>(groups_.size()); }
    hzlb_ensemble *group(int g) { return g >= 0 && g < count() ? groups_[g].get() : nullptr; }

    void step(const double *dt, uint64_t nsteps) {
        check_dt(dt);
        for (int g = 0; g < count(); ++g)
            groups_[g]->engine->prepare_steps(dt[g]);
        constexpr int kBatch = 8;
        uint64_t left = nsteps;
        while (left >= kBatch) {
            cuda_check(cudaGraphLaunch(graph_for(dt, kBatch), main_), "launch mixed graph");
            left -= kBatch;
        }
        if (left)
            cuda_check(cudaGraphLaunch(graph_for(dt, static_cast<int>(left)), main_),
                       "launch mixed graph");
        cuda_check(cudaStreamSynchronize(main_), "mixed step");
        for (int g = 0; g < count(); ++g)
            groups_[g]->engine->finish_steps(dt[g], nsteps);
    }

    // Returns the best step time (ms per step); the chosen schedule stays in effect.
    double tune(const double *dt, int repeats) {
        check_dt(dt);
        repeats = std::max(1, repeats);
        // save every group's state and clock (restored below)
        std::vector<DeviceBuffer> saved(count());
        std::vector<std::pair<double, uint64_t>> clocks(count());
        for (int g = 0; g < count(); ++g) {
            Engine &e = *groups_[g]->engine;
            const hzlb_config &c = e.config();
            saved[g].ensure(e.compact_size() * 2 * c.precision * static_cast<size_t>(e.members()),
                            "allocate tuning snapshot");
            e.get_state_compact(saved[g].ptr, 0, e.members());
            clocks[g] = {e.time, e.step_index};
        }
        for (int g = 0; g < count(); ++g)
            groups_[g]->engine->prepare_steps(dt[g]);
        // serial schedule
        set_schedule(true, std::vector<GroupCaps>(count()));
        const double serial = measure(dt, repeats);
        // concurrent schedule: coordinate descent over grid-cap fractions
        std::vector<GroupCaps> best(count());
        set_schedule(false, best);
        double best_ms = measure(dt, repeats);
        std::vector<int> order(count());
        for (int g = 0; g < count(); ++g)
            order[g] = g;
        std::sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
        const double fracs[] = {1.0, 0.75, 0.5, 0.25, 0.125};
        for (int pass = 0; pass < 2; ++pass)
            for (int g : order)
                for (double f : fracs) {
                    std::vector<GroupCaps> trial = best;
                    trial[g].col = std::max(1, static_cast<int>(std::lround(resident_[g].col * f)));
                    trial[g].row = std::max(1, static_cast<int>(std::lround(resident_[g].row * f)));
                    set_schedule(false, trial);
                    const double ms = measure(dt, repeats);
                    if (ms < best_ms) {
                        best_ms = ms;
                        best = trial;
                    }
                }
        // the row kernel's block shape per resolution, 64 or 128 threads (both compiled), the
        // grid cap carried over as the same fraction of that shape's resident blocks
        for (int g : order) {
            std::vector<GroupCaps> trial = best;
            const int cur = row_threads(g, best[g].row_threads), alt = cur == 64 ? 128 : 64;
            trial[g].row_threads = alt;
            if (best[g].row > 0)
                trial[g].row = std::max(1, static_cast<int>(std::lround(
                                               static_cast<double>(best[g].row) *
                                               row_resident(g, alt) / row_resident(g, cur))));
            set_schedule(false, trial);
            const double ms = measure(dt, repeats);
            if (ms < best_ms) {
                best_ms = ms;
                best = trial;
            }
        }
        // the fused kernels over the mixed work list, and with the 512^2 resolution on a branch
        // whose grid cap is searched too
        Mode best_mode = Mode::Concurrent;
        std::vector<GroupCaps> best_caps = best;
        GroupCaps best_fused{};
        tried_.clear();
        tried_.push_back({Mode::Serial, serial});
        tried_.push_back({Mode::Concurrent, best_ms});
        if (fusable()) {
            set_mode(Mode::Fused, std::vector<GroupCaps>(count()));
            const double f = measure(dt, repeats);
            tried_.push_back({Mode::Fused, f});
            if (f < best_ms) {
                best_ms = f;
                best_mode = Mode::Fused;
                best_caps = std::vector<GroupCaps>(count());
            }
            const int g5 = group_512();
            if (g5 >= 0) {
                // the branch's grid, then the fused kernels' grid, each as a fraction of its
                // resident blocks
                double fb_best = 0;
                std::vector<GroupCaps> fb_caps(count());
                GroupCaps fb_fused{};
                auto try_fb = [&](const std::vector<GroupCaps> &caps, GroupCaps fused) {
                    set_mode(Mode::FusedBranch, caps, fused);
                    const double ms = measure(dt, repeats);
                    if (fb_best == 0 || ms < fb_best) {
                        fb_best = ms;
                        fb_caps = caps;
                        fb_fused = fused;
                    }
                };
                for (double frac : {0.125, 0.25, 0.5, 1.0}) {
                    std::vector<GroupCaps> trial(count());
                    trial[g5].col = std::max(1, static_cast<int>(std::lround(resident_[g5].col * frac)));
                    trial[g5].row = std::max(1, static_cast<int>(std::lround(resident_[g5].row * frac)));
                    try_fb(trial, GroupCaps{});
                }
                const std::vector<GroupCaps> branch_caps = fb_caps;
                for (double frac : {0.9, 0.8, 0.7}) {
                    GroupCaps f;
                    f.col = std::max(1, static_cast<int>(std::lround(fused_resident_.col * frac)));
                    f.row = std::max(1, static_cast<int>(std::lround(fused_resident_.row * frac)));
                    try_fb(branch_caps, f);
                }
                tried_.push_back({Mode::FusedBranch, fb_best});
                if (fb_best < best_ms) {
                    best_ms = fb_best;
                    best_mode = Mode::FusedBranch;
                    best_caps = fb_caps;
                    best_fused = fb_fused;
                }
            }
        }
        if (serial <= best_ms) {
            set_mode(Mode::Serial, std::vector<GroupCaps>(count()));
            best_ms = serial;
        } else {
            set_mode(best_mode, best_caps, best_fused);
        }
        tuned_serial_ms_ = serial;
        for (int g = 0; g < count(); ++g) {
            Engine &e = *groups_[g]->engine;
            e.set_state_compact(saved[g].ptr, 0, e.members());
            e.set_time(clocks[g].first, clocks[g].second);
            e.synchronize();
            e.status();   // clears status bits raised while tuning
        }
        return best_ms;
    }
    void schedule(int *serial, int *col_caps, int *row_caps) const {
        if (serial)
            *serial = serial_ ? 1 : 0;
        for (int g = 0; g < count(); ++g) {
            if (col_caps)
                col_caps[g] = caps_[g].col ? caps_[g].col : resident_[g].col;
            if (row_caps)
                row_caps[g] = caps_[g].row ? caps_[g].row : resident_[g].row;
        }
    }
    // the row kernel block shape group g runs with `threads` (0: its default) resolves to
    int row_threads(int g, int threads) const {
        const hzlb_config &c = groups_[g]->engine->config();
        return c.precision == 4 ? row_block_threads<float>(c.n, threads)
                                : row_block_threads<double>(c.n, threads);
    }
    int row_threads(int g) const { return row_threads(g, caps_[g].row_threads); }
    void set_row_threads(const int *threads) {
        if (!threads)
            raise(HZLB_EINVAL, "null row block shapes");
        for (int g = 0; g < count(); ++g)
            if (threads[g] != 0 && threads[g] != 64 && threads[g] != 128)
                raise(HZLB_EINVAL, "row block shape must be 0 (default), 64 or 128 threads");
        for (int g = 0; g < count(); ++g)
            caps_[g].row_threads = threads[g];
        drop();
    }
    // resident blocks of group g's row kernel in blocks of `threads`
    int row_resident(int g, int threads) const {
        const hzlb_config &c = groups_[g]->engine->config();
        int col = 0, row = 0;
        cuda_check(c.precision == 4 ? resident_blocks<float>(c.n, &col, &row, threads)
                                    : resident_blocks<double>(c.n, &col, &row, threads),
                   "query resident blocks");
        return row > 0 ? row : 1;
    }
    void set_schedule(bool serial, const std::vector<GroupCaps> &caps) {
        set_mode(serial ? Mode::Serial : Mode::Concurrent, caps);
    }
    // caps: per group, used by the concurrent schedule and by the 512^2 branch of fused_branch
    // fused: the grid caps of the fused kernels (0: every resident block)
    void set_mode(Mode mode, const std::vector<GroupCaps> &caps, GroupCaps fused = GroupCaps{}) {
        fused_caps_ = fused;
        if ((mode == Mode::Fused || mode == Mode::FusedBranch) && !fusable())
            raise(HZLB_EINVAL, "fused schedules need FP32 resolutions among 64, 128, 256 and 512 "
                               "(one ensemble each, no device OU forcing)");
        if (mode == Mode::FusedBranch && group_512() < 0)
            raise(HZLB_EINVAL, "the fused schedule with a branch needs a 512^2 ensemble");
        if (mode == Mode::Fused || mode == Mode::FusedBranch) {
            int cres = 0, rres = 0;
            cuda_check(cudaSetDevice(device_), "select CUDA device");
            cuda_check(prepare_mixed(3, &cres, &rres), "configure mixed kernels");
            if (mode == Mode::Fused && group_512() >= 0)
                cuda_check(prepare_mixed(4, &cres, &rres), "configure mixed kernels");
            fused_resident_.col = cres;
            fused_resident_.row = rres;
        }
        mode_ = mode;
        serial_ = mode == Mode::Serial;
        caps_ = caps;
        drop();
    }
    Mode mode() const { return mode_; }

  private:
    struct Graph {
        std::vector<double> dt;
        int steps;
        cudaGraphExec_t exec;
    };
    void check_dt(const double *dt) const {
        if (!dt)
            raise(HZLB_EINVAL, "null time steps");
        for (int g = 0; g < count(); ++g)
            if (!std::isfinite(dt[g]) || dt[g] <= 0)
                raise(HZLB_EINVAL, "time steps must be positive and finite");
    }
    // bytes moved per step by a resolution (members x compact size), for the tuning order
    double work(int g) const {
        const hzlb_config &c = groups_[g]->engine->config();
        const int K = (c.n - 1) / 3;
        return static_cast<double>(c.members) * c.n * (K + 1) * c.precision;
    }
    void drop() {
        for (auto &g : graphs_)
            if (g.exec)
                cudaGraphExecDestroy(g.exec);
        graphs_.clear();
    }
    cudaGraphExec_t graph_for(const double *dt, int steps) {
        for (auto &g : graphs_)
            if (g.steps == steps && std::equal(g.dt.begin(), g.dt.end(), dt))
                return g.exec;
        // graphs are kept for the current time steps only (an adaptive caller changes them)
        if (!graphs_.empty() && !std::equal(graphs_.front().dt.begin(), graphs_.front().dt.end(), dt))
            drop();
        cudaGraph_t graph = nullptr;
        cuda_check(cudaStreamBeginCapture(main_, cudaStreamCaptureModeThreadLocal),
                   "begin mixed capture");
        try {
            if (mode_ == Mode::Fused) {
                enqueue_fused(dt, steps, main_, -1);
            } else if (mode_ == Mode::FusedBranch) {
                const int g5 = group_512();
                cuda_check(cudaEventRecord(fork_, main_), "fork");
                cuda_check(cudaStreamWaitEvent(branch_[g5], fork_, 0), "branch wait");
                groups_[g5]->engine->enqueue_steps_on(dt[g5], steps, branch_[g5], caps_[g5].col,
                                                      caps_[g5].row, caps_[g5].row_threads);
                cuda_check(cudaEventRecord(join_[g5], branch_[g5]), "join record");
                enqueue_fused(dt, steps, main_, g5);
                cuda_check(cudaStreamWaitEvent(main_, join_[g5], 0), "join wait");
            } else if (serial_) {
                for (int g = 0; g < count(); ++g)
                    groups_[g]->engine->enqueue_steps_on(dt[g], steps, main_, 0, 0,
                                                         caps_[g].row_threads);
            } else {
                cuda_check(cudaEventRecord(fork_, main_), "fork");
                for (int g = 0; g < count(); ++g) {
                    cuda_check(cudaStreamWaitEvent(branch_[g], fork_, 0), "branch wait");
                    groups_[g]->engine->enqueue_steps_on(dt[g], steps, branch_[g], caps_[g].col,
                                                         caps_[g].row, caps_[g].row_threads);
                    cuda_check(cudaEventRecord(join_[g], branch_[g]), "join record");
                    cuda_check(cudaStreamWaitEvent(main_, join_[g], 0), "join wait");
                }
            }
        } catch (...) {
            cudaStreamEndCapture(main_, &graph);
            if (graph)
                cudaGraphDestroy(graph);
            throw;
        }
        cuda_check(cudaStreamEndCapture(main_, &graph), "end mixed capture");
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        cuda_check(e, "instantiate mixed graph");
        graphs_.push_back({std::vector<double>(dt, dt + count()), steps, exec});
        return exec;
    }
    double measure(const double *dt, int repeats) {
        constexpr int kSteps = 8;
        cudaGraphExec_t exec = graph_for(dt, kSteps);
        cuda_check(cudaGraphLaunch(exec, main_), "warm-up mixed graph");
        cudaEvent_t a, b;
        cuda_check(cudaEventCreate(&a), "create event");
        cuda_check(cudaEventCreate(&b), "create event");
        cuda_check(cudaEventRecord(a, main_), "record");
        for (int i = 0; i < repeats; ++i)
            cuda_check(cudaGraphLaunch(exec, main_), "launch mixed graph");
        cuda_check(cudaEventRecord(b, main_), "record");
        cuda_check(cudaEventSynchronize(b), "time mixed graph");
        float ms = 0;
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        for (int g = 0; g < count(); ++g)
            groups_[g]->engine->finish_steps(dt[g], static_cast<uint64_t>(kSteps) * (repeats + 1));
        return ms / (static_cast<double>(repeats) * kSteps);
    }

    // ---- fused kernels over the mixed work list ------------------------------------
    // class of group g in the fused kernels (resolution 64 << class), or -1
    int class_of(int g) const {
        const int n = groups_[g]->engine->config().n;
        return n == 64 ? 0 : n == 128 ? 1 : n == 256 ? 2 : n == 512 ? 3 : -1;
    }
    // every group FP32 without device OU forcing, resolutions 64..512, one group per resolution
    bool fusable() const {
        if (count() > MIXED_CLASSES)
            return false;
        bool seen[MIXED_CLASSES] = {};
        for (int g = 0; g < count(); ++g) {
            const Engine &e = *groups_[g]->engine;
            const int c = class_of(g);
            if (c < 0 || seen[c] || e.config().precision != 4 || e.ou_enabled())
                return false;
            seen[c] = true;
        }
        return true;
    }
    int group_512() const {
        for (int g = 0; g < count(); ++g)
            if (class_of(g) == 3)
                return g;
        return -1;
    }
    // `steps` RK4 steps of every group except `skip` through the fused kernels on stream s
    void enqueue_fused(const double *dt, int steps, cudaStream_t s, int skip) {
        const int ccap = fused_caps_.col, rcap = fused_caps_.row;
        MixedRowArgs<float> ra{};
        MixedColumnArgs<float> ca{};
        std::array<double, MIXED_CLASSES> cfl{};
        int rtot = 0, ctot = 0, classes = 3;
        for (int g = 0; g < count(); ++g) {
            if (g == skip)
                continue;
            const int c = class_of(g), n = 64 << c;
            Engine &e = *groups_[g]->engine;
            e.stage_args(dt[g], &ca.cls[c], &ra.cls[c]);
            const KernelShape k = kernel_shape<float>(n);
            ra.items[c] = e.members() * (n / k.rows_per_block);
            ca.items[c] = e.members() * k.col_blocks_per_member;
            cfl[c] = dt[g] * n / (2 * 3.141592653589793238462643383279502884);
            if (c == 3)
                classes = 4;
        }
        // the work list in the kernels' processing order, largest resolution first
        for (int c = MIXED_CLASSES - 1; c >= 0; --c) {
            ra.offset[c] = rtot;
            ca.offset[c] = ctot;
            rtot += ra.items[c];
            ctot += ca.items[c];
        }
        for (int i = 0; i < steps; ++i)
            for (int st = 1; st <= 4; ++st) {
                for (int c = 0; c < MIXED_CLASSES; ++c)
                    ra.cls[c].cfl_scale = st == 1 ? cfl[c] : 0.0;
                cuda_check(launch_mixed_row(ra, classes, rtot, s, rcap), "launch mixed row pass");
                for (int c = 0; c < MIXED_CLASSES; ++c)
                    ca.cls[c].stage = st;
                cuda_check(launch_mixed_column(ca, st, classes, ctot, s, ccap),
                           "launch mixed column pass");
            }
    }

    int device_ = 0;
    Mode mode_ = Mode::Concurrent;
    GroupCaps fused_caps_, fused_resident_;   // grid cap of the fused kernels (0: all resident)
    std::vector<std::unique_ptr<hzlb_ensemble>> groups_;
    cudaStream_t main_ = nullptr;
    std::vector<cudaStream_t> branch_;
    std::vector<cudaEvent_t> join_;
    cudaEvent_t fork_ = nullptr;
    std::vector<GroupCaps> caps_, resident_;
    bool serial_ = false;
    double tuned_serial_ms_ = 0;
    std::vector<std::pair<Mode, double>> tried_;   // best ms per step of each schedule kind

  public:
    // the tuner's best time per step for each schedule kind it measured (ms; 0 if not measured)
    void tuned_times(double *out4) const {
        for (int i = 0; i < 4; ++i)
            out4[i] = 0;
        for (const auto &t : tried_)
            out4[static_cast<int>(t.first)] = t.second;
    }

  private:
    std::vector<Graph> graphs_;
};

} // namespace hzlb

struct hzlb_mixed {
    std::unique_ptr<hzlb::Mixed> mixed;
};

namespace {
template <class F> int guarded_mixed(F &&f) {
    try {
        f();
        return HZLB_OK;
    } catch (const hzlb::Error &e) {
        hzlb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception &e) {
        hzlb::set_last_error(e.what());
        return HZLB_ERUNTIME;
    }
}
hzlb::Mixed &mixed(hzlb_mixed *h) {
    if (!h || !h->mixed)
        hzlb::raise(HZLB_EINVAL, "null mixed handle");
    return *h->mixed;
}
} // namespace

extern "C" {
HZLB_API int hzlb_mixed_create(const hzlb_config *configs, int count, hzlb_mixed **out) {
    return guarded_mixed([&] {
        if (!out)
            hzlb::raise(HZLB_EINVAL, "null output");
        auto h = std::make_unique<hzlb_mixed>();
        h->mixed = std::make_unique<hzlb::Mixed>(configs, count);
        *out = h.release();
    });
}
HZLB_API void hzlb_mixed_destroy(hzlb_mixed *h) { delete h; }
HZLB_API hzlb_ensemble *hzlb_mixed_group(hzlb_mixed *h, int group) {
    return h && h->mixed ? h->mixed->group(group) : nullptr;
}
HZLB_API int hzlb_mixed_step(hzlb_mixed *h, const double *dt, uint64_t nsteps) {
    return guarded_mixed([&] { mixed(h).step(dt, nsteps); });
}
HZLB_API int hzlb_mixed_tune(hzlb_mixed *h, const double *dt, int repeats, double *ms_per_step) {
    return guarded_mixed([&] {
        const double ms = mixed(h).tune(dt, repeats);
        if (ms_per_step)
            *ms_per_step = ms;
    });
}
HZLB_API int hzlb_mixed_schedule(hzlb_mixed *h, int *serial, int *col_caps, int *row_caps) {
    return guarded_mixed([&] { mixed(h).schedule(serial, col_caps, row_caps); });
}
HZLB_API int hzlb_mixed_set_mode(hzlb_mixed *h, int mode, const int *col_caps,
                                 const int *row_caps) {
    return guarded_mixed([&] {
        auto &m = mixed(h);
        if (mode < 0 || mode > 3)
            hzlb::raise(HZLB_EINVAL, "mixed schedule mode must be 0..3");
        std::vector<hzlb::GroupCaps> caps(m.count());
        for (int g = 0; g < m.count(); ++g) {
            caps[g].col = col_caps ? std::max(0, col_caps[g]) : 0;
            caps[g].row = row_caps ? std::max(0, row_caps[g]) : 0;
        }
        m.set_mode(static_cast<hzlb::Mode>(mode), caps);
    });
}
HZLB_API int hzlb_mixed_row_threads(hzlb_mixed *h, int *threads) {
    return guarded_mixed([&] {
        auto &m = mixed(h);
        if (!threads)
            hzlb::raise(HZLB_EINVAL, "null output");
        for (int g = 0; g < m.count(); ++g)
            threads[g] = m.row_threads(g);
    });
}
HZLB_API int hzlb_mixed_set_row_threads(hzlb_mixed *h, const int *threads) {
    return guarded_mixed([&] { mixed(h).set_row_threads(threads); });
}
HZLB_API int hzlb_mixed_mode(hzlb_mixed *h, int *mode, double *tuned_ms) {
    return guarded_mixed([&] {
        auto &m = mixed(h);
        if (mode)
            *mode = static_cast<int>(m.mode());
        if (tuned_ms)
            m.tuned_times(tuned_ms);
    });
}
HZLB_API int hzlb_mixed_set_schedule(hzlb_mixed *h, int serial, const int *col_caps,
                                     const int *row_caps) {
    return guarded_mixed([&] {
        auto &m = mixed(h);
        std::vector<hzlb::GroupCaps> caps(m.count());
        for (int g = 0; g < m.count(); ++g) {
            caps[g].col = col_caps ? std::max(0, col_caps[g]) : 0;
            caps[g].row = row_caps ? std::max(0, row_caps[g]) : 0;
        }
        m.set_schedule(serial != 0, caps);
    });
}
} // extern "C"
