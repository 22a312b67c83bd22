// Observation dataset files in the reference's formats, HZL_OBSERVATIONS_V2 (written) and
// HZL_OBSERVATIONS_V1/V2 (read): the behaviour of hzl::Dataset::validate, save and load
// (src/inference.cpp:197-257).  Host code only; the files are byte-identical with the
// reference's because the same standard-stream formatting (17 significant digits) and the same
// whitespace-token parsing are used, and the same checks raise the same errors
// (std::invalid_argument -> HZLB_EINVAL, std::runtime_error -> HZLB_ERUNTIME).
#include "engine.h"

#include <algorithm>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

namespace hzlb {
namespace {

struct DatasetRecord {
    size_t n = 16;
    double dt = 0.01;
    bool stochastic = false;
    int forcing_min = 2, forcing_max = 3;
    std::vector<hzlb_observation> observations;
};

bool power_of_two(size_t n) { return n && !(n & (n - 1)); }

// Dataset::validate (src/inference.cpp:197-213): the grid of the spectral transform, the forcing
// shell inside the dealiased band, then the dataset itself.
void validate(const DatasetRecord &d) {
    if (d.n < 8 || d.n > 4096 || !power_of_two(d.n))
        raise(HZLB_EINVAL, "grid must be a power of two between 8 and 4096");
    if (d.forcing_min < 1 || d.forcing_max < d.forcing_min ||
        3 * static_cast<long long>(d.forcing_max) >= static_cast<long long>(d.n))
        raise(HZLB_EINVAL, "forcing shell must lie strictly inside the dealiased grid");
    if (d.n < 16 || !std::isfinite(d.dt) || d.dt <= 0 || d.observations.empty())
        raise(HZLB_EINVAL, "invalid observation dataset");
    uint64_t previous = 0;
    for (const auto &o : d.observations) {
        if (o.step < previous || o.x >= d.n || o.y >= d.n || !std::isfinite(o.value) ||
            !std::isfinite(o.standard_deviation) || o.standard_deviation <= 0)
            raise(HZLB_EINVAL, "observations must be time ordered, finite, in bounds, and "
                               "have positive uncertainty");
        previous = o.step;
    }
}

DatasetRecord from_c(const hzlb_dataset *d) {
    if (!d || (d->count && !d->observations))
        raise(HZLB_EINVAL, "invalid observation dataset");
    if (d->n < 0)
        raise(HZLB_EINVAL, "grid must be a power of two between 8 and 4096");
    DatasetRecord r;
    r.n = static_cast<size_t>(d->n);
    r.dt = d->dt;
    r.stochastic = d->stochastic != 0;
    r.forcing_min = d->forcing_min;
    r.forcing_max = d->forcing_max;
    r.observations.assign(d->observations, d->observations + d->count);
    return r;
}

// Dataset::save (src/inference.cpp:214-226)
void save(const DatasetRecord &d, const std::string &path) {
    validate(d);
    std::ofstream out(path);
    out << std::setprecision(17);
    out << "HZL_OBSERVATIONS_V2," << d.n << ',' << d.dt << ',' << d.stochastic << ','
        << d.forcing_min << ',' << d.forcing_max << "\nstep,x,y,vorticity,standard_deviation\n";
    for (const auto &o : d.observations)
        out << o.step << ',' << o.x << ',' << o.y << ',' << o.value << ',' << o.standard_deviation
            << '\n';
    if (!out)
        raise(HZLB_ERUNTIME, "observation write failed");
}

// Dataset::load (src/inference.cpp:227-257): comma-separated fields read as whitespace tokens,
// a V1 header carrying n and dt only (deterministic data, forcing shell 2..3).
DatasetRecord load(const std::string &path) {
    std::ifstream in(path);
    std::string line, magic;
    DatasetRecord d;
    if (!std::getline(in, line))
        raise(HZLB_ERUNTIME, "cannot read observation dataset");
    std::replace(line.begin(), line.end(), ',', ' ');
    std::istringstream header(line);
    if (!(header >> magic >> d.n >> d.dt) ||
        (magic != "HZL_OBSERVATIONS_V1" && magic != "HZL_OBSERVATIONS_V2"))
        raise(HZLB_ERUNTIME, "invalid dataset header");
    if (magic == "HZL_OBSERVATIONS_V2" &&
        !(header >> d.stochastic >> d.forcing_min >> d.forcing_max))
        raise(HZLB_ERUNTIME, "invalid stochastic dataset metadata");
    if (!std::getline(in, line) || line != "step,x,y,vorticity,standard_deviation")
        raise(HZLB_ERUNTIME, "invalid dataset columns");
    while (std::getline(in, line)) {
        if (line.empty())
            continue;
        std::replace(line.begin(), line.end(), ',', ' ');
        std::istringstream row(line);
        size_t step = 0, x = 0, y = 0;
        double value = 0, sd = 0;
        std::string extra;
        if (!(row >> step >> x >> y >> value >> sd) || (row >> extra))
            raise(HZLB_ERUNTIME, "invalid observation row");
        // positions beyond the grid fail validation below; keep them out of range when narrowed
        const uint32_t xs = x > 0xFFFFFFFFu ? 0xFFFFFFFFu : static_cast<uint32_t>(x);
        const uint32_t ys = y > 0xFFFFFFFFu ? 0xFFFFFFFFu : static_cast<uint32_t>(y);
        d.observations.push_back({static_cast<uint64_t>(step), xs, ys, value, sd});
    }
    validate(d);
    return d;
}

thread_local std::string dataset_error;
template <class F> int guarded(F &&f) {
    try {
        f();
        return HZLB_OK;
    } catch (const Error &e) {
        dataset_error = e.what();
        set_last_error(dataset_error);
        return e.code;
    } catch (const std::exception &e) {
        dataset_error = e.what();
        set_last_error(dataset_error);
        return HZLB_ERUNTIME;
    }
}

} // namespace
} // namespace hzlb

using namespace hzlb;

extern "C" {

HZLB_API int hzlb_dataset_save(const hzlb_dataset *data, const char *path) {
    return guarded([&] {
        if (!path)
            raise(HZLB_EINVAL, "null path");
        save(from_c(data), path);
    });
}

HZLB_API int hzlb_dataset_validate(const hzlb_dataset *data) {
    return guarded([&] { validate(from_c(data)); });
}

HZLB_API int hzlb_dataset_load(const char *path, hzlb_dataset *header,
                               hzlb_observation *observations, size_t capacity, size_t *count) {
    return guarded([&] {
        if (!path || !header || !count)
            raise(HZLB_EINVAL, "null argument");
        const DatasetRecord d = load(path);
        *count = d.observations.size();
        if (observations && capacity < d.observations.size())
            raise(HZLB_EINVAL, "observation buffer too small");
        header->n = static_cast<int>(d.n);
        header->dt = d.dt;
        header->stochastic = d.stochastic ? 1 : 0;
        header->forcing_min = d.forcing_min;
        header->forcing_max = d.forcing_max;
        header->count = observations ? d.observations.size() : 0;
        header->observations = observations;
        if (observations)
            std::copy(d.observations.begin(), d.observations.end(), observations);
    });
}

} // extern "C"
