// Host-side declarations of the kernel launchers (implemented in launch.cu).
#pragma once
#include "spectral_step.cuh"

#include <cmath>
#include <vector>

namespace hzlb {

struct KernelShape {
    int col_threads, row_threads;
    int col_blocks_per_member, row_blocks_per_member;
    size_t col_smem, row_smem;
    int elements_per_thread, rows_per_block;
};

// The transform's twiddle table W_N^k = exp(-2 pi i k / N), k < N, built on the host in double
// precision as the reference builds its roots (std::polar, fft.cpp:25-27), then rounded to R.
template <typename R> std::vector<cx<R>> host_twiddles(int n) {
    std::vector<cx<R>> tw(n);
    for (int k = 0; k < n; ++k) {
        const double theta = -2.0 * 3.141592653589793238462643383279502884 * static_cast<double>(k) /
                             static_cast<double>(n);
        tw[k] = mk<R>(static_cast<R>(std::cos(theta)), static_cast<R>(std::sin(theta)));
    }
    return tw;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda);
// null when the driver does not provide it.
using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                 const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                 const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                 CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled tensor_map_encoder();

template <typename R> cudaError_t prepare_kernels(int n);
// cap > 0 limits the persistent grid to cap blocks (default: all resident blocks of the device)
template <typename R>
cudaError_t launch_column(int n, const ColumnArgs<R> &a, cudaStream_t s, int cap = 0);
// threads: the row kernel's block shape, 64 or 128 (0: the resolution's default,
// row_kernel_threads); both are compiled for every resolution
template <typename R>
cudaError_t launch_row(int n, const RowArgs<R> &a, cudaStream_t s, int cap = 0, int threads = 0);
// resident blocks of the column kernel and of the row kernel of that shape on the current
// device (after prepare_kernels)
template <typename R> cudaError_t resident_blocks(int n, int *column, int *row, int threads = 0);
// the block shape `threads` resolves to at resolution n (64 or 128)
template <typename R> int row_block_threads(int n, int threads);
template <typename R>
cudaError_t launch_physical(int n, const cx<R> *field, long long stride, cx<R> *cols, R *phys,
                            const cx<R> *tw, int members, cudaStream_t s);
template <typename R>
cudaError_t launch_velocity_max(int n, const cx<R> *w, unsigned long long *bits, const cx<R> *tw,
                                int members, cudaStream_t s);
template <typename R>
cudaError_t launch_diagnostics(int n, const cx<R> *omega, const cx<R> *forcing, long long fstride,
                               int fcols, int members, double *out, cudaStream_t s);
template <typename R>
cudaError_t launch_gather(const R *phys, int n, const unsigned *xs, const unsigned *ys, int p,
                          int members, double *out, cudaStream_t s);
// The physical rows of the listed row pairs at p points (the observation operator of a point
// set): column inverse transforms of every member, row transforms of the pairs only, gather.
template <typename R>
cudaError_t launch_observe_rows(int n, const cx<R> *field, long long stride, cx<R> *cols,
                                R *rows, const int *pairs, int npairs, const unsigned *xs,
                                const unsigned *slots, int p, const cx<R> *tw, int members,
                                double *out, cudaStream_t s);
template <typename R> KernelShape kernel_shape(int n);

// One persistent kernel per RK stage over a mixed-resolution work list (FP32, class c at
// resolution 64 << c): `classes` 3 (64..256) or 4 (64..512).  prepare_mixed sets the kernels'
// shared memory and returns their resident grids; the launchers take the total items of the
// pass (every class's items) for the grid's cap.
cudaError_t prepare_mixed(int classes, int *column_resident, int *row_resident);
cudaError_t launch_mixed_row(const MixedRowArgs<float> &a, int classes, int total_items,
                             cudaStream_t s, int cap = 0);
cudaError_t launch_mixed_column(const MixedColumnArgs<float> &a, int stage, int classes,
                                int total_items, cudaStream_t s, int cap = 0);

} // namespace hzlb
