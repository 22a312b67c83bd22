// Template instantiation and launch dispatch for the spectral kernels, N = 8..512, float and
// double.  Grids put members on x (no 65535 limit) and column blocks / row tiles on y.
#include "launch.h"
#include "physical.cuh"

#include <algorithm>
#include <mutex>

namespace hzlb {

EncodeTiled tensor_map_encoder() {
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}

namespace {

// The tensor map through which the row pass of resolution N stores a tile's product spectra
// (RowArgs::nlmap); nothing to do for resolutions that store them with plain stores.
template <typename R, int N, int RT = 128> cudaError_t row_store_map(RowArgs<R> &a) {
    using G = Cfg<R, N, RT>;
    if constexpr (!G::ROW_TMA) {
        return cudaSuccess;
    } else {
        constexpr cuuint32_t W = sizeof(cx<R>) / 4;   // 4-byte words per complex entry
        EncodeTiled fn = tensor_map_encoder();
        if (!fn || a.members < 1 || (reinterpret_cast<uintptr_t>(a.nl) & 15))
            return cudaErrorInvalidValue;
        const cuuint64_t dims[3] = {static_cast<cuuint64_t>(N) * W, 2 * G::C,
                                    static_cast<cuuint64_t>(a.members)};
        const cuuint64_t strides[2] = {static_cast<cuuint64_t>(N) * sizeof(cx<R>),
                                       static_cast<cuuint64_t>(2 * G::C) * N * sizeof(cx<R>)};
        const cuuint32_t box[3] = {static_cast<cuuint32_t>(G::TY) * W, 2 * G::C, 1};
        const cuuint32_t estr[3] = {1, 1, 1};
        const CUtensorMapSwizzle sw = G::ROW_SPAN == 32   ? CU_TENSOR_MAP_SWIZZLE_32B
                                      : G::ROW_SPAN == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                                          : CU_TENSOR_MAP_SWIZZLE_128B;
        return fn(&a.nlmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, a.nl, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS
                   ? cudaSuccess
                   : cudaErrorInvalidValue;
    }
}

// The standalone row kernel of resolution N in blocks of RT threads: shared memory, resident
// grid per device, launch.
template <typename R, int N, int RT> struct RowShape {
    using GR = Cfg<R, N, RT>;
    static constexpr size_t smem = hzlb::row_smem<R, N, RT>();
    static_assert(smem <= 227 * 1024, "row kernel shared memory");
    static inline int resident[64] = {};
    static cudaError_t prepare(int dev, int sms) {
        cudaError_t e = cudaFuncSetAttribute(row_kernel<R, N, RT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        int rb = 0;
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rb, row_kernel<R, N, RT>,
                                                              GR::ROW_THREADS, smem);
        if (e == cudaSuccess && rb < 1)
            e = cudaErrorInvalidConfiguration;
        if (e == cudaSuccess && dev >= 0 && dev < 64)
            resident[dev] = rb * sms;
        return e;
    }
    static int resident_blocks() {
        int dev = 0;
        cudaGetDevice(&dev);
        return dev >= 0 && dev < 64 && resident[dev] > 0 ? resident[dev] : 148;
    }
    static cudaError_t run(const RowArgs<R> &args, cudaStream_t s, int cap) {
        RowArgs<R> a = args;
        if (cudaError_t e = row_store_map<R, N, RT>(a))
            return e;
        const int items = a.members * (N / GR::TY);
        const int res = resident_blocks();
        const int grid = std::min(items, cap > 0 ? std::min(cap, res) : res);
        row_kernel<R, N, RT><<<grid, GR::ROW_THREADS, smem, s>>>(a, items);
        return cudaGetLastError();
    }
};

template <typename R, int N> struct L {
    using G = Cfg<R, N>;
    static constexpr size_t col_smem = hzlb::column_smem<R, N>();
    // the standalone row kernel's default block shape (RT threads)
    static constexpr int RT = row_kernel_threads<R, N>();
    static constexpr size_t prow_smem = sizeof(cx<R>) * (G::TWE + G::GROUPS * G::BUF);
    static constexpr size_t pcol_smem = sizeof(cx<R>) * (G::TWE + G::LPB * G::BUF);
    // persistent grid of the column pass: resident blocks per SM x SMs, per device
    static inline int col_resident[64] = {};
    // one column kernel per RK stage
    static constexpr void (*col_kernels[5])(const ColumnArgs<R>, int) = {
        column_kernel<R, N, 0>, column_kernel<R, N, 1>, column_kernel<R, N, 2>,
        column_kernel<R, N, 3>, column_kernel<R, N, 4>};
    static cudaError_t prepare() {
        cudaError_t e = cudaSuccess;
        for (int st = 0; st < 5 && e == cudaSuccess; ++st)
            e = cudaFuncSetAttribute(col_kernels[st], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(col_smem));
        int dev = 0, sms = 0, cb = 0;
        if (e == cudaSuccess)
            e = cudaGetDevice(&dev);
        if (e == cudaSuccess)
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        // persistent grid of the column pass: the fewest resident blocks over the stages
        cb = 1 << 30;
        for (int st = 0; st < 5 && e == cudaSuccess; ++st) {
            int b = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, col_kernels[st], G::COL_THREADS,
                                                              col_smem);
            cb = std::min(cb, b);
        }
        if (e == cudaSuccess && cb < 1)
            e = cudaErrorInvalidConfiguration;
        if (e == cudaSuccess && dev < 64)
            col_resident[dev] = cb * sms;
        if (e == cudaSuccess)
            e = RowShape<R, N, 64>::prepare(dev, sms);
        if (e == cudaSuccess)
            e = RowShape<R, N, 128>::prepare(dev, sms);
        return e;
    }
    static int resident(const int *table) {
        int dev = 0;
        cudaGetDevice(&dev);
        return dev < 64 && table[dev] > 0 ? table[dev] : 148;
    }
    static dim3 col_grid(int members) { return dim3(members, (G::C + G::LPB - 1) / G::LPB); }
    static dim3 row_grid(int members) { return dim3(members, N / G::TY); }
    static cudaError_t column(const ColumnArgs<R> &a, cudaStream_t s, int cap) {
        const int items = a.members * G::NCG;
        const int res = resident(col_resident);
        const int grid = std::min(items, cap > 0 ? std::min(cap, res) : res);
        if (a.stage < 0 || a.stage > 4)
            return cudaErrorInvalidValue;
        col_kernels[a.stage]<<<grid, G::COL_THREADS, col_smem, s>>>(a, items);
        return cudaGetLastError();
    }
    // threads: 64 or 128 (0: the default shape)
    static int row_threads(int threads) { return threads == 64 || threads == 128 ? threads : RT; }
    static cudaError_t row(const RowArgs<R> &args, cudaStream_t s, int cap, int threads) {
        return row_threads(threads) == 64 ? RowShape<R, N, 64>::run(args, s, cap)
                                          : RowShape<R, N, 128>::run(args, s, cap);
    }
    static int row_resident(int threads) {
        return row_threads(threads) == 64 ? RowShape<R, N, 64>::resident_blocks()
                                          : RowShape<R, N, 128>::resident_blocks();
    }
    static cudaError_t physical(const cx<R> *field, long long stride, cx<R> *cols, R *phys,
                                const cx<R> *tw, int members, cudaStream_t s) {
        field_column_inverse<R, N><<<col_grid(members), G::COL_THREADS, pcol_smem, s>>>(
            field, stride, cols, tw);
        field_row_inverse<R, N><<<row_grid(members), G::ROW_THREADS, prow_smem, s>>>(cols, phys, tw);
        return cudaGetLastError();
    }
    static cudaError_t observe_rows(const cx<R> *field, long long stride, cx<R> *cols, R *rows,
                                    const int *pairs, int npairs, const cx<R> *tw, int members,
                                    cudaStream_t s) {
        field_column_inverse<R, N><<<col_grid(members), G::COL_THREADS, pcol_smem, s>>>(
            field, stride, cols, tw);
        const dim3 grid(members, (npairs + G::TY / 2 - 1) / (G::TY / 2));
        field_row_pairs_inverse<R, N><<<grid, G::ROW_THREADS, prow_smem, s>>>(cols, pairs, npairs,
                                                                              rows, tw);
        return cudaGetLastError();
    }
    static cudaError_t vmax(const cx<R> *w, unsigned long long *bits, const cx<R> *tw, int members,
                            cudaStream_t s) {
        velocity_max<R, N><<<row_grid(members), G::ROW_THREADS, prow_smem, s>>>(w, bits, tw);
        return cudaGetLastError();
    }
    static void shape(KernelShape &k) {
        k.col_threads = G::COL_THREADS;
        k.row_threads = G::ROW_THREADS;
        k.col_blocks_per_member = (G::C + G::LPB - 1) / G::LPB;
        k.row_blocks_per_member = N / G::TY;
        k.col_smem = col_smem;
        k.row_smem = hzlb::row_smem<R, N>();
        k.elements_per_thread = G::E;
        k.rows_per_block = G::TY;
    }
};

template <typename R, template <typename, int> class F, typename... A>
cudaError_t dispatch(int n, A &&...args) {
    switch (n) {
    case 8: return F<R, 8>::run(args...);
    case 16: return F<R, 16>::run(args...);
    case 32: return F<R, 32>::run(args...);
    case 64: return F<R, 64>::run(args...);
    case 128: return F<R, 128>::run(args...);
    case 256: return F<R, 256>::run(args...);
    case 512: return F<R, 512>::run(args...);
    default: return cudaErrorInvalidValue;
    }
}
template <typename R, int N> struct DoPrepare {
    static cudaError_t run() { return L<R, N>::prepare(); }
};
template <typename R, int N> struct DoColumn {
    static cudaError_t run(const ColumnArgs<R> &a, cudaStream_t s, int cap) {
        return L<R, N>::column(a, s, cap);
    }
};
template <typename R, int N> struct DoRow {
    static cudaError_t run(const RowArgs<R> &a, cudaStream_t s, int cap, int threads) {
        return L<R, N>::row(a, s, cap, threads);
    }
};
template <typename R, int N> struct DoResident {
    static cudaError_t run(int *c, int *r, int threads) {
        *c = L<R, N>::resident(L<R, N>::col_resident);
        *r = L<R, N>::row_resident(threads);
        return cudaSuccess;
    }
};
template <typename R, int N> struct DoRowShape {
    static cudaError_t run(int threads, int *out) {
        *out = L<R, N>::row_threads(threads);
        return cudaSuccess;
    }
};
template <typename R, int N> struct DoPhysical {
    static cudaError_t run(const cx<R> *f, long long st, cx<R> *c, R *p, const cx<R> *tw, int m,
                           cudaStream_t s) {
        return L<R, N>::physical(f, st, c, p, tw, m, s);
    }
};
template <typename R, int N> struct DoObserveRows {
    static cudaError_t run(const cx<R> *f, long long st, cx<R> *c, R *rows, const int *pairs,
                           int npairs, const cx<R> *tw, int m, cudaStream_t s) {
        return L<R, N>::observe_rows(f, st, c, rows, pairs, npairs, tw, m, s);
    }
};
template <typename R, int N> struct DoVmax {
    static cudaError_t run(const cx<R> *w, unsigned long long *b, const cx<R> *tw, int m,
                           cudaStream_t s) {
        return L<R, N>::vmax(w, b, tw, m, s);
    }
};
template <typename R, int N> struct DoShape {
    static cudaError_t run(KernelShape &k) {
        L<R, N>::shape(k);
        return cudaSuccess;
    }
};
} // namespace

template <typename R> cudaError_t prepare_kernels(int n) { return dispatch<R, DoPrepare>(n); }
template <typename R>
cudaError_t launch_column(int n, const ColumnArgs<R> &a, cudaStream_t s, int cap) {
    return dispatch<R, DoColumn>(n, a, s, cap);
}
template <typename R>
cudaError_t launch_row(int n, const RowArgs<R> &a, cudaStream_t s, int cap, int threads) {
    return dispatch<R, DoRow>(n, a, s, cap, threads);
}
template <typename R> cudaError_t resident_blocks(int n, int *column, int *row, int threads) {
    return dispatch<R, DoResident>(n, column, row, threads);
}
template <typename R> int row_block_threads(int n, int threads) {
    int out = 0;
    return dispatch<R, DoRowShape>(n, threads, &out) == cudaSuccess ? out : 0;
}
template <typename R>
cudaError_t launch_physical(int n, const cx<R> *field, long long stride, cx<R> *cols, R *phys,
                            const cx<R> *tw, int members, cudaStream_t s) {
    return dispatch<R, DoPhysical>(n, field, stride, cols, phys, tw, members, s);
}
template <typename R>
cudaError_t launch_velocity_max(int n, const cx<R> *w, unsigned long long *bits, const cx<R> *tw,
                                int members, cudaStream_t s) {
    return dispatch<R, DoVmax>(n, w, bits, tw, members, s);
}
template <typename R>
cudaError_t launch_diagnostics(int n, const cx<R> *omega, const cx<R> *forcing, long long fstride,
                               int fcols, int members, double *out, cudaStream_t s) {
    integral_diagnostics<R><<<members, 256, 0, s>>>(omega, forcing, fstride, fcols, n, out);
    return cudaGetLastError();
}
template <typename R>
cudaError_t launch_gather(const R *phys, int n, const unsigned *xs, const unsigned *ys, int p,
                          int members, double *out, cudaStream_t s) {
    const long long total = static_cast<long long>(members) * p;
    if (total == 0)
        return cudaSuccess;
    gather_points<R><<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(phys, n, xs, ys, p,
                                                                              members, out);
    return cudaGetLastError();
}
template <typename R>
cudaError_t launch_observe_rows(int n, const cx<R> *field, long long stride, cx<R> *cols,
                                R *rows, const int *pairs, int npairs, const unsigned *xs,
                                const unsigned *slots, int p, const cx<R> *tw, int members,
                                double *out, cudaStream_t s) {
    if (npairs <= 0 || p <= 0)
        return cudaSuccess;
    cudaError_t e = dispatch<R, DoObserveRows>(n, field, stride, cols, rows, pairs, npairs, tw,
                                               members, s);
    if (e != cudaSuccess)
        return e;
    const long long total = static_cast<long long>(members) * p;
    gather_rows<R><<<static_cast<unsigned>((total + 255) / 256), 256, 0, s>>>(
        rows, 2 * npairs, n, xs, slots, p, members, out);
    return cudaGetLastError();
}
template <typename R> KernelShape kernel_shape(int n) {
    KernelShape k{};
    dispatch<R, DoShape>(n, k);
    return k;
}

#define HZLB_INSTANTIATE(R)                                                                        \
    template cudaError_t prepare_kernels<R>(int);                                                  \
    template cudaError_t launch_column<R>(int, const ColumnArgs<R> &, cudaStream_t, int);          \
    template cudaError_t launch_row<R>(int, const RowArgs<R> &, cudaStream_t, int, int);           \
    template cudaError_t resident_blocks<R>(int, int *, int *, int);                               \
    template int row_block_threads<R>(int, int);                                                   \
    template cudaError_t launch_physical<R>(int, const cx<R> *, long long, cx<R> *, R *,          \
                                            const cx<R> *, int, cudaStream_t);                     \
    template cudaError_t launch_velocity_max<R>(int, const cx<R> *, unsigned long long *,         \
                                                const cx<R> *, int, cudaStream_t);                 \
    template cudaError_t launch_diagnostics<R>(int, const cx<R> *, const cx<R> *, long long, int, \
                                               int, double *, cudaStream_t);                       \
    template cudaError_t launch_gather<R>(const R *, int, const unsigned *, const unsigned *, int, \
                                          int, double *, cudaStream_t);                            \
    template cudaError_t launch_observe_rows<R>(int, const cx<R> *, long long, cx<R> *, R *,       \
                                                const int *, int, const unsigned *,                \
                                                const unsigned *, int, const cx<R> *, int,         \
                                                double *, cudaStream_t);                           \
    template KernelShape kernel_shape<R>(int);
HZLB_INSTANTIATE(float)
HZLB_INSTANTIATE(double)

} // namespace hzlb

// ---- mixed-resolution kernels ----------------------------------------------------------
namespace hzlb {
namespace {
// The fused kernels of a pack of resolutions: shared memory is the largest over the pack;
// CMINB column blocks per SM (6, or 5 with 512^2 in the pack, whose 40.2 KB per block allow
// no more) bound the registers of the column kernel; the row kernel keeps 6 blocks.
template <int CMINB, int... Ns> struct MixedL {
    static constexpr size_t row_smem = std::max({hzlb::row_smem<float, Ns>()...});
    static constexpr size_t col_smem = std::max({hzlb::column_smem<float, Ns>()...});
    static inline int row_res[64] = {}, col_res[64] = {};
    static constexpr void (*cols[5])(const MixedColumnArgs<float>) = {
        mixed_column_kernel<float, 0, CMINB, Ns...>, mixed_column_kernel<float, 1, CMINB, Ns...>,
        mixed_column_kernel<float, 2, CMINB, Ns...>, mixed_column_kernel<float, 3, CMINB, Ns...>,
        mixed_column_kernel<float, 4, CMINB, Ns...>};
    static constexpr void (*rowk)(const MixedRowArgs<float>) = mixed_row_kernel<float, 6, Ns...>;
    static cudaError_t prepare(int *cres, int *rres) {
        cudaError_t e = cudaSuccess;
        for (int st = 0; st < 5 && e == cudaSuccess; ++st)
            e = cudaFuncSetAttribute(cols[st], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(col_smem));
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(rowk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     static_cast<int>(row_smem));
        int dev = 0, sms = 0, cb = 1 << 30, rb = 0;
        if (e == cudaSuccess)
            e = cudaGetDevice(&dev);
        if (e == cudaSuccess)
            e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        for (int st = 0; st < 5 && e == cudaSuccess; ++st) {
            int b = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, cols[st], 64, col_smem);
            cb = std::min(cb, b);
        }
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rb, rowk, 128, row_smem);
        if (e == cudaSuccess && (cb < 1 || rb < 1))
            e = cudaErrorInvalidConfiguration;
        if (e == cudaSuccess && dev >= 0 && dev < 64) {
            col_res[dev] = cb * sms;
            row_res[dev] = rb * sms;
        }
        if (cres)
            *cres = cb * sms;
        if (rres)
            *rres = rb * sms;
        return e;
    }
    static int resident(const int *table) {
        int dev = 0;
        cudaGetDevice(&dev);
        return dev >= 0 && dev < 64 && table[dev] > 0 ? table[dev] : 148;
    }
    static cudaError_t row(const MixedRowArgs<float> &args, int total, cudaStream_t s, int cap) {
        MixedRowArgs<float> a = args;
        cudaError_t e = cudaSuccess;
        ((e = e == cudaSuccess && a.items[mixed_class(Ns)] > 0
                  ? row_store_map<float, Ns>(a.cls[mixed_class(Ns)])
                  : e),
         ...);
        if (e != cudaSuccess)
            return e;
        const int res = cap > 0 ? std::min(cap, resident(row_res)) : resident(row_res);
        const int grid = std::max(1, std::min(total, res));
        rowk<<<grid, 128, row_smem, s>>>(a);
        return cudaGetLastError();
    }
    static cudaError_t column(const MixedColumnArgs<float> &a, int stage, int total, cudaStream_t s,
                              int cap) {
        if (stage < 0 || stage > 4)
            return cudaErrorInvalidValue;
        const int res = cap > 0 ? std::min(cap, resident(col_res)) : resident(col_res);
        const int grid = std::max(1, std::min(total, res));
        cols[stage]<<<grid, 64, col_smem, s>>>(a);
        return cudaGetLastError();
    }
};
using Mixed3 = MixedL<6, 256, 128, 64>;
using Mixed4 = MixedL<5, 512, 256, 128, 64>;
} // namespace

cudaError_t prepare_mixed(int classes, int *column_resident, int *row_resident) {
    if (classes == 3)
        return Mixed3::prepare(column_resident, row_resident);
    if (classes == 4)
        return Mixed4::prepare(column_resident, row_resident);
    return cudaErrorInvalidValue;
}
cudaError_t launch_mixed_row(const MixedRowArgs<float> &a, int classes, int total_items,
                             cudaStream_t s, int cap) {
    if (classes == 3)
        return Mixed3::row(a, total_items, s, cap);
    if (classes == 4)
        return Mixed4::row(a, total_items, s, cap);
    return cudaErrorInvalidValue;
}
cudaError_t launch_mixed_column(const MixedColumnArgs<float> &a, int stage, int classes,
                                int total_items, cudaStream_t s, int cap) {
    if (classes == 3)
        return Mixed3::column(a, stage, total_items, s, cap);
    if (classes == 4)
        return Mixed4::column(a, stage, total_items, s, cap);
    return cudaErrorInvalidValue;
}
} // namespace hzlb
