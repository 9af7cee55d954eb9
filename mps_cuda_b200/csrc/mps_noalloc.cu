// mps_noalloc.cu -- bucket build that allocates nothing (mps_bucket_build_noalloc).
//
// Some callers cannot allocate device memory at the point where they need the buckets:
// code running inside another framework's memory pool (the pool owns every byte of the
// device and a cudaMalloc behind its back can fail or fragment it), real-time loops that
// must not allocate after start-up, and plug-ins handed only input and output buffers by
// their host. This entry point gives them MkBkt (kernel.cu:516-550) with every temporary
// -- bucket counters, per-item ranks, bucket segments and scan partials -- kept in one
// file-scope __device__ array of fixed size instead of memory allocated per call.
//
// Limits and sharing:
//   * at most MPS_NOALLOC_MAX_ITEMS particles and MPS_NOALLOC_MAX_BUCKETS buckets (the
//     array is about 21 MB and every GPU that loads the library holds it until exit);
//   * every call on a device uses the same array, so calls whose work overlaps on that
//     GPU (different streams, or different host threads) race and corrupt each other's
//     results; serialise them on one stream;
//   * the array keeps the previous call's contents; each call clears the counters it
//     needs before using them;
//   * the first call on a device looks up the array's device address there
//     (cudaGetSymbolAddress); make that first call before any stream capture. The address
//     is kept per device ordinal for the life of the process: after a cudaDeviceReset the
//     library's module is loaded again in the new context and the kept address no longer
//     names the array, so a process that resets a device must not call this entry point
//     on that device afterwards;
//   * like the reference's cell index (kernel.cu:521-524), a particle outside the bucket
//     grid gets the nearest edge bucket: cell_of clamps its coordinates. Nothing reports
//     that here (the solver counts such particles in err_cell_range); a caller whose
//     particles may leave the domain checks their positions itself.
#include <mutex>

#include "mps_solver.cuh"

namespace mps {
namespace {

constexpr size_t kScratchInts =
    3 * size_t(MPS_NOALLOC_MAX_ITEMS) + 2 * (size_t(MPS_NOALLOC_MAX_BUCKETS) + 2) +
    (size_t(MPS_NOALLOC_MAX_BUCKETS) + 1) / kScanTile + 2;

// the scratch: [key | rnk | seg | count | cs | partials]
__device__ __align__(256) int g_scratch[kScratchInts];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int* g_addr[kMaxDevices] = {};

// host-side address of g_scratch on the current device; a failing CUDA call's error is
// returned in *err (it is consumed here and cannot be read again with cudaGetLastError)
int scratch_on_current_device(int* dev_out, int** out, cudaError_t* err) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *err = e;
        return MPS_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return MPS_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) {
            *err = e != cudaSuccess ? e : cudaErrorInvalidSymbol;
            return MPS_ERR_CUDA;
        }
        g_addr[dev] = static_cast<int*>(p);
    }
    *dev_out = dev;
    *out = g_addr[dev];
    return MPS_OK;
}

template <class R> struct SoaKeySrc {
    SceneDev<R, R> sc;  // by value: no device copy of the scene constants is needed
    int n, dead;
    const int8_t* typ;
    const R* pos;  // SoA x[n], y[n], z[n]
    __device__ __forceinline__ int key(int t, DevCounters* cnt) const {
        if (typ[t] == kGST) return dead;
        int ix, iy, iz;
        cell_of(sc, pos[t], pos[size_t(n) + t], pos[2 * size_t(n) + t], ix, iy, iz);
        return iz * sc.nbxy + iy * sc.nbx + ix;
    }
    __device__ __forceinline__ int id(int t) const { return t; }
};

struct OrderGather {
    const int* key;
    int dead;
    int* order;
    int* cell;
    __device__ __forceinline__ void operator()(int t, int d) const {
        int c = key[t];
        cell[t] = c == dead ? -1 : c;
        if (c != dead) order[d] = t;
    }
};

__global__ void k_zero(int* p, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0;
}

__global__ void k_copy_starts(const int* cs, int nb, int* start) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= nb; i += gridDim.x * blockDim.x)
        start[i] = cs[i];
}

template <class R>
int run(const mps_params& p, int n, const int8_t* typ, const void* pos, int32_t* cell,
        int32_t* order, int32_t* start, cudaStream_t st, cudaError_t* err) {
    SceneDev<R, R> sc;
    mps_info inf;
    try {
        derive_scene<R, R>(p, 0, 0, 0, n, sc, inf);  // host only: checks the grid's size
    } catch (const ApiError& e) {
        return e.code;
    }
    const int C = inf.nbxyz;
    if (C > MPS_NOALLOC_MAX_BUCKETS) return MPS_ERR_OVERFLOW;
    int dev = 0, *base = nullptr;
    int rc = scratch_on_current_device(&dev, &base, err);
    if (rc) return rc;
    const int L = C + 1;  // buckets + the bucket of GST particles
    int* key = base;
    int* rnk = key + MPS_NOALLOC_MAX_ITEMS;
    int* seg = rnk + MPS_NOALLOC_MAX_ITEMS;
    int* count = seg + MPS_NOALLOC_MAX_ITEMS;
    int* cs = count + (MPS_NOALLOC_MAX_BUCKETS + 2);
    int* part = cs + (MPS_NOALLOC_MAX_BUCKETS + 2);
    SoaKeySrc<R> src{sc, n, C, typ, static_cast<const R*>(pos)};
    OrderGather g{key, C, order, cell};
    const int gi = std::max(1, std::min((n + 255) / 256, 148 * 32));
    const int gc = std::max(1, std::min((L + 255) / 256, 148 * 8));
    const int nb = (L + kScanTile - 1) / kScanTile;
    // counters start at zero: the array still holds the previous call's values
    k_zero<<<gc, 256, 0, st>>>(count, L);
    if (n > 0) k_bin_key<SoaKeySrc<R>><<<gi, 256, 0, st>>>(src, nullptr, n, key, rnk, count, nullptr, nullptr);
    k_scan_reduce<<<nb, kScanThreads, 0, st>>>(count, L, part);
    k_scan_apply<<<nb, kScanThreads, 0, st>>>(count, L, part, cs);
    if (n > 0) {
        k_bin_seg<SoaKeySrc<R>><<<gi, 256, 0, st>>>(src, nullptr, n, key, rnk, cs, seg);
        k_bin_fin<SoaKeySrc<R>, OrderGather><<<gi, 256, 0, st>>>(src, g, nullptr, n, key, rnk, cs,
                                                                  seg, C);
    }
    k_copy_starts<<<gc, 256, 0, st>>>(cs, C, start);
    *err = cudaGetLastError();
    return *err == cudaSuccess ? MPS_OK : MPS_ERR_CUDA;
}

}  // namespace
}  // namespace mps

extern "C" int mps_bucket_build_noalloc(const mps_params* p, int32_t n, const int8_t* typ,
                                        const void* pos, int32_t* cell, int32_t* order,
                                        int32_t* start, void* stream) {
    if (!p || n < 0 || (n > 0 && (!typ || !pos || !cell || !order)) || !start) {
        mps::g_last_error = "mps_bucket_build_noalloc: null argument or negative count";
        return MPS_ERR_ARG;
    }
    // The size checks stay ahead of every device access: a caller may pass buffers that
    // were sized for the limit, and a size beyond it must fail before any kernel or copy
    // touches them.
    if (n > MPS_NOALLOC_MAX_ITEMS) {
        mps::g_last_error = "mps_bucket_build_noalloc: more than MPS_NOALLOC_MAX_ITEMS particles";
        return MPS_ERR_OVERFLOW;
    }
    bool domain_ok = true;
    for (int d = 0; d < 3; ++d) domain_ok = domain_ok && p->max[d] > p->min[d];
    if (!(p->pcl_dst > 0) || !domain_ok || p->precision < 0 || p->precision > 2) {
        mps::g_last_error = "mps_bucket_build_noalloc: invalid parameters";
        return MPS_ERR_ARG;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t err = cudaSuccess;
    int rc = p->precision == MPS_F64
                 ? mps::run<double>(*p, n, typ, pos, cell, order, start, st, &err)
                 : mps::run<float>(*p, n, typ, pos, cell, order, start, st, &err);
    if (rc == MPS_ERR_OVERFLOW)
        mps::g_last_error = "mps_bucket_build_noalloc: the grid has more than "
                            "MPS_NOALLOC_MAX_BUCKETS buckets";
    else if (rc == MPS_ERR_CUDA)
        mps::g_last_error = std::string("mps_bucket_build_noalloc: ") + cudaGetErrorString(err);
    else if (rc == MPS_ERR_UNSUPPORTED)
        mps::g_last_error = "mps_bucket_build_noalloc: device ordinal beyond 63";
    return rc;
}
