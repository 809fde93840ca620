// qx_noalloc.cu -- density statistics of a caller-owned device psi array
// without any allocation.
//
// Who needs it: code that holds psi in its own device memory and must not
// allocate while it runs -- a host application that hands all device memory
// to its own pool or caching allocator, a time-step loop that cannot afford
// the implicit device synchronisation of cudaMalloc/cudaFree, or a process
// working under a fixed memory budget.  Creating a qx field would allocate
// the field's buffers; this entry point needs none of them.
//
// The per-block partial sums live in the file-scope array below (fixed size,
// held by every GPU that loads this library until the process exits).  Host
// code must not pass the array's name to a kernel: on the host that name is
// only a stand-in, not a device address.  The device address is looked up
// with cudaGetSymbolAddress while the device is current, on the first call
// made for that device (make that first call before any stream capture
// begins), and looked up again only if the device's context has changed
// since (a cudaDeviceReset between calls gives the device a new context in
// which the array has a new address).  Every call writes each partial slot it
// later reads, so nothing needs clearing between calls; calls that overlap on
// the GPU share the array and race.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/qaxions_b200.h"
#include "qx_kernels.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 32;  // sites per thread
constexpr int kMaxBlocks = QX_NOALLOC_MAX_SITES / (kThreads * kPerThread);
constexpr int kMaxDevices = 64;

// two partials (sum, max) per block
static __device__ __align__(256) double g_noalloc_partials[2 * kMaxBlocks];

struct DevScratch {
    double* addr = nullptr;
    unsigned long long ctx_id = 0;  // context in which addr was looked up
};
DevScratch g_scratch[kMaxDevices];
std::mutex g_mu;
thread_local std::string g_err;

template <typename R>
__global__ void __launch_bounds__(kThreads) k_rho_partials(const qx::cx_t<R>* psi, long n, double* part) {
    __shared__ double red[32];
    double s = 0.0, m = 0.0;
    const long base = (long)blockIdx.x * kThreads * kPerThread + threadIdx.x;
#pragma unroll 4
    for (int k = 0; k < kPerThread; ++k) {
        const long i = base + (long)k * kThreads;
        if (i < n) {
            const qx::cx_t<R> p = psi[i];
            const double r = (double)p.x * p.x + (double)p.y * p.y;
            s += r;
            m = qx::fmax_nan(m, r);
        }
    }
    const double bs = qx::block_reduce<0>(s, red);
    const double bm = qx::block_reduce<1>(m, red);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = bs;
        part[kMaxBlocks + blockIdx.x] = bm;
    }
}

// one warp folds the block partials in a fixed order (NaN-propagating max)
__global__ void k_rho_fold(const double* part, int nblk, long n, double* out) {
    const double s = qx::warp_fold<0>(part, nblk);
    const double m = qx::warp_fold<1>(part + kMaxBlocks, nblk);
    if (threadIdx.x == 0) {
        out[0] = s;
        out[1] = m;
        out[2] = m / (s / (double)n);
    }
}

template <typename F> F driver_fn(const char* name) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return nullptr;
    return reinterpret_cast<F>(p);
}

// `ptr` .. `ptr + bytes` must lie inside one device allocation of device `dev`
bool device_extent_ok(const void* ptr, size_t bytes, int dev, const char* what) {
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, ptr) != cudaSuccess ||
        (pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) || pa.device != dev) {
        cudaGetLastError();
        g_err = std::string(what) + " is not device memory of the current device (select it with qx_set_device)";
        return false;
    }
    static const auto range = driver_fn<PFN_cuMemGetAddressRange_v3020>("cuMemGetAddressRange");
    CUdeviceptr base = 0;
    size_t size = 0;
    if (!range || range(&base, &size, reinterpret_cast<CUdeviceptr>(ptr)) != CUDA_SUCCESS) {
        g_err = std::string("cannot determine the allocation that holds ") + what;
        return false;
    }
    const uintptr_t p = reinterpret_cast<uintptr_t>(ptr);
    if (p < (uintptr_t)base || p - (uintptr_t)base > size || bytes > size - (p - (uintptr_t)base)) {
        g_err = std::string(what) + " extends past the end of its device allocation";
        return false;
    }
    return true;
}

// id of the current context (0 if it cannot be read)
unsigned long long current_ctx_id() {
    static const auto get_cur = driver_fn<PFN_cuCtxGetCurrent_v4000>("cuCtxGetCurrent");
    static const auto get_id = driver_fn<PFN_cuCtxGetId_v12000>("cuCtxGetId");
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur && get_id && get_cur(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS) return id;
    return 0;
}

}  // namespace

extern "C" const char* qx_noalloc_last_error(void) { return g_err.c_str(); }

extern "C" int qx_rho_stats_noalloc(const void* psi, long long sites, int dtype, double* out, void* stream) {
    if (!psi || !out) {
        g_err = "psi and out must be device pointers";
        return QX_ERR_INVALID;
    }
    if (dtype != QX_C128 && dtype != QX_C64) {
        g_err = "dtype must be QX_C128 or QX_C64";
        return QX_ERR_INVALID;
    }
    if (sites < 1 || sites > QX_NOALLOC_MAX_SITES) {
        g_err = "sites must be in [1, " + std::to_string((long long)QX_NOALLOC_MAX_SITES) +
                "]: the fixed scratch holds partials for at most that many sites";
        return QX_ERR_INVALID;
    }
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        g_err = "no usable current CUDA device";
        return QX_ERR_CUDA;
    }
    const size_t elem = dtype == QX_C64 ? sizeof(float2) : sizeof(double2);
    if (!device_extent_ok(psi, (size_t)sites * elem, dev, "psi")) return QX_ERR_INVALID;
    if (!device_extent_ok(out, 3 * sizeof(double), dev, "out")) return QX_ERR_INVALID;
    double* part = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        const unsigned long long ctx = current_ctx_id();
        DevScratch& ds = g_scratch[dev];
        if (!ds.addr || ds.ctx_id != ctx) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
            if (e != cudaSuccess || !p) {
                cudaGetLastError();
                g_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return QX_ERR_CUDA;
            }
            ds.addr = static_cast<double*>(p);
            ds.ctx_id = ctx;
        }
        part = ds.addr;
    }
    const int nblk = (int)((sites + (long long)kThreads * kPerThread - 1) / ((long long)kThreads * kPerThread));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dtype == QX_C64)
        k_rho_partials<float><<<nblk, kThreads, 0, st>>>(static_cast<const float2*>(psi), (long)sites, part);
    else
        k_rho_partials<double><<<nblk, kThreads, 0, st>>>(static_cast<const double2*>(psi), (long)sites, part);
    k_rho_fold<<<1, 32, 0, st>>>(part, nblk, (long)sites, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_err = std::string("kernel launch: ") + cudaGetErrorString(e);
        return QX_ERR_CUDA;
    }
    g_err.clear();
    return QX_OK;
}
