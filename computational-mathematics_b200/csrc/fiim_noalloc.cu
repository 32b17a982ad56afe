// Preconditioner application that allocates no device memory.
//
// fiim_prec_apply needs one scratch vector (tm = IDv o (H r), n doubles) and leaves it
// to the caller. Some callers cannot provide or allocate it: a host application that
// hands all device memory to its own pool at start-up and forbids allocations behind
// that pool's back, or a service that runs under a fixed per-process device-memory
// budget. fiim_prec_apply_noalloc serves them from a fixed array compiled into this
// library instead. The array is a file-scope __device__ variable, so every GPU that
// loads this library's device code holds it (kNoAllocMaxRows doubles, 8 MiB) until
// the process exits.
//
// Host code must not pass the array's name to a kernel: on the host it names a
// host-side stand-in, not device memory. Its device address is looked up once per
// device with cudaGetSymbolAddress (with that device current) on the first call made
// on that device, then reused.

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "fiim_b200.h"
#include "fiim_internal.h"
#include "fiim_kernels.cuh"

namespace {

constexpr long kNoAllocMaxRows = 1L << 20;   // 1,048,576 rows -> 8 MiB of doubles
constexpr int kMaxDevices = 64;

// tm for fiim_prec_apply_noalloc. Shared by every call on a device; each call writes
// tm[0..n) in full (one value per row of H) before reading it, so nothing needs to be
// cleared between calls. Calls that overlap on the GPU (concurrent streams, or several
// host threads) race on it.
__device__ __align__(256) double g_noalloc_tm[kNoAllocMaxRows];

std::mutex g_mu;
double *g_tm_addr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_tm on the current device (looked up once per device).
int noalloc_scratch(double **out) {
    int dev = 0;
    FIIM_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return fiim::set_error(FIIM_EARG, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_tm_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_tm);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            return fiim::set_error(FIIM_ECUDA, "cudaGetSymbolAddress(g_noalloc_tm): %s", cudaGetErrorString(e));
        }
        g_tm_addr[dev] = static_cast<double *>(p);
    }
    *out = g_tm_addr[dev];
    return FIIM_OK;
}

int grid_rows(long n, int rows_per_block) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
        cudaGetLastError();
        sms = 148;
    }
    const long need = (n + rows_per_block - 1) / rows_per_block;
    return (int)std::max<long>(1, std::min<long>(need, 8L * sms));
}

}  // namespace

extern "C" int fiim_prec_apply_noalloc(int n, const int *Gi, const int *Gj, const double *Gv,
                                       const double *IDv, const int *Hi, const int *Hj,
                                       const double *Hv, const double *r, double *z, void *stream) {
    if (n <= 0 || !Gi || !Gj || !Gv || !IDv || !Hi || !Hj || !Hv || !r || !z)
        return fiim::set_error(FIIM_EARG, "null array or n <= 0");
    if (n > kNoAllocMaxRows)
        return fiim::set_error(FIIM_EARG,
                               "n = %d exceeds the %ld rows fiim_prec_apply_noalloc serves; "
                               "use fiim_prec_apply with caller scratch", n, kNoAllocMaxRows);
    FIIM_TRY(fiim::check_device(nullptr));
    double *tm = nullptr;
    FIIM_TRY(noalloc_scratch(&tm));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Eight lanes per row; every lane count gives the same sums (storage order).
    constexpr int kVec = 8;
    const int g = grid_rows(n, (32 / kVec) * fiim::kWarps);
    fiim::k_spmv_vec<kVec, fiim::EpiScale, 2><<<g, fiim::kThreads, 0, s>>>(
        fiim::CsrView<double>{Hi, Hj, Hv, n}, r, fiim::EpiScale{tm, IDv}, nullptr, nullptr);
    FIIM_CUDA(cudaGetLastError());
    fiim::k_spmv_vec<kVec, fiim::EpiStore, 1><<<g, fiim::kThreads, 0, s>>>(
        fiim::CsrView<double>{Gi, Gj, Gv, n}, tm, fiim::EpiStore{z}, nullptr, nullptr);
    FIIM_CUDA(cudaGetLastError());
    return FIIM_OK;
}
