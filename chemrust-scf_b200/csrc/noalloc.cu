// chfsi_zgemm_cn_noalloc: the complex projection / overlap GEMM
// (C = conj(A) B^T, the op::C ZGEMM) for callers that cannot allocate device
// memory — a host code that hands the whole GPU to its own memory pool
// (a Fortran SCF driver that preallocates, or a framework's caching
// allocator), or a caller on a latency-critical path where cudaMalloc and
// cudaFree would synchronise the device.  The caller passes the inputs and
// the output; the split-K partial sums go to one file-scope device array of
// kNoAllocScratchBytes (4 MiB), which every GPU that loads this library keeps
// until the process exits.
//
// Set-up: the first call on a device (with that device current) looks the
// array's device address up with cudaGetSymbolAddress and caches it per
// device; make that first call before any stream capture.  The cached address
// belongs to the device's primary context: cudaDeviceReset while the library
// is loaded is not supported (the next call would write to a stale address).
// Calls share the array, so calls that overlap on the GPU (different streams,
// or different host threads on one device) race; serialise them.  Nothing
// needs clearing
// between calls: every partial the reduction reads is written earlier in the
// same call.
#include "chfsi.h"
#include "gemm.hpp"

#include <cuda_runtime.h>

#include <mutex>
#include <string>

namespace chfsi {
chfsi_status cuda_fail(cudaError_t e, const char* expr, const char* file, int line);
void set_last_error(const char* msg);
}

namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)CHFSI_NOALLOC_SCRATCH_BYTES;
constexpr size_t kNoAllocScratchElems = kNoAllocScratchBytes / sizeof(double2);
constexpr int kMaxDevices = 64;
// split-K chunk arithmetic is 32-bit; this bound keeps it far from overflow
constexpr int kMaxK = 1 << 30;

static __device__ __align__(256) double2 g_noalloc_scratch[kNoAllocScratchElems];

std::mutex g_setup_mutex;
double2* g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (host code only
// sees a stand-in for the symbol, never its device address).
chfsi_status scratch_for_current_device(double2** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return chfsi::cuda_fail(e, "cudaGetDevice", __FILE__, __LINE__);
    if (dev < 0 || dev >= kMaxDevices) {
        chfsi::set_last_error("chfsi_zgemm_cn_noalloc: device ordinal above 63");
        return CHFSI_ERR_BAD_INPUT;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return chfsi::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)", __FILE__, __LINE__);
        g_scratch_addr[dev] = static_cast<double2*>(p);
    }
    *out = g_scratch_addr[dev];
    return CHFSI_OK;
}

}  // namespace

extern "C" chfsi_status chfsi_zgemm_cn_noalloc(const chfsi_c128* a_dev, int lda,
                                               const chfsi_c128* b_dev, int ldb, int m, int n,
                                               int k, chfsi_c128* c_dev, void* stream) {
    if (!a_dev || !b_dev || !c_dev) {
        chfsi::set_last_error("chfsi_zgemm_cn_noalloc: null device pointer");
        return CHFSI_ERR_BAD_INPUT;
    }
    if (m <= 0 || n <= 0 || k <= 0 || k > kMaxK) {
        chfsi::set_last_error("chfsi_zgemm_cn_noalloc: m, n and k must be in 1..2^30");
        return CHFSI_ERR_BAD_INPUT;
    }
    if (lda < k || ldb < k) {
        chfsi::set_last_error("chfsi_zgemm_cn_noalloc: lda and ldb must be at least k");
        return CHFSI_ERR_BAD_INPUT;
    }
    const size_t mn = (size_t)m * (size_t)n;
    if (mn > kNoAllocScratchElems) {
        // one split needs m*n partials; larger outputs need the allocating entry point
        chfsi::set_last_error("chfsi_zgemm_cn_noalloc: m*n exceeds the 262144-element static "
                              "scratch (use chfsi_zgemm_cn)");
        return CHFSI_ERR_BAD_INPUT;
    }
    double2* scratch = nullptr;
    chfsi_status s = scratch_for_current_device(&scratch);
    if (s != CHFSI_OK) return s;
    cudaStream_t st = (cudaStream_t)stream;
    const int max_splits = (int)(kNoAllocScratchElems / mn);
    chfsi::gemm_cn_capped(reinterpret_cast<const double2*>(a_dev), lda,
                          reinterpret_cast<const double2*>(b_dev), ldb, m, n, k, max_splits, scratch,
                          reinterpret_cast<double2*>(c_dev), st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return chfsi::cuda_fail(e, "gemm_cn_capped", __FILE__, __LINE__);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return chfsi::cuda_fail(e, "cudaStreamSynchronize", __FILE__, __LINE__);
    return CHFSI_OK;
}
