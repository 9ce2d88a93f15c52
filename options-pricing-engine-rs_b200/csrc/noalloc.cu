// Allocation-free variant of the batched pricing entry point.
//
// Some callers cannot let a library allocate device memory.  A host that hands
// all of a GPU's memory to one allocator (a framework's caching allocator, or
// a fixed arena sized at start-up) has none left for a library's own
// cudaMalloc, and a latency-critical request path cannot afford
// cudaMalloc/cudaFree in the middle of a request, since either may wait for
// the whole device.  ope_price_surfaces_noalloc serves them: the caller
// passes device buffers for inputs and outputs, and the pricing kernel's
// scratch (one integral pair and one completion counter per contract, plus
// the work-queue head) lives in the file-scope device array below, which
// every GPU that loads this library holds until the process exits.
//
// Limits and rules (also in include/ope.h):
//  * at most OPE_NOALLOC_MAX_CONTRACTS contracts per call; larger calls are
//    rejected with OPE_ERR_INVALID_ARG and a message;
//  * the first call on a device does the set-up, with that device current:
//    it looks up the array's device address (cudaGetSymbolAddress) and sets
//    up both models' kernels; make that first call before any stream capture;
//  * all calls share the one array: calls whose work overlaps on the GPU race
//    and corrupt each other's results; serialise them (one stream, or events);
//  * the array keeps the last call's contents; the parts that must start at
//    zero (completion counters, queue head) are cleared by every call.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "internal.h"

namespace ope {

namespace {

constexpr size_t kNoallocMax = OPE_NOALLOC_MAX_CONTRACTS;
// integ (2 doubles per contract) | done (one uint32 per contract) | queue head
constexpr size_t kIntegBytes = 2 * kNoallocMax * sizeof(double);
constexpr size_t kDoneBytes = kNoallocMax * sizeof(unsigned int);
constexpr size_t kScratchBytes = kIntegBytes + kDoneBytes + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// Per-device set-up: the device address of the scratch array (the host-side
// name g_noalloc_scratch is only a stand-in, never a device address).
int scratch_for_current_device(void** addr) {
    int dev = -1;
    OPE_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(OPE_ERR_NO_DEVICE, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        int major = 0, minor = 0;
        OPE_CHECK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
        OPE_CHECK(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev));
        if (major != 10 || minor != 0)
            return set_error(OPE_ERR_NO_DEVICE, "this library is built for sm_100a (B200)");
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr) return check_cuda(e == cudaSuccess ? cudaErrorInvalidSymbol : e,
                                                                "cudaGetSymbolAddress(noalloc scratch)");
        // both models' kernels set up now, so later calls make no CUDA
        // runtime calls besides the memset and the launch
        OPE_TRY(prepare_price_kernels());
        g_addr[dev] = p;
    }
    *addr = g_addr[dev];
    return OPE_OK;
}

}  // namespace

}  // namespace ope

using namespace ope;

extern "C" int ope_price_surfaces_noalloc(int32_t model, const ope_contract* d_contracts, size_t n,
                                          const int64_t* d_surf_offsets, size_t n_surf, const void* d_params,
                                          double* d_out_prices, double tol, void* stream) {
    if (model != OPE_MODEL_HESTON && model != OPE_MODEL_BATES)
        return set_error(OPE_ERR_INVALID_ARG, "model must be OPE_MODEL_HESTON or OPE_MODEL_BATES");
    if (n > kNoallocMax)
        return set_error(OPE_ERR_INVALID_ARG, "ope_price_surfaces_noalloc: n exceeds OPE_NOALLOC_MAX_CONTRACTS (" +
                                                  std::to_string(kNoallocMax) + "); use ope_price_surfaces");
    // the tolerance rule of every other entry point: <= 0 selects the
    // reference's 1e-8, NaN and infinity are rejected
    if (std::isnan(tol)) return set_error(OPE_ERR_INVALID_ARG, "tol is NaN");
    if (!(tol > 0.0)) tol = OPE_REF_TOL;
    if (!std::isfinite(tol)) return set_error(OPE_ERR_INVALID_ARG, "tol must be finite");
    if (n == 0) return OPE_OK;
    if (!d_contracts || !d_surf_offsets || !d_params || !d_out_prices || n_surf == 0)
        return set_error(OPE_ERR_INVALID_ARG, "NULL argument or n_surf == 0");
    void* base = nullptr;
    OPE_TRY(scratch_for_current_device(&base));
    char* p = static_cast<char*>(base);
    PriceScratch s;
    s.integ = reinterpret_cast<double*>(p);
    s.done = reinterpret_cast<unsigned int*>(p + kIntegBytes);
    s.head = reinterpret_cast<unsigned long long*>(p + kIntegBytes + kDoneBytes);
    // launch_price_persistent clears s.done[0..n) and s.head on the stream first
    return launch_price_persistent(model, d_contracts, n, d_surf_offsets, n_surf, nullptr,
                                   static_cast<const double*>(d_params), tol,
                                   d_out_prices, s, static_cast<cudaStream_t>(stream));
}
