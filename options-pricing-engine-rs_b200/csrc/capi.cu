// C-ABI implementation (include/ope.h): per-thread context, argument
// validation, host<->device staging and dispatch to the kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "checked.cuh"
#include "internal.h"

#ifndef OPE_ZERO_COPY
#define OPE_ZERO_COPY 1
#endif

namespace ope {

#if OPE_CHECKED
__device__ unsigned int g_ope_check_word = 0;
#endif

ThreadCtx& tctx() {
    static thread_local ThreadCtx c;
    return c;
}

int set_error(int code, const std::string& msg) {
    tctx().last_error = msg;
    return code;
}

int check_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return OPE_OK;
    std::string msg = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    if (e == cudaErrorMemoryAllocation) return set_error(OPE_ERR_OUT_OF_MEMORY, msg);
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return set_error(OPE_ERR_NO_DEVICE, msg);
    return set_error(OPE_ERR_DEVICE, msg);
}

int ensure_device() {
    ThreadCtx& c = tctx();
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(OPE_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (c.device == cur) return OPE_OK;
    int major = 0, minor = 0, sms = 0;
    OPE_CHECK(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, cur));
    OPE_CHECK(cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, cur));
    OPE_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, cur));
    if (major != 10 || minor != 0) {
        return set_error(OPE_ERR_NO_DEVICE, "this library is built for sm_100a (B200); device " + std::to_string(cur) +
                                                " is sm_" + std::to_string(major) + std::to_string(minor));
    }
    // A new device for this thread: drop the old device's resources (leaked
    // rather than freed on the wrong device).
    c.ws = nullptr;
    c.ws_bytes = 0;
    c.last_probe = nullptr;
    OPE_CHECK(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    c.device = cur;
    c.sm_count = sms;
    c.cc_major = major;
    c.cc_minor = minor;
    return OPE_OK;
}

ApiScope::ApiScope() { ++tctx().api_depth; }

ApiScope::~ApiScope() {
    ThreadCtx& c = tctx();
    if (--c.api_depth == 0 && c.ws_taken) {
        c.ws_taken = false;
        c.ws_recorded = cudaEventRecord(c.ws_event, c.ws_stream) == cudaSuccess;
    }
}

int ensure_workspace(size_t bytes, void** out, cudaStream_t st) {
    ThreadCtx& c = tctx();
    if (!c.ws_event) OPE_CHECK(cudaEventCreateWithFlags(&c.ws_event, cudaEventDisableTiming));
    if (c.ws_limit && bytes > c.ws_limit)
        return set_error(OPE_ERR_OUT_OF_MEMORY, "call needs " + std::to_string(bytes) +
                                                    " bytes of device workspace, above this thread's limit of " +
                                                    std::to_string(c.ws_limit) + " (ope_set_workspace_limit)");
    // order st after the previous call's use of the workspace (another stream)
    if (c.ws_recorded && c.ws_stream != st) OPE_CHECK(cudaStreamWaitEvent(st, c.ws_event, 0));
    if (bytes > c.ws_bytes) {
        size_t want = std::max(bytes, c.ws_bytes + c.ws_bytes / 2);
        want = align_up(want, 1 << 20);
        if (c.ws_limit) want = std::max(bytes, std::min(want, c.ws_limit));
        // Stream-ordered: the old block is freed on st after every earlier use
        // of it (they are all ordered before st by the wait above, or were
        // enqueued on st by this call), and the new block is valid for work
        // enqueued on st from here on.  Neither call synchronises the device,
        // so growing one thread's workspace never stalls other streams.
        if (c.ws) {
            OPE_CHECK(cudaFreeAsync(c.ws, st));
            c.ws = nullptr;
            c.ws_bytes = 0;
            c.last_probe = nullptr;  // lived in the old block
        }
        OPE_CHECK(cudaMallocAsync(&c.ws, want, st));
        c.ws_bytes = want;
    }
    c.ws_stream = st;
    c.ws_taken = true;
    *out = c.ws;
    return OPE_OK;
}

int current_device_sms(int* sms) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static int cache[kMaxDevices] = {};
    int dev = -1;
    OPE_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) return set_error(OPE_ERR_NO_DEVICE, "device index out of range");
    std::lock_guard<std::mutex> g(mu);
    if (cache[dev] == 0) OPE_CHECK(cudaDeviceGetAttribute(&cache[dev], cudaDevAttrMultiProcessorCount, dev));
    *sms = cache[dev];
    return OPE_OK;
}

int blocks_per_sm(const void* kernel, int threads, size_t smem, int* per_sm) {
    static std::mutex mu;
    static std::map<std::tuple<const void*, int, int, size_t>, int> cache;
    int dev = -1;
    OPE_CHECK(cudaGetDevice(&dev));
    const auto key = std::make_tuple(kernel, dev, threads, smem);
    {
        std::lock_guard<std::mutex> g(mu);
        const auto it = cache.find(key);
        if (it != cache.end()) {
            *per_sm = it->second;
            return OPE_OK;
        }
    }
    int b = 0;
    OPE_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    OPE_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, threads, smem));
    if (b < 1) b = 1;
    std::lock_guard<std::mutex> g(mu);
    cache[key] = b;
    *per_sm = b;
    return OPE_OK;
}

int ensure_pinned(size_t bytes, void** out) {
    ThreadCtx& c = tctx();
    if (bytes > c.pinned_bytes) {
        if (c.pinned) {
            OPE_CHECK(cudaFreeHost(c.pinned));
            c.pinned = nullptr;
            c.pinned_bytes = 0;
        }
        size_t want = align_up(std::max(bytes, (size_t)1 << 20), 1 << 20);
        OPE_CHECK(cudaMallocHost(&c.pinned, want));
        c.pinned_bytes = want;
    }
    *out = c.pinned;
    return OPE_OK;
}

namespace {

int resolve_tol(const ope_options* o, double* tol) {
    double t = (o && o->tol > 0.0) ? o->tol : OPE_REF_TOL;
    if (o && std::isnan(o->tol)) return set_error(OPE_ERR_INVALID_ARG, "tol is NaN");
    if (!std::isfinite(t)) return set_error(OPE_ERR_INVALID_ARG, "tol must be finite");
    *tol = t;
    return OPE_OK;
}

int check_model(int32_t model) {
    if (model != OPE_MODEL_HESTON && model != OPE_MODEL_BATES)
        return set_error(OPE_ERR_INVALID_ARG, "model must be OPE_MODEL_HESTON or OPE_MODEL_BATES");
    return OPE_OK;
}

bool device_ptrs(const ope_options* o) { return o && (o->flags & OPE_FLAG_DEVICE_PTRS); }
cudaStream_t user_stream(const ope_options* o) { return o ? static_cast<cudaStream_t>(o->stream) : nullptr; }

// Device address of a pinned (page-locked, mapped) host buffer, or nullptr
// for pageable memory.  The pricing kernel reads each contract once and
// writes each price once, so from pinned host buffers it works in place over
// PCIe (zero-copy): the transfer overlaps the compute instead of preceding
// and following it.
void* pinned_device_ptr(const void* host) {
    if (!OPE_ZERO_COPY) return nullptr;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, host) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

// Calls from pageable host contracts of at least this many contracts take
// the pipelined path below.
constexpr size_t kPipelineMin = 262144;
// Calls from pageable host contracts of at most this many contracts stage them
// through the thread's pinned buffer (a host memcpy) and let the kernel read
// them and write the prices there in place (zero-copy), instead of a staged
// pageable copy each way around the launch: a small call's time is mostly
// these fixed costs.
constexpr size_t kStagedMax = 16384;

// The staged small-call setup: contracts copied into the pinned buffer
// (*k_con points at them); *h_out is the pinned slot for the prices (NULL
// when the caller's output is pinned already, *k_out).
int stage_small(const ope_contract* contracts, size_t n, const ope_contract** k_con, double** k_out,
                double** h_out) {
    const size_t b_con = align_up(n * sizeof(ope_contract), 256);
    void* pin;
    OPE_TRY(ensure_pinned(b_con + align_up(n * sizeof(double), 256), &pin));
    std::memcpy(pin, contracts, n * sizeof(ope_contract));
    *k_con = static_cast<const ope_contract*>(pinned_device_ptr(pin));
    *h_out = nullptr;
    if (!*k_out) {
        *h_out = reinterpret_cast<double*>(static_cast<char*>(pin) + b_con);
        *k_out = static_cast<double*>(pinned_device_ptr(*h_out));
    }
    if (!*k_con || !*k_out) return set_error(OPE_ERR_DEVICE, "pinned staging buffer is not device-accessible");
    return OPE_OK;
}

// Pageable host contracts (what a Rust Vec is), large calls: the contract copy
// no longer precedes the whole launch.  The first eighth of the contracts is
// copied and priced; the other seven eighths copy on the thread's copy stream
// while that first launch runs, then price; each part's prices come back as
// soon as its launch ends (from a pageable output the host waits for each;
// into pinned memory the kernel writes them in place).  Two launches instead
// of one cost one extra queue tail.  The parts split the contracts anywhere:
// each gets its own rebased surface offsets (contract ranges clipped to the
// part) and its parameter rows; every unit's arithmetic is that of a single
// launch, so prices are bit-identical.  off_h == NULL: one parameter set
// (d_par) for all contracts.  d_off2 holds room for n_surf + 3 offsets;
// d_nb (NULL or 2n bisection counts) and out_nb follow the same parts;
// scratch holds price_scratch_bytes(n) bytes and run_bytes of run cache.
int price_pipelined(int model, const ope_contract* contracts, size_t n, const int64_t* off_h, size_t n_surf,
                    const double* d_par, double tol, ope_contract* d_con, int64_t* d_off2, double* d_out,
                    double* out_prices, double* k_out, int32_t* d_nb, int32_t* out_nb, void* scratch,
                    size_t run_bytes) {
    ThreadCtx& c = tctx();
    if (!c.copy_stream) OPE_CHECK(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
    for (auto& e : c.pipe_ev)
        if (!e) OPE_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    cudaStream_t st = c.stream, cs = c.copy_stream;
    const int stride = param_stride(model);
    const size_t c1 = n / 8;  // part A: [0, c1), part B: [c1, n)
    // parts' surfaces and rebased offsets
    size_t nsA = 1, nsB = 1, sB = 0;
    std::vector<int64_t> offs;
    if (off_h) {
        const size_t sA_last = (size_t)(std::upper_bound(off_h, off_h + n_surf + 1, (int64_t)c1 - 1) - off_h) - 1;
        sB = (size_t)(std::upper_bound(off_h, off_h + n_surf + 1, (int64_t)c1) - off_h) - 1;
        nsA = sA_last + 1;
        nsB = n_surf - sB;
        offs.resize(nsA + 1 + nsB + 1);
        for (size_t j = 0; j < nsA; ++j) offs[j] = std::min<int64_t>(off_h[j], (int64_t)c1);
        offs[nsA] = (int64_t)c1;
        for (size_t j = 0; j <= nsB; ++j) offs[nsA + 1 + j] = std::max<int64_t>(off_h[sB + j], (int64_t)c1) - (int64_t)c1;
        OPE_CHECK(cudaMemcpyAsync(d_off2, offs.data(), offs.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    }
    const int64_t* offA = off_h ? d_off2 : nullptr;
    const int64_t* offB = off_h ? d_off2 + nsA + 1 : nullptr;
    const PriceScratch sc = carve_price_scratch(scratch, n, run_bytes);
    double* oA = k_out ? k_out : d_out;
    // part A: copy, then price
    OPE_CHECK(cudaMemcpyAsync(d_con, contracts, c1 * sizeof(ope_contract), cudaMemcpyHostToDevice, cs));
    OPE_CHECK(cudaEventRecord(c.pipe_ev[0], cs));
    OPE_CHECK(cudaStreamWaitEvent(st, c.pipe_ev[0], 0));
    OPE_TRY(launch_price_persistent(model, d_con, c1, offA, nsA, nullptr, d_par, tol, oA, sc, st, d_nb));
    OPE_CHECK(cudaEventRecord(c.pipe_ev[2], st));
    // part B: its copy overlaps part A's pricing
    OPE_CHECK(cudaMemcpyAsync(d_con + c1, contracts + c1, (n - c1) * sizeof(ope_contract), cudaMemcpyHostToDevice,
                              cs));
    OPE_CHECK(cudaEventRecord(c.pipe_ev[1], cs));
    OPE_CHECK(cudaStreamWaitEvent(st, c.pipe_ev[1], 0));
    OPE_TRY(launch_price_persistent(model, d_con + c1, n - c1, offB, nsB, nullptr, d_par + sB * stride, tol, oA + c1,
                                    sc, st, d_nb ? d_nb + 2 * c1 : nullptr));
    OPE_CHECK(cudaEventRecord(c.pipe_ev[3], st));
    // results: part A's while part B prices, then part B's
    if (!k_out) {
        OPE_CHECK(cudaStreamWaitEvent(cs, c.pipe_ev[2], 0));
        OPE_CHECK(cudaMemcpyAsync(out_prices, d_out, c1 * sizeof(double), cudaMemcpyDeviceToHost, cs));
        OPE_CHECK(cudaStreamWaitEvent(cs, c.pipe_ev[3], 0));
        OPE_CHECK(cudaMemcpyAsync(out_prices + c1, d_out + c1, (n - c1) * sizeof(double), cudaMemcpyDeviceToHost, cs));
    }
    if (out_nb) OPE_CHECK(cudaMemcpyAsync(out_nb, d_nb, 2 * n * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    OPE_CHECK(cudaStreamSynchronize(cs));
    OPE_CHECK(cudaStreamSynchronize(st));
    return OPE_OK;
}

// Plain (one parameter set) pricing, host or device pointers.
int batch_price(int32_t model, const ope_contract* contracts, size_t n, const void* params, double* out,
                const ope_options* opts) {
    OPE_RANGE("ope.batch_price");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n == 0) return OPE_OK;
    if (!contracts || !params || !out) return set_error(OPE_ERR_INVALID_ARG, "NULL array argument");
    OPE_TRY(ensure_device());
    const int stride = param_stride(model);
    if (device_ptrs(opts)) {
        void* ws;
        const size_t b_run = price_run_bytes(model, n, price_scratch_bytes(n));
        OPE_TRY(ensure_workspace(price_scratch_bytes(n) + b_run, &ws, user_stream(opts)));
        return launch_price_persistent(model, contracts, n, nullptr, 1, nullptr, static_cast<const double*>(params),
                                       tol, out, carve_price_scratch(ws, n, b_run), user_stream(opts));
    }
    ThreadCtx& c = tctx();
    const size_t b_con = align_up(n * sizeof(ope_contract), 256), b_par = 256, b_out = align_up(n * sizeof(double), 256);
    const size_t b_run = price_run_bytes(model, n, b_con + b_par + b_out + price_scratch_bytes(n));
    void* ws;
    OPE_TRY(ensure_workspace(b_con + b_par + b_out + price_scratch_bytes(n) + b_run, &ws, c.stream));
    char* p = static_cast<char*>(ws);
    ope_contract* d_con = reinterpret_cast<ope_contract*>(p);
    double* d_par = reinterpret_cast<double*>(p + b_con);
    double* d_out = reinterpret_cast<double*>(p + b_con + b_par);
    void* scratch = p + b_con + b_par + b_out;
    // contracts and prices in pinned host memory are used in place (zero-copy)
    const ope_contract* k_con = static_cast<const ope_contract*>(pinned_device_ptr(contracts));
    double* k_out = static_cast<double*>(pinned_device_ptr(out));
    OPE_CHECK(cudaMemcpyAsync(d_par, params, stride * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    if (!k_con && n >= kPipelineMin)
        return price_pipelined(model, contracts, n, nullptr, 1, d_par, tol, d_con, nullptr, d_out, out, k_out, nullptr,
                               nullptr, scratch, b_run);
    double* h_out = nullptr;
    if (!k_con && n <= kStagedMax) {
        OPE_TRY(stage_small(contracts, n, &k_con, &k_out, &h_out));
        OPE_TRY(launch_price_persistent(model, k_con, n, nullptr, 1, nullptr, d_par, tol, k_out,
                                        carve_price_scratch(scratch, n, b_run), c.stream));
        OPE_CHECK(cudaStreamSynchronize(c.stream));
        if (h_out) std::memcpy(out, h_out, n * sizeof(double));
        return OPE_OK;
    }
    if (!k_con) {
        OPE_CHECK(cudaMemcpyAsync(d_con, contracts, n * sizeof(ope_contract), cudaMemcpyHostToDevice, c.stream));
        k_con = d_con;
    }
    OPE_TRY(launch_price_persistent(model, k_con, n, nullptr, 1, nullptr, d_par, tol, k_out ? k_out : d_out,
                                    carve_price_scratch(scratch, n, b_run), c.stream));
    if (!k_out) OPE_CHECK(cudaMemcpyAsync(out, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    return OPE_OK;
}

int batch_greeks(int32_t model, const ope_contract* contracts, size_t n, const void* params,
                 ope_pricing_result* out, const ope_options* opts, bool ad = false) {
    OPE_RANGE(ad ? "ope.batch_greeks_ad" : "ope.batch_greeks");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n == 0) return OPE_OK;
    if (!contracts || !params || !out) return set_error(OPE_ERR_INVALID_ARG, "NULL array argument");
    OPE_TRY(ensure_device());
    const int stride = param_stride(model);
    const bool analytic = ad && opts && (opts->flags & OPE_FLAG_ANALYTIC_GREEKS);
    const size_t g_bytes = analytic ? greeks_analytic_workspace_bytes(n)
                                    : (ad ? greeks_ad_workspace_bytes(n, stride) : greeks_workspace_bytes(n));
    auto launch = [&](const ope_contract* con, const double* par, ope_pricing_result* o, void* gws, cudaStream_t st) {
        if (analytic) return launch_greeks_analytic(model, con, n, par, tol, o, gws, st);
        return ad ? launch_greeks_ad(model, con, n, par, tol, o, gws, st) : launch_greeks(model, con, n, par, tol, o, gws, st);
    };
    if (device_ptrs(opts)) {
        void* ws;
        OPE_TRY(ensure_workspace(g_bytes, &ws, user_stream(opts)));
        return launch(contracts, static_cast<const double*>(params), out, ws, user_stream(opts));
    }
    ThreadCtx& c = tctx();
    const size_t b_con = align_up(n * sizeof(ope_contract), 256), b_par = 256,
                 b_out = align_up(n * sizeof(ope_pricing_result), 256);
    void* ws;
    OPE_TRY(ensure_workspace(b_con + b_par + b_out + g_bytes, &ws, c.stream));
    char* p = static_cast<char*>(ws);
    ope_contract* d_con = reinterpret_cast<ope_contract*>(p);
    double* d_par = reinterpret_cast<double*>(p + b_con);
    ope_pricing_result* d_out = reinterpret_cast<ope_pricing_result*>(p + b_con + b_par);
    void* gws = p + b_con + b_par + b_out;
    OPE_CHECK(cudaMemcpyAsync(d_con, contracts, n * sizeof(ope_contract), cudaMemcpyHostToDevice, c.stream));
    OPE_CHECK(cudaMemcpyAsync(d_par, params, stride * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    OPE_TRY(launch(d_con, d_par, d_out, gws, c.stream));
    OPE_CHECK(cudaMemcpyAsync(out, d_out, n * sizeof(ope_pricing_result), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    return OPE_OK;
}

}  // namespace
}  // namespace ope

using namespace ope;

extern "C" {

const char* ope_last_error(void) { return tctx().last_error.c_str(); }

const char* ope_version(void) { return "ope-b200 0.1.0 (sm_100a, FP64 greedy GK15)"; }

uint64_t ope_kernel_launch_count(void) { return tctx().launches; }

int ope_check_word(uint32_t* out_word, int32_t* out_checked_build) {
    if (!out_word) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    *out_word = 0;
    if (out_checked_build) *out_checked_build = OPE_CHECKED;
#if OPE_CHECKED
    OPE_TRY(ensure_device());
    unsigned int w = 0;
    OPE_CHECK(cudaMemcpyFromSymbol(&w, g_ope_check_word, sizeof(w)));
    const unsigned int zero = 0;
    OPE_CHECK(cudaMemcpyToSymbol(g_ope_check_word, &zero, sizeof(zero)));
    *out_word = w;
#endif
    return OPE_OK;
}

int ope_set_workspace_limit(uint64_t bytes) {
    ThreadCtx& c = tctx();
    c.ws_limit = (size_t)bytes;
    if (bytes && c.ws && c.ws_bytes > bytes) {  // give back a workspace above the new cap
        // stream-ordered after the workspace's last use (its event), on this
        // thread's own stream (created with the workspace's device)
        if (c.last_probe) {  // the run probe's word lives in the workspace: keep what it said
            int32_t pu = 1;
            OPE_TRY(ope_last_per_unit(&pu));
            c.last_per_unit = pu;
            c.last_probe = nullptr;
        }
        if (c.ws_recorded) OPE_CHECK(cudaStreamWaitEvent(c.stream, c.ws_event, 0));
        OPE_CHECK(cudaFreeAsync(c.ws, c.stream));
        c.ws = nullptr;
        c.ws_bytes = 0;
        c.ws_recorded = false;
        c.ws_stream = nullptr;
    }
    return OPE_OK;
}

uint64_t ope_workspace_bytes(void) { return tctx().ws_bytes; }

int ope_device_info(int32_t* sm_count, int32_t* cc_major, int32_t* cc_minor) {
    OPE_TRY(ensure_device());
    if (sm_count) *sm_count = tctx().sm_count;
    if (cc_major) *cc_major = tctx().cc_major;
    if (cc_minor) *cc_minor = tctx().cc_minor;
    return OPE_OK;
}

int ope_heston_price(double spot, double strike, double expiry, double rate, double div_yield,
                     const ope_heston_params* params, int32_t opt_type, double* out_price) {
    if (!params || !out_price) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (opt_type != OPE_CALL && opt_type != OPE_PUT) return set_error(OPE_ERR_INVALID_ARG, "bad opt_type");
    ope_contract c{spot, strike, expiry, rate, div_yield, 0.0, opt_type, 0};
    return batch_price(OPE_MODEL_HESTON, &c, 1, params, out_price, nullptr);
}

int ope_bates_price(double spot, double strike, double expiry, double rate, double div_yield,
                    const ope_bates_params* params, int32_t opt_type, double* out_price) {
    if (!params || !out_price) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (opt_type != OPE_CALL && opt_type != OPE_PUT) return set_error(OPE_ERR_INVALID_ARG, "bad opt_type");
    ope_contract c{spot, strike, expiry, rate, div_yield, 0.0, opt_type, 0};
    return batch_price(OPE_MODEL_BATES, &c, 1, params, out_price, nullptr);
}

int ope_batch_heston(const ope_contract* contracts, size_t n, const ope_heston_params* params, double* out) {
    return batch_price(OPE_MODEL_HESTON, contracts, n, params, out, nullptr);
}

int ope_batch_bates(const ope_contract* contracts, size_t n, const ope_bates_params* params, double* out) {
    return batch_price(OPE_MODEL_BATES, contracts, n, params, out, nullptr);
}

int ope_batch_heston_greeks(const ope_contract* contracts, size_t n, const ope_heston_params* params,
                            ope_pricing_result* out) {
    return batch_greeks(OPE_MODEL_HESTON, contracts, n, params, out, nullptr);
}

int ope_batch_bates_greeks(const ope_contract* contracts, size_t n, const ope_bates_params* params,
                           ope_pricing_result* out) {
    return batch_greeks(OPE_MODEL_BATES, contracts, n, params, out, nullptr);
}

int ope_batch_price_ex(int32_t model, const ope_contract* contracts, size_t n, const void* params,
                       double* out_prices, const ope_options* opts) {
    return batch_price(model, contracts, n, params, out_prices, opts);
}

int ope_batch_greeks_ex(int32_t model, const ope_contract* contracts, size_t n, const void* params,
                        ope_pricing_result* out, const ope_options* opts) {
    return batch_greeks(model, contracts, n, params, out, opts);
}

int ope_batch_greeks_ad(int32_t model, const ope_contract* contracts, size_t n, const void* params,
                        ope_pricing_result* out, const ope_options* opts) {
    return batch_greeks(model, contracts, n, params, out, opts, true);
}

int ope_batch_implied_vol(const ope_contract* contracts, size_t n, const double* market_prices, double* out_iv,
                          int32_t* out_ok, const ope_options* opts) {
    OPE_RANGE("ope.batch_implied_vol");
    if (n == 0) return OPE_OK;
    if (!contracts || !market_prices || !out_iv || !out_ok) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    OPE_TRY(ensure_device());
    if (device_ptrs(opts)) return launch_batch_iv(contracts, market_prices, n, out_iv, out_ok, user_stream(opts));
    ThreadCtx& c = tctx();
    const size_t b_con = align_up(n * sizeof(ope_contract), 256), b_d = align_up(n * sizeof(double), 256),
                 b_i = align_up(n * sizeof(int32_t), 256);
    void* ws;
    OPE_TRY(ensure_workspace(b_con + 2 * b_d + b_i, &ws, c.stream));
    char* p = static_cast<char*>(ws);
    ope_contract* d_con = reinterpret_cast<ope_contract*>(p);
    double* d_px = reinterpret_cast<double*>(p + b_con);
    double* d_iv = reinterpret_cast<double*>(p + b_con + b_d);
    int32_t* d_ok = reinterpret_cast<int32_t*>(p + b_con + 2 * b_d);
    OPE_CHECK(cudaMemcpyAsync(d_con, contracts, n * sizeof(ope_contract), cudaMemcpyHostToDevice, c.stream));
    OPE_CHECK(cudaMemcpyAsync(d_px, market_prices, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    OPE_TRY(launch_batch_iv(d_con, d_px, n, d_iv, d_ok, c.stream));
    OPE_CHECK(cudaMemcpyAsync(out_iv, d_iv, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaMemcpyAsync(out_ok, d_ok, n * sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    return OPE_OK;
}

int ope_calibrate_surfaces(int32_t model, const ope_contract* quotes, const double* iv_market, const double* weights,
                           size_t n_quotes, const int64_t* surf_offsets, size_t n_surf, const double* p0,
                           ope_calib_result* out, const ope_options* opts) {
    OPE_RANGE("ope.calibrate_surfaces");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n_surf == 0) return OPE_OK;
    if (!quotes || !iv_market || !surf_offsets || !p0 || !out) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (n_quotes == 0) return set_error(OPE_ERR_INVALID_ARG, "nothing to calibrate");  // calibration.rs:438
    OPE_TRY(ensure_device());
    return run_calibration(model, quotes, iv_market, weights, n_quotes, surf_offsets, n_surf, p0, out, tol,
                           device_ptrs(opts), user_stream(opts));
}

int ope_calibrate_surfaces_reg(int32_t model, const ope_contract* quotes, const double* iv_market,
                               const double* weights, size_t n_quotes, const int64_t* surf_offsets, size_t n_surf,
                               const double* p0, const double* prior, const double* reg_weight,
                               ope_calib_result* out, const ope_options* opts) {
    OPE_RANGE("ope.calibrate_surfaces_reg");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n_surf == 0) return OPE_OK;
    if (!quotes || !iv_market || !surf_offsets || !p0 || !out || !prior || !reg_weight)
        return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (n_quotes == 0) return set_error(OPE_ERR_INVALID_ARG, "nothing to calibrate");  // calibration.rs:438
    for (size_t s = 0; s < n_surf; ++s)
        if (!(reg_weight[s] >= 0.0)) return set_error(OPE_ERR_INVALID_ARG, "reg_weight must be >= 0");
    OPE_TRY(ensure_device());
    CalibExtra ex;
    ex.prior = prior;
    ex.reg_weight = reg_weight;
    return run_calibration(model, quotes, iv_market, weights, n_quotes, surf_offsets, n_surf, p0, out, tol,
                           device_ptrs(opts), user_stream(opts), &ex);
}

int ope_calibrate_multistart(int32_t model, const ope_contract* quotes, const double* iv_market,
                             const double* weights, size_t n_quotes, const int64_t* surf_offsets, size_t n_surf,
                             const double* p0, int32_t n_restarts, uint64_t seed, const double* shared_best0,
                             ope_multistart_result* out, ope_calib_result* out_restarts, const ope_options* opts) {
    OPE_RANGE("ope.calibrate_multistart");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n_surf == 0) return OPE_OK;
    if (!quotes || !iv_market || !surf_offsets || !p0 || !out) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (device_ptrs(opts)) return set_error(OPE_ERR_INVALID_ARG, "ope_calibrate_multistart takes host pointers");
    if (n_quotes == 0) return set_error(OPE_ERR_INVALID_ARG, "nothing to calibrate");
    OPE_TRY(ensure_device());
    return run_multistart(model, quotes, iv_market, weights, n_quotes, surf_offsets, n_surf, p0, n_restarts, seed,
                          shared_best0, out, out_restarts, tol);
}

int ope_calibrate_global(int32_t model, const ope_contract* quotes, const double* iv_market, const double* weights,
                         size_t n_quotes, const int64_t* surf_offsets, size_t n_surf, int32_t n_pop, int32_t n_gen,
                         uint64_t seed, const double* prior, const double* reg_weight, ope_global_result* out,
                         const ope_options* opts) {
    OPE_RANGE("ope.calibrate_global");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n_surf == 0) return OPE_OK;
    if (!quotes || !iv_market || !surf_offsets || !out) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (device_ptrs(opts)) return set_error(OPE_ERR_INVALID_ARG, "ope_calibrate_global takes host pointers");
    if (n_quotes == 0) return set_error(OPE_ERR_INVALID_ARG, "nothing to calibrate");
    if (prior)
        for (size_t s = 0; s < n_surf; ++s)
            if (!reg_weight || !(reg_weight[s] >= 0.0)) return set_error(OPE_ERR_INVALID_ARG, "reg_weight must be >= 0");
    OPE_TRY(ensure_device());
    return run_global(model, quotes, iv_market, weights, n_quotes, surf_offsets, n_surf, n_pop, n_gen, seed, prior,
                      reg_weight, out, tol);
}

int ope_calib_jacobian(int32_t model, const ope_contract* quotes, const double* iv_market, size_t n_quotes,
                       const int64_t* surf_offsets, size_t n_surf, const double* params, double* out_jac,
                       double* out_res, const ope_options* opts) {
    OPE_RANGE("ope.calib_jacobian");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n_quotes == 0) return OPE_OK;
    if (!quotes || !iv_market || !surf_offsets || !params || !out_jac || n_surf == 0)
        return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (device_ptrs(opts)) return set_error(OPE_ERR_INVALID_ARG, "ope_calib_jacobian takes host pointers");
    if (surf_offsets[0] != 0 || surf_offsets[n_surf] != (int64_t)n_quotes)
        return set_error(OPE_ERR_INVALID_ARG, "surf_offsets must span [0, n)");
    OPE_TRY(ensure_device());
    return run_calib_jacobian(model, quotes, iv_market, n_quotes, surf_offsets, n_surf, params, out_jac, out_res, tol);
}

int ope_price_gradient_surfaces(int32_t model, const ope_contract* contracts, size_t n, const int64_t* surf_offsets,
                                size_t n_surf, const void* params, double* out_prices, double* out_grad,
                                const ope_options* opts) {
    OPE_RANGE("ope.price_gradient_surfaces");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n == 0) return OPE_OK;
    if (!contracts || !params || !out_prices || !out_grad || !surf_offsets)
        return set_error(OPE_ERR_INVALID_ARG, "NULL array argument");
    if (n_surf == 0) return set_error(OPE_ERR_INVALID_ARG, "n_surf must be >= 1 when n > 0");
    OPE_TRY(ensure_device());
    const int dim = param_stride(model);
    if (device_ptrs(opts)) {
        void* ws;
        OPE_TRY(ensure_workspace(grad_scratch_bytes(n, dim), &ws, user_stream(opts)));
        return launch_price_grad(model, contracts, n, surf_offsets, n_surf, nullptr, static_cast<const double*>(params),
                                 tol, out_prices, out_grad, ws, user_stream(opts));
    }
    if (surf_offsets[0] != 0 || surf_offsets[n_surf] != (int64_t)n)
        return set_error(OPE_ERR_INVALID_ARG, "surf_offsets must start at 0 and end at n");
    for (size_t s = 0; s < n_surf; ++s)
        if (surf_offsets[s + 1] < surf_offsets[s]) return set_error(OPE_ERR_INVALID_ARG, "surf_offsets not sorted");
    ThreadCtx& c = tctx();
    const size_t b_con = align_up(n * sizeof(ope_contract), 256), b_off = align_up((n_surf + 1) * sizeof(int64_t), 256),
                 b_par = align_up(n_surf * dim * sizeof(double), 256), b_out = align_up(n * sizeof(double), 256),
                 b_g = align_up(n * dim * sizeof(double), 256);
    void* ws;
    OPE_TRY(ensure_workspace(b_con + b_off + b_par + b_out + b_g + grad_scratch_bytes(n, dim), &ws, c.stream));
    char* p = static_cast<char*>(ws);
    ope_contract* d_con = reinterpret_cast<ope_contract*>(p);
    int64_t* d_off = reinterpret_cast<int64_t*>(p + b_con);
    double* d_par = reinterpret_cast<double*>(p + b_con + b_off);
    double* d_out = reinterpret_cast<double*>(p + b_con + b_off + b_par);
    double* d_g = reinterpret_cast<double*>(p + b_con + b_off + b_par + b_out);
    void* scratch = p + b_con + b_off + b_par + b_out + b_g;
    OPE_CHECK(cudaMemcpyAsync(d_con, contracts, n * sizeof(ope_contract), cudaMemcpyHostToDevice, c.stream));
    OPE_CHECK(cudaMemcpyAsync(d_off, surf_offsets, (n_surf + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c.stream));
    OPE_CHECK(cudaMemcpyAsync(d_par, params, n_surf * dim * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    OPE_TRY(launch_price_grad(model, d_con, n, d_off, n_surf, nullptr, d_par, tol, d_out, d_g, scratch, c.stream));
    OPE_CHECK(cudaMemcpyAsync(out_prices, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaMemcpyAsync(out_grad, d_g, n * dim * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    return OPE_OK;
}

int ope_selftest_math(uint64_t* max_ulp_rcp, uint64_t* max_ulp_sqrt) {
    OPE_RANGE("ope.selftest_math");
    if (!max_ulp_rcp || !max_ulp_sqrt) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    OPE_TRY(ensure_device());
    return selftest_math(max_ulp_rcp, max_ulp_sqrt);
}

int ope_selftest_atan2(uint64_t* max_ulp) {
    OPE_RANGE("ope.selftest_atan2");
    if (!max_ulp) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    OPE_TRY(ensure_device());
    return selftest_atan2(max_ulp);
}

int ope_selftest_log(uint64_t* max_ulp) {
    OPE_RANGE("ope.selftest_log");
    if (!max_ulp) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    OPE_TRY(ensure_device());
    return selftest_log(max_ulp);
}

int ope_selftest_node_u(uint64_t* mismatches) {
    OPE_RANGE("ope.selftest_node_u");
    if (!mismatches) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    OPE_TRY(ensure_device());
    return selftest_node_u(mismatches);
}

int ope_selftest_log_cr(const double* args, size_t n, double* out_log_cr, double* out_log_cuda) {
    OPE_RANGE("ope.selftest_log_cr");
    if (n == 0) return OPE_OK;
    if (!args || !out_log_cr || !out_log_cuda) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (n > ((size_t)1 << 26)) return set_error(OPE_ERR_INVALID_ARG, "n above 2^26");
    OPE_TRY(ensure_device());
    return selftest_log_cr(args, n, out_log_cr, out_log_cuda);
}

int ope_measure_fp64_peak(double* flops_per_s, double* elapsed_ms) {
    OPE_RANGE("ope.measure_fp64_peak");
    if (!flops_per_s || !elapsed_ms) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    OPE_TRY(ensure_device());
    return measure_fp64_peak(flops_per_s, elapsed_ms);
}

int ope_price_surfaces(int32_t model, const ope_contract* contracts, size_t n, const int64_t* surf_offsets,
                       size_t n_surf, const void* params, double* out_prices, const ope_options* opts) {
    return ope_price_surfaces_stats(model, contracts, n, surf_offsets, n_surf, params, out_prices, nullptr, opts);
}

int ope_price_surfaces_stats(int32_t model, const ope_contract* contracts, size_t n, const int64_t* surf_offsets,
                             size_t n_surf, const void* params, double* out_prices, int32_t* out_bisections,
                             const ope_options* opts) {
    OPE_RANGE("ope.price_surfaces");
    OPE_TRY(check_model(model));
    double tol;
    OPE_TRY(resolve_tol(opts, &tol));
    if (n == 0) return OPE_OK;
    if (!contracts || !params || !out_prices || !surf_offsets)
        return set_error(OPE_ERR_INVALID_ARG, "NULL array argument");
    if (n_surf == 0) return set_error(OPE_ERR_INVALID_ARG, "n_surf must be >= 1 when n > 0");
    OPE_TRY(ensure_device());
    const int stride = param_stride(model);
    if (device_ptrs(opts)) {
        void* ws;
        const size_t b_run = price_run_bytes(model, n, price_scratch_bytes(n));
        OPE_TRY(ensure_workspace(price_scratch_bytes(n) + b_run, &ws, user_stream(opts)));
        return launch_price_persistent(model, contracts, n, surf_offsets, n_surf, nullptr,
                                       static_cast<const double*>(params), tol, out_prices,
                                       carve_price_scratch(ws, n, b_run), user_stream(opts), out_bisections);
    }
    if (surf_offsets[0] != 0 || surf_offsets[n_surf] != (int64_t)n)
        return set_error(OPE_ERR_INVALID_ARG, "surf_offsets must start at 0 and end at n");
    for (size_t s = 0; s < n_surf; ++s)
        if (surf_offsets[s + 1] < surf_offsets[s]) return set_error(OPE_ERR_INVALID_ARG, "surf_offsets not sorted");
    ThreadCtx& c = tctx();
    const size_t b_con = align_up(n * sizeof(ope_contract), 256), b_off = align_up((n_surf + 3) * sizeof(int64_t), 256),
                 b_par = align_up(n_surf * stride * sizeof(double), 256), b_out = align_up(n * sizeof(double), 256),
                 b_nb = out_bisections ? align_up(2 * n * sizeof(int32_t), 256) : 0;
    const size_t b_run = price_run_bytes(model, n, b_con + b_off + b_par + b_out + b_nb + price_scratch_bytes(n));
    void* ws;
    OPE_TRY(ensure_workspace(b_con + b_off + b_par + b_out + b_nb + price_scratch_bytes(n) + b_run, &ws, c.stream));
    char* p = static_cast<char*>(ws);
    ope_contract* d_con = reinterpret_cast<ope_contract*>(p);
    int64_t* d_off = reinterpret_cast<int64_t*>(p + b_con);
    double* d_par = reinterpret_cast<double*>(p + b_con + b_off);
    double* d_out = reinterpret_cast<double*>(p + b_con + b_off + b_par);
    int32_t* d_nb = out_bisections ? reinterpret_cast<int32_t*>(p + b_con + b_off + b_par + b_out) : nullptr;
    void* scratch = p + b_con + b_off + b_par + b_out + b_nb;
    // contracts and prices in pinned host memory are used in place (zero-copy)
    const ope_contract* k_con = static_cast<const ope_contract*>(pinned_device_ptr(contracts));
    double* k_out = static_cast<double*>(pinned_device_ptr(out_prices));
    OPE_CHECK(cudaMemcpyAsync(d_par, params, n_surf * stride * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    if (!k_con && n >= kPipelineMin)
        return price_pipelined(model, contracts, n, surf_offsets, n_surf, d_par, tol, d_con, d_off, d_out, out_prices,
                               k_out, d_nb, out_bisections, scratch, b_run);
    double* h_out = nullptr;
    if (!k_con && n <= kStagedMax) OPE_TRY(stage_small(contracts, n, &k_con, &k_out, &h_out));
    if (!k_con) {
        OPE_CHECK(cudaMemcpyAsync(d_con, contracts, n * sizeof(ope_contract), cudaMemcpyHostToDevice, c.stream));
        k_con = d_con;
    }
    OPE_CHECK(cudaMemcpyAsync(d_off, surf_offsets, (n_surf + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, c.stream));
    OPE_TRY(launch_price_persistent(model, k_con, n, d_off, n_surf, nullptr, d_par, tol, k_out ? k_out : d_out,
                                    carve_price_scratch(scratch, n, b_run), c.stream, d_nb));
    if (!k_out)
        OPE_CHECK(cudaMemcpyAsync(out_prices, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    if (out_bisections)
        OPE_CHECK(cudaMemcpyAsync(out_bisections, d_nb, 2 * n * sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    OPE_CHECK(cudaStreamSynchronize(c.stream));
    if (h_out) std::memcpy(out_prices, h_out, n * sizeof(double));
    return OPE_OK;
}

}  // extern "C"
