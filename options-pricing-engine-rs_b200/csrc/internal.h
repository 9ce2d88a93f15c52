// Internal host-side interfaces shared by the C-ABI translation units.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stddef.h>
#include <stdint.h>

#include <string>

#include "../../include/ope.h"

namespace ope {

// Per-thread library state: current device, an internal stream for the
// synchronous host-pointer calls, a growable device workspace and the text
// of the last error.  Thread-local so concurrent host threads never share a
// workspace.
struct ThreadCtx {
    int device = -1;
    int sm_count = 0;
    int cc_major = 0, cc_minor = 0;
    cudaStream_t stream = nullptr;
    void* ws = nullptr;      // device workspace
    size_t ws_bytes = 0;
    void* pinned = nullptr;  // pinned host staging
    size_t pinned_bytes = 0;
    std::string last_error;
    uint64_t launches = 0;
    size_t ws_limit = 0;         // cap on the device workspace (0: none), ope_set_workspace_limit
    double grid_fraction = 1.0;  // persistent launches fill at most this share of the block slots
    // Stream order of the workspace: the stream of its last user, an event
    // recorded there when that user's C-ABI call returned, and whether the
    // current call has taken the workspace (the event is recorded on exit).
    cudaStream_t ws_stream = nullptr;
    cudaEvent_t ws_event = nullptr;
    bool ws_recorded = false;
    bool ws_taken = false;
    int api_depth = 0;
    // Copy stream and events of the pipelined pageable-host pricing path
    // (created on first use with this thread's device).
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t pipe_ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // contracts per unit of this thread's last plain pricing launch: fixed
    // (last_per_unit), or the run probe's choice in the workspace word
    // last_probe (on last_probe_stream) for an automatic launch
    int last_per_unit = 1;
    const unsigned long long* last_probe = nullptr;
    cudaStream_t last_probe_stream = nullptr;
};

ThreadCtx& tctx();
int set_error(int code, const std::string& msg);
int check_cuda(cudaError_t e, const char* what);
int ensure_device();                               // OPE_OK or OPE_ERR_NO_DEVICE
// The per-thread device workspace, grown to `bytes`, for work enqueued on
// `st`.  If the previous call of this thread used it on another stream, `st`
// first waits (on the device) for that call's work.  Growth is stream-ordered
// (cudaFreeAsync of the old block and cudaMallocAsync of the new one on
// `st`), so it never waits for, or stalls, work on other streams.
int ensure_workspace(size_t bytes, void** out, cudaStream_t st);
int ensure_pinned(size_t bytes, void** out);       // grows the pinned staging buffer
// Resident blocks per SM of `kernel` (threads per block, dynamic shared
// memory) on the current device, with its dynamic-shared-memory attribute
// set; queried once per kernel and device, then cached.
int blocks_per_sm(const void* kernel, int threads, size_t smem, int* per_sm);
// SM count of the current device (queried once per device, then cached).
// Persistent grids are sized from it, so a launch is sized for the device it
// runs on whichever thread makes it.
int current_device_sms(int* sms);
// Sets up both models' plain pricing kernels on the current device (their
// shared-memory attribute and occupancy query), so that later launches of
// them make no CUDA runtime calls besides the launch and its memset.
int prepare_price_kernels();

// Profiler ranges (NVTX, header-only: free when no tool is attached), one
// per C-ABI call and per server micro-batch.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
// One per C-ABI call: when the outermost call returns, records the
// workspace's event on the stream its work was enqueued on.
struct ApiScope {
    ApiScope();
    ~ApiScope();
    ApiScope(const ApiScope&) = delete;
    ApiScope& operator=(const ApiScope&) = delete;
};
#define OPE_RANGE(name)                           \
    ::ope::NvtxRange _ope_nvtx_range(name);       \
    ::ope::ApiScope _ope_api_scope

#define OPE_CHECK(call)                                        \
    do {                                                       \
        int _rc = ::ope::check_cuda((call), #call);            \
        if (_rc != OPE_OK) return _rc;                         \
    } while (0)

#define OPE_TRY(expr)                                          \
    do {                                                       \
        int _rc = (expr);                                      \
        if (_rc != OPE_OK) return _rc;                         \
    } while (0)

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Scratch needed by one pricing launch over n contracts: per-contract integral
// pair + completion counter, and the work-queue head.
// With order/bucket/hist set (carve_price_scratch sets them), a launch may
// queue its contracts deepest-first (LaunchShape::deepest_first); left NULL
// (the allocation-free entry point) it always uses the natural order.
struct PriceScratch {
    double* integ;                 // 2n
    unsigned int* done;            // n   (must be zero before launch)
    unsigned long long* head;      // 1   (must be zero before launch; persistent only)
    uint32_t* order = nullptr;     // n   queue position -> contract
    uint32_t* bucket = nullptr;    // n   depth bucket of each contract
    unsigned int* hist = nullptr;  // 2 x 64 bucket counts and fill counters
    // run cache of the run kernel (optional; run_cache_bytes() bytes): without
    // it a launch takes one contract per unit whatever its shape asks
    void* runcache = nullptr;
    size_t runcache_bytes = 0;
};
size_t price_scratch_bytes(size_t n);
PriceScratch carve_price_scratch(void* base, size_t n);
// The same with the run cache (run_bytes of it, 0: none) right after the
// price_scratch_bytes(n) bytes; price_run_bytes(model, n, other_bytes): the
// run cache a plain launch of n contracts wants under the current launch
// shape (0 or run_cache_bytes(); 0 too when it would take a workspace of
// other_bytes past the thread's limit).  Callers size and carve with one
// value of it.
PriceScratch carve_price_scratch(void* base, size_t n, size_t run_bytes);
size_t price_run_bytes(int model, size_t n, size_t other_bytes);

// Launch shape of a plain pricing launch: warps per block (each warp one
// integral, so warps / 2 contracts per block) of the persistent grid, whether
// the work queue takes contracts deepest-first (by |ln(K/S)| / sqrt(v0 T),
// which ranks the bisection counts with a Spearman correlation of 0.9) or in
// input order, and the share of the resident blocks per SM the grid fills.
// Every shape gives bit-identical prices (a unit's arithmetic does not depend
// on scheduling).
struct LaunchShape {
    int warps = 4;
    int deepest_first = 0;
    double occupancy = 1.0;
    // contracts per unit: 1 = one contract per unit (k_price_persistent);
    // 2..32 = blocks of that many consecutive contracts per warp, runs of
    // equal (parameter set, expiry, rate) sharing a run cache (k_price_runs,
    // input order); 0 = automatic: a call of 32,768 contracts or more probes
    // its contracts on the device and takes the run kernel when its runs
    // average 4 contracts or more
    int per_unit = 0;
};
// Bytes of the run cache for the current device (every warp the run
// kernel's grid can hold); 0 without a device.
size_t run_cache_bytes();
constexpr int kTuneClasses = 16;  // OPE_TUNE_CLASSES
// Size classes of the tuning table: calls of at most kTuneClassMax[i]
// contracts (64, 128, ..., 2^20; the last class: all larger calls).
extern const uint64_t kTuneClassMax[kTuneClasses];
// The shape a plain pricing launch of n contracts of `model` uses on the
// current device: the tuned table's entry for n's class when this device has
// been tuned and tuning is enabled, else the default shape.
LaunchShape price_shape(int model, size_t n);

// Device launchers (stream-ordered; all pointers are device pointers).
// Contract c is priced with params + stride * p(c), where p(c) = param_idx[c]
// when param_idx is non-NULL, else the surface of c under surf_offsets
// (n_surf + 1 entries), else 0.  With surf_mask non-NULL, units whose p(c)
// has surf_mask[p(c)] == 0 are skipped (their outputs are left untouched).
// Final live-panel lists of the integrals (the adjoint's backward pass runs
// over them).  Unit u = 2c + which of parameter set p(c) uses slot k =
// slot[p(c)] (slot NULL: 0) of n_slots: its bisection count is
// nbis[u * n_slots + k] and its panels the (a, b) pairs at
// panels + (u * n_slots + k) * 2 * kMaxPanels (kMaxPanels = 200).  Two slots
// let a calibration keep the lists of its current parameters while a trial
// step writes the other.
struct PanelSink {
    double* panels;
    int32_t* nbis;
    const int32_t* slot;
    int n_slots;
};
size_t panel_sink_bytes(size_t n, int n_slots);  // panels + nbis for n contracts
PanelSink carve_panel_sink(void* base, size_t n, int n_slots, const int32_t* slot);
// sink (non-NULL): also store every priced integral's panel list there.
// shape (non-NULL): this launch shape instead of price_shape(model, n); a
// launch that stores panel lists (sink) or skips surfaces (surf_mask) always
// uses 4 warps per block in input order.
int launch_price_persistent(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets,
                            size_t n_surf, const int32_t* param_idx, const double* params, double tol, double* out,
                            const PriceScratch& s, cudaStream_t st, int32_t* nbis_out = nullptr,
                            const int32_t* surf_mask = nullptr, const PanelSink* sink = nullptr,
                            const LaunchShape* shape = nullptr);
// The adjoint's backward pass and combine (adjoint.cu) over panel lists a
// pricing launch stored in `src`: out_grad (n x dim) = d price / d params.
// bscratch: grad_backward_bytes(n, dim) bytes (chunk list, partial sums).
size_t grad_backward_bytes(size_t n, int dim);
int launch_grad_backward(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                         const int32_t* param_idx, const double* params, const PanelSink& src, void* bscratch,
                         double* out_grad, cudaStream_t st, const int32_t* surf_mask = nullptr);
// Price + reverse-mode parameter gradient (adjoint.cu); `scratch` must hold
// grad_scratch_bytes(n, dim) bytes; out_grad is n x dim (dim 5 or 8).
size_t grad_scratch_bytes(size_t n, int dim);
int launch_price_grad(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                      const int32_t* param_idx, const double* params, double tol, double* out_price,
                      double* out_grad, void* scratch, cudaStream_t st, const int32_t* surf_mask = nullptr);
// Batched LM calibration (calib.cu).
struct CalibGraph;  // an instantiated LM graph (one per stream of use)
// Optional parts of calibrate_inner for a calibration batch (host pointers).
// prior / reg_weight: per surface, a Tikhonov pull toward prior[s] (ns x dim)
// with weight reg_weight[s] (calibration.rs:448-470).  group: per surface, a
// restart group in [0, n_group) whose members share a best SSE and prune
// against it (calibration.rs:482-490, 520-523); gbest0: n_group initial shared
// best values (NULL: +inf).
struct CalibExtra {
    const double* prior = nullptr;
    const double* reg_weight = nullptr;
    const int32_t* group = nullptr;
    const double* gbest0 = nullptr;
    int n_group = 0;
};
size_t calib_workspace_bytes(size_t nq, size_t ns, int dim);
size_t calib_pinned_bytes(size_t nq, size_t ns, int dim);
int calib_enqueue(int model, const ope_contract* quotes, const double* iv_market, const double* weights, size_t nq,
                  const int64_t* surf_offsets, const int64_t* off_h, size_t ns, const double* p0,
                  ope_calib_result* out, double tol, cudaMemcpyKind kind, cudaMemcpyKind out_kind, char* dev,
                  char* pin, cudaStream_t st, CalibGraph* G, const CalibExtra* ex = nullptr);
CalibGraph* calib_graph_new();
void calib_graph_release(CalibGraph* G);
void calib_graph_delete(CalibGraph* G);
int run_calibration(int model, const ope_contract* quotes, const double* iv_market, const double* weights, size_t nq,
                    const int64_t* surf_offsets, size_t ns, const double* p0, ope_calib_result* out, double tol,
                    bool device_ptrs, cudaStream_t st, const CalibExtra* ex = nullptr);
// Multistart and differential-evolution calibration (calib_global.cu), host pointers.
int run_multistart(int model, const ope_contract* quotes, const double* iv_market, const double* weights, size_t nq,
                   const int64_t* surf_offsets, size_t ns, const double* p0, int n_restarts, uint64_t seed,
                   const double* shared_best0, ope_multistart_result* out, ope_calib_result* out_restarts, double tol);
int run_global(int model, const ope_contract* quotes, const double* iv_market, const double* weights, size_t nq,
               const int64_t* surf_offsets, size_t ns, int n_pop, int n_gen, uint64_t seed, const double* prior,
               const double* reg_weight, ope_global_result* out, double tol);
int run_calib_jacobian(int model, const ope_contract* quotes, const double* iv_market, size_t nq,
                       const int64_t* surf_offsets, size_t ns, const double* params, double* out_jac,
                       double* out_res, double tol);
// batch.rs:51-56 on the device (calib.cu).
int launch_batch_iv(const ope_contract* con, const double* price, size_t n, double* iv, int32_t* ok, cudaStream_t st);
// DFMA throughput probe: FP64 flop/s (2 per FMA) over ~`ms_target` ms.
int measure_fp64_peak(double* flops, double* ms);
int selftest_math(uint64_t* ulp_rcp, uint64_t* ulp_sqrt);
int selftest_atan2(uint64_t* ulp);
int selftest_log(uint64_t* ulp);
int selftest_log_cr(const double* v, size_t n, double* out_cr, double* out_cuda);
int selftest_node_u(uint64_t* mismatches);
// Bump-and-reprice Greeks (greeks.rs:19-72) for n contracts under one
// parameter set; `ws` must hold greeks_workspace_bytes(n) bytes.
size_t greeks_workspace_bytes(size_t n);
int launch_greeks(int model, const ope_contract* con, size_t n, const double* params, double tol,
                  ope_pricing_result* out, void* ws, cudaStream_t st);
// AD Greeks (ad.rs:736-795, 809-865) for n contracts under one parameter set;
// `ws` must hold greeks_ad_workspace_bytes(n, dim) bytes.
size_t greeks_ad_workspace_bytes(size_t n, int dim);
int launch_greeks_ad(int model, const ope_contract* con, size_t n, const double* params, double tol,
                     ope_pricing_result* out, void* ws, cudaStream_t st);

// All eight Greeks analytically (adjoint.cu): one pricing launch that keeps
// the panel lists, one backward pass of the seven Greek integrals, one
// combine; n contracts under one parameter set; `ws` must hold
// greeks_analytic_workspace_bytes(n) bytes.
size_t greeks_analytic_workspace_bytes(size_t n);
int launch_greeks_analytic(int model, const ope_contract* con, size_t n, const double* params, double tol,
                           ope_pricing_result* out, void* ws, cudaStream_t st);

inline int param_stride(int model) { return model == OPE_MODEL_BATES ? 8 : 5; }

}  // namespace ope
