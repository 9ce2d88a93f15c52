/*
 * ope.h — C ABI of the B200 (sm_100a) Heston/Bates characteristic-function
 * pricer.  This is the drop-in boundary: the reference crate
 * (options_pricing_engine 0.1.0, Rust) binds these symbols over `extern "C"`
 * in place of its CPU pricing path.  Every entry point cites the reference
 * item it replaces as `file:line` within the reference crate.
 *
 * Conventions
 *  - Every call returns an int status (OPE_OK = 0); nothing aborts.  The
 *    text of the last error on the calling thread is ope_last_error().
 *  - Arrays are caller-owned.  Plain calls take HOST pointers and return
 *    once results are in the caller's buffer.  With OPE_FLAG_DEVICE_PTRS in
 *    ope_options.flags every array argument is a DEVICE pointer and the call
 *    is stream-ordered on ope_options.stream (it returns after enqueueing).
 *  - All arithmetic is IEEE binary64.  The quadrature is the reference's
 *    greedy globally-adaptive Gauss-Kronrod-15 with at most 200 live panels
 *    (heston.rs:193-212); the absolute tolerance defaults to the reference's
 *    hard-coded 1e-8 (heston.rs:228) and is settable through ope_options.tol.
 *  - Thread safety: calls may come from any host thread.  Each thread owns
 *    a private device workspace.  Calls of one thread are ordered through
 *    it: a call whose work goes to a different stream than the previous
 *    call's (a device-pointer call on another stream, or a host-pointer call
 *    after a device-pointer one) first makes its stream wait, on the device,
 *    for the previous call's work.  Calls from different threads run
 *    independently.
 *  - Single GPU: the current CUDA device of the calling thread.
 */
#ifndef OPE_H
#define OPE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
    OPE_OK = 0,
    OPE_ERR_INVALID_ARG = 1,   /* NULL pointer, n/size mismatch, bad enum, tol not finite */
    OPE_ERR_OUT_OF_MEMORY = 2, /* device allocation failed */
    OPE_ERR_DEVICE = 3,        /* CUDA runtime/kernel error (see ope_last_error) */
    OPE_ERR_NO_DEVICE = 4,     /* no CUDA device, or the device is not sm_100 */
    OPE_ERR_TIMEOUT = 5,       /* a bounded device/host wait expired */
    OPE_ERR_REJECTED = 6,      /* admission control refused the request (serving) */
    OPE_ERR_CANCELLED = 7,     /* request cancelled before completion (serving) */
    OPE_ERR_NOT_FOUND = 8      /* unknown request id (serving) */
};

enum { OPE_CALL = 0, OPE_PUT = 1 };                /* types.rs:5-13 OptionType */
enum { OPE_MODEL_HESTON = 0, OPE_MODEL_BATES = 1 };

#define OPE_REF_TOL 1e-8          /* heston.rs:228 */
#define OPE_MAX_PANELS 200        /* heston.rs:194 */
#define OPE_FLAG_DEVICE_PTRS 1u
#define OPE_FLAG_ANALYTIC_GREEKS 2u  /* ope_batch_greeks_ad: all eight Greeks by adjoint, no bumps */

/* ------------------------------------------------------------- records */
/* types.rs:16-25 OptionContract (`vol` is carried but unused by Heston/Bates,
 * exactly as in batch.rs:25; it seeds the IV solver in calibration). 56 B. */
typedef struct {
    double spot, strike, expiry, rate, div_yield, vol;
    int32_t opt_type; /* OPE_CALL / OPE_PUT */
    int32_t pad;
} ope_contract;

/* types.rs:48-54 HestonParams (v0 is a variance). 40 B. */
typedef struct {
    double v0, kappa, theta, sigma, rho;
} ope_heston_params;

/* types.rs:66-72 BatesParams. 64 B. */
typedef struct {
    ope_heston_params heston;
    double lambda, mu_j, sigma_j;
} ope_bates_params;

/* types.rs:29-39 PricingResult. 64 B. */
typedef struct {
    double price, delta, gamma, vega, theta, rho, vanna, volga;
} ope_pricing_result;

/* calibration.rs:44-68 CalibResult.  params holds (v0, kappa, theta, sigma,
 * rho[, lambda, mu_j, sigma_j]); status: 1 converged (gradient or step
 * test), 2 stopped on the damping cap, 3 stopped on the iteration cap,
 * 4 pruned by multistart (early_stopped). */
typedef struct {
    double params[8];
    double rmse, max_err, condition_number;
    double weakest_direction[8];
    int32_t iters, converged, early_stopped, status;
} ope_calib_result;

/* calibration.rs:70-76 MultistartResult (+ the index of the best restart). */
typedef struct {
    ope_calib_result best;
    int32_t n_restarts, n_converged, n_pruned, best_restart;
} ope_multistart_result;

/* calibration.rs:296-300 GlobalCalibResult (+ the population size used). */
typedef struct {
    ope_calib_result best;  /* after the LM polish */
    double de_best_sse;     /* SSE of the DE winner, before the polish */
    int32_t de_generations, n_pop;
} ope_global_result;

typedef struct {
    double tol;        /* absolute GK15 tolerance; <= 0 selects OPE_REF_TOL */
    uint32_t flags;    /* OPE_FLAG_DEVICE_PTRS, OPE_FLAG_ANALYTIC_GREEKS */
    uint32_t reserved;
    void* stream;      /* cudaStream_t; used with OPE_FLAG_DEVICE_PTRS; NULL = default stream */
} ope_options;

/* ------------------------------------------------ library / diagnostics */
const char* ope_last_error(void);            /* thread-local text of the last failure */
const char* ope_version(void);
int ope_device_info(int32_t* sm_count, int32_t* cc_major, int32_t* cc_minor);
/* Device kernels launched by this library on the calling thread since load. */
uint64_t ope_kernel_launch_count(void);

/* No reference counterpart.  Caps the device workspace the calling thread's
 * calls may hold (bytes; 0 = no cap).  A call that needs more fails with
 * OPE_ERR_OUT_OF_MEMORY before allocating anything; a workspace already held
 * above the new cap is freed.  The request server's slab and the
 * allocation-free entry point are not affected. */
int ope_set_workspace_limit(uint64_t bytes);
/* Bytes of device workspace the calling thread holds. */
uint64_t ope_workspace_bytes(void);
/* No reference counterpart.  Reads and clears the device check word of a
 * bounds-checked build (make CHECKED=1, lib/checked/): each set bit is a
 * kernel invariant that failed and was contained (1 panel index, 2 panel
 * count, 4 surface index, 8 panel-list slot, 16 stored panel count, 32
 * run-cache entry).
 * *out_checked_build: 1 for that build; the ordinary build reports 0 and a
 * zero word. */
int ope_check_word(uint32_t* out_word, int32_t* out_checked_build);

/* ------------------------------------------------ reference drop-ins */
/* heston.rs:61-72 heston_price.  One contract. */
int ope_heston_price(double spot, double strike, double expiry, double rate, double div_yield,
                     const ope_heston_params* params, int32_t opt_type, double* out_price);

/* bates.rs:29-39 bates_price. */
int ope_bates_price(double spot, double strike, double expiry, double rate, double div_yield,
                    const ope_bates_params* params, int32_t opt_type, double* out_price);

/* batch.rs:23-27 batch_heston: one parameter set for the whole slice; output
 * in input order.  The "plain per-surface" launch: one warp per integral. */
int ope_batch_heston(const ope_contract* contracts, size_t n, const ope_heston_params* params,
                     double* out_prices);

/* batch.rs:38-42 batch_bates. */
int ope_batch_bates(const ope_contract* contracts, size_t n, const ope_bates_params* params,
                    double* out_prices);

/* batch.rs:32-36 batch_heston_greeks (greeks.rs:19-72 bump-and-reprice: 14
 * pricings per contract, priced as extra work units in one launch). */
int ope_batch_heston_greeks(const ope_contract* contracts, size_t n, const ope_heston_params* params,
                            ope_pricing_result* out);

/* batch.rs:44-48 batch_bates_greeks. */
int ope_batch_bates_greeks(const ope_contract* contracts, size_t n, const ope_bates_params* params,
                           ope_pricing_result* out);

/* The two batch entry points above with explicit options (tolerance, device
 * pointers, stream).  `model` selects the params type. */
int ope_batch_price_ex(int32_t model, const ope_contract* contracts, size_t n, const void* params,
                       double* out_prices, const ope_options* opts);

/* batch.rs:32-36 / 44-48 with explicit options (tolerance, device pointers,
 * stream); the reference's greeks always use the 1e-8 tolerance. */
int ope_batch_greeks_ex(int32_t model, const ope_contract* contracts, size_t n, const void* params,
                        ope_pricing_result* out, const ope_options* opts);

/* --------------------------------------- batched multi-surface pricing */
/* No single reference twin: many batch_heston/batch_bates calls (batch.rs:23,
 * 38), one per surface, fused into ONE persistent launch.  Surface s owns
 * contracts [surf_offsets[s], surf_offsets[s+1]) and prices them with
 * params[s] (ope_heston_params[] or ope_bates_params[] by `model`).
 * surf_offsets has n_surf+1 entries, starts at 0, ends at n, non-decreasing.
 * A device work queue hands (contract, integral) units to warps. */
int ope_price_surfaces(int32_t model, const ope_contract* contracts, size_t n,
                       const int64_t* surf_offsets, size_t n_surf, const void* params,
                       double* out_prices, const ope_options* opts);

/* ad.rs:736-795 heston_greeks_ad / ad.rs:809-865 bates_greeks_ad, batched
 * over contracts under one parameter set: price and vega from the exact
 * d price / d v0 (reverse-mode adjoint kernel; vega = dP/dv0 * 2 sqrt(v0)),
 * volga from the same derivative at v0 = (sqrt(v0) +- 0.01)^2 (lower leg
 * floored at 1e-6), delta / gamma (spot +- 1%), theta (T - 1 day, floored at
 * 1e-6), rho (r +- 1bp) and vanna by the reference's finite differences.
 * With OPE_FLAG_ANALYTIC_GREEKS: every Greek is an exact derivative instead
 * (the analytic S/r/T sensitivities that ad.rs:751-763 leaves to finite
 * differences): one pricing and one backward pass of seven derivative
 * integrals over the pricing's own panels -- in x = ln(S/K) (first and
 * second order), r, T and v0 (first and second order, and mixed with x) --
 * combined with the discount and parity terms of heston.rs:70, 95-98, in the
 * same conventions: delta = dP/dS, gamma = d2P/dS2, vega = dP/dsqrt(v0),
 * theta = -dP/dT per year, rho = dP/dr, vanna = d2P/dS dsqrt(v0),
 * volga = d2P/dsqrt(v0)^2.
 * Host or device pointers (OPE_FLAG_DEVICE_PTRS). */
int ope_batch_greeks_ad(int32_t model, const ope_contract* contracts, size_t n, const void* params,
                        ope_pricing_result* out, const ope_options* opts);

/* batch.rs:51-56 batch_implied_vol (iv.rs:14-95 per contract): BSM implied
 * volatility of market_prices[i] for contracts[i]; out_ok[i] = 0 where the
 * reference returns None (out_iv[i] is then 0). */
int ope_batch_implied_vol(const ope_contract* contracts, size_t n, const double* market_prices, double* out_iv,
                          int32_t* out_ok, const ope_options* opts);

/* calibration.rs:204-210 calibrate_heston / calibrate_bates (calibrate_inner,
 * calibration.rs:433-569), for many independent quote surfaces at once:
 * Levenberg-Marquardt in implied-vol space, one state machine per surface,
 * Jacobian from the adjoint kernel (d price/d p / BSM vega), the whole
 * iteration loop run on the device as one CUDA graph (conditional WHILE).
 * Surface s owns quotes [surf_offsets[s], surf_offsets[s+1]); iv_market[i]
 * is quote i's market IV; weights may be NULL (all 1.0); p0 is n_surf x dim.
 * out receives n_surf results.  Pricing tolerance: opts->tol (default 1e-8,
 * the tolerance the reference calibrates with). */
int ope_calibrate_surfaces(int32_t model, const ope_contract* quotes, const double* iv_market,
                           const double* weights, size_t n_quotes, const int64_t* surf_offsets,
                           size_t n_surf, const double* p0, ope_calib_result* out,
                           const ope_options* opts);

/* calibration.rs:220-230 calibrate_heston_regularized /
 * calibrate_bates_regularized, batched like ope_calibrate_surfaces: surface s
 * is pulled toward prior[s * dim ...] with weight reg_weight[s] (Tikhonov
 * pseudo-rows (p_k - prior_k) / scale_k, scale = calibration.rs:130, 174-177);
 * rmse, max_err and the J'J diagnostics stay data-only, as in the reference.
 * prior and reg_weight are host pointers. */
int ope_calibrate_surfaces_reg(int32_t model, const ope_contract* quotes, const double* iv_market,
                               const double* weights, size_t n_quotes, const int64_t* surf_offsets, size_t n_surf,
                               const double* p0, const double* prior, const double* reg_weight,
                               ope_calib_result* out, const ope_options* opts);

/* calibration.rs:246-314 calibrate_heston_multistart /
 * calibrate_bates_multistart, batched over surfaces (host pointers).  Every
 * surface runs n_restarts LM fits: restart 0 from p0[s], restart i from
 * CalibModel::random_guess (calibration.rs:131-141, 179-185) under rand 0.8's
 * SmallRng::seed_from_u64(splitmix64(seed ^ i)) (every surface gets the same
 * starts, as one reference call per surface would).  The restarts of a
 * surface share a best SSE and prune as the reference does (every 10
 * iterations, SSE > 8x the shared best); on the device they advance in
 * lockstep, one LM iteration each per pass.  shared_best0: NULL (+inf, the
 * reference) or n_surf initial values.  out: n_surf records; out_restarts:
 * NULL or n_surf x n_restarts records. */
int ope_calibrate_multistart(int32_t model, const ope_contract* quotes, const double* iv_market,
                             const double* weights, size_t n_quotes, const int64_t* surf_offsets, size_t n_surf,
                             const double* p0, int32_t n_restarts, uint64_t seed, const double* shared_best0,
                             ope_multistart_result* out, ope_calib_result* out_restarts, const ope_options* opts);

/* calibration.rs:316-427 calibrate_heston_global / calibrate_bates_global
 * (prior == NULL) and calibrate_*_global_regularized (prior: n_surf x dim,
 * reg_weight: n_surf), batched over surfaces (host pointers): differential
 * evolution DE/rand/1/bin (F 0.6, CR 0.9) over the parameter box with
 * max(n_pop, 4 dim) members for n_gen generations, every member's SSE a
 * device pricing + IV pass and the generation loop one CUDA graph launch,
 * then one device LM polish from each surface's winner. */
int ope_calibrate_global(int32_t model, const ope_contract* quotes, const double* iv_market, const double* weights,
                         size_t n_quotes, const int64_t* surf_offsets, size_t n_surf, int32_t n_pop, int32_t n_gen,
                         uint64_t seed, const double* prior, const double* reg_weight, ope_global_result* out,
                         const ope_options* opts);

/* calibration.rs:613-652 jacobian (host pointers): the IV-space Jacobian the
 * device LM uses, d iv_i / d p = (d price_i / d p) / vega_BSM(iv_i), rows of
 * dim doubles, and the IV residuals iv_i - iv_market_i (out_res may be NULL),
 * at params (n_surf x dim). */
int ope_calib_jacobian(int32_t model, const ope_contract* quotes, const double* iv_market, size_t n_quotes,
                       const int64_t* surf_offsets, size_t n_surf, const double* params, double* out_jac,
                       double* out_res, const ope_options* opts);

/* ad.rs:695-731 forward_pass (all parameters at once) / ad.rs:882-895
 * bates_jump_sensitivities_ad, batched over surfaces like ope_price_surfaces:
 * prices plus d price / d params by a reverse-mode adjoint kernel over the
 * primal's final panel set.  out_grad is n x dim, dim = 5 for Heston
 * (v0, kappa, theta, sigma, rho) and 8 for Bates (+ lambda, mu_j, sigma_j). */
int ope_price_gradient_surfaces(int32_t model, const ope_contract* contracts, size_t n,
                                const int64_t* surf_offsets, size_t n_surf, const void* params,
                                double* out_prices, double* out_grad, const ope_options* opts);

/* ----------------------------------------------------------- serving */
/* No reference twin (the reference is synchronous, batch.rs / calibration.rs):
 * a device-resident request server with continuous batching.  Requests are
 * queued by submit (non-blocking) and collected by wait.  A scheduler thread
 * packs everything pending into micro-batches (one persistent pricing launch
 * for reprices, one device-LM graph for calibrations) whenever a stream slot
 * and device memory are free, so new requests are admitted while earlier ones
 * are still running and their work overlaps on the GPU.  Admission is by
 * device memory: the server reserves hbm_fraction of the FREE HBM at creation
 * (capped by hbm_cap_bytes) and launches a batch when its buffers fit; a
 * request that can never fit is rejected (OPE_ERR_REJECTED).  Reprices run
 * on high-priority streams; calibrations one batch at a time on a
 * low-priority stream, its kernels' grids capped at calib_sm_fraction of the
 * block slots, so a reprice's blocks find free slots while a calibration runs.  A request's
 * results do not depend on what it was batched with. */
typedef struct ope_server ope_server;

typedef struct {
    double tol;                    /* pricing tolerance; <= 0 selects OPE_REF_TOL */
    double hbm_fraction;           /* share of free HBM to reserve (0 -> 0.5) */
    uint64_t hbm_cap_bytes;        /* upper bound on that reservation (0 -> none) */
    uint32_t max_inflight;         /* concurrent micro-batches = streams (0 -> 4) */
    uint32_t max_batch_contracts;  /* contracts per micro-batch (0 -> 2^20) */
    uint64_t pinned_bytes;         /* host staging (0 -> 256 MiB) */
    double calib_sm_fraction;      /* share of the GPU's block slots a calibration batch's kernels may fill,
                                      leaving the rest to reprices (<= 0 or > 1 -> 0.5) */
} ope_server_config;

typedef struct {
    uint64_t submitted, completed, rejected, cancelled, failed;
    uint64_t batches, batched_requests, max_inflight;
    uint64_t hbm_budget_bytes, hbm_peak_bytes, pending, inflight;
} ope_server_stats;

int ope_server_create(const ope_server_config* cfg, ope_server** out);
int ope_server_destroy(ope_server* server);
/* Reprice one surface: n contracts under one parameter set (batch.rs:23 / 38). */
int ope_server_submit_price(ope_server* server, int32_t model, const ope_contract* contracts, size_t n,
                            const void* params, uint64_t* out_id);
/* Calibrate one quote surface from p0 (calibration.rs:204-210). */
int ope_server_submit_calibrate(ope_server* server, int32_t model, const ope_contract* quotes,
                                const double* iv_market, size_t n, const void* p0, uint64_t* out_id);
/* Wait up to timeout_ms (< 0: forever) for a request; on OPE_OK the results go
 * to out_prices (n doubles, reprice) or out_calib (calibration) and the
 * request's latency (submit -> results on the host) to out_latency_ms.  The
 * request is forgotten after a non-timeout return. */
int ope_server_wait(ope_server* server, uint64_t id, double timeout_ms, double* out_prices,
                    ope_calib_result* out_calib, double* out_latency_ms);
/* Cancel a request that has not started yet. */
int ope_server_cancel(ope_server* server, uint64_t id);
int ope_server_get_stats(ope_server* server, ope_server_stats* out);

/* ope_price_surfaces plus diagnostics: out_bisections (may be NULL) receives
 * 2n int32 — the bisection count of each contract's P1 and P2 integral (the
 * loop iterations of heston.rs:200-210), from which the nodes evaluated are
 * 15 * (1 + 2 * count). */
int ope_price_surfaces_stats(int32_t model, const ope_contract* contracts, size_t n,
                             const int64_t* surf_offsets, size_t n_surf, const void* params,
                             double* out_prices, int32_t* out_bisections, const ope_options* opts);

/* No reference twin (measurement support): the FP64 throughput of this GPU,
 * measured by a DFMA-chain kernel (2 flops per DFMA) on the calling thread's
 * device.  The roofline denominator for the FP64-bound pricing kernels. */
int ope_measure_fp64_peak(double* flops_per_s, double* elapsed_ms);

/* No counterpart in the reference.  For callers that cannot let a library
 * allocate device memory: a host that hands all of a GPU's memory to one
 * allocator (a framework's caching allocator, or a fixed arena sized at
 * start-up) has none left for a library's own cudaMalloc, and a latency-
 * critical request path cannot afford cudaMalloc/cudaFree, either of which
 * may wait for the whole device.  This is ope_price_surfaces with DEVICE
 * pointers only that allocates nothing: the kernel's scratch lives in a static
 * device array of this library (about 1.25 MiB on every GPU that loads it,
 * held until exit), so n is limited to OPE_NOALLOC_MAX_CONTRACTS (larger n:
 * OPE_ERR_INVALID_ARG).  tol <= 0 selects OPE_REF_TOL; NaN or infinity is
 * OPE_ERR_INVALID_ARG.  Stream-ordered on `stream` (cudaStream_t, NULL =
 * legacy default stream).  The first call on a device does the set-up, with
 * that device current: it looks up the array's device address and sets up
 * both models' kernels; make that first call before any stream capture.
 * Every call shares the one array, so calls whose work overlaps on the GPU
 * race: serialise them on one stream (or order them with events). */
#define OPE_NOALLOC_MAX_CONTRACTS 65536
int ope_price_surfaces_noalloc(int32_t model, const ope_contract* d_contracts, size_t n,
                               const int64_t* d_surf_offsets, size_t n_surf, const void* d_params,
                               double* d_out_prices, double tol, void* stream);

/* No counterpart in the reference (its batch calls hand contracts to
 * rayon's work-stealing pool, batch.rs:23-42): the launch-shape autotuner of
 * the pricing kernel.  A shape is the persistent grid's warps per block (each
 * warp integrates one of a contract's two integrals), whether the work queue
 * takes contracts deepest-first (by |ln(K/S)| / sqrt(v0 T)) or in input
 * order, and the share of the resident blocks per SM the grid fills.  Every
 * shape gives bit-identical prices; only the time differs.
 * ope_autotune measures every candidate shape (1, 2 or 4 warps x order x
 * occupancy 1 or 1/2) on seeded synthetic batches of each size class (at the
 * class's geometric interior) on the calling thread's device, keeps per class
 * the fastest shape if it beats the default (4, input order, 1) by more than
 * 3 %, installs the table for that device and model in this process, and
 * writes the OPE_TUNE_CLASSES entries to out_entries (may be NULL).  Takes
 * about 10 s (about 1 s with OPE_TUNE_QUICK).  Plain pricing calls (ope_batch_*,
 * ope_price_surfaces, Greeks, the server's reprices) then launch with their
 * class's shape; calibration passes keep the default shape.
 * ope_set_autotune(0) returns every call to the default shape (1: the tuned
 * tables again); ope_get_tune_table reads the current device's table
 * (*out_tuned = 0: not tuned, the default entries); ope_set_tune_table
 * installs one. */
typedef struct {
    int32_t warps_per_block; /* 1, 2 or 4 */
    int32_t deepest_first;   /* 1: queue deepest-first, 0: input order */
    double occupancy;        /* share of the resident blocks per SM, (0, 1] */
    int32_t per_unit;        /* contracts per work unit, 0..32.  1: one.  From 2, a warp integrates blocks
                              * of that many consecutive contracts, and a run of contracts of one parameter
                              * set with the same expiry and rate (the strikes of one expiry of a surface
                              * laid out expiry by expiry) evaluates the characteristic function once per
                              * panel for the whole run (4 warps, input order).  0 (the default):
                              * automatic -- a call of 32,768 contracts or more counts its runs on the
                              * device and takes blocks of 16 when they average 4 contracts or more.
                              * Prices are bit-identical in every mode. */
    int32_t reserved;        /* 0 */
} ope_launch_shape;
typedef struct {
    uint64_t max_contracts;  /* the class: calls of at most this many contracts (the last: all larger) */
    ope_launch_shape shape;  /* the shape calls of this class use */
    double ms_default;       /* measured kernel time of the default shape on the class's batch */
    double ms_tuned;         /* measured kernel time of `shape` (ms_default when it is the default) */
} ope_tune_entry;
#define OPE_TUNE_CLASSES 16  /* calls of up to 64, 128, 256, ..., 2^20 contracts, and larger */
#define OPE_TUNE_QUICK 1u    /* ope_autotune flag: measure the classes up to 2^17 contracts only (the
                              * larger ones keep the default shape) */
int ope_autotune(int32_t model, uint32_t flags, ope_tune_entry* out_entries);
/* Contracts per unit that this thread's last plain pricing call launched
 * with (1: one per unit; for an automatic launch, the run probe's choice --
 * read after that call's work, so it waits for it).  Ask before the thread's
 * next call. */
int ope_last_per_unit(int32_t* out_per_unit);
int ope_set_autotune(int32_t enabled);
int ope_get_tune_table(int32_t model, ope_tune_entry* out_entries, int32_t* out_tuned);
/* Installs OPE_TUNE_CLASSES entries (e.g. a table saved from
 * ope_get_tune_table in an earlier process) as the current device's tuned
 * table for `model`; each shape must be valid (1, 2 or 4 warps; 0 or 1;
 * occupancy in (0, 1]; per_unit 0..32), max_contracts is ignored. */
int ope_set_tune_table(int32_t model, const ope_tune_entry* entries);

/* No reference twin (diagnostic of heston.rs:193-212 adaptive_gk): the step
 * by step record of the greedy GK15 quadrature on integral `which` (0 = P1,
 * 1 = P2) of one contract, made by the pricing kernel's own warp routine and
 * node evaluation.  Host pointers; synchronous.  Per step j (0 = the first
 * panel [0, 1], j >= 1 = the j-th bisection) OPE_TRACE_FIELDS doubles:
 * a, b and the error estimate of the bisected panel (0, 1, 0 at j = 0); K and
 * error estimate of the left and right children (j = 0: the first panel's K
 * and error, 0, 0); the running error and total after the step; the 15
 * integrand values of the left child and the 15 of the right child (zeros at
 * j = 0).  At most min(max_steps, OPE_MAX_PANELS) steps are written;
 * *out_n_steps receives the number of steps the integral took and
 * *out_integral the integral.  tol <= 0 selects OPE_REF_TOL. */
#define OPE_TRACE_FIELDS 39
int ope_trace_integral(int32_t model, const ope_contract* contract, const void* params, int32_t which, double tol,
                       double* out_steps, int32_t max_steps, int32_t* out_n_steps, double* out_integral);

/* No reference twin (numerics self-check): the worst error, in ulps, of the
 * kernels' Newton-refined reciprocal and square root against IEEE 1/x and
 * sqrt over 2^20 inputs spanning 1e-300 .. 1e300. */
int ope_selftest_math(uint64_t* max_ulp_rcp, uint64_t* max_ulp_sqrt);

/* No reference twin (numerics self-check): the worst difference, in ulps, of
 * the node evaluation's own branch-free atan2 (used for arg A of the Albrecher
 * CF, heston.rs:120) from CUDA's atan2 over 2^24 argument pairs with
 * magnitudes 2^-60 .. 2^60 and ratios 2^-45 .. 2^45. */
int ope_selftest_atan2(uint64_t* max_ulp);

/* No reference twin (numerics self-check): the worst difference, in ulps, of
 * the node evaluation's own log (used for log|A| of the Albrecher CF,
 * heston.rs:120) from CUDA's log over 2^24 arguments from 2^-1000 to 2^1000
 * and around 1. */
int ope_selftest_log(uint64_t* max_ulp);

/* No reference twin (numerics self-check of heston.rs:223, u = (1 - t)/t):
 * the number of 2^24 node positions t, uniform in (0, 1) and log-uniform down
 * to 2^-200, at which the kernels' u differs from the IEEE quotient. */
int ope_selftest_node_u(uint64_t* mismatches);

/* No reference twin (numerics self-check of heston.rs:86, x = ln(S/K)): the
 * kernels' correctly rounded logarithm, and CUDA's log for comparison, of n
 * host arguments (n <= 2^26).  The pricing kernels take x from the former, so
 * that it rounds as the platform libm's log does in the reference. */
int ope_selftest_log_cr(const double* args, size_t n, double* out_log_cr, double* out_log_cuda);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* OPE_H */
