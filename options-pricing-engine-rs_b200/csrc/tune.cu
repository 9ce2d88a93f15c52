// Launch-shape autotuner of the pricing kernel (no counterpart in the
// reference, whose batch calls hand contracts to rayon's work-stealing pool,
// batch.rs:23-42).
//
// A call's pricing time depends on its launch shape mostly through its tail:
// the integrals take 0 to 199 bisections each, serial chains of panel steps,
// and a call is done when its deepest chain is.  The tuner measures, on the
// device in use, every candidate shape on seeded synthetic batches of each
// size class (powers of two from 64 to 2^20 contracts, and larger;
// benchmark-configuration parameter ranges)
// and keeps, per class, the fastest shape when it beats the default by more
// than 3 % (else the default):
//   * warps per block: 1, 2 or 4 (each warp one integral), i.e. how finely
//     a small call's units spread over the SMs;
//   * queue order: input order, or deepest-first by |ln(K/S)| / sqrt(v0 T);
//   * occupancy: all resident blocks per SM, or half (fewer warps sharing an
//     SM sub-partition run each chain faster).
// The panel list keeps the reference's 200-panel capacity (a smaller one
// would change results; shared memory does not limit occupancy at the
// 64-register budget), and each integral keeps one warp (several warps per
// integral were measured slower).  The table lives per device in this
// process; ope_autotune fills it, ope_set_autotune switches it on or off.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "internal.h"

namespace ope {

namespace {

struct TuneTable {
    bool tuned[2] = {false, false};
    ope_tune_entry e[2][kTuneClasses];
};

std::mutex g_mu;
std::map<int, TuneTable> g_tables;
std::atomic<int> g_enabled{1};

int class_of(size_t n) {
    int i = 0;
    while (i < kTuneClasses - 1 && n > kTuneClassMax[i]) ++i;
    return i;
}

// Size measured for each class: the class's geometric interior, 2^(k - 1/2)
// for the class (2^(k-1), 2^k] (the last class, above 2^20: 1.5 x 2^20).
constexpr size_t kClassN[kTuneClasses] = {45,    91,    181,    362,    724,    1448,   2896,   5793,
                                          11585, 23170, 46341, 92682, 185364, 370728, 741455, 1572864};
// OPE_TUNE_QUICK measures the classes up to 2^17 contracts only.
constexpr int kQuickClasses = 12;

// splitmix64 stream of uniform doubles in [0, 1)
struct Rng {
    uint64_t s;
    double uniform() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        return (double)(z >> 11) * 0x1.0p-53;
    }
    double range(double lo, double hi) { return lo + (hi - lo) * uniform(); }
};

// Synthetic batch of n contracts in surfaces of up to 256: the benchmark
// configurations' ranges (Bates: the deep-wing batch, ln(K/F) in [-1.2, 0.7],
// T log-uniform in [1/365, 3] y, jumps; Heston: the uneven-grid batch,
// ln(K/F) in [-0.8, 0.5], T log-uniform in [1/252, 5] y).
void synth(int model, size_t n, uint64_t seed, std::vector<ope_contract>& con, std::vector<int64_t>& off,
           std::vector<double>& par) {
    const bool bates = model == OPE_MODEL_BATES;
    const int dim = bates ? 8 : 5;
    Rng g{seed};
    const size_t per = std::min<size_t>(256, n);
    const size_t ns = (n + per - 1) / per;
    con.resize(n);
    off.assign(ns + 1, 0);
    par.resize(ns * dim);
    for (size_t s = 0; s < ns; ++s) {
        double* p = &par[s * dim];
        p[0] = g.range(0.01, 0.2);
        p[1] = g.range(0.2, 5.0);
        p[2] = g.range(0.01, 0.2);
        p[3] = g.range(0.1, 1.0);
        p[4] = g.range(-0.95, 0.2);
        if (bates) {
            p[5] = g.range(0.0, 1.5);
            p[6] = g.range(-0.3, 0.1);
            p[7] = g.range(0.05, 0.4);
        }
        const double r = g.range(0.0, 0.06), q = g.range(0.0, 0.03);
        off[s] = (int64_t)(s * per);
        off[s + 1] = (int64_t)std::min(n, (s + 1) * per);
        for (size_t c = s * per; c < std::min(n, (s + 1) * per); ++c) {
            const double t = bates ? std::exp(g.range(std::log(1.0 / 365.0), std::log(3.0)))
                                   : std::exp(g.range(std::log(1.0 / 252.0), std::log(5.0)));
            const double m = bates ? g.range(-1.2, 0.7) : g.range(-0.8, 0.5);
            ope_contract k{};
            k.spot = 100.0;
            k.strike = 100.0 * std::exp((r - q) * t + m);
            k.expiry = t;
            k.rate = r;
            k.div_yield = q;
            k.vol = 0.2;
            k.opt_type = g.uniform() < 0.5 ? OPE_CALL : OPE_PUT;
            con[c] = k;
        }
    }
}

ope_tune_entry default_entry(int cls) {
    ope_tune_entry e{};
    e.max_contracts = kTuneClassMax[cls];
    e.shape.warps_per_block = 4;
    e.shape.deepest_first = 0;
    e.shape.occupancy = 1.0;
    e.shape.per_unit = 0;
    e.shape.reserved = 0;
    e.ms_default = 0.0;
    e.ms_tuned = 0.0;
    return e;
}

struct DevBatch {
    ope_contract* con = nullptr;
    int64_t* off = nullptr;
    double* par = nullptr;
    double* out = nullptr;
    void* scratch = nullptr;
};

// Median kernel time (ms) of `reps` launches of one shape, after `warm`.
int time_shape(int model, const DevBatch& B, size_t n, size_t ns, double tol, const LaunchShape& sh, int warm,
               int reps, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, double* ms) {
    const PriceScratch s = carve_price_scratch(B.scratch, n);
    std::vector<float> t(reps);
    for (int i = 0; i < warm + reps; ++i) {
        OPE_CHECK(cudaEventRecord(e0, st));
        OPE_TRY(launch_price_persistent(model, B.con, n, B.off, ns, nullptr, B.par, tol, B.out, s, st, nullptr,
                                        nullptr, nullptr, &sh));
        OPE_CHECK(cudaEventRecord(e1, st));
        OPE_CHECK(cudaEventSynchronize(e1));
        if (i >= warm) OPE_CHECK(cudaEventElapsedTime(&t[i - warm], e0, e1));
    }
    std::sort(t.begin(), t.end());
    *ms = t[reps / 2];
    return OPE_OK;
}

}  // namespace

LaunchShape price_shape(int model, size_t n) {
    LaunchShape sh;
    if (!g_enabled.load(std::memory_order_relaxed)) return sh;
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return sh;
    }
    const int m = model == OPE_MODEL_BATES ? 1 : 0;
    std::lock_guard<std::mutex> g(g_mu);
    const auto it = g_tables.find(dev);
    if (it == g_tables.end() || !it->second.tuned[m]) return sh;
    const ope_tune_entry& e = it->second.e[m][class_of(n)];
    sh.warps = e.shape.warps_per_block;
    sh.deepest_first = e.shape.deepest_first;
    sh.occupancy = e.shape.occupancy;
    sh.per_unit = e.shape.per_unit;
    return sh;
}

}  // namespace ope

using namespace ope;

extern "C" {

int ope_autotune(int32_t model, uint32_t flags, ope_tune_entry* out_entries) {
    OPE_RANGE("ope.autotune");
    if (model != OPE_MODEL_HESTON && model != OPE_MODEL_BATES)
        return set_error(OPE_ERR_INVALID_ARG, "model must be OPE_MODEL_HESTON or OPE_MODEL_BATES");
    OPE_TRY(ensure_device());
    ThreadCtx& c = tctx();
    const int n_cls = (flags & OPE_TUNE_QUICK) ? kQuickClasses : kTuneClasses;
    const size_t nmax = kClassN[n_cls - 1];
    std::vector<ope_contract> con;
    std::vector<int64_t> off;
    std::vector<double> par;
    synth(model, nmax, 0x5EEDull + (uint64_t)model, con, off, par);
    // the tuner's own buffers, stream-ordered on this thread's stream, freed before it returns
    DevBatch B;
    const size_t b_con = align_up(nmax * sizeof(ope_contract), 256), b_off = align_up(off.size() * 8, 256),
                 b_par = align_up(par.size() * 8, 256), b_out = align_up(nmax * 8, 256);
    const size_t total = b_con + b_off + b_par + b_out + price_scratch_bytes(nmax);
    char* base = nullptr;
    OPE_CHECK(cudaMallocAsync(reinterpret_cast<void**>(&base), total, c.stream));
    B.con = reinterpret_cast<ope_contract*>(base);
    B.off = reinterpret_cast<int64_t*>(base + b_con);
    B.par = reinterpret_cast<double*>(base + b_con + b_off);
    B.out = reinterpret_cast<double*>(base + b_con + b_off + b_par);
    B.scratch = base + b_con + b_off + b_par + b_out;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = OPE_OK;
    TuneTable T;
    {
        std::lock_guard<std::mutex> g(g_mu);
        int dev = c.device;
        if (g_tables.count(dev)) T = g_tables[dev];
    }
    const int m = model == OPE_MODEL_BATES ? 1 : 0;
    for (int i = 0; i < kTuneClasses; ++i) T.e[m][i] = default_entry(i);
    do {
        if ((rc = check_cuda(cudaEventCreate(&e0), "cudaEventCreate")) != OPE_OK) break;
        if ((rc = check_cuda(cudaEventCreate(&e1), "cudaEventCreate")) != OPE_OK) break;
        if ((rc = check_cuda(cudaMemcpyAsync(B.con, con.data(), nmax * sizeof(ope_contract), cudaMemcpyHostToDevice,
                                             c.stream), "cudaMemcpyAsync")) != OPE_OK)
            break;
        if ((rc = check_cuda(cudaMemcpyAsync(B.par, par.data(), par.size() * 8, cudaMemcpyHostToDevice, c.stream),
                             "cudaMemcpyAsync")) != OPE_OK)
            break;
        for (int cls = 0; cls < n_cls && rc == OPE_OK; ++cls) {
            // the first n contracts: whole surfaces, offsets of this prefix
            const size_t n = kClassN[cls];
            const size_t per = std::min<size_t>(256, n);
            const size_t ns = (n + per - 1) / per;
            std::vector<int64_t> o(ns + 1);
            for (size_t s = 0; s <= ns; ++s) o[s] = (int64_t)std::min(n, s * per);
            if ((rc = check_cuda(cudaMemcpyAsync(B.off, o.data(), o.size() * 8, cudaMemcpyHostToDevice, c.stream),
                                 "cudaMemcpyAsync")) != OPE_OK)
                break;
            const int warm = n >= 185364 ? 1 : 3, reps = n >= 185364 ? 3 : (n >= 11585 ? 5 : 9);
            LaunchShape def;
            double t_def = 0.0;
            if ((rc = time_shape(model, B, n, ns, 1e-10, def, warm, reps, c.stream, e0, e1, &t_def)) != OPE_OK) break;
            LaunchShape best = def;
            double t_best = t_def;
            for (int w : {1, 2, 4})
                for (int df : {0, 1})
                    for (double occ : {1.0, 0.5}) {
                        const LaunchShape sh{w, df, occ};
                        if (w == 4 && df == 0 && occ == 1.0) continue;
                        double t = 0.0;
                        if ((rc = time_shape(model, B, n, ns, 1e-10, sh, warm, reps, c.stream, e0, e1, &t)) != OPE_OK)
                            break;
                        if (t < t_best) {
                            t_best = t;
                            best = sh;
                        }
                    }
            if (rc != OPE_OK) break;
            ope_tune_entry& e = T.e[m][cls];
            e.ms_default = t_def;
            if (t_best < 0.97 * t_def) {
                e.shape.warps_per_block = best.warps;
                e.shape.deepest_first = best.deepest_first;
                e.shape.occupancy = best.occupancy;
                e.shape.per_unit = best.per_unit;
                e.ms_tuned = t_best;
            } else {
                e.ms_tuned = t_def;
            }
        }
    } while (false);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    const int rc_free = check_cuda(cudaFreeAsync(base, c.stream), "cudaFreeAsync");
    if (rc == OPE_OK) rc = rc_free;
    if (rc == OPE_OK) rc = check_cuda(cudaStreamSynchronize(c.stream), "cudaStreamSynchronize");
    if (rc != OPE_OK) return rc;
    T.tuned[m] = true;
    {
        std::lock_guard<std::mutex> g(g_mu);
        g_tables[c.device] = T;
    }
    if (out_entries)
        for (int i = 0; i < kTuneClasses; ++i) out_entries[i] = T.e[m][i];
    return OPE_OK;
}

int ope_set_autotune(int32_t enabled) {
    g_enabled.store(enabled ? 1 : 0);
    return OPE_OK;
}

int ope_set_tune_table(int32_t model, const ope_tune_entry* entries) {
    if (model != OPE_MODEL_HESTON && model != OPE_MODEL_BATES)
        return set_error(OPE_ERR_INVALID_ARG, "model must be OPE_MODEL_HESTON or OPE_MODEL_BATES");
    if (!entries) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    for (int i = 0; i < kTuneClasses; ++i) {
        const ope_launch_shape& sh = entries[i].shape;
        if (sh.warps_per_block != 1 && sh.warps_per_block != 2 && sh.warps_per_block != 4)
            return set_error(OPE_ERR_INVALID_ARG, "warps_per_block must be 1, 2 or 4");
        if (sh.deepest_first != 0 && sh.deepest_first != 1)
            return set_error(OPE_ERR_INVALID_ARG, "deepest_first must be 0 or 1");
        if (!(sh.occupancy > 0.0 && sh.occupancy <= 1.0))
            return set_error(OPE_ERR_INVALID_ARG, "occupancy must be in (0, 1]");
        if (sh.per_unit < 0 || sh.per_unit > 32) return set_error(OPE_ERR_INVALID_ARG, "per_unit must be in 0..32");
    }
    OPE_TRY(ensure_device());
    const int m = model == OPE_MODEL_BATES ? 1 : 0;
    std::lock_guard<std::mutex> g(g_mu);
    TuneTable& T = g_tables[tctx().device];
    for (int i = 0; i < kTuneClasses; ++i) {
        T.e[m][i] = entries[i];
        T.e[m][i].max_contracts = kTuneClassMax[i];
    }
    T.tuned[m] = true;
    return OPE_OK;
}

int ope_last_per_unit(int32_t* out_per_unit) {
    if (!out_per_unit) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    ThreadCtx& c = tctx();
    if (!c.last_probe) {
        *out_per_unit = c.last_per_unit;
        return OPE_OK;
    }
    unsigned long long v = 0;
    OPE_CHECK(cudaStreamSynchronize(c.last_probe_stream));
    OPE_CHECK(cudaMemcpy(&v, c.last_probe, sizeof(v), cudaMemcpyDeviceToHost));
    *out_per_unit = v ? (int32_t)v : 1;
    return OPE_OK;
}

int ope_get_tune_table(int32_t model, ope_tune_entry* out_entries, int32_t* out_tuned) {
    if (model != OPE_MODEL_HESTON && model != OPE_MODEL_BATES)
        return set_error(OPE_ERR_INVALID_ARG, "model must be OPE_MODEL_HESTON or OPE_MODEL_BATES");
    if (!out_entries || !out_tuned) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    OPE_TRY(ensure_device());
    const int m = model == OPE_MODEL_BATES ? 1 : 0;
    std::lock_guard<std::mutex> g(g_mu);
    const auto it = g_tables.find(tctx().device);
    const bool tuned = it != g_tables.end() && it->second.tuned[m];
    for (int i = 0; i < kTuneClasses; ++i) out_entries[i] = tuned ? it->second.e[m][i] : default_entry(i);
    *out_tuned = tuned ? 1 : 0;
    return OPE_OK;
}

}  // extern "C"
