// Multistart and differential-evolution (global) calibration on the device.
//
// Reference: calibration.rs:246-314 (calibrate_multistart), 316-427
// (calibrate_global, DE/rand/1/bin + LM polish), 131-141 / 179-185
// (CalibModel::random_guess), 115-126 / 158-173 (bounds), mc.rs:337-343
// (splitmix64), and the random-number generator of rand 0.8 (below).
//
// Multistart: every restart of every surface is one surface of ONE batched
// device LM run (calib.cu) over replicated quotes, with the restarts of a
// surface in one pruning group, so all of them advance in lockstep inside
// one conditional-WHILE graph.
//
// DE: a member's fitness is the weighted IV-space SSE of the surface's
// quotes at the member's parameters (INFINITY out of bounds).  All members
// of all surfaces are priced by one persistent pricing launch per generation
// (each member a "surface" of its own over a replicated copy of the quotes,
// out-of-bounds trials masked off), followed by an IV-residual kernel and a
// per-member selection kernel; the generation loop is one CUDA graph with a
// conditional WHILE node.  Trials are built on the device from the
// generation's own seeded generator exactly as the reference builds them, so
// the population evolves as the reference's does up to the pricing's
// rounding.  The polish is the batched device LM (calib.cu), regularised
// when a prior is given.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "internal.h"
#include "iv_device.cuh"

namespace ope {

namespace {

// ---------------------------------------------------------------------------
// rand 0.8 SmallRng (on 64-bit targets: xoshiro256++, Blackman & Vigna)
// seeded by rand_core 0.6's default SeedableRng::seed_from_u64 (eight PCG32
// XSH-RR outputs, little endian; SmallRng does not forward seed_from_u64 to
// the inner generator), and the samplers calibration.rs calls:
//   gen::<f64>()            (next >> 11) * 2^-53
//   gen_range(lo..hi), f64  v in [1, 2) from the top 52 bits of next,
//                           (v - 1) * (hi - lo) + lo, redrawn while >= hi
//   gen_range(0..n), usize  widening multiply, rejected while the low word
//                           exceeds (n << leading_zeros(n)) - 1
// The reference's lock file does not pin rand (Cargo.toml:19 asks for 0.8),
// so these follow the published 0.8.5 algorithms.
// ---------------------------------------------------------------------------
struct SmallRng {
    uint64_t s[4];
};

__host__ __device__ inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__host__ __device__ inline uint64_t splitmix64(uint64_t x) { return mix64(x + 0x9e3779b97f4a7c15ull); }

__host__ __device__ inline SmallRng rng_from_u64(uint64_t state) {
    SmallRng r;
    for (int k = 0; k < 4; ++k) {
        uint64_t word = 0;
        for (int half = 0; half < 2; ++half) {
            state = state * 6364136223846793005ull + 11634580027462260723ull;
            const uint32_t xs = (uint32_t)(((state >> 18) ^ state) >> 27);
            const uint32_t rot = (uint32_t)(state >> 59);
            const uint32_t x = (xs >> rot) | (xs << ((32u - rot) & 31u));
            word |= (uint64_t)x << (32 * half);
        }
        r.s[k] = word;
    }
    if ((r.s[0] | r.s[1] | r.s[2] | r.s[3]) == 0) {  // xoshiro256++'s own seeding of 0
        uint64_t st = 0;
        for (int k = 0; k < 4; ++k) {
            st += 0x9e3779b97f4a7c15ull;
            r.s[k] = mix64(st);
        }
    }
    return r;
}

__host__ __device__ inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

__host__ __device__ inline uint64_t rng_next(SmallRng& r) {
    const uint64_t out = rotl64(r.s[0] + r.s[3], 23) + r.s[0];
    const uint64_t t = r.s[1] << 17;
    r.s[2] ^= r.s[0];
    r.s[3] ^= r.s[1];
    r.s[1] ^= r.s[2];
    r.s[0] ^= r.s[3];
    r.s[2] ^= t;
    r.s[3] = rotl64(r.s[3], 45);
    return out;
}

__host__ __device__ inline double rng_unit(SmallRng& r) {
    return (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0);  // exact: 53-bit integer x 2^-53
}

__host__ __device__ inline uint64_t mulhi64(uint64_t a, uint64_t b) {
#ifdef __CUDA_ARCH__
    return __umul64hi(a, b);
#else
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

__host__ __device__ inline int clz64(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

// gen_range(0..n), n >= 1.  The rejection zone keeps at least half of all
// draws, so 64 draws fail with probability < 2^-64; false then (the caller
// reports it) instead of looping without bound.
__host__ __device__ inline bool rng_below(SmallRng& r, uint64_t n, uint64_t* out) {
    const uint64_t zone = (n << clz64(n)) - 1;
    for (int t = 0; t < 64; ++t) {
        const uint64_t v = rng_next(r);
        if (v * n <= zone) {
            *out = mulhi64(v, n);
            return true;
        }
    }
    return false;
}

// gen_range(lo..hi) on f64 (host only: the initial population and restarts).
double rng_uniform(SmallRng& r, double lo, double hi) {
    const double scale = hi - lo;
    for (;;) {
        const uint64_t bits = (rng_next(r) >> 12) | 0x3ff0000000000000ull;
        double v;
        std::memcpy(&v, &bits, sizeof(v));
        const double res = (v - 1.0) * scale + lo;  // host code is built without FMA contraction
        if (res < hi) return res;
    }
}

// calibration.rs:131-141, 179-185
void random_guess(int dim, SmallRng& r, double* v) {
    v[0] = rng_uniform(r, 0.005, 0.5);
    v[1] = rng_uniform(r, 0.3, 8.0);
    v[2] = rng_uniform(r, 0.005, 0.5);
    const double cap = std::fmax(std::sqrt((2.0 * v[1]) * v[2]) * 0.9, 0.05);
    v[3] = rng_uniform(r, 0.02, cap);
    v[4] = rng_uniform(r, -0.9, 0.9);
    if (dim == 8) {
        v[5] = rng_uniform(r, 0.0, 2.0);
        v[6] = rng_uniform(r, -0.3, 0.1);
        v[7] = rng_uniform(r, 0.02, 0.4);
    }
}

// calibration.rs:124-126, 169-173 param_bounds
__host__ __device__ inline void param_bounds(int k, double* lo, double* hi) {
    constexpr double L[8] = {1e-8, 1e-6, 1e-8, 1e-6, -0.9999, 0.0, -2.0, 1e-6};
    constexpr double H[8] = {5.0, 50.0, 5.0, 10.0, 0.9999, 10.0, 2.0, 2.0};
    *lo = L[k];
    *hi = H[k];
}

// calibration.rs:115-122, 158-163 bounds_ok (Feller: types.rs:60-62)
__host__ __device__ inline bool in_bounds(const double* v, int dim) {
    const bool feller = (2.0 * v[1]) * v[2] > v[3] * v[3];
    const bool h = feller && v[0] > 1e-8 && v[0] < 5.0 && v[1] > 1e-6 && v[1] < 50.0 && v[2] > 1e-8 &&
                   v[2] < 5.0 && v[3] > 1e-6 && v[3] < 10.0 && v[4] > -0.9999 && v[4] < 0.9999;
    if (dim == 5) return h;
    return h && v[5] >= 0.0 && v[5] < 10.0 && fabs(v[6]) < 2.0 && v[7] > 1e-6 && v[7] < 2.0;
}

// f64::total_cmp order as a signed key
__host__ __device__ inline long long total_key(double x) {
#ifdef __CUDA_ARCH__
    long long b = __double_as_longlong(x);
#else
    long long b;
    std::memcpy(&b, &x, sizeof(b));
#endif
    return b ^ (long long)(((unsigned long long)(b >> 63)) >> 1);
}

// ---------------------------------------------------------------------------
// DE on the device
// ---------------------------------------------------------------------------
constexpr double kDeF = 0.6, kDeCr = 0.9;  // calibration.rs:324-325

struct DEDev {
    const ope_contract* con;  // replicated quotes: member u owns [off[u], off[u+1])
    const int32_t* unit;      // member of each replicated quote
    const int32_t* qidx;      // original quote of each replicated quote
    const int64_t* off;
    const double* iv;         // market IVs (original quotes)
    const double* w;          // weights (original quotes)
    double* pop;              // members x dim
    double* fit;              // members
    double* trial;            // members x dim
    int32_t* mask;            // members: trial in bounds (priced)
    double* price;            // replicated quotes
    double* res;              // replicated quotes
    int* state;               // [0] generation, [1] sampler gave up
    int ns, np, dim, n_gen;
    long long nr;
    unsigned long long seed;
};

// One trial per member (calibration.rs:370-392): the generator of (gen, i),
// three distinct partners other than i, one forced dimension, binomial
// crossover, clamped to the box.
__global__ void k_de_trials(DEDev D) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= D.ns * D.np) return;
    const int s = u / D.np, i = u - s * D.np;
    const int dim = D.dim;
    const unsigned long long gen = (unsigned long long)D.state[0];
    SmallRng rng = rng_from_u64(splitmix64(D.seed ^ (gen << 32) ^ (unsigned long long)i));
    uint64_t idx[3] = {0, 0, 0};
    bool ok = true;
    for (int slot = 0; slot < 3 && ok; ++slot) {
        bool found = false;
        for (int t = 0; t < 64 && !found && ok; ++t) {
            uint64_t cand;
            ok = rng_below(rng, (uint64_t)D.np, &cand);
            if (!ok) break;
            bool seen = false;
            for (int k = 0; k < slot; ++k) seen = seen || idx[k] == cand;
            if (cand != (uint64_t)i && !seen) {
                idx[slot] = cand;
                found = true;
            }
        }
        ok = ok && found;
    }
    uint64_t forced = 0;
    ok = ok && rng_below(rng, (uint64_t)dim, &forced);
    double* tr = D.trial + (size_t)u * dim;
    const double* me = D.pop + (size_t)u * dim;
    for (int d = 0; d < dim; ++d) tr[d] = me[d];
    if (!ok) {  // probability < 2^-64 per draw; reported to the host
        atomicExch(D.state + 1, 1);
        D.mask[u] = 0;
        return;
    }
    const double* pa = D.pop + ((size_t)s * D.np + idx[0]) * dim;
    const double* pb = D.pop + ((size_t)s * D.np + idx[1]) * dim;
    const double* pc = D.pop + ((size_t)s * D.np + idx[2]) * dim;
    for (int d = 0; d < dim; ++d) {
        if ((uint64_t)d == forced || rng_unit(rng) < kDeCr) {
            double lo, hi;
            param_bounds(d, &lo, &hi);
            double v = __dadd_rn(pa[d], __dmul_rn(kDeF, __dsub_rn(pb[d], pc[d])));
            if (v < lo) v = lo;  // f64::clamp
            if (v > hi) v = hi;
            tr[d] = v;
        }
    }
    D.mask[u] = in_bounds(tr, dim) ? 1 : 0;
}

// The initial population's "trials" are the members themselves.
__global__ void k_de_init(DEDev D) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= D.ns * D.np) return;
    for (int d = 0; d < D.dim; ++d) D.trial[(size_t)u * D.dim + d] = D.pop[(size_t)u * D.dim + d];
    D.mask[u] = in_bounds(D.pop + (size_t)u * D.dim, D.dim) ? 1 : 0;
}

// calibration.rs:573-581: IV residual of every replicated quote of a priced member.
__global__ void k_de_resid(DEDev D) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.nr) return;
    if (D.mask[D.unit[i]] == 0) return;
    double iv;
    D.res[i] = implied_vol_d(iv_contract(D.con[i]), D.price[i], &iv) ? iv - D.iv[D.qidx[i]] : 0.0;
}

// Fitness (calibration.rs:355-359, 589-591: weighted SSE summed in quote
// order, INFINITY out of bounds) and greedy selection (calibration.rs:391).
// init: the fitness of the initial population (calibration.rs:369).
__global__ void k_de_select(DEDev D, int init, cudaGraphConditionalHandle handle) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u < D.ns * D.np) {
        double sse = __longlong_as_double(0x7ff0000000000000ll);
        if (D.mask[u]) {
            sse = 0.0;
            for (long long i = D.off[u]; i < D.off[u + 1]; ++i) {
                const double t = D.w[D.qidx[i]] * D.res[i];
                sse = __dadd_rn(sse, __dmul_rn(t, t));
            }
        }
        if (init) {
            D.fit[u] = sse;
        } else if (sse < D.fit[u]) {
            for (int d = 0; d < D.dim; ++d) D.pop[(size_t)u * D.dim + d] = D.trial[(size_t)u * D.dim + d];
            D.fit[u] = sse;
        }
    }
    if (!init && u == 0) {  // no thread of this kernel reads the generation counter
        const int g = D.state[0] + 1;
        D.state[0] = g;
        cudaGraphSetConditional(handle, g < D.n_gen ? 1u : 0u);
    }
}

// Per surface: the first member of minimal fitness (min_by(total_cmp)).
__global__ void k_de_best(DEDev D, double* best_sse, double* winner) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= D.ns) return;
    const int base = s * D.np;
    int b = 0;
    for (int i = 1; i < D.np; ++i)
        if (total_key(D.fit[base + i]) < total_key(D.fit[base + b])) b = i;
    best_sse[s] = D.fit[base + b];
    for (int d = 0; d < D.dim; ++d) winner[s * D.dim + d] = D.pop[(size_t)(base + b) * D.dim + d];
}

int enqueue_generation(int model, const DEDev& D, const PriceScratch& ps, double tol, cudaStream_t st,
                       cudaGraphConditionalHandle handle, bool init) {
    const int members = D.ns * D.np;
    const int mb = (members + 127) / 128;
    if (init) k_de_init<<<mb, 128, 0, st>>>(D);
    else k_de_trials<<<mb, 128, 0, st>>>(D);
    OPE_CHECK(cudaGetLastError());
    OPE_TRY(launch_price_persistent(model, D.con, (size_t)D.nr, D.off, (size_t)members, nullptr, D.trial, tol,
                                    D.price, ps, st, nullptr, D.mask));
    k_de_resid<<<(unsigned)((D.nr + 127) / 128), 128, 0, st>>>(D);
    OPE_CHECK(cudaGetLastError());
    k_de_select<<<mb, 128, 0, st>>>(D, init ? 1 : 0, handle);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 3;
    return OPE_OK;
}

// The generation loop as one graph: a conditional WHILE node whose body is
// one generation (trials, pricing, residuals, selection).
int run_generations(int model, const DEDev& D, const PriceScratch& ps, double tol, cudaStream_t st) {
    cudaGraph_t g;
    OPE_CHECK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle handle;
    cudaError_t e = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return check_cuda(e, "cudaGraphConditionalHandleCreate"); }
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return check_cuda(e, "cudaGraphAddNode"); }
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return check_cuda(e, "cudaStreamBeginCaptureToGraph"); }
    const int rc = enqueue_generation(model, D, ps, tol, st, handle, false);
    cudaGraph_t captured = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(st, &captured);
    if (rc != OPE_OK) { cudaGraphDestroy(g); return rc; }
    if (ec != cudaSuccess) { cudaGraphDestroy(g); return check_cuda(ec, "cudaStreamEndCapture"); }
    cudaGraphExec_t exec;
    e = cudaGraphInstantiate(&exec, g, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return check_cuda(e, "cudaGraphInstantiate"); }
    e = cudaGraphLaunch(exec, st);
    const cudaError_t es = cudaStreamSynchronize(st);
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return check_cuda(e, "cudaGraphLaunch");
    return check_cuda(es, "DE generations");
}

int check_offsets(const int64_t* off, size_t ns, size_t nq) {
    if (off[0] != 0 || off[ns] != (int64_t)nq) return set_error(OPE_ERR_INVALID_ARG, "surf_offsets must span [0, n)");
    for (size_t s = 0; s < ns; ++s) {
        if (off[s + 1] < off[s]) return set_error(OPE_ERR_INVALID_ARG, "surf_offsets not sorted");
        if (off[s + 1] == off[s]) return set_error(OPE_ERR_INVALID_ARG, "nothing to calibrate");  // calibration.rs:438
    }
    return OPE_OK;
}

}  // namespace

int run_multistart(int model, const ope_contract* quotes, const double* iv_market, const double* weights, size_t nq,
                   const int64_t* off, size_t ns, const double* p0, int n_restarts, uint64_t seed,
                   const double* shared_best0, ope_multistart_result* out, ope_calib_result* out_restarts,
                   double tol) {
    OPE_TRY(check_offsets(off, ns, nq));
    const int dim = param_stride(model);
    const size_t nr = (size_t)std::max(n_restarts, 1);  // calibration.rs:269
    // restart i > 0 starts at random_guess(SmallRng::seed_from_u64(splitmix64(seed ^ i))) (calibration.rs:277-283)
    std::vector<double> guess(nr * dim);
    for (size_t i = 1; i < nr; ++i) {
        SmallRng rng = rng_from_u64(splitmix64(seed ^ (uint64_t)i));
        random_guess(dim, rng, guess.data() + i * dim);
    }
    // LM surface s * nr + i = restart i of surface s, over its own copy of the quotes
    const size_t nq_rep = nq * nr, ns_rep = ns * nr;
    std::vector<ope_contract> con(nq_rep);
    std::vector<double> iv(nq_rep), w(nq_rep), p(ns_rep * dim);
    std::vector<int64_t> off_rep(ns_rep + 1);
    std::vector<int32_t> group(ns_rep);
    size_t at = 0;
    for (size_t s = 0; s < ns; ++s) {
        const size_t a = (size_t)off[s], len = (size_t)(off[s + 1] - off[s]);
        for (size_t i = 0; i < nr; ++i) {
            const size_t u = s * nr + i;
            off_rep[u] = (int64_t)at;
            std::memcpy(con.data() + at, quotes + a, len * sizeof(ope_contract));
            std::memcpy(iv.data() + at, iv_market + a, len * sizeof(double));
            for (size_t k = 0; k < len; ++k) w[at + k] = weights ? weights[a + k] : 1.0;
            std::memcpy(p.data() + u * dim, i == 0 ? p0 + s * dim : guess.data() + i * dim, dim * sizeof(double));
            group[u] = (int32_t)s;
            at += len;
        }
    }
    off_rep[ns_rep] = (int64_t)at;
    CalibExtra ex;
    ex.group = group.data();
    ex.gbest0 = shared_best0;
    ex.n_group = (int)ns;
    std::vector<ope_calib_result> res(ns_rep);
    OPE_TRY(run_calibration(model, con.data(), iv.data(), w.data(), nq_rep, off_rep.data(), ns_rep, p.data(),
                            res.data(), tol, false, nullptr, &ex));
    for (size_t s = 0; s < ns; ++s) {
        const ope_calib_result* r = res.data() + s * nr;
        int best = 0, n_conv = 0, n_pruned = 0;
        for (size_t i = 0; i < nr; ++i) {
            n_conv += r[i].converged;
            n_pruned += r[i].early_stopped;
            if (total_key(r[i].rmse) < total_key(r[best].rmse)) best = (int)i;  // min_by: first minimum
        }
        out[s].best = r[best];
        out[s].n_restarts = (int32_t)nr;
        out[s].n_converged = n_conv;
        out[s].n_pruned = n_pruned;
        out[s].best_restart = best;
    }
    if (out_restarts) std::memcpy(out_restarts, res.data(), ns_rep * sizeof(ope_calib_result));
    return OPE_OK;
}

int run_global(int model, const ope_contract* quotes, const double* iv_market, const double* weights, size_t nq,
               const int64_t* off, size_t ns, int n_pop, int n_gen, uint64_t seed, const double* prior,
               const double* reg_weight, ope_global_result* out, double tol) {
    OPE_TRY(check_offsets(off, ns, nq));
    if (n_gen < 0) return set_error(OPE_ERR_INVALID_ARG, "n_gen must be >= 0");
    if (prior && !reg_weight) return set_error(OPE_ERR_INVALID_ARG, "a prior needs its reg_weight");
    ThreadCtx& c = tctx();
    const int dim = param_stride(model);
    const int np = std::max(n_pop, 4 * dim);  // calibration.rs:353
    // Initial population (calibration.rs:361-368), the same for every surface:
    // up to 20 draws for a member whose SSE is finite, else a 21st draw.  With
    // finite market IVs and weights the SSE is finite exactly when the draw
    // is in bounds (residuals are IV differences or 0), so in_bounds decides.
    std::vector<double> pop0((size_t)np * dim);
    {
        SmallRng rng = rng_from_u64(splitmix64(seed));
        double lo[8], hi[8];
        for (int d = 0; d < dim; ++d) param_bounds(d, &lo[d], &hi[d]);
        for (int i = 0; i < np; ++i) {
            double* v = pop0.data() + (size_t)i * dim;
            bool got = false;
            for (int attempt = 0; attempt < 20 && !got; ++attempt) {
                for (int d = 0; d < dim; ++d) v[d] = rng_uniform(rng, lo[d], hi[d]);
                got = in_bounds(v, dim);
            }
            if (!got)
                for (int d = 0; d < dim; ++d) v[d] = rng_uniform(rng, lo[d], hi[d]);
        }
    }
    // Replicated quotes: member u = s * np + i owns a copy of surface s's quotes.
    const size_t members = ns * (size_t)np;
    const size_t nr = nq * (size_t)np;
    std::vector<ope_contract> con(nr);
    std::vector<int32_t> unit(nr), qidx(nr);
    std::vector<int64_t> off_rep(members + 1);
    std::vector<double> pop(members * dim);
    size_t at = 0;
    for (size_t s = 0; s < ns; ++s) {
        const size_t a = (size_t)off[s], len = (size_t)(off[s + 1] - off[s]);
        for (int i = 0; i < np; ++i) {
            const size_t u = s * np + i;
            off_rep[u] = (int64_t)at;
            std::memcpy(con.data() + at, quotes + a, len * sizeof(ope_contract));
            for (size_t k = 0; k < len; ++k) {
                unit[at + k] = (int32_t)u;
                qidx[at + k] = (int32_t)(a + k);
            }
            std::memcpy(pop.data() + u * dim, pop0.data() + (size_t)i * dim, dim * sizeof(double));
            at += len;
        }
    }
    off_rep[members] = (int64_t)at;
    std::vector<double> wv(nq);
    for (size_t i = 0; i < nq; ++i) wv[i] = weights ? weights[i] : 1.0;
    // Device layout
    size_t o = 0;
    auto take = [&](size_t bytes) { const size_t r = o; o += align_up(bytes, 256); return r; };
    const size_t o_con = take(nr * sizeof(ope_contract)), o_unit = take(nr * sizeof(int32_t)),
                 o_qidx = take(nr * sizeof(int32_t)), o_off = take((members + 1) * sizeof(int64_t)),
                 o_iv = take(nq * sizeof(double)), o_w = take(nq * sizeof(double)),
                 o_pop = take(members * dim * sizeof(double)), o_fit = take(members * sizeof(double)),
                 o_trial = take(members * dim * sizeof(double)), o_mask = take(members * sizeof(int32_t)),
                 o_price = take(nr * sizeof(double)), o_res = take(nr * sizeof(double)),
                 o_state = take(4 * sizeof(int)), o_bsse = take(ns * sizeof(double)),
                 o_win = take(ns * dim * sizeof(double)), o_scr = take(price_scratch_bytes(nr));
    cudaStream_t st = c.stream;
    void* ws;
    OPE_TRY(ensure_workspace(o, &ws, st));
    char* b = static_cast<char*>(ws);
    OPE_CHECK(cudaMemcpyAsync(b + o_con, con.data(), nr * sizeof(ope_contract), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(b + o_unit, unit.data(), nr * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(b + o_qidx, qidx.data(), nr * sizeof(int32_t), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(b + o_off, off_rep.data(), (members + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(b + o_iv, iv_market, nq * sizeof(double), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(b + o_w, wv.data(), nq * sizeof(double), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemcpyAsync(b + o_pop, pop.data(), members * dim * sizeof(double), cudaMemcpyHostToDevice, st));
    OPE_CHECK(cudaMemsetAsync(b + o_state, 0, 4 * sizeof(int), st));
    DEDev D;
    D.con = reinterpret_cast<const ope_contract*>(b + o_con);
    D.unit = reinterpret_cast<const int32_t*>(b + o_unit);
    D.qidx = reinterpret_cast<const int32_t*>(b + o_qidx);
    D.off = reinterpret_cast<const int64_t*>(b + o_off);
    D.iv = reinterpret_cast<const double*>(b + o_iv);
    D.w = reinterpret_cast<const double*>(b + o_w);
    D.pop = reinterpret_cast<double*>(b + o_pop);
    D.fit = reinterpret_cast<double*>(b + o_fit);
    D.trial = reinterpret_cast<double*>(b + o_trial);
    D.mask = reinterpret_cast<int32_t*>(b + o_mask);
    D.price = reinterpret_cast<double*>(b + o_price);
    D.res = reinterpret_cast<double*>(b + o_res);
    D.state = reinterpret_cast<int*>(b + o_state);
    D.ns = (int)ns;
    D.np = np;
    D.dim = dim;
    D.n_gen = n_gen;
    D.nr = (long long)nr;
    D.seed = seed;
    const PriceScratch ps = carve_price_scratch(b + o_scr, nr);
    // fitness of the initial population (calibration.rs:369), then the generations
    OPE_TRY(enqueue_generation(model, D, ps, tol, st, cudaGraphConditionalHandle{}, true));
    if (n_gen > 0) OPE_TRY(run_generations(model, D, ps, tol, st));
    double* d_bsse = reinterpret_cast<double*>(b + o_bsse);
    double* d_win = reinterpret_cast<double*>(b + o_win);
    k_de_best<<<(unsigned)((ns + 127) / 128), 128, 0, st>>>(D, d_bsse, d_win);
    OPE_CHECK(cudaGetLastError());
    c.launches += 1;
    std::vector<double> bsse(ns), win(ns * dim);
    int state[4] = {0, 0, 0, 0};
    OPE_CHECK(cudaMemcpyAsync(bsse.data(), d_bsse, ns * sizeof(double), cudaMemcpyDeviceToHost, st));
    OPE_CHECK(cudaMemcpyAsync(win.data(), d_win, ns * dim * sizeof(double), cudaMemcpyDeviceToHost, st));
    OPE_CHECK(cudaMemcpyAsync(state, D.state, sizeof(state), cudaMemcpyDeviceToHost, st));
    OPE_CHECK(cudaStreamSynchronize(st));
    if (state[1]) return set_error(OPE_ERR_DEVICE, "DE: index sampler exceeded its rejection limit");
    // LM polish from each winner (calibration.rs:422-426), regularised when a prior is given
    std::vector<ope_calib_result> res(ns);
    CalibExtra ex;
    ex.prior = prior;
    ex.reg_weight = reg_weight;
    OPE_TRY(run_calibration(model, quotes, iv_market, weights, nq, off, ns, win.data(), res.data(), tol, false,
                            nullptr, prior ? &ex : nullptr));
    for (size_t s = 0; s < ns; ++s) {
        out[s].best = res[s];
        out[s].de_best_sse = bsse[s];
        out[s].de_generations = n_gen;
        out[s].n_pop = np;
    }
    return OPE_OK;
}

}  // namespace ope
