// The pricing kernel: a persistent grid of warps pulling (contract, integral)
// units from a device work queue.  The same kernel serves the plain
// per-surface drop-in (batch.rs:23-42: one launch per parameter set) and the
// batched multi-surface launch, so a contract's price is bit-identical
// whichever way, and whatever else, it is launched with.
//
// Work unit = one Gil-Pelaez integral of one contract (P1 or P2,
// heston.rs:92-93 / bates.rs:58-59), integrated by one warp.  The two
// integrals of a contract run on different warps; whichever finishes second
// combines them into the price (heston.rs:95-98) through a per-contract
// completion counter.  The queue takes contracts in input order, or
// deepest-first (a counting sort of the contracts by a depth key, three small
// kernels ahead of the launch) when the launch shape asks for it: the
// reference's rayon pool (batch.rs:23-42) steals work per contract; here the
// longest serial bisection chains start first, so a call's tail is not one
// deep integral that started last.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "quadrature.cuh"

// Register budget of the pricing kernel: per model, the minimum resident
// blocks per SM of the 4-warp shape handed to __launch_bounds__ (registers
// per thread capped at 65536 / (32 * 4 * MINB)); the 1- and 2-warp shapes get
// 4 / warps times as many blocks, the same 64 registers.  8 for both models:
// the fastest of 5-9 blocks on each model's full batch (within 2 % of one
// another; kept per model because the optimum has moved apart and back with
// changes to the node evaluation).
#ifndef OPE_KERNEL_MINB_BATES
#define OPE_KERNEL_MINB_BATES 8
#endif
#ifndef OPE_KERNEL_MINB_HESTON
#define OPE_KERNEL_MINB_HESTON 8
#endif
// The same for the run kernel (both models).
#ifndef OPE_RUNS_MINB
#define OPE_RUNS_MINB 8
#endif

namespace ope {

namespace {
constexpr int kOrderBuckets = 64;
// Run cache entries per warp (panels of one run), and warps per SM it is
// sized for (the 64-register budget holds at most 32).
#ifndef OPE_RUN_CACHE_ENTRIES
#define OPE_RUN_CACHE_ENTRIES 128
#endif
constexpr int kRunCacheEntries = OPE_RUN_CACHE_ENTRIES;
constexpr int kRunWarpsPerSm = 32;
// Automatic launches (per_unit 0): calls of at least kRunsMinContracts
// contracts probe for runs (k_run_probe), which picks kRunsMinPerUnit to
// kRunsMaxPerUnit contracts per unit, or the per-contract kernel.
constexpr size_t kRunsMinContracts = 32768;
constexpr int kRunsMinPerUnit = 4;
constexpr int kRunsMaxPerUnit = 16;
constexpr int kRunsUnitsPerWarp = 24;
constexpr size_t kRunCacheWarpBytes = (size_t)kRunCacheEntries * (2 * 16 * sizeof(double) + sizeof(uint32_t));
}

// Layout: integ (2n doubles) | done (n) | head (256 B) | hist (2 x kOrderBuckets
// counters, 512 B) | order (n) | bucket (n); done, head and hist are adjacent
// so one memset clears them.
size_t price_scratch_bytes(size_t n) {
    return align_up(2 * n * sizeof(double), 256) + align_up(n * sizeof(unsigned int), 256) + 256 + 512 +
           2 * align_up(n * sizeof(uint32_t), 256);
}

size_t panel_sink_bytes(size_t n, int n_slots) {
    return align_up(2 * n * n_slots * 2 * kMaxPanels * sizeof(double), 256) + align_up(2 * n * n_slots * sizeof(int32_t), 256);
}

PriceScratch carve_price_scratch(void* base, size_t n, size_t run_bytes) {
    PriceScratch s = carve_price_scratch(base, n);
    if (run_bytes) {
        s.runcache = static_cast<char*>(base) + price_scratch_bytes(n);
        s.runcache_bytes = run_bytes;
    }
    return s;
}

size_t price_run_bytes(int model, size_t n, size_t other_bytes) {
    const int pu = price_shape(model, n).per_unit;
    if (!(pu > 1 || (pu == 0 && n >= kRunsMinContracts))) return 0;
    const size_t b = run_cache_bytes();
    // under a workspace limit the run cache is optional: without it the call
    // takes one contract per unit, with the same prices
    const size_t limit = tctx().ws_limit;
    return (limit && other_bytes + b > limit) ? 0 : b;
}

PanelSink carve_panel_sink(void* base, size_t n, int n_slots, const int32_t* slot) {
    PanelSink k;
    k.panels = static_cast<double*>(base);
    k.nbis = reinterpret_cast<int32_t*>(static_cast<char*>(base) +
                                        align_up(2 * n * n_slots * 2 * kMaxPanels * sizeof(double), 256));
    k.slot = slot;
    k.n_slots = n_slots;
    return k;
}

PriceScratch carve_price_scratch(void* base, size_t n) {
    char* p = static_cast<char*>(base);
    PriceScratch s;
    s.integ = reinterpret_cast<double*>(p);
    p += align_up(2 * n * sizeof(double), 256);
    s.done = reinterpret_cast<unsigned int*>(p);
    p += align_up(n * sizeof(unsigned int), 256);
    s.head = reinterpret_cast<unsigned long long*>(p);
    p += 256;
    s.hist = reinterpret_cast<unsigned int*>(p);
    p += 512;
    s.order = reinterpret_cast<uint32_t*>(p);
    p += align_up(n * sizeof(uint32_t), 256);
    s.bucket = reinterpret_cast<uint32_t*>(p);
    return s;
}

namespace {

struct ContractView {
    double s, k, t, r, q;
    int opt_type;
};

// The 56-byte contract record staged cooperatively for the per-integral
// constants: lanes 0-6 each load one of its seven 8-byte words (one coalesced
// request), shuffles hand every lane the fields.  (The lane that combines a
// contract's integrals at the end re-reads the fields it needs, so they are
// not held across the integration.)
__device__ __forceinline__ ContractView load_contract(const ope_contract* con, long long c, int lane) {
    const unsigned FULL = 0xffffffffu;
    const long long* w = reinterpret_cast<const long long*>(con + c);
    const long long mine = lane < 7 ? __ldg(w + lane) : 0ll;
    ContractView v;
    v.s = __longlong_as_double(__shfl_sync(FULL, mine, 0));
    v.k = __longlong_as_double(__shfl_sync(FULL, mine, 1));
    v.t = __longlong_as_double(__shfl_sync(FULL, mine, 2));
    v.r = __longlong_as_double(__shfl_sync(FULL, mine, 3));
    v.q = __longlong_as_double(__shfl_sync(FULL, mine, 4));
    v.opt_type = (int)(unsigned)(__shfl_sync(FULL, mine, 6) & 0xffffffffll);  // low word of {opt_type, pad}
    return v;
}

// Integrate unit (contract c, integral `which`) and, if it completes the
// contract, write the price.  SAVE: also store the final live-panel list
// and the bisection count in `sink` (slot `slot`), for the adjoint's backward
// pass.
// CACHED: through the run cache `rc` (the run kernel).
template <bool BATES, bool SAVE, bool CACHED = false>
__device__ __forceinline__ void run_unit(long long c, int which, const ope_contract* con, const double* p,
                                         double tol, double* out, double* integ, unsigned int* done,
                                         int32_t* nbis_out, const PanelSink& sink, int slot, PanelStore& L,
                                         CfConsts& Cs, int lane, const LaneRule& R, RunCacheWarp* rc = nullptr) {
    {
        const ContractView v = load_contract(con, c, lane);
        double pl[8];
#pragma unroll
        for (int i = 0; i < (BATES ? 8 : 5); ++i) pl[i] = __ldg(p + i);
        const CfConsts Cl = make_consts(v.s, v.k, v.t, v.r, pl, BATES, which);
        __syncwarp();
        if (lane == 0) Cs = Cl;
        __syncwarp();
    }
    const CfConsts& C = Cs;
    int nb;
    const double I = gk_integrate_warp<BATES, CACHED>(C, tol, L, lane, R, &nb, NoTrace(), rc);
    if (SAVE) {
        const size_t idx = (size_t)(2 * c + which) * sink.n_slots + slot;
        double* dst = sink.panels + idx * (2 * kMaxPanels);
        for (int i = lane; i <= nb; i += 32) {
            dst[2 * i] = L.a[i];
            dst[2 * i + 1] = L.b[i];
        }
        if (lane == 0) sink.nbis[idx] = nb;
        __syncwarp();  // the list is read before the next unit rewrites it
    }
    if (lane == 0) {
        if (nbis_out) nbis_out[2 * c + which] = nb;
        integ[2 * c + which] = I;
        __threadfence();
        const unsigned int prev = atomicAdd(done + c, 1u);
        if (prev == 1u) {
            __threadfence();
            const double other = __ldcg(integ + 2 * c + (1 - which));
            const double i1 = which == 0 ? I : other;
            const double i2 = which == 0 ? other : I;
            const ope_contract* k = con + c;
            out[c] = finish_price(__ldg(&k->spot), __ldg(&k->strike), __ldg(&k->expiry), __ldg(&k->rate),
                                  __ldg(&k->div_yield), __ldg(&k->opt_type), i1, i2);
        }
    }
}

// Surface of contract c: the s with off[s] <= c < off[s+1] (upper_bound - 1).
__device__ __forceinline__ long long find_surface(const int64_t* off, long long n_surf, long long c) {
    long long lo = 1, hi = n_surf;  // search [1, n_surf] for the first off[j] > c
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (__ldg(off + mid) > c) hi = mid; else lo = mid + 1;
    }
    return lo - 1;
}

__device__ __forceinline__ long long param_set(const int32_t* param_idx, const int64_t* surf_off, long long n_surf,
                                               long long c) {
    return param_idx ? (long long)__ldg(param_idx + c) : (n_surf > 1 ? find_surface(surf_off, n_surf, c) : 0);
}

// Every warp pulls units from the device queue until it drains; the grid is
// the resident capacity of the GPU (or the launch shape's share of it), or
// fewer warps than units for small calls.  Queue position q holds contract
// order[q] (input order when order is NULL); its two integrals are units 2q
// and 2q + 1, so a contract's pair starts together.
template <bool BATES, bool SAVE, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, (BATES ? OPE_KERNEL_MINB_BATES : OPE_KERNEL_MINB_HESTON) * 4 / WARPS)
    k_price_persistent(const ope_contract* __restrict__ con, long long n, const int64_t* __restrict__ surf_off,
                       long long n_surf, const int32_t* __restrict__ param_idx, const int32_t* __restrict__ surf_mask,
                       const double* __restrict__ params, double tol, double* __restrict__ out, double* integ,
                       unsigned int* done, unsigned long long* head, int32_t* nbis_out, PanelSink sink,
                       const uint32_t* __restrict__ order) {
    extern __shared__ PanelStore smem_panels[];
    // Per warp: the unit's integrand constants.  They are warp-uniform, so the
    // node evaluation reads them from shared memory (broadcast loads) and
    // leaves its registers to the per-lane values: at the 72-register cap
    // that cut the spills by half and the Bates batch's time by 4 %.
    __shared__ CfConsts s_consts[WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const LaneRule R = lane_rule(lane);
    const int stride = BATES ? 8 : 5;
    const unsigned long long n_units = 2ull * (unsigned long long)n;
    while (true) {
        unsigned long long unit = 0;
        if (lane == 0) unit = atomicAdd(head, 1ull);
        unit = __shfl_sync(0xffffffffu, unit, 0);
        if (unit >= n_units) break;
        const long long q = (long long)(unit >> 1);
        const long long c = order ? (long long)__ldg(order + q) : q;
        const long long s = param_set(param_idx, surf_off, n_surf, c);
        if (surf_mask && __ldg(surf_mask + s) == 0) {
            // a skipped surface's units are contiguous in input order: move the
            // queue head past all of them with one atomic instead of one per unit
            if (lane == 0 && !param_idx && surf_off && !order)
                atomicMax(head, 2ull * (unsigned long long)__ldg(surf_off + s + 1));
            continue;
        }
        if (!param_idx && n_surf > 1 && !ope_check(s >= 0 && s < n_surf, CHK_SURFACE)) continue;
        int slot = (SAVE && sink.slot) ? __ldg(sink.slot + s) : 0;
        if (SAVE && !ope_check(slot >= 0 && slot < sink.n_slots, CHK_SLOT)) slot = 0;
        run_unit<BATES, SAVE>(c, (int)(unit & 1), con, params + s * stride, tol, out, integ, done, nbis_out,
                              sink, slot, smem_panels[warp], s_consts[warp], lane, R);
    }
}

// The run kernel: the queue hands out blocks of `per_unit` consecutive
// contracts (unit 2b + which: integral `which` of block b), and one warp
// integrates a block's contracts one after another.  A block splits into runs
// -- maximal stretches of contracts with the same parameter set, expiry and
// rate, whose integrands differ only in the phase u ln(S/K) -- and each run of
// two or more contracts shares one run cache (quadrature.cuh), so a surface
// laid out expiry by expiry evaluates the characteristic function once per
// panel and expiry instead of once per panel and strike.  A run never
// reaches across blocks; contracts alone in their run are integrated
// uncached.  Prices are bit-identical to k_price_persistent's.
struct RunCacheMem {
    double* vals;     // per warp of the grid: [2][cap][16] (w, a)
    uint32_t* child;  // per warp of the grid: [cap]
    int cap;
};

template <bool BATES, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, OPE_RUNS_MINB * 4 / WARPS)
    k_price_runs(const ope_contract* __restrict__ con, long long n, const int64_t* __restrict__ surf_off,
                 long long n_surf, const int32_t* __restrict__ param_idx, const double* __restrict__ params,
                 double tol, double* __restrict__ out, double* integ, unsigned int* done, unsigned long long* head,
                 int32_t* nbis_out, int per_unit_arg, RunCacheMem mem) {
    extern __shared__ PanelStore smem_panels[];  // [WARPS], then the entry slots [WARPS][kMaxPanels]
    __shared__ CfConsts s_consts[WARPS];
    const unsigned FULL = 0xffffffffu;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const LaneRule R = lane_rule(lane);
    const int stride = BATES ? 8 : 5;
    const size_t gw = (size_t)blockIdx.x * WARPS + warp;
    RunCacheWarp rc;
    rc.cap = mem.cap;
    rc.w = mem.vals + gw * 2 * (size_t)mem.cap * 16;
    rc.a = rc.w + (size_t)mem.cap * 16;
    rc.child = mem.child + gw * (size_t)mem.cap;
    rc.slot = reinterpret_cast<uint16_t*>(smem_panels + WARPS) + warp * kMaxPanels;
    rc.n_alloc = 0;
    rc.on = false;
    // contracts per unit: the launch's, or (0) the run probe's choice; with
    // no choice (the probe kept the per-contract kernel) the queue is closed
    int per_unit = per_unit_arg;
    if (per_unit <= 0) per_unit = (int)min(__ldcg(head + 9), 32ull);  // head + 9 = the probe's head[25]
    if (per_unit <= 0) per_unit = 1;
    const unsigned long long n_blocks = ((unsigned long long)n + per_unit - 1) / per_unit;
    const PanelSink none{nullptr, nullptr, nullptr, 1};
    while (true) {
        unsigned long long unit = 0;
        if (lane == 0) unit = atomicAdd(head, 1ull);
        unit = __shfl_sync(FULL, unit, 0);
        if (unit >= 2ull * n_blocks) {
            run_cache_discard(rc, lane);
            break;
        }
        const long long c0 = (long long)(unit >> 1) * per_unit;
        const int which = (int)(unit & 1);
        const int cnt = (int)min((long long)per_unit, n - c0);
        // run keys of the block's contracts, one lane each; a contract starts
        // a run when its key differs from its predecessor's
        long long ps = -1, tb = 0, rb = 0;
        if (lane < cnt) {
            ps = param_set(param_idx, surf_off, n_surf, c0 + lane);
            tb = __double_as_longlong(__ldg(&con[c0 + lane].expiry));
            rb = __double_as_longlong(__ldg(&con[c0 + lane].rate));
        }
        const long long pps = __shfl_up_sync(FULL, ps, 1), ptb = __shfl_up_sync(FULL, tb, 1),
                        prb = __shfl_up_sync(FULL, rb, 1);
        const unsigned starts = __ballot_sync(FULL, lane < cnt && (lane == 0 || ps != pps || tb != ptb || rb != prb));
        for (int i = 0; i < cnt; ++i) {
            const long long c = c0 + i;
            const long long s = __shfl_sync(FULL, ps, i);
            if ((starts >> i) & 1u) {
                const unsigned later = i < 31 ? starts >> (i + 1) : 0u;
                const int next = later ? i + __ffs((int)later) : cnt;
                run_cache_discard(rc, lane);
                rc.on = next - i >= 2 && rc.cap > 0;
            }
            if (!param_idx && n_surf > 1 && !ope_check(s >= 0 && s < n_surf, CHK_SURFACE)) continue;
            run_unit<BATES, false, true>(c, which, con, params + s * stride, tol, out, integ, done, nbis_out, none,
                                         0, smem_panels[warp], s_consts[warp], lane, R, &rc);
        }
    }
}

// Run probe of an automatic launch: counts, on a sample of the call, the
// contracts that start a run (the first of a surface, or a change of
// expiry or rate) and, in its last block to finish, picks the contracts per
// unit: the largest power of two up to 16 that is at most the sample's mean
// run length and leaves every warp of the run kernel's grid (run_warps) at
// least kRunsUnitsPerWarp units, so that the queue's tail stays short.
// Below kRunsMinPerUnit it keeps the per-contract kernel.  The sample: up to
// kProbeChunks chunks of 32 consecutive contracts spread evenly over the
// call, one warp each, every lane reading one contract's expiry and rate
// (the predecessor's come by shuffle; contracts in pinned host memory are
// read over PCIe, so the probe reads as little as it can).  It closes the
// work queue of the kernel that is not to run (head[0]: the per-contract
// kernel's, head[16]: the run kernel's) and leaves the choice in head[25]
// for the run kernel; head[26..27] hold its counters.  Both kernels are
// launched after it; the one whose queue is closed ends after one atomic
// per warp.  The choice only moves time: prices are the same either way.
constexpr unsigned long long kQueueClosed = 1ull << 62;
constexpr long long kProbeChunks = 2048;

__global__ void __launch_bounds__(256) k_run_probe(const ope_contract* __restrict__ con, long long n,
                                                   const int64_t* __restrict__ surf_off, long long n_surf,
                                                   const int32_t* __restrict__ param_idx, unsigned long long* head,
                                                   long long run_warps) {
    __shared__ unsigned int part[2][8];
    const unsigned FULL = 0xffffffffu;
    unsigned int* cnt = reinterpret_cast<unsigned int*>(head + 26);  // [0] starts, [1] sampled, [2] blocks done
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long chunks = (n + 31) / 32;
    const long long samples = chunks < kProbeChunks ? chunks : kProbeChunks;
    unsigned int starts = 0, seen = 0;
    for (long long k = (long long)blockIdx.x * (blockDim.x >> 5) + wib; k < samples;
         k += (long long)gridDim.x * (blockDim.x >> 5)) {
        const long long c0 = (k * chunks / samples) * 32;
        const long long c = c0 + lane;
        const bool in = c < n;
        long long ps = -1, tb = 0, rb = 0;
        if (in) {
            ps = param_set(param_idx, surf_off, n_surf, c);
            tb = __double_as_longlong(__ldg(&con[c].expiry));
            rb = __double_as_longlong(__ldg(&con[c].rate));
        }
        long long pps = __shfl_up_sync(FULL, ps, 1), ptb = __shfl_up_sync(FULL, tb, 1), prb = __shfl_up_sync(FULL, rb, 1);
        bool start = true;
        if (lane == 0 && c0 > 0) {
            pps = param_set(param_idx, surf_off, n_surf, c0 - 1);
            ptb = __double_as_longlong(__ldg(&con[c0 - 1].expiry));
            prb = __double_as_longlong(__ldg(&con[c0 - 1].rate));
        }
        if (c > 0) start = ps != pps || tb != ptb || rb != prb;
        starts += __popc(__ballot_sync(FULL, in && start));
        seen += __popc(__ballot_sync(FULL, in));
    }
    if (lane == 0) {
        part[0][wib] = starts;
        part[1][wib] = seen;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned int st = 0, se = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            st += part[0][i];
            se += part[1][i];
        }
        atomicAdd(cnt, st);
        atomicAdd(cnt + 1, se);
        __threadfence();
        if (atomicAdd(cnt + 2, 1u) == gridDim.x - 1) {
            __threadfence();
            const unsigned long long s_starts = atomicAdd(cnt, 0u), s_seen = atomicAdd(cnt + 1, 0u);
            int pu = kRunsMaxPerUnit;
            while (pu >= kRunsMinPerUnit &&
                   (s_seen < (unsigned long long)pu * s_starts ||
                    2ull * (unsigned long long)n < (unsigned long long)pu * kRunsUnitsPerWarp * (unsigned long long)run_warps))
                pu >>= 1;
            const bool runs = pu >= kRunsMinPerUnit;
            head[25] = runs ? (unsigned long long)pu : 0ull;
            __threadfence();
            atomicExch(head + (runs ? 0 : 16), kQueueClosed);
        }
    }
}

// Depth bucket of a contract: 0 for the deepest.  The key |ln(K/S)| /
// sqrt(v0 T) -- how many standard deviations of the initial variance over the
// expiry the strike lies out -- ranks the integrals' bisection counts with a
// Spearman correlation of 0.9 on the benchmark batches (short expiries and
// deep wings need the most panels); 8 buckets per doubling of 1 + key.
__device__ __forceinline__ unsigned depth_bucket(const ope_contract* con, long long c, double v0) {
    const double x = fabs(log(__ldg(&con[c].strike) / __ldg(&con[c].spot)));
    const double key = x / sqrt(fmax(v0, 0.0) * __ldg(&con[c].expiry));
    if (!(key == key)) return kOrderBuckets - 1;  // NaN (e.g. 0/0): last
    const int b = (int)fmin(8.0 * log2(1.0 + key), (double)(kOrderBuckets - 1));
    return (unsigned)(kOrderBuckets - 1 - b);
}

__global__ void __launch_bounds__(256) k_order_bucket(const ope_contract* __restrict__ con, long long n,
                                                      const int64_t* __restrict__ surf_off, long long n_surf,
                                                      const int32_t* __restrict__ param_idx,
                                                      const double* __restrict__ params, int stride,
                                                      uint32_t* __restrict__ bucket, unsigned int* hist) {
    __shared__ unsigned int h[kOrderBuckets];
    for (int i = threadIdx.x; i < kOrderBuckets; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const long long s = param_set(param_idx, surf_off, n_surf, c);
        const unsigned b = depth_bucket(con, c, __ldg(params + s * stride));
        bucket[c] = b;
        atomicAdd(&h[b], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kOrderBuckets; i += blockDim.x)
        if (h[i]) atomicAdd(hist + i, h[i]);
}

// Queue positions: each block forms the buckets' starting positions (an
// exclusive prefix sum of the kOrderBuckets counts hist[0..64), one warp),
// then each contract takes the next free slot of its bucket through the fill
// counters hist[64..128) (the order inside a bucket is arbitrary, and
// irrelevant to the prices).
__global__ void __launch_bounds__(256) k_order_scatter(long long n, const uint32_t* __restrict__ bucket,
                                                       unsigned int* hist, uint32_t* __restrict__ order) {
    __shared__ unsigned int start[kOrderBuckets];
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        const unsigned a = __ldcg(hist + 2 * lane), b = __ldcg(hist + 2 * lane + 1);
        unsigned incl = a + b;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += v;
        }
        start[2 * lane] = incl - (a + b);
        start[2 * lane + 1] = incl - b;
    }
    __syncthreads();
    unsigned int* fill = hist + kOrderBuckets;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const uint32_t b = bucket[c];
        order[start[b] + atomicAdd(fill + b, 1u)] = (uint32_t)c;
    }
}

template <class K>
int persistent_grid(K kernel, int threads, size_t smem, double occupancy, int* grid) {
    int per_sm = 0, sms = 0;
    OPE_TRY(blocks_per_sm(reinterpret_cast<const void*>(kernel), threads, smem, &per_sm));
    OPE_TRY(current_device_sms(&sms));
    const int blocks = std::max(1, (int)(per_sm * occupancy));
    *grid = std::max(1, (int)(blocks * sms * tctx().grid_fraction));
    return OPE_OK;
}

template <bool BATES, bool SAVE, int WARPS>
int launch_impl(const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                const int32_t* param_idx, const double* params, double tol, double* out, const PriceScratch& s,
                cudaStream_t st, int32_t* nbis_out, const int32_t* surf_mask, const PanelSink& sink,
                const uint32_t* order, double occupancy) {
    const int threads = WARPS * 32;
    const size_t smem = WARPS * sizeof(PanelStore);
    int grid = 0;
    OPE_TRY(persistent_grid(k_price_persistent<BATES, SAVE, WARPS>, threads, smem, occupancy, &grid));
    const unsigned long long need = (2ull * n + WARPS - 1) / WARPS;
    grid = (int)std::min<unsigned long long>((unsigned long long)grid, need);
    k_price_persistent<BATES, SAVE, WARPS><<<grid, threads, smem, st>>>(
        con, (long long)n, surf_offsets, (long long)n_surf, param_idx, surf_mask, params, tol, out, s.integ, s.done,
        s.head, nbis_out, sink, order);
    OPE_CHECK(cudaGetLastError());
    return OPE_OK;
}

// Grid of the run kernel (blocks of WARPS warps): the persistent grid,
// capped by the warps the run cache holds and by the units of a launch of
// per_unit contracts (the smallest the run probe may pick when automatic).
template <bool BATES, int WARPS>
int runs_grid(size_t n, const PriceScratch& s, int per_unit, double occupancy, int* grid) {
    const int threads = WARPS * 32;
    const size_t smem = WARPS * (sizeof(PanelStore) + kMaxPanels * sizeof(uint16_t));
    OPE_TRY(persistent_grid(k_price_runs<BATES, WARPS>, threads, smem, occupancy, grid));
    const int pu = per_unit > 0 ? per_unit : kRunsMinPerUnit;
    const unsigned long long blocks = ((unsigned long long)n + pu - 1) / pu;
    const unsigned long long need = (2ull * blocks + WARPS - 1) / WARPS;
    const size_t cache_warps = s.runcache_bytes / kRunCacheWarpBytes;
    *grid = (int)std::min<unsigned long long>({(unsigned long long)*grid, need, cache_warps / WARPS});
    if (*grid < 1) return set_error(OPE_ERR_INVALID_ARG, "run cache too small for one block of warps");
    return OPE_OK;
}

// per_unit 0: the run probe's choice (automatic launches).
template <bool BATES, int WARPS>
int launch_runs(const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                const int32_t* param_idx, const double* params, double tol, double* out, const PriceScratch& s,
                cudaStream_t st, int32_t* nbis_out, int per_unit, double occupancy) {
    const int threads = WARPS * 32;
    const size_t smem = WARPS * (sizeof(PanelStore) + kMaxPanels * sizeof(uint16_t));
    int grid = 0;
    OPE_TRY((runs_grid<BATES, WARPS>(n, s, per_unit, occupancy, &grid)));
    const size_t cache_warps = s.runcache_bytes / kRunCacheWarpBytes;
    RunCacheMem mem;
    mem.cap = kRunCacheEntries;
    mem.vals = static_cast<double*>(s.runcache);
    mem.child = reinterpret_cast<uint32_t*>(static_cast<char*>(s.runcache) +
                                            cache_warps * (size_t)kRunCacheEntries * 2 * 16 * sizeof(double));
    k_price_runs<BATES, WARPS><<<grid, threads, smem, st>>>(con, (long long)n, surf_offsets, (long long)n_surf,
                                                             param_idx, params, tol, out, s.integ, s.done,
                                                             s.head + 16, nbis_out, per_unit, mem);
    OPE_CHECK(cudaGetLastError());
    return OPE_OK;
}

template <bool BATES>
int launch_plain(int warps, const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                 const int32_t* param_idx, const double* params, double tol, double* out, const PriceScratch& s,
                 cudaStream_t st, int32_t* nbis_out, const uint32_t* order, double occupancy) {
    const PanelSink none{nullptr, nullptr, nullptr, 1};
    switch (warps) {
        case 1:
            return launch_impl<BATES, false, 1>(con, n, surf_offsets, n_surf, param_idx, params, tol, out, s, st,
                                                nbis_out, nullptr, none, order, occupancy);
        case 2:
            return launch_impl<BATES, false, 2>(con, n, surf_offsets, n_surf, param_idx, params, tol, out, s, st,
                                                nbis_out, nullptr, none, order, occupancy);
        default:
            return launch_impl<BATES, false, 4>(con, n, surf_offsets, n_surf, param_idx, params, tol, out, s, st,
                                                nbis_out, nullptr, none, order, occupancy);
    }
}

// Deepest-first queue order of the n contracts into s.order (s.hist, zeroed
// by the caller, and s.bucket as scratch).
int build_order(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                const int32_t* param_idx, const double* params, const PriceScratch& s, cudaStream_t st) {
    int sms = 0;
    OPE_TRY(current_device_sms(&sms));
    const long long want = (long long)((n + 255) / 256);
    const unsigned blocks = (unsigned)std::max(1ll, std::min<long long>(want, 8ll * sms));
    k_order_bucket<<<blocks, 256, 0, st>>>(con, (long long)n, surf_offsets, (long long)n_surf, param_idx, params,
                                           param_stride(model), s.bucket, s.hist);
    OPE_CHECK(cudaGetLastError());
    k_order_scatter<<<blocks, 256, 0, st>>>((long long)n, s.bucket, s.hist, s.order);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 2;
    return OPE_OK;
}

}  // namespace

const uint64_t kTuneClassMax[kTuneClasses] = {1ull << 6,  1ull << 7,  1ull << 8,  1ull << 9,  1ull << 10, 1ull << 11,
                                               1ull << 12, 1ull << 13, 1ull << 14, 1ull << 15, 1ull << 16, 1ull << 17,
                                               1ull << 18, 1ull << 19, 1ull << 20, ~0ull};

size_t run_cache_bytes() {
    int sms = 0;
    if (current_device_sms(&sms) != OPE_OK) return 0;
    return (size_t)sms * kRunWarpsPerSm * kRunCacheWarpBytes;
}

int prepare_price_kernels() {
    int grid = 0;
    const int threads = 4 * 32;
    const size_t smem = 4 * sizeof(PanelStore);
    OPE_TRY(persistent_grid(k_price_persistent<false, false, 4>, threads, smem, 1.0, &grid));
    OPE_TRY(persistent_grid(k_price_persistent<true, false, 4>, threads, smem, 1.0, &grid));
    return OPE_OK;
}

int launch_price_persistent(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets,
                            size_t n_surf, const int32_t* param_idx, const double* params, double tol, double* out,
                            const PriceScratch& s, cudaStream_t st, int32_t* nbis_out, const int32_t* surf_mask,
                            const PanelSink* sink, const LaunchShape* shape) {
    if (n == 0) return OPE_OK;
    const bool bates = model == OPE_MODEL_BATES;
    // stored panel lists and skipped surfaces keep the fixed shape (4 warps,
    // input order); the allocation-free entry point has no order scratch
    LaunchShape sh;
    if (!sink && !surf_mask) sh = shape ? *shape : price_shape(model, n);
    if (!s.order || n > 0xffffffffull) sh.deepest_first = 0;
    // contracts per unit: fixed (2..32), automatic (0: probe for runs in
    // calls of kRunsMinContracts or more), or one per unit; the run kernel
    // needs the run cache and serves plain launches only
    if (!s.runcache || sink || surf_mask || sh.per_unit < 0 || (sh.per_unit == 0 && n < kRunsMinContracts))
        sh.per_unit = 1;
    if (sh.per_unit > 32) sh.per_unit = 32;
    const bool probe = sh.per_unit == 0;
    if (sh.per_unit > 1) sh.deepest_first = 0;
    if (sh.warps != 1 && sh.warps != 2) sh.warps = 4;
    if (!(sh.occupancy > 0.0 && sh.occupancy <= 1.0)) sh.occupancy = 1.0;
    // completion counters, queue head and (for a deepest-first order) the
    // bucket counters start at zero: one memset where they are adjacent
    const size_t done_bytes = align_up(n * sizeof(unsigned int), 256);
    const bool adjacent = reinterpret_cast<char*>(s.head) == reinterpret_cast<char*>(s.done) + done_bytes;
    const bool hist_adjacent = sh.deepest_first && reinterpret_cast<char*>(s.hist) == reinterpret_cast<char*>(s.head) + 256;
    const size_t head_bytes = 256;  // both queue heads and the probe's words
    if (adjacent) {
        OPE_CHECK(cudaMemsetAsync(s.done, 0, done_bytes + (hist_adjacent ? 256 + 512 : head_bytes), st));
    } else {
        OPE_CHECK(cudaMemsetAsync(s.done, 0, n * sizeof(unsigned int), st));
        OPE_CHECK(cudaMemsetAsync(s.head, 0, head_bytes, st));
    }
    if (sh.deepest_first && !(adjacent && hist_adjacent))
        OPE_CHECK(cudaMemsetAsync(s.hist, 0, 2 * kOrderBuckets * sizeof(unsigned int), st));
    if (!sink && !surf_mask) {
        tctx().last_per_unit = sh.per_unit;
        tctx().last_probe = nullptr;
    }
    const uint32_t* order = nullptr;
    if (sh.deepest_first) {
        OPE_TRY(build_order(model, con, n, surf_offsets, n_surf, param_idx, params, s, st));
        order = s.order;
    }
    if (sink) {
        OPE_TRY((bates ? launch_impl<true, true, 4> : launch_impl<false, true, 4>)(
            con, n, surf_offsets, n_surf, param_idx, params, tol, out, s, st, nbis_out, surf_mask, *sink, nullptr,
            1.0));
    } else if (surf_mask) {
        const PanelSink none{nullptr, nullptr, nullptr, 1};
        OPE_TRY((bates ? launch_impl<true, false, 4> : launch_impl<false, false, 4>)(
            con, n, surf_offsets, n_surf, param_idx, params, tol, out, s, st, nbis_out, surf_mask, none, nullptr,
            1.0));
    } else if (sh.per_unit > 1) {
        OPE_TRY((bates ? launch_runs<true, 4> : launch_runs<false, 4>)(con, n, surf_offsets, n_surf, param_idx, params,
                                                                       tol, out, s, st, nbis_out, sh.per_unit,
                                                                       sh.occupancy));
    } else if (probe) {
        // the probe closes one of the two queues; both kernels launch
        tctx().last_probe = s.head + 25;
        tctx().last_probe_stream = st;
        int sms = 0;
        OPE_TRY(current_device_sms(&sms));
        const long long probe_warps = std::min<long long>((long long)((n + 31) / 32), kProbeChunks);
        const unsigned pb = (unsigned)std::max(1ll, std::min<long long>((probe_warps + 7) / 8, 2ll * sms));
        int rgrid = 0;
        OPE_TRY((bates ? runs_grid<true, 4> : runs_grid<false, 4>)(n, s, 0, sh.occupancy, &rgrid));
        k_run_probe<<<pb, 256, 0, st>>>(con, (long long)n, surf_offsets, (long long)n_surf, param_idx, s.head,
                                        4ll * rgrid);
        OPE_CHECK(cudaGetLastError());
        OPE_TRY((bates ? launch_plain<true> : launch_plain<false>)(sh.warps, con, n, surf_offsets, n_surf, param_idx,
                                                                   params, tol, out, s, st, nbis_out, order,
                                                                   sh.occupancy));
        OPE_TRY((bates ? launch_runs<true, 4> : launch_runs<false, 4>)(con, n, surf_offsets, n_surf, param_idx, params,
                                                                       tol, out, s, st, nbis_out, 0, sh.occupancy));
        tctx().launches += 2;
    } else {
        OPE_TRY((bates ? launch_plain<true> : launch_plain<false>)(sh.warps, con, n, surf_offsets, n_surf, param_idx,
                                                                   params, tol, out, s, st, nbis_out, order,
                                                                   sh.occupancy));
    }
    tctx().launches += 1;
    return OPE_OK;
}

}  // namespace ope
