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
// completion counter.
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"
#include "quadrature.cuh"

// Launch shape of the pricing kernel: warps per block and, per model, the
// minimum resident blocks per SM handed to __launch_bounds__ (which caps
// registers per thread at 65536 / (32 * WARPS * MINB)): 64 registers x 8
// blocks for both models, the fastest of 5-8 blocks on each model's full
// batch (within 2 % of one another; kept per model because the optimum has
// moved apart and back with changes to the node evaluation).
#ifndef OPE_KERNEL_WARPS
#define OPE_KERNEL_WARPS 4
#endif
#ifndef OPE_KERNEL_MINB_BATES
#define OPE_KERNEL_MINB_BATES 8
#endif
#ifndef OPE_KERNEL_MINB_HESTON
#define OPE_KERNEL_MINB_HESTON 8
#endif

namespace ope {

size_t price_scratch_bytes(size_t n) {
    return align_up(2 * n * sizeof(double), 256) + align_up(n * sizeof(unsigned int), 256) + 256;
}

size_t panel_sink_bytes(size_t n, int n_slots) {
    return align_up(2 * n * n_slots * 2 * kMaxPanels * sizeof(double), 256) + align_up(2 * n * n_slots * sizeof(int32_t), 256);
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
    return s;
}

namespace {

struct ContractView {
    double s, k, t, r, q;
    int opt_type;
};

__device__ __forceinline__ ContractView load_contract(const ope_contract* con, long long c) {
    const ope_contract* p = con + c;
    ContractView v;
    v.s = __ldg(&p->spot);
    v.k = __ldg(&p->strike);
    v.t = __ldg(&p->expiry);
    v.r = __ldg(&p->rate);
    v.q = __ldg(&p->div_yield);
    v.opt_type = __ldg(&p->opt_type);
    return v;
}

// Integrate unit (contract c, integral `which`) and, if it completes the
// contract, write the price.  SAVE: also store the final live-panel list
// and the bisection count in `sink` (slot `slot`), for the adjoint's backward
// pass.
template <bool BATES, bool SAVE>
__device__ __forceinline__ void run_unit(long long c, int which, const ope_contract* con, const double* p,
                                         double tol, double* out, double* integ, unsigned int* done,
                                         int32_t* nbis_out, const PanelSink& sink, int slot, PanelStore& L,
                                         CfConsts& Cs, int lane, const LaneRule& R) {
    const ContractView v = load_contract(con, c);
    double pl[8];
#pragma unroll
    for (int i = 0; i < (BATES ? 8 : 5); ++i) pl[i] = __ldg(p + i);
    {
        const CfConsts Cl = make_consts(v.s, v.k, v.t, v.r, pl, BATES, which);
        __syncwarp();
        if (lane == 0) Cs = Cl;
        __syncwarp();
    }
    const CfConsts& C = Cs;
    int nb;
    const double I = gk_integrate_warp<BATES>(C, tol, L, lane, R, &nb);
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
            out[c] = finish_price(v.s, v.k, v.t, v.r, v.q, v.opt_type, i1, i2);
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

// Every warp pulls units from the device queue until it drains; the grid is
// the resident capacity of the GPU, or fewer warps than units for small calls.
template <bool BATES, bool SAVE>
__global__ void __launch_bounds__(OPE_KERNEL_WARPS * 32, BATES ? OPE_KERNEL_MINB_BATES : OPE_KERNEL_MINB_HESTON) k_price_persistent(const ope_contract* __restrict__ con, long long n,
                                                          const int64_t* __restrict__ surf_off, long long n_surf,
                                                          const int32_t* __restrict__ param_idx,
                                                          const int32_t* __restrict__ surf_mask,
                                                          const double* __restrict__ params, double tol,
                                                          double* __restrict__ out, double* integ,
                                                          unsigned int* done, unsigned long long* head,
                                                          int32_t* nbis_out, PanelSink sink) {
    extern __shared__ PanelStore smem_panels[];
    // Per warp: the unit's integrand constants.  They are warp-uniform, so the
    // node evaluation reads them from shared memory (broadcast loads) and
    // leaves its registers to the per-lane values: at the 72-register cap
    // that cut the spills by half and the Bates batch's time by 4 %.
    __shared__ CfConsts s_consts[OPE_KERNEL_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const LaneRule R = lane_rule(lane);
    const int stride = BATES ? 8 : 5;
    const unsigned long long n_units = 2ull * (unsigned long long)n;
    while (true) {
        unsigned long long unit = 0;
        if (lane == 0) unit = atomicAdd(head, 1ull);
        unit = __shfl_sync(0xffffffffu, unit, 0);
        if (unit >= n_units) break;
        const long long c = (long long)(unit >> 1);
        const long long s = param_idx ? (long long)__ldg(param_idx + c)
                                      : (n_surf > 1 ? find_surface(surf_off, n_surf, c) : 0);
        if (surf_mask && __ldg(surf_mask + s) == 0) {
            // a skipped surface's units are contiguous: move the queue head past
            // all of them with one atomic instead of one per unit
            if (lane == 0 && !param_idx && surf_off)
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

template <class K>
int persistent_grid(K kernel, int threads, size_t smem, int* grid) {
    int per_sm = 0, sms = 0;
    OPE_TRY(blocks_per_sm(reinterpret_cast<const void*>(kernel), threads, smem, &per_sm));
    OPE_TRY(current_device_sms(&sms));
    *grid = std::max(1, (int)(per_sm * sms * tctx().grid_fraction));
    return OPE_OK;
}

template <bool BATES, bool SAVE>
int launch_impl(const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                const int32_t* param_idx, const double* params, double tol, double* out, const PriceScratch& s,
                cudaStream_t st, int32_t* nbis_out, const int32_t* surf_mask, const PanelSink& sink) {
    const int warps = OPE_KERNEL_WARPS, threads = warps * 32;
    const size_t smem = warps * sizeof(PanelStore);
    int grid = 0;
    OPE_TRY(persistent_grid(k_price_persistent<BATES, SAVE>, threads, smem, &grid));
    const unsigned long long need = (2ull * n + warps - 1) / warps;
    grid = (int)std::min<unsigned long long>((unsigned long long)grid, need);
    k_price_persistent<BATES, SAVE><<<grid, threads, smem, st>>>(con, (long long)n, surf_offsets, (long long)n_surf,
                                                                 param_idx, surf_mask, params, tol, out, s.integ,
                                                                 s.done, s.head, nbis_out, sink);
    OPE_CHECK(cudaGetLastError());
    return OPE_OK;
}

}  // namespace

int prepare_price_kernels() {
    const int threads = OPE_KERNEL_WARPS * 32;
    const size_t smem = OPE_KERNEL_WARPS * sizeof(PanelStore);
    int grid = 0;
    OPE_TRY(persistent_grid(k_price_persistent<false, false>, threads, smem, &grid));
    OPE_TRY(persistent_grid(k_price_persistent<true, false>, threads, smem, &grid));
    return OPE_OK;
}

int launch_price_persistent(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets,
                            size_t n_surf, const int32_t* param_idx, const double* params, double tol, double* out,
                            const PriceScratch& s, cudaStream_t st, int32_t* nbis_out, const int32_t* surf_mask,
                            const PanelSink* sink) {
    if (n == 0) return OPE_OK;
    // completion counters and queue head start at zero (one memset when adjacent)
    const size_t done_bytes = align_up(n * sizeof(unsigned int), 256);
    if (reinterpret_cast<char*>(s.head) == reinterpret_cast<char*>(s.done) + done_bytes) {
        OPE_CHECK(cudaMemsetAsync(s.done, 0, done_bytes + sizeof(unsigned long long), st));
    } else {
        OPE_CHECK(cudaMemsetAsync(s.done, 0, n * sizeof(unsigned int), st));
        OPE_CHECK(cudaMemsetAsync(s.head, 0, sizeof(unsigned long long), st));
    }
    const bool bates = model == OPE_MODEL_BATES;
    if (sink) {
        OPE_TRY((bates ? launch_impl<true, true> : launch_impl<false, true>)(
            con, n, surf_offsets, n_surf, param_idx, params, tol, out, s, st, nbis_out, surf_mask, *sink));
    } else {
        const PanelSink none{nullptr, nullptr, nullptr, 1};
        OPE_TRY((bates ? launch_impl<true, false> : launch_impl<false, false>)(
            con, n, surf_offsets, n_surf, param_idx, params, tol, out, s, st, nbis_out, surf_mask, none));
    }
    tctx().launches += 1;
    return OPE_OK;
}

}  // namespace ope
