// Price + reverse-mode gradient kernel: d price / d(v0, kappa, theta, sigma,
// rho[, lambda, mu_j, sigma_j]) for every contract of many surfaces.
//
// Reference: ad.rs:695-731 (forward_pass: derivative integrated by Leibniz
// over the primal's adaptive panel set, error control on the primal only),
// ad.rs:736-745 / 821-825 (the five Heston-parameter passes) and ad.rs:882-895
// (the three jump-parameter passes).  One unit = one integral, one warp:
//   1. the primal greedy GK15 integration (identical to the pricing kernel),
//      leaving the final live-panel list in shared memory;
//   2. the derivative integral over those panels: the 15 * len nodes are
//      spread over the 32 lanes, each lane recomputes the CF at its node and
//      runs the backward pass (cf_adjoint.cuh), accumulating all parameter
//      derivatives at once; a warp reduction finishes the sums.
// The price combination is heston.rs:95-98 and the derivative combination is
// ad.rs:713-730: d price = S e^{-qT} dI1/pi - K e^{-rT} dI2/pi for calls and
// puts alike (parity terms do not depend on the model parameters).
#include <cuda_runtime.h>

#include <algorithm>

#include "cf_adjoint.cuh"
#include "internal.h"
#include "quadrature.cuh"

// Minimum resident blocks per SM for the adjoint kernel's __launch_bounds__
// (caps registers per thread at 65536 / (128 * OPE_GRAD_MINB)).
#ifndef OPE_GRAD_MINB
#define OPE_GRAD_MINB 7
#endif

namespace ope {

namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

__device__ __forceinline__ long long find_surface_g(const int64_t* off, long long n_surf, long long c) {
    long long lo = 1, hi = n_surf;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (__ldg(off + mid) > c) hi = mid; else lo = mid + 1;
    }
    return lo - 1;
}

template <bool BATES>
__global__ void __launch_bounds__(128, OPE_GRAD_MINB) k_price_grad(const ope_contract* __restrict__ con, long long n,
                                                    const int64_t* __restrict__ surf_off, long long n_surf,
                                                    const int32_t* __restrict__ param_idx,
                                                    const int32_t* __restrict__ surf_mask,
                                                    const double* __restrict__ params, double tol,
                                                    double* __restrict__ out_price, double* __restrict__ out_grad,
                                                    double* integ, double* ginteg, unsigned int* done,
                                                    unsigned long long* head) {
    constexpr int DIM = BATES ? 8 : 5;
    extern __shared__ PanelStore smem_panels[];
    __shared__ double s_norm[4][16];  // per warp: the P1 normaliser's dLog CF(-i)/dp (complex, DIM <= 8)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    PanelStore& L = smem_panels[warp];
    const LaneRule R = lane_rule(lane);
    const unsigned long long n_units = 2ull * (unsigned long long)n;
    while (true) {
        unsigned long long unit = 0;
        if (lane == 0) unit = atomicAdd(head, 1ull);
        unit = __shfl_sync(0xffffffffu, unit, 0);
        if (unit >= n_units) break;
        const long long c = (long long)(unit >> 1);
        const int which = (int)(unit & 1);
        const long long s = param_idx ? (long long)__ldg(param_idx + c)
                                      : (n_surf > 1 ? find_surface_g(surf_off, n_surf, c) : 0);
        if (surf_mask && __ldg(surf_mask + s) == 0) {
            // a skipped surface's units are contiguous: move the queue head past
            // all of them with one atomic instead of one per unit
            if (lane == 0 && !param_idx && surf_off)
                atomicMax(head, 2ull * (unsigned long long)__ldg(surf_off + s + 1));
            continue;
        }
        const double* p = params + s * DIM;
        double pl[8];
#pragma unroll
        for (int i = 0; i < DIM; ++i) pl[i] = __ldg(p + i);
        const ope_contract* cp = con + c;
        const double S = __ldg(&cp->spot), K = __ldg(&cp->strike), T = __ldg(&cp->expiry), r = __ldg(&cp->rate),
                     q = __ldg(&cp->div_yield);
        const int ot = __ldg(&cp->opt_type);
        const CfConsts C = make_consts(S, K, T, r, pl, BATES, which);
        int nb;
        const double I = gk_integrate_warp<BATES>(C, tol, L, lane, R, &nb);
        const int len = nb + 1;

        // derivative integral over the final panel set; for P1 one extra work
        // item evaluates the normaliser's dLog CF(-i)/dp (u = 0), so that the
        // kernel holds ONE inlined copy of exponent_and_grad
        const GradParams G = make_grad_params(pl, BATES);
        double acc[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) acc[k] = 0.0;
        double sw_re = 0.0, sw_im = 0.0;
        const int total = 15 * len;
        const int items = total + (which == 0 ? 1 : 0);
        for (int base = 0; base < items; base += 32) {
            const int idx = base + lane;
            const int pi = idx / 15, j = idx - 15 * (idx / 15);
            const double xj = __shfl_sync(0xffffffffu, R.x, j & 15);
            const double wj = __shfl_sync(0xffffffffu, R.wk, j & 15);
            if (idx < items) {
                const bool normaliser = idx == total;
                double tn = 0.0, hw = 0.0, u = 0.0;
                if (!normaliser) {
                    const double a = L.a[pi], b = L.b[pi];
                    const double cc = 0.5 * (a + b), h = 0.5 * (b - a);
                    tn = __dadd_rn(cc, __dmul_rn(h, xj));
                    hw = h * wj;
                    u = (1.0 - tn) / tn;
                }
                C2 dz[8];
                const C2 Z = exponent_and_grad<BATES>(C, G, u, dz);
                if (normaliser) {
#pragma unroll
                    for (int k = 0; k < DIM; ++k) { s_norm[warp][2 * k] = dz[k].re; s_norm[warp][2 * k + 1] = dz[k].im; }
                } else {
                    node_accumulate<BATES>(Z, dz, tn, u, hw, acc, sw_re, sw_im);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < DIM; ++k) acc[k] = warp_sum(acc[k]);
        sw_re = warp_sum(sw_re);
        sw_im = warp_sum(sw_im);
        if (which == 0) {
            // -d Log CF(-i)/dp, constant over the integral (zero up to rounding for a
            // regular normaliser; ad.rs:705-706 carries it through the Dual division)
            __syncwarp();
#pragma unroll
            for (int k = 0; k < DIM; ++k)
                acc[k] -= (c2(s_norm[warp][2 * k], s_norm[warp][2 * k + 1]) * c2(sw_re, sw_im)).im;
            __syncwarp();
        }
        if (lane == 0) {
            integ[2 * c + which] = I;
#pragma unroll
            for (int k = 0; k < DIM; ++k) ginteg[(2 * c + which) * DIM + k] = acc[k];
            __threadfence();
            const unsigned int prev = atomicAdd(done + c, 1u);
            if (prev == 1u) {
                __threadfence();
                const int o = 1 - which;
                const double other = __ldcg(integ + 2 * c + o);
                const double i1 = which == 0 ? I : other, i2 = which == 0 ? other : I;
                out_price[c] = finish_price(S, K, T, r, q, ot, i1, i2);
                const double PI = 3.14159265358979323846;
                const double seq = S * exp(-q * T), ker = K * exp(-r * T);
#pragma unroll
                for (int k = 0; k < DIM; ++k) {
                    const double og = __ldcg(ginteg + (2 * c + o) * DIM + k);
                    const double d1 = which == 0 ? acc[k] : og, d2 = which == 0 ? og : acc[k];
                    out_grad[c * DIM + k] = seq * (d1 / PI) - ker * (d2 / PI);
                }
            }
        }
    }
}

template <class K>
int grad_grid(K kernel, size_t smem, unsigned long long need, int* grid) {
    int per_sm = 0;
    OPE_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    OPE_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 128, smem));
    if (per_sm < 1) per_sm = 1;
    const int cap = std::max(1, (int)(per_sm * tctx().sm_count * tctx().grid_fraction));
    *grid = (int)std::min<unsigned long long>((unsigned long long)cap, need);
    return OPE_OK;
}

}  // namespace

size_t grad_scratch_bytes(size_t n, int dim) {
    return price_scratch_bytes(n) + align_up(2 * n * dim * sizeof(double), 256);
}

int launch_price_grad(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                      const int32_t* param_idx, const double* params, double tol, double* out_price,
                      double* out_grad, void* scratch, cudaStream_t st, const int32_t* surf_mask) {
    if (n == 0) return OPE_OK;
    const PriceScratch s = carve_price_scratch(scratch, n);
    double* ginteg = reinterpret_cast<double*>(static_cast<char*>(scratch) + price_scratch_bytes(n));
    OPE_CHECK(cudaMemsetAsync(s.done, 0, n * sizeof(unsigned int), st));
    OPE_CHECK(cudaMemsetAsync(s.head, 0, sizeof(unsigned long long), st));
    const size_t smem = 4 * sizeof(PanelStore);
    const unsigned long long need = (2ull * n + 3) / 4;
    int grid = 0;
    if (model == OPE_MODEL_BATES) {
        OPE_TRY(grad_grid(k_price_grad<true>, smem, need, &grid));
        k_price_grad<true><<<grid, 128, smem, st>>>(con, (long long)n, surf_offsets, (long long)n_surf, param_idx,
                                                    surf_mask, params, tol, out_price, out_grad, s.integ, ginteg, s.done, s.head);
    } else {
        OPE_TRY(grad_grid(k_price_grad<false>, smem, need, &grid));
        k_price_grad<false><<<grid, 128, smem, st>>>(con, (long long)n, surf_offsets, (long long)n_surf, param_idx,
                                                     surf_mask, params, tol, out_price, out_grad, s.integ, ginteg, s.done, s.head);
    }
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 1;
    return OPE_OK;
}

}  // namespace ope
