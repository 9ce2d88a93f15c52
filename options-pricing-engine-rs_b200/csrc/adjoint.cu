// Price + reverse-mode gradient: d price / d(v0, kappa, theta, sigma, rho[,
// lambda, mu_j, sigma_j]) for every contract of many surfaces.
//
// Reference: ad.rs:695-731 (forward_pass: derivative integrated by Leibniz
// over the primal's adaptive panel set, error control on the primal only),
// ad.rs:736-745 / 821-825 (the five Heston-parameter passes) and ad.rs:882-895
// (the three jump-parameter passes).  Three launches:
//   1. the pricing kernel itself (pricing.cu), which also stores every
//      integral's final live-panel list (prices are therefore bit-identical
//      to a plain pricing call);
//   2. the backward pass over chunks of up to 64 stored panels: a small
//      kernel lists every integral's chunks (ceil(len / 64) of them), then
//      warps pull chunks from that list; the 15 nodes of each panel are
//      spread over the 32 lanes, each lane recomputes the CF at its node and
//      runs the backward pass (cf_adjoint.cuh), accumulating all parameter
//      derivatives at once; for P1 one extra work item of the first chunk
//      evaluates the normaliser's dLog CF(-i)/dp; a warp reduction finishes
//      each chunk's partial sums.  Chunking spreads a long integral over
//      several warps, which matters when few integrals are left (the tail of
//      a calibration): the LM batch ran 126.5 -> 94.4 ms at unchanged
//      gradient throughput;
//   3. a per-contract combine: the chunks' partial sums in chunk order, the
//      P1 normaliser term, then ad.rs:713-730, d price = S e^{-qT} dI1/pi -
//      K e^{-rT} dI2/pi for calls and puts alike (parity terms do not depend
//      on the model parameters).
// Splitting the primal from the backward pass keeps each kernel's code small
// (the fused form stalled on instruction fetch) and lets each run at its own
// occupancy.
#include <cuda_runtime.h>

#include <algorithm>

#include "cf_adjoint.cuh"
#include "internal.h"
#include "quadrature.cuh"

// Minimum resident blocks per SM for the backward kernels' __launch_bounds__
// (caps registers per thread at 65536 / (128 * OPE_GRAD_MINB)): 5, i.e. 96
// registers.  The kernel time is flat from 4 to 7 blocks (within 0.5 % on the
// 262k-contract Bates gradient, 1 % on the Heston one), but at 7 blocks (72
// registers) its spills overflow L1: 274 MB of DRAM writes per 65,536 Bates
// contracts against 12 MB at 5 blocks (ncu, one launch).
#ifndef OPE_GRAD_MINB
#define OPE_GRAD_MINB 5
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

// Work items of the backward pass: chunks of kChunkPanels final panels of one
// integral (an integral of len panels has ceil(len / kChunkPanels) chunks),
// so a long integral's nodes are spread over several warps instead of
// running as one warp's serial loop.  64 panels per chunk: 32 gave the same
// calibration tail but cost 3 % of gradient throughput in per-chunk set-up.
constexpr int kChunkPanels = 64;
constexpr int kMaxChunks = (kMaxPanels + kChunkPanels - 1) / kChunkPanels;

// Per launch: the chunk list and each chunk's partial sums.
struct BackScratch {
    uint32_t* unit_base;        // first chunk slot of each integral
    uint8_t* nch;               // chunks of each integral (0 on masked surfaces)
    unsigned long long* work;   // chunk list: integral * 8 + chunk, in slot order
    double* part;               // per chunk slot: dim derivative sums, then sum W (re, im)
    double* normd;              // per contract: the P1 normaliser's dLog CF(-i)/dp (re, im)
    unsigned long long* count;  // [0] chunk slots allocated, [1] queue head
};

__device__ __forceinline__ long long unit_surface(const int32_t* param_idx, const int64_t* surf_off, long long n_surf,
                                                  long long c) {
    return param_idx ? (long long)__ldg(param_idx + c) : (n_surf > 1 ? find_surface_g(surf_off, n_surf, c) : 0);
}

// One thread per integral: its chunk count from the stored panel count, and a
// contiguous run of chunk slots (one atomic per warp after a warp scan).
__global__ void k_grad_chunks(long long n, const int64_t* __restrict__ surf_off, long long n_surf,
                              const int32_t* __restrict__ param_idx, const int32_t* __restrict__ surf_mask,
                              PanelSink src, BackScratch B) {
    const long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned lane = threadIdx.x & 31;
    int nch = 0;
    if (u < 2 * n) {
        const long long s = unit_surface(param_idx, surf_off, n_surf, u >> 1);
        if (!(surf_mask && __ldg(surf_mask + s) == 0)) {
            int slot = src.slot ? __ldg(src.slot + s) : 0;
            if (!ope_check(slot >= 0 && slot < src.n_slots, CHK_SLOT)) slot = 0;
            int len = __ldg(src.nbis + (size_t)u * src.n_slots + slot) + 1;
            if (!ope_check(len >= 1 && len <= kMaxPanels, CHK_PANEL_LEN)) len = len < 1 ? 1 : kMaxPanels;
            nch = (len + kChunkPanels - 1) / kChunkPanels;
        }
    }
    int incl = nch;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, off);
        if ((int)lane >= off) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    unsigned long long base = 0;
    if (lane == 31 && total > 0) base = atomicAdd(B.count, (unsigned long long)total);
    base = __shfl_sync(0xffffffffu, base, 31);
    if (u < 2 * n) {
        const unsigned long long first = base + (unsigned long long)(incl - nch);
        B.unit_base[u] = (uint32_t)first;
        B.nch[u] = (uint8_t)nch;
        for (int j = 0; j < nch; ++j) B.work[first + j] = (unsigned long long)u * 8ull + (unsigned long long)j;
    }
}

template <bool BATES>
__global__ void __launch_bounds__(128, OPE_GRAD_MINB) k_grad_backward(const ope_contract* __restrict__ con, long long n,
                                                      const int64_t* __restrict__ surf_off, long long n_surf,
                                                      const int32_t* __restrict__ param_idx,
                                                      const double* __restrict__ params, PanelSink src,
                                                      BackScratch B) {
    constexpr int DIM = BATES ? 8 : 5;
    __shared__ double s_norm[4][16];  // per warp: the P1 normaliser's dLog CF(-i)/dp (complex, DIM <= 8)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const LaneRule R = lane_rule(lane);
    const unsigned long long n_work = *(volatile unsigned long long*)B.count;  // final: set by k_grad_chunks
    while (true) {
        unsigned long long w = 0;
        if (lane == 0) w = atomicAdd(B.count + 1, 1ull);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= n_work) break;
        const unsigned long long e = __ldg(B.work + w);
        const unsigned long long unit = e >> 3;
        const int chunk = (int)(e & 7ull);
        if (!ope_check(unit < 2ull * (unsigned long long)n && chunk < kMaxChunks, CHK_PANEL_INDEX)) continue;
        const long long c = (long long)(unit >> 1);
        const int which = (int)(unit & 1);
        const long long s = unit_surface(param_idx, surf_off, n_surf, c);
        const double* p = params + s * DIM;
        double pl[8];
#pragma unroll
        for (int i = 0; i < DIM; ++i) pl[i] = __ldg(p + i);
        const ope_contract* cp = con + c;
        const CfConsts C = make_consts(__ldg(&cp->spot), __ldg(&cp->strike), __ldg(&cp->expiry), __ldg(&cp->rate),
                                       pl, BATES, which);
        const GradParams G = make_grad_params(pl, BATES);
        int slot = src.slot ? __ldg(src.slot + s) : 0;
        if (!ope_check(slot >= 0 && slot < src.n_slots, CHK_SLOT)) slot = 0;
        const size_t pidx = (size_t)unit * src.n_slots + slot;
        int len = __ldg(src.nbis + pidx) + 1;
        if (!ope_check(len >= 1 && len <= kMaxPanels, CHK_PANEL_LEN)) len = len < 1 ? 1 : kMaxPanels;
        const int p0 = chunk * kChunkPanels, p1 = min(len, p0 + kChunkPanels);
        const double* P = src.panels + pidx * (2 * kMaxPanels) + 2 * p0;
        double acc[DIM];
#pragma unroll
        for (int k = 0; k < DIM; ++k) acc[k] = 0.0;
        double sw_re = 0.0, sw_im = 0.0;
        const bool with_norm = which == 0 && chunk == 0;
        const int total = 15 * max(p1 - p0, 0);
        const int items = total + (with_norm ? 1 : 0);
        for (int base = 0; base < items; base += 32) {
            const int idx = base + lane;
            const int pi = idx / 15, j = idx - 15 * (idx / 15);
            const double xj = __shfl_sync(0xffffffffu, R.x, j & 15);
            const double wj = __shfl_sync(0xffffffffu, R.wk, j & 15);
            if (idx < items) {
                const bool normaliser = idx == total;
                double tn = 0.0, hw = 0.0, u = 0.0, itt = 0.0;
                if (!normaliser) {
                    const double a = __ldg(P + 2 * pi), b = __ldg(P + 2 * pi + 1);
                    const double cc = 0.5 * (a + b), h = 0.5 * (b - a);
                    tn = __dadd_rn(cc, __dmul_rn(h, xj));
                    hw = h * wj;
                    const double omt = 1.0 - tn;
                    itt = rcp_nr(omt * tn);  // 1 / ((1 - t) t), as the pricing node evaluation
                    u = (omt * omt) * itt;   // (1 - t) / t
                }
                C2 dz[8];
                const C2 Z = exponent_and_grad<BATES>(C, G, u, dz);
                if (normaliser) {
#pragma unroll
                    for (int k = 0; k < DIM; ++k) { s_norm[warp][2 * k] = dz[k].re; s_norm[warp][2 * k + 1] = dz[k].im; }
                } else {
                    node_accumulate<BATES>(Z, dz, (tn > 0.0) && (u >= 1e-12), itt, hw, acc, sw_re, sw_im);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < DIM; ++k) acc[k] = warp_sum(acc[k]);
        sw_re = warp_sum(sw_re);
        sw_im = warp_sum(sw_im);
        __syncwarp();
        if (lane == 0) {
            double* out = B.part + w * (DIM + 2);
#pragma unroll
            for (int k = 0; k < DIM; ++k) out[k] = acc[k];
            out[DIM] = sw_re;
            out[DIM + 1] = sw_im;
            if (with_norm) {
#pragma unroll
                for (int k = 0; k < 2 * DIM; ++k) B.normd[c * 2 * DIM + k] = s_norm[warp][k];
            }
        }
        __syncwarp();  // s_norm is read before the next work item rewrites it
    }
}

// ad.rs:713-730 per contract; contracts of masked surfaces are left untouched.
// Each integral's derivative is the sum of its chunks' partial sums, in chunk
// order.  For P1 the normaliser term -dLog CF(-i)/dp * sum W (constant over
// the integral; zero up to rounding for a regular normaliser, ad.rs:705-706
// carries it through the Dual division) is applied here; where it is not
// finite (e.g. kappa < rho sigma puts xi + d = 0 at phi = -i), every P1 node's
// derivative is non-finite in the reference, so every node is dropped
// (ad.rs:679-682) and the component is 0.
template <int DIM>
__global__ void k_grad_combine(const ope_contract* __restrict__ con, long long n, const int64_t* __restrict__ surf_off,
                               long long n_surf, const int32_t* __restrict__ param_idx,
                               const int32_t* __restrict__ surf_mask, BackScratch B,
                               double* __restrict__ out_grad) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    if (surf_mask) {
        const long long s = unit_surface(param_idx, surf_off, n_surf, c);
        if (surf_mask[s] == 0) return;
    }
    double d[2][DIM];
#pragma unroll
    for (int which = 0; which < 2; ++which) {
        const long long u = 2 * c + which;
        const double* part = B.part + (size_t)B.unit_base[u] * (DIM + 2);
        const int nc = B.nch[u];
        double sw_re = 0.0, sw_im = 0.0;
#pragma unroll
        for (int k = 0; k < DIM; ++k) d[which][k] = 0.0;
        for (int j = 0; j < nc; ++j) {
#pragma unroll
            for (int k = 0; k < DIM; ++k) d[which][k] += part[j * (DIM + 2) + k];
            sw_re += part[j * (DIM + 2) + DIM];
            sw_im += part[j * (DIM + 2) + DIM + 1];
        }
        if (which == 0) {
#pragma unroll
            for (int k = 0; k < DIM; ++k) {
                const C2 dl = c2(B.normd[c * 2 * DIM + 2 * k], B.normd[c * 2 * DIM + 2 * k + 1]);
                d[0][k] = (isfinite(dl.re) && isfinite(dl.im)) ? d[0][k] - (dl * c2(sw_re, sw_im)).im : 0.0;
            }
        }
    }
    const ope_contract& cp = con[c];
    const double PI = 3.14159265358979323846;
    const double seq = cp.spot * exp(-cp.div_yield * cp.expiry), ker = cp.strike * exp(-cp.rate * cp.expiry);
#pragma unroll
    for (int k = 0; k < DIM; ++k) out_grad[c * DIM + k] = seq * (d[0][k] / PI) - ker * (d[1][k] / PI);
}

// The analytic Greeks' backward pass: the work list of k_grad_backward
// (chunks of stored panels), per node the seven Greek integrands of
// cf_adjoint.cuh (d/dx, d2/dx2, d/dr, d/dT, d/dv0, d2/dx dv0, d2/dv0^2 of the
// node value), a warp sum per chunk.  One parameter set per contract, as the
// reference's AD Greeks take (ad.rs:736-865).
template <bool BATES>
__global__ void __launch_bounds__(128, OPE_GRAD_MINB) k_greeks_backward(const ope_contract* __restrict__ con, long long n,
                                                        const int64_t* __restrict__ surf_off, long long n_surf,
                                                        const int32_t* __restrict__ param_idx,
                                                        const double* __restrict__ params, PanelSink src,
                                                        BackScratch B) {
    constexpr int DIM = BATES ? 8 : 5;
    const int lane = threadIdx.x & 31;
    const LaneRule R = lane_rule(lane);
    const unsigned long long n_work = *(volatile unsigned long long*)B.count;  // final: set by k_grad_chunks
    while (true) {
        unsigned long long w = 0;
        if (lane == 0) w = atomicAdd(B.count + 1, 1ull);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= n_work) break;
        const unsigned long long e = __ldg(B.work + w);
        const unsigned long long unit = e >> 3;
        const int chunk = (int)(e & 7ull);
        if (!ope_check(unit < 2ull * (unsigned long long)n && chunk < kMaxChunks, CHK_PANEL_INDEX)) continue;
        const long long c = (long long)(unit >> 1);
        const int which = (int)(unit & 1);
        const long long s = unit_surface(param_idx, surf_off, n_surf, c);
        const double* p = params + s * DIM;
        double pl[8];
#pragma unroll
        for (int i = 0; i < DIM; ++i) pl[i] = __ldg(p + i);
        const ope_contract* cp = con + c;
        const double r = __ldg(&cp->rate);
        const CfConsts C = make_consts(__ldg(&cp->spot), __ldg(&cp->strike), __ldg(&cp->expiry), r, pl, BATES, which);
        const double is2 = 1.0 / (pl[3] * pl[3]);
        const double lambda = BATES ? pl[5] : 0.0;
        int slot = src.slot ? __ldg(src.slot + s) : 0;
        if (!ope_check(slot >= 0 && slot < src.n_slots, CHK_SLOT)) slot = 0;
        const size_t pidx = (size_t)unit * src.n_slots + slot;
        int len = __ldg(src.nbis + pidx) + 1;
        if (!ope_check(len >= 1 && len <= kMaxPanels, CHK_PANEL_LEN)) len = len < 1 ? 1 : kMaxPanels;
        const int p0 = chunk * kChunkPanels, p1 = min(len, p0 + kChunkPanels);
        const double* P = src.panels + pidx * (2 * kMaxPanels) + 2 * p0;
        double acc[7];
#pragma unroll
        for (int k = 0; k < 7; ++k) acc[k] = 0.0;
        const int items = 15 * max(p1 - p0, 0);
        for (int base = 0; base < items; base += 32) {
            const int idx = base + lane;
            const int pi = idx / 15, j = idx - 15 * (idx / 15);
            const double xj = __shfl_sync(0xffffffffu, R.x, j & 15);
            const double wj = __shfl_sync(0xffffffffu, R.wk, j & 15);
            if (idx < items) {
                const double a = __ldg(P + 2 * pi), b = __ldg(P + 2 * pi + 1);
                const double cc = 0.5 * (a + b), h = 0.5 * (b - a);
                const double tn = __dadd_rn(cc, __dmul_rn(h, xj));
                const double omt = 1.0 - tn;
                const double itt = rcp_nr(omt * tn);  // 1 / ((1 - t) t)
                const double u = node_u(omt, tn, itt);
                C2 Zv, ZT;
                const C2 Z = exponent_and_greeks<BATES>(C, u, r, lambda, is2, Zv, ZT);
                greeks_accumulate(Z, Zv, ZT, u, C.t, (tn > 0.0) && (u >= 1e-12), itt, h * wj, acc);
            }
        }
#pragma unroll
        for (int k = 0; k < 7; ++k) acc[k] = warp_sum(acc[k]);
        if (lane == 0) {
            double* out = B.part + w * 7;
#pragma unroll
            for (int k = 0; k < 7; ++k) out[k] = acc[k];
        }
    }
}

// Per contract: the eight Greeks from the two integrals (I1, I2 of the
// pricing launch), their seven derivative integrals and the Gil-Pelaez
// combination (heston.rs:95-98, 70), in the reference's conventions
// (greeks.rs:19-72): delta = dP/dS, gamma = d2P/dS2, vega = dP/dsqrt(v0),
// theta = -dP/dT (per year), rho = dP/dr, vanna = d2P/dS dsqrt(v0),
// volga = d2P/dsqrt(v0)^2.  With a = S e^{-qT}, b = K e^{-rT},
// P_j = 1/2 + I_j/pi and x = ln(S/K), the call a P1 - b P2 gives
//   dC/dS  = e^{-qT} P1 + e^{-qT} I1x/pi - b I2x/(pi S)
//   dC2/dS2 = e^{-qT} (I1x + I1xx)/(pi S) - b (I2xx - I2x)/(pi S^2)
//   dC/dr  = a I1r/pi + T b P2 - b I2r/pi,  dC/dT = -q a P1 + a I1T/pi + r b P2 - b I2T/pi
// and the v0 terms alike; where the reference clamps the call at 0 its
// derivatives are 0; the put (C - a + b) adds -e^{-qT}, -T b and q a - r b.
template <int DIM>
__global__ void k_greeks_combine(const ope_contract* __restrict__ con, long long n, const double* __restrict__ integ,
                                 const double* __restrict__ price, const double* __restrict__ params, BackScratch B,
                                 ope_pricing_result* __restrict__ out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    double G[2][7];
#pragma unroll
    for (int which = 0; which < 2; ++which) {
        const long long u = 2 * c + which;
        const double* part = B.part + (size_t)B.unit_base[u] * 7;
        const int nc = B.nch[u];
#pragma unroll
        for (int k = 0; k < 7; ++k) G[which][k] = 0.0;
        for (int j = 0; j < nc; ++j)
#pragma unroll
            for (int k = 0; k < 7; ++k) G[which][k] += part[j * 7 + k];
    }
    const ope_contract& k = con[c];
    const double PI = 3.14159265358979323846;
    const double S = k.spot, T = k.expiry, r = k.rate, q = k.div_yield, v0 = params[0];
    const double eq = exp(-q * T), er = exp(-r * T);
    const double a = S * eq, b = k.strike * er;
    const double p1 = 0.5 + integ[2 * c] / PI, p2 = 0.5 + integ[2 * c + 1] / PI;
    const bool live = a * p1 - b * p2 > 0.0;  // heston.rs:98: the call is clamped at 0
    double dS = 0.0, dSS = 0.0, dr = 0.0, dT = 0.0, dv = 0.0, dSv = 0.0, dvv = 0.0;
    if (live) {
        dS = eq * p1 + eq * G[0][0] / PI - b * G[1][0] / (PI * S);
        dSS = eq * (G[0][0] + G[0][1]) / (PI * S) - b * (G[1][1] - G[1][0]) / (PI * S * S);
        dr = a * G[0][2] / PI + T * b * p2 - b * G[1][2] / PI;
        dT = -q * a * p1 + a * G[0][3] / PI + r * b * p2 - b * G[1][3] / PI;
        dv = (a * G[0][4] - b * G[1][4]) / PI;
        dSv = eq * G[0][4] / PI + eq * G[0][5] / PI - b * G[1][5] / (PI * S);
        dvv = (a * G[0][6] - b * G[1][6]) / PI;
    }
    if (k.opt_type != 0) {  // put = call - S e^{-qT} + K e^{-rT} (heston.rs:70)
        dS -= eq;
        dr -= T * b;
        dT += q * a - r * b;
    }
    const double sv = sqrt(v0);
    ope_pricing_result o;
    o.price = price[c];
    o.delta = dS;
    o.gamma = dSS;
    o.vega = 2.0 * sv * dv;
    o.theta = -dT;
    o.rho = dr;
    o.vanna = 2.0 * sv * dSv;
    o.volga = 2.0 * dv + 4.0 * v0 * dvv;
    out[c] = o;
}

template <class K>
int grad_grid(K kernel, size_t smem, unsigned long long need, int* grid) {
    int per_sm = 0;
    OPE_TRY(blocks_per_sm(reinterpret_cast<const void*>(kernel), 128, smem, &per_sm));
    int sms = 0;
    OPE_TRY(current_device_sms(&sms));
    const int cap = std::max(1, (int)(per_sm * sms * tctx().grid_fraction));
    *grid = (int)std::min<unsigned long long>((unsigned long long)cap, need);
    return OPE_OK;
}

}  // namespace

size_t grad_backward_bytes(size_t n, int dim) {
    const size_t units = 2 * n, slots = units * kMaxChunks;
    return align_up(units * sizeof(uint32_t), 256) + align_up(units, 256) +
           align_up(slots * sizeof(unsigned long long), 256) + align_up(slots * (dim + 2) * sizeof(double), 256) +
           align_up(n * 2 * dim * sizeof(double), 256) + 256;
}

namespace {

BackScratch carve_back_scratch(void* base, size_t n, int dim) {
    const size_t units = 2 * n, slots = units * kMaxChunks;
    char* p = static_cast<char*>(base);
    BackScratch B;
    B.unit_base = reinterpret_cast<uint32_t*>(p);
    p += align_up(units * sizeof(uint32_t), 256);
    B.nch = reinterpret_cast<uint8_t*>(p);
    p += align_up(units, 256);
    B.work = reinterpret_cast<unsigned long long*>(p);
    p += align_up(slots * sizeof(unsigned long long), 256);
    B.part = reinterpret_cast<double*>(p);
    p += align_up(slots * (dim + 2) * sizeof(double), 256);
    B.normd = reinterpret_cast<double*>(p);
    p += align_up(n * 2 * dim * sizeof(double), 256);
    B.count = reinterpret_cast<unsigned long long*>(p);
    return B;
}

}  // namespace

size_t grad_scratch_bytes(size_t n, int dim) {
    return price_scratch_bytes(n) + panel_sink_bytes(n, 1) + grad_backward_bytes(n, dim);
}

int launch_grad_backward(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                         const int32_t* param_idx, const double* params, const PanelSink& src, void* bscratch,
                         double* out_grad, cudaStream_t st, const int32_t* surf_mask) {
    if (n == 0) return OPE_OK;
    const int dim = param_stride(model);
    const BackScratch B = carve_back_scratch(bscratch, n, dim);
    OPE_CHECK(cudaMemsetAsync(B.count, 0, 2 * sizeof(unsigned long long), st));
    const unsigned long long units = 2ull * n;
    k_grad_chunks<<<(unsigned)((units + 127) / 128), 128, 0, st>>>((long long)n, surf_offsets, (long long)n_surf,
                                                                   param_idx, surf_mask, src, B);
    OPE_CHECK(cudaGetLastError());
    const unsigned long long need = (units * kMaxChunks + 3) / 4;
    int grid = 0;
    if (model == OPE_MODEL_BATES) {
        OPE_TRY(grad_grid(k_grad_backward<true>, 0, need, &grid));
        k_grad_backward<true><<<grid, 128, 0, st>>>(con, (long long)n, surf_offsets, (long long)n_surf, param_idx,
                                                    params, src, B);
    } else {
        OPE_TRY(grad_grid(k_grad_backward<false>, 0, need, &grid));
        k_grad_backward<false><<<grid, 128, 0, st>>>(con, (long long)n, surf_offsets, (long long)n_surf, param_idx,
                                                     params, src, B);
    }
    OPE_CHECK(cudaGetLastError());
    const unsigned cb = (unsigned)((n + 127) / 128);
    if (dim == 8)
        k_grad_combine<8><<<cb, 128, 0, st>>>(con, (long long)n, surf_offsets, (long long)n_surf, param_idx, surf_mask,
                                              B, out_grad);
    else
        k_grad_combine<5><<<cb, 128, 0, st>>>(con, (long long)n, surf_offsets, (long long)n_surf, param_idx, surf_mask,
                                              B, out_grad);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 3;
    return OPE_OK;
}

size_t greeks_analytic_workspace_bytes(size_t n) {
    return align_up(n * sizeof(double), 256) + price_scratch_bytes(n) + panel_sink_bytes(n, 1) +
           grad_backward_bytes(n, 5);  // 5 + 2 = 7 sums per chunk
}

int launch_greeks_analytic(int model, const ope_contract* con, size_t n, const double* params, double tol,
                           ope_pricing_result* out, void* ws, cudaStream_t st) {
    if (n == 0) return OPE_OK;
    char* p = static_cast<char*>(ws);
    double* price = reinterpret_cast<double*>(p);
    p += align_up(n * sizeof(double), 256);
    const PriceScratch s = carve_price_scratch(p, n);
    p += price_scratch_bytes(n);
    const PanelSink sink = carve_panel_sink(p, n, 1, nullptr);
    p += panel_sink_bytes(n, 1);
    const BackScratch B = carve_back_scratch(p, n, 5);
    // 1. prices, the integrals I1, I2 (s.integ) and the final panel lists
    OPE_TRY(launch_price_persistent(model, con, n, nullptr, 1, nullptr, params, tol, price, s, st, nullptr, nullptr,
                                    &sink));
    // 2. the Greek integrals over those panels, 3. the combination
    OPE_CHECK(cudaMemsetAsync(B.count, 0, 2 * sizeof(unsigned long long), st));
    const unsigned long long units = 2ull * n;
    k_grad_chunks<<<(unsigned)((units + 127) / 128), 128, 0, st>>>((long long)n, nullptr, 1, nullptr, nullptr, sink, B);
    OPE_CHECK(cudaGetLastError());
    const unsigned long long need = (units * kMaxChunks + 3) / 4;
    int grid = 0;
    if (model == OPE_MODEL_BATES) {
        OPE_TRY(grad_grid(k_greeks_backward<true>, 0, need, &grid));
        k_greeks_backward<true><<<grid, 128, 0, st>>>(con, (long long)n, nullptr, 1, nullptr, params, sink, B);
    } else {
        OPE_TRY(grad_grid(k_greeks_backward<false>, 0, need, &grid));
        k_greeks_backward<false><<<grid, 128, 0, st>>>(con, (long long)n, nullptr, 1, nullptr, params, sink, B);
    }
    OPE_CHECK(cudaGetLastError());
    const unsigned cb = (unsigned)((n + 127) / 128);
    if (model == OPE_MODEL_BATES)
        k_greeks_combine<8><<<cb, 128, 0, st>>>(con, (long long)n, s.integ, price, params, B, out);
    else
        k_greeks_combine<5><<<cb, 128, 0, st>>>(con, (long long)n, s.integ, price, params, B, out);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 3;
    return OPE_OK;
}

int launch_price_grad(int model, const ope_contract* con, size_t n, const int64_t* surf_offsets, size_t n_surf,
                      const int32_t* param_idx, const double* params, double tol, double* out_price,
                      double* out_grad, void* scratch, cudaStream_t st, const int32_t* surf_mask) {
    if (n == 0) return OPE_OK;
    char* p = static_cast<char*>(scratch);
    const PriceScratch s = carve_price_scratch(p, n);
    p += price_scratch_bytes(n);
    const PanelSink sink = carve_panel_sink(p, n, 1, nullptr);
    p += panel_sink_bytes(n, 1);
    // 1. prices and the final panel lists, 2. the backward pass and combine
    OPE_TRY(launch_price_persistent(model, con, n, surf_offsets, n_surf, param_idx, params, tol, out_price, s, st,
                                    nullptr, surf_mask, &sink));
    return launch_grad_backward(model, con, n, surf_offsets, n_surf, param_idx, params, sink, p, out_grad, st,
                                surf_mask);
}

}  // namespace ope
