// Bump-and-reprice Greeks on the device (greeks.rs:19-72, reached through
// batch.rs:32-36 / 44-48).
//
// Each contract expands into the reference's 14 pricings (price, spot +-1%,
// vol +-1pt, T - 1 day, r +-1bp, the 4 spot x vol cross bumps and vol
// +-2pt).  All 14n virtual contracts go through ONE persistent pricing launch
// as ordinary work units (5 parameter sets: base and the four v0 bumps), and
// a combine kernel applies the reference's finite-difference formulas.  Bump
// arithmetic is rounded as the reference rounds it (no FMA contraction).
#include <cuda_runtime.h>

#include <algorithm>

#include "internal.h"

namespace ope {

namespace {

constexpr int kVariants = 14;

struct GreeksLayout {
    ope_contract* vcon;  // 14n
    int32_t* vidx;       // 14n
    double* vparams;     // 5 x 8
    double* vprice;      // 14n
    void* scratch;       // price scratch for 14n
};

GreeksLayout carve(void* ws, size_t n) {
    const size_t nv = kVariants * n;
    char* p = static_cast<char*>(ws);
    GreeksLayout L;
    L.vcon = reinterpret_cast<ope_contract*>(p);
    p += align_up(nv * sizeof(ope_contract), 256);
    L.vidx = reinterpret_cast<int32_t*>(p);
    p += align_up(nv * sizeof(int32_t), 256);
    L.vparams = reinterpret_cast<double*>(p);
    p += align_up(5 * 8 * sizeof(double), 256);
    L.vprice = reinterpret_cast<double*>(p);
    p += align_up(nv * sizeof(double), 256);
    L.scratch = p;
    return L;
}

// The five parameter sets: 0 base, 1 vol+dv, 2 vol-dv, 3 vol+2dv, 4 vol-2dv
// (v0 = (sqrt(v0) +- dv)^2 with the lower bump floored at 1e-8).
__global__ void k_greeks_params(const double* __restrict__ params, int stride, double* __restrict__ vp) {
    const int i = threadIdx.x;
    if (i >= 5) return;
    const double dv = 0.01;
    const double v_cur = sqrt(params[0]);
    double vol;
    switch (i) {
        case 1: vol = __dadd_rn(v_cur, dv); break;
        case 2: vol = fmax(__dsub_rn(v_cur, dv), 1e-8); break;
        case 3: vol = __dadd_rn(v_cur, 2.0 * dv); break;
        case 4: vol = fmax(__dsub_rn(v_cur, 2.0 * dv), 1e-8); break;
        default: vol = 0.0; break;
    }
    for (int k = 0; k < stride; ++k) vp[i * stride + k] = params[k];
    if (i > 0) vp[i * stride] = __dmul_rn(vol, vol);
}

__global__ void k_greeks_expand(const ope_contract* __restrict__ con, long long n, ope_contract* __restrict__ vcon,
                                int32_t* __restrict__ vidx) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n * kVariants) return;
    const long long c = g / kVariants;
    const int v = (int)(g % kVariants);
    ope_contract b = con[c];
    const double ds = __dmul_rn(0.01, b.spot);
    const double up = __dadd_rn(b.spot, ds), dn = __dsub_rn(b.spot, ds);
    const double dr = 1e-4, dt = 1.0 / 365.0;
    int pidx = 0;
    switch (v) {
        case 0: break;                                      // price
        case 1: b.spot = up; break;                         // pu
        case 2: b.spot = dn; break;                         // pd
        case 3: pidx = 1; break;                            // p_vup
        case 4: pidx = 2; break;                            // p_vdn
        case 5: b.expiry = fmax(__dsub_rn(b.expiry, dt), 1e-6); break;  // theta leg
        case 6: b.rate = __dadd_rn(b.rate, dr); break;      // rho up
        case 7: b.rate = __dsub_rn(b.rate, dr); break;      // rho down
        case 8: b.spot = up; pidx = 1; break;               // delta at vol up
        case 9: b.spot = dn; pidx = 1; break;
        case 10: b.spot = up; pidx = 2; break;              // delta at vol down
        case 11: b.spot = dn; pidx = 2; break;
        case 12: pidx = 3; break;                           // vol up 2
        case 13: pidx = 4; break;                           // vol down 2
    }
    vcon[g] = b;
    vidx[g] = pidx;
}

__global__ void k_greeks_combine(const ope_contract* __restrict__ con, long long n, const double* __restrict__ vp,
                                 ope_pricing_result* __restrict__ out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double* p = vp + c * kVariants;
    const double spot = con[c].spot;
    const double ds = __dmul_rn(0.01, spot), dv = 0.01, dr = 1e-4, dt = 1.0 / 365.0;
    const double price = p[0];
    ope_pricing_result r;
    r.price = price;
    r.delta = (p[1] - p[2]) / (2.0 * ds);
    r.gamma = __dadd_rn(__dsub_rn(p[1], 2.0 * price), p[2]) / __dmul_rn(ds, ds);
    r.vega = (p[3] - p[4]) / (2.0 * dv);
    r.theta = (p[5] - price) / dt;
    r.rho = (p[6] - p[7]) / (2.0 * dr);
    const double delta_vup = (p[8] - p[9]) / (2.0 * ds);
    const double delta_vdn = (p[10] - p[11]) / (2.0 * ds);
    r.vanna = (delta_vup - delta_vdn) / (2.0 * dv);
    const double vega_up = (p[12] - price) / (2.0 * dv);
    const double vega_dn = (price - p[13]) / (2.0 * dv);
    r.volga = (vega_up - vega_dn) / (2.0 * dv);
    out[c] = r;
}

// ---------------------------------------------------------------------------
// AD Greeks (ad.rs:736-795 heston_greeks_ad, 809-865 bates_greeks_ad): vega
// and volga from the exact d price / d v0 (the adjoint kernel, at the base
// v0 and at the two vol bumps), delta / gamma / theta / rho / vanna by the
// reference's finite differences.  Per contract: 9 pricings (r +- 1bp,
// spot +- 1%, T - 1 day, spot +- 1% at each vol bump) as work units of one
// persistent pricing launch, and 3 adjoint evaluations (base, vol up, vol
// down) as work units of one adjoint launch; then a combine kernel.
constexpr int kAdPricings = 9, kAdGrads = 3;

struct GreeksAdLayout {
    ope_contract* pcon;  // 9n
    int32_t* pidx;       // 9n
    double* pprice;      // 9n
    ope_contract* acon;  // 3n
    int32_t* aidx;       // 3n
    double* aprice;      // 3n
    double* agrad;       // 3n x dim
    double* vparams;     // 3 x 8
    void* scratch;       // pricing scratch for 9n, then adjoint scratch for 3n
};

GreeksAdLayout carve_ad(void* ws, size_t n, int dim) {
    char* p = static_cast<char*>(ws);
    GreeksAdLayout L;
    auto take = [&](size_t bytes) { char* r = p; p += align_up(bytes, 256); return r; };
    L.pcon = reinterpret_cast<ope_contract*>(take(kAdPricings * n * sizeof(ope_contract)));
    L.pidx = reinterpret_cast<int32_t*>(take(kAdPricings * n * sizeof(int32_t)));
    L.pprice = reinterpret_cast<double*>(take(kAdPricings * n * sizeof(double)));
    L.acon = reinterpret_cast<ope_contract*>(take(kAdGrads * n * sizeof(ope_contract)));
    L.aidx = reinterpret_cast<int32_t*>(take(kAdGrads * n * sizeof(int32_t)));
    L.aprice = reinterpret_cast<double*>(take(kAdGrads * n * sizeof(double)));
    L.agrad = reinterpret_cast<double*>(take(kAdGrads * n * dim * sizeof(double)));
    L.vparams = reinterpret_cast<double*>(take(3 * 8 * sizeof(double)));
    L.scratch = p;
    return L;
}

// Parameter sets: 0 base, 1 v0 = (vol + 0.01)^2, 2 v0 = max(vol - 0.01, 1e-6)^2 (ad.rs:768-769).
__global__ void k_greeks_ad_params(const double* __restrict__ params, int stride, double* __restrict__ vp) {
    const int i = threadIdx.x;
    if (i >= 3) return;
    const double vol = sqrt(params[0]);
    for (int k = 0; k < stride; ++k) vp[i * stride + k] = params[k];
    if (i == 1) { const double v = __dadd_rn(vol, 0.01); vp[i * stride] = __dmul_rn(v, v); }
    if (i == 2) { const double v = fmax(__dsub_rn(vol, 0.01), 1e-6); vp[i * stride] = __dmul_rn(v, v); }
}

__global__ void k_greeks_ad_expand(const ope_contract* __restrict__ con, long long n, ope_contract* __restrict__ pcon,
                                   int32_t* __restrict__ pidx, ope_contract* __restrict__ acon,
                                   int32_t* __restrict__ aidx) {
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n * (kAdPricings + kAdGrads)) return;
    const long long c = g / (kAdPricings + kAdGrads);
    const int v = (int)(g % (kAdPricings + kAdGrads));
    ope_contract b = con[c];
    if (v >= kAdPricings) {  // adjoint units: base, vol up, vol down
        const int a = v - kAdPricings;
        acon[c * kAdGrads + a] = b;
        aidx[c * kAdGrads + a] = a;
        return;
    }
    const double ds = __dmul_rn(0.01, b.spot);
    const double up = __dadd_rn(b.spot, ds), dn = __dsub_rn(b.spot, ds);
    const double dr = 1e-4, dt = 1.0 / 365.0;
    int pi = 0;
    switch (v) {
        case 0: b.rate = __dadd_rn(b.rate, dr); break;                  // rho legs (ad.rs:753-756)
        case 1: b.rate = __dsub_rn(b.rate, dr); break;
        case 2: b.spot = up; break;                                      // delta / gamma (ad.rs:760-764)
        case 3: b.spot = dn; break;
        case 4: b.expiry = fmax(__dsub_rn(b.expiry, dt), 1e-6); break;  // theta (ad.rs:766-768)
        case 5: b.spot = up; pi = 1; break;                              // vanna legs (ad.rs:771-779)
        case 6: b.spot = dn; pi = 1; break;
        case 7: b.spot = up; pi = 2; break;
        default: b.spot = dn; pi = 2; break;
    }
    pcon[c * kAdPricings + v] = b;
    pidx[c * kAdPricings + v] = pi;
}

__global__ void k_greeks_ad_combine(const ope_contract* __restrict__ con, long long n, const double* __restrict__ params,
                                    const double* __restrict__ pp, const double* __restrict__ ap,
                                    const double* __restrict__ ag, int dim, ope_pricing_result* __restrict__ out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double* p = pp + c * kAdPricings;
    const double spot = con[c].spot;
    const double ds = __dmul_rn(0.01, spot), dr = 1e-4, dt = 1.0 / 365.0;
    const double vol = sqrt(params[0]);
    const double price = ap[c * kAdGrads];
    const double dv0 = ag[(c * kAdGrads + 0) * dim], dv0_up = ag[(c * kAdGrads + 1) * dim],
                 dv0_dn = ag[(c * kAdGrads + 2) * dim];
    ope_pricing_result r;
    r.price = price;
    r.vega = __dmul_rn(dv0 * 2.0, vol);
    r.rho = (p[0] - p[1]) / (2.0 * dr);
    r.delta = (p[2] - p[3]) / (2.0 * ds);
    r.gamma = __dadd_rn(__dsub_rn(p[2], 2.0 * price), p[3]) / __dmul_rn(ds, ds);
    r.theta = (p[4] - price) / dt;
    const double delta_vup = (p[5] - p[6]) / (2.0 * ds);
    const double delta_vdn = (p[7] - p[8]) / (2.0 * ds);
    r.vanna = (delta_vup - delta_vdn) / (2.0 * 0.01);
    const double vega_up = __dmul_rn(dv0_up * 2.0, __dadd_rn(vol, 0.01));
    const double vega_dn = __dmul_rn(dv0_dn * 2.0, fmax(__dsub_rn(vol, 0.01), 1e-6));
    r.volga = (vega_up - vega_dn) / (2.0 * 0.01);
    out[c] = r;
}

}  // namespace

size_t greeks_ad_workspace_bytes(size_t n, int dim) {
    size_t b = 0;
    for (size_t x : {kAdPricings * n * sizeof(ope_contract), kAdPricings * n * sizeof(int32_t),
                     kAdPricings * n * sizeof(double), kAdGrads * n * sizeof(ope_contract),
                     kAdGrads * n * sizeof(int32_t), kAdGrads * n * sizeof(double),
                     kAdGrads * n * dim * sizeof(double), (size_t)3 * 8 * sizeof(double)})
        b += align_up(x, 256);
    return b + std::max(price_scratch_bytes(kAdPricings * n), grad_scratch_bytes(kAdGrads * n, dim));
}

int launch_greeks_ad(int model, const ope_contract* con, size_t n, const double* params, double tol,
                     ope_pricing_result* out, void* ws, cudaStream_t st) {
    if (n == 0) return OPE_OK;
    const int stride = param_stride(model);
    const GreeksAdLayout L = carve_ad(ws, n, stride);
    k_greeks_ad_params<<<1, 32, 0, st>>>(params, stride, L.vparams);
    OPE_CHECK(cudaGetLastError());
    const size_t nv = (kAdPricings + kAdGrads) * n;
    k_greeks_ad_expand<<<(unsigned)((nv + 255) / 256), 256, 0, st>>>(con, (long long)n, L.pcon, L.pidx, L.acon, L.aidx);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 2;
    OPE_TRY(launch_price_persistent(model, L.pcon, kAdPricings * n, nullptr, 3, L.pidx, L.vparams, tol, L.pprice,
                                    carve_price_scratch(L.scratch, kAdPricings * n), st));
    OPE_TRY(launch_price_grad(model, L.acon, kAdGrads * n, nullptr, 3, L.aidx, L.vparams, tol, L.aprice, L.agrad,
                              L.scratch, st));
    k_greeks_ad_combine<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(con, (long long)n, params, L.pprice, L.aprice,
                                                                     L.agrad, stride, out);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 1;
    return OPE_OK;
}

size_t greeks_workspace_bytes(size_t n) {
    const size_t nv = kVariants * n;
    return align_up(nv * sizeof(ope_contract), 256) + align_up(nv * sizeof(int32_t), 256) +
           align_up(5 * 8 * sizeof(double), 256) + align_up(nv * sizeof(double), 256) + price_scratch_bytes(nv);
}

int launch_greeks(int model, const ope_contract* con, size_t n, const double* params, double tol,
                  ope_pricing_result* out, void* ws, cudaStream_t st) {
    if (n == 0) return OPE_OK;
    const int stride = param_stride(model);
    GreeksLayout L = carve(ws, n);
    const size_t nv = kVariants * n;
    k_greeks_params<<<1, 32, 0, st>>>(params, stride, L.vparams);
    OPE_CHECK(cudaGetLastError());
    k_greeks_expand<<<(unsigned)((nv + 255) / 256), 256, 0, st>>>(con, (long long)n, L.vcon, L.vidx);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 2;
    OPE_TRY(launch_price_persistent(model, L.vcon, nv, nullptr, 5, L.vidx, L.vparams, tol, L.vprice,
                                    carve_price_scratch(L.scratch, nv), st));
    k_greeks_combine<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(con, (long long)n, L.vprice, out);
    OPE_CHECK(cudaGetLastError());
    tctx().launches += 1;
    return OPE_OK;
}

}  // namespace ope
