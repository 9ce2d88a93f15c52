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

}  // namespace

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
