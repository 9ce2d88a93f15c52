// Device implied volatility: the calibration residuals are in IV space.
//
// Reference: iv.rs:14-95 (implied_vol: bounds check, Brenner-Subrahmanyam
// seed, Halley with at most 10 steps at 1e-10, bisection fallback of 60
// steps), bsm.rs:8-12, 55-60 (bsm_price), bsm.rs:15-40 (vega), math.rs:10-19
// (npdf, ncdf via erfc).  Same control flow and constants; the arithmetic
// uses CUDA's exp/log/erfc/sqrt (agreement with the CPU libm is at the ulp
// level).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "../../include/ope.h"

namespace ope {

struct IvC {
    double s, k, t, r, q;
    int opt;
};

__device__ __forceinline__ double npdf_d(double x) { return 0.3989422804014327 * exp((-0.5 * x) * x); }
__device__ __forceinline__ double ncdf_d(double x) { return 0.5 * erfc(-x * 0.70710678118654752440); }

// bsm.rs:55-60
__device__ __forceinline__ double bsm_price_d(const IvC& c, double v) {
    const double vt = v * sqrt(c.t);
    const double d1 = (log(c.s / c.k) + ((c.r - c.q) + (0.5 * v) * v) * c.t) / vt;
    const double d2 = d1 - vt;
    const double phi = c.opt == 0 ? 1.0 : -1.0;
    return phi * ((c.s * exp(-c.q * c.t)) * ncdf_d(phi * d1) - (c.k * exp(-c.r * c.t)) * ncdf_d(phi * d2));
}

// bsm.rs:15-40 vega (per unit vol)
__device__ __forceinline__ double bsm_vega_d(const IvC& c, double v) {
    const double sqt = sqrt(c.t);
    const double vt = v * sqt;
    const double d1 = (log(c.s / c.k) + ((c.r - c.q) + (0.5 * v) * v) * c.t) / vt;
    return ((c.s * exp(-c.q * c.t)) * npdf_d(d1)) * sqt;
}

// iv.rs:85-95
__device__ __forceinline__ void vega_volga_d(const IvC& c, double v, double* vega, double* volga) {
    const double vt = v * sqrt(c.t);
    const double d1 = (log(c.s / c.k) + ((c.r - c.q) + (0.5 * v) * v) * c.t) / vt;
    const double d2 = d1 - vt;
    const double vg = ((c.s * exp(-c.q * c.t)) * npdf_d(d1)) * sqrt(c.t);
    *vega = vg;
    *volga = ((vg * d1) * d2) / v;
}

// iv.rs:52-63
__device__ __forceinline__ bool bisect_d(const IvC& c, double target, double* out) {
    double lo = 1e-4, hi = 10.0;
    if ((bsm_price_d(c, lo) - target) * (bsm_price_d(c, hi) - target) > 0.0) return false;
    for (int i = 0; i < 60; ++i) {
        const double mid = 0.5 * (lo + hi);
        if (bsm_price_d(c, mid) - target < 0.0) lo = mid; else hi = mid;
        if (hi - lo < 1e-9) { *out = mid; return true; }
    }
    *out = 0.5 * (lo + hi);
    return true;
}

// iv.rs:14-49, 65-83
__device__ __forceinline__ bool implied_vol_d(const IvC& c, double mkt, double* out) {
    // price_in_bounds (iv.rs:22-31)
    if (!(mkt > 0.0)) return false;
    const double er = exp(-c.r * c.t), eq = exp(-c.q * c.t);
    const double intrinsic = c.opt == 0 ? fmax(c.s * eq - c.k * er, 0.0) : fmax(c.k * er - c.s * eq, 0.0);
    if (!(mkt >= intrinsic)) return false;
    // initial_guess (iv.rs:36-49)
    const double fwd = (c.s * eq) / er;
    const double bs = (mkt * sqrt((2.0 * 3.14159265358979323846) / c.t)) / (fwd * er);
    const double x = log(fwd / c.k);
    double v = bs / fmax(exp((-0.5 * x) * x), 0.01);
    v = fmin(fmax(v, 0.001), 10.0);
    if (!(fabs(bsm_price_d(c, v) - mkt) < 0.2 * mkt)) {
        if (!bisect_d(c, mkt, &v)) return false;
    }
    // halley_solve (iv.rs:65-83)
    for (int it = 0; it < 10; ++it) {
        const double err = bsm_price_d(c, v) - mkt;
        if (fabs(err) < 1e-10) { *out = v; return true; }
        double vega, volga;
        vega_volga_d(c, v, &vega, &volga);
        if (fabs(vega) < 1e-14) return false;
        double denom = 1.0 - (err * volga) / ((2.0 * vega) * vega);
        denom = fmin(fmax(denom, 0.5), 2.0);
        v -= err / (vega * denom);
        if (v <= 0.0) v = 1e-8;
    }
    if (fabs(bsm_price_d(c, v) - mkt) < 1e-6) { *out = v; return true; }
    return false;
}

__device__ __forceinline__ IvC iv_contract(const ope_contract& q) {
    return IvC{q.spot, q.strike, q.expiry, q.rate, q.div_yield, q.opt_type};
}

}  // namespace ope
