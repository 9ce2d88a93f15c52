// Reverse-mode derivative of one Gil-Pelaez node with respect to the model
// parameters (v0, kappa, theta, sigma, rho[, lambda, mu_j, sigma_j]).
//
// Reference: ad.rs:609-731 (forward-mode Dual through stable_cf_dual,
// jump_factor and dual_integrand, integrated over the primal's adaptive
// panel set).  Same quantity, computed backwards: the node value is
//
//     g(t) = Im(W) / (u t^2),  W = exp(Z),  Z = kts*Ch + v0s*Dh + i r phi T + i u x - Log CF(-i) [+ J]
//
// with Ch = (xi-d)T - 2 Log A and Dh = (xi-d)(1-e)/(1-g e) (the C and D of
// heston.rs:123-124 without their real prefactors kappa*theta/sigma^2 and
// v0/sigma^2).  Every intermediate is a holomorphic function of the two
// complex inputs xi and z = xi^2 + sigma^2 phi(phi+i), so the whole backward
// pass reduces to two complex partials Z_xi, Z_z (chain rule through
// d = sqrt z, g = (xi-d)/(xi+d), e = exp(-dT), A = (ge-1)/(g-1)), which are
// then chained to each real parameter:
//
//   dZ/dv0    = Dh / sigma^2
//   dZ/dkappa = Y + Ch * theta / sigma^2          Y = Z_xi + 2 xi Z_z
//   dZ/dtheta = Ch * kappa / sigma^2
//   dZ/dsigma = Y rho s + Z_z 2 sigma w - 2 kts Ch / sigma - 2 v0s Dh / sigma
//   dZ/drho   = Y sigma s                          s = phi_im - i u, w = phi(phi+i)
//
// and dg/dp = Im(W dZ/dp) / (u t^2).  The CF is recomputed here, nothing from
// the primal pass is stored.  The P1 normaliser term -dLog CF(-i)/dp is the
// same expression at phi = -i; since it is constant over the integral its
// contribution is applied once per integral to the sum of W/(u t^2) weights.
#pragma once

#include "cf_device.cuh"

namespace ope {

struct C2 {
    double re, im;
};
__device__ __forceinline__ C2 c2(double re, double im) { return C2{re, im}; }
__device__ __forceinline__ C2 operator+(C2 a, C2 b) { return C2{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ C2 operator-(C2 a, C2 b) { return C2{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ C2 operator*(C2 a, C2 b) { return C2{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ C2 operator*(C2 a, double s) { return C2{a.re * s, a.im * s}; }
__device__ __forceinline__ C2 operator*(double s, C2 a) { return C2{a.re * s, a.im * s}; }
// 1/a with one refined reciprocal (rcp_nr); a = 0 gives a non-finite result,
// which drops the node as a division by zero does in the reference.
__device__ __forceinline__ C2 crcp(C2 a) {
    const double inv = rcp_nr(a.re * a.re + a.im * a.im);
    return C2{a.re * inv, -a.im * inv};
}

// Real model parameters for the chain to (v0, kappa, theta, sigma, rho, ...).
struct GradParams {
    double v0, kappa, theta, sigma, rho;
    double sigma_j;
    double is2;     // 1 / sigma^2
    double sk, sv;  // 2 kts / sigma and 2 v0s / sigma (kts, v0s as in make_consts)
};

__device__ __forceinline__ GradParams make_grad_params(const double* p, bool bates) {
    GradParams G;
    G.v0 = p[0];
    G.kappa = p[1];
    G.theta = p[2];
    G.sigma = p[3];
    G.rho = p[4];
    G.sigma_j = bates ? p[7] : 0.0;
    G.is2 = 1.0 / (p[3] * p[3]);
    G.sk = 2.0 * ((p[1] * p[2]) / (p[3] * p[3])) / p[3];
    G.sv = 2.0 * (p[0] / (p[3] * p[3])) / p[3];
    return G;
}

// dZ/dp at (u, phi_im) for every parameter (dim = 5 or 8), plus W = exp(Z)
// (W only meaningful for u > 0).  `out` receives dZ/dp as complex numbers.
template <bool BATES>
__device__ __forceinline__ C2 exponent_and_grad(const CfConsts& C, const GradParams& P, double u, C2* out) {
    const double T = C.t;
    const C2 xi = c2(C.kappa + C.rs * C.phi_im, -C.rs * u);
    const C2 wphi = c2(u * u, C.sgn * u);  // phi(phi+i)
    const C2 z = xi * xi + wphi * C.sig2;
    C2 d;
    csqrt_node(z.re, z.im, d.re, d.im);
    const C2 m = xi - d, p = xi + d;
    const C2 ip = crcp(p);
    const C2 g = m * ip;
    double sn, cs;
    sincos(-d.im * T, &sn, &cs);
    const double em = exp(-d.re * T);
    const C2 e = c2(em * cs, em * sn);
    const C2 ge = g * e;
    const C2 N = c2(ge.re - 1.0, ge.im);  // g e - 1  (= -(1 - g e))
    const C2 M = c2(g.re - 1.0, g.im);    // g - 1
    const C2 iM = crcp(M);
    const C2 iN = crcp(N);
    const C2 A = N * iM;
    const C2 lnA = c2(0.5 * log(A.re * A.re + A.im * A.im), atan2_node(A.im, A.re));
    const C2 om = c2(1.0 - e.re, -e.im);  // 1 - e
    const C2 iQ = c2(-iN.re, -iN.im);     // 1/(1 - g e)
    const C2 Ch = m * T - lnA * 2.0;
    const C2 Dh = m * om * iQ;
    // Z (without the Log CF(-i) normaliser, added by the caller through C.lnm)
    C2 Z = Ch * C.kts + Dh * C.v0s + c2(-C.rt * C.phi_im + C.lnm_re, C.rt * u + u * C.x + C.lnm_im);

    // backward: holomorphic partials through d, g, e, A
    const C2 ip2 = ip * ip;
    const C2 g_xi = d * ip2 * 2.0;
    const C2 g_d = xi * ip2 * (-2.0);
    const C2 e_d = e * (-T);
    const C2 iMN = iM * iN;
    const C2 C_xi = (c2(T, 0.0) - om * g_xi * iMN * 2.0) * C.kts;
    const C2 C_d = (c2(-T, 0.0) - (om * g_d * iMN + g * e_d * iN) * 2.0) * C.kts;
    const C2 iQ2 = iQ * iQ;
    const C2 mom = m * om;
    const C2 D_xi = (om * iQ + mom * e * g_xi * iQ2) * C.v0s;
    const C2 D_d = (c2(-om.re, -om.im) * iQ - m * e_d * iQ + mom * (g_d * e + g * e_d) * iQ2) * C.v0s;
    const C2 Z_xi = C_xi + D_xi;
    const C2 Z_z = (C_d + D_d) * crcp(d * 2.0);
    const C2 Y = Z_xi + xi * Z_z * 2.0;
    const C2 s = c2(C.phi_im, -u);
    const double is2 = P.is2;
    out[0] = Dh * is2;                                                     // v0
    out[1] = Y + Ch * (P.theta * is2);                                     // kappa
    out[2] = Ch * (P.kappa * is2);                                         // theta
    out[3] = Y * s * P.rho + Z_z * wphi * (2.0 * P.sigma) - Ch * P.sk - Dh * P.sv;  // sigma
    out[4] = Y * s * P.sigma;                                              // rho
    if (BATES) {
        const C2 iphi = c2(-C.phi_im, u);
        const C2 phi2 = c2(u * u - C.phi_im * C.phi_im, 2.0 * u * C.phi_im);
        const double jr_in = -C.phi_im * C.mu_j - C.hs2 * phi2.re;
        const double ji_in = u * C.mu_j - C.hs2 * phi2.im;
        double js, jc;
        sincos(ji_in, &js, &jc);
        const double je = exp(jr_in);
        const C2 jump = c2(je * jc, je * js);
        const C2 base = jump - c2(1.0, 0.0) - iphi * C.comp;
        Z = Z + base * C.lt;
        out[5] = base * T;                                                            // lambda
        out[6] = iphi * (jump - c2(1.0 + C.comp, 0.0)) * C.lt;                        // mu_j
        out[7] = (c2(-(jump * phi2).re, -(jump * phi2).im) - iphi * (1.0 + C.comp)) *
                 (C.lt * P.sigma_j);                                                  // sigma_j
    }
    return Z;
}

// One node of the derivative integral from its exponent Z and dZ/dp (from
// exponent_and_grad at u = (1 - tn)/tn, with itt = 1/((1 - tn) tn) =
// 1/(u tn^2)): adds hw * dg/dp into acc[0..dim) and hw * W/(u t^2) into sw
// (for the P1 normaliser term).  A node outside the substitution's domain
// (`inside` false: t <= 0 or u < 1e-12, heston.rs:222-225) or whose value or
// derivative is not finite contributes zero, as in gk_integrate_dual
// (ad.rs:679-682).
template <bool BATES>
__device__ __forceinline__ void node_accumulate(const C2& Z, const C2* dz, bool inside, double itt, double hw,
                                                double* acc, double& sw_re, double& sw_im) {
    constexpr int DIM = BATES ? 8 : 5;
    double sn, cs;
    sincos(Z.im, &sn, &cs);
    const double ez = exp(Z.re);
    const C2 Wf = c2(ez * cs * itt, ez * sn * itt);
    const double v = Wf.im;
    bool ok = inside && isfinite(v);
    double gk[8];
#pragma unroll
    for (int k = 0; k < DIM; ++k) {
        gk[k] = (Wf * dz[k]).im;
        ok = ok && isfinite(gk[k]);
    }
    if (ok) {
#pragma unroll
        for (int k = 0; k < DIM; ++k) acc[k] += hw * gk[k];
        sw_re += hw * Wf.re;
        sw_im += hw * Wf.im;
    }
}

// The exponent Z of one node with its derivatives with respect to v0 and
// to the expiry T, for the analytic Greeks (x = ln(S/K) and r enter Z as
// i u x and i u r T -- the P1 normaliser's r T cancels the real part of
// i r phi T -- so their derivatives need nothing from here):
//   dZ/dv0 = Dh / sigma^2
//   dZ/dT  = kts (m - 2 g d e / (1 - g e)) + v0s m d e (1 - g) / (1 - g e)^2 + i r u [+ lambda base]
// with m = xi - d, e = exp(-d T) (de/dT = -d e), and for Bates J = lambda T base
// (the normaliser's own T-dependence, r T, is already taken out: the jump
// factor at phi = -i is 1 and C, D vanish there).
template <bool BATES>
__device__ __forceinline__ C2 exponent_and_greeks(const CfConsts& C, double u, double r, double lambda, double is2,
                                                  C2& Zv, C2& ZT) {
    const double T = C.t;
    const C2 xi = c2(C.kappa + C.rs * C.phi_im, -C.rs * u);
    const C2 wphi = c2(u * u, C.sgn * u);  // phi(phi+i)
    const C2 z = xi * xi + wphi * C.sig2;
    C2 d;
    csqrt_node(z.re, z.im, d.re, d.im);
    const C2 m = xi - d, p = xi + d;
    const C2 g = m * crcp(p);
    double sn, cs;
    sincos(-d.im * T, &sn, &cs);
    const double em = exp(-d.re * T);
    const C2 e = c2(em * cs, em * sn);
    const C2 ge = g * e;
    const C2 N = c2(ge.re - 1.0, ge.im);  // g e - 1
    const C2 A = N * crcp(c2(g.re - 1.0, g.im));
    const C2 lnA = c2(0.5 * log(A.re * A.re + A.im * A.im), atan2_node(A.im, A.re));
    const C2 iN = crcp(N);
    const C2 iQ = c2(-iN.re, -iN.im);  // 1/(1 - g e)
    const C2 om = c2(1.0 - e.re, -e.im);
    const C2 Ch = m * T - lnA * 2.0;
    const C2 Dh = m * om * iQ;
    C2 Z = Ch * C.kts + Dh * C.v0s + c2(-C.rt * C.phi_im + C.lnm_re, C.rt * u + u * C.x + C.lnm_im);
    Zv = Dh * is2;
    const C2 de = d * e;
    const C2 dCh = m - g * de * iQ * 2.0;
    const C2 dDh = m * de * c2(1.0 - g.re, -g.im) * (iQ * iQ);
    ZT = dCh * C.kts + dDh * C.v0s + c2(0.0, r * u);
    if (BATES) {
        const C2 iphi = c2(-C.phi_im, u);
        const C2 phi2 = c2(u * u - C.phi_im * C.phi_im, 2.0 * u * C.phi_im);
        double js, jc;
        sincos(u * C.mu_j - C.hs2 * phi2.im, &js, &jc);
        const double je = exp(-C.phi_im * C.mu_j - C.hs2 * phi2.re);
        const C2 base = c2(je * jc, je * js) - c2(1.0, 0.0) - iphi * C.comp;
        Z = Z + base * C.lt;
        ZT = ZT + base * lambda;
    }
    return Z;
}

// Sums of the analytic-Greek integrands of one node into acc[0..7):
// d/dx, d2/dx2, d/dr, d/dT, d/dv0, d2/dx dv0, d2/dv0^2 of g = Im(W) / (u t^2),
// weighted by hw; with Z linear in x (i u x) and in v0 (v0 Dh / sigma^2) the
// second derivatives are Im(W Zp Zq) / (u t^2).  A node outside the
// substitution's domain or with a non-finite value contributes zero.
__device__ __forceinline__ void greeks_accumulate(const C2& Z, const C2& Zv, const C2& ZT, double u, double T,
                                                  bool inside, double itt, double hw, double* acc) {
    double sn, cs;
    sincos(Z.im, &sn, &cs);
    const double ez = exp(Z.re);
    const C2 Wf = c2(ez * cs * itt, ez * sn * itt);
    const C2 Wv = Wf * Zv;
    double g[7];
    g[0] = u * Wf.re;        // Im(W i u)
    g[1] = -u * u * Wf.im;   // Im(W (i u)^2)
    g[2] = u * T * Wf.re;    // Im(W i u T)
    g[3] = (Wf * ZT).im;
    g[4] = Wv.im;
    g[5] = u * Wv.re;        // Im(W Zv i u)
    g[6] = (Wv * Zv).im;
    bool ok = inside && isfinite(Wf.im);
#pragma unroll
    for (int k = 0; k < 7; ++k) ok = ok && isfinite(g[k]);
    if (ok) {
#pragma unroll
        for (int k = 0; k < 7; ++k) acc[k] += hw * g[k];
    }
}

}  // namespace ope
