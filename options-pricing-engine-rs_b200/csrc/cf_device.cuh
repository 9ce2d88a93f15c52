// Device-side characteristic functions and Gil-Pelaez integrand (FP64).
//
// Reference: heston.rs:101-127 (cf_integrand, stable_cf), heston.rs:155-175
// (fast_csqrt), heston.rs:220-227 (the [0,inf) -> [0,1] substitution),
// bates.rs:65-83 (bates_integrand, jump_cf).
//
// One call of `node_value` evaluates gk_integrate's g(t) at one GK node:
// u = (1-t)/t, f(u)/t^2, non-finite -> 0.  The Albrecher stable CF is
// evaluated with its per-contract constants hoisted into CfConsts.  The
// three exponential factors the reference multiplies together per node
// (stable_cf's exp, the jump factor's outer exp and e^{iux}), the division
// by the P1 normaliser CF(-i) and the final division by iu are merged into
// ONE complex exponent Z:
//
//     Re[ e^{iux} * CF(phi) / CF(-i) / (iu) ] = e^{Re Z} * sin(Im Z) / u,
//     Z = i r phi T + C + D [+ J] + i u x - Log CF(-i)
//
// which is the same number up to rounding (exp(a)exp(b) = exp(a+b)), and
// trades four complex exponentials and two complex divisions per node for
// one real exp and one sin.  Log CF(-i) is computed once per integral from
// CF(-i) evaluated with the reference's own operation sequence, so the
// degenerate cases (CF(-i) = 0, inf or NaN) zero the P1 integrand exactly as
// the reference's division does.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace ope {

struct Cx {
    double re, im;
};

__device__ __forceinline__ Cx cadd(Cx a, Cx b) { return Cx{a.re + b.re, a.im + b.im}; }
__device__ __forceinline__ Cx csub(Cx a, Cx b) { return Cx{a.re - b.re, a.im - b.im}; }
__device__ __forceinline__ Cx cmul(Cx a, Cx b) {
    return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ Cx cscale(Cx a, double s) { return Cx{a.re * s, a.im * s}; }
// conj/|b|^2 division (the num-complex algorithm), with one reciprocal.
__device__ __forceinline__ Cx cdiv(Cx a, Cx b) {
    double inv = 1.0 / (b.re * b.re + b.im * b.im);
    return Cx{(a.re * b.re + a.im * b.im) * inv, (a.im * b.re - a.re * b.im) * inv};
}
__device__ __forceinline__ Cx cexp(Cx z) {
    double s, c;
    sincos(z.im, &s, &c);
    double e = exp(z.re);
    return Cx{e * c, e * s};
}
__device__ __forceinline__ Cx clog(Cx z) { return Cx{log(hypot(z.re, z.im)), atan2(z.im, z.re)}; }

// heston.rs:155-175 fast_csqrt, branch-free: the safe component is
// w = sqrt((|a| + r)/2); the other is b/(2w) (its magnitude when a < 0).
// Same values as the reference's two branches, including the b == 0 cases.
__device__ __forceinline__ Cx fast_csqrt(double a, double b) {
    double r = hypot(a, b);
    double w = sqrt(0.5 * (r + fabs(a)));
    double q = (w > 0.0) ? (0.5 * b) / w : b;
    return (a >= 0.0) ? Cx{w, q} : Cx{fabs(q), copysign(w, b)};
}

// Per-integral constants (everything that does not depend on the node).
struct CfConsts {
    double kappa;    // kappa
    double rs;       // rho * sigma
    double sig2;     // sigma^2
    double kts;      // kappa * theta / sigma^2
    double v0s;      // v0 / sigma^2
    double t;        // expiry T
    double rt;       // r * T
    double x;        // ln(S/K)
    double phi_im;   // -1 for P1 (phi = u - i), 0 for P2 (phi = u)
    double sgn;      // Im of phi*(phi+i) / u: -1 for P1, +1 for P2
    double lnm_re;   // -Re Log CF(-i) for P1, 0 for P2
    double lnm_im;   // -Im Log CF(-i) for P1, 0 for P2
    // Bates (bates.rs:77-83); lt = 0 switches the jump factor off.
    double lt;       // lambda * T
    double mu_j;     // mu_j
    double hs2;      // 0.5 * sigma_j^2
    double comp;     // e^{mu_j + sigma_j^2/2} - 1
};

// stable_cf at a general complex phi, following heston.rs:113-127's operation
// order (used once per integral for the P1 normaliser CF(-i)).
__device__ __forceinline__ Cx stable_cf_ref(Cx phi, double t, double r, double v0, double kappa,
                                            double theta, double sigma, double rho) {
    const Cx I{0.0, 1.0};
    Cx xi = csub(Cx{kappa, 0.0}, cmul(cscale(phi, rho * sigma), I));
    Cx z = cadd(cmul(xi, xi), cmul(cscale(phi, sigma * sigma), cadd(phi, I)));
    Cx d = fast_csqrt(z.re, z.im);
    Cx g = cdiv(csub(xi, d), cadd(xi, d));
    Cx edt = cexp(cscale(Cx{-d.re, -d.im}, t));
    Cx ge = cmul(g, edt);
    Cx a = cdiv(Cx{ge.re - 1.0, ge.im}, Cx{g.re - 1.0, g.im});
    Cx la = clog(a);
    Cx xmd = csub(xi, d);
    Cx c = cscale(Cx{xmd.re * t - 2.0 * la.re, xmd.im * t - 2.0 * la.im}, (kappa * theta) / (sigma * sigma));
    Cx num = cmul(cscale(xmd, v0), Cx{1.0 - edt.re, 0.0 - edt.im});
    Cx den = cscale(Cx{1.0 - ge.re, 0.0 - ge.im}, sigma * sigma);
    Cx dd = cdiv(num, den);
    Cx e = cadd(cadd(cscale(cmul(cscale(phi, r), I), t), c), dd);
    return cexp(e);
}

// bates.rs:77-83 jump_cf at a general complex phi (normaliser only).
__device__ __forceinline__ Cx jump_cf_ref(Cx phi, double t, double lambda, double mu_j, double sigma_j) {
    const Cx I{0.0, 1.0};
    double comp = exp(mu_j + (0.5 * sigma_j) * sigma_j) - 1.0;
    Cx a = cscale(cmul(phi, I), mu_j);
    Cx b = cscale(cscale(cmul(cscale(phi, 0.5), phi), sigma_j), sigma_j);
    Cx jump = cexp(csub(a, b));
    Cx inner = csub(Cx{jump.re - 1.0, jump.im}, cscale(cmul(I, phi), comp));
    return cexp(cscale(inner, lambda * t));
}

// Build the per-integral constants.  which: 0 = P1 (stock measure), 1 = P2.
__device__ __forceinline__ CfConsts make_consts(double s, double k, double t, double r, const double* p,
                                                bool bates, int which) {
    const double v0 = p[0], kappa = p[1], theta = p[2], sigma = p[3], rho = p[4];
    CfConsts C;
    C.kappa = kappa;
    C.rs = rho * sigma;
    C.sig2 = sigma * sigma;
    C.kts = (kappa * theta) / (sigma * sigma);
    C.v0s = v0 / (sigma * sigma);
    C.t = t;
    C.rt = r * t;
    C.x = log(s / k);
    C.phi_im = (which == 0) ? -1.0 : 0.0;
    C.sgn = (which == 0) ? -1.0 : 1.0;
    if (bates) {
        C.lt = p[5] * t;
        C.mu_j = p[6];
        C.hs2 = 0.5 * p[7] * p[7];
        C.comp = exp(p[6] + (0.5 * p[7]) * p[7]) - 1.0;
    } else {
        C.lt = 0.0;
        C.mu_j = 0.0;
        C.hs2 = 0.0;
        C.comp = 0.0;
    }
    C.lnm_re = 0.0;
    C.lnm_im = 0.0;
    if (which == 0) {
        const Cx phi_mi{0.0, -1.0};
        Cx m = stable_cf_ref(phi_mi, t, r, v0, kappa, theta, sigma, rho);
        if (bates) m = cmul(m, jump_cf_ref(phi_mi, t, p[5], p[6], p[7]));
        Cx lm = clog(m);
        C.lnm_re = -lm.re;
        C.lnm_im = -lm.im;
    }
    return C;
}

// gk_integrate's g(t) (heston.rs:221-227) with the merged-exponent integrand.
template <bool BATES>
__device__ __forceinline__ double node_value(const CfConsts& C, double tn) {
    const double u = (1.0 - tn) / tn;
    // xi = kappa - i*rho*sigma*phi,  phi = u + i*phi_im
    const double xr = C.kappa + C.rs * C.phi_im;
    const double xi = -C.rs * u;
    // z = xi^2 + sigma^2 * phi*(phi+i);  phi*(phi+i) = (u^2, sgn*u) for both integrals
    const double zr = (xr * xr - xi * xi) + C.sig2 * (u * u);
    const double zi = 2.0 * xr * xi + C.sig2 * (C.sgn * u);
    const Cx d = fast_csqrt(zr, zi);
    const double amr = xr - d.re, ami = xi - d.im;  // xi - d
    const double apr = xr + d.re, api = xi + d.im;  // xi + d
    // g = (xi - d) / (xi + d)
    const double ig = 1.0 / (apr * apr + api * api);
    const double gr = (amr * apr + ami * api) * ig;
    const double gi = (ami * apr - amr * api) * ig;
    // e = exp(-d T)
    double sn, cs;
    sincos(-d.im * C.t, &sn, &cs);
    const double em = exp(-d.re * C.t);
    const double er = em * cs, ei = em * sn;
    // g e
    const double ger = gr * er - gi * ei;
    const double gei = gr * ei + gi * er;
    // A = (g e - 1) / (g - 1)
    const double nr = ger - 1.0, ni = gei;
    const double dr = gr - 1.0, di = gi;
    const double ia = 1.0 / (dr * dr + di * di);
    const double ar = (nr * dr + ni * di) * ia;
    const double ai = (ni * dr - nr * di) * ia;
    // Log A
    const double lr = 0.5 * log(ar * ar + ai * ai);
    const double li = atan2(ai, ar);
    // D = v0/sigma^2 * (xi - d)(1 - e) / (1 - g e)
    const double omr = 1.0 - er, omi = -ei;
    const double pr = amr * omr - ami * omi;
    const double pim = amr * omi + ami * omr;
    const double qr = 1.0 - ger, qi = -gei;
    const double iq = 1.0 / (qr * qr + qi * qi);
    const double Dr = C.v0s * (pr * qr + pim * qi) * iq;
    const double Di = C.v0s * (pim * qr - pr * qi) * iq;
    // C = kappa theta / sigma^2 * ((xi - d) T - 2 Log A)
    const double Cr = C.kts * (amr * C.t - 2.0 * lr);
    const double Ci = C.kts * (ami * C.t - 2.0 * li);
    // i r phi T = (-rT*phi_im, rT*u);  i u x;  minus Log CF(-i)
    double zre = Cr + Dr - C.rt * C.phi_im + C.lnm_re;
    double zim = Ci + Di + C.rt * u + u * C.x + C.lnm_im;
    if (BATES) {
        // J = lambda T (exp(i phi mu_j - phi^2 sigma_j^2/2) - 1 - i phi comp)
        const double jr_in = -C.phi_im * C.mu_j - C.hs2 * (u * u - C.phi_im * C.phi_im);
        const double ji_in = u * C.mu_j - C.hs2 * (2.0 * u * C.phi_im);
        double js, jc;
        sincos(ji_in, &js, &jc);
        const double je = exp(jr_in);
        zre += C.lt * (je * jc - 1.0 + C.phi_im * C.comp);
        zim += C.lt * (je * js - u * C.comp);
    }
    const double v = (exp(zre) * sin(zim) / u) / (tn * tn);
    const bool ok = (tn > 0.0) && (u >= 1e-12) && isfinite(v);
    return ok ? v : 0.0;
}

}  // namespace ope
