// Device-side characteristic functions and Gil-Pelaez integrand (FP64).
//
// Reference: heston.rs:101-127 (cf_integrand, stable_cf), heston.rs:155-175
// (fast_csqrt), heston.rs:220-227 (the [0,inf) -> [0,1] substitution),
// bates.rs:65-83 (bates_integrand, jump_cf).
//
// `node_cf` + `node_finish` evaluate gk_integrate's g(t) at one GK node:
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
//
// Of Z only the phase u x depends on the strike (x = ln(S/K)); the rest is a
// function of the node, the expiry, the rate, the parameters and the
// integral.  So the evaluation is split: node_cf gives the strike-free part
// (e^{Re Z} and Im Z without u x), node_finish adds one strike's phase and
// forms the value.  Contracts of one surface that share
// an expiry and a rate share node_cf's values at every panel they both
// bisect (the run cache of quadrature.cuh).
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace ope {

struct Cx {
    double re, im;
};

// Reciprocal and reciprocal square root: the hardware approximation
// (rcp/rsqrt.approx.ftz.f64, about 2^-22 relative error) refined by two
// Newton-Raphson steps, y <- y + y(1 - x y) and y <- y + y(1/2 - x y^2 / 2),
// each of which squares the relative error, so the result is within an ulp
// or two of the correctly rounded value (checked against IEEE division and
// sqrt by ope_selftest_math).  Used for the complex reciprocals and the
// square root of the node evaluation; a zero or infinite argument gives a
// non-finite result, which zeroes the node exactly as the reference's
// division by zero does.
__device__ __forceinline__ double rcp_nr(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}
__device__ __forceinline__ double rsqrt_nr(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double hx = 0.5 * x;
    double e = fma(-hx * y, y, 0.5);
    y = fma(y, e, y);
    e = fma(-hx * y, y, 0.5);
    return fma(y, e, y);
}

// arg(A) of the node evaluation's Log A: atan2(y, x), branch-free, written
// for this use (CUDA's atan2 was the costliest call of a node: replacing it
// cut the Bates batch by 4 %).  Method (the classical argument reduction of
// Cody and Waite's elementary-function manual): octant symmetry reduces it
// to atan(q), q = min(|x|,|y|)/max(|x|,|y|) in [0, 1]; above tan(pi/8),
// atan(q) = pi/4 + atan((q - 1)/(q + 1)); on |t| <= tan(pi/8),
// atan(t) = t + t s P(s), s = t^2, with the degree-10 Chebyshev interpolant P
// of node_math_coeffs.py (5e-18 relative).  The two quotients use rcp_nr.  At most
// 4 ulp from CUDA's atan2 over finite arguments whose larger magnitude is at
// least 2^-1022 (ope_selftest_atan2); outside that (a NaN or infinite
// argument, or both below 2^-1022) it returns NaN.  In the node evaluation
// those cases come only from an A that is 0, infinite or NaN, where log|A| is
// not finite and the node's value is 0 with either function.
__device__ __forceinline__ double atan2_node(double y, double x) {
    const double ax = fabs(x), ay = fabs(y);
    const bool swap = ay > ax;
    const double q = (swap ? ax : ay) * rcp_nr(swap ? ay : ax);
    const bool big = q > 0.41421356237309503;  // tan(pi/8)
    const double t = big ? (q - 1.0) * rcp_nr(q + 1.0) : q;
    const double s = t * t;
    double p = -0.01917688711906226;
    p = fma(p, s, 0.03923165829558719);
    p = fma(p, s, -0.0508544973794026);
    p = fma(p, s, 0.0585814891280221);
    p = fma(p, s, -0.06664511447381948);
    p = fma(p, s, 0.07692183190826087);
    p = fma(p, s, -0.09090904578123903);
    p = fma(p, s, 0.11111111015256361);
    p = fma(p, s, -0.14285714284666542);
    p = fma(p, s, 0.1999999999999552);
    p = fma(p, s, -0.3333333333333333);
    double r = fma(t * s, p, t);                       // atan(t)
    r = big ? r + 0.78539816339744831 : r;            // atan(q)
    r = swap ? 1.5707963267948966 - r : r;            // first quadrant
    r = (x < 0.0) ? 3.1415926535897931 - r : r;       // upper half plane
    return copysign(r, y);
}

// log|A|^2 of the node evaluation's Log A: log(v), written for this use
// (2.4 % off the Bates batch against CUDA's log).  Method (the atanh form of
// the logarithm of Cody and Waite's manual): v = 2^k m with m in
// [sqrt(1/2), sqrt 2), read off the IEEE exponent and mantissa bits;
// log v = k ln 2 + 2 atanh(s), s = (m - 1)/(m + 1) (m - 1 is exact, the
// quotient uses rcp_nr), 2 atanh(s) = 2 s + s w R(w), w = s^2, with the
// degree-6 Chebyshev interpolant R of node_math_coeffs.py (4.5e-18 relative),
// and k ln 2 added through two FMAs with ln 2 split into a double and its
// remainder.  At most 2 ulp from CUDA's log (ope_selftest_log).  Arguments
// outside the normal range (0, subnormal, infinite, NaN) take CUDA's log.
__device__ __forceinline__ double log_node(double v) {
    const int hi = __double2hiint(v), lo = __double2loint(v);
    const int k = (hi - 0x3FE6A09E) >> 20;  // 0x3FE6A09E: high word of sqrt(1/2)
    const double m = __hiloint2double(hi - k * 0x100000, lo);
    const double f = m - 1.0;
    const double s = f * rcp_nr(2.0 + f);
    const double w = s * s;
    double r = 0.14616449685043406;
    r = fma(r, w, 0.15331721600556042);
    r = fma(r, w, 0.18182889125261723);
    r = fma(r, w, 0.2222221113479508);
    r = fma(r, w, 0.28571428625975487);
    r = fma(r, w, 0.39999999999899505);
    r = fma(r, w, 0.666666666666667);
    const double lm = fma(s * w, r, 2.0 * s);  // log m
    const double kd = (double)k;
    double out = fma(kd, 0.6931471805599453, fma(kd, 2.3190468138462996e-17, lm));
    if (!(v >= 0x1p-1022 && v <= 0x1.fffffffffffffp+1023)) out = log(v);
    return out;
}

// Error-free transformations (Knuth's TwoSum, Dekker's Fast2Sum, the FMA
// product residual) and double-double arithmetic, for log_cr below.
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
    s = __dadd_rn(a, b);
    const double bb = __dsub_rn(s, a);
    e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ void fast_two_sum(double a, double b, double& s, double& e) {  // |a| >= |b|
    s = __dadd_rn(a, b);
    e = __dsub_rn(b, __dsub_rn(s, a));
}
struct DD {
    double hi, lo;
};
__device__ __forceinline__ DD dd_add(DD a, DD b) {
    double s, e;
    two_sum(a.hi, b.hi, s, e);
    e = __dadd_rn(e, __dadd_rn(a.lo, b.lo));
    DD r;
    fast_two_sum(s, e, r.hi, r.lo);
    return r;
}
__device__ __forceinline__ DD dd_mul(DD a, DD b) {
    const double p = __dmul_rn(a.hi, b.hi);
    double e = fma(a.hi, b.hi, -p);
    e = fma(a.hi, b.lo, fma(a.lo, b.hi, e));
    DD r;
    fast_two_sum(p, e, r.hi, r.lo);
    return r;
}

// ln(v) correctly rounded (to nearest) for positive normal v, other arguments
// through CUDA's log.  Used once per integral for x = ln(S/K): the integrand's
// phase u x reaches 1e7 and beyond on short-dated deep-wing contracts, where
// one ulp of x moves a node value by 1e-9 relative, so x must be the value
// the reference's own libm log returns -- the correctly rounded one.  Method
// (the atanh series of the logarithm, in double-double): v = 2^k m with m in
// [sqrt(1/2), sqrt 2); s = (m - 1)/(m + 1) as a double-double;
// ln m = 2s + 2s^3/3 + 2s^5/5 + s^7 q(s^2), q(w) = sum_j 2 w^j/(2j + 7)
// (|s| <= 0.1716, the first three terms in double-double, q in double); plus
// k ln 2 with ln 2 as a double-double.  The sum carries about 2^-68 relative
// error, so the final rounding is correct unless ln v lies within that of a
// rounding midpoint.
__device__ __forceinline__ double log_cr(double v) {
    if (!(v >= 0x1p-1022 && v <= 0x1.fffffffffffffp+1023)) return log(v);
    const int hi = __double2hiint(v), lo = __double2loint(v);
    const int k = (hi - 0x3FE6A09E) >> 20;  // 0x3FE6A09E: high word of sqrt(1/2)
    const double m = __hiloint2double(hi - k * 0x100000, lo);
    const double f = __dsub_rn(m, 1.0);  // exact (Sterbenz)
    double dh, dl;
    fast_two_sum(2.0, f, dh, dl);  // m + 1 = 2 + f exactly
    const double sh = __ddiv_rn(f, dh);
    const double res = __dsub_rn(fma(-sh, dh, f), __dmul_rn(sh, dl));  // f - sh (dh + dl)
    DD S;
    fast_two_sum(sh, __ddiv_rn(res, dh), S.hi, S.lo);
    const DD W = dd_mul(S, S);
    const DD S3 = dd_mul(S, W);
    const DD S5 = dd_mul(S3, W);
    const double w = W.hi;
    double q = 0.07407407407407407;
    q = fma(q, w, 0.08);
    q = fma(q, w, 0.08695652173913043);
    q = fma(q, w, 0.09523809523809523);
    q = fma(q, w, 0.10526315789473684);
    q = fma(q, w, 0.11764705882352941);
    q = fma(q, w, 0.13333333333333333);
    q = fma(q, w, 0.15384615384615385);
    q = fma(q, w, 0.18181818181818182);
    q = fma(q, w, 0.2222222222222222);
    q = fma(q, w, 0.2857142857142857);
    const double rest = __dmul_rn(__dmul_rn(S5.hi, w), q);
    DD acc{__dmul_rn(2.0, S.hi), __dmul_rn(2.0, S.lo)};
    acc = dd_add(acc, dd_mul(S3, DD{0.6666666666666666, 3.700743415417188e-17}));  // 2/3
    acc = dd_add(acc, dd_mul(S5, DD{0.4, -2.2204460492503132e-17}));               // 2/5
    acc = dd_add(acc, DD{rest, 0.0});
    const double kd = (double)k;
    DD kl;
    kl.hi = __dmul_rn(kd, 0.6931471805599453);  // ln 2 = 0.6931471805599453 + 2.3190468138462996e-17
    kl.lo = fma(kd, 2.3190468138462996e-17, fma(kd, 0.6931471805599453, -kl.hi));
    acc = dd_add(kl, acc);
    return __dadd_rn(acc.hi, acc.lo);
}

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

// d = fast_csqrt(z) of the node evaluations (heston.rs:155-175), branch-free
// and without hypot, a division or an IEEE square root: |z| and
// w = sqrt((|zr| + |z|)/2) through refined reciprocal square roots, the other
// component zi / (2 w).  z = 0 gives d = 0 as the reference's b == 0 branch
// does.
__device__ __forceinline__ void csqrt_node(double zr, double zi, double& dre, double& dim) {
    const double zz = fma(zr, zr, zi * zi);
    const double r = (zz > 0.0) ? zz * rsqrt_nr(zz) : zz;  // |z| (zz = 0 stays 0)
    const double s2 = 0.5 * (r + fabs(zr));
    const double iw = rsqrt_nr(s2);
    const double w = (s2 > 0.0) ? s2 * iw : 0.0;
    const double q = (s2 > 0.0) ? (0.5 * zi) * iw : zi;
    dre = (zr >= 0.0) ? w : fabs(q);
    dim = (zr >= 0.0) ? q : copysign(w, zi);
}

// Per-integral constants (everything that does not depend on the node),
// folded so that the node evaluation does as little as possible:
//   xi   = (xr, -rs u)                       xi = kappa - i rho sigma phi, phi = u + i phi_im
//   z    = xi^2 + (sig2 u^2, sig2s u)       sigma^2 phi(phi+i)
//   Re Z = kts Re Ch + v0s Re Dh + z0re      z0re = r T + Re(-Log CF(-i)) for P1, 0 for P2
//   Im Z = kts Im Ch + v0s Im Dh + r T u + z0im + (x u mod 2 pi)      x = ln(S/K)
//   Bates: jump = exp(jr0 - hs2 u^2 + i jmu u);  J = (lt Re jump + jre0, lt Im jump - ltc u)
struct CfConsts {
    double xr, rs, sig2, sig2s, kts, v0s, t, z0re, z0im;
    double jr0, hs2, jmu, lt, jre0, ltc;
    // raw values kept for the adjoint chain
    double kappa, phi_im, sgn, rt, x, lnm_re, lnm_im, mu_j, comp;
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
    C.x = log_cr(s / k);  // heston.rs:86, rounded as the platform libm rounds it
    C.phi_im = (which == 0) ? -1.0 : 0.0;
    C.sgn = (which == 0) ? -1.0 : 1.0;
    C.xr = kappa + C.rs * C.phi_im;
    C.sig2s = C.sig2 * C.sgn;
    double lt = 0.0, mu_j = 0.0, hs2 = 0.0, comp = 0.0;
    if (bates) {
        lt = p[5] * t;
        mu_j = p[6];
        hs2 = 0.5 * p[7] * p[7];
        comp = exp(p[6] + (0.5 * p[7]) * p[7]) - 1.0;
    }
    C.lt = lt;
    C.mu_j = mu_j;
    C.hs2 = hs2;
    C.comp = comp;
    C.jr0 = -C.phi_im * mu_j + hs2 * (C.phi_im * C.phi_im);
    C.jmu = mu_j - 2.0 * hs2 * C.phi_im;
    C.jre0 = lt * (C.phi_im * comp - 1.0);
    C.ltc = lt * comp;
    C.lnm_re = 0.0;
    C.lnm_im = 0.0;
    if (which == 0) {
        // CF(-i) = e^{rT} in exact arithmetic (C = D = 0 there, jump factor 1),
        // and the reference's operation sequence reproduces that to the last
        // ulp or so whenever xi(-i) = kappa - rho sigma (C.xr) is a positive
        // normal number and the other terms are moderate: then Log CF(-i) is
        // rT.  Everywhere else -- xi(-i) <= 0, where xi + d = 0 makes the
        // reference's CF(-i) NaN and drops every P1 node, and any extreme or
        // non-finite parameter -- it is evaluated with the reference's own
        // sequence.  (The regular case skips two complex exponentials, three
        // complex divisions and two complex logarithms per P1 integral.)
        bool regular = C.xr > 1e-100 && C.xr < 1e100 && C.sig2 > 1e-100 && C.kts < 1e4 &&
                       C.v0s * C.xr < 1e4 && fabs(C.rt) < 700.0 && t < 1e3;
        if (bates) regular = regular && fabs(p[6] + 0.5 * p[7] * p[7]) < 50.0 && fabs(lt) * (comp + 1.0) < 1e4;
        if (regular) {
            C.lnm_re = -C.rt;
        } else {
            const Cx phi_mi{0.0, -1.0};
            Cx m = stable_cf_ref(phi_mi, t, r, v0, kappa, theta, sigma, rho);
            if (bates) m = cmul(m, jump_cf_ref(phi_mi, t, p[5], p[6], p[7]));
            Cx lm = clog(m);
            C.lnm_re = -lm.re;
            C.lnm_im = -lm.im;
        }
    }
    C.z0re = -C.rt * C.phi_im + C.lnm_re;
    C.z0im = C.lnm_im;
    return C;
}

// u = (1 - t)/t of a node, rounded as heston.rs:223 rounds it (the IEEE
// quotient): at large u the phase u x makes every ulp of u count.  From
// y ~ 1/t (= (1 - t) itt with itt ~ 1/((1 - t) t), a few ulps) the quotient
// u0 = (1 - t) y is within a few ulps; one correction with the exact residual
// (1 - t) - u0 t (an FMA) lands within about 1e-15 ulp of the true quotient,
// so its rounding is the IEEE one short of a midpoint that close (checked
// against IEEE division by ope_selftest_node_u).
__device__ __forceinline__ double node_u(double omt, double tn, double itt) {
    const double yt = omt * itt;
    const double u0 = omt * yt;
    return fma(fma(-u0, tn, omt), yt, u0);
}

// The strike-free part of a node (heston.rs:221-227 with the merged-exponent
// integrand): E = e^{Re Z}, A = Im Z - (u x mod 2 pi), and the node's
// u = (1 - t)/t and itt = 1/((1 - t) t) (node_geom computes the last two
// alone, bit for bit).
struct NodeCf {
    double e, a, u, itt;
};

__device__ __forceinline__ void node_geom(double tn, double& u, double& itt) {
    const double omt = 1.0 - tn;
    itt = rcp_nr(omt * tn);
    u = node_u(omt, tn, itt);
}

// u of a node alone (bit for bit node_geom's).
__device__ __forceinline__ double node_u_of(double tn) {
    double u, itt;
    node_geom(tn, u, itt);
    return u;
}

template <bool BATES>
__device__ __forceinline__ NodeCf node_cf(const CfConsts& C, double tn) {
    double u, itt;  // (1 - t) / t and 1 / ((1 - t) t)
    node_geom(tn, u, itt);
    const double u2 = u * u;
    // xi = (xr, xi_) ; z = xi^2 + sigma^2 phi(phi+i)
    const double xr = C.xr, xi_ = -C.rs * u;
    const double zr = fma(xr, xr, fma(-xi_, xi_, C.sig2 * u2));
    const double zi = fma(2.0 * xr, xi_, C.sig2s * u);
    double dre, dim;
    csqrt_node(zr, zi, dre, dim);
    const double amr = xr - dre, ami = xi_ - dim;  // xi - d
    const double apr = xr + dre, api = xi_ + dim;  // xi + d
    // g = (xi - d) / (xi + d)
    const double ig = rcp_nr(fma(apr, apr, api * api));
    const double gr = fma(amr, apr, ami * api) * ig;
    const double gi = fma(ami, apr, -amr * api) * ig;
    // e = exp(-d T)
    double sn, cs;
    sincos(-dim * C.t, &sn, &cs);
    const double em = exp(-dre * C.t);
    const double er = em * cs, ei = em * sn;
    // g e
    const double ger = fma(gr, er, -gi * ei);
    const double gei = fma(gr, ei, gi * er);
    // A = (g e - 1) / (g - 1)
    const double nr = ger - 1.0, ni = gei;
    const double dr = gr - 1.0, di = gi;
    const double mm = fma(dr, dr, di * di);
    double lr, li, iqc;
    if (BATES) {
        // |A|^2 = |N|^2/|M|^2 and 1/|1 - g e|^2 = 1/|N|^2 from one reciprocal;
        // arg A = arg(N conj(M)) (faster for the Bates instantiation only)
        const double nn = fma(nr, nr, ni * ni);
        const double inv = rcp_nr(nn * mm);
        lr = 0.5 * log_node((nn * nn) * inv);
        li = atan2_node(fma(ni, dr, -nr * di), fma(nr, dr, ni * di));
        iqc = mm * inv;
    } else {
        const double ia = rcp_nr(mm);
        const double ar = fma(nr, dr, ni * di) * ia;
        const double ai = fma(ni, dr, -nr * di) * ia;
        lr = 0.5 * log_node(fma(ar, ar, ai * ai));
        li = atan2_node(ai, ar);
        iqc = 0.0;
    }
    // Dh = (xi - d)(1 - e) / (1 - g e)
    const double omr = 1.0 - er, omi = -ei;
    const double pr = fma(amr, omr, -ami * omi);
    const double pim = fma(amr, omi, ami * omr);
    const double qr = 1.0 - ger, qi = -gei;
    const double iq = BATES ? iqc : rcp_nr(fma(qr, qr, qi * qi));
    const double Dr = fma(pr, qr, pim * qi) * iq;
    const double Di = fma(pim, qr, -pr * qi) * iq;
    // Ch = (xi - d) T - 2 Log A
    const double Cr = fma(amr, C.t, -2.0 * lr);
    const double Ci = fma(ami, C.t, -2.0 * li);
    double zre = fma(C.kts, Cr, fma(C.v0s, Dr, C.z0re));
    double zim = fma(C.kts, Ci, fma(C.v0s, Di, fma(C.rt, u, C.z0im)));
    if (BATES) {
        double js, jc;
        sincos(C.jmu * u, &js, &jc);
        const double je = C.lt * exp(fma(-C.hs2, u2, C.jr0));
        zre += fma(je, jc, C.jre0);
        zim += fma(je, js, -C.ltc * u);
    }
    return NodeCf{exp(zre), zim, u, itt};
}

// One strike's node value from the strike-free part: Im(e^Z) / u / t^2 =
// e^{Re Z} sin(Im Z) / ((1 - t) t) = sin(A + phase) W with W = E itt; 0
// where the reference's g(t) is 0 (t <= 0, u < 1e-12) or the value is not
// finite.  The phase of e^{iux} (heston.rs:107): u x rounded as the
// reference rounds it, reduced modulo 2 pi without loss (Cody and Waite's
// argument reduction, 2 pi split into two doubles and the products taken
// exactly by FMA: |u x - n 2 pi| < 4 makes the first step exact), so that
// adding the CF's own phase costs an ulp of a number below 4 however large
// u x is.  The reference adds the two phases exactly too, through the
// complex product e^{iux} CF (an unreduced sum would lose ulp(u x), 1e-9 at
// u x = 1e7, on short-dated deep-wing contracts).
// LIVE_IN_W: w already carries the liveness (NaN where the node is not live,
// see node_w_live), as the run cache stores it; the value is then 0 exactly
// where the explicit test gives 0.
template <bool LIVE_IN_W = false>
__device__ __forceinline__ double node_finish_w(double x, double tn, double w, double a, double u) {
    const double ux = __dmul_rn(u, x);
    const double nq = rint(ux * 0.15915494309189535);  // 1 / (2 pi)
    const double uxr = fma(-nq, 2.4492935982947064e-16, fma(-nq, 6.283185307179586, ux));
    const double v = __dmul_rn(sin(__dadd_rn(a, uxr)), w);
    const bool ok = (LIVE_IN_W || ((tn > 0.0) && (u >= 1e-12))) && isfinite(v);
    return ok ? v : 0.0;
}

// W with the node's liveness folded in: NaN where the reference's g(t) is 0
// whatever the strike (t <= 0, u < 1e-12).
__device__ __forceinline__ double node_w_live(double tn, const NodeCf& n) {
    return ((tn > 0.0) && (n.u >= 1e-12)) ? __dmul_rn(n.e, n.itt) : __longlong_as_double(0x7ff8000000000000ll);
}

__device__ __forceinline__ double node_w(const NodeCf& n) { return __dmul_rn(n.e, n.itt); }

__device__ __forceinline__ double node_finish(double x, double tn, const NodeCf& n) {
    return node_finish_w(x, tn, node_w(n), n.a, n.u);
}



}  // namespace ope
