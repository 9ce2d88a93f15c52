// TEST INFRASTRUCTURE ONLY — the CPU oracle.
//
// A plain C++ restatement of the reference crate's Heston/Bates pricing path
// (options_pricing_engine 0.1.0, Rust).  It exists to check the CUDA product
// path, and as the timed CPU baseline in bench.py.  Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
// product library never links or calls it.
//
// Every function cites the reference file:line it follows.  Expression trees
// are kept as the Rust source writes them (same association order, no FMA
// contraction: build with -ffp-contract=off) so that, on the same platform
// libm, values agree with the reference to the last bit wherever the Rust
// code calls the same libm routine.  Complex arithmetic restates the
// published algorithms of num-complex 0.4.6 (the crate version the reference
// lock file pins): textbook multiply, conj/|c|^2 division (not Smith's),
// exp = from_polar(e^re, im) with its +-inf/NaN corner cases, and
// ln = (ln hypot(re,im), atan2(im,re)).  The crate source is not vendored in
// the reference tree, so those four are restated from the published algorithm.
//
// Exported with C linkage for ctypes (oracle/oracle.py).

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <vector>
#include <algorithm>
#include <limits>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double PI = 3.14159265358979323846;

// ---------------------------------------------------------------------------
// num-complex 0.4.6 Complex<f64> semantics (heston.rs:13, bates.rs:11)
// ---------------------------------------------------------------------------
struct Cx { double re, im; };

inline Cx cx(double re, double im) { return Cx{re, im}; }
inline Cx operator+(Cx a, Cx b) { return Cx{a.re + b.re, a.im + b.im}; }
inline Cx operator-(Cx a, Cx b) { return Cx{a.re - b.re, a.im - b.im}; }
inline Cx operator-(Cx a) { return Cx{-a.re, -a.im}; }
inline Cx operator*(Cx a, Cx b) {
    return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
inline Cx operator/(Cx a, Cx b) {
    double n = b.re * b.re + b.im * b.im;
    double re = a.re * b.re + a.im * b.im;
    double im = a.im * b.re - a.re * b.im;
    return Cx{re / n, im / n};
}
// mixed real/complex ops (num-complex real_arithmetic macro)
inline Cx operator+(Cx a, double x) { return Cx{a.re + x, a.im}; }
inline Cx operator-(Cx a, double x) { return Cx{a.re - x, a.im}; }
inline Cx operator*(Cx a, double x) { return Cx{a.re * x, a.im * x}; }
inline Cx operator*(double x, Cx a) { return Cx{x * a.re, x * a.im}; }
inline Cx operator-(double x, Cx a) { return Cx{x - a.re, 0.0 - a.im}; }
inline Cx operator+(double x, Cx a) { return Cx{x + a.re, a.im}; }

inline Cx cexp(Cx z) {
    double re = z.re, im = z.im;
    if (std::isinf(re)) {
        if (re < 0.0) {
            if (!std::isfinite(im)) return Cx{0.0, 0.0};
        } else if (im == 0.0 || !std::isfinite(im)) {
            if (std::isinf(im)) im = std::numeric_limits<double>::quiet_NaN();
            return Cx{re, im};
        }
    } else if (std::isnan(re) && im == 0.0) {
        return z;
    }
    double r = std::exp(re);
    return Cx{r * std::cos(im), r * std::sin(im)};
}
inline Cx cln(Cx z) { return Cx{std::log(std::hypot(z.re, z.im)), std::atan2(z.im, z.re)}; }
const Cx I = {0.0, 1.0};

// ---------------------------------------------------------------------------
// heston.rs:29-59 — GK15 nodes/weights in the reference's order, G7 subset.
// ---------------------------------------------------------------------------
const double GK_NODES[15] = {
    0.0,
    0.2077849550078985, -0.2077849550078985,
    0.4058451513773972, -0.4058451513773972,
    0.5860872354676911, -0.5860872354676911,
    0.7415311855993945, -0.7415311855993945,
    0.8648644233597691, -0.8648644233597691,
    0.9491079123427585, -0.9491079123427585,
    0.9914553711208126, -0.9914553711208126,
};
const double GK_WEIGHTS[15] = {
    0.2094821410847278,
    0.2044329400752989, 0.2044329400752989,
    0.1903505780647854, 0.1903505780647854,
    0.1690047266392679, 0.1690047266392679,
    0.1406532597155259, 0.1406532597155259,
    0.1047900103222502, 0.1047900103222502,
    0.0630920926299786, 0.0630920926299786,
    0.0229353220105292, 0.0229353220105292,
};
const int G7_IDX[7] = {0, 3, 4, 7, 8, 11, 12};
const double G7_WEIGHTS[7] = {
    0.4179591836734694,
    0.3818300505051189, 0.3818300505051189,
    0.2797053914892766, 0.2797053914892766,
    0.1294849661688697, 0.1294849661688697,
};
constexpr int MAX_PANELS = 200;  // heston.rs:194
constexpr double REF_TOL = 1e-8; // heston.rs:228

struct Heston { double v0, kappa, theta, sigma, rho; };  // types.rs:48-54
struct Bates { Heston h; double lambda, mu_j, sigma_j; }; // types.rs:66-72

// OptionContract (types.rs:16-25) with the C-ABI layout of include/ope.h.
struct Contract {
    double spot, strike, expiry, rate, div_yield, vol;
    int32_t opt_type;  // 0 = Call, 1 = Put
    int32_t pad;
};
static_assert(sizeof(Contract) == 56, "contract layout");

// heston.rs:155-175
inline Cx fast_csqrt(Cx z) {
    double a = z.re, b = z.im;
    if (b == 0.0) {
        if (a >= 0.0) return Cx{std::sqrt(a), b};
        double m = std::sqrt(-a);
        return Cx{0.0, std::signbit(b) ? -m : m};
    }
    double r = std::hypot(a, b);
    if (a >= 0.0) {
        double re = std::sqrt((r + a) / 2.0);
        double im = b / (2.0 * re);
        return Cx{re, im};
    } else {
        double im = std::copysign(std::sqrt((r - a) / 2.0), b);
        double re = b / (2.0 * im);
        return Cx{re, im};
    }
}

// heston.rs:113-127
inline Cx stable_cf(Cx phi, double t, double r, const Heston& p) {
    const double v0 = p.v0, kappa = p.kappa, theta = p.theta, sigma = p.sigma, rho = p.rho;
    Cx xi = kappa - ((rho * sigma) * phi) * I;
    Cx d = fast_csqrt(xi * xi + ((sigma * sigma) * phi) * (phi + I));
    Cx g = (xi - d) / (xi + d);
    Cx edt = cexp((-d) * t);
    Cx a = (g * edt - 1.0) / (g - 1.0);
    Cx c = ((kappa * theta) / (sigma * sigma)) * ((xi - d) * t - 2.0 * cln(a));
    Cx dd = ((v0 * (xi - d)) * (1.0 - edt)) / ((sigma * sigma) * (1.0 - g * edt));
    return cexp((((r * phi) * I) * t + c) + dd);
}

// bates.rs:77-83
inline Cx jump_cf(Cx phi, double t, const Bates& bp) {
    const double lambda = bp.lambda, mu_j = bp.mu_j, sigma_j = bp.sigma_j;
    double comp = std::exp(mu_j + (0.5 * sigma_j) * sigma_j) - 1.0;
    Cx jump = cexp((phi * I) * mu_j - (((0.5 * phi) * phi) * sigma_j) * sigma_j);
    return cexp((lambda * t) * ((jump - 1.0) - (I * phi) * comp));
}

// heston.rs:180-187.  fv_out (optional): the 15 integrand values, for the
// step trace below.
template <class F>
inline void gk15_panel(const F& f, double a, double b, double* k_out, double* e_out, double* fv_out = nullptr) {
    double c = 0.5 * (a + b);
    double h = 0.5 * (b - a);
    double fv[15];
    for (int i = 0; i < 15; ++i) fv[i] = f(c + h * GK_NODES[i]);
    double k = 0.0;
    for (int i = 0; i < 15; ++i) k = k + GK_WEIGHTS[i] * fv[i];
    double g = 0.0;
    for (int j = 0; j < 7; ++j) g = g + G7_WEIGHTS[j] * fv[G7_IDX[j]];
    *k_out = k * h;
    *e_out = std::fabs(k - g) * h;
    if (fv_out) std::memcpy(fv_out, fv, sizeof(fv));
}

// Step record of adaptive_gk (a diagnostic of the greedy QAG's decisions,
// field for field what the device library's ope_trace_integral records):
// per step j (0 = the first panel [0, 1], j >= 1 = the j-th bisection)
// TRACE_FIELDS doubles: the bisected panel a, b and its error estimate
// (0, 1, 0 at j = 0), the children's K and error estimates kl, el, kr, er
// (j = 0: the first panel's K, err, 0, 0), the running error and total after
// the step, then the 15 integrand values of the left child and the 15 of the
// right child (j = 0: the first panel's 15, then zeros).
constexpr int TRACE_FIELDS = 39;
struct QagTrace {
    double* out;
    int max_steps;
    int steps = 0;
    void record(int j, double a, double b, double ew, double kl, double el, double kr, double er, double err,
                double total, const double* fl, const double* fr) {
        steps = j + 1;
        if (j >= max_steps) return;
        double* r = out + (size_t)j * TRACE_FIELDS;
        const double head[9] = {a, b, ew, kl, el, kr, er, err, total};
        std::memcpy(r, head, sizeof(head));
        for (int i = 0; i < 15; ++i) {
            r[9 + i] = fl[i];
            r[24 + i] = fr ? fr[i] : 0.0;
        }
    }
};

// f64::total_cmp key (Rust core::f64::total_cmp)
inline int64_t total_key(double x) {
    int64_t i;
    std::memcpy(&i, &x, 8);
    i ^= (int64_t)(((uint64_t)(i >> 63)) >> 1);
    return i;
}

struct Panel { double err, k, a, b; };

// heston.rs:193-212.  `bisections` (optional) counts loop iterations.
template <class F>
inline double adaptive_gk(const F& f, double a, double b, double tol, int* bisections, QagTrace* tr = nullptr) {
    double k0, e0;
    double fl[15], fr[15];
    gk15_panel(f, a, b, &k0, &e0, tr ? fl : nullptr);
    Panel panels[MAX_PANELS + 1];
    int len = 0;
    panels[len++] = Panel{e0, k0, a, b};
    double total = k0;
    double err = e0;
    int nb = 0;
    if (tr) tr->record(0, a, b, 0.0, k0, e0, 0.0, 0.0, err, total, fl, nullptr);
    while (err > tol && len < MAX_PANELS) {
        // (0..len).max_by(total_cmp): the LAST maximum wins ties
        int w = 0;
        int64_t best = total_key(panels[0].err);
        for (int i = 1; i < len; ++i) {
            int64_t ki = total_key(panels[i].err);
            if (ki >= best) { best = ki; w = i; }
        }
        Panel pw = panels[w];
        panels[w] = panels[len - 1];  // swap_remove
        --len;
        double m = 0.5 * (pw.a + pw.b);
        double kl, el, kr, er;
        gk15_panel(f, pw.a, m, &kl, &el, tr ? fl : nullptr);
        gk15_panel(f, m, pw.b, &kr, &er, tr ? fr : nullptr);
        total += (kl + kr) - pw.k;
        err += (el + er) - pw.err;
        panels[len++] = Panel{el, kl, pw.a, m};
        panels[len++] = Panel{er, kr, m, pw.b};
        ++nb;
        if (tr) tr->record(nb, pw.a, pw.b, pw.err, kl, el, kr, er, err, total, fl, fr);
    }
    if (bisections) *bisections = nb;
    return total;
}

// heston.rs:220-229 (tol made a parameter; the reference hard-codes 1e-8)
template <class F>
inline double gk_integrate(const F& f, double tol, int* bisections, QagTrace* tr = nullptr) {
    auto g = [&](double t) -> double {
        if (t <= 0.0) return 0.0;
        double u = (1.0 - t) / t;
        if (u < 1e-12) return 0.0;
        double v = f(u) / (t * t);
        return std::isfinite(v) ? v : 0.0;
    };
    return adaptive_gk(g, 0.0, 1.0, tol, bisections, tr);
}

// heston.rs:101-109
inline double cf_integrand(double u, double x, double t, double r, const Heston& p, bool is_p1,
                           const Cx* cf_mi) {
    Cx phi = is_p1 ? Cx{u, -1.0} : Cx{u, 0.0};
    Cx cf = stable_cf(phi, t, r, p);
    if (cf_mi) cf = cf / *cf_mi;
    Cx num = cexp(Cx{0.0, u * x}) * cf;
    return (num / Cx{0.0, u}).re;
}

// bates.rs:65-73
inline double bates_integrand(double u, double x, double t, double r, const Bates& bp, bool is_p1,
                              const Cx* cf_mi) {
    Cx phi = is_p1 ? Cx{u, -1.0} : Cx{u, 0.0};
    Cx cf = stable_cf(phi, t, r, bp.h) * jump_cf(phi, t, bp);
    if (cf_mi) cf = cf / *cf_mi;
    Cx num = cexp(Cx{0.0, u * x}) * cf;
    return (num / Cx{0.0, u}).re;
}

// heston.rs:82-99
inline double heston_call(double s, double k, double t, double r, double q, const Heston& p,
                          double tol, int* nb) {
    double x = std::log(s / k);
    Cx cf_mi = stable_cf(Cx{0.0, -1.0}, t, r, p);
    double i1 = gk_integrate([&](double u) { return cf_integrand(u, x, t, r, p, true, &cf_mi); },
                             tol, nb ? nb : nullptr);
    double i2 = gk_integrate([&](double u) { return cf_integrand(u, x, t, r, p, false, nullptr); },
                             tol, nb ? nb + 1 : nullptr);
    double p1 = 0.5 + i1 / PI;
    double p2 = 0.5 + i2 / PI;
    return std::fmax((s * std::exp(-q * t)) * p1 - (k * std::exp(-r * t)) * p2, 0.0);
}

// bates.rs:49-63
inline double bates_call(double s, double k, double t, double r, double q, const Bates& bp,
                         double tol, int* nb) {
    double x = std::log(s / k);
    Cx phi_mi{0.0, -1.0};
    Cx cf_mi = stable_cf(phi_mi, t, r, bp.h) * jump_cf(phi_mi, t, bp);
    double i1 = gk_integrate([&](double u) { return bates_integrand(u, x, t, r, bp, true, &cf_mi); },
                             tol, nb ? nb : nullptr);
    double i2 = gk_integrate([&](double u) { return bates_integrand(u, x, t, r, bp, false, nullptr); },
                             tol, nb ? nb + 1 : nullptr);
    double p1 = 0.5 + i1 / PI;
    double p2 = 0.5 + i2 / PI;
    return std::fmax((s * std::exp(-q * t)) * p1 - (k * std::exp(-r * t)) * p2, 0.0);
}

// heston.rs:61-72
inline double heston_price(double spot, double strike, double expiry, double rate, double div_yield,
                           const Heston& p, int opt_type, double tol, int* nb) {
    double call = heston_call(spot, strike, expiry, rate, div_yield, p, tol, nb);
    if (opt_type == 0) return call;
    return (call - spot * std::exp(-div_yield * expiry)) + strike * std::exp(-rate * expiry);
}

// bates.rs:29-39
inline double bates_price(double spot, double strike, double expiry, double rate, double div_yield,
                          const Bates& p, int opt_type, double tol, int* nb) {
    double call = bates_call(spot, strike, expiry, rate, div_yield, p, tol, nb);
    if (opt_type == 0) return call;
    return (call - spot * std::exp(-div_yield * expiry)) + strike * std::exp(-rate * expiry);
}

// ---------------------------------------------------------------------------
// math.rs / bsm.rs / iv.rs (needed by the IV-space residuals of calibration)
// ---------------------------------------------------------------------------
constexpr double SQRT_2PI_INV = 0.3989422804014327;  // math.rs:8
constexpr double SQRT_2_INV = 0.70710678118654752440;  // math.rs:9 (FRAC_1_SQRT_2)

inline double npdf(double x) { return SQRT_2PI_INV * std::exp((-0.5 * x) * x); }  // math.rs:10-12
inline double ncdf(double x) { return 0.5 * std::erfc(-x * SQRT_2_INV); }          // math.rs:17-19

// math.rs:24-51 (Acklam)
double ncdf_inv(double p) {
    const double A1 = -3.969683028665376e1, A2 = 2.209460984245205e2, A3 = -2.759285104469687e2,
                 A4 = 1.38357751867269e2, A5 = -3.066479806614716e1, A6 = 2.506628277459239;
    const double B1 = -5.447609879822406e1, B2 = 1.615858368580409e2, B3 = -1.556989798598866e2,
                 B4 = 6.680131188771972e1, B5 = -1.328068155288572e1;
    const double C1 = -7.784894002430293e-3, C2 = -3.223964580411365e-1, C3 = -2.400758277161838,
                 C4 = -2.549732539343734, C5 = 4.374664141464968, C6 = 2.938163982698783;
    const double D1 = 7.784695709041462e-3, D2 = 3.224671290700398e-1, D3 = 2.445134137142996,
                 D4 = 3.754408661907416;
    const double P_LO = 0.02425;
    if (p >= P_LO && p <= 1.0 - P_LO) {
        double q = p - 0.5;
        double r = q * q;
        return q * (((((A1 * r + A2) * r + A3) * r + A4) * r + A5) * r + A6) /
               (1.0 + ((((B1 * r + B2) * r + B3) * r + B4) * r + B5) * r);
    }
    double r = p < P_LO ? std::sqrt(-2.0 * std::log(p)) : std::sqrt(-2.0 * std::log(1.0 - p));
    double x = (((((C1 * r + C2) * r + C3) * r + C4) * r + C5) * r + C6) /
               ((((D1 * r + D2) * r + D3) * r + D4) * r + 1.0);
    return p < P_LO ? x : -x;
}

inline double sign_of(int opt_type) { return opt_type == 0 ? 1.0 : -1.0; }  // types.rs:9-12

// bsm.rs:8-12
inline void d_terms(double s, double k, double t, double r, double q, double v, double* d1, double* d2) {
    double vt = v * std::sqrt(t);
    double dd1 = (std::log(s / k) + ((r - q) + (0.5 * v) * v) * t) / vt;
    *d1 = dd1;
    *d2 = dd1 - vt;
}

// bsm.rs:55-60
inline double bsm_price(const Contract& c) {
    double d1, d2;
    d_terms(c.spot, c.strike, c.expiry, c.rate, c.div_yield, c.vol, &d1, &d2);
    double phi = sign_of(c.opt_type);
    return phi * ((c.spot * std::exp(-c.div_yield * c.expiry)) * ncdf(phi * d1) -
                  (c.strike * std::exp(-c.rate * c.expiry)) * ncdf(phi * d2));
}

struct Result8 { double price, delta, gamma, vega, theta, rho, vanna, volga; };  // types.rs:29-39

// bsm.rs:15-52
inline Result8 bsm_price_and_greeks(const Contract& c) {
    double s = c.spot, k = c.strike, t = c.expiry, r = c.rate, q = c.div_yield, v = c.vol;
    double d1, d2;
    d_terms(s, k, t, r, q, v, &d1, &d2);
    double phi = sign_of(c.opt_type);
    double nd1 = ncdf(phi * d1), nd2 = ncdf(phi * d2), npd1 = npdf(d1);
    double eq = std::exp(-q * t), er = std::exp(-r * t);
    double seq = s * eq, ker = k * er, sqt = std::sqrt(t);
    Result8 o;
    o.price = phi * (seq * nd1 - ker * nd2);
    o.delta = (phi * eq) * nd1;
    o.gamma = (eq * npd1) / ((s * v) * sqt);
    o.vega = (seq * npd1) * sqt;
    double vsqt = v * sqt;
    o.theta = ((-seq) * npd1) * vsqt / (2.0 * t) - phi * ((q * seq) * nd1 - (r * ker) * nd2);
    o.rho = (((phi * k) * t) * er) * nd2;
    o.vanna = (((-eq) * npd1) * d2) / v;
    o.volga = ((o.vega * d1) * d2) / v;
    return o;
}

// iv.rs:85-95
inline void vega_and_volga(const Contract& c, double v, double* vega, double* volga) {
    double vt = v * std::sqrt(c.expiry);
    double d1 = (std::log(c.spot / c.strike) + ((c.rate - c.div_yield) + (0.5 * v) * v) * c.expiry) / vt;
    double d2 = d1 - vt;
    double eq = std::exp(-c.div_yield * c.expiry);
    double npd1 = npdf(d1);
    double sqt = std::sqrt(c.expiry);
    double vg = ((c.spot * eq) * npd1) * sqt;
    *vega = vg;
    *volga = ((vg * d1) * d2) / v;
}

inline Contract with_vol(const Contract& c, double v) { Contract o = c; o.vol = v; return o; }

// iv.rs:22-31
inline bool price_in_bounds(const Contract& c, double price) {
    if (price <= 0.0) return false;
    double er = std::exp(-c.rate * c.expiry);
    double eq = std::exp(-c.div_yield * c.expiry);
    double intrinsic = c.opt_type == 0 ? std::fmax(c.spot * eq - c.strike * er, 0.0)
                                       : std::fmax(c.strike * er - c.spot * eq, 0.0);
    return price >= intrinsic;
}

// iv.rs:52-63
inline bool bisect(const Contract& c, double target, double* out) {
    double lo = 1e-4, hi = 10.0;
    auto f = [&](double v) { return bsm_price(with_vol(c, v)) - target; };
    if (f(lo) * f(hi) > 0.0) return false;
    for (int i = 0; i < 60; ++i) {
        double mid = 0.5 * (lo + hi);
        if (f(mid) < 0.0) lo = mid; else hi = mid;
        if (hi - lo < 1e-9) { *out = mid; return true; }
    }
    *out = 0.5 * (lo + hi);
    return true;
}

// iv.rs:36-49
inline bool initial_guess(const Contract& c, double price, double* out) {
    double er = std::exp(-c.rate * c.expiry);
    double eq = std::exp(-c.div_yield * c.expiry);
    double fwd = (c.spot * eq) / er;
    double bs = (price * std::sqrt((2.0 * PI) / c.expiry)) / (fwd * er);
    double x = std::log(fwd / c.strike);
    double v0 = bs / std::fmax(std::exp((-0.5 * x) * x), 0.01);
    v0 = std::min(std::max(v0, 0.001), 10.0);  // f64::clamp
    if (std::fabs(bsm_price(with_vol(c, v0)) - price) < 0.2 * price) { *out = v0; return true; }
    return bisect(c, price, out);
}

// iv.rs:65-83
inline bool halley_solve(const Contract& c, double target, double v0, double* out) {
    const int MAX_ITER = 10;
    const double TOL = 1e-10;
    double v = v0;
    for (int it = 0; it < MAX_ITER; ++it) {
        double err = bsm_price(with_vol(c, v)) - target;
        if (std::fabs(err) < TOL) { *out = v; return true; }
        double vega, volga;
        vega_and_volga(c, v, &vega, &volga);
        if (std::fabs(vega) < 1e-14) return false;
        double denom = 1.0 - (err * volga) / ((2.0 * vega) * vega);
        denom = std::min(std::max(denom, 0.5), 2.0);
        v -= err / (vega * denom);
        if (v <= 0.0) v = 1e-8;
    }
    if (std::fabs(bsm_price(with_vol(c, v)) - target) < 1e-6) { *out = v; return true; }
    return false;
}

// iv.rs:14-20
inline bool implied_vol(const Contract& c, double mkt, double* out) {
    if (!price_in_bounds(c, mkt)) return false;
    double v0;
    if (!initial_guess(c, mkt, &v0)) return false;
    return halley_solve(c, mkt, v0, out);
}

// ---------------------------------------------------------------------------
// greeks.rs:19-72 — bump-and-reprice through a generic pricer.
// ---------------------------------------------------------------------------
template <class P, class PriceFn, class WithV0>
Result8 bump_and_reprice(double spot, double strike, double expiry, double rate, double div_yield,
                         const P& params, double v0, int opt_type, const PriceFn& price_fn,
                         const WithV0& with_v0) {
    auto px = [&](const P& pp, double s, double t, double r) {
        return price_fn(s, strike, t, r, div_yield, pp, opt_type);
    };
    double price = px(params, spot, expiry, rate);
    double ds = 0.01 * spot, dv = 0.01, dr = 1e-4, dt = 1.0 / 365.0;
    double pu = px(params, spot + ds, expiry, rate);
    double pd = px(params, spot - ds, expiry, rate);
    double delta = (pu - pd) / (2.0 * ds);
    double gamma = ((pu - 2.0 * price) + pd) / (ds * ds);
    double v_cur = std::sqrt(v0);
    double vu = v_cur + dv;
    double vd = std::fmax(v_cur - dv, 1e-8);
    P p_vup = with_v0(params, vu * vu);
    P p_vdn = with_v0(params, vd * vd);
    double vega = (px(p_vup, spot, expiry, rate) - px(p_vdn, spot, expiry, rate)) / (2.0 * dv);
    double t_dn = std::fmax(expiry - dt, 1e-6);
    double theta = (px(params, spot, t_dn, rate) - price) / dt;
    double rho = (px(params, spot, expiry, rate + dr) - px(params, spot, expiry, rate - dr)) / (2.0 * dr);
    double delta_vup = (px(p_vup, spot + ds, expiry, rate) - px(p_vup, spot - ds, expiry, rate)) / (2.0 * ds);
    double delta_vdn = (px(p_vdn, spot + ds, expiry, rate) - px(p_vdn, spot - ds, expiry, rate)) / (2.0 * ds);
    double vanna = (delta_vup - delta_vdn) / (2.0 * dv);
    double vu2 = v_cur + 2.0 * dv;
    double vd2 = std::fmax(v_cur - 2.0 * dv, 1e-8);
    P p_vup2 = with_v0(params, vu2 * vu2);
    P p_vdn2 = with_v0(params, vd2 * vd2);
    double vega_up = (px(p_vup2, spot, expiry, rate) - price) / (2.0 * dv);
    double vega_dn = (price - px(p_vdn2, spot, expiry, rate)) / (2.0 * dv);
    double volga = (vega_up - vega_dn) / (2.0 * dv);
    return Result8{price, delta, gamma, vega, theta, rho, vanna, volga};
}

// ---------------------------------------------------------------------------
// ad.rs — forward-mode AD (scalar Dual), the oracle for the adjoint kernel.
// ---------------------------------------------------------------------------
struct Dual { double val, dot; };  // ad.rs:29-33
inline Dual dc(double v) { return Dual{v, 0.0}; }
inline Dual da(double v) { return Dual{v, 1.0}; }
inline Dual operator+(Dual a, Dual b) { return Dual{a.val + b.val, a.dot + b.dot}; }  // ad.rs:57
inline Dual operator-(Dual a, Dual b) { return Dual{a.val - b.val, a.dot - b.dot}; }  // ad.rs:58
inline Dual operator-(Dual a) { return Dual{-a.val, -a.dot}; }                         // ad.rs:59
inline Dual operator*(Dual a, Dual b) { return Dual{a.val * b.val, a.val * b.dot + a.dot * b.val}; }  // ad.rs:62
inline Dual operator/(Dual a, Dual b) {  // ad.rs:63-65
    return Dual{a.val / b.val, (a.dot * b.val - a.val * b.dot) / (b.val * b.val)};
}
inline Dual dexp(Dual a) { double e = std::exp(a.val); return Dual{e, e * a.dot}; }  // ad.rs:39-43
inline Dual dsqrt(Dual a) { double s = std::sqrt(a.val); return Dual{s, a.dot / (2.0 * s)}; }  // ad.rs:50-54

struct CD { Dual re, im; };  // Complex<Dual> with num-complex generic ops
inline CD operator+(CD a, CD b) { return CD{a.re + b.re, a.im + b.im}; }
inline CD operator-(CD a, CD b) { return CD{a.re - b.re, a.im - b.im}; }
inline CD operator*(CD a, CD b) { return CD{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline CD operator/(CD a, CD b) {
    Dual n = b.re * b.re + b.im * b.im;
    Dual re = a.re * b.re + a.im * b.im;
    Dual im = a.im * b.re - a.re * b.im;
    return CD{re / n, im / n};
}
inline CD cd(double re, double im) { return CD{dc(re), dc(im)}; }  // ad.rs:95-97
inline CD cd_i() { return cd(0.0, 1.0); }                          // ad.rs:100

// ad.rs:104-120
inline CD cexp_d(CD z) {
    double ea = std::exp(z.re.val);
    double cs = std::cos(z.im.val);
    double sn = std::sin(z.im.val);
    double re_val = ea * cs;
    double im_val = ea * sn;
    double re_dot = ea * (z.re.dot * cs - z.im.dot * sn);
    double im_dot = ea * (z.re.dot * sn + z.im.dot * cs);
    return CD{Dual{re_val, re_dot}, Dual{im_val, im_dot}};
}

// ad.rs:131-153
inline CD csqrt_d(CD z) {
    Dual a = z.re, b = z.im;
    if (b.val == 0.0) {
        if (a.val >= 0.0) return CD{dsqrt(a), b};
        Dual m = dsqrt(-a);
        return CD{dc(0.0), std::signbit(b.val) ? -m : m};
    }
    Dual r = dsqrt(a * a + b * b);
    if (a.val >= 0.0) {
        Dual re = dsqrt((r + a) * dc(0.5));
        Dual im = b / (re * dc(2.0));
        return CD{re, im};
    } else {
        Dual mag = dsqrt((r - a) * dc(0.5));
        Dual im = std::signbit(b.val) ? -mag : mag;
        Dual re = b / (im * dc(2.0));
        return CD{re, im};
    }
}

// ad.rs:156-171
inline CD cln_d(CD z) {
    double a = z.re.val, b = z.im.val, dA = z.re.dot, dB = z.im.dot;
    double r2 = a * a + b * b;
    double r = std::sqrt(r2);
    double ln_val = std::log(r);
    double arg_val = std::atan2(b, a);
    double ln_dot = (a * dA + b * dB) / r2;
    double arg_dot = (a * dB - b * dA) / r2;
    return CD{Dual{ln_val, ln_dot}, Dual{arg_val, arg_dot}};
}

struct DualParams { Dual v0, kappa, theta, sigma, rho; };  // ad.rs:585-591

// ad.rs:593-602
inline DualParams dual_params(const Heston& p, int active) {
    auto d = [&](double v, int i) { return i == active ? da(v) : dc(v); };
    return DualParams{d(p.v0, 0), d(p.kappa, 1), d(p.theta, 2), d(p.sigma, 3), d(p.rho, 4)};
}

// ad.rs:178-195
inline CD stable_cf_dual(CD phi, double t, double r, const DualParams& p) {
    CD i = cd_i();
    auto c = [](double v) { return CD{dc(v), dc(0.0)}; };
    auto cp = [](Dual d) { return CD{d, dc(0.0)}; };
    CD xi = cp(p.kappa) - (cp(p.rho * p.sigma) * phi) * i;
    CD d = csqrt_d(xi * xi + (cp(p.sigma * p.sigma) * phi) * (phi + i));
    CD g = (xi - d) / (xi + d);
    CD edt = cexp_d(d * c(-t));
    CD one = c(1.0);
    CD a = cln_d((g * edt - one) / (g - one));
    CD cc = cp((p.kappa * p.theta) / (p.sigma * p.sigma)) * ((xi - d) * c(t) - a * c(2.0));
    CD dd = ((cp(p.v0) * (xi - d)) * (one - edt)) / (cp(p.sigma * p.sigma) * (one - g * edt));
    return cexp_d(((c(r * t) * phi) * i + cc) + dd);
}

// ad.rs:211-216
struct JumpSpec { int mode; double lambda, mu_j, sigma_j; int active; };  // mode 0 Off, 1 Const, 2 Active

// ad.rs:218-234
inline CD jump_factor(CD phi, double t, const JumpSpec& spec) {
    if (spec.mode == 0) return cd(1.0, 0.0);
    int active = spec.mode == 2 ? spec.active : -1;
    CD i = cd_i();
    Dual dl = active == 0 ? da(spec.lambda) : dc(spec.lambda);
    Dual dmj = active == 1 ? da(spec.mu_j) : dc(spec.mu_j);
    Dual dsj = active == 2 ? da(spec.sigma_j) : dc(spec.sigma_j);
    auto c0 = [](Dual d) { return CD{d, dc(0.0)}; };
    Dual half_sj2 = (dsj * dsj) * dc(0.5);
    Dual comp = dexp(dmj + half_sj2) - dc(1.0);
    CD jump = cexp_d((phi * i) * c0(dmj) - (c0(half_sj2) * phi) * phi);
    return cexp_d((c0(dl) * c0(dc(t))) * ((jump - c0(dc(1.0))) - (i * phi) * c0(comp)));
}

// ad.rs:609-630
inline void dual_integrand(double u, double x, double t, double r, const DualParams& dp, bool is_p1,
                           const CD* cf_mi, const JumpSpec& jump, double* val, double* dot) {
    CD phi = is_p1 ? CD{dc(u), dc(-1.0)} : CD{dc(u), dc(0.0)};
    CD cf = stable_cf_dual(phi, t, r, dp);
    cf = cf * jump_factor(phi, t, jump);
    if (cf_mi) cf = cf / *cf_mi;
    CD exp_term = cexp_d(CD{dc(0.0), dc(u * x)});
    CD num = exp_term * cf;
    CD dv = CD{dc(0.0), dc(u)};
    CD res = num / dv;
    *val = res.re.val;
    *dot = res.re.dot;
}

// ad.rs:639-647
template <class F>
inline void gk15_panel_dual(const F& f, double a, double b, double* kv, double* kd, double* e) {
    double c = 0.5 * (a + b);
    double h = 0.5 * (b - a);
    double fv[15], fd[15];
    for (int i = 0; i < 15; ++i) f(c + h * GK_NODES[i], &fv[i], &fd[i]);
    double k_val = 0.0, k_dot = 0.0, g_val = 0.0;
    for (int i = 0; i < 15; ++i) k_val = k_val + GK_WEIGHTS[i] * fv[i];
    for (int i = 0; i < 15; ++i) k_dot = k_dot + GK_WEIGHTS[i] * fd[i];
    for (int j = 0; j < 7; ++j) g_val = g_val + G7_WEIGHTS[j] * fv[G7_IDX[j]];
    *kv = k_val * h;
    *kd = k_dot * h;
    *e = std::fabs(k_val - g_val) * h;
}

struct PanelD { double err, val, dot, a, b; };

// ad.rs:649-670
template <class F>
inline void adaptive_gk_dual(const F& f, double a, double b, double tol, double* tv, double* td) {
    double v0, d0, e0;
    gk15_panel_dual(f, a, b, &v0, &d0, &e0);
    PanelD panels[MAX_PANELS + 1];
    int len = 0;
    panels[len++] = PanelD{e0, v0, d0, a, b};
    double total_val = v0, total_dot = d0, err = e0;
    while (err > tol && len < MAX_PANELS) {
        int w = 0;
        int64_t best = total_key(panels[0].err);
        for (int i = 1; i < len; ++i) {
            int64_t ki = total_key(panels[i].err);
            if (ki >= best) { best = ki; w = i; }
        }
        PanelD pw = panels[w];
        panels[w] = panels[len - 1];
        --len;
        double m = 0.5 * (pw.a + pw.b);
        double vl, dl, el, vr, dr, er;
        gk15_panel_dual(f, pw.a, m, &vl, &dl, &el);
        gk15_panel_dual(f, m, pw.b, &vr, &dr, &er);
        total_val += (vl + vr) - pw.val;
        total_dot += (dl + dr) - pw.dot;
        err += (el + er) - pw.err;
        panels[len++] = PanelD{el, vl, dl, pw.a, m};
        panels[len++] = PanelD{er, vr, dr, m, pw.b};
    }
    *tv = total_val;
    *td = total_dot;
}

// ad.rs:673-684
template <class F>
inline void gk_integrate_dual(const F& f, double tol, double* tv, double* td) {
    auto g = [&](double t, double* v, double* d) {
        if (t <= 0.0) { *v = 0.0; *d = 0.0; return; }
        double u = (1.0 - t) / t;
        if (u < 1e-12) { *v = 0.0; *d = 0.0; return; }
        double vv, ddv;
        f(u, &vv, &ddv);
        double jac = t * t;
        vv = vv / jac;
        ddv = ddv / jac;
        if (std::isfinite(vv) && std::isfinite(ddv)) { *v = vv; *d = ddv; }
        else { *v = 0.0; *d = 0.0; }
    };
    adaptive_gk_dual(g, 0.0, 1.0, tol, tv, td);
}

// ad.rs:695-731
inline void forward_pass(double s, double k, double t, double r, double q, const Heston& p,
                         int opt_type, int active, const JumpSpec& jump, double tol,
                         double* price, double* dprice) {
    double x = std::log(s / k);
    DualParams dp = dual_params(p, active);
    CD phi_mi = CD{dc(0.0), dc(-1.0)};
    CD cf_mi = stable_cf_dual(phi_mi, t, r, dp) * jump_factor(phi_mi, t, jump);
    double i1v, i1d, i2v, i2d;
    gk_integrate_dual([&](double u, double* v, double* d) {
        dual_integrand(u, x, t, r, dp, true, &cf_mi, jump, v, d);
    }, tol, &i1v, &i1d);
    gk_integrate_dual([&](double u, double* v, double* d) {
        dual_integrand(u, x, t, r, dp, false, nullptr, jump, v, d);
    }, tol, &i2v, &i2d);
    double p1v = 0.5 + i1v / PI, p2v = 0.5 + i2v / PI;
    double p1d = i1d / PI, p2d = i2d / PI;
    double eq = std::exp(-q * t), er = std::exp(-r * t);
    double seq = s * eq, ker = k * er;
    double call_val = std::fmax(seq * p1v - ker * p2v, 0.0);
    double call_dot = seq * p1d - ker * p2d;
    if (opt_type == 0) { *price = call_val; *dprice = call_dot; }
    else { *price = (call_val - seq) + ker; *dprice = call_dot; }
}

// ---------------------------------------------------------------------------
// calibration.rs — LM in IV space (single start; optional Tikhonov pull).
// ---------------------------------------------------------------------------
struct Quote { Contract c; double iv_market; double weight; };  // calibration.rs:38-42

struct Model {  // CalibModel (calibration.rs:79-199) for Heston (dim 5) and Bates (dim 8)
    int dim;
    double price(const double* v, const Contract& c) const {
        if (dim == 5) {
            Heston h{v[0], v[1], v[2], v[3], v[4]};
            return heston_price(c.spot, c.strike, c.expiry, c.rate, c.div_yield, h, c.opt_type, REF_TOL, nullptr);
        }
        Bates b{{v[0], v[1], v[2], v[3], v[4]}, v[5], v[6], v[7]};
        return bates_price(c.spot, c.strike, c.expiry, c.rate, c.div_yield, b, c.opt_type, REF_TOL, nullptr);
    }
    // calibration.rs:115-122, 158-163
    bool bounds_ok(const double* v) const {
        bool feller = (2.0 * v[1]) * v[2] > v[3] * v[3];  // types.rs:60-62
        bool h = feller && v[0] > 1e-8 && v[0] < 5.0 && v[1] > 1e-6 && v[1] < 50.0 && v[2] > 1e-8 &&
                 v[2] < 5.0 && v[3] > 1e-6 && v[3] < 10.0 && v[4] > -0.9999 && v[4] < 0.9999;
        if (dim == 5) return h;
        return h && v[5] >= 0.0 && v[5] < 10.0 && std::fabs(v[6]) < 2.0 && v[7] > 1e-6 && v[7] < 2.0;
    }
    // calibration.rs:123, 164-168
    double bump(int i) const {
        static const double b[8] = {1e-4, 1e-3, 1e-4, 1e-3, 1e-4, 1e-4, 1e-4, 1e-4};
        return b[i];
    }
    // calibration.rs:124-126, 169-173
    void bounds(int i, double* lo, double* hi) const {
        static const double l[8] = {1e-8, 1e-6, 1e-8, 1e-6, -0.9999, 0.0, -2.0, 1e-6};
        static const double h[8] = {5.0, 50.0, 5.0, 10.0, 0.9999, 10.0, 2.0, 2.0};
        *lo = l[i];
        *hi = h[i];
    }
    // calibration.rs:130, 174-178
    double reg_scale(int i) const {
        static const double s[8] = {0.04, 2.0, 0.04, 0.3, 0.3, 0.5, 0.1, 0.15};
        return s[i];
    }
    // calibration.rs:186-198 (Bates jump columns through AD); Heston: none.
    bool ad_price_derivative(const double* v, const Contract& c, int col, double* out) const {
        if (dim == 5 || col < 5) return false;
        Heston h{v[0], v[1], v[2], v[3], v[4]};
        double price, d;
        JumpSpec js{2, v[5], v[6], v[7], col - 5};
        forward_pass(c.spot, c.strike, c.expiry, c.rate, c.div_yield, h, c.opt_type, -1, js, REF_TOL, &price, &d);
        *out = d;
        return true;
    }
};

// calibration.rs:573-581
double single_residual(const Model& m, const Contract& c, double iv_mkt, const double* p) {
    double px = m.price(p, c);
    Contract cfi = with_vol(c, iv_mkt);
    double iv;
    if (implied_vol(cfi, px, &iv)) return iv - iv_mkt;
    return 0.0;
}

// calibration.rs:583-587
void residuals(const Model& m, const Quote* q, int n, const double* p, double* out) {
    for (int i = 0; i < n; ++i) out[i] = single_residual(m, q[i].c, q[i].iv_market, p);
}

// calibration.rs:589-591
double weighted_sse(const double* res, const double* w, int n) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) { double t = w[i] * res[i]; s = s + t * t; }
    return s;
}

// calibration.rs:598-605
bool model_iv_and_vega(const Model& m, const Contract& c, double iv_seed, const double* p, double* iv,
                       double* vega) {
    double px = m.price(p, c);
    double v;
    if (!implied_vol(with_vol(c, iv_seed), px, &v)) return false;
    *iv = v;
    *vega = bsm_price_and_greeks(with_vol(c, v)).vega;
    return true;
}

// calibration.rs:613-652 — J is row-major [n_quotes][dim].
void jacobian(const Model& m, const Quote* q, int n, const double* p, double* j) {
    int dim = m.dim;
    std::fill(j, j + (size_t)n * dim, 0.0);
    std::vector<double> colv(n), ru(n), rd(n);
    for (int col = 0; col < dim; ++col) {
        bool ok = true;
        for (int row = 0; row < n && ok; ++row) {
            double dpr, iv, vega;
            if (!m.ad_price_derivative(p, q[row].c, col, &dpr)) { ok = false; break; }
            if (!model_iv_and_vega(m, q[row].c, q[row].iv_market, p, &iv, &vega)) { ok = false; break; }
            if (std::fabs(vega) < 1e-10) { ok = false; break; }
            colv[row] = dpr / vega;
        }
        if (ok) {
            for (int row = 0; row < n; ++row) j[(size_t)row * dim + col] = colv[row];
            continue;
        }
        double lo, hi;
        m.bounds(col, &lo, &hi);
        double vu[8], vd[8];
        for (int i = 0; i < dim; ++i) { vu[i] = p[i]; vd[i] = p[i]; }
        vu[col] = std::min(p[col] + m.bump(col), hi);
        vd[col] = std::max(p[col] - m.bump(col), lo);
        double h = vu[col] - vd[col];
        if (h <= 0.0) continue;
        residuals(m, q, n, vu, ru.data());
        residuals(m, q, n, vd, rd.data());
        for (int row = 0; row < n; ++row) j[(size_t)row * dim + col] = (ru[row] - rd[row]) / h;
    }
}

// calibration.rs:655-668
void jtj_and_grad(const double* j, int rows, const double* res, const double* w, int n, double* jtj,
                  double* grad) {
    std::fill(jtj, jtj + n * n, 0.0);
    std::fill(grad, grad + n, 0.0);
    for (int row = 0; row < rows; ++row) {
        double w2 = w[row] * w[row];
        const double* jr = j + (size_t)row * n;
        for (int c1 = 0; c1 < n; ++c1) {
            grad[c1] += (w2 * jr[c1]) * res[row];
            for (int c2 = 0; c2 < n; ++c2) jtj[c1 * n + c2] += (w2 * jr[c1]) * jr[c2];
        }
    }
}

// calibration.rs:673-703
void lm_step(const double* jtj, const double* grad, double lam, int n, double* dp) {
    double a[8][8], b[8];
    for (int i = 0; i < n; ++i) {
        for (int k = 0; k < n; ++k) a[i][k] = jtj[i * n + k];
        b[i] = grad[i];
    }
    for (int i = 0; i < n; ++i) { a[i][i] *= 1.0 + lam; b[i] = -b[i]; }
    for (int col = 0; col < n; ++col) {
        // max_by(partial_cmp) over rows col..n: last maximum wins
        int pivot = col;
        for (int i = col + 1; i < n; ++i)
            if (std::fabs(a[i][col]) >= std::fabs(a[pivot][col])) pivot = i;
        for (int k = 0; k < n; ++k) std::swap(a[col][k], a[pivot][k]);
        std::swap(b[col], b[pivot]);
        if (std::fabs(a[col][col]) < 1e-15) continue;
        double inv = 1.0 / a[col][col];
        for (int row = col + 1; row < n; ++row) {
            double f = a[row][col] * inv;
            for (int k = col; k < n; ++k) a[row][k] -= f * a[col][k];
            b[row] -= f * b[col];
        }
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = b[i];
        for (int k = i + 1; k < n; ++k) s -= a[i][k] * dp[k];
        dp[i] = std::fabs(a[i][i]) > 1e-15 ? s / a[i][i] : 0.0;
    }
}

// calibration.rs:717-768 (eigenvector i is column i of v)
void jacobi_eigen(const double* a_in, int n, double* evals, double* evecs /* [i][k] = v[k][i] */) {
    double a[8][8], v[8][8];
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) { a[i][k] = a_in[i * n + k]; v[i][k] = (i == k) ? 1.0 : 0.0; }
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < n; ++i) {
            double row = 0.0;
            for (int jj = i + 1; jj < n; ++jj) row = row + a[i][jj] * a[i][jj];
            off = off + row;
        }
        if (std::sqrt(off) < 1e-14) break;
        for (int p = 0; p < n; ++p) {
            for (int q = p + 1; q < n; ++q) {
                if (std::fabs(a[p][q]) < 1e-300) continue;
                double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
                double t = theta >= 0.0 ? 1.0 / (theta + std::sqrt(theta * theta + 1.0))
                                        : -1.0 / (-theta + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0);
                double s = t * c;
                double apq = a[p][q];
                a[p][p] -= t * apq;
                a[q][q] += t * apq;
                a[p][q] = 0.0;
                a[q][p] = 0.0;
                for (int i = 0; i < n; ++i) {
                    if (i != p && i != q) {
                        double aip = a[i][p], aiq = a[i][q];
                        a[i][p] = c * aip - s * aiq; a[p][i] = a[i][p];
                        a[i][q] = s * aip + c * aiq; a[q][i] = a[i][q];
                    }
                }
                for (int row = 0; row < n; ++row) {
                    double vip = v[row][p], viq = v[row][q];
                    v[row][p] = c * vip - s * viq;
                    v[row][q] = s * vip + c * viq;
                }
            }
        }
    }
    for (int i = 0; i < n; ++i) evals[i] = a[i][i];
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) evecs[i * n + k] = v[k][i];
}

struct CalibOut {
    double params[8];
    double rmse, max_err, condition_number;
    double weakest[8];
    int32_t iters, converged, early_stopped, pad;
};

// The device LM's Jacobian restated on the CPU (not the reference's): every
// column exact, d iv / d p = (d price / d p by forward-mode AD) / BSM vega at
// the model IV, and a zero row where that IV solve fails or |vega| < 1e-10.
// The reference (jacobian above) uses central differences for the Heston
// columns; this variant lets a test follow the device LM iteration for
// iteration.
void jacobian_exact(const Model& m, const Quote* q, int n, const double* p, double* j) {
    int dim = m.dim;
    Heston h{p[0], p[1], p[2], p[3], p[4]};
    bool bates = dim == 8;
    for (int row = 0; row < n; ++row) {
        const Contract& c = q[row].c;
        double* jr = j + (size_t)row * dim;
        double px = m.price(p, c);
        double iv, vega = 0.0;
        bool ok = implied_vol(with_vol(c, q[row].iv_market), px, &iv);
        if (ok) vega = bsm_price_and_greeks(with_vol(c, iv)).vega;
        if (!ok || std::fabs(vega) < 1e-10) {
            for (int k = 0; k < dim; ++k) jr[k] = 0.0;
            continue;
        }
        JumpSpec js = bates ? JumpSpec{1, p[5], p[6], p[7], -1} : JumpSpec{0, 0, 0, 0, -1};
        for (int a = 0; a < 5; ++a) {
            double pv, dv;
            forward_pass(c.spot, c.strike, c.expiry, c.rate, c.div_yield, h, c.opt_type, a, js, REF_TOL, &pv, &dv);
            jr[a] = dv / vega;
        }
        for (int a = 0; bates && a < 3; ++a) {
            double pv, dv;
            JumpSpec ja{2, p[5], p[6], p[7], a};
            forward_pass(c.spot, c.strike, c.expiry, c.rate, c.div_yield, h, c.opt_type, -1, ja, REF_TOL, &pv, &dv);
            jr[5 + a] = dv / vega;
        }
    }
}

// calibration.rs:433-569 as a resumable state machine: init() is the set-up
// (lines 438-479), step() one pass of the iteration loop (481-538), finish()
// the data-only diagnostics (541-568).  Running step() until done() is
// exactly calibrate_inner; multistart runs several machines in lockstep.
// prior == nullptr: no Tikhonov rows (calibration.rs:448-470).  jac_mode 0:
// the reference's Jacobian; 1: jacobian_exact.
struct LMRun {
    static constexpr int MAX_ITER = 200;                                          // calibration.rs:30
    static constexpr double TOL_GRAD = 1e-8, TOL_PARAMS = 1e-10, LM_INIT = 1e-3,  // calibration.rs:31-36
        LM_UP = 10.0, LM_DOWN = 0.1, LM_MAX = 1e8, PRUNE_FACTOR = 8.0;           // calibration.rs:263
    static constexpr int PRUNE_CHECK_EVERY = 10;                                  // calibration.rs:264

    const Model* m = nullptr;
    const Quote* q = nullptr;
    int n = 0, dim = 0, rows = 0, jac_mode = 0;
    const double* prior = nullptr;
    double reg_weight = 0.0;
    std::vector<double> base_w, res, w, res_new, w_new, j;
    double p[8] = {0};
    double lam = LM_INIT, sse = 0.0;
    int iters = 0, iter = 0;
    bool converged = false, early_stopped = false, finished = false;

    void jac(const double* pv, double* jj) const {
        if (jac_mode == 1) jacobian_exact(*m, q, n, pv, jj);
        else jacobian(*m, q, n, pv, jj);
    }
    void aug_res(const double* pv, double* r, double* ww) const {
        residuals(*m, q, n, pv, r);
        for (int i = 0; i < n; ++i) ww[i] = base_w[i];
        if (prior) {
            double rw = std::sqrt(reg_weight);
            for (int i = 0; i < dim; ++i) { r[n + i] = (pv[i] - prior[i]) / m->reg_scale(i); ww[n + i] = rw; }
        }
    }
    void aug_jac(const double* pv, double* jj) const {
        jac(pv, jj);
        if (prior)
            for (int i = 0; i < dim; ++i)
                for (int c = 0; c < dim; ++c) jj[(size_t)(n + i) * dim + c] = (c == i) ? 1.0 / m->reg_scale(i) : 0.0;
    }
    void init(const Model& model, const Quote* quotes, int nq, const double* p0, const double* pr, double rw, int jm) {
        m = &model; q = quotes; n = nq; dim = model.dim; prior = pr; reg_weight = rw; jac_mode = jm;
        rows = n + (prior ? dim : 0);
        base_w.resize(n);
        for (int i = 0; i < n; ++i) base_w[i] = q[i].weight;
        res.resize(rows); w.resize(rows); res_new.resize(rows); w_new.resize(rows); j.resize((size_t)rows * dim);
        for (int i = 0; i < dim; ++i) p[i] = p0[i];
        lam = LM_INIT;
        aug_res(p, res.data(), w.data());
        sse = weighted_sse(res.data(), w.data(), rows);
    }
    bool done() const { return finished || iter >= MAX_ITER; }
    // One loop iteration.  prune: this run takes part in multistart pruning,
    // against `shared_best` (the shared best SSE as it reads at the top of the
    // iteration).  *accepted_sse receives the new SSE after an accepted step,
    // else NaN (it is what the run would publish to the shared best).
    void step(bool prune, double shared_best, double* accepted_sse) {
        *accepted_sse = std::numeric_limits<double>::quiet_NaN();
        if (done()) return;
        iters = iter + 1;
        int this_iter = iter++;
        if (prune && this_iter > 0 && this_iter % PRUNE_CHECK_EVERY == 0) {
            if (std::isfinite(shared_best) && sse > shared_best * PRUNE_FACTOR) {
                early_stopped = true;
                finished = true;
                return;
            }
        }
        aug_jac(p, j.data());
        double jtj[64], grad[8];
        jtj_and_grad(j.data(), rows, res.data(), w.data(), dim, jtj, grad);
        double gn = 0.0;
        for (int i = 0; i < dim; ++i) gn = gn + grad[i] * grad[i];
        if (std::sqrt(gn) < TOL_GRAD) { converged = true; finished = true; return; }
        double dp[8];
        lm_step(jtj, grad, lam, dim, dp);
        double p_new[8];
        for (int i = 0; i < dim; ++i) p_new[i] = p[i] + dp[i];
        if (!m->bounds_ok(p_new)) { lam = std::min(lam * LM_UP, LM_MAX); return; }
        aug_res(p_new, res_new.data(), w_new.data());
        double sse_new = weighted_sse(res_new.data(), w_new.data(), rows);
        if (sse_new < sse) {
            for (int i = 0; i < dim; ++i) p[i] = p_new[i];
            res.swap(res_new);
            w.swap(w_new);
            sse = sse_new;
            lam = std::max(lam * LM_DOWN, 1e-12);
            *accepted_sse = sse;
            double sn = 0.0;
            for (int i = 0; i < dim; ++i) sn = sn + dp[i] * dp[i];
            if (std::sqrt(sn) < TOL_PARAMS) { converged = true; finished = true; }
        } else {
            lam = std::min(lam * LM_UP, LM_MAX);
            if (lam >= LM_MAX) finished = true;
        }
    }
    CalibOut finish() const {
        CalibOut o{};
        for (int i = 0; i < dim; ++i) o.params[i] = p[i];
        std::vector<double> rd(n);
        residuals(*m, q, n, p, rd.data());
        double wsum = 0.0;
        for (int i = 0; i < n; ++i) wsum = wsum + base_w[i] * base_w[i];
        o.rmse = std::sqrt(weighted_sse(rd.data(), base_w.data(), n) / wsum);
        double mx = 0.0;
        for (int i = 0; i < n; ++i) mx = std::fmax(mx, std::fabs(rd[i]));
        o.max_err = mx;
        std::vector<double> fj((size_t)n * dim);
        jac(p, fj.data());
        double jtj[64], grad[8], ev[8], evec[64];
        jtj_and_grad(fj.data(), n, rd.data(), base_w.data(), dim, jtj, grad);
        jacobi_eigen(jtj, dim, ev, evec);
        double mx_e = -std::numeric_limits<double>::max(), mn_e = std::numeric_limits<double>::max();
        for (int i = 0; i < dim; ++i) { mx_e = std::fmax(mx_e, ev[i]); mn_e = std::fmin(mn_e, ev[i]); }
        o.condition_number = std::fabs(mn_e) > 1e-300 ? std::fabs(mx_e / mn_e) : INFINITY;
        int weakest = 0;
        for (int i = 1; i < dim; ++i)
            if (total_key(std::fabs(ev[i])) < total_key(std::fabs(ev[weakest]))) weakest = i;  // min_by: first min
        for (int k = 0; k < dim; ++k) o.weakest[k] = evec[weakest * dim + k];
        o.iters = iters;
        o.converged = converged ? 1 : 0;
        o.early_stopped = early_stopped ? 1 : 0;
        return o;
    }
};

// calibration.rs:433-569.  shared_best: initial shared best SSE for a run
// that takes part in pruning (calibration.rs:482-490); NaN: no pruning.
CalibOut calibrate_inner(const Model& m, const Quote* q, int n, const double* p0, const double* prior,
                         double reg_weight, int jac_mode = 0, double shared_best = NAN) {
    LMRun r;
    r.init(m, q, n, p0, prior, reg_weight, jac_mode);
    const bool prune = !std::isnan(shared_best);
    double acc;
    while (!r.done()) {
        r.step(prune, shared_best, &acc);
        if (prune && acc < shared_best) shared_best = acc;
    }
    return r.finish();
}

// ---------------------------------------------------------------------------
// rand 0.8 SmallRng + the samplers the calibration calls (calibration.rs:
// 131-141, 179-185, 284, 372-392).  The reference lock file does not pin
// rand (Cargo.toml:19 asks for 0.8 with small_rng), so this restates the
// published 0.8.5 algorithms: SmallRng on 64-bit targets is xoshiro256++
// (Blackman & Vigna), seeded by rand_core's default seed_from_u64 (PCG32);
// gen::<f64>() = (next_u64 >> 11) * 2^-53; gen_range(lo..hi) on f64
// draws v in [1,2) from the top 52 bits, res = (v - 1) * (hi - lo) + lo,
// redrawn while res >= hi; gen_range(lo..hi) on usize is the widening-
// multiply method with the (range << leading_zeros) - 1 rejection zone.
// ---------------------------------------------------------------------------
inline uint64_t splitmix64(uint64_t x) {  // mc.rs:337-343
    x = x + 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct SmallRng {
    uint64_t s[4];
    // xoshiro256++'s own seed_from_u64 (four SplitMix64 outputs); rand uses it
    // only for an all-zero seed (Xoshiro256PlusPlus::from_seed).
    static SmallRng xoshiro_seed_from_u64(uint64_t state) {
        SmallRng r;
        for (int k = 0; k < 4; ++k) {
            state = state + 0x9e3779b97f4a7c15ull;
            uint64_t z = state;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            r.s[k] = z ^ (z >> 31);
        }
        return r;
    }
    // SmallRng::seed_from_u64 in rand 0.8 is rand_core 0.6's default
    // SeedableRng::seed_from_u64 (SmallRng does not forward it to the inner
    // generator): the 32-byte seed is eight PCG32 (XSH-RR) outputs, little
    // endian, then Xoshiro256PlusPlus::from_seed.
    static SmallRng seed_from_u64(uint64_t state) {
        uint32_t x[8];
        for (int k = 0; k < 8; ++k) {
            state = state * 6364136223846793005ull + 11634580027462260723ull;
            uint32_t xorshifted = (uint32_t)(((state >> 18) ^ state) >> 27);
            uint32_t rot = (uint32_t)(state >> 59);
            x[k] = (xorshifted >> rot) | (xorshifted << ((32 - rot) & 31));
        }
        SmallRng r;
        for (int k = 0; k < 4; ++k) r.s[k] = (uint64_t)x[2 * k] | ((uint64_t)x[2 * k + 1] << 32);
        if ((r.s[0] | r.s[1] | r.s[2] | r.s[3]) == 0) return xoshiro_seed_from_u64(0);
        return r;
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next_u64() {
        uint64_t result = rotl(s[0] + s[3], 23) + s[0];
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return result;
    }
    double gen_f64() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
    double gen_range_f64(double lo, double hi) {
        double scale = hi - lo;
        for (;;) {
            uint64_t bits = (next_u64() >> 12) | 0x3ff0000000000000ull;
            double v12;
            std::memcpy(&v12, &bits, 8);
            double res = (v12 - 1.0) * scale + lo;
            if (res < hi) return res;
        }
    }
    uint64_t gen_range_usize(uint64_t lo, uint64_t hi) {  // [lo, hi)
        uint64_t range = (hi - 1) - lo + 1;
        if (range == 0) return next_u64();
        uint64_t zone = (range << __builtin_clzll(range)) - 1;
        for (;;) {
            uint64_t v = next_u64();
            unsigned __int128 mm = (unsigned __int128)v * range;
            if ((uint64_t)mm <= zone) return lo + (uint64_t)(mm >> 64);
        }
    }
};

// calibration.rs:131-141 (Heston) and 179-185 (Bates)
void random_guess(int dim, SmallRng& rng, double* v) {
    double v0 = rng.gen_range_f64(0.005, 0.5);
    double kappa = rng.gen_range_f64(0.3, 8.0);
    double theta = rng.gen_range_f64(0.005, 0.5);
    double sigma_cap = std::fmax(std::sqrt((2.0 * kappa) * theta) * 0.9, 0.05);
    double sigma = rng.gen_range_f64(0.02, sigma_cap);
    double rho = rng.gen_range_f64(-0.9, 0.9);
    v[0] = v0; v[1] = kappa; v[2] = theta; v[3] = sigma; v[4] = rho;
    if (dim == 8) {
        v[5] = rng.gen_range_f64(0.0, 2.0);
        v[6] = rng.gen_range_f64(-0.3, 0.1);
        v[7] = rng.gen_range_f64(0.02, 0.4);
    }
}

inline double rust_clamp(double x, double lo, double hi) {  // f64::clamp
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}

inline int threads_or_default(int nthreads) {
#ifdef _OPENMP
    return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

inline Heston heston_from(const double* hp) { return Heston{hp[0], hp[1], hp[2], hp[3], hp[4]}; }
inline Bates bates_from(const double* bp) { return Bates{{bp[0], bp[1], bp[2], bp[3], bp[4]}, bp[5], bp[6], bp[7]}; }

}  // namespace

// ===========================================================================
// C exports (ctypes).  Parameter packs: Heston = 5 doubles (v0,kappa,theta,
// sigma,rho); Bates = 8 doubles (Heston + lambda, mu_j, sigma_j).
// ===========================================================================
extern "C" {

void orc_fast_csqrt(double re, double im, double* out) {
    Cx z = fast_csqrt(Cx{re, im});
    out[0] = z.re; out[1] = z.im;
}

void orc_stable_cf(double phi_re, double phi_im, double t, double r, const double* hp, double* out) {
    Cx z = stable_cf(Cx{phi_re, phi_im}, t, r, heston_from(hp));
    out[0] = z.re; out[1] = z.im;
}

void orc_jump_cf(double phi_re, double phi_im, double t, const double* bp, double* out) {
    Cx z = jump_cf(Cx{phi_re, phi_im}, t, bates_from(bp));
    out[0] = z.re; out[1] = z.im;
}

double orc_cf_integrand(double u, double s, double k, double t, double r, const double* hp, int is_p1) {
    Heston p = heston_from(hp);
    double x = std::log(s / k);
    Cx cf_mi = stable_cf(Cx{0.0, -1.0}, t, r, p);
    return cf_integrand(u, x, t, r, p, is_p1 != 0, is_p1 ? &cf_mi : nullptr);
}

double orc_heston_price(double spot, double strike, double expiry, double rate, double div_yield,
                        const double* hp, int opt_type, double tol, int* bisections2) {
    return heston_price(spot, strike, expiry, rate, div_yield, heston_from(hp), opt_type, tol, bisections2);
}

double orc_bates_price(double spot, double strike, double expiry, double rate, double div_yield,
                       const double* bp, int opt_type, double tol, int* bisections2) {
    return bates_price(spot, strike, expiry, rate, div_yield, bates_from(bp), opt_type, tol, bisections2);
}

// Step trace of one Gil-Pelaez integral (which: 0 = P1, 1 = P2) of one
// contract, with the integrand built as heston_call / bates_call build it
// (heston.rs:86-93, bates.rs:53-59).  out: max_steps x TRACE_FIELDS doubles
// (QagTrace).  Returns the number of steps (1 + bisections); *integral
// receives the integral.
int orc_trace_integral(const void* contract, const double* params, int bates, int which, double tol,
                       double* out, int max_steps, double* integral) {
    const Contract& c = *static_cast<const Contract*>(contract);
    const double x = std::log(c.spot / c.strike);
    const double t = c.expiry, r = c.rate;
    QagTrace tr{out, max_steps};
    double v;
    if (bates) {
        const Bates bp = bates_from(params);
        const Cx phi_mi{0.0, -1.0};
        const Cx cf_mi = stable_cf(phi_mi, t, r, bp.h) * jump_cf(phi_mi, t, bp);
        v = gk_integrate([&](double u) { return bates_integrand(u, x, t, r, bp, which == 0, which == 0 ? &cf_mi : nullptr); },
                         tol, nullptr, &tr);
    } else {
        const Heston p = heston_from(params);
        const Cx cf_mi = stable_cf(Cx{0.0, -1.0}, t, r, p);
        v = gk_integrate([&](double u) { return cf_integrand(u, x, t, r, p, which == 0, which == 0 ? &cf_mi : nullptr); },
                         tol, nullptr, &tr);
    }
    if (integral) *integral = v;
    return tr.steps;
}

// batch.rs:23-27 / 38-42 generalised to many parameter sets: contract i uses
// params[surf_idx[i]] (surf_idx may be NULL: all use params[0]).  `stride` is
// 5 (Heston) or 8 (Bates); bates != 0 selects the Bates pricer.  OpenMP
// dynamic schedule, one contract per iteration (the rayon par_iter analogue).
void orc_batch_price(const void* contracts, int64_t n, const int32_t* surf_idx, const double* params,
                     int bates, double tol, double* out, int32_t* bisections, int nthreads) {
    const Contract* c = static_cast<const Contract*>(contracts);
    int nt = threads_or_default(nthreads);
    const int stride = bates ? 8 : 5;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t i = 0; i < n; ++i) {
        const double* pp = params + (size_t)(surf_idx ? surf_idx[i] : 0) * stride;
        int nb[2] = {0, 0};
        const Contract& ci = c[i];
        double v = bates ? bates_price(ci.spot, ci.strike, ci.expiry, ci.rate, ci.div_yield, bates_from(pp),
                                       ci.opt_type, tol, nb)
                         : heston_price(ci.spot, ci.strike, ci.expiry, ci.rate, ci.div_yield, heston_from(pp),
                                        ci.opt_type, tol, nb);
        out[i] = v;
        if (bisections) { bisections[2 * i] = nb[0]; bisections[2 * i + 1] = nb[1]; }
    }
}

// batch.rs:32-36 / 44-48 via greeks.rs:19-72.  out: 8 doubles per contract.
void orc_batch_greeks(const void* contracts, int64_t n, const double* params, int bates, double tol,
                      double* out, int nthreads) {
    const Contract* c = static_cast<const Contract*>(contracts);
    int nt = threads_or_default(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t i = 0; i < n; ++i) {
        const Contract& ci = c[i];
        Result8 r;
        if (bates) {
            Bates b = bates_from(params);
            r = bump_and_reprice(ci.spot, ci.strike, ci.expiry, ci.rate, ci.div_yield, b, b.h.v0, ci.opt_type,
                [&](double s, double k, double t, double rr, double q, const Bates& pp, int ot) {
                    return bates_price(s, k, t, rr, q, pp, ot, tol, nullptr); },
                [](const Bates& pp, double v0) { Bates o = pp; o.h.v0 = v0; return o; });
        } else {
            Heston h = heston_from(params);
            r = bump_and_reprice(ci.spot, ci.strike, ci.expiry, ci.rate, ci.div_yield, h, h.v0, ci.opt_type,
                [&](double s, double k, double t, double rr, double q, const Heston& pp, int ot) {
                    return heston_price(s, k, t, rr, q, pp, ot, tol, nullptr); },
                [](const Heston& pp, double v0) { Heston o = pp; o.v0 = v0; return o; });
        }
        std::memcpy(out + 8 * i, &r, sizeof(r));
    }
}

double orc_npdf(double x) { return npdf(x); }
double orc_ncdf(double x) { return ncdf(x); }
double orc_ncdf_inv(double p) { return ncdf_inv(p); }
double orc_bsm_price(const void* contract) { return bsm_price(*static_cast<const Contract*>(contract)); }
void orc_bsm_price_and_greeks(const void* contract, double* out8) {
    Result8 r = bsm_price_and_greeks(*static_cast<const Contract*>(contract));
    std::memcpy(out8, &r, sizeof(r));
}
void orc_batch_implied_vol(const void* contracts, int64_t n, const double* prices, double* out, int32_t* ok,
                           int nthreads) {
    const Contract* c = static_cast<const Contract*>(contracts);
    int nt = threads_or_default(nthreads);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt)
    for (int64_t i = 0; i < n; ++i) {
        double v = 0.0;
        ok[i] = implied_vol(c[i], prices[i], &v) ? 1 : 0;
        out[i] = v;
    }
}

int orc_implied_vol(const void* contract, double market_price, double* out) {
    return implied_vol(*static_cast<const Contract*>(contract), market_price, out) ? 1 : 0;
}

// ad.rs:695-731.  active: 0..4 = Heston param index, -1 = none.
// jump_mode: 0 Off, 1 Const, 2 Active (jump_active: 0 lambda, 1 mu_j, 2 sigma_j).
void orc_forward_pass(double s, double k, double t, double r, double q, const double* hp, int opt_type,
                      int active, int jump_mode, double lambda, double mu_j, double sigma_j, int jump_active,
                      double tol, double* price, double* dprice) {
    JumpSpec js{jump_mode, lambda, mu_j, sigma_j, jump_active};
    forward_pass(s, k, t, r, q, heston_from(hp), opt_type, active, js, tol, price, dprice);
}

// The full price gradient the adjoint kernel computes, assembled from
// forward passes: d/d(v0,kappa,theta,sigma,rho) (ad.rs:736-745, 821-825) and,
// for Bates, d/d(lambda,mu_j,sigma_j) (ad.rs:882-895).  One contract; out has
// 5 (Heston) or 8 (Bates) entries; *price from the first pass.
void orc_price_gradient(const void* contract, const double* params, int bates, double tol, double* price,
                        double* grad) {
    const Contract& c = *static_cast<const Contract*>(contract);
    Heston h = heston_from(params);
    JumpSpec js = bates ? JumpSpec{1, params[5], params[6], params[7], -1} : JumpSpec{0, 0, 0, 0, -1};
    for (int a = 0; a < 5; ++a) {
        double pv, dv;
        forward_pass(c.spot, c.strike, c.expiry, c.rate, c.div_yield, h, c.opt_type, a, js, tol, &pv, &dv);
        grad[a] = dv;
        if (a == 0) *price = pv;
    }
    if (bates) {
        for (int a = 0; a < 3; ++a) {
            double pv, dv;
            JumpSpec ja{2, params[5], params[6], params[7], a};
            forward_pass(c.spot, c.strike, c.expiry, c.rate, c.div_yield, h, c.opt_type, -1, ja, tol, &pv, &dv);
            grad[5 + a] = dv;
        }
    }
}

void orc_batch_price_gradient(const void* contracts, int64_t n, const int32_t* surf_idx, const double* params,
                              int bates, double tol, double* price, double* grad, int nthreads) {
    const Contract* c = static_cast<const Contract*>(contracts);
    int nt = threads_or_default(nthreads);
    const int stride = bates ? 8 : 5;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int64_t i = 0; i < n; ++i) {
        const double* pp = params + (size_t)(surf_idx ? surf_idx[i] : 0) * stride;
        orc_price_gradient(&c[i], pp, bates, tol, price + i, grad + (size_t)i * stride);
    }
}

// ad.rs:736-795 (heston_greeks_ad) and ad.rs:809-865 (bates_greeks_ad); the
// FD legs use the plain pricer at the reference tolerance, as the reference does.
void orc_greeks_ad(const void* contract, const double* params, int bates, double tol, double* out8) {
    const Contract& c = *static_cast<const Contract*>(contract);
    double spot = c.spot, strike = c.strike, expiry = c.expiry, rate = c.rate, dy = c.div_yield;
    int ot = c.opt_type;
    Heston h = heston_from(params);
    JumpSpec js = bates ? JumpSpec{1, params[5], params[6], params[7], -1} : JumpSpec{0, 0, 0, 0, -1};
    auto px = [&](double s, double t, double r, const Heston& hh) {
        if (bates) {
            Bates b{hh, params[5], params[6], params[7]};
            return bates_price(s, strike, t, r, dy, b, ot, tol, nullptr);
        }
        return heston_price(s, strike, t, r, dy, hh, ot, tol, nullptr);
    };
    double price, dv0;
    forward_pass(spot, strike, expiry, rate, dy, h, ot, 0, js, tol, &price, &dv0);
    double vol = std::sqrt(h.v0);
    double vega = (dv0 * 2.0) * vol;
    double dr = 1e-4;
    double rho_g = (px(spot, expiry, rate + dr, h) - px(spot, expiry, rate - dr, h)) / (2.0 * dr);
    double ds = 0.01 * spot;
    double p_sup = px(spot + ds, expiry, rate, h), p_sdn = px(spot - ds, expiry, rate, h);
    double delta = (p_sup - p_sdn) / (2.0 * ds);
    double gamma = ((p_sup - 2.0 * price) + p_sdn) / (ds * ds);
    double t_dn = std::fmax(expiry - 1.0 / 365.0, 1e-6);
    double theta = (px(spot, t_dn, rate, h) - price) / (1.0 / 365.0);
    double vu = vol + 0.01, vd = std::fmax(vol - 0.01, 1e-6);
    Heston h_up = h; h_up.v0 = vu * vu;
    Heston h_dn = h; h_dn.v0 = vd * vd;
    double delta_vup = (px(spot + ds, expiry, rate, h_up) - px(spot - ds, expiry, rate, h_up)) / (2.0 * ds);
    double delta_vdn = (px(spot + ds, expiry, rate, h_dn) - px(spot - ds, expiry, rate, h_dn)) / (2.0 * ds);
    double vanna = (delta_vup - delta_vdn) / (2.0 * 0.01);
    double pv, dup, ddn;
    forward_pass(spot, strike, expiry, rate, dy, h_up, ot, 0, js, tol, &pv, &dup);
    forward_pass(spot, strike, expiry, rate, dy, h_dn, ot, 0, js, tol, &pv, &ddn);
    double vega_up = (dup * 2.0) * (vol + 0.01);
    double vega_dn = (ddn * 2.0) * std::fmax(vol - 0.01, 1e-6);
    double volga = (vega_up - vega_dn) / (2.0 * 0.01);
    double o[8] = {price, delta, gamma, vega, theta, rho_g, vanna, volga};
    std::memcpy(out8, o, sizeof(o));
}

// One LM calibration (calibration.rs:204-210, 220-230, 433-569).
// quotes: contracts[n] + iv_market[n] + weight[n].  dim 5 = Heston, 8 = Bates.
// prior may be NULL (no regularisation).  out: CalibOut (see above).
void orc_calibrate(int dim, const void* contracts, const double* iv_market, const double* weight, int n,
                   const double* p0, const double* prior, double reg_weight, void* out) {
    const Contract* c = static_cast<const Contract*>(contracts);
    std::vector<Quote> q(n);
    for (int i = 0; i < n; ++i) q[i] = Quote{c[i], iv_market[i], weight ? weight[i] : 1.0};
    Model m{dim};
    CalibOut o = calibrate_inner(m, q.data(), n, p0, prior, reg_weight);
    std::memcpy(out, &o, sizeof(o));
}

// One LM calibration with every option of calibrate_inner: Tikhonov prior
// (calibration.rs:220-230; prior NULL = none), the Jacobian variant
// (jac_mode, see LMRun) and a fixed shared best SSE to prune against
// (calibration.rs:482-490; NaN = no pruning, as calibrate_heston does).
void orc_calibrate_ex(int dim, const void* contracts, const double* iv_market, const double* weight, int n,
                      const double* p0, const double* prior, double reg_weight, int jac_mode, double shared_best,
                      void* out) {
    const Contract* c = static_cast<const Contract*>(contracts);
    std::vector<Quote> q(n);
    for (int i = 0; i < n; ++i) q[i] = Quote{c[i], iv_market[i], weight ? weight[i] : 1.0};
    Model m{dim};
    CalibOut o = calibrate_inner(m, q.data(), n, p0, prior, reg_weight, jac_mode, shared_best);
    std::memcpy(out, &o, sizeof(o));
}

// calibration.rs:246-314 calibrate_multistart.  Restart 0 starts at p0,
// restart i at random_guess(SmallRng::seed_from_u64(splitmix64(seed ^ i))).
// The reference runs restarts on rayon threads against a mutex-guarded
// shared best, so which pruning checks see which updates depends on thread
// timing.  Here the restarts advance in lockstep, one iteration each per
// round, and every check of round k sees the updates of rounds < k: one of
// the schedules the reference allows, and the one the device runs.
// shared_best0: the shared best's initial value (the reference: +inf).
// out_best: CalibOut of the lowest-RMSE restart (min_by: first minimum);
// out_all (NULL or n_restarts records); counts = {n_converged, n_pruned,
// index of the best restart}.
void orc_calibrate_multistart(int dim, const void* contracts, const double* iv_market, const double* weight, int n,
                              const double* p0, int n_restarts, uint64_t seed, int jac_mode, double shared_best0,
                              void* out_best, void* out_all, int32_t* counts, int nthreads) {
    const Contract* c = static_cast<const Contract*>(contracts);
    std::vector<Quote> q(n);
    for (int i = 0; i < n; ++i) q[i] = Quote{c[i], iv_market[i], weight ? weight[i] : 1.0};
    Model m{dim};
    const int nr = std::max(n_restarts, 1);
    std::vector<double> starts((size_t)nr * dim);
    for (int i = 0; i < nr; ++i) {
        double* v = starts.data() + (size_t)i * dim;
        if (i == 0) {
            for (int k = 0; k < dim; ++k) v[k] = p0[k];
        } else {
            SmallRng rng = SmallRng::seed_from_u64(splitmix64(seed ^ (uint64_t)i));
            random_guess(dim, rng, v);
        }
    }
    std::vector<LMRun> runs(nr);
    int nt = threads_or_default(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int i = 0; i < nr; ++i) runs[i].init(m, q.data(), n, starts.data() + (size_t)i * dim, nullptr, 0.0, jac_mode);
    double shared = shared_best0;
    std::vector<double> acc(nr);
    for (;;) {
        bool any = false;
        for (int i = 0; i < nr; ++i) any = any || !runs[i].done();
        if (!any) break;
        const double snap = shared;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
        for (int i = 0; i < nr; ++i) runs[i].step(true, snap, &acc[i]);
        for (int i = 0; i < nr; ++i)
            if (acc[i] < shared) shared = acc[i];
    }
    std::vector<CalibOut> res(nr);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int i = 0; i < nr; ++i) res[i] = runs[i].finish();
    int best = 0, n_conv = 0, n_pruned = 0;
    for (int i = 0; i < nr; ++i) {
        n_conv += res[i].converged;
        n_pruned += res[i].early_stopped;
        if (total_key(res[i].rmse) < total_key(res[best].rmse)) best = i;
    }
    std::memcpy(out_best, &res[best], sizeof(CalibOut));
    if (out_all) std::memcpy(out_all, res.data(), sizeof(CalibOut) * nr);
    counts[0] = n_conv;
    counts[1] = n_pruned;
    counts[2] = best;
}

// calibration.rs:349-427 calibrate_global: DE/rand/1/bin (F 0.6, CR 0.9,
// calibration.rs:324-325) over the parameter box, then one LM polish from
// the DE winner, regularised toward prior when prior != NULL
// (calibration.rs:335-347).  out: CalibOut of the polish; *de_best_sse the
// winner's SSE; pop_out / fit_out (NULL or n_pop_used x dim / n_pop_used):
// the final population and its fitness; *n_pop_used = max(n_pop, 4 dim).
void orc_calibrate_global(int dim, const void* contracts, const double* iv_market, const double* weight, int n,
                          int n_pop, int n_gen, uint64_t seed, const double* prior, double reg_weight, int jac_mode,
                          void* out, double* de_best_sse, double* pop_out, double* fit_out, int32_t* n_pop_used,
                          int nthreads) {
    const Contract* c = static_cast<const Contract*>(contracts);
    std::vector<Quote> q(n);
    for (int i = 0; i < n; ++i) q[i] = Quote{c[i], iv_market[i], weight ? weight[i] : 1.0};
    Model m{dim};
    const int np = std::max(n_pop, 4 * dim);
    std::vector<double> base_w(n);
    for (int i = 0; i < n; ++i) base_w[i] = q[i].weight;
    auto sse_of = [&](const double* v) -> double {
        if (!m.bounds_ok(v)) return INFINITY;
        std::vector<double> r(n);
        residuals(m, q.data(), n, v, r.data());
        return weighted_sse(r.data(), base_w.data(), n);
    };
    double lo[8], hi[8];
    for (int d = 0; d < dim; ++d) m.bounds(d, &lo[d], &hi[d]);
    SmallRng init_rng = SmallRng::seed_from_u64(splitmix64(seed));
    std::vector<double> pop((size_t)np * dim), fit(np);
    for (int i = 0; i < np; ++i) {
        double* v = pop.data() + (size_t)i * dim;
        bool got = false;
        for (int attempt = 0; attempt < 20 && !got; ++attempt) {
            for (int d = 0; d < dim; ++d) v[d] = init_rng.gen_range_f64(lo[d], hi[d]);
            got = std::isfinite(sse_of(v));
        }
        if (!got)
            for (int d = 0; d < dim; ++d) v[d] = init_rng.gen_range_f64(lo[d], hi[d]);
    }
    int nt = threads_or_default(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int i = 0; i < np; ++i) fit[i] = sse_of(pop.data() + (size_t)i * dim);
    const double DE_F = 0.6, DE_CR = 0.9;
    std::vector<double> npop(pop.size()), nfit(np);
    for (int gen = 0; gen < n_gen; ++gen) {
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
        for (int i = 0; i < np; ++i) {
            SmallRng rng = SmallRng::seed_from_u64(splitmix64(seed ^ ((uint64_t)gen << 32) ^ (uint64_t)i));
            uint64_t idx[3] = {0, 0, 0};
            for (int slot = 0; slot < 3; ++slot) {
                for (;;) {
                    uint64_t cand = rng.gen_range_usize(0, (uint64_t)np);
                    bool seen = false;
                    for (int k = 0; k < slot; ++k) seen = seen || idx[k] == cand;
                    if (cand != (uint64_t)i && !seen) { idx[slot] = cand; break; }
                }
            }
            const double* pa = pop.data() + idx[0] * dim;
            const double* pb = pop.data() + idx[1] * dim;
            const double* pc = pop.data() + idx[2] * dim;
            uint64_t forced = rng.gen_range_usize(0, (uint64_t)dim);
            double trial[8];
            for (int d = 0; d < dim; ++d) trial[d] = pop[(size_t)i * dim + d];
            for (int d = 0; d < dim; ++d)
                if ((uint64_t)d == forced || rng.gen_f64() < DE_CR)
                    trial[d] = rust_clamp(pa[d] + DE_F * (pb[d] - pc[d]), lo[d], hi[d]);
            double tf = sse_of(trial);
            double* dst = npop.data() + (size_t)i * dim;
            if (tf < fit[i]) {
                for (int d = 0; d < dim; ++d) dst[d] = trial[d];
                nfit[i] = tf;
            } else {
                for (int d = 0; d < dim; ++d) dst[d] = pop[(size_t)i * dim + d];
                nfit[i] = fit[i];
            }
        }
        pop.swap(npop);
        fit.swap(nfit);
    }
    int best = 0;
    for (int i = 1; i < np; ++i)
        if (total_key(fit[i]) < total_key(fit[best])) best = i;
    *de_best_sse = fit[best];
    *n_pop_used = np;
    if (pop_out) std::memcpy(pop_out, pop.data(), sizeof(double) * pop.size());
    if (fit_out) std::memcpy(fit_out, fit.data(), sizeof(double) * np);
    CalibOut o = calibrate_inner(m, q.data(), n, pop.data() + (size_t)best * dim, prior, reg_weight, jac_mode);
    std::memcpy(out, &o, sizeof(o));
}

// The random-number restatement, exposed for its tests.
uint64_t orc_splitmix64(uint64_t x) { return splitmix64(x); }
void orc_small_rng_u64(uint64_t seed, int n, uint64_t* out) {
    SmallRng r = SmallRng::seed_from_u64(seed);
    for (int i = 0; i < n; ++i) out[i] = r.next_u64();
}
void orc_xoshiro_from_state(const uint64_t* state4, int n, uint64_t* out) {
    SmallRng r;
    for (int k = 0; k < 4; ++k) r.s[k] = state4[k];
    for (int i = 0; i < n; ++i) out[i] = r.next_u64();
}
void orc_rng_gen_range_f64(uint64_t seed, double lo, double hi, int n, double* out) {
    SmallRng r = SmallRng::seed_from_u64(seed);
    for (int i = 0; i < n; ++i) out[i] = r.gen_range_f64(lo, hi);
}
void orc_rng_gen_range_usize(uint64_t seed, uint64_t lo, uint64_t hi, int n, uint64_t* out) {
    SmallRng r = SmallRng::seed_from_u64(seed);
    for (int i = 0; i < n; ++i) out[i] = r.gen_range_usize(lo, hi);
}
void orc_random_guess(int dim, uint64_t seed, double* out) {
    SmallRng r = SmallRng::seed_from_u64(seed);
    random_guess(dim, r, out);
}

// Many independent calibrations (one per surface) over the host cores; the
// CPU analogue of the batched device LM.  surface s owns quotes
// [offsets[s], offsets[s+1]).  outs: n_surf CalibOut records.
void orc_calibrate_many(int dim, const void* contracts, const double* iv_market, const int64_t* offsets,
                        int n_surf, const double* p0s, void* outs, int nthreads) {
    const Contract* c = static_cast<const Contract*>(contracts);
    int nt = threads_or_default(nthreads);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (int s = 0; s < n_surf; ++s) {
        int64_t lo = offsets[s], hi = offsets[s + 1];
        orc_calibrate(dim, c + lo, iv_market + lo, nullptr, (int)(hi - lo), p0s + (size_t)s * dim, nullptr, 0.0,
                      static_cast<char*>(outs) + (size_t)s * sizeof(CalibOut));
    }
}

// calibration.rs:613-652 at params p (row-major n x dim).
void orc_jacobian(int dim, const void* contracts, const double* iv_market, int n, const double* p, double* j) {
    const Contract* c = static_cast<const Contract*>(contracts);
    std::vector<Quote> q(n);
    for (int i = 0; i < n; ++i) q[i] = Quote{c[i], iv_market[i], 1.0};
    Model m{dim};
    jacobian(m, q.data(), n, p, j);
}

void orc_jacobi_eigen(const double* a, int n, double* evals, double* evecs) { jacobi_eigen(a, n, evals, evecs); }
void orc_lm_step(const double* jtj, const double* grad, double lam, int n, double* dp) { lm_step(jtj, grad, lam, n, dp); }

int orc_calib_out_size() { return (int)sizeof(CalibOut); }
int orc_max_threads() { return threads_or_default(0); }

}  // extern "C"
