// The reference crate's own unit tests for the CF pricing path, written
// against the C++ mirror (options-pricing-engine-rs_b200/host/ope.hpp) and so
// run on the GPU: heston.rs:309-427, bates.rs:98-173, batch.rs:246-319,
// calibration.rs:870-1071, 1073-1131, 1216-1234.  Same inputs, same assertions, same tolerances.
// Exit status 0 when every test passes.
#include <cmath>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "../../options-pricing-engine-rs_b200/host/ope.hpp"

using namespace ope;

static int g_fail = 0;
#define EXPECT(cond, ...)                                         \
    do {                                                          \
        if (!(cond)) {                                            \
            std::printf("  assertion failed: %s: ", #cond);       \
            std::printf(__VA_ARGS__);                             \
            std::printf("\n");                                    \
            throw std::runtime_error("assertion");                \
        }                                                         \
    } while (0)

static void run(const char* name, const std::function<void()>& f) {
    try {
        f();
        std::printf("PASS %s\n", name);
    } catch (const std::exception& e) {
        std::printf("FAIL %s (%s)\n", name, e.what());
        ++g_fail;
    }
}

// bsm.rs:55-60, for the BSM-limit tests (BSM itself stays on the CPU)
static double bsm_price(double s, double k, double t, double r, double q, double v, OptionType ot) {
    const double vt = v * std::sqrt(t);
    const double d1 = (std::log(s / k) + (r - q + 0.5 * v * v) * t) / vt;
    const double d2 = d1 - vt;
    const double phi = sign(ot);
    auto N = [](double x) { return 0.5 * std::erfc(-x / std::sqrt(2.0)); };
    return phi * (s * std::exp(-q * t) * N(phi * d1) - k * std::exp(-r * t) * N(phi * d2));
}

static HestonParams params() { return HestonParams{0.04, 2.0, 0.04, 0.3, -0.7}; }  // heston.rs:236-239
static BatesParams bp_with_jumps() { return BatesParams{params(), 0.5, -0.1, 0.15}; }  // bates.rs:94-96

static std::vector<OptionContract> chain(int n) {  // batch.rs:238-244
    std::vector<OptionContract> v;
    for (int i = 0; i < n; ++i) v.push_back(OptionContract{100.0, 80.0 + i * 2.0, 0.5, 0.03, 0.0, 0.20, OptionType::Call});
    return v;
}

int main() {
    // ---------------------------------------------------------------- heston.rs
    run("heston::put_call_parity", [] {
        const auto p = params();
        const double call = heston_price(100.0, 100.0, 0.5, 0.03, 0.0, p, OptionType::Call);
        const double put = heston_price(100.0, 100.0, 0.5, 0.03, 0.0, p, OptionType::Put);
        const double er = std::exp(-0.03 * 0.5);
        EXPECT(std::fabs(call - put - (100.0 - 100.0 * er)) < 0.01, "call %g put %g", call, put);
    });
    run("heston::price_sanity", [] {
        const auto p = params();
        const double call = heston_price(100.0, 100.0, 1.0, 0.05, 0.0, p, OptionType::Call);
        const double put = heston_price(100.0, 100.0, 1.0, 0.05, 0.0, p, OptionType::Put);
        const double pcp = std::fabs(call - put - 100.0 + 100.0 * std::exp(-0.05));
        EXPECT(pcp < 0.05, "pcp err = %g", pcp);
        EXPECT(call >= 0.0, "call %g", call);
    });
    run("heston::feller_condition", [] { EXPECT(params().feller_ok(), "feller"); });
    run("heston::greeks_signs", [] {
        const auto r = heston_price_and_greeks(100.0, 100.0, 1.0, 0.05, 0.0, params(), OptionType::Call);
        EXPECT(r.delta > 0.0 && r.delta < 1.0, "delta=%g", r.delta);
        EXPECT(r.gamma > 0.0, "gamma=%g", r.gamma);
        EXPECT(r.vega > 0.0, "vega=%g", r.vega);
        EXPECT(r.rho > 0.0, "rho=%g", r.rho);
    });
    run("heston::greeks_put_delta_negative", [] {
        const auto r = heston_price_and_greeks(100.0, 100.0, 1.0, 0.05, 0.0, params(), OptionType::Put);
        EXPECT(r.delta < 0.0 && r.delta > -1.0, "put delta=%g", r.delta);
        EXPECT(r.gamma > 0.0, "gamma=%g", r.gamma);
    });
    run("heston::delta_close_to_bsm", [] {
        const HestonParams p{0.04, 0.1, 0.04, 0.01, 0.0};
        const auto h = heston_price_and_greeks(100.0, 100.0, 1.0, 0.05, 0.0, p, OptionType::Call);
        // BSM delta and vega (bsm.rs:15-40)
        const double vt = 0.2, d1 = (std::log(1.0) + (0.05 + 0.5 * 0.04) * 1.0) / vt;
        const double delta = 0.5 * std::erfc(-d1 / std::sqrt(2.0));
        const double vega = 100.0 * 0.3989422804014327 * std::exp(-0.5 * d1 * d1);
        EXPECT(std::fabs(h.delta - delta) < 0.01, "heston delta=%g bsm delta=%g", h.delta, delta);
        const double damp = (1.0 - std::exp(-p.kappa * 1.0)) / p.kappa;
        EXPECT(std::fabs(h.vega - vega * damp) < 0.5, "heston vega=%g bsm vega*damp=%g", h.vega, vega * damp);
    });
    run("heston::no_static_arbitrage", [] {
        const HestonParams sets[] = {{0.04, 2.0, 0.04, 0.3, -0.7}, {0.09, 1.0, 0.09, 0.8, -0.5}, {0.04, 0.5, 0.04, 0.5, -0.7}};
        const double s = 100.0, r = 0.03, q = 0.0;
        for (const auto& p : sets)
            for (double t : {0.02, 0.1, 0.25, 0.5, 1.0, 2.0}) {
                const double cap = s * std::exp(-q * t);
                double prev = INFINITY;
                for (double k : {70.0, 85.0, 100.0, 115.0, 130.0, 150.0, 200.0}) {
                    const double c = heston_price(s, k, t, r, q, p, OptionType::Call);
                    const double intrinsic = std::fmax(s * std::exp(-q * t) - k * std::exp(-r * t), 0.0);
                    EXPECT(c >= intrinsic - 1e-4, "call %g < intrinsic %g (T=%g K=%g)", c, intrinsic, t, k);
                    EXPECT(c <= cap + 1e-4, "call %g > spot cap %g (T=%g K=%g)", c, cap, t, k);
                    EXPECT(c <= prev + 1e-4, "call not monotone in K (T=%g K=%g)", t, k);
                    prev = c;
                }
            }
    });
    run("heston::zero_vol_of_vol_matches_bsm", [] {
        const HestonParams p{0.04, 1.0, 0.04, 1e-4, 0.0};
        for (double t : {0.25, 1.0, 2.0})
            for (double k : {70.0, 85.0, 100.0, 115.0, 130.0}) {
                const double h = heston_price(100.0, k, t, 0.03, 0.0, p, OptionType::Call);
                const double b = bsm_price(100.0, k, t, 0.03, 0.0, 0.2, OptionType::Call);
                EXPECT(std::fabs(h - b) < 0.02, "heston %.5f vs bsm %.5f (T=%g K=%g)", h, b, t, k);
            }
    });
    // ----------------------------------------------------------------- bates.rs
    run("bates::recovers_heston_no_jumps", [] {
        const BatesParams bp{params(), 0.0, 0.0, 1e-8};
        const double b = bates_price(100.0, 100.0, 1.0, 0.05, 0.0, bp, OptionType::Call);
        const double h = heston_price(100.0, 100.0, 1.0, 0.05, 0.0, params(), OptionType::Call);
        EXPECT(std::fabs(b - h) < 0.02, "bates=%.4f heston=%.4f", b, h);
    });
    run("bates::put_call_parity", [] {
        const auto bp = bp_with_jumps();
        const double call = bates_price(100.0, 100.0, 0.5, 0.03, 0.0, bp, OptionType::Call);
        const double put = bates_price(100.0, 100.0, 0.5, 0.03, 0.0, bp, OptionType::Put);
        EXPECT(std::fabs(call - put - (100.0 - 100.0 * std::exp(-0.03 * 0.5))) < 0.02, "parity");
    });
    run("bates::greeks_signs", [] {
        const auto r = bates_price_and_greeks(100.0, 100.0, 1.0, 0.05, 0.0, bp_with_jumps(), OptionType::Call);
        EXPECT(r.delta > 0.0 && r.delta < 1.0 && r.gamma > 0.0 && r.vega > 0.0 && r.rho > 0.0, "signs");
    });
    run("bates::greeks_put_delta_negative", [] {
        const auto r = bates_price_and_greeks(100.0, 100.0, 1.0, 0.05, 0.0, bp_with_jumps(), OptionType::Put);
        EXPECT(r.delta < 0.0 && r.delta > -1.0 && r.gamma > 0.0, "put delta=%g", r.delta);
    });
    run("bates::greeks_match_heston_no_jumps", [] {
        const BatesParams bp{params(), 0.0, 0.0, 1e-8};
        const auto b = bates_price_and_greeks(100.0, 100.0, 1.0, 0.05, 0.0, bp, OptionType::Call);
        const auto h = heston_price_and_greeks(100.0, 100.0, 1.0, 0.05, 0.0, params(), OptionType::Call);
        EXPECT(std::fabs(b.delta - h.delta) < 0.01, "delta: bates=%.4f heston=%.4f", b.delta, h.delta);
        EXPECT(std::fabs(b.vega - h.vega) < 1.0, "vega: bates=%.4f heston=%.4f", b.vega, h.vega);
    });
    run("bates::no_static_arbitrage", [] {
        const BatesParams sets[] = {{params(), 0.5, -0.1, 0.15}, {{0.09, 1.0, 0.09, 0.8, -0.5}, 1.0, -0.2, 0.25}};
        const double s = 100.0, r = 0.03, q = 0.0;
        for (const auto& bp : sets)
            for (double t : {0.02, 0.1, 0.25, 0.5, 1.0, 2.0}) {
                const double cap = s * std::exp(-q * t);
                double prev = INFINITY;
                for (double k : {70.0, 85.0, 100.0, 115.0, 130.0, 150.0, 200.0}) {
                    const double c = bates_price(s, k, t, r, q, bp, OptionType::Call);
                    const double intrinsic = std::fmax(s * std::exp(-q * t) - k * std::exp(-r * t), 0.0);
                    EXPECT(c >= intrinsic - 1e-4 && c <= cap + 1e-4 && c <= prev + 1e-4, "T=%g K=%g c=%g", t, k, c);
                    prev = c;
                }
            }
    });
    // ----------------------------------------------------------------- batch.rs
    run("batch::iv_roundtrip", [] {
        auto c = chain(10);
        std::vector<double> prices;
        for (const auto& x : c) prices.push_back(bsm_price(x.spot, x.strike, x.expiry, x.rate, x.div_yield, x.vol, x.opt_type));
        const auto ivs = batch_implied_vol(c, prices);
        for (size_t i = 0; i < c.size(); ++i) {
            EXPECT(ivs[i].has_value(), "solver bailed");
            EXPECT(std::fabs(*ivs[i] - c[i].vol) < 1e-6, "got %.8f", *ivs[i]);
        }
    });
    run("batch::batch_heston_greeks_matches_scalar", [] {
        const auto c = chain(15);
        const auto out = batch_heston_greeks(c, params());
        for (size_t i = 0; i < c.size(); ++i) {
            const auto s = heston_price_and_greeks(c[i].spot, c[i].strike, c[i].expiry, c[i].rate, c[i].div_yield,
                                                   params(), c[i].opt_type);
            EXPECT(std::fabs(out[i].price - s.price) < 1e-12 && std::fabs(out[i].delta - s.delta) < 1e-12 &&
                       std::fabs(out[i].vega - s.vega) < 1e-12 && std::fabs(out[i].vanna - s.vanna) < 1e-12,
                   "mismatch at %zu", i);
        }
    });
    run("batch::batch_bates_greeks_matches_scalar", [] {
        const auto c = chain(15);
        const auto out = batch_bates_greeks(c, bp_with_jumps());
        for (size_t i = 0; i < c.size(); ++i) {
            const auto s = bates_price_and_greeks(c[i].spot, c[i].strike, c[i].expiry, c[i].rate, c[i].div_yield,
                                                  bp_with_jumps(), c[i].opt_type);
            EXPECT(std::fabs(out[i].price - s.price) < 1e-12 && std::fabs(out[i].delta - s.delta) < 1e-12 &&
                       std::fabs(out[i].vega - s.vega) < 1e-12, "mismatch at %zu", i);
        }
    });
    run("batch::batch_heston_price_matches_batch_heston_greeks", [] {
        const auto c = chain(12);
        const auto px = batch_heston(c, params());
        const auto g = batch_heston_greeks(c, params());
        for (size_t i = 0; i < c.size(); ++i) EXPECT(std::fabs(px[i] - g[i].price) < 1e-12, "at %zu", i);
    });
    // ----------------------------------------------------------- calibration.rs
    auto make_quotes = [](bool bates, const BatesParams& bp, std::vector<OptionContract>& store) {
        store.clear();
        std::vector<double> ivs;
        for (double t : {0.25, 0.5, 1.0})
            for (double k : {80.0, 90.0, 95.0, 100.0, 105.0, 110.0, 120.0}) {
                const OptionType ot = k >= 100.0 ? OptionType::Call : OptionType::Put;
                const double px = bates ? bates_price(100.0, k, t, 0.03, 0.0, bp, ot)
                                        : heston_price(100.0, k, t, 0.03, 0.0, bp.heston, ot);
                store.push_back(OptionContract{100.0, k, t, 0.03, 0.0, 0.2, ot});
                ivs.push_back(px);
            }
        const auto iv = batch_implied_vol(store, ivs);
        std::vector<OptionContract> kept;
        std::vector<double> kept_iv;
        for (size_t i = 0; i < store.size(); ++i)
            if (iv[i] && *iv[i] > 0.01 && *iv[i] < 2.0) { kept.push_back(store[i]); kept_iv.push_back(*iv[i]); }
        store = kept;
        return kept_iv;
    };
    run("calibration::recovers_params_from_synthetic_surface", [&] {
        std::vector<OptionContract> store;
        const HestonParams truth{0.04, 2.0, 0.04, 0.3, -0.5};
        const auto iv = make_quotes(false, BatesParams{truth, 0, 0, 0}, store);
        std::vector<CalibInput> q;
        for (size_t i = 0; i < store.size(); ++i) q.push_back(CalibInput{&store[i], iv[i], 1.0});
        const auto res = calibrate_heston(q, HestonParams{0.05, 1.5, 0.05, 0.4, -0.3});
        EXPECT(res.converged, "did not converge after %d iters", res.iters);
        EXPECT(res.rmse < 0.005, "rmse=%g", res.rmse);
        EXPECT(std::fabs(res.params[0] - truth.v0) < 0.005, "v0 off");
        EXPECT(std::fabs(res.params[4] - truth.rho) < 0.05, "rho off");
        EXPECT(2.0 * res.params[1] * res.params[2] > res.params[3] * res.params[3], "Feller violated");
    });
    run("calibration::recovers_bates_params_from_synthetic_surface", [&] {
        std::vector<OptionContract> store;
        const BatesParams truth{{0.04, 2.0, 0.04, 0.3, -0.5}, 0.5, -0.1, 0.15};
        const auto iv = make_quotes(true, truth, store);
        std::vector<CalibInput> q;
        for (size_t i = 0; i < store.size(); ++i) q.push_back(CalibInput{&store[i], iv[i], 1.0});
        const auto res = calibrate_bates(q, BatesParams{{0.05, 1.5, 0.05, 0.4, -0.3}, 0.3, -0.05, 0.1});
        EXPECT(res.converged, "did not converge after %d iters", res.iters);
        EXPECT(res.rmse < 0.01, "rmse=%g", res.rmse);
        EXPECT(std::fabs(res.params[0] - 0.04) < 0.01, "v0 off");
    });
    auto quotes_of = [](const std::vector<OptionContract>& store, const std::vector<double>& iv) {
        std::vector<CalibInput> q;
        for (size_t i = 0; i < store.size(); ++i) q.push_back(CalibInput{&store[i], iv[i], 1.0});
        return q;
    };
    const BatesParams truth_b{{0.04, 2.0, 0.04, 0.3, -0.5}, 0.5, -0.1, 0.15};
    std::vector<OptionContract> store_h, store_b;
    const auto iv_h = make_quotes(false, truth_b, store_h);
    const auto iv_b = make_quotes(true, truth_b, store_b);
    run("calibration::regularization_recovers_plausible_params_in_the_degenerate_case", [&] {
        const BatesParams prior{{0.035, 1.8, 0.04, 0.35, -0.45}, 0.4, -0.08, 0.12};
        const auto reg = calibrate_bates_global_regularized(quotes_of(store_b, iv_b), 60, 80, 999, prior, 1e-3);
        EXPECT(reg.best.rmse < 0.005, "rmse=%g", reg.best.rmse);
        EXPECT(std::isfinite(reg.best.condition_number) && reg.best.condition_number < 1e9, "cond=%g",
               reg.best.condition_number);
        const auto& p = reg.best.params;
        EXPECT(std::fabs(p[0] - 0.04) < 0.01, "v0=%g", p[0]);
        EXPECT(std::fabs(p[1] - 2.0) < 0.5, "kappa=%g", p[1]);
        EXPECT(std::fabs(p[5] - 0.5) < 0.15, "lambda=%g", p[5]);
        EXPECT(std::fabs(p[6] + 0.1) < 0.05, "mu_j=%g", p[6]);
        EXPECT(std::fabs(p[7] - 0.15) < 0.05, "sigma_j=%g", p[7]);
    });
    run("calibration::regularization_does_not_hurt_a_well_identified_case", [&] {
        const auto q = quotes_of(store_h, iv_h);
        const HestonParams p0{0.05, 1.5, 0.05, 0.4, -0.3};
        const auto unreg = calibrate_heston(q, p0);
        const auto reg = calibrate_heston_regularized(q, p0, HestonParams{0.045, 1.8, 0.045, 0.32, -0.45}, 1e-3);
        EXPECT(reg.rmse < 0.002, "rmse=%g", reg.rmse);
        EXPECT(std::fabs(reg.params[0] - unreg.params[0]) < 0.005, "v0 drifted");
    });
    run("calibration::condition_number_flags_the_degenerate_bates_case", [&] {
        const auto h = calibrate_heston(quotes_of(store_h, iv_h), HestonParams{0.05, 1.5, 0.05, 0.4, -0.3});
        EXPECT(std::isfinite(h.condition_number) && h.condition_number < 1e9, "cond=%g", h.condition_number);
        const auto qb = quotes_of(store_b, iv_b);
        const auto good = calibrate_bates(qb, BatesParams{{0.05, 1.5, 0.05, 0.4, -0.3}, 0.3, -0.05, 0.1});
        EXPECT(std::isfinite(good.condition_number), "good p0 degenerate");
        const auto de = calibrate_bates_global(qb, 60, 80, 999);
        EXPECT(de.best.condition_number > 1e10 || !std::isfinite(de.best.condition_number), "cond=%g",
               de.best.condition_number);
        EXPECT(de.best.condition_number > 100.0 * good.condition_number, "de=%g good=%g", de.best.condition_number,
               good.condition_number);
    });
    run("calibration::de_global_recovers_heston_params_without_any_initial_guess", [&] {
        const auto res = calibrate_heston_global(quotes_of(store_h, iv_h), 40, 60, 777);
        const auto& p = res.best.params;
        EXPECT(res.best.rmse < 0.01, "rmse=%g", res.best.rmse);
        EXPECT(std::fabs(p[0] - 0.04) < 0.01, "v0 off: %g", p[0]);
        EXPECT(std::fabs(p[4] + 0.5) < 0.1, "rho off: %g", p[4]);
        EXPECT(2.0 * p[1] * p[2] > p[3] * p[3], "Feller");
        const double de_rmse = std::sqrt(res.de_best_sse / (double)iv_h.size());
        EXPECT(res.best.rmse <= de_rmse + 1e-9, "polished=%g de_raw=%g", res.best.rmse, de_rmse);
    });
    run("calibration::de_global_bates_finds_an_excellent_fit_not_necessarily_the_true_params", [&] {
        const auto res = calibrate_bates_global(quotes_of(store_b, iv_b), 60, 80, 999);
        const auto& p = res.best.params;
        EXPECT(res.best.rmse < 0.005, "rmse=%g", res.best.rmse);
        EXPECT(2.0 * p[1] * p[2] > p[3] * p[3], "Feller");
        EXPECT(p[0] > 0.0 && p[5] >= 0.0, "sanity bounds");
    });
    run("calibration::multistart_beats_bad_single_start", [&] {
        const auto q = quotes_of(store_h, iv_h);
        const HestonParams bad{0.25, 6.0, 0.3, 0.15, 0.6};
        const auto single = calibrate_heston(q, bad);
        const auto multi = calibrate_heston_multistart(q, bad, 8, 12345);
        EXPECT(multi.n_converged >= 1, "no restart converged at all");
        EXPECT(multi.best.rmse <= single.rmse + 1e-9, "multistart=%g single=%g", multi.best.rmse, single.rmse);
        EXPECT(multi.best.rmse < 0.01, "rmse=%g", multi.best.rmse);
    });
    // ------------------------------------------------------------- error path
    run("errors::invalid_argument_throws", [] {
        bool threw = false;
        try {
            batch_implied_vol(chain(2), {1.0});
        } catch (const Error& e) {
            threw = e.status() == OPE_ERR_INVALID_ARG;
        }
        EXPECT(threw, "expected ope::Error(OPE_ERR_INVALID_ARG)");
    });
    std::printf("%s: %d failed\n", g_fail ? "FAILED" : "OK", g_fail);
    return g_fail ? 1 : 0;
}
