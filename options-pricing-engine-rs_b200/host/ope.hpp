// ope.hpp — C++ mirror of the reference crate's pricing API over the C ABI.
//
// Same names, argument order and meaning as the reference's public surface
// (lib.rs:18-35): heston_price / bates_price (heston.rs:61-72,
// bates.rs:29-39), batch_heston / batch_heston_greeks / batch_bates /
// batch_bates_greeks / batch_implied_vol (batch.rs:23-56),
// calibrate_heston / calibrate_bates (calibration.rs:204-210) and the
// records OptionType, OptionContract, PricingResult, HestonParams,
// BatesParams, CalibResult (types.rs, calibration.rs:44-68).  Where the
// reference panics (it has no Result on this path) this throws ope::Error
// carrying the C ABI status and message; there is no CPU fallback.  The
// quadrature tolerance is the reference's 1e-8 unless *_tol overloads are
// used.  Header-only: link against libope_b200.so.
#pragma once

#include <cstdint>
#include <optional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ope.h"

namespace ope {

class Error : public std::runtime_error {
   public:
    Error(int status, const std::string& what) : std::runtime_error(what), status_(status) {}
    int status() const { return status_; }

   private:
    int status_;
};

inline void check(int rc) {
    if (rc != OPE_OK) throw Error(rc, std::string("ope: ") + ope_last_error());
}

enum class OptionType : int32_t { Call = OPE_CALL, Put = OPE_PUT };  // types.rs:5-13

inline double sign(OptionType t) { return t == OptionType::Call ? 1.0 : -1.0; }

struct OptionContract {  // types.rs:16-25
    double spot, strike, expiry, rate, div_yield, vol;
    OptionType opt_type;
};

struct HestonParams {  // types.rs:48-63
    double v0, kappa, theta, sigma, rho;
    bool feller_ok() const { return 2.0 * kappa * theta > sigma * sigma; }
};

struct BatesParams {  // types.rs:66-72
    HestonParams heston;
    double lambda, mu_j, sigma_j;
};

using PricingResult = ope_pricing_result;  // types.rs:29-39 (same field order)

struct CalibInput {  // calibration.rs:38-42
    const OptionContract* contract;
    double iv_market;
    double weight;
};

struct CalibResult {  // calibration.rs:44-68
    std::vector<double> params;
    double rmse, max_err;
    int iters;
    bool converged, early_stopped;
    double condition_number;
    std::vector<double> weakest_direction;
};

namespace detail {
inline ope_contract to_c(const OptionContract& c) {
    return ope_contract{c.spot, c.strike, c.expiry, c.rate, c.div_yield, c.vol, static_cast<int32_t>(c.opt_type), 0};
}
inline std::vector<ope_contract> to_c(const std::vector<OptionContract>& v) {
    std::vector<ope_contract> out;
    out.reserve(v.size());
    for (const auto& c : v) out.push_back(to_c(c));
    return out;
}
inline ope_heston_params to_c(const HestonParams& p) { return ope_heston_params{p.v0, p.kappa, p.theta, p.sigma, p.rho}; }
inline ope_bates_params to_c(const BatesParams& p) {
    return ope_bates_params{to_c(p.heston), p.lambda, p.mu_j, p.sigma_j};
}
inline ope_options opts(double tol) { return ope_options{tol, 0u, 0u, nullptr}; }
}  // namespace detail

// heston.rs:61-72
inline double heston_price(double spot, double strike, double expiry, double rate, double div_yield,
                           const HestonParams& params, OptionType opt_type) {
    double out = 0.0;
    const ope_heston_params p = detail::to_c(params);
    check(ope_heston_price(spot, strike, expiry, rate, div_yield, &p, static_cast<int32_t>(opt_type), &out));
    return out;
}

// bates.rs:29-39
inline double bates_price(double spot, double strike, double expiry, double rate, double div_yield,
                          const BatesParams& params, OptionType opt_type) {
    double out = 0.0;
    const ope_bates_params p = detail::to_c(params);
    check(ope_bates_price(spot, strike, expiry, rate, div_yield, &p, static_cast<int32_t>(opt_type), &out));
    return out;
}

// batch.rs:23-27
inline std::vector<double> batch_heston(const std::vector<OptionContract>& contracts, const HestonParams& params,
                                        double tol = OPE_REF_TOL) {
    auto c = detail::to_c(contracts);
    const ope_heston_params p = detail::to_c(params);
    std::vector<double> out(c.size());
    const ope_options o = detail::opts(tol);
    check(ope_batch_price_ex(OPE_MODEL_HESTON, c.data(), c.size(), &p, out.data(), &o));
    return out;
}

// batch.rs:38-42
inline std::vector<double> batch_bates(const std::vector<OptionContract>& contracts, const BatesParams& params,
                                       double tol = OPE_REF_TOL) {
    auto c = detail::to_c(contracts);
    const ope_bates_params p = detail::to_c(params);
    std::vector<double> out(c.size());
    const ope_options o = detail::opts(tol);
    check(ope_batch_price_ex(OPE_MODEL_BATES, c.data(), c.size(), &p, out.data(), &o));
    return out;
}

// batch.rs:32-36 (greeks.rs:19-72)
inline std::vector<PricingResult> batch_heston_greeks(const std::vector<OptionContract>& contracts,
                                                      const HestonParams& params) {
    auto c = detail::to_c(contracts);
    const ope_heston_params p = detail::to_c(params);
    std::vector<PricingResult> out(c.size());
    check(ope_batch_heston_greeks(c.data(), c.size(), &p, out.data()));
    return out;
}

// batch.rs:44-48
inline std::vector<PricingResult> batch_bates_greeks(const std::vector<OptionContract>& contracts,
                                                     const BatesParams& params) {
    auto c = detail::to_c(contracts);
    const ope_bates_params p = detail::to_c(params);
    std::vector<PricingResult> out(c.size());
    check(ope_batch_bates_greeks(c.data(), c.size(), &p, out.data()));
    return out;
}

// heston.rs:74-80 / bates.rs:41-47: one contract's bump-and-reprice Greeks
inline PricingResult heston_price_and_greeks(double spot, double strike, double expiry, double rate, double div_yield,
                                             const HestonParams& params, OptionType opt_type) {
    return batch_heston_greeks({OptionContract{spot, strike, expiry, rate, div_yield, 0.0, opt_type}}, params)[0];
}
inline PricingResult bates_price_and_greeks(double spot, double strike, double expiry, double rate, double div_yield,
                                            const BatesParams& params, OptionType opt_type) {
    return batch_bates_greeks({OptionContract{spot, strike, expiry, rate, div_yield, 0.0, opt_type}}, params)[0];
}

// batch.rs:51-56 (None where the solver bails)
inline std::vector<std::optional<double>> batch_implied_vol(const std::vector<OptionContract>& contracts,
                                                            const std::vector<double>& market_prices) {
    if (contracts.size() != market_prices.size()) throw Error(OPE_ERR_INVALID_ARG, "length mismatch");
    auto c = detail::to_c(contracts);
    std::vector<double> iv(c.size());
    std::vector<int32_t> ok(c.size());
    check(ope_batch_implied_vol(c.data(), c.size(), market_prices.data(), iv.data(), ok.data(), nullptr));
    std::vector<std::optional<double>> out(c.size());
    for (size_t i = 0; i < c.size(); ++i)
        if (ok[i]) out[i] = iv[i];
    return out;
}

// ad.rs:736-795
inline PricingResult heston_greeks_ad(double spot, double strike, double expiry, double rate, double div_yield,
                                      const HestonParams& params, OptionType opt_type) {
    const ope_contract c{spot, strike, expiry, rate, div_yield, 0.0, static_cast<int32_t>(opt_type), 0};
    const double p[5] = {params.v0, params.kappa, params.theta, params.sigma, params.rho};
    PricingResult r;
    check(ope_batch_greeks_ad(OPE_MODEL_HESTON, &c, 1, p, &r, nullptr));
    return r;
}

// ad.rs:809-865
inline PricingResult bates_greeks_ad(double spot, double strike, double expiry, double rate, double div_yield,
                                     const HestonParams& heston, double lambda, double mu_j, double sigma_j,
                                     OptionType opt_type) {
    const ope_contract c{spot, strike, expiry, rate, div_yield, 0.0, static_cast<int32_t>(opt_type), 0};
    const double p[8] = {heston.v0, heston.kappa, heston.theta, heston.sigma, heston.rho, lambda, mu_j, sigma_j};
    PricingResult r;
    check(ope_batch_greeks_ad(OPE_MODEL_BATES, &c, 1, p, &r, nullptr));
    return r;
}

// All eight Greeks as exact derivatives (OPE_FLAG_ANALYTIC_GREEKS): the
// analytic S / r / T sensitivities ad.rs:751-763 leaves to finite differences,
// for many contracts under one parameter set (5 or 8 doubles by model).
inline std::vector<PricingResult> batch_greeks_analytic(int32_t model, const std::vector<OptionContract>& contracts,
                                                        const double* params, double tol = OPE_REF_TOL) {
    std::vector<PricingResult> out(contracts.size());
    if (contracts.empty()) return out;
    std::vector<ope_contract> c;
    c.reserve(contracts.size());
    for (const auto& k : contracts)
        c.push_back(ope_contract{k.spot, k.strike, k.expiry, k.rate, k.div_yield, k.vol,
                                 static_cast<int32_t>(k.opt_type), 0});
    ope_options o{tol, OPE_FLAG_ANALYTIC_GREEKS, 0, nullptr};
    check(ope_batch_greeks_ad(model, c.data(), c.size(), params, out.data(), &o));
    return out;
}

// ad.rs heston_greeks_ad5: the joint five-parameter pass returns what
// heston_greeks_ad returns (ad.rs:1295-1322), so it is the same computation.
inline PricingResult heston_greeks_ad5(double spot, double strike, double expiry, double rate, double div_yield,
                                       const HestonParams& params, OptionType opt_type) {
    return heston_greeks_ad(spot, strike, expiry, rate, div_yield, params, opt_type);
}

struct BatesJumpSensitivities {  // ad.rs:866-871
    double price, d_lambda, d_mu_j, d_sigma_j;
};

// ad.rs:882-895, through the reverse-mode adjoint
inline BatesJumpSensitivities bates_jump_sensitivities_ad(double spot, double strike, double expiry, double rate,
                                                          double div_yield, const HestonParams& heston, double lambda,
                                                          double mu_j, double sigma_j, OptionType opt_type) {
    const ope_contract c{spot, strike, expiry, rate, div_yield, 0.0, static_cast<int32_t>(opt_type), 0};
    const double p[8] = {heston.v0, heston.kappa, heston.theta, heston.sigma, heston.rho, lambda, mu_j, sigma_j};
    const int64_t off[2] = {0, 1};
    double price = 0.0, grad[8];
    check(ope_price_gradient_surfaces(OPE_MODEL_BATES, &c, 1, off, 1, p, &price, grad, nullptr));
    return BatesJumpSensitivities{price, grad[5], grad[6], grad[7]};
}

struct MultistartResult {  // calibration.rs:70-76
    CalibResult best;
    size_t n_restarts, n_converged, n_pruned;
};

struct GlobalCalibResult {  // calibration.rs:296-300
    CalibResult best;
    double de_best_sse;
    size_t de_generations;
};

namespace detail {
struct Quotes {
    std::vector<ope_contract> c;
    std::vector<double> iv, w;
    int64_t off[2];
    explicit Quotes(const std::vector<CalibInput>& quotes) {
        if (quotes.empty()) throw Error(OPE_ERR_INVALID_ARG, "nothing to calibrate");  // calibration.rs:438
        for (const auto& q : quotes) {
            c.push_back(to_c(*q.contract));
            iv.push_back(q.iv_market);
            w.push_back(q.weight);
        }
        off[0] = 0;
        off[1] = (int64_t)c.size();
    }
};
inline CalibResult from_c(const ope_calib_result& r, size_t dim) {
    return CalibResult{std::vector<double>(r.params, r.params + dim), r.rmse, r.max_err, r.iters,
                       r.converged != 0, r.early_stopped != 0, r.condition_number,
                       std::vector<double>(r.weakest_direction, r.weakest_direction + dim)};
}
inline std::vector<double> vec(const HestonParams& p) { return {p.v0, p.kappa, p.theta, p.sigma, p.rho}; }
inline std::vector<double> vec(const BatesParams& p) {
    return {p.heston.v0, p.heston.kappa, p.heston.theta, p.heston.sigma, p.heston.rho, p.lambda, p.mu_j, p.sigma_j};
}
inline CalibResult calibrate(int model, const std::vector<CalibInput>& quotes, const std::vector<double>& p0) {
    Quotes q(quotes);
    ope_calib_result r;
    check(ope_calibrate_surfaces(model, q.c.data(), q.iv.data(), q.w.data(), q.c.size(), q.off, 1, p0.data(), &r,
                                 nullptr));
    return from_c(r, p0.size());
}
inline CalibResult calibrate_reg(int model, const std::vector<CalibInput>& quotes, const std::vector<double>& p0,
                                 const std::vector<double>& prior, double reg_weight) {
    Quotes q(quotes);
    ope_calib_result r;
    check(ope_calibrate_surfaces_reg(model, q.c.data(), q.iv.data(), q.w.data(), q.c.size(), q.off, 1, p0.data(),
                                     prior.data(), &reg_weight, &r, nullptr));
    return from_c(r, p0.size());
}
inline MultistartResult multistart(int model, const std::vector<CalibInput>& quotes, const std::vector<double>& p0,
                                   size_t n_restarts, uint64_t seed) {
    Quotes q(quotes);
    ope_multistart_result r;
    check(ope_calibrate_multistart(model, q.c.data(), q.iv.data(), q.w.data(), q.c.size(), q.off, 1, p0.data(),
                                   (int32_t)n_restarts, seed, nullptr, &r, nullptr, nullptr));
    return MultistartResult{from_c(r.best, p0.size()), (size_t)r.n_restarts, (size_t)r.n_converged,
                            (size_t)r.n_pruned};
}
inline GlobalCalibResult global(int model, const std::vector<CalibInput>& quotes, size_t n_pop, size_t n_gen,
                                uint64_t seed, const std::vector<double>* prior, double reg_weight) {
    Quotes q(quotes);
    ope_global_result r;
    check(ope_calibrate_global(model, q.c.data(), q.iv.data(), q.w.data(), q.c.size(), q.off, 1, (int32_t)n_pop,
                               (int32_t)n_gen, seed, prior ? prior->data() : nullptr, prior ? &reg_weight : nullptr,
                               &r, nullptr));
    return GlobalCalibResult{from_c(r.best, model == OPE_MODEL_BATES ? 8 : 5), r.de_best_sse,
                             (size_t)r.de_generations};
}
}  // namespace detail

// calibration.rs:204-206
inline CalibResult calibrate_heston(const std::vector<CalibInput>& quotes, const HestonParams& p0) {
    return detail::calibrate(OPE_MODEL_HESTON, quotes, detail::vec(p0));
}

// calibration.rs:208-210
inline CalibResult calibrate_bates(const std::vector<CalibInput>& quotes, const BatesParams& p0) {
    return detail::calibrate(OPE_MODEL_BATES, quotes, detail::vec(p0));
}

// calibration.rs:220-224
inline CalibResult calibrate_heston_regularized(const std::vector<CalibInput>& quotes, const HestonParams& p0,
                                                const HestonParams& prior, double reg_weight) {
    return detail::calibrate_reg(OPE_MODEL_HESTON, quotes, detail::vec(p0), detail::vec(prior), reg_weight);
}

// calibration.rs:226-230
inline CalibResult calibrate_bates_regularized(const std::vector<CalibInput>& quotes, const BatesParams& p0,
                                               const BatesParams& prior, double reg_weight) {
    return detail::calibrate_reg(OPE_MODEL_BATES, quotes, detail::vec(p0), detail::vec(prior), reg_weight);
}

// calibration.rs:246-250
inline MultistartResult calibrate_heston_multistart(const std::vector<CalibInput>& quotes, const HestonParams& p0,
                                                    size_t n_restarts, uint64_t seed) {
    return detail::multistart(OPE_MODEL_HESTON, quotes, detail::vec(p0), n_restarts, seed);
}

// calibration.rs:252-256
inline MultistartResult calibrate_bates_multistart(const std::vector<CalibInput>& quotes, const BatesParams& p0,
                                                   size_t n_restarts, uint64_t seed) {
    return detail::multistart(OPE_MODEL_BATES, quotes, detail::vec(p0), n_restarts, seed);
}

// calibration.rs:316-320
inline GlobalCalibResult calibrate_heston_global(const std::vector<CalibInput>& quotes, size_t n_pop, size_t n_gen,
                                                 uint64_t seed) {
    return detail::global(OPE_MODEL_HESTON, quotes, n_pop, n_gen, seed, nullptr, 0.0);
}

// calibration.rs:322-326
inline GlobalCalibResult calibrate_bates_global(const std::vector<CalibInput>& quotes, size_t n_pop, size_t n_gen,
                                                uint64_t seed) {
    return detail::global(OPE_MODEL_BATES, quotes, n_pop, n_gen, seed, nullptr, 0.0);
}

// calibration.rs:335-340
inline GlobalCalibResult calibrate_heston_global_regularized(const std::vector<CalibInput>& quotes, size_t n_pop,
                                                             size_t n_gen, uint64_t seed, const HestonParams& prior,
                                                             double reg_weight) {
    const auto pr = detail::vec(prior);
    return detail::global(OPE_MODEL_HESTON, quotes, n_pop, n_gen, seed, &pr, reg_weight);
}

// calibration.rs:342-347
inline GlobalCalibResult calibrate_bates_global_regularized(const std::vector<CalibInput>& quotes, size_t n_pop,
                                                            size_t n_gen, uint64_t seed, const BatesParams& prior,
                                                            double reg_weight) {
    const auto pr = detail::vec(prior);
    return detail::global(OPE_MODEL_BATES, quotes, n_pop, n_gen, seed, &pr, reg_weight);
}

}  // namespace ope
