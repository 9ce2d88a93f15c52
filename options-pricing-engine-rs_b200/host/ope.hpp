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

namespace detail {
inline CalibResult calibrate(int model, const std::vector<CalibInput>& quotes, const std::vector<double>& p0) {
    if (quotes.empty()) throw Error(OPE_ERR_INVALID_ARG, "nothing to calibrate");  // calibration.rs:438
    std::vector<ope_contract> c;
    std::vector<double> iv, w;
    for (const auto& q : quotes) {
        c.push_back(to_c(*q.contract));
        iv.push_back(q.iv_market);
        w.push_back(q.weight);
    }
    const int64_t off[2] = {0, (int64_t)c.size()};
    ope_calib_result r;
    check(ope_calibrate_surfaces(model, c.data(), iv.data(), w.data(), c.size(), off, 1, p0.data(), &r, nullptr));
    const size_t dim = p0.size();
    return CalibResult{std::vector<double>(r.params, r.params + dim), r.rmse, r.max_err, r.iters,
                       r.converged != 0, r.early_stopped != 0, r.condition_number,
                       std::vector<double>(r.weakest_direction, r.weakest_direction + dim)};
}
}  // namespace detail

// calibration.rs:204-206
inline CalibResult calibrate_heston(const std::vector<CalibInput>& quotes, const HestonParams& p0) {
    return detail::calibrate(OPE_MODEL_HESTON, quotes, {p0.v0, p0.kappa, p0.theta, p0.sigma, p0.rho});
}

// calibration.rs:208-210
inline CalibResult calibrate_bates(const std::vector<CalibInput>& quotes, const BatesParams& p0) {
    return detail::calibrate(OPE_MODEL_BATES, quotes,
                             {p0.heston.v0, p0.heston.kappa, p0.heston.theta, p0.heston.sigma, p0.heston.rho,
                              p0.lambda, p0.mu_j, p0.sigma_j});
}

}  // namespace ope
