// Prices of the reference crate itself (options_pricing_engine, built from
// its own sources) for the contracts of tests/golden/ref_inputs.txt, one per
// line, through its public single-contract API (heston_price, heston.rs:61;
// bates_price, bates.rs:29; quadrature tolerance fixed at 1e-8, heston.rs:228).
// Input line: "heston|bates p0 .. p4|p7 ; spot strike expiry rate div_yield call|put".
// Output line: the price in Rust's shortest round-trip form.
use options_pricing_engine::{bates_price, heston_price, BatesParams, HestonParams, OptionType};
use std::io::{self, BufRead, Write};

fn main() {
    let stdin = io::stdin();
    let mut out = io::BufWriter::new(io::stdout());
    for line in stdin.lock().lines() {
        let line = line.expect("read");
        let line = line.trim();
        if line.is_empty() || line.starts_with('#') {
            continue;
        }
        let (lhs, rhs) = line.split_once(';').expect("';' between parameters and contract");
        let mut l = lhs.split_whitespace();
        let model = l.next().expect("model");
        let p: Vec<f64> = l.map(|x| x.parse().expect("parameter")).collect();
        let c: Vec<&str> = rhs.split_whitespace().collect();
        let f = |i: usize| -> f64 { c[i].parse().expect("contract field") };
        let ot = if c[5] == "put" { OptionType::Put } else { OptionType::Call };
        let h = HestonParams { v0: p[0], kappa: p[1], theta: p[2], sigma: p[3], rho: p[4] };
        let v = if model == "bates" {
            let b = BatesParams { heston: h, lambda: p[5], mu_j: p[6], sigma_j: p[7] };
            bates_price(f(0), f(1), f(2), f(3), f(4), &b, ot)
        } else {
            heston_price(f(0), f(1), f(2), f(3), f(4), &h, ot)
        };
        writeln!(out, "{}", v).expect("write");
    }
}
