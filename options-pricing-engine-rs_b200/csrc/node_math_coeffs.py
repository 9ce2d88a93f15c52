"""Coefficients of the node evaluation's own atan2 and log (cf_device.cuh:
atan2_node, log_node), computed in 60-digit arithmetic (mpmath).

atan2_node reduces atan2(y, x) to atan(t) with |t| <= tan(pi/8): first to
q = min(|x|,|y|) / max(|x|,|y|) in [0, 1] (octant symmetry), then, for
q > tan(pi/8), to t = (q - 1)/(q + 1) with atan(q) = pi/4 + atan(t).  There
atan(t) = t + t s P(s), s = t^2, where P is the degree-10 polynomial that
interpolates f(s) = (atan(sqrt s)/sqrt s - 1)/s at the 11 Chebyshev nodes of
[0, (sqrt 2 - 1)^2]: 5e-18 relative error on atan(t).

log_node writes v = 2^k m with m in [sqrt(1/2), sqrt(2)), so that
log v = k ln 2 + 2 atanh(s), s = (m - 1)/(m + 1), |s| <= 3 - 2 sqrt 2, and
2 atanh(s) = 2 s + s w R(w), w = s^2, where R is the degree-6 polynomial that
interpolates (2 atanh(s) - 2 s)/(s w) at the 7 Chebyshev nodes of
[0, (3 - 2 sqrt 2)^2]: 4.5e-18 relative error on log m.

Both are far below the 1.1e-16 rounding unit; the evaluation in double
precision then adds a few ulps (checked against CUDA's functions on the
device by ope_selftest_atan2 / ope_selftest_log and in numpy by
tests/test_node_math_cpu.py).

Run: python node_math_coeffs.py  (prints the coefficients, highest degree
first, as they appear in cf_device.cuh, and the approximation errors).
"""
import mpmath as mp

mp.mp.dps = 60
ATAN_DEG = 10
LOG_DEG = 6


def _chebyshev_interpolant(fn, hi, deg):
    n = deg + 1
    xs = [hi / 2 * (1 - mp.cos(mp.pi * (k + mp.mpf(1) / 2) / n)) for k in range(n)]
    a = mp.matrix([[x ** j for j in range(n)] for x in xs])
    b = mp.matrix([fn(x) for x in xs])
    c = mp.lu_solve(a, b)
    return [c[j] for j in range(n)]


def _atan_f(s):
    if s == 0:
        return mp.mpf(-1) / 3
    r = mp.sqrt(s)
    return (mp.atan(r) / r - 1) / s


def _log_r(w):
    if w == 0:
        return mp.mpf(2) / 3
    s = mp.sqrt(w)
    return (2 * mp.atanh(s) - 2 * s) / (s * w)


def atan_coefficients(deg=ATAN_DEG):
    """P(s), lowest degree first, and the interval end (sqrt 2 - 1)^2."""
    smax = (mp.sqrt(2) - 1) ** 2
    return _chebyshev_interpolant(_atan_f, smax, deg), smax


def log_coefficients(deg=LOG_DEG):
    """R(w), lowest degree first, and the interval end (3 - 2 sqrt 2)^2."""
    wmax = (3 - 2 * mp.sqrt(2)) ** 2
    return _chebyshev_interpolant(_log_r, wmax, deg), wmax


def _poly(c, x):
    return sum(c[j] * x ** j for j in range(len(c)))


def atan_error(c, smax, samples=2000):
    return max(abs((mp.sqrt(s) + mp.sqrt(s) * s * _poly(c, s)) / mp.atan(mp.sqrt(s)) - 1)
               for s in (smax * i / samples for i in range(1, samples + 1)))


def log_error(c, wmax, samples=2000):
    return max(abs((2 * mp.sqrt(w) + mp.sqrt(w) * w * _poly(c, w)) / (2 * mp.atanh(mp.sqrt(w))) - 1)
               for w in (wmax * i / samples for i in range(1, samples + 1)))


if __name__ == "__main__":
    for name, (c, hi), err in (("atan2_node P(s)", atan_coefficients(), atan_error),
                               ("log_node R(w)", log_coefficients(), log_error)):
        print(name)
        for j in reversed(range(len(c))):
            print(f"    {float(c[j])!r},  // ^{j}")
        print("  max relative error:", mp.nstr(err(c, hi), 3))
