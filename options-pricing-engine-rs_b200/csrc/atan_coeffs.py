"""Coefficients of atan2_node's polynomial (cf_device.cuh).

atan2_node reduces atan2(y, x) to atan(t) with |t| <= tan(pi/8): first to
q = min(|x|,|y|) / max(|x|,|y|) in [0, 1] (octant symmetry), then, for
q > tan(pi/8), to t = (q - 1)/(q + 1) with atan(q) = pi/4 + atan(t).  On that
interval atan(t) = t + t s P(s), s = t^2, where P approximates
f(s) = (atan(sqrt s)/sqrt s - 1)/s on [0, (sqrt 2 - 1)^2].  P is the degree-10
polynomial interpolating f at the 11 Chebyshev nodes of the interval,
computed here in 60-digit arithmetic (mpmath); its relative error on
atan(t) is 5e-18, far below the 1.1e-16 rounding unit.

Run: python atan_coeffs.py  (prints the coefficients, highest degree first,
in the form pasted into atan2_node, and the approximation error).
"""
import mpmath as mp

mp.mp.dps = 60
DEG = 10


def f(s):
    if s == 0:
        return mp.mpf(-1) / 3
    r = mp.sqrt(s)
    return (mp.atan(r) / r - 1) / s


def coefficients(deg=DEG):
    smax = (mp.sqrt(2) - 1) ** 2
    n = deg + 1
    xs = [smax / 2 * (1 - mp.cos(mp.pi * (k + mp.mpf(1) / 2) / n)) for k in range(n)]
    a = mp.matrix([[x ** j for j in range(n)] for x in xs])
    b = mp.matrix([f(x) for x in xs])
    c = mp.lu_solve(a, b)
    return [c[j] for j in range(n)], smax


def max_rel_error(c, smax, samples=4000):
    err = 0
    for i in range(1, samples + 1):
        s = smax * i / samples
        t = mp.sqrt(s)
        p = sum(c[j] * s ** j for j in range(len(c)))
        err = max(err, abs((t + t * s * p) / mp.atan(t) - 1))
    return err


if __name__ == "__main__":
    c, smax = coefficients()
    for j in reversed(range(len(c))):
        print(f"    {float(c[j])!r},  // s^{j}")
    print("max relative error on atan(t):", mp.nstr(max_rel_error(c, smax), 3))
