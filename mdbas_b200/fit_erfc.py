"""Derivation of the FP32 erfc used by the mixed-precision pair kernel.

Form (Abramowitz & Stegun 7.1.26, refitted here):

    erfc(x) ~= t * P(t) * exp(-x^2),   t = 1 / (1 + p x),   x in [0, 6],

with P of degree 7.  p and the coefficients minimise the maximum RELATIVE
error of t*P(t) against the scaled complementary error function
erfcx(x) = erfc(x) exp(x^2) (scipy.special.erfcx, FP64) on 20,001 points:
p by a bounded scalar search, the coefficients by Lawson's iteratively
reweighted least squares toward the minimax solution.  Running this script
prints the constants compiled into csrc/pair_fp32.cu and the fit's maximum
relative error (2.4e-8).
"""
import numpy as np
from scipy.optimize import minimize_scalar
from scipy.special import erfcx

X0, X1, DEG = 0.0, 6.0, 7


def fit(p, deg=DEG, iters=60):
    x = np.linspace(X0, X1, 20001)
    t = 1.0 / (1.0 + p * x)
    y = erfcx(x)
    a = np.stack([t ** (k + 1) for k in range(deg + 1)], 1)
    w = 1.0 / y
    for _ in range(iters):
        c, *_ = np.linalg.lstsq(a * w[:, None], y * w, rcond=None)
        err = (a @ c - y) / y
        w = w * (np.abs(err) + 1e-3 * np.abs(err).max()) ** 0.5
        w /= w.max() / (1.0 / y).max()
    err = (a @ c - y) / y
    return float(np.abs(err).max()), c


def main():
    res = minimize_scalar(lambda p: fit(p, DEG, 20)[0], bounds=(0.2, 1.5), method="bounded",
                          options={"xatol": 1e-5})
    e, c = fit(res.x, DEG, 120)
    print(f"p = {res.x:.9e}f")
    for k, v in enumerate(c):
        print(f"c{k} = {v:.9e}f")
    print(f"max relative error on [{X0}, {X1}]: {e:.3e}")


if __name__ == "__main__":
    main()
