"""Derives the single-precision erfc used by the real-space pair kernel (the coefficients of
`erfc_poly` and `pair_terms_x2` in pair_math.cuh).

erfc(x) = exp(-x^2) * erfcx(x), and erfcx is smooth and bounded on [0, inf), so it is fitted
as a degree-7 polynomial in t = 1 / (1 + p x), p = 0.46, over x in [0, 4.2] (alpha * cutoff
for Ewald tolerances down to ~1e-8), by iteratively reweighted least squares on the relative
error.  The fit itself is good to ~6e-8 relative; evaluated in float with Horner's rule it is
good to ~4e-7 relative.  This is our own fit of the mathematical function (scipy's erfcx as
the target), not a reproduction of any vendor library's constants.

Run:  python openmm-rs_b200/csrc/fit_erfc.py   (prints the coefficient table)
"""
import numpy as np
from scipy.special import erfcx

P = 0.46
DEGREE = 7
XMAX = 4.2


def fit(p=P, degree=DEGREE, xmax=XMAX):
    x = np.linspace(0.0, xmax, 20001)
    t = 1.0 / (1.0 + p * x)
    y = erfcx(x)
    v = np.vander(t, degree + 1, increasing=True)
    w = 1.0 / y
    c, *_ = np.linalg.lstsq(v * w[:, None], y * w, rcond=None)
    for _ in range(40):
        err = (v @ c - y) / y
        ww = w * (np.abs(err) / np.abs(err).max() + 0.05) ** 0.5
        c, *_ = np.linalg.lstsq(v * ww[:, None], y * ww, rcond=None)
    return c, float(np.abs((v @ c - y) / y).max())


if __name__ == "__main__":
    coef, err = fit()
    print(f"// p = {P}, degree {DEGREE}, max relative error of the fit {err:.3e}")
    for k, c in enumerate(coef):
        print(f"  {float(c)!r:>24}f,  // t^{k}")
