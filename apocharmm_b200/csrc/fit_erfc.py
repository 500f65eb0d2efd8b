"""Fits the erfc approximation used by the direct-space kernel.

erfc(x) = exp(-x^2) * t * P(t),  t = 1 / (1 + p x),  P a polynomial of
degree K-1, the form of Hastings' approximation (Abramowitz & Stegun 7.1.26)
with coefficients refitted here for relative accuracy on 0 <= x <= XMAX,
the range kappa*r takes inside the cutoff.  Prints the coefficients in the
form pasted into nonbonded.cu and the maximum relative error.
"""
import numpy as np
from scipy.special import erfcx

XMAX, K = 6.0, 9
best = None
for p in np.linspace(0.2, 0.8, 121):
    x = np.linspace(0.0, XMAX, 20001)
    t = 1.0 / (1.0 + p * x)
    y = erfcx(x) / t                      # target for P(t)
    # relative-error weighting: minimise (P - y)/y
    A = np.vander(t, K, increasing=True) / y[:, None]
    c, *_ = np.linalg.lstsq(A, np.ones_like(y), rcond=None)
    rel = np.abs(np.polyval(c[::-1], t) * t / erfcx(x) - 1.0).max()
    if best is None or rel < best[0]:
        best = (rel, p, c)
rel, p, c = best
c32 = c.astype(np.float32)
x = np.linspace(0.0, XMAX, 200001)
t = (1.0 / (1.0 + np.float32(p) * x)).astype(np.float32)
approx = np.polyval(c32[::-1].astype(np.float64), t) * t
print(f"p = {p!r}")
print("coefficients (t^0 .. t^%d):" % (K - 1), ", ".join(f"{v:.9e}f" for v in c32))
print(f"max relative error (fp64 eval) {rel:.3e}; with fp32 coefficients {np.abs(approx / erfcx(x) - 1).max():.3e}")
