"""Kostrov circular expanding crack, analytic slip rate (cst/kostrov.py),
with the C constant of Dahlen (1974) eq. (44) by numerical integration."""
import numpy as np


def _cee_integrand(x, a2, b2):
    return ((x + 0.5 * b2) ** 2.0 - x * np.sqrt((x + b2) * (x + a2))) / ((x + 1.0) * (x + 1.0) * np.sqrt(x + b2))


def _cee_integral(a2, b2):
    import scipy.integrate
    return scipy.integrate.quad(_cee_integrand, 0.0, float('inf'), args=(a2, b2))[0]


def cee(a, b):
    """C for a = vrup / vp and b = vrup / vs (cst/kostrov.py:21-31)."""
    a2 = np.asarray(a) * a
    b2 = np.asarray(b) * b
    d = np.vectorize(_cee_integral)(a2, b2) + 0.25 * b2 * (b + np.arccos(b) / np.sqrt(1.0 - b2))
    return b * b2 / d


def slip_rate(rho, vp, vs, vrup, dtau, r, t, C=None):
    """Slip rate at hypocentral distance r and reduced time t (t = 0 at the
    rupture arrival) for density rho, wave speeds vp, vs, rupture speed vrup
    and stress drop dtau (cst/kostrov.py:34-48)."""
    t0 = r / vrup
    if C is None:
        C = cee(vrup / vp, vrup / vs)
    t = np.asarray(t)
    return C * dtau / (rho * vs) * (t + t0) / np.sqrt(t * (t + 2.0 * t0))
