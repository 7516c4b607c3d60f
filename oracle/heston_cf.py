"""FP64 prices of European puts under the Heston model, by the characteristic function. Test infrastructure only.

The published method (Heston 1993, the probabilities P1, P2 by Fourier inversion), with the characteristic function
written in the form that stays on the principal branch of the complex logarithm (Albrecher, Mayer, Schoutens and
Tistaert 2007, "the little Heston trap"). The reference's finance bench prices its Heston batches against the same
closed form (bench/finance.py:72-90); this is a fresh restatement with scipy's adaptive quadrature.
"""
import math

import numpy as np
from scipy import integrate


def _cf(phi, s0, v0, kappa, theta, sigma, rho, r, T):
    """E[exp(i phi ln S_T)] under the risk-neutral Heston dynamics."""
    i = 1j
    a = kappa - rho * sigma * i * phi
    d = np.sqrt(a * a + sigma * sigma * (i * phi + phi * phi))
    g = (a - d) / (a + d)
    e = np.exp(-d * T)
    c = (kappa * theta / (sigma * sigma)) * ((a - d) * T - 2.0 * np.log((1.0 - g * e) / (1.0 - g)))
    dterm = (v0 / (sigma * sigma)) * (a - d) * (1.0 - e) / (1.0 - g * e)
    return np.exp(i * phi * (math.log(s0) + r * T) + c + dterm)


def put(s0, K, T, v0, kappa, theta, sigma, rho, r):
    """The European put (FP64)."""
    lnk = math.log(K)
    fwd = s0 * math.exp(r * T)

    def p1(phi):
        return (np.exp(-1j * phi * lnk) * _cf(phi - 1j, s0, v0, kappa, theta, sigma, rho, r, T) / (1j * phi * fwd)).real

    def p2(phi):
        return (np.exp(-1j * phi * lnk) * _cf(phi, s0, v0, kappa, theta, sigma, rho, r, T) / (1j * phi)).real

    i1 = integrate.quad(p1, 1e-10, 200.0, limit=400, epsabs=1e-12, epsrel=1e-12)[0]
    i2 = integrate.quad(p2, 1e-10, 200.0, limit=400, epsabs=1e-12, epsrel=1e-12)[0]
    P1 = 0.5 + i1 / math.pi
    P2 = 0.5 + i2 / math.pi
    call = s0 * P1 - K * math.exp(-r * T) * P2
    return call - s0 + K * math.exp(-r * T)


def black_scholes_put(s0, K, T, vol, r):
    """The Black-Scholes put, for the limit checks of the quadrature."""
    from scipy.stats import norm
    d1 = (math.log(s0 / K) + (r + 0.5 * vol * vol) * T) / (vol * math.sqrt(T))
    d2 = d1 - vol * math.sqrt(T)
    return K * math.exp(-r * T) * norm.cdf(-d2) - s0 * norm.cdf(-d1)
