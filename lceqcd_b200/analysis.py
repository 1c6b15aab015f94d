"""Statistics of Monte Carlo time series: autocorrelation-corrected errors.

* tau_int: integrated autocorrelation time with the automatic window of
  Madras & Sokal (J. Stat. Phys. 50 (1988) 109): sum the normalised
  autocorrelation function up to the first W with W >= c * tau_int(W).
* mean_err: mean and its error sqrt(2 tau_int var / N).
* z_score: difference of two independent estimates in units of the combined
  error (the "within n sigma" test used to compare ensembles).
* effective_mass: cosh effective mass of a periodic correlator,
  m(z) = arccosh((C(z-1) + C(z+1)) / (2 C(z))).
"""
from __future__ import annotations

import numpy as np


def autocorrelation(x: np.ndarray) -> np.ndarray:
    x = np.asarray(x, np.float64)
    n = x.size
    d = x - x.mean()
    f = np.fft.rfft(d, 2 * n)
    acf = np.fft.irfft(f * np.conj(f))[:n] / np.arange(n, 0, -1)
    return acf / acf[0] if acf[0] > 0 else np.ones(n)


def tau_int(x: np.ndarray, c: float = 5.0) -> float:
    rho = autocorrelation(x)
    tau = 0.5
    for w in range(1, rho.size):
        tau += rho[w]
        if w >= c * tau:
            break
    return max(tau, 0.5)


def mean_err(x: np.ndarray, c: float = 5.0):
    x = np.asarray(x, np.float64)
    t = tau_int(x, c)
    return float(x.mean()), float(np.sqrt(2.0 * t * x.var(ddof=1) / x.size)), t


def z_score(a, b) -> float:
    (ma, ea), (mb, eb) = a[:2], b[:2]
    return float((ma - mb) / np.sqrt(ea * ea + eb * eb))


def effective_mass(corr: np.ndarray) -> np.ndarray:
    c = np.asarray(corr, np.float64)
    n = c.size
    out = np.full(n, np.nan)
    for z in range(1, n // 2):
        r = (c[z - 1] + c[z + 1]) / (2.0 * c[z])
        if r >= 1.0:
            out[z] = np.arccosh(r)
    return out


def jackknife(fn, samples: np.ndarray, nbins: int = 20):
    """Jackknife mean and error of fn(mean of samples) over nbins contiguous
    bins (bins long against the autocorrelation time keep the error honest).
    samples: [n, ...]; returns (estimate, error)."""
    x = np.asarray(samples, np.float64)
    n = (x.shape[0] // nbins) * nbins
    bins = x[:n].reshape((nbins, n // nbins) + x.shape[1:]).mean(axis=1)
    tot = bins.sum(axis=0)
    vals = np.array([fn((tot - bins[i]) / (nbins - 1)) for i in range(nbins)])
    est = fn(tot / nbins)
    err = np.sqrt((nbins - 1) / nbins * ((vals - vals.mean(axis=0)) ** 2).sum(axis=0))
    return est, err
