"""Autocorrelation analysis used by the ensemble comparisons (CPU only)."""
import numpy as np

from lceqcd_b200.analysis import effective_mass, mean_err, tau_int, z_score


def test_tau_int_of_white_noise_and_ar1():
    rng = np.random.default_rng(1)
    assert abs(tau_int(rng.standard_normal(20000)) - 0.5) < 0.1
    x = np.zeros(50000)
    for i in range(1, x.size):
        x[i] = 0.8 * x[i - 1] + rng.standard_normal()
    assert abs(tau_int(x) - 0.5 * (1 + 0.8) / (1 - 0.8)) < 1.0   # AR(1): (1+phi)/(2(1-phi)) = 4.5


def test_mean_err_and_z():
    rng = np.random.default_rng(2)
    a = mean_err(1.0 + rng.standard_normal(10000))
    b = mean_err(1.0 + rng.standard_normal(10000))
    assert abs(a[0] - 1.0) < 5 * a[1] and abs(z_score(a, b)) < 5


def test_effective_mass_of_cosh():
    n, m = 16, 0.3
    z = np.arange(n)
    c = np.cosh(m * (z - n / 2))
    np.testing.assert_allclose(effective_mass(c)[1:n // 2], m, rtol=1e-10)


def test_jackknife_mean_error_and_nonlinear_function():
    import numpy as np
    from lceqcd_b200.analysis import jackknife
    rng = np.random.default_rng(1)
    x = rng.normal(2.0, 1.0, size=(20000, 2))
    est, err = jackknife(lambda c: c[0], x, nbins=50)
    assert abs(est - 2.0) < 0.05 and 0.7 * 1 / np.sqrt(20000) < err < 1.3 / np.sqrt(20000)
    # ratio of means: error by propagation ~ sqrt(2) * sigma / (2 sqrt(n))
    est, err = jackknife(lambda c: c[0] / c[1], x, nbins=50)
    assert abs(est - 1.0) < 0.02 and 0.6 * np.sqrt(2) / 2 / np.sqrt(20000) < err < 1.5 * np.sqrt(2) / 2 / np.sqrt(20000)
