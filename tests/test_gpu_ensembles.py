"""Production ensembles against the CPU oracle's ensembles and the FP64 GPU
path: plaquette, <Tr A0^2>, Polyakov loop and the Tr A0^2 slice correlator
agree within autocorrelation-corrected errors (|z| < 3 per observable, so that
a run of several comparisons is not flaky; the z-scores are printed)."""
import numpy as np
import pytest

from lceqcd_b200.analysis import mean_err, tau_int, z_score
from oracle.oracle import Oracle, hot_config

pytestmark = pytest.mark.gpu
lce = pytest.importorskip("lceqcd_b200")
from lceqcd_b200 import Lattice  # noqa: E402

L = (8, 8, 8)
COUP = dict(beta=9.0, x=0.1, y=0.45)
NTHERM, NMEAS = 300, 3000


def gpu_series(precision: str, seed: int):
    g = Lattice(L, **COUP, precision=precision, seed=seed)
    g.init_unit(0.0)
    g.sweeps(NTHERM, 0)
    plaq, a2, pol, sc1 = [], [], [], []
    for _ in range(NMEAS):
        m = g.sweep(1)
        plaq.append(m["plaq"])
        a2.append(m["a2"])
        _, _, mean2 = g.polyakov()
        pol.append(np.sqrt(mean2))
        sc1.append(g.scalarcorr()[1][1])
    return {k: np.array(v) for k, v in dict(plaq=plaq, a2=a2, pol=pol, sc1=sc1).items()}


def oracle_series(seed: int):
    o = Oracle(L, COUP["beta"], COUP["x"], COUP["y"], bits=32, threads=4)
    o.unitconf(0.0)
    o.set_philox(seed, 0)
    for _ in range(NTHERM):
        o.sweep(0)
    plaq, a2, pol, sc1 = [], [], [], []
    for _ in range(NMEAS):
        m = o.sweep(1)
        plaq.append(m["plaq"])
        a2.append(m["a2"])
        _, _, mean2 = o.polyakov()
        pol.append(np.sqrt(mean2))
        sc1.append(o.scalarcorr()[1][1])
    return {k: np.array(v) for k, v in dict(plaq=plaq, a2=a2, pol=pol, sc1=sc1).items()}


@pytest.fixture(scope="module")
def series():
    return {"f32": gpu_series("f32", 11), "f64": gpu_series("f64", 12), "oracle": oracle_series(13)}


@pytest.mark.parametrize("other", ["oracle", "f64"])
@pytest.mark.parametrize("obs", ["plaq", "a2", "pol", "sc1"])
def test_fp32_ensemble_matches(series, other, obs):
    a = mean_err(series["f32"][obs])
    b = mean_err(series[other][obs])
    z = z_score(a, b)
    print(f"{obs}: f32 {a[0]:.6f}+-{a[1]:.6f} (tau {a[2]:.1f})  {other} {b[0]:.6f}+-{b[1]:.6f}  z={z:+.2f}")
    assert abs(z) < 3.0
