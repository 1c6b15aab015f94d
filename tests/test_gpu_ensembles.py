"""Production ensembles against the CPU oracle's ensembles and the FP64 GPU
path: plaquette, <Tr A0^2>, Polyakov loop and the Tr A0^2 slice correlator
agree within autocorrelation-corrected errors.  These are the secondary
comparisons (many observables, forms and precisions), held to |z| < 3 so
that the suite of them is not flaky; the 2-sigma comparison of the
production ensembles with the reference's CPU ensembles is
tests/test_gpu_reference_ensembles.py.  The z-scores are printed."""
import os

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


# ---- the plain-method workload: 16^3, beta 9.0, x 0.1, y 0.45, cold start
# (U = 1, A0 = 0); per sweep one link heatbath, 4 link overrelaxation steps,
# a Higgs Metropolis step whose step size f/ahiggs1.f tunes towards 50%
# acceptance and 2 Higgs overrelaxation steps; 200 + 1000 sweeps.  Composed
# from the single-routine entry points (lce_agauge, lce_link_or, lce_ahiggs1,
# lce_ahiggs3, lce_renorm) in that order, on the device and in the oracle.
L16 = (16, 16, 16)
N16T, N16M = 200, 1000


def composed_series(lat, polyakov):
    delta, accs = 0.5, []
    plaq, a2, pol = [], [], []
    for k in range(N16T + N16M):
        meas = 1 if k >= N16T else 0
        lat.agauge(meas)
        if meas:
            plaq.append(lat_meas(lat)["plaq"])
        for _ in range(4):
            lat.link_or(0)
        acc, delta = lat.ahiggs1(delta, 0)
        accs.append(acc)
        lat.ahiggs3(0)
        lat.ahiggs3(meas)
        lat.renorm()
        if meas:
            a2.append(lat_meas(lat)["a2"])
            pol.append(np.sqrt(polyakov(lat)))
    return {"plaq": np.array(plaq), "a2": np.array(a2), "pol": np.array(pol), "acc_metro": np.array(accs[N16T:])}


def lat_meas(lat):
    return lat.meas() if isinstance(lat, Oracle) else lat.meas1()


# three independent chains per side, Philox keys declared here once
COMPOSED_KEYS = {"f32": (21, 121, 221), "f64": (22, 122, 222), "oracle": (23, 123, 223)}


@pytest.fixture(scope="module")
def composed():
    out = {}
    for prec in ("f32", "f64"):
        out[prec] = []
        for seed in COMPOSED_KEYS[prec]:
            g = Lattice(L16, beta=9.0, x=0.1, y=0.45, precision=prec, seed=seed)
            g.init_unit(0.0)
            out[prec].append(composed_series(g, lambda h: h.polyakov()[2]))
            g.close()
    out["oracle"] = []
    for seed in COMPOSED_KEYS["oracle"]:
        o = Oracle(L16, 9.0, 0.1, 0.45, bits=64, threads=os.cpu_count() or 1)
        o.unitconf(0.0)
        o.set_philox(seed, 0)
        out["oracle"].append(composed_series(o, lambda h: h.polyakov()[2]))
    return out


def pooled(chains, obs):
    """Mean of the chains' means; error from their autocorrelation-corrected errors."""
    ests = [mean_err(c[obs]) for c in chains]
    return (float(np.mean([e[0] for e in ests])), float(np.sqrt(sum(e[1] ** 2 for e in ests)) / len(ests)),
            float(np.mean([e[2] for e in ests])))


@pytest.mark.parametrize("one,other", [("f32", "oracle"), ("f32", "f64"), ("f64", "oracle")])
@pytest.mark.parametrize("obs", ["plaq", "a2", "pol"])
def test_composed_sweep_ensemble_matches(composed, one, other, obs):
    a = pooled(composed[one], obs)
    b = pooled(composed[other], obs)
    z = z_score(a, b)
    print(f"{obs}: {one} {a[0]:.6f}+-{a[1]:.6f} (tau {a[2]:.1f})  {other} {b[0]:.6f}+-{b[1]:.6f}  z={z:+.2f}")
    assert abs(z) < 3.0


@pytest.mark.parametrize("obs", ["plaq", "a2", "pol"])
def test_composed_sweep_from_the_reference_init2_start(composed, obs):
    """The same workload from the reference's init = 2 cold start
    (f/confget.f unitconf: U = 1, A0 = (0, 0, 1)) thermalises to the
    ensemble of the A0 = 0 start (the FP64 run above)."""
    if "init2" not in composed:
        g = Lattice(L16, beta=9.0, x=0.1, y=0.45, precision="f32", seed=24)
        g.init_unit(1.0)
        composed["init2"] = [composed_series(g, lambda h: h.polyakov()[2])]
        g.close()
    a = pooled(composed["init2"], obs)
    b = pooled(composed["f64"], obs)
    z = z_score(a, b)
    print(f"{obs}: init2 f32 {a[0]:.6f}+-{a[1]:.6f}  A0=0 f64 {b[0]:.6f}+-{b[1]:.6f}  z={z:+.2f}")
    assert abs(z) < 3.0


def test_composed_sweep_metropolis_step_is_tuned(composed):
    """f/ahiggs1.f:117-123 rescales the step while |acceptance - 1/2| > 0.1."""
    for k in ("f32", "f64", "oracle"):
        for chain in composed[k]:
            acc = chain["acc_metro"]
            assert 0.35 < acc.mean() < 0.65, (k, acc.mean())


# ---- the mixed-precision single-chain workload: 64^3, beta 12, x 0.09,
# y 0.3, hot start, 500 sweeps (the headline sweep); FP32 fields with FP64
# reunitarisation and sums against the FP64 path, measured over the last
# 400 sweeps of two chains started alike
L64 = (64, 64, 64)


@pytest.fixture(scope="module")
def mixed64():
    out = {}
    for prec, seed in (("f32", 41), ("f64", 42)):
        g = Lattice(L64, beta=12.0, x=0.09, y=0.3, precision=prec, seed=seed)
        g.init_hot(seed)
        rows = [g.sweep(1) for _ in range(500)][100:]
        out[prec] = {k: np.array([r[k] for r in rows]) for k in ("plaq", "a2", "a4")}
        g.close()
    return out


@pytest.mark.parametrize("obs", ["plaq", "a2", "a4"])
def test_mixed_precision_64cubed_observables_match_fp64(mixed64, obs):
    a, b = mean_err(mixed64["f32"][obs]), mean_err(mixed64["f64"][obs])
    z = z_score(a, b)
    print(f"64^3 {obs}: f32 {a[0]:.7f}+-{a[1]:.7f} (tau {a[2]:.1f})  f64 {b[0]:.7f}+-{b[1]:.7f}  z={z:+.2f}")
    assert abs(z) < 3.0
