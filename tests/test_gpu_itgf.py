"""The reference's iterative gauge fixing, f/it_gauge_fixing.f, on the device
(lce_it_gauge_fixing, lce_it_landau_gauge) against the oracle's restatement:
single iterations in every form (as written, component corrected, ascent),
the reunitarised loop of f/landau_gauge.f, transform tracking, FP32."""
import numpy as np
import pytest

from oracle.oracle import Oracle, hot_config

pytestmark = pytest.mark.gpu
lce = pytest.importorskip("lceqcd_b200")
from lceqcd_b200 import Lattice, LceError  # noqa: E402

FORMS = [(False, False), (True, False), (False, True), (True, True)]
THERM = dict(beta=12.0, x=0.09, y=0.3)


def rel_err(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b))))


def flags(fix, asc):
    return (1 if fix else 0) | (2 if asc else 0)


def thermalised(L, sweeps=30, seed=5):
    o = Oracle(L, THERM["beta"], THERM["x"], THERM["y"], lam=1.7, limit_or=1e-10)
    o.set_fields(*hot_config(L, seed=seed))
    o.set_philox(seed + 2)
    for _ in range(sweeps):
        o.sweep(0)
    return o.get_fields()


@pytest.mark.parametrize("L", [(4, 4, 4), (6, 4, 8)])
@pytest.mark.parametrize("fix,asc", FORMS)
@pytest.mark.parametrize("step", [0.0, 0.2])
def test_single_iterations_fp64(L, fix, asc, step):
    """Three iterations of the subroutine (no reunitarisation) from a hot
    configuration; step 0 takes the context's alpha (0.9) like the reference."""
    u, a = hot_config(L, seed=21)
    o = Oracle(L, 9.0, 0.1, 0.45, lam=1.7, alpha=0.9, limit_or=1e-10)
    o.set_fields(u, a)
    o.landau_copy()
    g = Lattice(L, beta=9.0, x=0.1, y=0.45, precision="f64", lam=1.7, alpha=0.9, limit_or=1e-10)
    g.upload(u, a, which=1)
    for _ in range(3):
        do = o.it_gauge_fixing(step if step > 0 else 0.9, flags(fix, asc))
        dg = g.it_gauge_fixing(step, fix_component=fix, ascend=asc)
        assert abs(dg - do) <= 1e-12 * do
        uf, af = g.download(which=1, dtype=np.float64)
        uo, ao = o.get_fields(which=1)
        assert rel_err(uf, uo) < 1e-12 and rel_err(af, ao) < 1e-12


@pytest.mark.parametrize("fix,asc", [(True, True), (True, False)])
def test_loop_converges_like_the_oracle_fp64(fix, asc):
    L = (8, 8, 6)
    u, a = thermalised(L)
    o = Oracle(L, THERM["beta"], THERM["x"], THERM["y"], lam=1.7, limit_or=1e-10)
    o.set_fields(u, a)
    do, it_o = o.it_landau_gauge(0.3, flags(fix, asc), max_iters=5000)
    g = Lattice(L, **THERM, precision="f64", lam=1.7, limit_or=1e-10)
    g.upload(u, a)
    dg, it_g = g.it_landau_gauge(0.3, fix_component=fix, ascend=asc)
    assert it_g == it_o and dg <= 1e-10
    assert abs(dg - do) <= 1e-8 * do
    assert rel_err(g.download(which=1, dtype=np.float64)[0], o.get_fields(which=1)[0]) < 1e-10
    F = g.gauge_functional()
    assert abs(F - o.gauge_functional()) < 1e-12
    assert (F > 0) == asc


def test_loop_as_written_does_not_converge():
    """The component as written (f/it_gauge_fixing.f:110): the capped loop
    reports non-convergence and has followed the oracle's iterates."""
    L = (6, 6, 6)
    u, a = thermalised(L, sweeps=20, seed=8)
    o = Oracle(L, THERM["beta"], THERM["x"], THERM["y"], lam=1.7, limit_or=1e-10)
    o.set_fields(u, a)
    do, it_o = o.it_landau_gauge(0.1, 0, max_iters=20)
    g = Lattice(L, **THERM, precision="f64", lam=1.7, limit_or=1e-10)
    g.upload(u, a)
    with pytest.raises(LceError) as e:
        g.it_landau_gauge(0.1, max_iters=20)
    assert e.value.code == lce._lib.LCE_ERR_GF_NOT_CONVERGED
    assert it_o == 20 and do > 1e-3
    assert rel_err(g.download(which=1, dtype=np.float64)[0], o.get_fields(which=1)[0]) < 1e-10


@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32", 2e-5)])
def test_tracked_transform(precision, tol):
    L = (8, 6, 4)
    u, a = thermalised(L, sweeps=20, seed=11)
    g = Lattice(L, **THERM, precision=precision, lam=1.7, limit_or=1e-10)
    g.upload(u, a)
    da1, it = g.it_landau_gauge(0.3, fix_component=True, ascend=True, track=True)
    assert da1 <= 1e-10 and it > 5
    uf, af = g.download(which=1, dtype=np.float64)
    g.apply_transform()
    u2, a2 = g.download(which=1, dtype=np.float64)
    np.testing.assert_allclose(u2, uf, atol=100 * tol)
    np.testing.assert_allclose(a2, af, atol=100 * tol * max(1, np.abs(af).max()))


def test_fp32_against_fp64_oracle():
    L = (8, 8, 6)
    u, a = thermalised(L)
    o = Oracle(L, THERM["beta"], THERM["x"], THERM["y"], lam=1.7, limit_or=1e-10)
    o.set_fields(u, a)
    o.landau_copy()
    g = Lattice(L, **THERM, precision="f32", lam=1.7, limit_or=1e-10)
    g.upload(u, a, which=1)
    do = o.it_gauge_fixing(0.3, 3)
    dg = g.it_gauge_fixing(0.3, fix_component=True, ascend=True)
    assert abs(dg - do) <= 1e-5 * do
    assert rel_err(g.download(which=1, dtype=np.float64)[0], o.get_fields(which=1)[0]) < 2e-6
    o.set_fields(u, a)
    _, it_o = o.it_landau_gauge(0.3, 3, max_iters=5000)
    g.upload(u, a)
    dg, it_g = g.it_landau_gauge(0.3, fix_component=True, ascend=True)
    assert dg <= 1e-10 and abs(it_g - it_o) <= max(3, it_o // 10)


def test_invalid_flags():
    g = Lattice((4, 4, 4), precision="f64")
    g.init_unit()
    with pytest.raises(LceError):
        g._ck(g.lib.lce_it_gauge_fixing(g.h, 0, 0.1, 8, None))
    with pytest.raises(LceError):
        g._ck(g.lib.lce_it_landau_gauge(g.h, 0, 0.1, 16, None, None, 10))
