"""Derived known answers for the oracle (the reference ships no golden vectors
beyond RANLUX, so these pin the restatement by physics identities):

* unit configuration (f/confget.f unitconf): staple = 4*1, plaquette = 1,
  Higgs force = 6*A, theta = 0 and one gauge-fixing iteration;
* gauge invariance: a random gauge transformation leaves the plaquette,
  Tr A^2, cos(4|A|) slices and the agauge/ahiggs updates' measured scalars
  unchanged, and gauge fixing drives theta below limit_or;
* testconf (f/confget.f:528-575): closed-form slice correlators;
* stream consumption: 29*V uniforms per sweep, RANLUX source == same numbers
  supplied as a stream; FP32 and FP64 builds agree to single precision.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, hot_config, random_gauge_transform, reference_stream, uniforms_per_sweep

LAT = [(4, 4, 4), (4, 6, 8), (6, 4, 2), (2, 2, 2)]


@pytest.mark.parametrize("L", LAT)
def test_unit_configuration(L):
    o = Oracle(L, 9.0, 0.1, 0.45)
    o.unitconf(1.0)
    for eo in range(2):
        for mu in range(3):
            o.staples(eo, mu)
            v = o.staple()[mu, eo]
            np.testing.assert_allclose(v, np.tile([4.0, 0, 0, 0], (o.nh, 1)), atol=1e-14)
    assert abs(o.plaquette() - 1.0) < 1e-14
    u, a = o.get_fields()
    a[:] = np.array([0.3, -0.2, 0.7])
    o.set_fields(u, a)
    o.a_force(0)
    np.testing.assert_allclose(o.force(), np.tile(6 * np.array([0.3, -0.2, 0.7]), (o.nh, 1)), atol=1e-13)
    o.landau_copy()
    assert o.theta_direct() < 1e-28
    da1, it = o.landau_gauge()
    assert it == 1 and da1 < 1e-28
    assert abs(o.gauge_functional() - 1.0) < 1e-14


@pytest.mark.parametrize("L", [(4, 4, 4), (4, 6, 8)])
def test_gauge_invariance(L):
    u, a = hot_config(L, seed=7)
    o1 = Oracle(L, 9.0, 0.1, 0.45)
    o1.set_fields(u, a)
    ug, ag = random_gauge_transform(u, a, L, seed=11)
    o2 = Oracle(L, 9.0, 0.1, 0.45)
    o2.set_fields(ug, ag)
    assert abs(o1.plaquette() - o2.plaquette()) < 1e-13
    s1, c1, m1 = o1.scalarcorr()
    s2, c2, m2 = o2.scalarcorr()
    np.testing.assert_allclose(s1, s2, rtol=1e-12)
    p1, q1, _ = o1.polyakov()
    p2, q2, _ = o2.polyakov()
    np.testing.assert_allclose(p1, p2, rtol=1e-12)
    # Higgs overrelaxation is deterministic up to the accept test, whose
    # Boltzmann ratio is gauge invariant: the update commutes with the gauge
    # transformation (heatbaths draw directions in a fixed frame and do not).
    stream = reference_stream(2 * o1.nh, seed=99)
    o1.set_stream(stream)
    o2.set_stream(stream)
    acc1, acc2 = o1.ahiggs3(1), o2.ahiggs3(1)
    assert acc1 == acc2
    m1, m2 = o1.meas(), o2.meas()
    for k in ("a2", "a4", "akin"):
        assert abs(m1[k] - m2[k]) < 1e-11 * max(1.0, abs(m1[k])), k
    u1, a1 = o1.get_fields()
    _, a1g = random_gauge_transform(u1, a1, L, seed=11)
    np.testing.assert_allclose(o2.get_fields()[1], a1g, atol=1e-12)


@pytest.mark.parametrize("mode,limit", [(0, 1e-14), (1, 1e-24)])
def test_gauge_fixing_of_pure_gauge(mode, limit):
    """A gauge transform of the unit configuration is fixed back to theta ~ 0
    and functional 1 (Landau gauge of a pure gauge).  The reference's
    acos(Re Omega) angle (mode 0) cannot resolve rotations below ~sqrt(eps)
    and stalls near theta ~ 1e-14 in FP64; the atan2 angle (mode 1) does not."""
    L = (6, 6, 6)
    o = Oracle(L, 9.0, 0.1, 0.45, lam=1.7, limit_or=limit)
    o.set_gf_angle(mode)
    o.unitconf(0.0)
    u, a = o.get_fields()
    ug, ag = random_gauge_transform(u, a, L, seed=3)
    o.set_fields(ug, ag)
    da1, it = o.landau_gauge(max_iters=5000)
    assert da1 <= limit and it < 500
    assert abs(o.gauge_functional() - 1.0) < 1e-12
    assert o.theta_direct() < 100 * limit


def test_acos_angle_stalls_where_atan2_converges():
    L = (6, 6, 6)
    res = {}
    for mode in (0, 1):
        o = Oracle(L, 9.0, 0.1, 0.45, lam=1.7, limit_or=1e-20)
        o.set_gf_angle(mode)
        o.unitconf(0.0)
        u, a = o.get_fields()
        o.set_fields(*random_gauge_transform(u, a, L, seed=3))
        res[mode] = o.landau_gauge(max_iters=400)
    assert res[0][1] == 400 and res[0][0] > 1e-16   # capped, stalled
    assert res[1][1] < 400 and res[1][0] <= 1e-20


def test_theta_matches_or_iteration_value():
    """da1 returned by an iteration is theta of U_f before that iteration's odd
    half-step (f/or_gauge_fixing1.f:153-158); the direct evaluation after the
    even half-step must agree on a fresh copy."""
    L = (4, 4, 6)
    u, a = hot_config(L, seed=5)
    o = Oracle(L, 9.0, 0.1, 0.45, lam=1.7)
    o.set_fields(u, a)
    o.landau_copy()
    d1 = o.or_gauge_fixing()
    assert d1 > 0
    o.u_f_renorm()
    d2 = o.or_gauge_fixing()
    assert d2 < d1


def test_testconf_correlators():
    L = (4, 4, 6)
    o = Oracle(L, 9.0, 0.1, 0.45)
    o.testconf()
    o.landau_copy()
    ca, cu, c3 = o.correlator()
    L3 = L[2]
    z = np.arange(L3)
    s = np.array([np.sum(z * ((z + d) % L3)) for d in range(L3)], float)
    np.testing.assert_allclose(ca, np.ones(L3), rtol=1e-14)
    np.testing.assert_allclose(cu, (1 + 4) * s / L3, rtol=1e-14)
    np.testing.assert_allclose(c3, 2 * 9 * s / L3, rtol=1e-14)
    np.testing.assert_allclose(o.meas2(), np.full(3, 1 / np.sqrt(3)), rtol=1e-14)


def test_stream_consumption_and_sources():
    L = (4, 4, 4)
    n = uniforms_per_sweep(L)
    u, a = hot_config(L, seed=1)
    o1 = Oracle(L, 9.0, 0.1, 0.45)
    o1.set_fields(u, a)
    stream = reference_stream(n + 10, seed=314159)
    o1.set_stream(stream)
    o1.sweep(1)
    assert o1.stream_pos() == n  # 29*V per sweep (f/main.f:38-41 composition)
    # RANLUX source consumed sequentially == the same numbers as a stream
    from oracle.oracle import Ranlux
    Ranlux().rluxgo(3, 314159)
    o2 = Oracle(L, 9.0, 0.1, 0.45)
    o2.set_fields(u, a)
    o2.set_ranlux()
    o2.sweep(1)
    np.testing.assert_array_equal(o1.get_fields()[0], o2.get_fields()[0])
    np.testing.assert_array_equal(o1.get_fields()[1], o2.get_fields()[1])
    # an exhausted stream is an error, not a silent reuse
    o3 = Oracle(L, 9.0, 0.1, 0.45)
    o3.set_fields(u, a)
    o3.set_stream(stream[:100])
    with pytest.raises(RuntimeError):
        o3.sweep(1)


def test_fp32_build_tracks_fp64():
    L = (4, 4, 4)
    u, a = hot_config(L, seed=2)
    stream = reference_stream(uniforms_per_sweep(L), seed=4242)
    o64 = Oracle(L, 12.0, 0.09, 0.3, bits=64)
    o32 = Oracle(L, 12.0, 0.09, 0.3, bits=32)
    o64.set_fields(u, a)
    o32.set_fields(u.astype(np.float32), a.astype(np.float32))
    o64.set_stream(stream)
    o32.set_stream(stream)
    o64.sweep(1)
    o32.sweep(1)
    u64, a64 = o64.get_fields()
    u32, a32 = o32.get_fields()
    # a handful of accept decisions may flip in single precision; the bulk agrees
    close = np.abs(u64 - u32).max(axis=-1) < 1e-4
    assert close.mean() > 0.95


def test_philox_source_is_order_independent():
    """Counter-based draws depend on (pass, site, slot) only: running with
    1 or 4 threads gives identical fields."""
    L = (6, 6, 6)
    u, a = hot_config(L, seed=9)
    res = []
    for th in (1, 4):
        o = Oracle(L, 9.0, 0.1, 0.45, threads=th)
        o.set_fields(u, a)
        o.set_philox(12345, 0)
        o.sweep(1)
        o.sweep(1)
        res.append(o.get_fields())
        assert o.pass_ctr() == 20
    np.testing.assert_array_equal(res[0][0], res[1][0])
    np.testing.assert_array_equal(res[0][1], res[1][1])


def test_ahiggs1_step_adaptation():
    L = (4, 4, 4)
    u, a = hot_config(L, seed=3)
    o = Oracle(L, 9.0, 0.1, 0.45)
    o.set_fields(u, a)
    o.set_philox(5, 0)
    acc, d = o.ahiggs1(10.0, 1)
    assert acc < 0.4 and abs(d - 10.0 * 0.8989669) < 1e-5
    acc, d2 = o.ahiggs1(0.01, 1)
    assert acc > 0.6 and abs(d2 - 0.01 * 1.1131241) < 1e-8


# ---- the reference's iterative gauge fixing, f/it_gauge_fixing.f

def _thermalised(L, sweeps=30, seed=5):
    o = Oracle(L, 12.0, 0.09, 0.3, lam=1.7, limit_or=1e-10)
    o.set_fields(*hot_config(L, seed=seed))
    o.set_philox(seed + 2)
    for _ in range(sweeps):
        o.sweep(0)
    return o.get_fields()


def test_it_gauge_fixing_unit_configuration():
    """g = 0 on the unit configuration: Omega = 1 (the sin(t)/t -> 1 limit
    where the reference divides 0 by 0), da1 = 0, fields unchanged."""
    o = Oracle((4, 4, 6), 9.0, 0.1, 0.45)
    o.unitconf(1.0)
    o.landau_copy()
    u, a = o.get_fields(0)
    for flags in range(4):
        assert o.it_gauge_fixing(1.0, flags) == 0.0
    uf, af = o.get_fields(1)
    np.testing.assert_array_equal(uf, u)
    np.testing.assert_allclose(af, a, atol=1e-15)


def test_it_gauge_fixing_forms():
    """On a thermalised 8^3 configuration: the corrected steepest ascent
    (flags 3) converges to the overrelaxed iteration's Landau gauge; the
    reference's sign (flags 1) ends at its Z2 mirror, functional -F; the
    second component as written at f/it_gauge_fixing.f:110 (flags 0) does not
    converge; steps above ~1/3 diverge."""
    L = (8, 8, 8)
    u, a = _thermalised(L)

    def run(step, flags, cap):
        o = Oracle(L, 12.0, 0.09, 0.3, lam=1.7, limit_or=1e-10)
        o.set_fields(u, a)
        da1, it = o.it_landau_gauge(step, flags, max_iters=cap)
        return da1, it, o.gauge_functional()

    o = Oracle(L, 12.0, 0.09, 0.3, lam=1.7, limit_or=1e-10)
    o.set_fields(u, a)
    o.landau_gauge(max_iters=20000)
    F = o.gauge_functional()
    da1, it, F3 = run(0.3, 3, 2000)
    assert da1 <= 1e-10 and it < 200 and abs(F3 - F) < 1e-6
    da1, it, F1 = run(0.3, 1, 2000)
    assert da1 <= 1e-10 and abs(F1 + F) < 1e-6
    da1, it, _ = run(0.1, 0, 1000)
    assert it == 1000 and da1 > 1e-3
    da1, it, _ = run(0.5, 3, 1000)
    assert it == 1000 and da1 > 1.0


def test_it_gauge_fixing_da1_is_theta_for_small_steps():
    """With the component corrected, |g|^2 is theta of the overrelaxed form
    (alpha = 1): for a negligible step da1 equals the direct evaluation."""
    L = (4, 6, 4)
    u, a = hot_config(L, seed=9)
    o = Oracle(L, 9.0, 0.1, 0.45, alpha=1.0)
    o.set_fields(u, a)
    o.landau_copy()
    th = o.theta_direct()
    da1 = o.it_gauge_fixing(1e-13, 1)
    assert abs(da1 - th) <= 1e-9 * th
