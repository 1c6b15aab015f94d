"""GPU parity tests: the CUDA path through the C ABI against the CPU oracle.

FP64 validation mode consumes the host-supplied RANLUX stream in the
reference's consumption order (29*V uniforms per sweep) and must reproduce
the oracle to 1e-12 relative (the tolerance stated for the plain FP64 path);
the FP32 production path is compared with the FP32 oracle drawing the same
Philox stream, within single-precision tolerance.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle, hot_config, random_gauge_transform, reference_stream, uniforms_per_sweep

pytestmark = pytest.mark.gpu
lce = pytest.importorskip("lceqcd_b200")
from lceqcd_b200 import Ensemble, LceError, Lattice, Params  # noqa: E402

TOL64 = 1e-12
LATS = [(4, 4, 4), (4, 6, 8), (6, 4, 2), (2, 2, 2), (8, 8, 8)]
COUP = dict(beta=9.0, x=0.1, y=0.45)


def rel_err(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b))))


def pair(L, seed=1, rng="stream", precision="f64", **kw):
    u, a = hot_config(L, seed=seed)
    o = Oracle(L, COUP["beta"], COUP["x"], COUP["y"], lam=kw.get("lam", 1.8), alpha=kw.get("alpha", 1.0),
               limit_or=kw.get("limit_or", 1e-9), imode=kw.get("imode", 0))
    o.set_fields(u, a)
    g = Lattice(L, **COUP, precision=precision, rng=rng, **kw)
    g.upload(u, a)
    return o, g, u, a


@pytest.mark.parametrize("L", LATS)
def test_staple_and_force(L):
    o, g, _, _ = pair(L, seed=3)
    for eo in range(2):
        for mu in range(3):
            o.staples(eo, mu)
            assert rel_err(g.debug_staple(eo, mu), o.staple()[mu, eo]) < TOL64
        o.a_force(eo)
        assert rel_err(g.debug_force(eo), o.force()) < TOL64


@pytest.mark.parametrize("L", LATS)
@pytest.mark.parametrize("imode", [0, 1])
def test_routines_fp64_stream(L, imode):
    """ahiggs2, ahiggs3, agauge, renorm called one by one (f/main.f:38-41)."""
    o, g, _, _ = pair(L, seed=5, imode=imode)
    stream = reference_stream(uniforms_per_sweep(L) + 7, seed=314159)
    o.set_stream(stream)
    g.set_rng_stream(stream)
    for name in ("ahiggs2", "ahiggs3", "agauge"):
        ao = getattr(o, name)(1)
        ag = getattr(g, name)(1)
        assert abs(ao - ag) < 1e-6, name  # accept rates are returned as REAL
        uo, a_o = o.get_fields()
        ug, a_g = g.download(dtype=np.float64)
        assert rel_err(a_g, a_o) < TOL64, name
        assert rel_err(ug, uo) < TOL64, name
        mo, mg = o.meas(), g.meas1()
        for k in ("plaq", "akin", "a2", "a4") if name == "agauge" else ("akin", "a2", "a4"):
            assert abs(mo[k] - mg[k]) <= TOL64 * max(1, abs(mo[k])), (name, k)
    o.renorm()
    g.renorm()
    assert rel_err(g.download(dtype=np.float64)[0], o.get_fields()[0]) < TOL64
    assert g.rng_position()[1] == o.stream_pos() == uniforms_per_sweep(L)


@pytest.mark.parametrize("L", [(4, 4, 4), (6, 4, 8)])
def test_fused_sweeps_fp64_stream(L):
    """lce_sweep (CUDA graph, reunitarisation fused into the link writer)
    against three reference sweeps."""
    o, g, _, _ = pair(L, seed=7)
    stream = reference_stream(3 * uniforms_per_sweep(L), seed=27182)
    o.set_stream(stream)
    g.set_rng_stream(stream)
    for _ in range(3):
        mo = o.sweep(1)
        mg = g.sweep(1)
        for k in ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or"):
            assert abs(mo[k] - mg[k]) <= 1e-11 * max(1, abs(mo[k])), k
    uo, ao = o.get_fields()
    ug, ag = g.download(dtype=np.float64)
    assert rel_err(ug, uo) < 1e-11 and rel_err(ag, ao) < 1e-11
    with pytest.raises(LceError) as e:  # the stream is used up
        g.sweep(1)
    assert e.value.code == lce._lib.LCE_ERR_STREAM


@pytest.mark.parametrize("L", [(4, 4, 4), (8, 6, 4)])
def test_philox_stream_matches_oracle(L):
    """The device Philox4x32-10 counters (site, call, pass) equal the oracle's."""
    o, g, _, _ = pair(L, seed=9, rng="philox")
    o.set_philox(12345, 0)
    for _ in range(2):
        o.sweep(1)
        g.sweep(1)
    assert g.rng_position()[0] == o.pass_ctr() == 20
    assert rel_err(g.download(dtype=np.float64)[0], o.get_fields()[0]) < 1e-11


def test_composed_routines_philox_match_oracle():
    """Single-routine calls in a composed order (agauge, 4 x link_or, ahiggs1,
    2 x ahiggs3, renorm) draw the same Philox uniforms as the oracle: FP64
    fields agree after every routine, and the pass counters match."""
    L = (4, 6, 4)
    o, g, _, _ = pair(L, seed=15, rng="philox")
    o.set_philox(12345, 0)
    do = dg = 0.5
    for _ in range(3):
        steps = [("agauge", ()), *[("link_or", ())] * 4, ("ahiggs1", None), ("ahiggs3", ()), ("ahiggs3", ()),
                 ("renorm", None)]
        for name, args in steps:
            if name == "ahiggs1":
                _, do = o.ahiggs1(do, 1)
                _, dg = g.ahiggs1(dg, 1)
            elif name == "renorm":
                o.renorm()
                g.renorm()
            else:
                getattr(o, name)(1)
                getattr(g, name)(1)
            uo, ao = o.get_fields()
            ug, ag = g.download(dtype=np.float64)
            assert rel_err(ug, uo) < 1e-11 and rel_err(ag, ao) < 1e-11, name
            assert g.rng_position()[0] == o.pass_ctr(), name


def test_ahiggs1_and_link_or_fp64():
    L = (4, 6, 4)
    o, g, _, _ = pair(L, seed=11)
    stream = reference_stream(10 * 2 * 4 * 48 + 6 * 48 * 2, seed=99)
    o.set_stream(stream)
    g.set_rng_stream(stream)
    for d0 in (0.75, 5.0, 0.0625):  # REAL step (f/ahiggs1.f:30): float-exact values
        ao, do = o.ahiggs1(d0, 1)
        ag, dg = g.ahiggs1(d0, 1)
        assert abs(ao - ag) < 1e-6 and abs(do - dg) < 1e-6 * d0
        assert rel_err(g.download(dtype=np.float64)[1], o.get_fields()[1]) < TOL64
    ao, ag = o.link_or(1), g.link_or(1)
    assert abs(ao - ag) < 1e-6
    assert rel_err(g.download(dtype=np.float64)[0], o.get_fields()[0]) < TOL64


@pytest.mark.parametrize("angle", ["acos", "atan2"])
@pytest.mark.parametrize("L", [(4, 4, 4), (6, 4, 8)])
def test_gauge_fixing_iterations_fp64(L, angle):
    o, g, _, _ = pair(L, seed=13, lam=1.7, alpha=0.9, limit_or=1e-30, gf_angle=angle)
    o.set_gf_angle(0 if angle == "acos" else 1)
    o.landau_copy()
    done = 0
    for k in (1, 4, 20):
        for _ in range(k):
            da1 = o.or_gauge_fixing()
            o.u_f_renorm()
        done += k
        # restart from U on the GPU and run `done` iterations
        with pytest.raises(LceError) as e:
            g.landau_gauge(max_iters=done)
        assert e.value.code == lce._lib.LCE_ERR_GF_NOT_CONVERGED
        uf, af = g.download(which=1, dtype=np.float64)
        uo, ao = o.get_fields(which=1)
        assert rel_err(uf, uo) < 1e-11 and rel_err(af, ao) < 1e-11
        assert abs(g.theta() - o.theta_direct()) <= 1e-10 * o.theta_direct() + 1e-20
        assert abs(g.gauge_functional() - o.gauge_functional()) < 1e-12


@pytest.mark.parametrize("angle,limit", [("acos", 1e-8), ("atan2", 1e-12)])
def test_gauge_fixing_convergence_fp64(angle, limit):
    L = (6, 6, 6)
    o, g, _, _ = pair(L, seed=17, lam=1.7, limit_or=limit, gf_angle=angle)
    o.set_gf_angle(0 if angle == "acos" else 1)
    da_o, it_o = o.landau_gauge(max_iters=20000)
    da_g, it_g = g.landau_gauge()
    assert it_o == it_g and da_g <= limit
    assert abs(da_o - da_g) <= 1e-9 * da_o
    ca, cu, c3 = o.correlator()
    ga, gu, g3, af = g.correlator()
    for x, y in ((ca, ga), (cu, gu), (c3, g3)):
        assert rel_err(y, x) < 1e-10
    np.testing.assert_allclose(af, o.meas2(), rtol=1e-9, atol=1e-13)


@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32", 2e-5)])
def test_tracked_transform_reproduces_fixed_fields(precision, tol):
    """With transform tracking, U_f = G U G^+ and A_f = G A G^+ at every step:
    re-applying the final G to (U, A) gives the gauge-fixed fields, and a
    restart from G is converged at once."""
    L = (8, 6, 4)
    g = Lattice(L, **COUP, precision=precision, lam=1.7, limit_or=1e-11)
    g.init_hot(5)
    th0, th, it = g.landau_gauge_from("identity")
    assert th <= 1e-11 and it > 5 and th0 > th
    uf, af = g.download(which=1, dtype=np.float64)
    # identity start tracks the same iteration as the plain gauge fixing
    h = Lattice(L, **COUP, precision=precision, lam=1.7, limit_or=1e-11)
    h.upload(*g.download(dtype=np.float64))
    h.landau_gauge()
    np.testing.assert_allclose(h.download(which=1, dtype=np.float64)[0], uf, atol=tol)
    g.apply_transform()
    u2, a2 = g.download(which=1, dtype=np.float64)
    np.testing.assert_allclose(u2, uf, atol=100 * tol)
    np.testing.assert_allclose(a2, af, atol=100 * tol * max(1, np.abs(af).max()))
    ts, th2, it2 = g.landau_gauge_from("transform")
    assert ts <= 1e-10 and it2 <= 2
    gt = g.get_transform()
    np.testing.assert_allclose(np.linalg.norm(gt, axis=-1), 1.0, atol=1e-6)
    g.set_transform(gt)
    np.testing.assert_array_equal(g.get_transform(), gt)


@pytest.mark.parametrize("L", [(4, 4, 6), (8, 4, 4)])
def test_measurements_fp64(L):
    o, g, u, a = pair(L, seed=19)
    o.landau_copy()
    g.upload(u, a, which=1)
    ca, cu, c3 = o.correlator()
    ga, gu, g3, af = g.correlator()
    for x, y in ((ca, ga), (cu, gu), (c3, g3)):
        assert rel_err(y, x) < TOL64
    assert rel_err(af, o.meas2()) < TOL64
    for f in ("polyakov", "scalarcorr"):
        so, co, mo = getattr(o, f)()
        sg, cg, mg = getattr(g, f)()
        assert rel_err(sg, so) < TOL64 and rel_err(cg, co) < TOL64 and abs(mo - mg) < TOL64 * max(1, abs(mo))
    assert abs(g.plaquette() - o.plaquette()) < TOL64
    assert abs(g.gauge_functional() - o.gauge_functional()) < TOL64
    assert abs(g.theta() - o.theta_direct()) < TOL64 * max(1, o.theta_direct())


def test_testconf_correlators_on_gpu():
    L = (4, 4, 6)
    o = Oracle(L, 9.0, 0.1, 0.45)
    o.testconf()
    o.landau_copy()
    u, a = o.get_fields()
    g = Lattice(L, **COUP, precision="f64")
    g.upload(u, a, which=1)
    for x, y in zip(o.correlator(), g.correlator()[:3]):
        assert rel_err(y, x) < TOL64


def test_fp32_production_tracks_fp32_oracle():
    """Same Philox stream, FP32 arithmetic on both sides: the bulk of the sites
    agree to single precision after two sweeps (a few accept decisions near
    threshold may differ) and the measured scalars agree closely."""
    L = (8, 8, 8)
    u, a = hot_config(L, seed=21, dtype=np.float32)
    o = Oracle(L, 12.0, 0.09, 0.3, bits=32)
    o.set_fields(u, a)
    o.set_philox(777, 0)
    g = Lattice(L, beta=12.0, x=0.09, y=0.3, precision="f32", seed=777)
    g.upload(u, a)
    for _ in range(2):
        mo = o.sweep(1)
        mg = g.sweep(1)
    for k in ("plaq", "a2", "akin"):
        assert abs(mo[k] - mg[k]) < 2e-3 * max(1, abs(mo[k])), k
    ug, ag = g.download()
    uo, ao = o.get_fields()
    close = np.abs(ug.astype(np.float64) - uo).max(axis=-1) < 1e-4
    assert close.mean() > 0.97


def test_batch_equals_single_chains():
    """A batched context of uneven chains reproduces each chain run alone, bit
    for bit (per-chain Philox keys, per-chain reductions)."""
    specs = [Params(L=(4, 4, 4), beta=9.0, x=0.1, y=0.45, seed=1),
             Params(L=(6, 4, 8), beta=12.0, x=0.09, y=0.3, seed=2),
             Params(L=(8, 8, 8), beta=16.0, x=0.08, y=0.2, seed=3, imode=1)]
    ens = Ensemble(specs)
    ens.init_hot(42)
    starts = [ens.download(chain=i) for i in range(3)]
    for _ in range(3):
        ens.sweep(1)
    mb = ens.meas_batch()
    for i, sp in enumerate(specs):
        g = Lattice(sp.L, beta=sp.beta, x=sp.x, y=sp.y, seed=sp.seed, imode=sp.imode)
        g.upload(*starts[i])
        for _ in range(3):
            ms = g.sweep(1)
        ub, ab = ens.download(chain=i)
        us, as_ = g.download()
        np.testing.assert_array_equal(ub, us)
        np.testing.assert_array_equal(ab, as_)
        for k in ("plaq", "a2", "acc_gauge"):
            assert mb[i][k] == ms[k]


@pytest.mark.parametrize("L", [(4, 4, 4), (16, 16, 16), (32, 16, 24)])
def test_persistent_sweep_equals_pass_kernels(L):
    """The cooperative persistent sweep kernel (one launch per sweep, grid
    barriers between passes) reproduces the per-pass kernel graph bit for bit."""
    res = []
    for mode in ("passes", "persistent"):
        g = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=99, sweep_mode=mode)
        g.init_hot(7)
        for mf in (1, 0, 1):
            g.sweeps(2, mf)
        m = g.meas1()
        assert g.sweep_mode() == mode
        res.append((g.download(), m, g.rng_position()))
    (u0, a0), m0, r0 = res[0]
    (u1, a1), m1, r1 = res[1]
    np.testing.assert_array_equal(u0, u1)
    np.testing.assert_array_equal(a0, a1)
    assert m0 == m1 and r0 == r1


def test_persistent_batch_and_autotune():
    # a batch shares one sweep composition: here with a link-OR hit and ahiggs1
    specs = [Params(L=(16, 16, 16), beta=6.0, x=0.1, y=0.1, seed=5, n_link_or=1, n_higgs_metro=1),
             Params(L=(8, 12, 6), beta=16.0, x=0.08, y=0.5, seed=6, n_link_or=1, n_higgs_metro=1, imode=1)]
    outs = []
    for mode in ("passes", "persistent", "auto"):
        ens = Ensemble([Params(**{**s.__dict__, "sweep_mode": mode}) for s in specs])
        ens.init_hot(3)
        ens.sweeps(40, 1)
        if mode == "auto":
            assert ens.sweep_mode() in ("passes", "passes2", "persistent", "direct")
        outs.append(([ens.download(chain=i) for i in range(2)], ens.meas_batch()))
    for o in outs[1:]:
        for i in range(2):
            np.testing.assert_array_equal(o[0][i][0], outs[0][0][i][0])
            np.testing.assert_array_equal(o[0][i][1], outs[0][0][i][1])
        # the autotuner may pick the two-sites-per-thread form, whose FP64
        # measurement sums run in another order
        for m0, m1 in zip(o[1], outs[0][1]):
            for k in m0:
                if k != "af":
                    assert abs(m0[k] - m1[k]) <= 1e-12 * max(1.0, abs(m1[k])), k


def test_persistent_fp64_stream_matches_oracle():
    L = (6, 4, 8)
    o, g, _, _ = pair(L, seed=33, sweep_mode="persistent")
    stream = reference_stream(2 * uniforms_per_sweep(L), seed=4711)
    o.set_stream(stream)
    g.set_rng_stream(stream)
    for _ in range(2):
        mo, mg = o.sweep(1), g.sweep(1)
        for k in ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or"):
            assert abs(mo[k] - mg[k]) <= 1e-11 * max(1, abs(mo[k])), k
    assert rel_err(g.download(dtype=np.float64)[0], o.get_fields()[0]) < 1e-11


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_upload_download_roundtrip(precision):
    L = (6, 4, 4)
    u, a = hot_config(L, seed=23)
    g = Lattice(L, **COUP, precision=precision)
    for dt in (np.float32, np.float64):
        g.upload(u.astype(dt), a.astype(dt))
        for which in (0, 1):
            if which == 1:
                g.upload(u.astype(dt), a.astype(dt), which=1)
            uu, aa = g.download(which=which, dtype=np.float64)
            tol = 1e-7 if (precision == "f32" or dt == np.float32) else 0
            np.testing.assert_allclose(uu, u, atol=tol)
            np.testing.assert_allclose(aa, a, atol=tol)


def test_hot_and_unit_starts():
    L = (16, 16, 16)
    g = Lattice(L, **COUP)
    g.init_unit(0.0)
    assert abs(g.plaquette() - 1.0) < 1e-12
    u, a = g.download(dtype=np.float64)
    assert np.all(u[..., 0] == 1) and np.all(a == 0)
    g.init_hot(5)
    u, a = g.download(dtype=np.float64)
    np.testing.assert_allclose(np.linalg.norm(u, axis=-1), 1, atol=1e-6)
    # Haar measure: each quaternion component has mean 0 and variance 1/4
    assert abs(u.mean()) < 5e-3 and abs(u.var() - 0.25) < 5e-3
    assert abs(a.mean()) < 1e-2 and abs(a.var() - 1.0) < 2e-2
    assert abs(g.plaquette()) < 1e-2


def test_error_paths():
    L = (4, 4, 4)
    with pytest.raises(LceError):
        Lattice((4, 4, 5), **COUP)
    g = Lattice(L, **COUP, precision="f64", rng="stream")
    g.init_unit(1.0)
    g.set_rng_stream(np.full(10, 0.5))
    with pytest.raises(LceError) as e:
        g.ahiggs2(1)
    assert e.value.code == lce._lib.LCE_ERR_STREAM
    # a non-finite field shows up as LCE_ERR_NAN in the measured sums
    u, a = hot_config(L, seed=1)
    a[0, 3, 1] = np.nan
    h = Lattice(L, **COUP, precision="f64")
    h.upload(u, a)
    with pytest.raises(LceError) as e:
        h.sweep(1)
    assert e.value.code == lce._lib.LCE_ERR_NAN
    # the gauge-fixing cap returns a status instead of spinning
    k = Lattice(L, **COUP, precision="f64", limit_or=1e-40)
    k.init_hot(3)
    with pytest.raises(LceError) as e:
        k.landau_gauge(max_iters=3)
    assert e.value.code == lce._lib.LCE_ERR_GF_NOT_CONVERGED


def test_gauge_invariant_measurements_on_gpu():
    L = (8, 8, 8)
    u, a = hot_config(L, seed=29)
    ug, ag = random_gauge_transform(u, a, L, seed=31)
    g1 = Lattice(L, **COUP, precision="f64")
    g2 = Lattice(L, **COUP, precision="f64")
    g1.upload(u, a)
    g2.upload(ug, ag)
    assert abs(g1.plaquette() - g2.plaquette()) < 1e-12
    assert rel_err(g1.scalarcorr()[0], g2.scalarcorr()[0]) < 1e-12
    assert rel_err(g1.polyakov()[0], g2.polyakov()[0]) < 1e-12


@pytest.mark.parametrize("L", [(4, 4, 4), (16, 16, 16), (64, 32, 34)])
def test_two_sites_per_thread_equals_one(L):
    """LCE_SWEEP_PASSES2 (tiles of 512 sites, two per thread) updates every
    site exactly as the one-site-per-thread kernels; only the order of the
    FP64 measurement sums differs."""
    res = []
    for mode in ("passes", "passes2"):
        g = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=77, sweep_mode=mode, n_link_or=1, n_higgs_metro=1)
        g.init_hot(8)
        ms = [g.sweep(1) for _ in range(3)]
        assert g.sweep_mode() == mode
        res.append((g.download(), ms, g.rng_position()))
    np.testing.assert_array_equal(res[0][0][0], res[1][0][0])
    np.testing.assert_array_equal(res[0][0][1], res[1][0][1])
    assert res[0][2] == res[1][2]
    for m0, m1 in zip(res[0][1], res[1][1]):
        for k in ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or", "acc_metro", "acc_link_or"):
            assert abs(m0[k] - m1[k]) <= 1e-12 * max(1.0, abs(m0[k])), k


def test_two_sites_per_thread_batch_and_three_way_autotune():
    specs = [Params(L=(16, 16, 16), beta=6.0, x=0.1, y=0.1, seed=5),
             Params(L=(8, 12, 6), beta=16.0, x=0.08, y=0.5, seed=6, imode=1),
             Params(L=(34, 8, 8), beta=9.0, x=0.1, y=0.3, seed=7)]
    outs = []
    for mode in ("passes", "passes2", "auto"):
        ens = Ensemble([Params(**{**s.__dict__, "sweep_mode": mode}) for s in specs])
        ens.init_hot(3)
        ens.sweeps(40, 1)
        if mode == "auto":
            assert ens.sweep_mode() in ("passes", "passes2", "persistent", "direct")
        outs.append([ens.download(chain=i) for i in range(3)])
    for o in outs[1:]:
        for i in range(3):
            np.testing.assert_array_equal(o[i][0], outs[0][i][0])
            np.testing.assert_array_equal(o[i][1], outs[0][i][1])


SHAPES = [(256, "passes"), (128, "passes"), (512, "passes"), (448, "passes"), (128, "passes2"), (256, "passes2"),
          (256, "direct")]


@pytest.mark.parametrize("L", [(16, 8, 12), (64, 32, 34)])
def test_tile_shapes_update_identically(L):
    """Every tile shape of the per-pass kernels (128, 256 or 512 threads per
    block; one or two sites per thread; the 56-register 128-thread form)
    updates every site exactly as the others; only the grouping of the FP64
    measurement sums differs."""
    res = []
    for bs, mode in SHAPES + [(128, "passes56")]:
        regs = 56 if mode == "passes56" else 0
        g = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=77, sweep_mode=mode.replace("56", ""), tile_threads=bs,
                    tile_registers=regs, n_link_or=1, n_higgs_metro=1)
        g.init_hot(8)
        ms = [g.sweep(1) for _ in range(3)]
        assert g.tile_shape(registers=True) == (bs, 2 if mode == "passes2" else 1, regs or (72 if bs == 448 else 64))
        res.append((g.download(), ms, g.rng_position()))
        g.close()
    for (u, a), ms, pos in res[1:]:
        np.testing.assert_array_equal(u, res[0][0][0])
        np.testing.assert_array_equal(a, res[0][0][1])
        assert pos == res[0][2]
        for m0, m1 in zip(res[0][1], ms):
            for k in ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or", "acc_metro", "acc_link_or"):
                assert abs(m0[k] - m1[k]) <= 1e-12 * max(1.0, abs(m0[k])), k


def test_tile_shapes_batch_of_uneven_volumes():
    specs = [Params(L=(16, 16, 16), beta=6.0, x=0.1, y=0.1, seed=5),
             Params(L=(8, 12, 6), beta=16.0, x=0.08, y=0.5, seed=6, imode=1),
             Params(L=(34, 8, 8), beta=9.0, x=0.1, y=0.3, seed=7)]
    outs = []
    for bs, mode in SHAPES:
        ens = Ensemble([Params(**{**s.__dict__, "sweep_mode": mode, "tile_threads": bs}) for s in specs])
        ens.init_hot(3)
        ens.sweeps(4, 1)
        outs.append([ens.download(chain=i) for i in range(3)])
        ens.close()
    for o in outs[1:]:
        for i in range(3):
            np.testing.assert_array_equal(o[i][0], outs[0][i][0])
            np.testing.assert_array_equal(o[i][1], outs[0][i][1])


MEAS_KEYS = ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or", "acc_metro", "acc_link_or")


@pytest.mark.parametrize("L", [(64, 64, 64), (96, 64, 48)])
def test_reduce_behind_multichunk(L):
    """The 448-thread kernels sum each pass's tile partials in extra blocks of
    the next pass (reduce-behind), and the finalize combines routine groups
    in parallel lanes.  At these volumes a slot spans 3 chunks of 128 tiles
    (448 threads), 2 (512), 8 or 9 (128: the single-chain and the multi-block
    finalize kernels), and the persistent form sums everything in its own
    kernel.  Two ahiggs1 calls and a link-overrelaxation hit per sweep make
    five routine groups (the step adaptation runs as a chain over two of
    them); measflag 0 sweeps leave slots for the ahiggs1 passes only.  Every
    form updates every site identically and advances the RNG and the ahiggs1
    step identically; the measurements agree to the FP64 rounding of their
    different tile groupings."""
    res = []
    for bs, mode in ((448, "passes"), (128, "passes"), (512, "passes"), (256, "persistent")):
        g = Lattice(L, beta=9.0, x=0.1, y=0.45, seed=31, sweep_mode=mode, tile_threads=bs if mode == "passes" else 0,
                    n_link_or=1, n_higgs_metro=2, delta0=2.0)
        g.init_hot(12)
        ms = []
        for mf in (1, 0, 1, 1, 0, 1):
            g.sweeps(1, mf)
            if mf:
                ms.append(g.meas1())
        assert g.sweep_mode() == mode
        res.append((g.download(), ms, g.rng_position()))
        g.close()
    (u0, a0), ms0, pos0 = res[0]
    for (u, a), ms, pos in res[1:]:
        np.testing.assert_array_equal(u, u0)
        np.testing.assert_array_equal(a, a0)
        assert pos == pos0
        for m0, m1 in zip(ms0, ms):
            assert m0["delta"] == m1["delta"]
            for k in MEAS_KEYS:
                assert abs(m0[k] - m1[k]) <= 1e-12 * max(1.0, abs(m0[k])), k
    # the step moved: the acceptance of the two ahiggs1 calls was adapted to
    assert ms0[-1]["delta"] != 2.0


def test_reduce_behind_batch_of_multichunk_chains():
    """A batch whose chains span several chunks each: the reduce-behind
    blocks take the level-1 items of every chain, the multi-block finalize
    the rest.  448-thread tiles against 128-thread tiles."""
    specs = [Params(L=(64, 64, 64), beta=6.0, x=0.1, y=0.1, seed=5, n_link_or=1, n_higgs_metro=1),
             Params(L=(80, 64, 40), beta=16.0, x=0.08, y=0.5, seed=6, imode=1, n_link_or=1, n_higgs_metro=1),
             Params(L=(8, 12, 6), beta=9.0, x=0.1, y=0.3, seed=7, n_link_or=1, n_higgs_metro=1)]
    outs = []
    for bs in (448, 128):
        ens = Ensemble([Params(**{**s.__dict__, "sweep_mode": "passes", "tile_threads": bs}) for s in specs])
        ens.init_hot(3)
        ens.sweeps(3, 1)
        outs.append(([ens.download(chain=i) for i in range(3)], ens.meas_batch()))
        ens.close()
    for i in range(3):
        np.testing.assert_array_equal(outs[1][0][i][0], outs[0][0][i][0])
        np.testing.assert_array_equal(outs[1][0][i][1], outs[0][0][i][1])
    for m0, m1 in zip(outs[0][1], outs[1][1]):
        for k in MEAS_KEYS:
            assert abs(m0[k] - m1[k]) <= 1e-12 * max(1.0, abs(m0[k])), k


@pytest.mark.parametrize("case", ["passes", "persistent", "passes_448_64cubed", "f64_stream"])
def test_multi_sweep_graph_equals_single_sweeps(case):
    """lce_sweeps(n) replays graphs of 8 sweeps chained by programmatic
    launch; in the per-pass form each sweep's finalize but the last runs in
    an extra block of the next sweep's first pass, and the sweeps take fixed
    RNG offsets that only the graph's last finalize advances.  19 sweeps that
    way (two 8-sweep graphs and three single ones) give the same fields, RNG
    position (Philox counter or validation-stream position) and last
    measurements as 19 single lce_sweep calls, with ahiggs1 (its step adapted
    after every sweep) and a link-overrelaxation hit in the composition."""
    L, kw = (16, 16, 16), dict(sweep_mode="passes")
    if case == "persistent":
        kw = dict(sweep_mode="persistent")
    elif case == "passes_448_64cubed":
        L, kw = (64, 64, 64), dict(sweep_mode="passes", tile_threads=448)
    elif case == "f64_stream":
        L, kw = (8, 8, 8), dict(sweep_mode="passes", precision="f64", rng="stream")
    res = []
    for many in (True, False):
        g = Lattice(L, beta=9.0, x=0.1, y=0.45, seed=17, n_link_or=1, n_higgs_metro=1, delta0=3.0, **kw)
        g.init_hot(4)
        if case == "f64_stream":
            g.set_rng_stream(np.random.default_rng(5).random(40 * 19 * L[0] * L[1] * L[2]))
        if many:
            g.sweeps(19, 1)
        else:
            for _ in range(19):
                g.sweep(1)
        res.append((g.download(), g.meas1(), g.rng_position()))
        g.close()
    (u0, a0), m0, r0 = res[0]
    (u1, a1), m1, r1 = res[1]
    np.testing.assert_array_equal(u0, u1)
    np.testing.assert_array_equal(a0, a1)
    assert r0 == r1 and m0 == m1


@pytest.mark.parametrize("case", ["single_128cubed", "batch"])
def test_multi_sweep_graph_multichunk_and_batch(case):
    """Graphs of sweeps where each sweep keeps its own finalize kernel (the
    multi-block one): a chain of more than 8 chunks (128^3, 128-thread tiles:
    64 chunks) and a batch of chains.  19 sweeps through lce_sweeps equal 19
    single sweeps bit for bit."""
    if case == "single_128cubed":
        specs = [Params(L=(128, 128, 128), beta=12.0, x=0.09, y=0.3, seed=5, n_higgs_metro=1, delta0=2.0)]
    else:
        specs = [Params(L=(32, 32, 32), beta=6.0, x=0.1, y=0.1, seed=5, n_link_or=1, n_higgs_metro=1),
                 Params(L=(8, 12, 6), beta=16.0, x=0.08, y=0.5, seed=6, imode=1, n_link_or=1, n_higgs_metro=1),
                 Params(L=(48, 16, 16), beta=9.0, x=0.1, y=0.3, seed=7, n_link_or=1, n_higgs_metro=1)]
    res = []
    for many in (True, False):
        ens = Ensemble([Params(**{**s.__dict__, "sweep_mode": "passes", "tile_threads": 128}) for s in specs])
        ens.init_hot(3)
        if many:
            ens.sweeps(19, 1)
        else:
            for _ in range(19):
                ens.sweep(1)
        res.append(([ens.download(chain=i) for i in range(len(specs))], ens.meas_batch(), ens.rng_position()))
        ens.close()
    for i in range(len(specs)):
        np.testing.assert_array_equal(res[0][0][i][0], res[1][0][i][0])
        np.testing.assert_array_equal(res[0][0][i][1], res[1][0][i][1])
    assert res[0][1] == res[1][1] and res[0][2] == res[1][2]


def test_autotune_chooses_form_and_tile_shape():
    """LCE_SWEEP_AUTO times every candidate (per-pass forms at each tile
    shape, and the persistent form) on real sweeps and keeps one; with
    tile_threads fixed only that block size is a per-pass candidate.  The
    fields equal a fixed-shape run's."""
    L = (32, 32, 32)
    ref = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=3, sweep_mode="passes", tile_threads=256)
    ref.init_hot(1)
    ref.sweeps(40, 0)
    u_ref, a_ref = ref.download()
    ref.close()
    for req in (0, 128):
        g = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=3, sweep_mode="auto", tile_threads=req)
        g.init_hot(1)
        g.sweeps(40, 0)
        mode = g.sweep_mode()
        bs, spt = g.tile_shape()
        assert mode in ("passes", "passes2", "persistent", "direct")
        if mode == "persistent":
            assert (bs, spt) == (256, 1)
        else:
            assert bs in ((128, 256, 448, 512) if req == 0 else (req,)) and spt == (2 if mode == "passes2" else 1)
        u, a = g.download()
        g.close()
        np.testing.assert_array_equal(u, u_ref)
        np.testing.assert_array_equal(a, a_ref)


def test_tile_threads_rejected_when_invalid():
    with pytest.raises(LceError):
        Lattice((8, 8, 8), tile_threads=64)
    with pytest.raises(LceError):
        Lattice((8, 8, 8), tile_threads=256, tile_registers=56)
    with pytest.raises(LceError):
        Lattice((8, 8, 8), tile_threads=128, tile_registers=56, precision="f64")


def test_profiled_sweep_graph_is_an_ordinary_sweep():
    """lce_profile_sweep runs one sweep as a graph with timing events hung off
    the pass kernels: it updates the fields exactly as lce_sweep does, and
    returns one positive duration per pass (10 for the reference
    composition)."""
    L = (16, 8, 12)
    a = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=5, sweep_mode="passes")
    b = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=5, sweep_mode="passes")
    for g in (a, b):
        g.init_hot(6)
        g.sweeps(2, 1)
    a.sweeps(1, 1)
    ms = b.profile_sweep(1)
    assert len(ms) == 10 and np.all(ms > 0)
    assert a.rng_position() == b.rng_position()
    np.testing.assert_array_equal(a.download()[0], b.download()[0])
    np.testing.assert_array_equal(a.download()[1], b.download()[1])
    ms2 = b.profile_sweep(0)  # a second graph, without the measurements
    assert len(ms2) == 10 and np.all(ms2 > 0)
    a.close()
    b.close()
