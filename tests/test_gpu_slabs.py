"""z-slab decomposition (lce_slabs_*, the reference's MPI domain
decomposition with a halo exchange after every pass): the lattice split over
1, 2 or 4 slabs reproduces the undecomposed context's fields bit for bit
(whole-lattice Philox counters) and its measurements to summation order, in
FP64 and FP32; the slabs here share one GPU, so the halo copies are
device-to-device (peer copies between GPUs take the same path)."""
import numpy as np
import pytest

from oracle.oracle import hot_config

pytestmark = pytest.mark.gpu
lce = pytest.importorskip("lceqcd_b200")
from lceqcd_b200 import LceError, Lattice, SlabLattice  # noqa: E402

KEYS = ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or")


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("L,nslabs", [((4, 4, 8), 1), ((4, 4, 8), 2), ((8, 6, 8), 4), ((6, 4, 12), 3),
                                      ((8, 8, 16), 2)])
def test_slabs_reproduce_the_whole_lattice(precision, L, nslabs):
    dt = np.float64 if precision == "f64" else np.float32
    u, a = hot_config(L, seed=31, dtype=dt)
    kw = dict(beta=12.0, x=0.09, y=0.3, precision=precision, seed=4242, n_link_or=1, n_higgs_metro=1,
              delta0=0.75)
    g = Lattice(L, sweep_mode="passes", **kw)
    g.upload(u, a)
    s = SlabLattice(L, nslabs, **kw)
    s.upload(u, a)
    for k in range(3):
        mg, ms = g.sweep(1), s.sweep(1)
        ug, ag = g.download(dtype=dt)
        us, as_ = s.download(dtype=dt)
        np.testing.assert_array_equal(us, ug)
        np.testing.assert_array_equal(as_, ag)
        for key in KEYS + ("acc_link_or", "acc_metro", "delta"):
            assert abs(ms[key] - mg[key]) <= 1e-12 * max(1.0, abs(mg[key])), (k, key)
    s.sweep(0)
    g.sweep(0)
    np.testing.assert_array_equal(s.download(dtype=dt)[0], g.download(dtype=dt)[0])
    s.close()


def test_slabs_metropolis_step_adapts_to_the_whole_lattice():
    """The ahiggs1 step follows the whole lattice's acceptance (f/ahiggs1.f:
    113-123): a step far from 50% acceptance is rescaled identically on every
    slab and in the undecomposed run, over several sweeps."""
    L = (8, 4, 8)
    u, a = hot_config(L, seed=9)
    kw = dict(beta=9.0, x=0.1, y=0.45, precision="f64", seed=11, n_higgs_metro=2, delta0=5.0)
    g = Lattice(L, sweep_mode="passes", **kw)
    g.upload(u, a)
    s = SlabLattice(L, 4, **kw)
    s.upload(u, a)
    deltas = []
    for k in range(4):
        mg, ms = g.sweep(k % 2), s.sweep(k % 2)
        assert ms["delta"] == mg["delta"], k
        deltas.append(ms["delta"])
    assert deltas[-1] < 5.0  # a step of 5 is accepted rarely: it shrinks
    np.testing.assert_array_equal(s.download()[1], g.download()[1])


def test_slabs_three_hit_link_update():
    L = (4, 6, 8)
    u, a = hot_config(L, seed=5)
    kw = dict(beta=9.0, x=0.1, y=0.45, precision="f64", seed=7, agauge_hits=3)
    g = Lattice(L, sweep_mode="passes", **kw)
    g.upload(u, a)
    s = SlabLattice(L, 2, **kw)
    s.upload(u, a)
    for _ in range(2):
        mg, ms = g.sweep(1), s.sweep(1)
    np.testing.assert_array_equal(s.download()[0], g.download()[0])
    assert abs(ms["acc_gauge"] - mg["acc_gauge"]) <= 1e-12


def test_slabs_reject_what_they_cannot_do():
    for L, n in (((4, 4, 6), 2), ((4, 4, 8), 8), ((4, 4, 8), 3)):  # odd, too thin, not a divisor
        with pytest.raises(LceError):
            SlabLattice(L, n, precision="f64")
    with pytest.raises(LceError):
        SlabLattice((4, 4, 8), 2, rng="stream")


def _thermalised_pair(L, nslabs, precision, limit_or, sweeps=3, seed=17):
    dt = np.float64 if precision == "f64" else np.float32
    u, a = hot_config(L, seed=seed, dtype=dt)
    kw = dict(beta=9.0, x=0.1, y=0.45, lam=1.7, limit_or=limit_or, precision=precision, seed=seed + 1)
    g = Lattice(L, sweep_mode="passes", **kw)
    g.upload(u, a)
    s = SlabLattice(L, nslabs, **kw)
    s.upload(u, a)
    for _ in range(sweeps):
        g.sweep(0)
        s.sweep(0)
    return g, s, dt


@pytest.mark.parametrize("precision,limit_or", [("f64", 1e-10), ("f32", 1e-6)])
@pytest.mark.parametrize("L,nslabs", [((8, 8, 8), 1), ((8, 8, 8), 2), ((8, 6, 12), 3), ((6, 8, 16), 4)])
def test_slabs_landau_gauge_reproduces_the_whole_lattice(precision, limit_or, L, nslabs):
    """f/landau_gauge.f's overrelaxed fixing on the slabs: the same
    iteration count, theta to summation order, and u_f, a_f bit for bit
    (every site's update is the undecomposed one; the U_z links a slab's
    first plane updates in its halo go back to the slab below)."""
    g, s, dt = _thermalised_pair(L, nslabs, precision, limit_or)
    tg, ig = g.landau_gauge()
    ts, is_ = s.landau_gauge()
    assert is_ == ig and ig > 10
    assert tg <= limit_or and abs(ts - tg) <= 1e-9 * tg
    ug, ag = _fixed(g, dt)
    us, as_ = s.download(dtype=dt, fixed=True)
    np.testing.assert_array_equal(us, ug)
    np.testing.assert_array_equal(as_, ag)
    # the un-fixed fields are untouched
    np.testing.assert_array_equal(s.download(dtype=dt)[0], g.download(dtype=dt)[0])
    s.close()


def _fixed(g, dt):
    return g.download(which=1, dtype=dt)  # LCE_FIELDS_FIXED


@pytest.mark.parametrize("precision,limit_or", [("f64", 1e-10), ("f32", 1e-6)])
@pytest.mark.parametrize("L,nslabs", [((8, 8, 8), 2), ((8, 6, 12), 3), ((6, 8, 16), 4)])
def test_slabs_tracked_fixing_and_warm_start(precision, limit_or, L, nslabs):
    """lce_landau_gauge_from on the slabs: the fixing from G = 1 tracking the
    transform, three more sweeps, then the fixing from the previous
    transform (G exchanged across the slab boundaries and applied on every
    plane) -- the undecomposed run's iterations and u_f, a_f bit for bit."""
    g, s, dt = _thermalised_pair(L, nslabs, precision, limit_or)
    _, tg, ig = g.landau_gauge_from("identity")
    ts, is_ = s.landau_gauge_from("identity")
    assert is_ == ig and ig > 10 and abs(ts - tg) <= 1e-9 * tg
    for x, y in zip(s.download(dtype=dt, fixed=True), _fixed(g, dt)):
        np.testing.assert_array_equal(x, y)
    for _ in range(3):
        g.sweep(0)
        s.sweep(0)
    _, tg2, ig2 = g.landau_gauge_from("transform")
    ts2, is2 = s.landau_gauge_from("transform")
    assert is2 == ig2 and abs(ts2 - tg2) <= 1e-9 * tg2
    for x, y in zip(s.download(dtype=dt, fixed=True), _fixed(g, dt)):
        np.testing.assert_array_equal(x, y)
    with pytest.raises(LceError):  # LCE_GF_START_NET: no network on slabs
        s._ck(s.lib.lce_slabs_landau_gauge_from(s.h, 2, None, None, 0))
    s.close()


@pytest.mark.parametrize("precision,limit_or,switch", [("f64", 1e-10, 0.0), ("f32", 1e-6, 0.0),
                                                       ("f64", 1e-10, 1e-4)])
@pytest.mark.parametrize("L,nslabs", [((8, 8, 8), 2), ((8, 4, 16), 4), ((16, 8, 8), 2)])
def test_slabs_fourier_fixing_reproduces_the_whole_lattice(precision, limit_or, switch, L, nslabs):
    """The Fourier-accelerated fixing on the slabs (the per-site stages on
    every slab, the y/z transforms of the whole lattice's buffer on the first
    slab's device): from G = 1, then after three sweeps from the previous
    transform; with a switch theta the plain iteration finishes.  The
    undecomposed run's iteration counts and u_f, a_f bit for bit."""
    g, s, dt = _thermalised_pair(L, nslabs, precision, limit_or)
    for start in ("identity", "transform"):
        tg, fg, pg = g.landau_gauge_fourier(start, theta_switch=switch)
        ts, fs, ps = s.landau_gauge_fourier(start, theta_switch=switch)
        assert (fs, ps) == (fg, pg) and fg > 2
        assert (pg > 0) == (switch > 0)
        assert tg <= limit_or and abs(ts - tg) <= 1e-9 * tg
        for x, y in zip(s.download(dtype=dt, fixed=True), _fixed(g, dt)):
            np.testing.assert_array_equal(x, y)
        for _ in range(3):
            g.sweep(0)
            s.sweep(0)
    s.close()


@pytest.mark.parametrize("precision,limit_or", [("f64", 1e-10), ("f32", 1e-6)])
@pytest.mark.parametrize("L,nslabs", [((8, 8, 8), 2), ((6, 8, 12), 3)])
@pytest.mark.parametrize("fix,asc,track", [(True, True, True), (True, False, False)])
def test_slabs_iterative_fixing_reproduces_the_whole_lattice(precision, limit_or, L, nslabs, fix, asc, track):
    """f/it_gauge_fixing.f under f/landau_gauge.f on the slabs: the same
    iteration count, da1 to summation order, u_f, a_f bit for bit."""
    g, s, dt = _thermalised_pair(L, nslabs, precision, limit_or)
    dg, ig = g.it_landau_gauge(0.3, fix_component=fix, ascend=asc, track=track)
    ds, is_ = s.it_landau_gauge(0.3, fix_component=fix, ascend=asc, track=track)
    assert is_ == ig and ig > 10 and abs(ds - dg) <= 1e-9 * dg
    for x, y in zip(s.download(dtype=dt, fixed=True), _fixed(g, dt)):
        np.testing.assert_array_equal(x, y)
    s.close()


@pytest.mark.parametrize("precision,limit_or", [("f64", 1e-10), ("f32", 1e-6)])
@pytest.mark.parametrize("L,nslabs", [((8, 8, 8), 2), ((8, 4, 16), 4), ((16, 8, 8), 2)])
def test_slabs_fourier_cg_fixing_matches_the_whole_lattice(precision, limit_or, L, nslabs):
    """The conjugate-gradient form on the slabs, from G = 1 and after three
    sweeps from the previous transform: the line search's sums are grouped
    per slab, so the step differs from the undecomposed one in the last bits
    and the two runs stop at different points inside theta < limit_or --
    the same iteration counts, u_f, a_f equal within what the stopping
    criterion leaves free (|dU| ~ sqrt(limit_or): 1e-6 in FP64 at 1e-10,
    measured 1.8e-8; 2e-5 in FP32)."""
    g, s, dt = _thermalised_pair(L, nslabs, precision, limit_or)
    tol = 1e-6 if precision == "f64" else 2e-5
    for start in ("identity", "transform"):
        tg, fg, pg = g.landau_gauge_fourier_cg(start)
        ts, fs, ps = s.landau_gauge_fourier_cg(start)
        assert fs == fg and pg == ps == 0 and fg > 2
        assert ts <= limit_or and tg <= limit_or
        for x, y in zip(s.download(dtype=dt, fixed=True), _fixed(g, dt)):
            assert np.max(np.abs(x.astype(np.float64) - y.astype(np.float64))) <= tol * max(1.0, np.max(np.abs(y)))
        for _ in range(3):
            g.sweep(0)
            s.sweep(0)
    s.close()


def test_slabs_fourier_fixing_needs_powers_of_two():
    s = SlabLattice((12, 8, 8), 2, precision="f64")
    with pytest.raises(LceError):
        s.landau_gauge_fourier()
    s.close()


def test_slabs_landau_gauge_cap():
    """An iteration cap stops both runs at the same iteration with the
    reference's not-converged status and the same partly fixed u_f."""
    g, s, dt = _thermalised_pair((8, 8, 8), 2, "f64", 1e-12)
    with pytest.raises(LceError):
        g.landau_gauge(max_iters=7)
    with pytest.raises(LceError):
        s.landau_gauge(max_iters=7)
    np.testing.assert_array_equal(s.download(fixed=True)[0], _fixed(g, dt)[0])
    s.close()


@pytest.mark.parametrize("nslabs", [1, 2, 4])
def test_slabs_correlators_match_the_whole_lattice(nslabs):
    """f/correlator.f, f/polyakov.f and f/scalarcorr.f on the slabs: slice
    sums per slab gathered on the first slab's device, correlated there; the
    whole lattice's values to summation order."""
    L = (8, 6, 16)
    g, s, dt = _thermalised_pair(L, nslabs, "f64", 1e-10, seed=23)
    g.landau_gauge()
    s.landau_gauge()
    for vg, vs in zip(g.correlator(), s.correlator()):
        np.testing.assert_allclose(vs, vg, rtol=1e-12, atol=1e-13)
    for fn in ("polyakov", "scalarcorr"):
        rg, rs = getattr(g, fn)(), getattr(s, fn)()
        np.testing.assert_allclose(rs[0], rg[0], rtol=1e-12, atol=1e-13)
        np.testing.assert_allclose(rs[1], rg[1], rtol=1e-12, atol=1e-13)
        assert abs(rs[2] - rg[2]) <= 1e-12 * max(1.0, abs(rg[2]))
    s.close()


@pytest.mark.parametrize("L,nslabs", [((4, 4, 8), 2), ((6, 4, 12), 3), ((8, 6, 8), 4)])
def test_slab_validation_stream_matches_the_oracle(L, nslabs):
    """FP64 validation mode on slabs: each slab draws the whole lattice's
    stream slots of its own sites, so two sweeps reproduce the oracle (the
    reference's routines at one rank) at 1e-12 and consume the stream alike."""
    from oracle.oracle import Oracle, reference_stream, uniforms_per_sweep
    u, a = hot_config(L, seed=13)
    stream = reference_stream(2 * uniforms_per_sweep(L), seed=77)
    o = Oracle(L, 9.0, 0.1, 0.45)
    o.set_fields(u, a)
    o.set_stream(stream)
    s = SlabLattice(L, nslabs, beta=9.0, x=0.1, y=0.45, precision="f64", rng="stream")
    s.upload(u, a)
    s.set_rng_stream(stream)
    for _ in range(2):
        mo, ms = o.sweep(1), s.sweep(1)
        for key in ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or"):
            assert abs(ms[key] - mo[key]) <= 1e-12 * max(1.0, abs(mo[key])), key
    uo, ao = o.get_fields()
    us, as_ = s.download(dtype=np.float64)
    assert np.max(np.abs(us - uo)) < 1e-12 and np.max(np.abs(as_ - ao)) < 1e-12
    with pytest.raises(LceError):  # the stream is used up
        s.sweep(1)
    s.close()


def test_slabs_on_two_devices_reproduce_the_whole_lattice():
    """Two slabs on devices 0 and 1: the halo planes cross as peer copies
    (no multicast); the fields equal the undecomposed run's bit for bit."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    L = (8, 8, 16)
    u, a = hot_config(L, seed=17, dtype=np.float32)
    kw = dict(beta=12.0, x=0.09, y=0.3, precision="f32", seed=4343)
    g = Lattice(L, sweep_mode="passes", **kw)
    g.upload(u, a)
    s = SlabLattice(L, 2, devices=[0, 1], **kw)
    s.upload(u, a)
    for _ in range(3):
        mg, ms = g.sweep(1), s.sweep(1)
        for key in KEYS:
            assert abs(ms[key] - mg[key]) <= 1e-12 * max(1.0, abs(mg[key])), key
    np.testing.assert_array_equal(s.download(dtype=np.float32)[0], g.download(dtype=np.float32)[0])
    np.testing.assert_array_equal(s.download(dtype=np.float32)[1], g.download(dtype=np.float32)[1])
    s.close()
