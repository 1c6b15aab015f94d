"""Plane-synchronised chaining of the per-pass kernels (lce_set_plane_sync).

A tile of pass i starts once pass i-1 has finished the z-planes it reads,
instead of after the whole pass; the tiles are dispatched in a folded plane
order and keep their natural index for the partial sums.  None of this may
change a bit of the result: fields, measurements and RNG position equal the
whole-pass chaining's, for every compiled tile shape, for the extra pass kinds
(link overrelaxation, Higgs Metropolis, the three-hit link update of
f/agauge1.f) and for a batch of uneven volumes, and no tile falls back to the
whole-pass wait.  Shapes whose tiles are not plane-aligned keep the whole-pass
wait.
"""
import numpy as np
import pytest

from lceqcd_b200.lattice import Ensemble, Lattice, Params

pytestmark = pytest.mark.gpu

KEYS = ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or", "acc_metro", "acc_link_or", "delta")


def _run(L, bs, mode, on, sweeps=4, **kw):
    g = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=77, sweep_mode=mode, tile_threads=bs, **kw)
    g.set_plane_sync(on)
    g.init_hot(8)
    ms = [g.sweep(1) for _ in range(sweeps)]
    out = (g.download(), ms, g.rng_position(), g.plane_sync())
    g.close()
    return out


def _same(a, b):
    np.testing.assert_array_equal(a[0][0], b[0][0])
    np.testing.assert_array_equal(a[0][1], b[0][1])
    assert a[2] == b[2]
    for m0, m1 in zip(a[1], b[1]):
        for k in KEYS:
            assert m0[k] == m1[k], k


@pytest.mark.parametrize("L", [(32, 32, 32), (64, 32, 34), (32, 16, 4)])
@pytest.mark.parametrize("bs,mode", [(128, "passes"), (256, "passes"), (512, "passes"), (256, "passes2"),
                                     (256, "direct")])
def test_plane_sync_updates_identically(L, bs, mode):
    kw = dict(n_link_or=1, n_higgs_metro=1)
    off = _run(L, bs, mode, False, **kw)
    on = _run(L, bs, mode, True, **kw)
    tile = bs * (2 if mode == "passes2" else 1)
    aligned = (L[0] * L[1] // 2) % tile == 0
    assert on[3] == (True, aligned, 0)
    assert off[3][:2] == (False, False)
    _same(off, on)


def test_plane_sync_three_hit_link_update():
    off = _run((32, 32, 16), 256, "passes", False, agauge_hits=3)
    on = _run((32, 32, 16), 256, "passes", True, agauge_hits=3)
    assert on[3] == (True, True, 0)
    _same(off, on)


def test_plane_sync_long_run_alternating_measurements():
    """60 sweeps, measurements every other sweep (graphs of both measflags
    replayed in turn): the plane counters are reset by every finalize."""
    res = []
    for on in (False, True):
        g = Lattice((64, 64, 64), beta=12.0, x=0.09, y=0.3, seed=5, sweep_mode="passes", tile_threads=512)
        g.set_plane_sync(on)
        g.init_hot(2)
        for k in range(30):
            g.sweeps(1, 0)
            g.sweeps(1, 1)
        res.append((g.download(), g.meas1(), g.plane_sync()))
        g.close()
    assert res[1][2] == (True, True, 0)
    np.testing.assert_array_equal(res[0][0][0], res[1][0][0])
    np.testing.assert_array_equal(res[0][0][1], res[1][0][1])
    for k in KEYS:
        assert res[0][1][k] == res[1][1][k], k


def test_plane_sync_batch_of_uneven_volumes():
    specs = [Params(L=(16, 16, 16), beta=6.0, x=0.1, y=0.1, seed=5),
             Params(L=(32, 16, 10), beta=16.0, x=0.08, y=0.5, seed=6, imode=1),
             Params(L=(16, 32, 6), beta=9.0, x=0.1, y=0.3, seed=7)]
    outs = []
    for on in (False, True):
        ens = Ensemble([Params(**{**s.__dict__, "sweep_mode": "passes", "tile_threads": 128}) for s in specs])
        ens.set_plane_sync(on)
        ens.init_hot(3)
        ens.sweeps(6, 1)
        outs.append(([ens.download(chain=i) for i in range(3)], ens.meas_batch(), ens.plane_sync()))
        ens.close()
    assert outs[1][2] == (True, True, 0)
    for i in range(3):
        np.testing.assert_array_equal(outs[0][0][i][0], outs[1][0][i][0])
        np.testing.assert_array_equal(outs[0][0][i][1], outs[1][0][i][1])
        for k in KEYS:
            assert outs[0][1][i][k] == outs[1][1][i][k], k


def test_plane_sync_switch_rebuilds_graphs():
    """Switching mid-run drops the cached sweep graphs; the run continues
    exactly as one that never switched."""
    L = (32, 32, 32)
    a = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=9, sweep_mode="passes", tile_threads=256)
    a.set_plane_sync(False)
    a.init_hot(4)
    a.sweeps(5, 1)
    b = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=9, sweep_mode="passes", tile_threads=256)
    b.set_plane_sync(False)
    b.init_hot(4)
    b.sweeps(2, 1)
    b.set_plane_sync(True)
    b.sweeps(2, 1)
    b.set_plane_sync(False)
    b.sweeps(1, 1)
    for x, y in zip(a.download(), b.download()):
        np.testing.assert_array_equal(x, y)
    a.close()
    b.close()
