"""Conjugate-gradient form of the Fourier-accelerated Landau gauge fixing
(lce_landau_gauge_fourier_cg): it reaches the plain iteration's stopping
criterion, tracks the transform, ends at a maximum of the same quality as
the steepest-ascent form, and runs from warm starts."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

COUP = dict(beta=12.0, x=0.09, y=0.3, lam=1.7)


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_cg_reaches_the_plain_criterion_and_tracks_the_transform(precision):
    from lceqcd_b200 import Lattice
    L = (16, 16, 16)
    g = Lattice(L, **COUP, precision=precision, limit_or=1e-11, seed=11)
    g.init_hot(3)
    g.sweeps(40, 0)
    th, itf, itp = g.landau_gauge_fourier_cg("identity")
    assert th <= 1e-11 and itf > 1 and itp == 0
    assert g.theta() <= 1e-10
    uf, _ = g.download(which=1, dtype=np.float64)
    g.apply_transform()
    uf2, _ = g.download(which=1, dtype=np.float64)
    tol = 1e-9 if precision == "f64" else 2e-3
    assert np.max(np.abs(uf - uf2)) < tol
    th0, th1, it1 = g.landau_gauge_from("transform")
    assert th0 <= 1e-10 and th1 <= 1e-11 and it1 < 100


@pytest.mark.parametrize("L", [(32, 32, 32), (16, 16, 64)])
def test_cg_against_steepest_ascent(L):
    """Same configurations, both forms from G = 1: both converge, to maxima of
    the functional of the same quality, the CG form in fewer iterations."""
    from lceqcd_b200 import Lattice
    g = Lattice(L, **COUP, limit_or=1e-10, seed=21)
    g.init_hot(5)
    g.sweeps(60, 0)
    sd, cg = 0, 0
    for _ in range(2):
        g.sweeps(5, 0)
        th, itf, itp = g.landau_gauge_fourier("identity")
        assert th <= 1e-10
        F_sd = g.gauge_functional()
        th, itc, itp2 = g.landau_gauge_fourier_cg("identity")
        assert th <= 1e-10 and itp2 == 0
        F_cg = g.gauge_functional()
        assert abs(F_cg - F_sd) < 5e-3
        sd += itf + itp
        cg += itc
    print("iterations steepest", sd, "cg", cg)
    assert cg < sd, (cg, sd)


def test_cg_from_a_warm_start_and_with_a_plain_finish():
    from lceqcd_b200 import GaugeNet, Lattice
    g = Lattice((16, 16, 32), **COUP, limit_or=1e-10, seed=8)
    g.init_hot(2)
    g.sweeps(40, 0)
    th, itf, itp = g.landau_gauge_fourier_cg("identity")
    assert th <= 1e-10 and itp == 0
    g.sweeps(3, 0)
    th, itf2, itp2 = g.landau_gauge_fourier_cg("transform")
    assert th <= 1e-10 and itp2 == 0
    g.sweeps(3, 0)
    th, itf3, itp3 = g.landau_gauge_fourier_cg("identity", theta_switch=1e-6)
    assert th <= 1e-10 and itp3 >= 1
    # the warm-start entry point with the CG flag, judged against identity
    net = GaugeNet(seed=3)
    g.sweeps(3, 0)
    start, F, th, it = g.landau_gauge_warm(net, use_net=True, judge=True, fourier=True, cg=True)
    assert th <= 1e-10 and start in ("identity", "transform", "net") and it > 0


def test_cg_needs_power_of_two_extents():
    from lceqcd_b200 import Lattice, LceError
    g = Lattice((8, 8, 12), **COUP, seed=1)
    g.init_hot(1)
    with pytest.raises(LceError):
        g.landau_gauge_fourier_cg("identity")


def test_cg_in_a_batch_of_uneven_volumes():
    """Chains of different volumes share the context's buffers (transforms,
    previous F, direction, CG state); the CG state restarts for each chain,
    and steepest-ascent and CG runs interleave with their graphs intact."""
    from lceqcd_b200 import Ensemble, Params
    specs = [Params(L=(16, 16, 16), **COUP, limit_or=1e-10, seed=1),
             Params(L=(32, 16, 8), **COUP, limit_or=1e-10, seed=2),
             Params(L=(8, 8, 8), **COUP, limit_or=1e-10, seed=3)]
    ens = Ensemble(specs)
    ens.init_hot(4)
    ens.sweeps(30, 0)
    for rnd in range(2):
        for c in (2, 0, 1) if rnd else (0, 1, 2):
            start = "identity" if rnd == 0 else "transform"
            th, itf, itp = ens.landau_gauge_fourier_cg(start, chain=c)
            assert th <= 1e-10 and itp == 0
            assert ens.theta(chain=c) <= 1e-10
            th, itf, itp = ens.landau_gauge_fourier(start, chain=c)
            assert th <= 1e-10
        ens.sweeps(2, 0)
