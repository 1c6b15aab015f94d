"""Fourier-accelerated Landau gauge fixing: the FFT-preconditioned direction
against numpy's FFT on the same U_f, convergence to the plain iteration's
stopping criterion, the tracked transform, and the gain in iterations."""
import numpy as np
import pytest

import net_reference as NR

pytestmark = pytest.mark.gpu

COUP = dict(beta=12.0, x=0.09, y=0.3, lam=1.7)


def numpy_direction(uf, L, alpha, step):
    """omega = step F^-1[F[Delta]/p_c^2] from links uf[mu][eo][s][4]."""
    L1, L2, L3 = L
    nh = L1 * L2 * L3 // 2
    x, y, z = NR.coords(L)
    flat = uf.reshape(3, 2 * nh, 4).astype(np.float64)
    c = np.array([1.0, 1.0, alpha])
    D = np.zeros((2 * nh, 3))  # a3, Re b, Im b
    for mu in range(3):
        d = [0, 0, 0]
        d[mu] = -1
        m = NR.flat_index(L, x + d[0], y + d[1], z + d[2])
        D[:, 0] += c[mu] * (flat[mu][:, 1] - flat[mu][m, 1])
        D[:, 1] += c[mu] * (flat[mu][:, 2] - flat[mu][m, 2])
        D[:, 2] += c[mu] * (flat[mu][:, 3] - flat[mu][m, 3])
    nat = np.zeros((3, L3, L2, L1))
    for k in range(3):
        nat[k][z, y, x] = D[:, k]
    kz, ky, kx = np.meshgrid(np.arange(L3), np.arange(L2), np.arange(L1), indexing="ij")
    p2 = 4 * (np.sin(np.pi * kx / L1) ** 2 + np.sin(np.pi * ky / L2) ** 2 + alpha * np.sin(np.pi * kz / L3) ** 2)
    p2[0, 0, 0] = np.inf
    out = np.zeros((2 * nh, 3))
    for k in range(3):
        w = np.fft.ifftn(np.fft.fftn(nat[k]) * step / p2).real
        out[:, k] = w[z, y, x]
    return out.reshape(2, nh, 3), D


# the transforms are FP32 (the divergence and the step's application FP64):
# the direction agrees with numpy's FP64 FFT to FP32 accuracy times the
# preconditioner's amplification of the longest wavelength, 1/p^2 ~ (L/2pi)^2
@pytest.mark.parametrize("precision,L,tol", [("f64", (8, 8, 8), 2e-6), ("f64", (16, 4, 8), 2e-6),
                                             ("f32", (8, 16, 4), 2e-6), ("f32", (32, 32, 32), 5e-6),
                                             ("f64", (4, 4, 64), 5e-6), ("f32", (128, 4, 2), 5e-6),
                                             ("f32", (1024, 2, 4), 5e-6), ("f64", (2, 512, 4), 5e-6),
                                             ("f32", (4, 2, 256), 5e-6)])
def test_preconditioned_direction_matches_numpy_fft(precision, L, tol):
    from lceqcd_b200 import Lattice
    # alpha exactly representable: FP32 contexts hold the couplings in FP32
    g = Lattice(L, **COUP, precision=precision, alpha=1.25, seed=3)
    g.init_hot(7)
    g.sweeps(3, 0)
    nh = L[0] * L[1] * L[2] // 2
    ident = np.zeros((2, nh, 4), np.float32)
    ident[..., 0] = 1.0
    g.set_transform(ident)
    g.apply_transform()  # U_f = U
    uf, _ = g.download(which=1, dtype=np.float64)
    om = g.debug_fourier_step(step=0.9)
    ref, _ = numpy_direction(uf, L, 1.25, 0.9)
    tol = max(tol, 1e-10 * max(L) ** 2)
    assert np.max(np.abs(om - ref)) <= tol * max(1.0, np.max(np.abs(ref)))


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_fourier_fixing_reaches_the_plain_criterion_and_tracks_the_transform(precision):
    from lceqcd_b200 import Lattice
    L = (16, 16, 16)
    g = Lattice(L, **COUP, precision=precision, limit_or=1e-11, seed=11)
    g.init_hot(3)
    g.sweeps(40, 0)
    th, itf, itp = g.landau_gauge_fourier("identity")
    assert th <= 1e-11 and itf > 1 and itp == 0
    assert g.theta() <= 1e-10
    uf, af = g.download(which=1, dtype=np.float64)
    g.apply_transform()
    uf2, af2 = g.download(which=1, dtype=np.float64)
    tol = 1e-9 if precision == "f64" else 2e-3
    assert np.max(np.abs(uf - uf2)) < tol
    # the tracked transform re-applied to (U, A) is in the Landau gauge; the
    # plain iteration started there stays converged (its overrelaxed first
    # sweeps overshoot, so it takes a few iterations to come back below the
    # limit)
    th0, th1, it1 = g.landau_gauge_from("transform")
    assert th0 <= 1e-10 and th1 <= 1e-11 and it1 < 100


def test_fourier_acceleration_cuts_iterations():
    """The plain iteration from G = 1 against the accelerated one on the same
    configurations at 32^3 (at 16^3 the gain is ~2x; it grows with L because
    the plain iteration's count does and the accelerated one's does not)."""
    from lceqcd_b200 import Lattice
    g = Lattice((32, 32, 32), **COUP, limit_or=1e-10, seed=21)
    g.init_hot(5)
    g.sweeps(60, 0)
    plain, fourier = 0, 0
    for _ in range(2):
        g.sweeps(5, 0)
        _, _, it = g.landau_gauge_from("identity")
        F_plain = g.gauge_functional()
        th, itf, itp = g.landau_gauge_fourier("identity")
        assert th <= 1e-10
        F_fa = g.gauge_functional()
        # both end at a Landau-gauge maximum of similar quality
        assert abs(F_fa - F_plain) < 5e-3
        plain += it
        fourier += itf + itp
    assert 3 * fourier < plain, (fourier, plain)


def test_fourier_needs_power_of_two_extents():
    from lceqcd_b200 import Lattice, LceError
    g = Lattice((8, 8, 12), **COUP, seed=1)
    g.init_hot(1)
    with pytest.raises(LceError):
        g.landau_gauge_fourier("identity")


def test_fourier_from_a_warm_start_and_with_a_plain_finish():
    """From the previous configuration's transform, and with a switch to the
    plain iteration at theta_switch above limit_or."""
    from lceqcd_b200 import Lattice
    g = Lattice((16, 16, 32), **COUP, limit_or=1e-10, seed=8)
    g.init_hot(2)
    g.sweeps(40, 0)
    th, itf, itp = g.landau_gauge_fourier("identity")
    assert th <= 1e-10 and itp == 0
    g.sweeps(3, 0)
    th, itf2, itp2 = g.landau_gauge_fourier("transform")
    assert th <= 1e-10 and itp2 == 0
    g.sweeps(3, 0)
    th, itf3, itp3 = g.landau_gauge_fourier("identity", theta_switch=1e-6)
    assert th <= 1e-10 and itp3 >= 1 and itf3 < itf


def test_fourier_in_a_batch_of_uneven_volumes():
    """Chains of different volumes share the context's buffers; each chain's
    captured iteration graphs stay valid when the others run in between."""
    from lceqcd_b200 import Ensemble, Params
    specs = [Params(L=(16, 16, 16), **COUP, limit_or=1e-10, seed=1),
             Params(L=(32, 16, 8), **COUP, limit_or=1e-10, seed=2),
             Params(L=(8, 8, 8), **COUP, limit_or=1e-10, seed=3)]
    ens = Ensemble(specs)
    ens.init_hot(4)
    ens.sweeps(30, 0)
    for rnd in range(2):
        for c in (2, 0, 1) if rnd else (0, 1, 2):
            th, itf, itp = ens.landau_gauge_fourier("identity" if rnd == 0 else "transform", chain=c)
            assert th <= 1e-10 and itp == 0
            assert ens.theta(chain=c) <= 1e-10
        ens.sweeps(2, 0)
