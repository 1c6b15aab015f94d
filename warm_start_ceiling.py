"""What a warm start must predict to shorten Landau gauge fixing.

    python warm_start_ceiling.py [--L 32] [--configs 6] [--fourier]

On thermalised L^3 configurations (beta = 12, x = 0.09, y = 0.3, 10 sweeps
apart, overrelaxation parameter 1.7, theta < 1e-10) each configuration is
fixed from the previous configuration's converged transform G_prev, giving
its own converged transform G*.  The correction R = G* G_prev^+ is what a
learned warm start would have to predict.  Its Lie-algebra field
theta(x) (R = exp(i theta . sigma)) is split by a Fourier filter into the
modes with |n|^2 <= cut (n the integer lattice momentum) and the rest, and
the same configuration is fixed again from

* G_prev (no prediction),
* exp(theta_low) G_prev: an exact prediction of the long wavelengths only,
* exp(theta_high) G_prev: an exact prediction of the short wavelengths only
  (what a network with a local receptive field can supply),
* exp(s theta) G_prev for s = 0.5, 0.9, 0.99: the whole correction predicted
  with a relative error 1 - s.

All fixings use the reference's overrelaxed iteration (or, with --fourier, the
Fourier-accelerated conjugate-gradient form) to the same theta.  Prints one
JSON object with the mean iterations of each start, i.e. the ceiling of what
any predictor of the correction can gain.
"""
from __future__ import annotations

import argparse
import json
import statistics

import numpy as np

from lceqcd_b200.lattice import Lattice


def natural_index(L):
    """For each parity-split slot (p, s), its natural x-fastest site index."""
    L1, L2, L3 = L
    hx, nxy = L1 // 2, L1 * L2 // 2
    nh = nxy * L3
    s = np.arange(nh)
    z, r = s // nxy, s % nxy
    y, xh = r // hx, r % hx
    out = np.empty((2, nh), np.int64)
    for p in range(2):
        x = 2 * xh + ((p + y + z) & 1)
        out[p] = x + L1 * (y + L2 * z)
    return out


def qmul_nd(u1, u2):
    """U1 U2^+ for SU(2) first rows (Re a, Im a, Re b, Im b), as the library's nd()."""
    a1 = u1[..., 0] + 1j * u1[..., 1]
    b1 = u1[..., 2] + 1j * u1[..., 3]
    a2 = u2[..., 0] + 1j * u2[..., 1]
    b2 = u2[..., 2] + 1j * u2[..., 3]
    a = a1 * np.conj(a2) + b1 * np.conj(b2)
    b = -(a1 * b2) + b1 * a2
    return np.stack([a.real, a.imag, b.real, b.imag], -1)


def qmul_nn(u1, u2):
    a1 = u1[..., 0] + 1j * u1[..., 1]
    b1 = u1[..., 2] + 1j * u1[..., 3]
    a2 = u2[..., 0] + 1j * u2[..., 1]
    b2 = u2[..., 2] + 1j * u2[..., 3]
    a = a1 * a2 - b1 * np.conj(b2)
    b = a1 * b2 + b1 * np.conj(a2)
    return np.stack([a.real, a.imag, b.real, b.imag], -1)


def log_map(q):
    """Unit quaternion (w = Re a; v = Im a, Re b, Im b) -> rotation vector."""
    w, v = q[..., 0], q[..., 1:]
    n = np.linalg.norm(v, axis=-1)
    ang = np.arctan2(n, w)
    f = np.where(n > 1e-12, ang / np.maximum(n, 1e-300), 1.0)
    return v * f[..., None]


def exp_map(t):
    ang = np.linalg.norm(t, axis=-1)
    f = np.where(ang > 1e-12, np.sin(ang) / np.maximum(ang, 1e-300), 1.0)
    return np.concatenate([np.cos(ang)[..., None], t * f[..., None]], -1)


def split_modes(theta, L, idx, cut):
    """theta (2, nh, 3) in parity-split order -> (low, high) parts, |n|^2 <= cut."""
    V = L[0] * L[1] * L[2]
    nat = np.zeros((V, 3))
    nat[idx.ravel()] = theta.reshape(-1, 3)
    f = np.fft.fftn(nat.reshape(L[2], L[1], L[0], 3), axes=(0, 1, 2))
    n3 = [np.fft.fftfreq(n) * n for n in (L[2], L[1], L[0])]
    nz, ny, nx = np.meshgrid(*n3, indexing="ij")
    mask = (nx ** 2 + ny ** 2 + nz ** 2) <= cut
    low = np.fft.ifftn(f * mask[..., None], axes=(0, 1, 2)).real.reshape(V, 3)
    low_ps = low[idx.ravel()].reshape(theta.shape)
    return low_ps, theta - low_ps


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=32)
    ap.add_argument("--configs", type=int, default=6)
    ap.add_argument("--cuts", default="1,3,12")
    ap.add_argument("--fourier", action="store_true", help="fix with the Fourier-accelerated CG form")
    ap.add_argument("--seed", type=int, default=5)
    a = ap.parse_args(argv)
    L = (a.L,) * 3
    g = Lattice(L, beta=12.0, x=0.09, y=0.3, lam=1.7, limit_or=1e-10, seed=a.seed)
    g.init_hot(a.seed + 1)
    g.sweeps(300, 0)
    idx = natural_index(L)

    def fix():
        if a.fourier:
            th, itf, itp = g.landau_gauge_fourier_cg("transform")
            return itf + itp, th
        _, th, it = g.landau_gauge_from("transform", max_iters=2000000)
        return it, th

    g.landau_gauge_from("identity", max_iters=2000000)
    cuts = [int(c) for c in a.cuts.split(",")]
    rows = {"previous": [], "exact": []}
    for c in cuts:
        rows[f"low_n2le{c}"] = []
        rows[f"high_n2gt{c}"] = []
    for s in (0.5, 0.9, 0.99):
        rows[f"scaled_{s}"] = []
    angle = []
    for k in range(a.configs):
        g.sweeps(10, 0)
        Gp = g.get_transform().astype(np.float64)
        it, th = fix()
        rows["previous"].append(it)
        Gs = g.get_transform().astype(np.float64)
        R = qmul_nd(Gs, Gp)
        theta = log_map(R)
        angle.append(float(np.degrees(np.linalg.norm(theta, axis=-1)).mean()))

        def start(Rs):
            g.set_transform(qmul_nn(Rs, Gp).astype(np.float32))
            return fix()[0]

        rows["exact"].append(start(R))
        for c in cuts:
            lo, hi = split_modes(theta, L, idx, c)
            rows[f"low_n2le{c}"].append(start(exp_map(lo)))
            rows[f"high_n2gt{c}"].append(start(exp_map(hi)))
        for s in (0.5, 0.9, 0.99):
            rows[f"scaled_{s}"].append(start(exp_map(s * theta)))
        # the chain goes on from this configuration's own converged transform
        g.set_transform(Gs.astype(np.float32))
    out = {"L": a.L, "configs": a.configs, "iteration": "fourier_cg" if a.fourier else "overrelaxation",
           "mean_rotation_deg_of_the_correction": statistics.mean(angle),
           "mean_iterations": {k: statistics.mean(v) for k, v in rows.items()},
           "iterations": rows}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
