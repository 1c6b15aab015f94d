"""The full production pipeline at scale, end to end on one GPU: an L^3
chain (default 256^3; beta = 16, x = 0.08, y = 0.2) in FP32 with FP64
reunitarisation and sums, each update the link heatbath, 4 link
overrelaxation hits, the Higgs heatbath, overrelaxation and Metropolis steps
(f/main.f:38-41 with the 3 link updates and ahiggs1), meas1 every sweep and
every `--meas-every` sweeps the gauge-fixed measurements of f/main.f:57-79:
warm-started Landau gauge fixing to theta < 1e-10 (the Fourier-accelerated
iteration, conjugate-gradient form unless --no-cg, from the previous
transform or the network's correction of it, whichever starts at the larger
functional) and the z-correlators, Polyakov loop and scalar correlator.

    python pipeline_study.py [--L 256] [--sweeps 100] [--meas-every 20]
        [--therm 200] [--pairs 4] [--judge-L 128]

Before the timed window: `--therm` sweeps from a hot start, the first
transform (Fourier from G = 1), and `--pairs` recorded pairs on which the
network trains (each 20 sweeps + a recorded fixing).  The window of
`--sweeps` sweeps is timed with the host clock around synchronised calls,
split into sweep time and measurement time; `total_2000_sweeps_s`
extrapolates it to a 2000-sweep run measured every 20 sweeps.  The judge is
the plain FP64 path at `--judge-L`^3 with the same couplings and update:
its plaquette and <A^2> against the FP32 run's, with autocorrelation-
corrected errors (z-scores).  Prints one JSON object.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from lceqcd_b200.analysis import mean_err, z_score
from lceqcd_b200.lattice import GaugeNet, Lattice

COUP = dict(beta=16.0, x=0.08, y=0.2)
# algorithmic bytes per site (FP32 storage): a link pass (one parity, one
# direction) 68, a Higgs pass (one parity) 66; the update has 6 link heatbath
# passes, 6 x 4 link overrelaxation passes and 6 Higgs passes
B_LINK, B_HIGGS = 68, 66


def hbm_peak():
    p = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def chain(L, precision, seed, n_or, metro):
    g = Lattice(L, **COUP, precision=precision, seed=seed, lam=1.7, limit_or=1e-10, n_link_or=n_or,
                n_higgs_metro=metro, delta0=0.5)
    g.init_hot(seed + 1)
    return g


def series(g, n):
    rows = [g.sweep(1) for _ in range(n)]
    return np.array([r["plaq"] for r in rows]), np.array([r["a2"] for r in rows])


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=256)
    ap.add_argument("--sweeps", type=int, default=100)
    ap.add_argument("--meas-every", type=int, default=20)
    ap.add_argument("--therm", type=int, default=200)
    ap.add_argument("--pairs", type=int, default=4)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--n-or", type=int, default=4)
    ap.add_argument("--metro", type=int, default=1)
    ap.add_argument("--judge-L", type=int, default=128)
    ap.add_argument("--judge-sweeps", type=int, default=300)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cg", dest="cg", action="store_false")
    a = ap.parse_args(argv)
    L = (a.L,) * 3
    V = a.L ** 3
    peak, peak_kind = hbm_peak()
    out = {"L": a.L, "couplings": COUP, "precision": "f32", "link_or_hits": a.n_or, "higgs_metro": a.metro,
           "cg": a.cg, "sweeps": a.sweeps, "meas_every": a.meas_every, "therm": a.therm, "limit": 1e-10}

    g = chain(L, "f32", a.seed, a.n_or, a.metro)
    g.sweeps(a.therm, 0)
    g.landau_gauge_fourier("identity")  # the chain's first transform
    net = GaugeNet(seed=a.seed + 2)
    t0 = time.perf_counter()
    for _ in range(a.pairs):
        g.sweeps(a.meas_every, 0)
        g.landau_gauge_warm(net, use_net=False, judge=False, record=True, fourier=True)
    loss = net.train(a.epochs, lr=1e-3) if a.pairs else None
    g.synchronize()
    out["net"] = {"pairs": a.pairs, "epochs": a.epochs, "final_loss": loss,
                  "record_and_train_s": time.perf_counter() - t0}

    # the timed window
    t_sweep = t_meas = 0.0
    plaq, a2, gf = [], [], []
    corr = {"corr_a": [], "corr_u": [], "pol": [], "sc": []}
    done = 0
    while done < a.sweeps:
        n = min(a.meas_every, a.sweeps - done)
        g.synchronize()
        t = time.perf_counter()
        for _ in range(n):
            m = g.sweep(1)
            plaq.append(m["plaq"])
            a2.append(m["a2"])
        g.synchronize()
        t_sweep += time.perf_counter() - t
        done += n
        if n == a.meas_every:
            t = time.perf_counter()
            start, F, theta, iters = g.landau_gauge_warm(net, use_net=True, judge=True, fourier=True, cg=a.cg)
            ca, cu, _, _ = g.correlator()
            _, pc, _ = g.polyakov()
            _, sc, _ = g.scalarcorr()
            g.synchronize()
            dt = time.perf_counter() - t
            t_meas += dt
            gf.append({"start": start, "iterations": iters, "theta": theta, "s": dt})
            corr["corr_a"].append(ca[:a.L // 2 + 1])
            corr["corr_u"].append(cu[:a.L // 2 + 1])
            corr["pol"].append(pc[:a.L // 2 + 1])
            corr["sc"].append(sc[:a.L // 2 + 1])
    n_meas = len(gf)
    bps = 6 * B_LINK * (1 + a.n_or) + (4 + 2 * a.metro) * B_HIGGS
    sps = V * a.sweeps / t_sweep
    out["window"] = {
        "sweep_s": t_sweep, "ms_per_sweep": 1e3 * t_sweep / a.sweeps, "site_updates_per_s": sps,
        "bytes_per_site": bps, "sweep_hbm_gbs": sps * bps / 1e9,
        "sweep_frac_of_hbm": sps * bps / 1e9 / peak, "hbm_peak_gbs": peak, "hbm_peak_kind": peak_kind,
        "measurements": n_meas, "meas_s": t_meas, "s_per_measurement": t_meas / n_meas if n_meas else None,
        "gauge_fix": gf, "starts": {s: sum(r["start"] == s for r in gf) for s in ("identity", "transform", "net")},
    }
    if n_meas:
        out["total_2000_sweeps_s"] = 2000 * t_sweep / a.sweeps + (2000 // a.meas_every) * t_meas / n_meas
    out["observables"] = {"plaq": mean_err(np.array(plaq))[:2], "a2": mean_err(np.array(a2))[:2],
                          "corr_a_mean": np.mean(corr["corr_a"], axis=0).tolist() if n_meas else None,
                          "pol_corr_mean": np.mean(corr["pol"], axis=0).tolist() if n_meas else None}
    g.close()
    net.close()

    if a.judge_L > 0:
        t = time.perf_counter()
        j = chain((a.judge_L,) * 3, "f64", a.seed + 10, a.n_or, a.metro)
        j.sweeps(a.therm, 0)
        jp, ja = series(j, a.judge_sweeps)
        j.close()
        mp, ma = mean_err(jp)[:2], mean_err(ja)[:2]
        out["judge"] = {"L": a.judge_L, "precision": "f64", "sweeps": a.judge_sweeps, "plaq": mp, "a2": ma,
                        "z_plaq": z_score(out["observables"]["plaq"], mp),
                        "z_a2": z_score(out["observables"]["a2"], ma), "s": time.perf_counter() - t}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
