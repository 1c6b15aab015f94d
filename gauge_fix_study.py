"""Landau gauge fixing of thermalised configurations to theta < limit_or:
the reference's method (overrelaxation from G = 1) against the same
iteration from the previous configuration's converged transform and the
Fourier-accelerated iteration (steepest ascent and conjugate gradients) from
G = 1 and from that transform.

    python gauge_fix_study.py [--L 64] [--configs 4] [--no-plain]

FP32 fields; beta = 12, x = 0.09, y = 0.3, overrelaxation parameter 1.7,
limit 1e-10; configurations 10 sweeps apart on one chain after 200
thermalisation sweeps.  Prints one JSON object: per method the mean
iterations, the mean seconds per configuration (host clock around
synchronised calls) and the mean final functional.
"""
from __future__ import annotations

import argparse
import json
import statistics
import time

from lceqcd_b200.lattice import Lattice


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=64)
    ap.add_argument("--configs", type=int, default=4)
    ap.add_argument("--no-plain", dest="plain", action="store_false",
                    help="skip the overrelaxed fixings (slow at large L)")
    ap.add_argument("--seed", type=int, default=21)
    a = ap.parse_args(argv)
    L = (a.L,) * 3
    g = Lattice(L, beta=12.0, x=0.09, y=0.3, precision="f32", seed=a.seed, lam=1.7, limit_or=1e-10)
    g.init_hot(a.seed + 1)
    g.sweeps(200, 0)
    g.landau_gauge_fourier("identity")  # the chain's first transform
    rows = {k: [] for k in ("plain_identity", "plain_warm", "fourier_identity", "fourier_warm",
                            "fourier_cg_identity", "fourier_cg_warm")}

    def timed(name, fn):
        g.synchronize()
        t0 = time.perf_counter()
        it = fn()
        g.synchronize()
        rows[name].append((it, time.perf_counter() - t0, g.gauge_functional()))

    for _ in range(a.configs):
        g.sweeps(10, 0)
        G = g.get_transform()
        if a.plain:
            timed("plain_identity", lambda: g.landau_gauge()[1])
            g.set_transform(G)
            timed("plain_warm", lambda: g.landau_gauge_from("transform")[2])
        timed("fourier_identity", lambda: sum(g.landau_gauge_fourier("identity")[1:]))
        timed("fourier_cg_identity", lambda: sum(g.landau_gauge_fourier_cg("identity")[1:]))
        g.set_transform(G)
        timed("fourier_warm", lambda: sum(g.landau_gauge_fourier("transform")[1:]))
        g.set_transform(G)
        timed("fourier_cg_warm", lambda: sum(g.landau_gauge_fourier_cg("transform")[1:]))
    out = {"L": a.L, "configs": a.configs, "limit": 1e-10}
    for k, rs in rows.items():
        if rs:
            out[k] = {"mean_iterations": statistics.mean(r[0] for r in rs),
                      "mean_s": statistics.mean(r[1] for r in rs),
                      "mean_functional": statistics.mean(r[2] for r in rs)}
    print(json.dumps(out), flush=True)
    g.close()


if __name__ == "__main__":
    main()
