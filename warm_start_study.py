"""Learned warm start for Landau gauge fixing, measured on the Landau-gauge
workload: thermalised L^3 configurations (beta = 12, x = 0.09, y = 0.3, 10
sweeps apart), overrelaxation parameter 1.7, theta < 1e-10.

    python warm_start_study.py [--L 128] [--pairs 400] [--test 50] [--epochs 10] [--cg]

Records `pairs` training pairs from the Fourier-accelerated fixing started at
the previous configuration's transform, trains the network on the device,
then fixes `test` new configurations from (a) the previous transform, (b) the
network's correction of it, (c) the judge's choice among identity / previous
/ network, all with the Fourier-accelerated iteration, and the first
`--plain` of them also with the reference's method (overrelaxation from
G = 1).  Prints one JSON object with iterations, times, functionals and the
network's training throughput.
"""
from __future__ import annotations

import argparse
import json
import statistics
import time

from lceqcd_b200.lattice import GaugeNet, Lattice

# forward FLOPs per site of the network: 4 layers of 27 offsets x 16 x 16
# multiply-adds (the last layer computes 16 outputs of which 4 are used)
FWD_FLOP_PER_SITE = 4 * 27 * 16 * 16 * 2


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--L", type=int, default=128)
    ap.add_argument("--pairs", type=int, default=400)
    ap.add_argument("--test", type=int, default=50)
    ap.add_argument("--plain", type=int, default=3)
    ap.add_argument("--epochs", type=int, default=10)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=3)
    ap.add_argument("--cg", action="store_true",
                    help="test fixings by the conjugate-gradient form (recording stays steepest ascent)")
    a = ap.parse_args(argv)
    L = (a.L,) * 3
    V = a.L ** 3
    g = Lattice(L, beta=12.0, x=0.09, y=0.3, lam=1.7, limit_or=1e-10, seed=a.seed)
    g.init_hot(a.seed + 1)
    g.sweeps(300, 0)
    g.landau_gauge_fourier("identity")
    net = GaugeNet(seed=a.seed + 2)

    t0 = time.perf_counter()
    rec_iters = []
    for _ in range(a.pairs):
        g.sweeps(10, 0)
        rec_iters.append(g.landau_gauge_warm(net, use_net=False, judge=False, record=True, fourier=True)[3])
    t_rec = time.perf_counter() - t0

    losses = []
    t0 = time.perf_counter()
    for _ in range(a.epochs):
        losses.append(net.train(1, lr=a.lr))
    t_train = time.perf_counter() - t0
    steps = a.epochs * a.pairs
    # forward + input gradient + weight gradient: three contractions of the forward's size
    train_tflops = 3 * FWD_FLOP_PER_SITE * V * steps / t_train / 1e12

    rows = {"fourier_previous": [], "fourier_network": [], "fourier_judge": [], "plain_identity": []}
    judged = {"identity": 0, "transform": 0, "net": 0}

    def run(name, fn):
        g.synchronize()
        t = time.perf_counter()
        it = fn()
        g.synchronize()
        rows[name].append((it, time.perf_counter() - t, g.gauge_functional()))

    def judge():
        start, _, _, it = g.landau_gauge_warm(net, use_net=True, judge=True, fourier=True, cg=a.cg)
        judged[start] += 1
        return it

    for k in range(a.test):
        g.sweeps(10, 0)
        G = g.get_transform()
        run("fourier_previous",
            lambda: g.landau_gauge_warm(net, use_net=False, judge=False, fourier=True, cg=a.cg)[3])
        g.set_transform(G)
        run("fourier_network",
            lambda: g.landau_gauge_warm(net, use_net=True, judge=False, fourier=True, cg=a.cg)[3])
        g.set_transform(G)
        run("fourier_judge", judge)
        if k < a.plain:
            run("plain_identity", lambda: g.landau_gauge(max_iters=1000000)[1])
        # the chain continues from the previous-transform result
        g.set_transform(G)
        g.landau_gauge_warm(net, use_net=False, judge=False, fourier=True)

    out = {"L": a.L, "pairs": a.pairs, "test_configs": a.test, "epochs": a.epochs, "cg": a.cg,
           "record_s": t_rec, "record_mean_iterations": statistics.mean(rec_iters),
           "train_s": t_train, "train_steps": steps, "train_tflops_bf16": train_tflops,
           "loss_per_epoch": losses, "judge_choices": judged}
    for k, rs in rows.items():
        if rs:
            out[k] = {"configs": len(rs), "mean_iterations": statistics.mean(r[0] for r in rs),
                      "mean_s": statistics.mean(r[1] for r in rs),
                      "mean_functional": statistics.mean(r[2] for r in rs)}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
