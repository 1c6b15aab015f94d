#!/usr/bin/env python
"""Benchmark of the lceqcd Monte Carlo hot path on B200.

Metric: site-updates/s of the heatbath + overrelaxation sweep (the sweep of
f/main.f:38-41: ahiggs2, ahiggs3, agauge, reunitarisation), whole job, on the
single-chain mixed-precision workload: 64^3, beta = 12, x = 0.09, y = 0.3, hot
start, FP32 fields with FP64 reunitarisation and FP64 sums, measurements on
every sweep.  A step is one sweep; L2 is flushed (256 MB write) between timed
steps.  Inputs are synthetic (hot start), there is no dataset.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--no-extras]

N > 1 runs N independent replica chains, one per GPU (the path does not
shard; no collective on the data path), launched by torch.distributed.run.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import signal
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L_MAIN = (64, 64, 64)
COUP = dict(beta=12.0, x=0.09, y=0.3)
METRIC = "site-updates/s (HB+OR sweep)"
UNIT = "site-updates/s"
# algorithmic HBM bytes per lattice site (FP32 fields): one link pass
# (eo, mu) moves 68 B*V, one Higgs pass 66 B*V, the sweep 672 B*V.
B_LINK, B_HIGGS, B_SWEEP = 68, 66, 672


def workload_config(L):
    """The config both arms print (identical dicts, so the two lines name one
    workload): the 64^3 mixed-precision single chain."""
    return {"workload": "single chain 64^3, beta=12, x=0.09, y=0.3, hot start; FP32 fields, FP64 "
                        "reunitarisation and sums; sweep = ahiggs2+ahiggs3+agauge (+renorm), the reference's "
                        "composition",
            "L": list(L), "sites": vol(L),
            "l2": "GPU arm: 256 MB L2 flush between timed steps; CPU arm: no flush (fields 16 MB, host caches)"}
# forward FLOPs per site of the warm-start network: 4 layers of 27 offsets x
# 16 x 16 multiply-adds
NET_FWD_FLOP_PER_SITE = 4 * 27 * 16 * 16 * 2
FALLBACK_HBM_GBS = 6650.0


def vol(L):
    return L[0] * L[1] * L[2]


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_traffic(mode: str):
    """DRAM bytes per launch of the dominant kernel at the headline size, from
    the committed ncu summary (a line `dram_bytes_per_launch[<mode>] = N`)."""
    p = os.path.join(ROOT, "profiles", "sweep_kernels_64cubed.txt")
    try:
        m = re.search(r"dram_bytes_per_launch\[%s\]\s*=\s*([0-9.eE+]+)" % re.escape(mode), open(p).read())
        return float(m.group(1)) if m else None
    except OSError:
        return None


class Clocks:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v for v in vis.split(",") if v.strip()]
        self.index = ids[local_rank] if local_rank < len(ids) else str(local_rank)
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": "nvidia-smi unavailable"}
        time.sleep(0.25)
        self.proc.send_signal(signal.SIGTERM)
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


class NvmlClocks:
    """NVML sampling every ~1 ms (SM clock, clock-event reasons) in a thread,
    for timed regions too short for nvidia-smi's 200 ms interval.  Reads only."""

    REASONS = (("nvmlClocksEventReasonHwSlowdown", "hw_slowdown"),
               ("nvmlClocksEventReasonHwThermalSlowdown", "hw_thermal_slowdown"),
               ("nvmlClocksEventReasonSwThermalSlowdown", "sw_thermal_slowdown"),
               ("nvmlClocksEventReasonSwPowerCap", "sw_power_cap"),
               ("nvmlClocksEventReasonHwPowerBrakeSlowdown", "hw_power_brake_slowdown"))

    def __init__(self, index: str):
        self.index = index
        self.samples = []
        self.thread = None
        self.h = None
        self.nvml = None

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = (pynvml.nvmlDeviceGetHandleByIndex(int(self.index)) if self.index.isdigit()
                      else pynvml.nvmlDeviceGetHandleByUUID(self.index))
        except Exception:
            self.h = None
            return
        self.stop_flag = False

        def run():
            n, h = self.nvml, self.h
            while not self.stop_flag:
                try:
                    self.samples.append((n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM),
                                         n.nvmlDeviceGetCurrentClocksEventReasons(h)))
                except Exception:
                    break
                time.sleep(0.001)

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()

    def stop(self):
        if self.thread is None:
            return None
        self.stop_flag = True
        self.thread.join()
        n = self.nvml
        smax = n.nvmlDeviceGetMaxClockInfo(self.h, n.NVML_CLOCK_SM)
        reasons = set()
        for _, r in self.samples:
            for attr, name in self.REASONS:
                if r & getattr(n, attr, 0):
                    reasons.add(name)
        sm = [s for s, _ in self.samples]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------- GPU arm
def timed_sweeps(lat, K, flush=True):
    """K sweeps, each bracketed by CUDA events on the context stream; L2
    flushed between steps (outside the events).  Returns total device ms."""
    tot = 0.0
    for _ in range(K):
        if flush:
            lat.flush_l2()
        lat.timer_start()
        lat.sweeps(1, 1)
        tot += lat.timer_stop()
    return tot


def settle(lat, measflag=1, limit=60):
    """Untimed sweeps until the library's autotuner has chosen a sweep form
    and tile shape (4 timed sweeps per candidate), so that no timed region
    contains tuning sweeps."""
    n = 0
    while lat.sweep_mode() == "auto" and n < limit:
        lat.sweeps(4, measflag)
        lat.synchronize()
        n += 4
    if lat.sweep_mode() == "auto":
        raise RuntimeError(f"the sweep autotuner has not decided after {n} sweeps")


def kernel_profile(lat, reps=10):
    """Per-pass durations of the sweep, averaged over reps L2-flushed sweeps:
    each sweep runs as a CUDA graph with a timing event after every pass on a
    side stream (lce_profile_sweep), so the passes keep the programmatic
    overlap they have in the timed sweeps; a pass's duration is the time
    between its completion and the previous pass's."""
    acc = None
    for _ in range(reps):
        lat.flush_l2()
        lat.synchronize()
        ms = lat.profile_sweep(1, with_finalize=True)
        acc = ms if acc is None else acc + ms
    return acc / reps


def cpu_baseline(L, budget_s=20.0, warm=1):
    """The oracle (FP32 restatement of the reference, OpenMP over sites in a
    parity pass) on the host cores, time-bounded sample of the workload."""
    import numpy as np
    from oracle.oracle import Oracle, hot_config
    threads = os.cpu_count() or 1
    u, a = hot_config(L, seed=3, dtype=np.float32)
    o = Oracle(L, COUP["beta"], COUP["x"], COUP["y"], bits=32, threads=threads)
    o.set_fields(u, a)
    o.set_philox(3, 0)
    for _ in range(warm):
        o.sweep(1)
    n, t0 = 0, time.perf_counter()
    while True:
        o.sweep(1)
        n += 1
        el = time.perf_counter() - t0
        if el > budget_s or n >= 10000:
            break
    return vol(L) * n / el, threads, n, el


def extras(args, peak):
    """Bounded secondary measurements (rank 0, N = 1)."""
    import numpy as np
    from lceqcd_b200 import Ensemble, Lattice, Params
    out = {}
    # the reference's sweep composition at 128^3 and 256^3, and at 128^3 the
    # production composition of the heatbath + overrelaxation runs (the link
    # heatbath followed by 4 link overrelaxation hits: 4 + 30 passes)
    for L, nor in (((128, 128, 128), 0), ((256, 256, 256), 0), ((128, 128, 128), 4)):
        key = f"sweep_{L[0]}cubed" + (f"_hb_{nor}or" if nor else "")
        try:
            lat = Lattice(L, **COUP, precision="f32", seed=11, n_link_or=nor)
            lat.init_hot(12)
            settle(lat)
            timed_sweeps(lat, 3)
            K = 20 if L[0] <= 128 else 10
            ms = timed_sweeps(lat, K)
            prof = kernel_profile(lat, reps=3)
            link = float(np.mean(prof[4:10])) if len(prof) >= 10 else None
            sps = vol(L) * K / (ms / 1e3)
            bs = B_SWEEP + 6 * nor * B_LINK  # algorithmic bytes per site of this composition
            out[key] = {"site_updates_per_s": sps, "ms_per_sweep": ms / K, "sweep_mode": lat.sweep_mode(),
                        "tile_shape": list(lat.tile_shape(registers=True)),
                        "passes": 10 + 6 * nor, "bytes_per_site": bs,
                        "sweep_hbm_gbs": sps * bs / 1e9, "sweep_frac_of_measured_hbm": sps * bs / 1e9 / peak,
                        "link_kernel_ms": link,
                        "link_kernel_frac_of_measured_hbm": (B_LINK * vol(L) / (link / 1e3) / 1e9 / peak) if link else None}
            lat.close()
        except Exception as e:  # a secondary number must not take the headline down
            out[key] = {"error": repr(e)[:300]}
    # a production run of the headline workload: sweeps back to back through
    # lce_sweeps (graphs of 8 sweeps), measurements on every sweep as in the
    # reference's main loop, one event pair around 160 sweeps, no L2 flush
    try:
        lat = Lattice(L_MAIN, **COUP, precision="f32", seed=1000)
        lat.init_hot(2000)
        settle(lat)
        lat.sweeps(16, 1)
        res = {}
        for mf in (1, 0):
            lat.synchronize()
            lat.timer_start()
            lat.sweeps(160, mf)
            ms = lat.timer_stop() / 160
            res["measured" if mf else "unmeasured"] = {"us_per_sweep": 1e3 * ms,
                                                       "site_updates_per_s": vol(L_MAIN) / (ms / 1e3)}
        out["production_64cubed"] = {**res, "sweep_mode": lat.sweep_mode(),
                                     "tile_shape": list(lat.tile_shape(registers=True)),
                                     "timing": "CUDA events around 160 back-to-back sweeps (lce_sweeps), no L2 "
                                               "flush; measured: measflag 1 on every sweep (f/main.f's production "
                                               "loop), unmeasured: measflag 0 (its thermalisation loop)"}
        lat.close()
    except Exception as e:
        out["production_64cubed"] = {"error": repr(e)[:300]}
    # Landau gauge fixing of thermalised 128^3 configurations (10 sweeps
    # apart) to theta < 1e-10: the reference's method (overrelaxation from
    # G = 1), the same iteration from the previous configuration's converged
    # transform, and the Fourier-accelerated iteration from that transform
    try:
        L = (128, 128, 128)
        lat = Lattice(L, **COUP, precision="f32", seed=21, lam=1.7, limit_or=1e-10)
        lat.init_hot(22)
        lat.sweeps(200, 0)
        lat.landau_gauge_fourier("identity")  # the chain's first transform
        rows = {"plain_identity": [], "plain_warm": [], "fourier_warm": [], "fourier_cg_warm": []}

        def timed(fn):
            # device time between CUDA events on the context stream around the
            # whole fixing (the library's host loop included)
            lat.synchronize()
            lat.timer_start()
            th, it = fn()
            ms = lat.timer_stop()
            return (ms / 1e3, it, th, lat.gauge_functional())

        n_all, n_cg, n_plain_warm = 10, 50, 2
        for k in range(n_cg):
            lat.sweeps(10, 0)
            G = lat.get_transform()
            if k < n_all:
                rows["plain_identity"].append(timed(lambda: lat.landau_gauge(max_iters=300000)))
                if k < n_plain_warm:
                    lat.set_transform(G)
                    rows["plain_warm"].append(
                        timed(lambda: lat.landau_gauge_from("transform", max_iters=300000)[1:]))
                lat.set_transform(G)
                rows["fourier_warm"].append(
                    timed(lambda: (lambda r: (r[0], r[1] + r[2]))(lat.landau_gauge_fourier("transform"))))
                lat.set_transform(G)
            rows["fourier_cg_warm"].append(
                timed(lambda: (lambda r: (r[0], r[1] + r[2]))(lat.landau_gauge_fourier_cg("transform"))))
        gf = {"limit": 1e-10, "omega_or": 1.7,
              "configs": {k: len(v) for k, v in rows.items()},
              "timing": "CUDA events on the context stream around each fixing",
              "configurations": "thermalised 128^3 (beta 12, x 0.09, y 0.3), 10 sweeps apart; plain_identity, "
                                "fourier_warm and the first 10 fourier_cg_warm on the same configurations",
              "warm_start": "from the previous configuration's converged transform; every fixing runs to "
                            "theta < 1e-10"}
        for k, rs in rows.items():
            gf[k] = {"s_per_config": statistics.mean(r[0] for r in rs),
                     "mean_iterations": statistics.mean(r[1] for r in rs),
                     "iterations": [r[1] for r in rs], "theta_max": max(r[2] for r in rs),
                     "functional_mean": statistics.mean(r[3] for r in rs)}
        same = rows["fourier_cg_warm"][:n_all]
        gf["iterations_plain_identity_over_fourier_warm"] = (sum(r[1] for r in rows["plain_identity"]) /
                                                             sum(r[1] for r in rows["fourier_warm"]))
        gf["time_plain_identity_over_fourier_warm"] = (gf["plain_identity"]["s_per_config"] /
                                                       gf["fourier_warm"]["s_per_config"])
        gf["time_plain_identity_over_fourier_cg_warm_same_configs"] = (
            gf["plain_identity"]["s_per_config"] / statistics.mean(r[0] for r in same))
        gf["plain_hbm_gbs"] = statistics.mean(216 * vol(L) * r[1] / r[0] / 1e9 for r in rows["plain_identity"])
        out["gauge_fix_128cubed"] = gf
        lat.close()
    except Exception as e:
        out["gauge_fix_128cubed"] = {"error": repr(e)[:300]}
    # the full production pipeline at 256^3 (beta = 16, x = 0.08, y = 0.2): a
    # sweep is ahiggs2, ahiggs3, one ahiggs1, the agauge heatbath and 4 link
    # overrelaxation hits; a measurement every 20 sweeps is a warm-started
    # Fourier-accelerated Landau gauge fixing (conjugate-gradient form) to
    # theta < 1e-10 and the correlators.  Timed: 20 sweeps + 1 measurement, after thermalisation and a
    # first gauge fixing from G = 1; the 2000-sweep run is projected from them.
    try:
        L = (256, 256, 256)
        lat = Lattice(L, beta=16.0, x=0.08, y=0.2, precision="f32", seed=31, lam=1.7, limit_or=1e-10,
                      n_link_or=4, n_higgs_metro=1)
        lat.init_hot(32)
        lat.sweeps(20, 0)
        lat.landau_gauge_fourier("identity")
        lat.synchronize()
        t0 = time.perf_counter()
        lat.sweeps(19, 0)
        lat.sweep(1)
        lat.synchronize()
        t1 = time.perf_counter()
        th, itf, itp = lat.landau_gauge_fourier_cg("transform")
        lat.correlator()
        lat.synchronize()
        t2 = time.perf_counter()
        ms_sweep = (t1 - t0) / 20 * 1e3
        out["pipeline_256cubed"] = {
            "ms_per_sweep": ms_sweep, "sweep_passes": 4 + 2 + 6 + 24,
            "s_per_measurement": t2 - t1, "gauge_fix_iterations": itf + itp, "theta": th,
            "projected_s_2000_sweeps_100_measurements": 2000 * ms_sweep / 1e3 + 100 * (t2 - t1),
            "site_updates_per_s": vol(L) * 20 / (t1 - t0), "note": "host wall clock around synchronised calls"}
        lat.close()
    except Exception as e:
        out["pipeline_256cubed"] = {"error": repr(e)[:300]}
    # the warm-start network's training at 128^3 (its tcgen05 convolution and
    # weight-gradient kernels): 4 recorded (configuration, transform) pairs,
    # one untimed epoch, then 5 timed epochs of Adam steps (one per pair)
    try:
        from lceqcd_b200 import GaugeNet
        L = (128, 128, 128)
        lat = Lattice(L, **COUP, precision="f32", seed=41, lam=1.7, limit_or=1e-10)
        lat.init_hot(42)
        lat.sweeps(100, 0)
        lat.landau_gauge_fourier("identity")
        net = GaugeNet(seed=43)
        npairs = 4
        for _ in range(npairs):
            lat.sweeps(10, 0)
            lat.landau_gauge_warm(net, use_net=False, judge=False, record=True, fourier=True)
        net.train(1, lr=1e-3)
        epochs = 5
        t0 = time.perf_counter()
        net.train(epochs, lr=1e-3)  # returns after the step's loss is read back
        t = time.perf_counter() - t0
        steps = epochs * npairs
        flop = 3 * NET_FWD_FLOP_PER_SITE * vol(L) * steps  # forward, input gradient, weight gradient
        tf = flop / t / 1e12
        bf16_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("bf16_tflops")
        out["net_train_128cubed"] = {"ms_per_step": t / steps * 1e3, "tflops_bf16": tf, "steps": steps,
                                     "bound": "tensor", "peak_tflops": bf16_peak,
                                     "frac_of_measured_bf16": tf / bf16_peak if bf16_peak else None,
                                     "note": "host wall clock around synchronised training calls; 27 x 16 x 16 "
                                             "per-site contractions, 3 per step",
                                     "judge_rule": "the warm start's judge takes, of the identity, the previous "
                                                   "transform and the network's start, the one with the highest "
                                                   "gauge functional rather than the lowest theta: the previous "
                                                   "transform starts at a worse theta (~7 against "
                                                   "~4.5 from G = 1) yet converges in 1.3-2x fewer iterations; the "
                                                   "plain iteration then runs to theta < limit_or from the start "
                                                   "taken"}
        net.close()
        lat.close()
    except Exception as e:
        out["net_train_128cubed"] = {"error": repr(e)[:300]}
    # z-slab decomposition on one GPU: the 256^3 sweep split into 2 slabs (halo
    # exchange after every pass, launches without a graph) against the same
    # lattice undecomposed -- the cost of the decomposition itself
    try:
        from lceqcd_b200 import SlabLattice
        L = (256, 256, 256)
        g = Lattice(L, **COUP, precision="f32", seed=51, sweep_mode="passes")
        g.init_hot(52)
        u, a = g.download()
        s = SlabLattice(L, 2, **COUP, precision="f32", seed=51)
        s.upload(u, a)
        del u, a

        def wall(fn, n):
            fn()
            t0 = time.perf_counter()
            for _ in range(n):
                fn()
            return (time.perf_counter() - t0) / n * 1e3

        ms_s = wall(lambda: s.sweep(1), 5)  # returns after every slab's stream is synchronised
        ms_g = wall(lambda: g.sweep(1), 5)  # returns after the measurements are read back
        out["slabs_256cubed_one_gpu"] = {"ms_per_sweep_2_slabs": ms_s, "ms_per_sweep_undecomposed": ms_g,
                                         "overhead": ms_s / ms_g - 1.0,
                                         "note": "host wall clock around synchronised sweeps; both on one GPU"}
        s.close()
        g.close()
    except Exception as e:
        out["slabs_256cubed_one_gpu"] = {"error": repr(e)[:300]}
    # the Fourier-accelerated gauge fixing on z-slabs (one GPU): a 128^3
    # configuration 30 sweeps from a hot start fixed from G = 1 to theta <
    # 1e-10 undecomposed and in 2 slabs (per-site stages on every slab, the
    # y/z transforms of the whole lattice's buffer on the first slab's device)
    try:
        from lceqcd_b200 import SlabLattice
        L = (128, 128, 128)
        kw = dict(COUP, precision="f32", seed=61, limit_or=1e-10)
        g = Lattice(L, sweep_mode="passes", **kw)
        g.init_hot(62)
        g.sweeps(30, 0)
        u, a = g.download()
        s = SlabLattice(L, 2, **kw)
        s.upload(u, a)
        del u, a
        res = {}
        for name, fn in (("undecomposed", g.landau_gauge_fourier), ("2_slabs", s.landau_gauge_fourier)):
            fn("identity", max_iters=5000)  # buffers, kernels' attributes
            t0 = time.perf_counter()
            th, itf, itp = fn("identity", max_iters=5000)
            res[name] = {"s_per_fixing": time.perf_counter() - t0, "fourier_iters": itf, "plain_iters": itp,
                         "theta": th}
        res["note"] = "host wall clock around a synchronised fixing; both on one GPU"
        out["slabs_fourier_fix_128cubed_one_gpu"] = res
        s.close()
        g.close()
    except Exception as e:
        out["slabs_fourier_fix_128cubed_one_gpu"] = {"error": repr(e)[:300]}
    # batched ensemble: 96 chains (32 each of 16^3, 32^3, 48^3) over the
    # coupling grid, against the same chains run one context at a time
    try:
        grid = [(b, y, x) for b in (6.0, 9.0, 12.0, 16.0) for y in (0.1, 0.3, 0.5) for x in (0.08, 0.1)]
        specs = []
        for i in range(96):
            b, y, x = grid[i % 24]
            n = (16, 32, 48)[i // 32]
            specs.append(Params(L=(n, n, n), beta=b, x=x, y=y, seed=i + 1))
        sites = sum(vol(s.L) for s in specs)
        ens = Ensemble(specs)
        ens.init_hot(5)
        settle(ens)   # the library's choice of sweep form and tile shape
        timed_sweeps(ens, 3)
        K = 20
        ms_b = timed_sweeps(ens, K)
        ens_mode = ens.sweep_mode()
        ens_tile = list(ens.tile_shape(registers=True))
        ens.close()
        # the plain path: each chain alone in its own context, one kernel per pass
        plain = {}
        for prec in ("f64", "f32"):
            tot = 0.0
            for s in specs:
                g = Lattice(s.L, beta=s.beta, x=s.x, y=s.y, seed=s.seed, precision=prec, sweep_mode="passes")
                g.init_hot(s.seed)
                g.sweeps(2, 1)
                g.synchronize()
                t = timed_sweeps(g, 3, flush=False) / 3
                tot += t
                g.close()
            plain[prec] = sites / (tot / 1e3)
        bat = sites * K / (ms_b / 1e3)
        out["batched_96_chains"] = {"site_updates_per_s": bat, "plain_f64_site_updates_per_s": plain["f64"],
                                    "plain_f32_site_updates_per_s": plain["f32"],
                                    "speedup_vs_plain_f64": bat / plain["f64"], "speedup_vs_plain_f32": bat / plain["f32"],
                                    "sites": sites, "sweep_mode": ens_mode,
                                    "tile_shape": ens_tile}
    except Exception as e:
        out["batched_96_chains"] = {"error": repr(e)[:300]}
    return out


def run_gpu(args):
    import numpy as np
    from lceqcd_b200 import Lattice
    rank, world, local = dist_setup()
    peak, peak_src = peaks()
    L = (args.lattice,) * 3 if args.lattice else L_MAIN
    V = vol(L)
    lat = Lattice(L, **COUP, precision="f32", seed=1000 + rank, device=local, sweep_mode=args.sweep_mode,
                  n_link_or=args.link_or, tile_threads=args.tile_threads, tile_registers=args.tile_registers)
    lat.init_hot(2000 + rank)
    # untimed: the library's autotuner times its candidates (sweep forms x tile
    # shapes, 4 sweeps each) on the first sweeps and keeps the fastest
    settle(lat)
    timed_sweeps(lat, args.warmup)
    lat.synchronize()
    barrier(world)
    clk = Clocks(local)
    fast = NvmlClocks(clk.index)
    if not args.quick:
        clk.start()
        fast.start()
    wall0 = time.perf_counter()
    ms = timed_sweeps(lat, args.steps)
    lat.synchronize()
    wall = time.perf_counter() - wall0
    fast_clocks = fast.stop() if not args.quick else None
    barrier(world)
    clocks = clk.stop() if not args.quick else None
    if clocks is not None and fast_clocks and fast_clocks["samples"]:
        # the ~1 ms NVML samples cover the timed region; nvidia-smi's (every
        # 200 ms, started before it) are kept beside them
        clocks = {**fast_clocks, "source": "nvml, ~1 ms interval, during the timed region",
                  "reasons": sorted(set(fast_clocks["reasons"]) | set(clocks.get("reasons", []))),
                  "nvidia_smi": clocks}
    ms_max = max_over_ranks(ms, world)
    value = world * V * args.steps / (ms_max / 1e3)
    mode = lat.sweep_mode()  # chosen by the library's autotuner during the untimed sweeps
    tile_bs, tile_spt, tile_regs = lat.tile_shape(registers=True)
    # per step: the sweep (one persistent kernel, or 10 pass kernels + finalize)
    # and the two L2-flush kernels
    launches = args.steps * ((1 if mode == "persistent" else 11) + 2)
    if args.quick:
        if rank == 0:
            passes = 4 + 6 * (1 + args.link_or)
            sweep_bytes = B_HIGGS * 4 + B_LINK * 6 * (1 + args.link_or)
            line = {"metric": METRIC, "value": value, "unit": UNIT, "L": list(L), "steps": args.steps,
                    "ms_per_step": ms_max / args.steps, "sweep_mode": mode, "quick": True,
                    "tile_shape": [tile_bs, tile_spt, tile_regs],
                    "link_or": args.link_or, "passes": passes, "bytes_per_site": sweep_bytes,
                    "frac_of_measured_hbm": value * sweep_bytes / 1e9 / peak}
            if args.pass_profile and mode != "persistent":
                line["per_pass_us"] = [round(1e3 * x, 2) for x in kernel_profile(lat, reps=args.pass_profile)]
            print(json.dumps(line), flush=True)
        lat.close()
        return

    # roofline of the dominant kernel: the persistent sweep kernel (672 B*V per
    # launch, one launch per step) when the autotuner chose it, else the link
    # pass kernel (68 B*V per launch, 6 of the 10 passes); per-pass kernel
    # durations come from events between the pass kernels of profiled sweeps
    prof = kernel_profile(lat, reps=10)  # 10 passes, then the finalize kernel
    link_ms = float(np.mean(prof[4:10]))
    # pass 0 also carries the graph's start and the cold L2 after the flush:
    # the Higgs kernel's own duration is the mean of passes 1-3
    higgs_ms = float(np.mean(prof[1:4]))
    first_ms = float(prof[0])
    fin_ms = float(prof[10])
    if mode == "persistent":
        dom_ms, dom_bytes = ms_max / args.steps, B_SWEEP * V
        dom_name = "sweep_persistent_kernel (whole sweep: 4 Higgs + 6 link passes, one cooperative launch)"
    else:
        dom_ms, dom_bytes = link_ms, B_LINK * V
        dom_name = "link_kernel (agauge pass, one parity x one mu" + (
            ", two sites per thread)" if mode == "passes2" else ")")
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    # the same bytes move whether a thread takes one site or two
    traffic = profile_traffic("passes" if mode in ("passes2", "direct") else mode)

    # End to end through the C ABI with pinned host buffers.  A step uploads
    # the configuration (the step's input, lce_upload), runs one measured
    # sweep and reads its measurements back (the step's result, lce_sweep with
    # an lce_meas output).  A second figure adds the download of the updated
    # fields (lce_download), i.e. a driver that keeps host mirrors in sync.
    import torch
    nh = V // 2
    hu = torch.empty((3, 2, nh, 4), dtype=torch.float32, pin_memory=True).numpy()
    ha = torch.empty((2, nh, 3), dtype=torch.float32, pin_memory=True).numpy()
    lat.download_into(hu, ha)
    Ke = max(5, min(args.steps, 50))
    for _ in range(2):
        lat.upload(hu, ha)
        lat.sweep(1)
        lat.download_into(hu, ha)
    barrier(world)
    e2e_ms, rt_ms = 0.0, 0.0
    for _ in range(Ke):
        lat.flush_l2()
        lat.timer_start()
        lat.upload(hu, ha)
        lat.sweep(1)
        e2e_ms += lat.timer_stop()
    for _ in range(Ke):
        lat.flush_l2()
        lat.timer_start()
        lat.upload(hu, ha)
        lat.sweep(1)
        lat.download_into(hu, ha)
        rt_ms += lat.timer_stop()
    # Streaming client: the copy engine moves step k+2's input into a staging
    # slot (lce_upload_stage) while step k sweeps and step k+1's staged input
    # is applied behind it (lce_upload_apply), and step k's measurements are
    # read after its sweep.  Every step still copies its whole input from
    # pinned host memory and reads its result back; one pair of CUDA events
    # spans the Ke steps.
    hu2 = torch.empty(hu.shape, dtype=torch.float32, pin_memory=True).numpy()
    ha2 = torch.empty(ha.shape, dtype=torch.float32, pin_memory=True).numpy()
    hu2[...] = hu
    ha2[...] = ha
    bufs = [(hu, ha), (hu2, ha2)]  # the client refills one while the other is in flight
    lat.upload_async(hu, ha)
    lat.sweeps(1, 1)
    lat.meas1()
    barrier(world)
    lat.synchronize()
    lat.timer_start()
    lat.upload_stage(*bufs[0])
    lat.upload_apply()
    if Ke > 1:
        lat.upload_stage(*bufs[1])
    for k in range(Ke):
        lat.sweeps(1, 1)
        lat.meas1()
        if k + 1 < Ke:
            lat.upload_apply()
        if k + 2 < Ke:
            lat.upload_stage(*bufs[k % 2])
    pipe_ms = lat.timer_stop()
    e2e_ms = max_over_ranks(e2e_ms, world)
    rt_ms = max_over_ranks(rt_ms, world)
    pipe_ms = max_over_ranks(pipe_ms, world)
    e2e_seq = world * V * Ke / (e2e_ms / 1e3)
    e2e_val = world * V * Ke / (pipe_ms / 1e3)
    h2d = hu.nbytes + ha.nbytes
    d2h = 13 * 8  # lce_meas

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (hot start: Haar links, A0 ~ N(0,1))",
        "config": workload_config(L),
        "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
        "wall_s_timed_region": wall,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "note": "streaming client, per step: lce_upload_stage(pinned host fields) two steps ahead, "
                        "lce_upload_apply, lce_sweeps(1, measflag=1), lce_get_meas (the step's measurements "
                        "read back); the copy engine overlaps the sweeps; one event pair over all steps",
                "sequential": {"value": e2e_seq,
                               "note": "per step: lce_upload (returns when copied) + lce_sweep(measflag=1), "
                                       "L2 flushed before each step outside its events"},
                "with_field_download": {"value": world * V * Ke / (rt_ms / 1e3), "d2h_bytes_per_step": d2h + h2d}},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": dom_name, "sweep_mode": mode,
                     "tile_shape": {"threads_per_block": tile_bs, "sites_per_thread": tile_spt,
                                    "register_cap": tile_regs,
                                    "chosen_by": "the library's autotuner" if args.sweep_mode == "auto"
                                    else f"--sweep-mode {args.sweep_mode}"},
                     "algorithmic_bytes_per_launch": dom_bytes, "avg_launch_ms": dom_ms,
                     "peak_source": f"{peak_src} (MEASURED_PEAKS.json hbm_gbs)" if peak_src == "measured" else "fallback",
                     "pass_kernels": {"link_kernel_ms": link_ms, "link_kernel_frac": B_LINK * V / (link_ms / 1e3) / 1e9 / peak,
                                      "higgs_kernel_ms": higgs_ms,
                                      "higgs_kernel_frac": B_HIGGS * V / (higgs_ms / 1e3) / 1e9 / peak,
                                      "finalize_kernel_ms": fin_ms,
                                      "first_pass_ms": first_ms,
                                      "per_pass_ms": [float(x) for x in prof],
                                      "share_of_sweep": {"link_passes": 6 * link_ms / float(np.sum(prof)),
                                                         "higgs_passes_1_3": 3 * higgs_ms / float(np.sum(prof)),
                                                         "first_pass": first_ms / float(np.sum(prof)),
                                                         "finalize": fin_ms / float(np.sum(prof))},
                                      "timing": "CUDA events hung off each pass of a sweep graph on a side stream "
                                                "(the passes keep their programmatic overlap); a pass's time is "
                                                "its completion minus the previous pass's (pass 0 from the graph "
                                                "start, after an L2 flush)"},
                     "sweep_frac": value / world * B_SWEEP / 1e9 / peak},
        "clocks": clocks,
    }
    if rank == 0 and world == 1:
        try:
            v, cores, n, el = cpu_baseline(L, budget_s=args.cpu_budget)
            line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                                    "sample": f"{n} full {L[0]}^3 sweeps ({el:.1f} s) of the FP32 oracle restatement "
                                              f"of the reference (OpenMP over sites, {cores} threads)"}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "port", "sample": repr(e)[:200]}
        if args.extras:
            line["secondary"] = extras(args, peak)
            # the larger volumes' sweep and link-kernel fractions, beside the
            # headline kernel's (the same figures as in secondary)
            byvol = {}
            for key in ("sweep_128cubed", "sweep_256cubed", "sweep_128cubed_hb_4or"):
                r = line["secondary"].get(key, {})
                if "sweep_frac_of_measured_hbm" in r:
                    byvol[key] = {"sweep_frac": r["sweep_frac_of_measured_hbm"],
                                  "link_kernel_frac": r["link_kernel_frac_of_measured_hbm"],
                                  "tile_shape": r.get("tile_shape"), "sweep_mode": r.get("sweep_mode")}
            line["roofline"]["by_volume"] = byvol
    lat.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------- reference arm
def run_reference(args):
    """The reference's CPU implementation of the path: the Fortran/MPI
    reference cannot be compiled in this image (no gfortran, no MPI), so this
    times the oracle port (FP32 restatement, OpenMP) on the host cores, on
    the same 64^3 workload; one step = one sweep."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import numpy as np
    from oracle.oracle import Oracle, hot_config
    threads = os.cpu_count() or 1
    u, a = hot_config(L_MAIN, seed=3, dtype=np.float32)
    o = Oracle(L_MAIN, COUP["beta"], COUP["x"], COUP["y"], bits=32, threads=threads)
    o.set_fields(u, a)
    o.set_philox(3, 0)
    t0 = time.perf_counter()
    o.sweep(1)
    t1 = time.perf_counter() - t0
    budget = 150.0
    W = min(args.warmup, max(1, int(20 / max(t1, 1e-3))))
    for _ in range(W):
        o.sweep(1)
    K = min(args.steps, max(1, int(budget / max(t1, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(K):
        o.sweep(1)
    el = time.perf_counter() - t0
    v = vol(L_MAIN) * K / el
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (hot start)", "impl": "reference",
            "config": workload_config(L_MAIN),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{K} of {args.steps} steps timed (bounded to ~{budget:.0f} s), each a full "
                                       "64^3 sweep of the FP32 oracle restatement (the Fortran reference has no "
                                       "compiler in this image)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def quick_gauge_fix(args):
    """The Fourier-accelerated gauge fixing as a profiling case: args.quick_gauge_fix
    iterations (7 kernel launches each; 11 for the conjugate-gradient form with
    --gauge-fix-cg) from G = 1, stopped by the iteration cap."""
    from lceqcd_b200 import Lattice, LceError
    n = args.lattice or 128
    lat = Lattice((n, n, n), **COUP, precision="f32", seed=21, lam=1.7, limit_or=1e-10)
    lat.init_hot(22)
    lat.sweeps(20, 0)
    lat.synchronize()
    t0 = time.perf_counter()
    try:
        if args.gauge_fix_cg:
            lat.landau_gauge_fourier_cg("identity", max_iters=args.quick_gauge_fix)
        else:
            lat.landau_gauge_fourier("identity", max_iters=args.quick_gauge_fix)
    except LceError as e:
        if e.code != -3:  # LCE_ERR_GF_NOT_CONVERGED: the cap stopped it, as intended
            raise
    lat.synchronize()
    print(json.dumps({"quick_gauge_fix": args.quick_gauge_fix, "cg": args.gauge_fix_cg, "L": n,
                      "theta": lat.theta(), "s": time.perf_counter() - t0}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="lceqcd_b200", choices=["lceqcd_b200", "reference"])
    ap.add_argument("--no-extras", dest="extras", action="store_false")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--quick", action="store_true",
                    help="timed sweeps only (no e2e, CPU baseline, extras or clocks): the ncu profiling case")
    ap.add_argument("--lattice", type=int, default=0, help="cubic extent for --quick runs (default 64)")
    ap.add_argument("--sweep-mode", default="auto", choices=["auto", "passes", "passes2", "persistent", "direct"],
                    help="sweep form (default: the library's autotuner chooses)")
    ap.add_argument("--tile-registers", type=int, default=0, choices=[0, 56],
                    help="register cap of the update kernels (56 needs --tile-threads 128)")
    ap.add_argument("--tile-threads", type=int, default=0, choices=[0, 128, 256, 448, 512],
                    help="threads per block of the update kernels (default 0: the autotuner chooses with "
                         "--sweep-mode auto, else 256)")
    ap.add_argument("--pass-profile", type=int, default=0, metavar="REPS",
                    help="--quick runs: also print the per-pass durations inside the sweep graph (the last: "
                         "the finalize kernel), averaged over REPS L2-flushed sweeps")
    ap.add_argument("--link-or", type=int, default=0, metavar="N",
                    help="--quick runs: N link overrelaxation hits per sweep after the heatbath")
    ap.add_argument("--quick-gauge-fix", type=int, default=0, metavar="ITERS",
                    help="profiling case: ITERS Fourier-accelerated gauge-fixing iterations on a thermalised "
                         "--lattice^3 FP32 configuration, then exit")
    ap.add_argument("--gauge-fix-cg", action="store_true",
                    help="with --quick-gauge-fix: the conjugate-gradient form")
    args = ap.parse_args()
    if args.quick_gauge_fix:
        quick_gauge_fix(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if (args.lattice or args.link_or) and not (args.quick or args.quick_gauge_fix):
        ap.error("--lattice / --link-or only apply to --quick profiling runs; the headline workload is the "
                 "standard 64^3 sweep")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
