"""The 3-hit link update of f/agauge1.f (lce_agauge1, and lce_sweep with
agauge_hits = 3) against the oracle's restatement: FP64 validation stream,
Philox stream, and the persistent form against the per-pass kernels."""
import numpy as np
import pytest

from oracle.oracle import Oracle, hot_config, reference_stream

pytestmark = pytest.mark.gpu
lce = pytest.importorskip("lceqcd_b200")
from lceqcd_b200 import Lattice  # noqa: E402

COUP = dict(beta=9.0, x=0.1, y=0.45)


def rel_err(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(1.0, np.max(np.abs(b))))


def pair(L, cfg_seed, **kw):
    u, a = hot_config(L, seed=cfg_seed)
    o = Oracle(L, COUP["beta"], COUP["x"], COUP["y"])
    o.set_fields(u, a)
    g = Lattice(L, **COUP, **kw)
    g.upload(u, a)
    return o, g


@pytest.mark.parametrize("L", [(4, 4, 4), (6, 4, 8)])
def test_agauge1_fp64_stream(L):
    V = L[0] * L[1] * L[2]
    o, g = pair(L, 3, precision="f64", rng="stream")
    stream = reference_stream(2 * 63 * V, seed=2024)  # 6 passes x 3 hits x 7 uniforms x V/2
    o.set_stream(stream)
    g.set_rng_stream(stream)
    for _ in range(2):
        ao, ag = o.agauge1(1), g.agauge1(1)
        assert abs(ao - ag) < 1e-6
        assert rel_err(g.download(dtype=np.float64)[0], o.get_fields()[0]) < 1e-12
        assert abs(o.meas()["plaq"] - g.meas1()["plaq"]) < 1e-12
    assert g.rng_position()[1] == o.stream_pos() == 2 * 63 * V


def test_agauge1_sweep_fp64_stream():
    """lce_sweep with agauge_hits = 3: ahiggs2, ahiggs3, agauge1, renorm."""
    L = (4, 6, 4)
    V = 96
    o, g = pair(L, 5, precision="f64", rng="stream", agauge_hits=3)
    stream = reference_stream(2 * 71 * V, seed=77)  # 7V + V + 63V per sweep
    o.set_stream(stream)
    g.set_rng_stream(stream)
    for _ in range(2):
        o.ahiggs2(1)
        o.ahiggs3(1)
        o.agauge1(1)
        o.renorm()
        mo, mg = o.meas(), g.sweep(1)
        for k in ("plaq", "akin", "a2", "a4", "acc_gauge", "acc_hb", "acc_or"):
            assert abs(mo[k] - mg[k]) <= 1e-11 * max(1, abs(mo[k])), k
    assert rel_err(g.download(dtype=np.float64)[0], o.get_fields()[0]) < 1e-11


def test_agauge1_philox_matches_oracle():
    L = (8, 4, 6)
    o, g = pair(L, 7, precision="f64", rng="philox", seed=12345)
    o.set_philox(12345, 0)
    for _ in range(2):
        o.agauge1(1)
        g.agauge1(1)
    assert g.rng_position()[0] == o.pass_ctr() == 2 * 18
    assert rel_err(g.download(dtype=np.float64)[0], o.get_fields()[0]) < 1e-11


def test_agauge1_persistent_equals_passes():
    res = []
    for mode in ("passes", "persistent"):
        g = Lattice((16, 8, 12), beta=12.0, x=0.09, y=0.3, seed=21, sweep_mode=mode, agauge_hits=3)
        g.init_hot(4)
        p0 = g.rng_position()[0]
        g.sweeps(3, 1)
        res.append((g.download(), g.meas1(), g.rng_position()[0] - p0))
    np.testing.assert_array_equal(res[0][0][0], res[1][0][0])
    assert res[0][1] == res[1][1] and res[0][2] == res[1][2]
    # 3 Philox passes per (parity, mu) of the link update: 4 + 18 per sweep
    assert res[0][2] == 3 * 22
