"""The GPU's FP64 validation path against the reference's own routines.

Replays the scripts of ``tests/golden/reference_runs.npz`` (what the
reference's unmodified Fortran computed, see tests/test_oracle_vs_reference.py)
on a Lattice with precision="f64" and rng="stream" through the C ABI, and
compares every recorded return value, field and stream position at 1e-12
relative, integers exactly.  This includes a 16^3 sweep at the plain-method
workload's couplings (beta = 9, x = 0.1, y = 0.45).

The gauge-fixing angle is the reference's acos of Re Omega
(f/or_gauge_fixing1.f:174), not the library's default atan2.  Not replayed
here: the single-iteration steps ``or_gauge_fixing`` and ``u_f_renorm`` (the
C ABI runs them only inside ``lce_landau_gauge``), the couplings and neighbour
tables (host functions of the library, replayed without a GPU in
tests/test_oracle_vs_reference.py), and the FP32 case (the FP32 production path uses
fast single-precision exp/log, so near-tie Metropolis decisions may differ
from the reference's; it is compared statistically in
tests/test_gpu_ensembles.py).
"""
import numpy as np
import pytest

from reference_cases import (CASES, FIELD_STEPS, apply_step, compare_arrays, compare_ret, inputs_sha256,
                             load_fixture, record_state)

pytestmark = pytest.mark.gpu
lce = pytest.importorskip("lceqcd_b200")
from lceqcd_b200 import Lattice  # noqa: E402

TOL64 = 1e-12
UNSUPPORTED = {"or_gauge_fixing", "u_f_renorm", "couplings", "tables"}
Z, MANIFEST = load_fixture()


class GpuLattice:
    """The GPU Lattice behind the method names the scripts use."""

    def __init__(self, p):
        self.g = Lattice(p["L"], beta=p["beta"], x=p["x"], y=p["y"], precision="f64", rng="stream",
                         lam=p.get("lam", 1.8), alpha=p.get("alpha", 1.0), limit_or=p.get("limit_or", 1e-9),
                         imode=p.get("imode", 0), gf_angle="acos", device=0)
        self.nh = self.g.nh()
        self._staple = np.zeros((3, 2, self.nh, 4))
        self._force = None
        self.landau_copy = None          # apply_step: call landau_gauge(0), no cap

    def close(self):
        self.g.close()

    def set_fields(self, u, a):
        self.g.upload(u, a)

    def set_stream(self, s):
        self.g.set_rng_stream(s)

    def stream_pos(self):
        return self.g.rng_position()[1]

    def get_fields(self, which=0):
        return self.g.download(which=which, dtype=np.float64)

    def meas(self):
        return self.g.meas1()

    def __getattr__(self, name):
        if name in ("ahiggs1", "ahiggs2", "ahiggs3", "agauge", "agauge1", "renorm", "sweep", "landau_gauge",
                    "polyakov", "scalarcorr", "meas2"):
            return getattr(self.g, name)
        raise AttributeError(name)

    def staples(self, eo, mu):
        self._staple[mu, eo] = self.g.debug_staple(eo, mu)

    def staple(self):
        return self._staple

    def a_force(self, eo):
        self._force = self.g.debug_force(eo)

    def force(self):
        return self._force

    def correlator(self):
        ca, cu, c3, _ = self.g.correlator()
        return ca, cu, c3

    def it_gauge_fixing(self, step, flags):
        assert flags == 0
        return self.g.it_gauge_fixing(step)


GPU_CASES = [c for c in CASES
             if c["params"].get("real_kind", 8) == 8 and not any(s[0] in UNSUPPORTED for s in c["steps"])]


@pytest.mark.parametrize("case", GPU_CASES, ids=[c["name"] for c in GPU_CASES])
def test_gpu_replays_reference(case):
    rec = MANIFEST[case["name"]]
    u, a, stream = case["inputs"]()
    assert inputs_sha256(u, a, stream) == rec["inputs_sha256"]
    g = GpuLattice(rec["params"])
    try:
        g.set_fields(u, a)
        g.set_stream(stream)
        for k, (step, r) in enumerate(zip(case["steps"], rec["steps"])):
            name = step[0]
            got = apply_step(g, step)
            measflag0 = name in FIELD_STEPS and name != "renorm" and len(step) > 1 and step[-1] == 0
            if not measflag0:
                # acceptance rates come back as the reference's REAL
                tol = 1e-6 if name in ("ahiggs1", "ahiggs2", "ahiggs3", "agauge", "agauge1") else TOL64
                compare_ret(got, r["ret"], tol, f"{case['name']}[{k}] {name}")
            assert g.stream_pos() == r["stream_pos"], f"{case['name']}[{k}] {name}: stream position"
            compare_arrays(record_state(g, step), Z, f"{case['name']}/{k}", TOL64)
    finally:
        g.close()


def test_gpu_cases_cover_the_reference_scripts():
    assert {c["name"] for c in GPU_CASES} >= {"sweep_imode0", "sweep_imode1", "sweep_c2_couplings", "routines",
                                               "agauge1", "gauge_fix", "it_gauge_fixing", "sweep_16cubed"}
