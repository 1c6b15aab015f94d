"""Scripts of reference calls shared by the golden-fixture generator
(tests/golden/make_reference_runs.py, which runs them on the reference's own
Fortran through oracle/fortran_runner.py) and the tests that replay them on the
oracle and on the GPU.

A step is a JSON list ``[method, *args]``; the method names are the
reference's subroutine names, which oracle.Oracle and
oracle.fortran_reference.FortranLattice share.
"""
from __future__ import annotations

import numpy as np

from oracle.oracle import hot_config, reference_stream, uniforms_per_sweep

C1 = dict(beta=9.0, x=0.1, y=0.45)        # the plain-method workload's couplings
C2 = dict(beta=12.0, x=0.09, y=0.3)       # the 64^3 mixed-precision workload's couplings

FIELD_STEPS = {"ahiggs1", "ahiggs2", "ahiggs3", "agauge", "agauge1", "renorm", "sweep"}
FIXED_STEPS = {"landau_gauge", "or_gauge_fixing", "u_f_renorm", "it_gauge_fixing"}


def _inputs(L, seed, stream_seed, sweeps, dtype=np.float64):
    def make():
        u, a = hot_config(L, seed=seed)
        n = int(sweeps * uniforms_per_sweep(L)) + 64
        s = reference_stream(n, seed=stream_seed)
        return u.astype(dtype).astype(np.float64), a.astype(dtype).astype(np.float64), s
    return make


def _case(name, L, params, seed, stream_seed, sweeps, steps, dtype=np.float64):
    p = dict(params)
    p["L"] = list(L)
    return {"name": name, "params": p, "inputs": _inputs(L, seed, stream_seed, sweeps, dtype), "steps": steps}


CASES = [
    _case("sweep_imode0", (4, 6, 8), C1, 1, 314159, 2.2,
          [["ahiggs2", 1], ["ahiggs3", 1], ["agauge", 1], ["renorm"], ["sweep", 1]]),
    _case("sweep_imode1", (4, 6, 8), dict(C1, imode=1), 2, 271828, 2.2,
          [["ahiggs2", 1], ["ahiggs3", 1], ["agauge", 1], ["renorm"], ["sweep", 1]]),
    _case("sweep_c2_couplings", (6, 4, 8), C2, 4, 4242, 2.2,
          [["sweep", 1], ["ahiggs2", 0], ["ahiggs3", 0], ["agauge", 0], ["renorm"]]),
    _case("routines", (4, 4, 6), C1, 3, 99, 1.2,
          [["staples", 0, 0], ["staples", 0, 1], ["staples", 0, 2], ["staples", 1, 0], ["staples", 1, 1],
           ["staples", 1, 2], ["a_force", 0], ["a_force", 1], ["ahiggs1", 0.75, 1], ["ahiggs1", 5.0, 1],
           ["ahiggs1", 0.0625, 1]]),
    _case("agauge1", (4, 4, 6), dict(C1, agauge1=True), 5, 11, 4.6,
          [["agauge1", 1], ["renorm"], ["agauge1", 1]]),
    _case("gauge_fix", (4, 6, 8), dict(C1, lam=1.7, limit_or=1e-6), 6, 2024, 2.2,
          [["sweep", 1], ["sweep", 1], ["landau_gauge"], ["correlator"], ["polyakov"], ["scalarcorr"],
           ["meas2"]]),
    _case("gauge_fix_steps", (4, 4, 6), dict(C1, lam=1.8, limit_or=5000.0), 7, 1, 0.1,
          [["landau_gauge"], ["or_gauge_fixing"], ["u_f_renorm"], ["or_gauge_fixing"], ["u_f_renorm"],
           ["correlator"]]),
    _case("it_gauge_fixing", (4, 4, 6), dict(C1, alpha=0.1, limit_or=5000.0), 8, 1, 0.1,
          [["landau_gauge"], ["it_gauge_fixing", 0.1, 0], ["it_gauge_fixing", 0.1, 0],
           ["it_gauge_fixing", 0.1, 0]]),
    _case("sweep_16cubed", (16, 16, 16), C1, 12345, 314159, 1.0, [["sweep", 1]]),
    _case("couplings_c1", (4, 4, 4), C1, 1, 1, 0.1, [["couplings"], ["tables"]]),
    _case("couplings_c2", (4, 4, 4), C2, 1, 1, 0.1, [["couplings"]]),
    _case("couplings_pipeline", (4, 4, 4), dict(beta=16.0, x=0.08, y=0.2), 1, 1, 0.1, [["couplings"]]),
    _case("couplings_grid", (4, 4, 4), dict(beta=6.0, x=0.08, y=0.1), 1, 1, 0.1, [["couplings"]]),
    _case("tables", (6, 4, 8), C1, 1, 1, 0.1, [["tables"]]),
    _case("sweep_fp32", (4, 4, 6), dict(C1, real_kind=4), 1, 314159, 2.2, [["sweep", 1], ["sweep", 1]],
          dtype=np.float32),
]


def inputs_sha256(u, a, stream) -> str:
    import hashlib
    h = hashlib.sha256()
    for arr in (u, a, stream):
        h.update(np.ascontiguousarray(arr, np.float64).tobytes())
    return h.hexdigest()


def _jsonable(x):
    if isinstance(x, (tuple, list)):
        return [_jsonable(v) for v in x]
    if isinstance(x, dict):
        return {k: _jsonable(v) for k, v in x.items()}
    if isinstance(x, np.ndarray):
        return x.tolist()
    if isinstance(x, (np.integer,)):
        return int(x)
    if isinstance(x, (np.floating,)):
        return float(x)
    return x


def apply_step(obj, step):
    """Call one step on an oracle.Oracle or a FortranLattice; return a
    JSON-able result in one canonical form for both."""
    name, args = step[0], step[1:]
    if name == "it_gauge_fixing":
        ret = obj.it_gauge_fixing(*args)
    elif name == "landau_gauge" and hasattr(obj, "landau_copy"):
        ret = obj.landau_gauge(0)           # the oracle: no iteration cap, as the reference
    elif name in ("polyakov", "scalarcorr"):
        r = getattr(obj, name)()
        ret = {"corr": r[1], "mean": r[2]}  # (slice means, correlator, first value written)
    elif name == "correlator":
        ca, cu, c3 = obj.correlator()
        ret = {"corr_a": ca, "corr_u": cu, "corr_3": c3}
    elif name == "tables":
        up, dn = obj.tables()
        ret = {"siteup": up, "sitedn": dn}
    else:
        ret = getattr(obj, name)(*args)
    return _jsonable(ret)


def record_state(obj, step):
    """Arrays that a step may change."""
    name = step[0]
    out = {}
    if name in FIELD_STEPS:
        u, a = obj.get_fields(0)
        out["u"], out["a"] = u, a
    if name in FIXED_STEPS:
        u, a = obj.get_fields(1)
        out["u_f"], out["a_f"] = u, a
    if name == "staples":
        eo, mu = step[1], step[2]
        out["staple"] = np.asarray(obj.staple())[mu, eo]
    if name == "a_force":
        out["force"] = np.asarray(obj.force())
    # /aver_loc/ after a measflag = 1 call, the quantities that call sets
    # (measflag = 0 calls zero the sums and leave them so; f/main.f:20-25
    # never reads them after those)
    if name in FIELD_STEPS and name != "renorm" and step[-1] == 1:
        m = obj.meas()
        keys = {"sweep": ("plaq", "akin", "a2", "a4"), "agauge": ("plaq",), "agauge1": ("plaq",)}.get(
            name, ("akin", "a2", "a4"))
        out["meas"] = np.array([m[k] for k in keys])
    return out


# ---------------------------------------------------------------------------
# replay

FIXTURE = __import__("os").path.join(__import__("os").path.dirname(__import__("os").path.abspath(__file__)),
                                     "golden", "reference_runs.npz")


def load_fixture():
    import json
    z = np.load(FIXTURE)
    manifest = json.loads(bytes(z["manifest"]).decode())
    return z, manifest


def case_by_name(name):
    for c in CASES:
        if c["name"] == name:
            return c
    raise KeyError(name)


def rel_err(x, ref):
    x, ref = np.asarray(x, np.float64), np.asarray(ref, np.float64)
    return float(np.max(np.abs(x - ref)) / max(1.0, float(np.max(np.abs(ref)))))


def compare_ret(got, want, tol, path="ret"):
    """Recorded return values against a replay's; integers and index tables
    exactly, reals to tol relative (scale: max(1, |values|))."""
    if want is None:
        return
    if isinstance(want, dict):
        for k, v in want.items():
            compare_ret(got[k], v, tol, f"{path}.{k}")
        return
    if isinstance(want, list) and want and isinstance(want[0], list) or path.endswith(("siteup", "sitedn")):
        assert np.array_equal(np.asarray(got), np.asarray(want)), path
        return
    if isinstance(want, list):
        assert len(got) == len(want), path
        for i, (g, w) in enumerate(zip(got, want)):
            compare_ret(g, w, tol, f"{path}[{i}]")
        return
    if isinstance(want, int) and not isinstance(want, bool):
        assert int(got) == want, f"{path}: {got} != {want}"
        return
    w = float(want)
    assert abs(float(got) - w) <= tol * max(1.0, abs(w)), f"{path}: {got} != {w} (tol {tol})"


def compare_arrays(got: dict, z, prefix, tol):
    for key, val in got.items():
        want = z[f"{prefix}/{key}"]
        err = rel_err(val, want)
        assert err <= tol, f"{prefix}/{key}: relative error {err:.3e} > {tol}"
