"""The oracle against the reference's own routines.

``tests/golden/reference_runs.npz`` holds what the reference's unmodified
Fortran computed (executed by oracle/fortran_runner.py, set up as
f/initialize.f does, on seeded hot configurations and a seeded RANLUX stream):
sweeps in both heatbath modes and at two coupling sets, the staples and
forces, ahiggs1 with its step adaptation, the 3-hit agauge1, the overrelaxed
Landau gauge fixing to convergence and step by step, the reference's
iterative gauge fixing, correlators, Polyakov and scalar correlators, meas2,
the couplings of paraminit and the neighbour tables of adresses, and a 16^3
sweep at the plain-method workload's couplings.

Every script is replayed on the FP64 oracle with the same inputs and stream
and compared at 1e-12 relative (max |x - ref| / max(1, max |ref|)), the
tolerance of the plain FP64 path; integers (iteration counts, stream
positions, neighbour tables) exactly.  The FP32 case compares the FP32 oracle
with the reference run at default REAL: 2e-5 on fields and 2e-6 on
measurements, because the FP32 oracle accumulates its sums in double where
the reference accumulates in single.
"""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from reference_cases import (CASES, FIELD_STEPS, apply_step, compare_arrays, compare_ret, inputs_sha256,
                             load_fixture, record_state)

TOL64 = 1e-12
TOL32_FIELDS, TOL32_MEAS = 2e-5, 2e-6

Z, MANIFEST = load_fixture()


def make_oracle(p):
    return Oracle(p["L"], p["beta"], p["x"], p["y"], lam=p.get("lam", 1.8), alpha=p.get("alpha", 1.0),
                  limit_or=p.get("limit_or", 1e-9), imode=p.get("imode", 0),
                  bits=32 if p.get("real_kind", 8) == 4 else 64)


def test_fixture_covers_every_case():
    assert sorted(MANIFEST) == sorted(c["name"] for c in CASES)


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_oracle_replays_reference(case):
    rec = MANIFEST[case["name"]]
    p = rec["params"]
    u, a, stream = case["inputs"]()
    assert inputs_sha256(u, a, stream) == rec["inputs_sha256"], "regenerated inputs differ from the fixture's"
    fp32 = p.get("real_kind", 8) == 4
    o = make_oracle(p)
    o.set_fields(u, a)
    o.set_stream(stream)
    for k, (step, r) in enumerate(zip(case["steps"], rec["steps"])):
        assert step == r["call"]
        name = step[0]
        got = apply_step(o, step)
        measflag0 = name in FIELD_STEPS and name != "renorm" and len(step) > 1 and step[-1] == 0
        if not measflag0:
            compare_ret(got, r["ret"], TOL32_MEAS if fp32 else TOL64, f"{case['name']}[{k}] {name}")
        assert o.stream_pos() == r["stream_pos"], f"{case['name']}[{k}] {name}: stream position"
        state = record_state(o, step)
        if fp32:
            meas = state.pop("meas", None)
            compare_arrays(state, Z, f"{case['name']}/{k}", TOL32_FIELDS)
            if meas is not None:
                compare_arrays({"meas": meas}, Z, f"{case['name']}/{k}", TOL32_MEAS)
        else:
            compare_arrays(state, Z, f"{case['name']}/{k}", TOL64)


@pytest.mark.skipif(not os.environ.get("LCEQCD_REFERENCE"),
                    reason="LCEQCD_REFERENCE names no checkout of the reference")
def test_reference_reruns_to_the_fixture():
    """With a checkout named in LCEQCD_REFERENCE, re-run one script on the
    reference through the interpreter and get the fixture back."""
    from oracle.fortran_reference import FortranLattice
    case = next(c for c in CASES if c["name"] == "sweep_imode0")
    rec = MANIFEST[case["name"]]
    p = rec["params"]
    f = FortranLattice(os.environ["LCEQCD_REFERENCE"], p["L"], p["beta"], p["x"], p["y"])
    u, a, stream = case["inputs"]()
    f.set_fields(u, a)
    f.set_stream(stream)
    for k, (step, r) in enumerate(zip(case["steps"], rec["steps"])):
        compare_ret(apply_step(f, step), r["ret"], 0.0)
        compare_arrays(record_state(f, step), Z, f"{case['name']}/{k}", 0.0)


def test_library_host_functions_replay_reference():
    """The C ABI's host-side couplings (lce_couplings) and neighbour tables
    (lce_geometry_tables) against the reference's paraminit and adresses."""
    lce = pytest.importorskip("lceqcd_b200")
    from lceqcd_b200.lattice import couplings, geometry_tables
    n = 0
    for case in CASES:
        rec = MANIFEST[case["name"]]
        p = rec["params"]
        for step, r in zip(case["steps"], rec["steps"]):
            if step[0] == "couplings":
                compare_ret(list(couplings(p["beta"], p["x"], p["y"])), r["ret"], 1e-14)
                n += 1
            elif step[0] == "tables":
                up, dn = geometry_tables(p["L"])
                assert np.array_equal(up, np.asarray(r["ret"]["siteup"]))
                assert np.array_equal(dn, np.asarray(r["ret"]["sitedn"]))
                n += 1
    assert n >= 6
