"""Write tests/golden/reference_runs.npz: the reference's own routines, run.

    python tests/golden/make_reference_runs.py <path to the lceqcd checkout>

Neither this container nor the GPU machine has a Fortran compiler, so the
reference's unmodified sources are executed by oracle/fortran_runner.py (a
interpreter for the Fortran subset they use), set up as f/initialize.f does
(paraminit, topology, adresses, measinit) with one MPI rank, promoted to
64-bit REAL/COMPLEX (real_kind=8) except where a case says otherwise.  Every
``call random_number`` draws from a RANLUX stream (oracle.reference_stream,
itself pinned to f/luxtst.f:88-162).

Each case is a script of calls that oracle.Oracle and the GPU Lattice also
have (see tests/reference_cases.py); after every step the script records what
the call returned, the fields it may change and the stream position.  The
inputs (a seeded hot configuration and a seeded RANLUX stream) are not stored:
the tests regenerate them and check their SHA-256 against the manifest.  The
tests replay the scripts on the oracle (CPU) and on the GPU's FP64 validation
path and compare at 1e-12 relative.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from oracle.fortran_reference import FortranLattice  # noqa: E402
from reference_cases import CASES, apply_step, inputs_sha256, record_state  # noqa: E402


def run_case(refdir, case, arrays, manifest):
    p = case["params"]
    f = FortranLattice(refdir, p["L"], p["beta"], p["x"], p["y"], lam=p.get("lam", 1.8),
                       alpha=p.get("alpha", 1.0), limit_or=p.get("limit_or", 1e-9), imode=p.get("imode", 0),
                       real_kind=p.get("real_kind", 8), agauge1=p.get("agauge1", False))
    name = case["name"]
    u, a, stream = case["inputs"]()
    f.set_fields(u, a)
    f.set_stream(stream)
    out = []
    for k, step in enumerate(case["steps"]):
        ret = apply_step(f, step)
        rec = {"call": step, "ret": ret, "stream_pos": f.stream_pos()}
        for key, arr in record_state(f, step).items():
            arrays[f"{name}/{k}/{key}"] = arr
        out.append(rec)
    manifest[name] = {"params": p, "steps": out, "inputs_sha256": inputs_sha256(u, a, stream)}


def main(argv):
    if len(argv) != 2:
        sys.exit("usage: python tests/golden/make_reference_runs.py <path to the lceqcd checkout>")
    refdir = argv[1]
    arrays, manifest = {}, {}
    for case in CASES:
        t0 = time.time()
        run_case(refdir, case, arrays, manifest)
        print(f"{case['name']}: {len(case['steps'])} steps, {time.time() - t0:.1f} s", flush=True)
    arrays["manifest"] = np.frombuffer(json.dumps(manifest, sort_keys=True).encode(), dtype=np.uint8)
    dst = os.path.join(HERE, "reference_runs.npz")
    np.savez_compressed(dst, **arrays)
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main(sys.argv)
