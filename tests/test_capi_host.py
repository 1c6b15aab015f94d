"""Host-side checks of the C ABI that need no GPU: every symbol declared in
include/lceqcd_gpu.h is exported by liblceqcd_gpu.so, the coupling
derivation (f/paraminit.f:150-153) and the neighbour arithmetic
(f/adresses.f:91-337) agree bit for bit with the oracle, and the inputfile
reader handles the reference's 20-line format."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from oracle.oracle import Oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
lce = pytest.importorskip("lceqcd_b200")


def _header_symbols():
    text = open(os.path.join(ROOT, "include", "lceqcd_gpu.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(lce_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(os.path.join(ROOT, "lceqcd_b200", "liblceqcd_gpu.so"))
    syms = _header_symbols()
    assert len(syms) >= 40
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    from lceqcd_b200._lib import SIGNATURES
    assert sorted(SIGNATURES) == syms


def test_version_and_errors():
    lib = lce.load()
    assert b"sm_100a" in lib.lce_version()
    assert lib.lce_strerror(-3) == b"gauge fixing did not converge"


@pytest.mark.parametrize("beta,x,y", [(9.0, 0.1, 0.45), (12.0, 0.09, 0.3), (16.0, 0.08, 0.2), (6.0, 0.1, 0.1)])
def test_couplings_match_oracle_bitwise(beta, x, y):
    for prec, bits in (("f64", 64), ("f32", 32)):
        got = lce.couplings(beta, x, y, precision=prec)
        want = Oracle((4, 4, 4), beta, x, y, bits=bits).couplings()
        assert got == want, (prec, got, want)


@pytest.mark.parametrize("L", [(4, 4, 4), (2, 2, 2), (4, 6, 8), (8, 2, 6), (16, 12, 10), (6, 6, 32)])
def test_geometry_matches_adresses(L):
    up, dn = lce.geometry_tables(L)
    oup, odn = Oracle(L, 9.0, 0.1, 0.45).tables()
    np.testing.assert_array_equal(up, oup)
    np.testing.assert_array_equal(dn, odn)


def test_geometry_large_extent_fastdiv():
    """The kernels' magic-number division over every site of a large ragged
    lattice: up/down along each direction must be inverse permutations."""
    L = (96, 34, 18)
    up, dn = lce.geometry_tables(L)
    nh = L[0] * L[1] * L[2] // 2
    for eo in range(2):
        for mu in range(3):
            # down from the other parity undoes up
            np.testing.assert_array_equal(dn[1 - eo, mu][up[eo, mu]], np.arange(nh))
            assert len(np.unique(up[eo, mu])) == nh


def test_invalid_lattice_is_rejected_without_gpu():
    lib = lce.load()
    from lceqcd_b200.lattice import Params
    p = Params(L=(5, 4, 4)).to_c()
    assert not lib.lce_create(C.byref(p))
    assert b"even" in lib.lce_last_error(None)


INPUTFILE = """16 16 16    !nx/ny/nz global lattice size
01 01 01    !dimproc
001         !nproc
2           ! init
0           !rand
0           !save
000000      !confstart
 9.000      !beta
0.1000      !x
0.4500      !y
1.7000      !lambda
1.000000    !alpha
0.100E-09   !limit_or
0.100E-04   !limit_it
001         !inorm
0           !nsweep_flag
240         !ntime
01000       !nsweep
00010       !imeas
000         !imode
"""


def test_inputfile_reader(tmp_path):
    p = tmp_path / "inputfile"
    p.write_text(INPUTFILE)
    cfg = lce.read_inputfile(str(p))
    assert cfg["n_lattice"] == [16, 16, 16] and cfg["nsweep"] == 1000 and cfg["imeas"] == 10
    assert cfg["beta"] == 9.0 and cfg["y"] == 0.45 and cfg["limit_or"] == 1e-10
    prm = lce.params_from_inputfile(cfg)
    assert prm.L == (16, 16, 16) and prm.lam == 1.7
    bad = tmp_path / "bad"
    bad.write_text("\n".join(INPUTFILE.splitlines()[:10]))
    with pytest.raises(ValueError):
        lce.read_inputfile(str(bad))
