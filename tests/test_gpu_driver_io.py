"""Configuration files in the reference's direct-access format and the C++
driver that restates f/main.f over the C ABI."""
import os
import re
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
lce = pytest.importorskip("lceqcd_b200")
from lceqcd_b200 import LceError, Lattice  # noqa: E402
from lceqcd_b200.confio import read_conf, write_conf  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "lceqcd_b200", "lce_main")


def test_confsave_format_and_roundtrip(tmp_path):
    L = (8, 6, 4)
    g = Lattice(L, beta=9.0, x=0.1, y=0.45)
    g.init_hot(3)
    fu, fa = str(tmp_path / "u"), str(tmp_path / "a")
    g.confsave(fu, fa)
    nxy = 8 * 6 // 2
    assert os.path.getsize(fu) == 3 * 2 * 4 * (16 * 2 * nxy)   # 6*L3 records of u_rl bytes
    assert os.path.getsize(fa) == 2 * 4 * (8 * 3 * nxy)        # 2*L3 records of a_rl bytes
    u, a = g.download()
    ur, ar = read_conf(fu, fa, L)
    np.testing.assert_array_equal(ur, u)
    np.testing.assert_array_equal(ar, a)
    # a file written by the numpy writer loads through lce_confget
    u2 = u.copy()
    u2[..., 0] *= -1
    write_conf(fu, fa, u2, a * 2, L)
    os.remove(fu + ".rng")
    g.confget(fu, fa)
    ug, ag = g.download()
    np.testing.assert_array_equal(ug, u2)
    np.testing.assert_array_equal(ag, a * 2)


def test_exact_resume_from_saved_configuration(tmp_path):
    L = (8, 8, 8)
    g = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=77)
    g.init_hot(1)
    g.sweeps(5, 1)
    fu, fa = str(tmp_path / "u"), str(tmp_path / "a")
    g.confsave(fu, fa)
    g.sweeps(4, 1)
    want = g.download()
    h = Lattice(L, beta=12.0, x=0.09, y=0.3, seed=77)
    h.confget(fu, fa)
    assert h.rng_position() == (g.rng_position()[0] - 40, 0)
    h.sweeps(4, 1)
    got = h.download()
    np.testing.assert_array_equal(got[0], want[0])
    np.testing.assert_array_equal(got[1], want[1])


def test_truncated_configuration_is_an_error(tmp_path):
    L = (4, 4, 4)
    g = Lattice(L, beta=9.0, x=0.1, y=0.45)
    g.init_hot(1)
    fu, fa = str(tmp_path / "u"), str(tmp_path / "a")
    g.confsave(fu, fa)
    with open(fu, "r+b") as f:
        f.truncate(os.path.getsize(fu) // 3)
    with pytest.raises(LceError):
        g.confget(fu, fa)


INPUT = """{L} {L} {L}    !nx/ny/nz global lattice size
01 01 01    !dimproc
001         !nproc
{init}           ! init
0           !rand
1           !save
{start:06d}      !confstart
 9.000      !beta
0.1000      !x
0.4500      !y
1.7000      !lambda
1.000000    !alpha
0.100E-08   !limit_or
0.100E-04   !limit_it
001         !inorm
0           !nsweep_flag
240         !ntime
00010       !nsweep
00005       !imeas
000         !imode
"""

E23 = r"[ -]\d\.\d{16}E[+-]\d\d"


def test_driver_writes_reference_files_and_resumes(tmp_path):
    assert os.path.exists(DRIVER)
    inp = tmp_path / "inputfile"
    inp.write_text(INPUT.format(L=8, init=2, start=0))
    env = dict(os.environ)
    r = subprocess.run([DRIVER, "--input", str(inp), "--dir", str(tmp_path), "--therm", "20"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    tag = "s08_be09000_x01000_y04500_u000000"
    action = (tmp_path / f"action_{tag}").read_text().splitlines()
    assert action[:3] == ["# 08 08 08 ", "#  9.0000  0.1000  0.4500 ", "# 00010"]
    assert len(action) == 3 + 10
    for line in action[3:]:
        assert re.fullmatch(r"\s*\d+ " + " ".join([E23] * 4) + " ", line), line
    vals = np.array([[float(v) for v in l.split()[1:]] for l in action[3:]])
    assert np.all((vals[:, 0] > 0.3) & (vals[:, 0] < 1.0))            # plaquette
    correl = (tmp_path / f"correl_{tag}").read_text().splitlines()
    assert correl[3] == "001" and len(correl) == 3 + 2 * (1 + 8)
    assert "number of iteration for or. gauge fixing" in (tmp_path / f"joblog_{tag}").read_text()
    afield = (tmp_path / f"afield_{tag}").read_text().splitlines()
    assert len(afield) == 3 + 2 and afield[3].startswith("00001 ")
    assert (tmp_path / "u_conf_s08_be09000_x01000_y04500_u000010").exists()
    # finalize rewrote the inputfile for a resume (init = 3, confstart advanced)
    new = inp.read_text().splitlines()
    assert new[3].startswith("3") and new[6].startswith("000010")
    r = subprocess.run([DRIVER, "--input", str(inp), "--dir", str(tmp_path), "--therm", "0"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert r.returncode == 0, r.stderr
    assert (tmp_path / "action_s08_be09000_x01000_y04500_u000010").exists()
    assert (tmp_path / "u_conf_s08_be09000_x01000_y04500_u000020").exists()


def test_driver_rejects_bad_inputfile(tmp_path):
    inp = tmp_path / "inputfile"
    inp.write_text("16 16 16\n1 1 1\n")
    r = subprocess.run([DRIVER, "--input", str(inp), "--dir", str(tmp_path)], capture_output=True, text=True,
                       timeout=60)
    assert r.returncode != 0 and "data input" in r.stderr


def test_driver_iterative_gauge_fixing(tmp_path):
    """--gauge-fix it: f/landau_gauge.f with the reference's iterative form
    (component corrected, ascending); same files as the overrelaxed run."""
    inp = tmp_path / "inputfile"
    inp.write_text(INPUT.format(L=8, init=2, start=0))
    r = subprocess.run([DRIVER, "--input", str(inp), "--dir", str(tmp_path), "--therm", "20",
                        "--gauge-fix", "it", "--it-step", "0.3"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    tag = "s08_be09000_x01000_y04500_u000000"
    correl = (tmp_path / f"correl_{tag}").read_text().splitlines()
    assert correl[3] == "001" and len(correl) == 3 + 2 * (1 + 8)
    vals = np.array([float(v) for l in correl[4:] if not l.strip().isdigit() for v in l.split()])
    assert vals.size > 0 and np.all(np.isfinite(vals))
    r = subprocess.run([DRIVER, "--input", str(inp), "--dir", str(tmp_path), "--gauge-fix", "sd"],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "gauge-fix" in r.stderr


@pytest.mark.parametrize("form", ["fourier", "fourier-cg"])
def test_driver_fourier_gauge_fixing(tmp_path, form):
    """--gauge-fix fourier / fourier-cg: the measurement files of the
    overrelaxed run, the Fourier-accelerated iteration (steepest ascent or
    conjugate gradients) from the previous transform."""
    inp = tmp_path / "inputfile"
    inp.write_text(INPUT.format(L=8, init=2, start=0))
    r = subprocess.run([DRIVER, "--input", str(inp), "--dir", str(tmp_path), "--therm", "20",
                        "--gauge-fix", form], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    tag = "s08_be09000_x01000_y04500_u000000"
    correl = (tmp_path / f"correl_{tag}").read_text().splitlines()
    assert correl[3] == "001" and len(correl) == 3 + 2 * (1 + 8)
    vals = np.array([float(v) for l in correl[4:] if not l.strip().isdigit() for v in l.split()])
    assert vals.size > 0 and np.all(np.isfinite(vals))
