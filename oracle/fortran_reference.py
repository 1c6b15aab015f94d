"""The reference's own routines, run by oracle/fortran_runner.py, behind the
same method names as oracle.Oracle.

TEST INFRASTRUCTURE ONLY: it needs a checkout of the reference (the Fortran
sources are read from it, never copied into this repository) and is used by
tests/golden/make_reference_runs.py to write golden fixtures, and by the tests
when a checkout is named in LCEQCD_REFERENCE.

The lattice is set up the way f/initialize.f:31-35 does it, minus the
configuration files: ``paraminit`` (reading a generated ``inputfile`` with the
20 positional values of f/paraminit.f:82-101), ``topology``, ``adresses`` and
``measinit`` (which fills ``normalsites`` and the file units), all unmodified,
with one MPI rank.  ``measinit``'s RANLUX seeding of ``random_number`` is
stubbed: every uniform comes from the stream the caller sets.  Fields are
exchanged in oracle.Oracle's layout (u[mu, eo, site, 4] = (Re a, Im a, Re b,
Im b), a[eo, site, 3]) and written into the COMMON arrays
u(2, maxarray, 0:1, 3) and a(3, maxarray, 0:1) of
f/INCLUDE/gaugefield.inc:21-26.
"""
from __future__ import annotations

import os

import numpy as np

from .fortran_runner import Arr, Ref, Runner

HOT_PATH_FILES = ["paraminit", "topology", "adresses", "measinit", "matmul", "staples", "heat_kpi", "agauge",
                  "a_force", "gauss", "ahiggs1", "ahiggs2", "ahiggs3", "renorm", "landau_gauge",
                  "or_gauge_fixing1", "u_f_renorm", "it_gauge_fixing", "correlator", "meas2a",
                  "polyakov", "scalarcorr"]



class FortranLattice:
    def __init__(self, refdir, L, beta, x, y, lam=1.8, alpha=1.0, limit_or=1e-9, imode=0,
                 real_kind: int = 8, agauge1: bool = False, nsweep: int = 1, imeas: int = 1,
                 confstart: int = 0):
        fdir = os.path.join(refdir, "f")
        files = [f for f in HOT_PATH_FILES if not (agauge1 and f == "agauge")]
        if agauge1:
            files.append("agauge1")
        self.r = Runner([os.path.join(fdir, f + ".f") for f in files], [os.path.join(fdir, "INCLUDE")],
                        real_kind=real_kind)
        self.r.stubs["paratypeconstruct"] = lambda *a: None
        self.L = tuple(int(v) for v in L)
        self.nh = self.L[0] * self.L[1] * self.L[2] // 2
        self.real = self.r.kinds.real
        vals = [f"{L[0]} {L[1]} {L[2]}", "1 1 1", "1", "0", "0", "0", str(confstart), repr(float(beta)),
                repr(float(x)), repr(float(y)), repr(float(lam)), repr(float(alpha)), repr(float(limit_or)),
                "1e-6", "1", "0", "1", str(nsweep), str(imeas), str(imode)]
        self.r.files_in["inputfile"] = vals
        self.r.call("paraminit")
        self.r.call("topology")
        self.r.call("adresses")
        self.r.stubs["rluxgo"] = lambda *a: None
        self.r.stubs["ranlux"] = lambda rvec, n: rvec.view().__setitem__(Ellipsis, 0)
        self.r.call("measinit")
        units = dict(self.r.commons["units"])
        self.unit = {k: int(units[k + "_unit"].get()) for k in ("corr", "checkp", "afield", "polyak", "corra2",
                                                                 "joblog")}
        self.r.capture_units = set(self.unit.values())
        self.r.captured.clear()

    # ---- COMMON access
    def common(self, block, name):
        return self.r.common_var(block, name)

    def scalar(self, block, name):
        return self.common(block, name).get()

    def couplings(self):
        return tuple(float(self.scalar("paramet", n)) for n in ("beta_a", "beta_2", "beta_4"))

    def tables(self):
        """siteup/sitedn as (eo, mu, site) 0-based, like oracle.Oracle.tables."""
        out = []
        for name in ("siteup", "sitedn"):
            t = self.common("pointer", name).view()      # (maxarray, 2, 3), 1-based values
            out.append(np.ascontiguousarray(t[:self.nh].transpose(1, 2, 0) - 1).astype(np.int32))
        return tuple(out)

    def _u(self, which):
        return self.common("linkvar", "u_f" if which else "u").view()   # (2, maxarray, 2, 3) complex

    def _a(self, which):
        return self.common("linkvar", "a_f" if which else "a").view()   # (3, maxarray, 2)

    def set_fields(self, u=None, a=None, which: int = 0):
        nh = self.nh
        if u is not None:
            u = np.asarray(u, np.float64).reshape(3, 2, nh, 4)
            U = self._u(which)
            U[0, :nh] = (u[..., 0] + 1j * u[..., 1]).transpose(2, 1, 0)
            U[1, :nh] = (u[..., 2] + 1j * u[..., 3]).transpose(2, 1, 0)
        if a is not None:
            a = np.asarray(a, np.float64).reshape(2, nh, 3)
            self._a(which)[:, :nh, :] = a.transpose(2, 1, 0)

    def get_fields(self, which: int = 0):
        nh = self.nh
        U = self._u(which)
        u = np.empty((3, 2, nh, 4))
        ua, ub = U[0, :nh].transpose(2, 1, 0), U[1, :nh].transpose(2, 1, 0)
        u[..., 0], u[..., 1], u[..., 2], u[..., 3] = ua.real, ua.imag, ub.real, ub.imag
        a = np.ascontiguousarray(self._a(which)[:, :nh, :].transpose(2, 1, 0)).astype(np.float64)
        return u, a

    def staple(self):
        nh = self.nh
        V = self.common("helpfields", "v").view()
        v = np.empty((3, 2, nh, 4))
        va, vb = V[0, :nh].transpose(2, 1, 0), V[1, :nh].transpose(2, 1, 0)
        v[..., 0], v[..., 1], v[..., 2], v[..., 3] = va.real, va.imag, vb.real, vb.imag
        return v

    def force(self):
        return np.ascontiguousarray(self.common("helpfields", "force").view()[:, :self.nh].T).astype(np.float64)

    # ---- uniforms
    def set_stream(self, u):
        self.r.set_stream(u)

    def stream_pos(self) -> int:
        return self.r.stream_pos

    # ---- routines (argument meaning as the reference's)
    def _acc(self):
        return Ref(np.zeros(1, self.real), 0)

    def ahiggs2(self, measflag: int = 1) -> float:
        acc = self._acc()
        self.r.call("ahiggs2", measflag, acc)
        return float(acc.get())

    def ahiggs3(self, measflag: int = 1) -> float:
        acc = self._acc()
        self.r.call("ahiggs3", measflag, acc)
        return float(acc.get())

    def ahiggs1(self, delta: float, measflag: int = 1):
        d = Ref(np.array([delta], self.real), 0)
        acc = self._acc()
        self.r.call("ahiggs1", d, measflag, acc)
        return float(acc.get()), float(d.get())

    def agauge(self, measflag: int = 1) -> float:
        acc = self._acc()
        self.r.call("agauge", measflag, acc)
        return float(acc.get())

    agauge1 = agauge     # the loaded file decides (agauge1=True loads f/agauge1.f)

    def renorm(self):
        self.r.call("renorm")

    def staples(self, eo: int, mu: int):
        self.r.call("staples", eo, 1 - eo, mu + 1)

    def a_force(self, eo: int):
        self.r.call("a_force", eo)

    def sweep(self, measflag: int = 1) -> dict:
        """f/main.f:38-41: ahiggs2, ahiggs3, agauge, renorm."""
        acc_hb = self.ahiggs2(measflag)
        acc_or = self.ahiggs3(measflag)
        acc_g = self.agauge(measflag)
        self.renorm()
        m = self.meas()
        m.update(acc_hb=acc_hb, acc_or=acc_or, acc_gauge=acc_g)
        return m

    def meas(self) -> dict:
        return {"plaq": float(self.scalar("aver_loc", "plaq0")), "akin": float(self.scalar("aver_loc", "a0kin")),
                "a2": float(self.scalar("aver_loc", "a02")), "a4": float(self.scalar("aver_loc", "a04"))}

    def landau_gauge(self):
        da1 = Ref(np.zeros(1, self.real), 0)
        it = Ref(np.zeros(1, np.int64), 0)
        self.r.call("landau_gauge", da1, it)
        return float(da1.get()), int(it.get())

    def or_gauge_fixing(self) -> float:
        da1 = Ref(np.zeros(1, self.real), 0)
        self.r.call("or_gauge_fixing", da1)
        return float(da1.get())

    def u_f_renorm(self):
        self.r.call("u_f_renorm")

    def it_gauge_fixing(self, step=None, flags: int = 0) -> float:
        """One iteration of f/it_gauge_fixing.f as written; its step is the
        input file's alpha, so ``step`` must equal it and ``flags`` be 0."""
        if flags != 0 or (step is not None and abs(step - float(self.scalar("paramet", "alpha"))) > 1e-6):
            raise ValueError("the reference's it_gauge_fixing takes alpha from the input file, as written")
        da1 = Ref(np.zeros(1, self.real), 0)
        self.r.call("it_gauge_fixing", da1)
        return float(da1.get())

    def _captured(self, unit):
        return self.r.captured.pop(unit, [])

    def correlator(self, meas: int = 1):
        """corr_a, corr_u (from unit corr_unit) and corr_3 (checkp_unit)."""
        self.r.call("correlator", meas, 0)
        rows = self._captured(self.unit['corr'])
        ca = np.array([r[0] for r in rows[1:]])
        cu = np.array([r[1] for r in rows[1:]])
        c3 = np.array([r[0] for r in self._captured(self.unit['checkp'])[1:]])
        return ca, cu, c3

    def meas2(self, meas: int = 1):
        """f/meas2a.f: the correlators and the average of A_f (afield file)."""
        self.r.call("meas2", meas)
        self._captured(self.unit['corr'])
        self._captured(self.unit['checkp'])
        self._captured(self.unit['joblog'])
        rows = self._captured(self.unit['afield'])
        return np.array(rows[-1][1:4])

    def polyakov(self, meas: int = 1):
        """(None, the slice correlator, (mean of cos(4|A|))^2) as written to
        the polyak file; the slice means themselves are not written."""
        self.r.call("polyakov", meas, 0)
        rows = self._captured(self.unit['polyak'])
        return None, np.array([r[0] for r in rows[2:]]), float(rows[1][0])

    def scalarcorr(self, meas: int = 1):
        """(None, the slice correlator, mean of |A|^2) as written to the
        corra2 file."""
        self.r.call("scalarcorr", meas, 0)
        rows = self._captured(self.unit['corra2'])
        return None, np.array([r[0] for r in rows[2:]]), float(rows[1][0])
