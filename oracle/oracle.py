"""ctypes wrapper for the CPU oracle (liblce_oracle64.so / liblce_oracle32.so).

TEST INFRASTRUCTURE ONLY.  This module is the correctness oracle for the CUDA
path and the CPU baseline of bench.py; only tests/, __graft_entry__.smoke()
and bench.py's CPU legs import it.  The product package lceqcd_b200 never
does.  Each method names the reference routine it restates (see
oracle/lce_oracle.h for file:line citations).

Field layout (both precisions): u[mu, eo, site, 4] with the last axis
(Re a, Im a, Re b, Im b) of the first row (a, b) of the SU(2) link, which is
the reference's COMPLEX u(2, site, eo, mu) order; a[eo, site, 3].
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict[int, C.CDLL] = {}


class LcoMeas(C.Structure):
    _fields_ = [
        ("plaq", C.c_double), ("akin", C.c_double), ("a2", C.c_double), ("a4", C.c_double),
        ("acc_gauge", C.c_double), ("acc_hb", C.c_double), ("acc_or", C.c_double),
        ("acc_metro", C.c_double), ("af", C.c_double * 3),
    ]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "af"}
        d["af"] = list(self.af)
        return d


def build() -> None:
    """Compile both oracle builds (make in oracle/)."""
    subprocess.check_call(["make", "-s", "-C", _HERE])


def _lib(bits: int) -> C.CDLL:
    if bits in _LIBS:
        return _LIBS[bits]
    path = os.path.join(_HERE, f"liblce_oracle{bits}.so")
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    R = C.c_double if bits == 64 else C.c_float
    P = C.c_void_p
    sig = {
        "lco_create": (P, [C.c_int, C.c_int, C.c_int] + [C.c_double] * 6 + [C.c_int]),
        "lco_destroy": (None, [P]),
        "lco_nh": (C.c_int, [P]),
        "lco_set_threads": (None, [P, C.c_int]),
        "lco_couplings": (None, [P, P]),
        "lco_set_stream": (None, [P, P, C.c_size_t]),
        "lco_stream_pos": (C.c_size_t, [P]),
        "lco_set_ranlux_source": (None, [P]),
        "lco_set_philox": (None, [P, C.c_uint64, C.c_uint64]),
        "lco_pass_ctr": (C.c_uint64, [P]),
        "lco_set_gf_angle": (None, [P, C.c_int]),
        "lco_set_fields": (None, [P, C.c_int, P, P]),
        "lco_get_fields": (None, [P, C.c_int, P, P]),
        "lco_get_staple": (None, [P, P]),
        "lco_get_force": (None, [P, P]),
        "lco_tables": (None, [P, P, P]),
        "lco_unitconf": (None, [P, C.c_double]),
        "lco_randomconf": (C.c_int, [P]),
        "lco_testconf": (None, [P]),
        "lco_staples": (C.c_int, [P, C.c_int, C.c_int]),
        "lco_a_force": (C.c_int, [P, C.c_int]),
        "lco_ahiggs1": (C.c_int, [P, P, C.c_int, P]),
        "lco_ahiggs2": (C.c_int, [P, C.c_int, P]),
        "lco_ahiggs3": (C.c_int, [P, C.c_int, P]),
        "lco_agauge": (C.c_int, [P, C.c_int, P]),
        "lco_agauge1": (C.c_int, [P, C.c_int, P]),
        "lco_link_or": (C.c_int, [P, C.c_int, P]),
        "lco_renorm": (None, [P]),
        "lco_sweep": (C.c_int, [P, C.c_int, P]),
        "lco_landau_copy": (None, [P]),
        "lco_or_gauge_fixing": (C.c_double, [P]),
        "lco_u_f_renorm": (None, [P]),
        "lco_landau_gauge": (C.c_int, [P, C.c_int, P]),
        "lco_it_gauge_fixing": (C.c_double, [P, C.c_double, C.c_int]),
        "lco_it_landau_gauge": (C.c_int, [P, C.c_double, C.c_int, C.c_int, P]),
        "lco_gauge_functional": (C.c_double, [P]),
        "lco_theta_direct": (C.c_double, [P]),
        "lco_correlator": (None, [P, P, P, P]),
        "lco_polyakov": (None, [P, P, P, P]),
        "lco_scalarcorr": (None, [P, P, P, P]),
        "lco_meas2": (None, [P, P]),
        "lco_plaquette": (C.c_double, [P]),
        "lco_get_meas": (None, [P, P]),
        "lco_ranlux_default": (None, []),
        "lco_rluxgo": (None, [C.c_int] * 4),
        "lco_ranlux": (None, [P, C.c_int]),
        "lco_rluxut": (None, [P]),
        "lco_rluxin": (None, [P]),
        "lco_rluxat": (None, [P, P, P, P]),
        "lco_philox4x32": (None, [P, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    lib._real = R
    _LIBS[bits] = lib
    return lib


def _ptr(arr: np.ndarray) -> C.c_void_p:
    assert arr.flags["C_CONTIGUOUS"]
    return C.c_void_p(arr.ctypes.data)


# ---------------------------------------------------------------- RANLUX
class Ranlux:
    """f/luxury.f restated (single precision, as the reference)."""

    def __init__(self):
        self.lib = _lib(64)

    def reset_default(self):
        self.lib.lco_ranlux_default()

    def rluxgo(self, lux: int, ins: int, k1: int = 0, k2: int = 0):
        self.lib.lco_rluxgo(lux, ins, k1, k2)

    def ranlux(self, n: int) -> np.ndarray:
        out = np.zeros(n, np.float32)
        self.lib.lco_ranlux(_ptr(out), n)
        return out

    def rluxut(self) -> np.ndarray:
        out = np.zeros(25, np.int32)
        self.lib.lco_rluxut(_ptr(out))
        return out

    def rluxin(self, isd) -> None:
        arr = np.ascontiguousarray(isd, np.int32)
        self.lib.lco_rluxin(_ptr(arr))

    def rluxat(self):
        v = [C.c_int() for _ in range(4)]
        self.lib.lco_rluxat(*[C.byref(x) for x in v])
        return tuple(x.value for x in v)


def philox4x32(ctr, key) -> np.ndarray:
    lib = _lib(64)
    c = np.ascontiguousarray(ctr, np.uint32)
    k = np.ascontiguousarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib.lco_philox4x32(_ptr(c), _ptr(k), _ptr(out))
    return out


def reference_stream(n: int, seed: int = 314159, lux: int = 3) -> np.ndarray:
    """n uniforms from RANLUX seeded like f/measinit.f:214 (rluxgo(3, seed))."""
    r = Ranlux()
    r.rluxgo(lux, seed, 0, 0)
    return r.ranlux(n).astype(np.float64)


def uniforms_per_sweep(L) -> int:
    """29*V uniforms per sweep in the reference's consumption order."""
    return 29 * int(L[0]) * int(L[1]) * int(L[2])


# ---------------------------------------------------------------- lattice
class Oracle:
    """One lattice with the reference's COMMON-block state (single rank)."""

    def __init__(self, L, beta, x, y, lam=1.8, alpha=1.0, limit_or=1e-9, imode=0,
                 bits: int = 64, threads: int = 1):
        self.lib = _lib(bits)
        self.bits = bits
        self.dtype = np.float64 if bits == 64 else np.float32
        self.L = tuple(int(v) for v in L)
        h = self.lib.lco_create(*self.L, float(beta), float(x), float(y), float(lam),
                                float(alpha), float(limit_or), int(imode))
        if not h:
            raise ValueError(f"oracle: invalid lattice {L}")
        self.h = C.c_void_p(h)
        self.nh = self.lib.lco_nh(self.h)
        self.vol = 2 * self.nh
        self._stream = None
        self.lib.lco_set_threads(self.h, threads)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.lco_destroy(self.h)
            self.h = None

    # --- couplings f/paraminit.f:150-153
    def couplings(self):
        out = np.zeros(3, np.float64)
        self.lib.lco_couplings(self.h, _ptr(out))
        return tuple(out)

    # --- random sources
    def set_stream(self, u: np.ndarray):
        self._stream = np.ascontiguousarray(u, np.float64)
        self.lib.lco_set_stream(self.h, _ptr(self._stream), self._stream.size)

    def stream_pos(self) -> int:
        return self.lib.lco_stream_pos(self.h)

    def set_ranlux(self):
        self.lib.lco_set_ranlux_source(self.h)

    def set_philox(self, seed: int, pass_ctr: int = 0):
        self.lib.lco_set_philox(self.h, seed, pass_ctr)

    def pass_ctr(self) -> int:
        return self.lib.lco_pass_ctr(self.h)

    def set_gf_angle(self, mode: int):
        """0: acos of Re Omega (the reference); 1: atan2 (small-angle accurate)."""
        self.lib.lco_set_gf_angle(self.h, mode)

    # --- fields
    def set_fields(self, u=None, a=None, which: int = 0):
        uu = None if u is None else np.ascontiguousarray(u, self.dtype).reshape(3, 2, self.nh, 4)
        aa = None if a is None else np.ascontiguousarray(a, self.dtype).reshape(2, self.nh, 3)
        self.lib.lco_set_fields(self.h, which, None if uu is None else _ptr(uu),
                                None if aa is None else _ptr(aa))

    def get_fields(self, which: int = 0):
        u = np.zeros((3, 2, self.nh, 4), self.dtype)
        a = np.zeros((2, self.nh, 3), self.dtype)
        self.lib.lco_get_fields(self.h, which, _ptr(u), _ptr(a))
        return u, a

    def staple(self):
        v = np.zeros((3, 2, self.nh, 4), self.dtype)
        self.lib.lco_get_staple(self.h, _ptr(v))
        return v

    def force(self):
        f = np.zeros((self.nh, 3), self.dtype)
        self.lib.lco_get_force(self.h, _ptr(f))
        return f

    def tables(self):
        up = np.zeros((2, 3, self.nh), np.int32)
        dn = np.zeros((2, 3, self.nh), np.int32)
        self.lib.lco_tables(self.h, _ptr(up), _ptr(dn))
        return up, dn

    # --- configurations f/confget.f
    def unitconf(self, a3: float = 1.0):
        self.lib.lco_unitconf(self.h, a3)

    def randomconf(self):
        self._check(self.lib.lco_randomconf(self.h))

    def testconf(self):
        self.lib.lco_testconf(self.h)

    # --- hot path
    def _check(self, rc):
        if rc != 0:
            raise RuntimeError("oracle: uniform stream exhausted")

    def _acc(self):
        return self.lib._real()

    def staples(self, eo: int, mu: int):
        self._check(self.lib.lco_staples(self.h, eo, mu))

    def a_force(self, eo: int):
        self._check(self.lib.lco_a_force(self.h, eo))

    def ahiggs1(self, delta: float, measflag: int = 1):
        d = self.lib._real(delta)
        acc = self._acc()
        self._check(self.lib.lco_ahiggs1(self.h, C.byref(d), measflag, C.byref(acc)))
        return acc.value, d.value

    def ahiggs2(self, measflag: int = 1) -> float:
        acc = self._acc()
        self._check(self.lib.lco_ahiggs2(self.h, measflag, C.byref(acc)))
        return acc.value

    def ahiggs3(self, measflag: int = 1) -> float:
        acc = self._acc()
        self._check(self.lib.lco_ahiggs3(self.h, measflag, C.byref(acc)))
        return acc.value

    def agauge(self, measflag: int = 1) -> float:
        acc = self._acc()
        self._check(self.lib.lco_agauge(self.h, measflag, C.byref(acc)))
        return acc.value

    def agauge1(self, measflag: int = 1) -> float:
        """f/agauge1.f: 3-hit link update."""
        acc = self._acc()
        self._check(self.lib.lco_agauge1(self.h, measflag, C.byref(acc)))
        return acc.value

    def link_or(self, measflag: int = 1) -> float:
        acc = self._acc()
        self._check(self.lib.lco_link_or(self.h, measflag, C.byref(acc)))
        return acc.value

    def renorm(self):
        self.lib.lco_renorm(self.h)

    def sweep(self, measflag: int = 1) -> dict:
        m = LcoMeas()
        self._check(self.lib.lco_sweep(self.h, measflag, C.byref(m)))
        return m.as_dict()

    def meas(self) -> dict:
        m = LcoMeas()
        self.lib.lco_get_meas(self.h, C.byref(m))
        return m.as_dict()

    # --- gauge fixing f/landau_gauge.f + f/or_gauge_fixing1.f
    def landau_copy(self):
        self.lib.lco_landau_copy(self.h)

    def or_gauge_fixing(self) -> float:
        return self.lib.lco_or_gauge_fixing(self.h)

    def u_f_renorm(self):
        self.lib.lco_u_f_renorm(self.h)

    def landau_gauge(self, max_iters: int = 0):
        da1 = C.c_double()
        it = self.lib.lco_landau_gauge(self.h, max_iters, C.byref(da1))
        return da1.value, it

    # f/it_gauge_fixing.f: flags 1 = second component from g1(2), 2 = ascend
    def it_gauge_fixing(self, step: float, flags: int = 0) -> float:
        return self.lib.lco_it_gauge_fixing(self.h, step, flags)

    def it_landau_gauge(self, step: float, flags: int = 0, max_iters: int = 0):
        da1 = C.c_double()
        it = self.lib.lco_it_landau_gauge(self.h, step, flags, max_iters, C.byref(da1))
        return da1.value, it

    def gauge_functional(self) -> float:
        return self.lib.lco_gauge_functional(self.h)

    def theta_direct(self) -> float:
        return self.lib.lco_theta_direct(self.h)

    # --- measurements
    def correlator(self):
        L3 = self.L[2]
        ca, cu, c3 = (np.zeros(L3) for _ in range(3))
        self.lib.lco_correlator(self.h, _ptr(ca), _ptr(cu), _ptr(c3))
        return ca, cu, c3

    def polyakov(self):
        L3 = self.L[2]
        sl, co, m = np.zeros(L3), np.zeros(L3), C.c_double()
        self.lib.lco_polyakov(self.h, _ptr(sl), _ptr(co), C.byref(m))
        return sl, co, m.value

    def scalarcorr(self):
        L3 = self.L[2]
        sl, co, m = np.zeros(L3), np.zeros(L3), C.c_double()
        self.lib.lco_scalarcorr(self.h, _ptr(sl), _ptr(co), C.byref(m))
        return sl, co, m.value

    def meas2(self):
        af = np.zeros(3)
        self.lib.lco_meas2(self.h, _ptr(af))
        return af

    def plaquette(self) -> float:
        return self.lib.lco_plaquette(self.h)


def hot_config(L, seed: int, dtype=np.float64):
    """Hot start: Haar links (normalised 4-Gaussians), A0 components ~ N(0,1).
    Returned in the oracle's layout; the same arrays are uploaded to the GPU."""
    nh = int(L[0]) * int(L[1]) * int(L[2]) // 2
    rng = np.random.default_rng(seed)
    q = rng.standard_normal((3, 2, nh, 4))
    q /= np.linalg.norm(q, axis=-1, keepdims=True)
    a = rng.standard_normal((2, nh, 3))
    return q.astype(dtype), a.astype(dtype)


def random_gauge_transform(u, a, L, seed: int):
    """Apply a random SU(2) gauge transformation g: U_mu(x) -> g(x) U_mu(x) g(x+mu)^+,
    A(x) -> g(x) A(x) g(x)^+ (numpy, float64).  Used by the gauge-invariance tests."""
    nh = u.shape[2]
    up = _up_tables(L)
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((2, nh, 4))
    g /= np.linalg.norm(g, axis=-1, keepdims=True)
    gc = g[..., 0] + 1j * g[..., 1], g[..., 2] + 1j * g[..., 3]
    uo = np.empty_like(u)
    for mu in range(3):
        for eo in range(2):
            oe = 1 - eo
            ua = u[mu, eo, :, 0] + 1j * u[mu, eo, :, 1]
            ub = u[mu, eo, :, 2] + 1j * u[mu, eo, :, 3]
            ga, gb = gc[0][eo], gc[1][eo]
            ha, hb = gc[0][oe][up[eo, mu]], gc[1][oe][up[eo, mu]]
            # g * U  (NN)
            ta = ga * ua - gb * np.conj(ub)
            tb = ga * ub + gb * np.conj(ua)
            # (g U) * h^+  (ND)
            ra = ta * np.conj(ha) + tb * np.conj(hb)
            rb = -ta * hb + tb * ha
            uo[mu, eo, :, 0], uo[mu, eo, :, 1] = ra.real, ra.imag
            uo[mu, eo, :, 2], uo[mu, eo, :, 3] = rb.real, rb.imag
    ao = np.empty_like(a)
    for eo in range(2):
        ga, gb = gc[0][eo], gc[1][eo]
        x = 1j * a[eo, :, 2]
        y = a[eo, :, 1] + 1j * a[eo, :, 0]
        # (iA) g^+  (AD)
        t1a = x * np.conj(ga) + y * np.conj(gb)
        t1b = -x * gb + y * ga
        # g (iA g^+)  (NN)
        t2a = ga * t1a - gb * np.conj(t1b)
        t2b = ga * t1b + gb * np.conj(t1a)
        ao[eo, :, 0], ao[eo, :, 1], ao[eo, :, 2] = t2b.imag, t2b.real, t2a.imag
    return uo, ao


def _up_tables(L):
    o = Oracle(L, 9.0, 0.1, 0.4)
    up, _ = o.tables()
    return up
