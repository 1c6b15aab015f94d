"""Python mirror of the reference's hot-path interface, over the C ABI.

`Lattice` exposes the subroutines f/main.f calls inside its sweep loop under
their reference names and argument meanings:

    ahiggs2(measflag) -> accept            f/ahiggs2.f:7
    ahiggs3(measflag) -> accept            f/ahiggs3.f:7
    ahiggs1(delta, measflag) -> (accept, delta)   f/ahiggs1.f:7
    agauge(measflag) -> accept             f/agauge.f:7
    renorm()                               f/renorm.f:6
    landau_gauge() -> (da1, iter_or1)      f/landau_gauge.f:6
    meas1() -> dict(plaq, akin, a2, a4)    f/meas1.f:7 (the reduced values)
    meas2() -> af(3)                       f/meas2a.f:9
    correlator() -> corr_a, corr_u, corr_3 f/correlator.f:11
    polyakov(), scalarcorr()               f/polyakov.f:10, f/scalarcorr.f:10

Errors raise LceError (the reference calls abort()).  Fields move in the
reference's array order: u[mu, eo, site, 4] = (Re a, Im a, Re b, Im b) of the
link's first row, a[eo, site, 3].
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import LceMeas, LceParams, check, load

PREC = {"f32": _lib.LCE_PREC_F32, "f64": _lib.LCE_PREC_F64}
RNG = {"philox": _lib.LCE_RNG_PHILOX, "stream": _lib.LCE_RNG_STREAM}
SWEEP_MODES = {"auto": _lib.LCE_SWEEP_AUTO, "passes": _lib.LCE_SWEEP_PASSES,
               "persistent": _lib.LCE_SWEEP_PERSISTENT, "passes2": _lib.LCE_SWEEP_PASSES2,
               "direct": _lib.LCE_SWEEP_DIRECT}


def _ptr(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


@dataclass
class Params:
    L: tuple = (16, 16, 16)
    beta: float = 9.0
    x: float = 0.1
    y: float = 0.5
    lam: float = 1.8
    alpha: float = 1.0
    limit_or: float = 1e-9
    imode: int = 0
    precision: str = "f32"
    rng: str = "philox"
    seed: int = 12345
    device: int = 0
    n_link_or: int = 0
    n_higgs_metro: int = 0
    delta0: float = 1.0
    gf_angle: str = "atan2"
    sweep_mode: str = "auto"
    agauge_hits: int = 1
    tile_threads: int = 0
    tile_registers: int = 0

    def to_c(self) -> LceParams:
        p = LceParams()
        load().lce_default_params(C.byref(p))
        for i in range(3):
            p.L[i] = int(self.L[i])
        p.beta, p.x, p.y = float(self.beta), float(self.x), float(self.y)
        p.lambda_, p.alpha, p.limit_or = float(self.lam), float(self.alpha), float(self.limit_or)
        p.imode = int(self.imode)
        p.precision = PREC[self.precision]
        p.rng = RNG[self.rng]
        p.seed = int(self.seed)
        p.device = int(self.device)
        p.n_link_or = int(self.n_link_or)
        p.n_higgs_metro = int(self.n_higgs_metro)
        p.delta0 = float(self.delta0)
        p.gf_angle = {"acos": _lib.LCE_GF_ACOS, "atan2": _lib.LCE_GF_ATAN2}[self.gf_angle]
        p.sweep_mode = SWEEP_MODES[self.sweep_mode]
        p.agauge_hits = int(self.agauge_hits)
        p.tile_threads = int(self.tile_threads)
        p.tile_registers = int(self.tile_registers)
        return p


def couplings(beta: float, x: float, y: float, precision: str = "f64"):
    """beta_a, beta_2, beta_4 of f/paraminit.f:150-153."""
    p = Params(beta=beta, x=x, y=y, precision=precision).to_c()
    out = np.zeros(3)
    check(load().lce_couplings(C.byref(p), _ptr(out)))
    return tuple(out)


def conf_filename(prefix: str, L3: int, beta: float, x: float, y: float, number: int) -> str:
    """f/measinit.f names, e.g. conf_filename('action', 16, 9.0, 0.1, 0.45, 0)."""
    buf = C.create_string_buffer(256)
    check(load().lce_conf_filename(buf, 256, prefix.encode(), int(L3), float(beta), float(x), float(y),
                                   int(number)))
    return buf.value.decode()


def geometry_tables(L):
    """siteup/sitedn of f/adresses.f (0-based), [eo, mu, site]."""
    nh = L[0] * L[1] * L[2] // 2
    up = np.zeros((2, 3, nh), np.int32)
    dn = np.zeros((2, 3, nh), np.int32)
    check(load().lce_geometry_tables(int(L[0]), int(L[1]), int(L[2]), _ptr(up), _ptr(dn)))
    return up, dn


class _Context:
    def __init__(self, params_list):
        self.lib = load()
        self.params = list(params_list)
        arr = (LceParams * len(self.params))(*[p.to_c() for p in self.params])
        if len(self.params) == 1:
            h = self.lib.lce_create(arr)
        else:
            h = self.lib.lce_create_batch(arr, len(self.params))
        if not h:
            raise _lib.LceError(_lib.LCE_ERR_INVALID, "lce_create: " + self.lib.lce_last_error(None).decode())
        self.h = C.c_void_p(h)
        self.dtype = np.float64 if self.params[0].precision == "f64" else np.float32
        # host arrays of asynchronous uploads: applied ones not yet known to be
        # copied (released by the next synchronising call), and staged ones
        # (oldest first; moved to _inflight by upload_apply)
        self._inflight = []
        self._staged = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.lce_destroy(self.h)  # synchronises the copy stream
            self.h = None
            self._inflight = []
            self._staged = []

    def __del__(self):
        self.close()

    def _ck(self, rc):
        return check(rc, self.h)

    # ---- fields
    def nh(self, chain: int = 0) -> int:
        L = self.params[chain].L
        return L[0] * L[1] * L[2] // 2

    def upload(self, u=None, a=None, which: int = 0, chain: int = 0):
        nh = self.nh(chain)
        f64 = (u is not None and np.asarray(u).dtype == np.float64) or \
              (a is not None and np.asarray(a).dtype == np.float64)
        dt = np.float64 if f64 else np.float32
        uu = None if u is None else np.ascontiguousarray(u, dt).reshape(3, 2, nh, 4)
        aa = None if a is None else np.ascontiguousarray(a, dt).reshape(2, nh, 3)
        fn = self.lib.lce_upload_f64 if f64 else self.lib.lce_upload
        self._ck(fn(self.h, chain, which, None if uu is None else _ptr(uu), None if aa is None else _ptr(aa), nh))

    def _async_args(self, u, a, chain, keep):
        nh = self.nh(chain)
        uu = None if u is None else np.ascontiguousarray(u, np.float32).reshape(3, 2, nh, 4)
        aa = None if a is None else np.ascontiguousarray(a, np.float32).reshape(2, nh, 3)
        keep.append((uu, aa))
        return None if uu is None else _ptr(uu), None if aa is None else _ptr(aa), nh

    def upload_async(self, u=None, a=None, which: int = 0, chain: int = 0):
        """lce_upload_async: FP32 fields, returns before the copy ends.  The
        arrays are kept referenced until the next synchronising call; pass
        pinned arrays for a copy that overlaps the work queued before it."""
        pu, pa, nh = self._async_args(u, a, chain, self._inflight)
        self._ck(self.lib.lce_upload_async(self.h, chain, which, pu, pa, nh))

    def upload_stage(self, u=None, a=None, which: int = 0, chain: int = 0):
        """lce_upload_stage: queue the host-to-device copy into a staging slot."""
        pu, pa, nh = self._async_args(u, a, chain, self._staged)
        rc = self.lib.lce_upload_stage(self.h, chain, which, pu, pa, nh)
        if rc < 0:
            self._staged.pop()
        self._ck(rc)

    def upload_apply(self):
        """lce_upload_apply: later update calls see the oldest staged upload."""
        self._ck(self.lib.lce_upload_apply(self.h))
        self._inflight.append(self._staged.pop(0))

    def download(self, which: int = 0, chain: int = 0, dtype=None):
        nh = self.nh(chain)
        dt = dtype or self.dtype
        u = np.zeros((3, 2, nh, 4), dt)
        a = np.zeros((2, nh, 3), dt)
        fn = self.lib.lce_download_f64 if dt == np.float64 else self.lib.lce_download
        self._ck(fn(self.h, chain, which, _ptr(u), _ptr(a), nh))
        self._inflight = []
        return u, a

    def download_into(self, u: np.ndarray, a: np.ndarray, which: int = 0, chain: int = 0):
        """Download into caller-owned (e.g. pinned) arrays of the reference layout."""
        nh = self.nh(chain)
        assert u.dtype == a.dtype and u.size == 24 * nh and a.size == 6 * nh
        fn = self.lib.lce_download_f64 if u.dtype == np.float64 else self.lib.lce_download
        self._ck(fn(self.h, chain, which, _ptr(u), _ptr(a), nh))
        self._inflight = []

    def extents(self, chain: int = 0):
        L = (C.c_int * 3)()
        self._ck(self.lib.lce_get_extents(self.h, chain, L))
        return tuple(L)

    def confsave(self, u_path: str, a_path: str, chain: int = 0):
        """f/confsave.f format (+ '<u_path>.rng' with the Philox position)."""
        self._ck(self.lib.lce_confsave(self.h, chain, u_path.encode(), a_path.encode()))

    def confget(self, u_path: str, a_path: str, chain: int = 0):
        """f/confget.f oldconf format; restores the Philox position if the sidecar exists."""
        self._ck(self.lib.lce_confget(self.h, chain, u_path.encode(), a_path.encode()))

    def init_unit(self, a3: float = 1.0):
        self._ck(self.lib.lce_init_unit(self.h, float(a3)))

    def init_hot(self, seed: int):
        self._ck(self.lib.lce_init_hot(self.h, int(seed)))

    # ---- random numbers
    def set_rng_stream(self, u: np.ndarray):
        self._stream = np.ascontiguousarray(u, np.float64)
        self._ck(self.lib.lce_set_rng_stream(self.h, _ptr(self._stream), self._stream.size))

    def rng_position(self):
        a, b = C.c_ulonglong(), C.c_ulonglong()
        self._ck(self.lib.lce_get_rng_position(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_rng_position(self, pass_ctr: int, stream_pos: int = 0):
        self._ck(self.lib.lce_set_rng_position(self.h, pass_ctr, stream_pos))

    # ---- updates (reference names)
    def ahiggs1(self, delta: float, measflag: int = 1):
        d, acc = C.c_float(delta), C.c_float()
        self._ck(self.lib.lce_ahiggs1(self.h, C.byref(d), measflag, C.byref(acc)))
        return acc.value, d.value

    def ahiggs2(self, measflag: int = 1) -> float:
        acc = C.c_float()
        self._ck(self.lib.lce_ahiggs2(self.h, measflag, C.byref(acc)))
        return acc.value

    def ahiggs3(self, measflag: int = 1) -> float:
        acc = C.c_float()
        self._ck(self.lib.lce_ahiggs3(self.h, measflag, C.byref(acc)))
        return acc.value

    def agauge(self, measflag: int = 1) -> float:
        acc = C.c_float()
        self._ck(self.lib.lce_agauge(self.h, measflag, C.byref(acc)))
        return acc.value

    def agauge1(self, measflag: int = 1) -> float:
        """f/agauge1.f: the 3-hit link update."""
        acc = C.c_float()
        self._ck(self.lib.lce_agauge1(self.h, measflag, C.byref(acc)))
        return acc.value

    def link_or(self, measflag: int = 1) -> float:
        acc = C.c_float()
        self._ck(self.lib.lce_link_or(self.h, measflag, C.byref(acc)))
        return acc.value

    def renorm(self):
        self._ck(self.lib.lce_renorm(self.h))

    def sweep(self, measflag: int = 1) -> dict:
        m = LceMeas()
        self._ck(self.lib.lce_sweep(self.h, measflag, C.byref(m)))
        self._inflight = []
        return m.as_dict()

    def sweeps(self, n: int, measflag: int = 0):
        self._ck(self.lib.lce_sweeps(self.h, int(n), measflag))

    def tile_shape(self, registers: bool = False):
        """(threads per block, sites per thread) of the update kernels in use,
        and with registers=True their per-thread register cap."""
        bs, spt, reg = C.c_int(), C.c_int(), C.c_int()
        self._ck(self.lib.lce_get_tile_shape(self.h, C.byref(bs), C.byref(spt), C.byref(reg)))
        return (bs.value, spt.value, reg.value) if registers else (bs.value, spt.value)

    def sweep_mode(self) -> str:
        m = self._ck(self.lib.lce_get_sweep_mode(self.h))
        return {v: k for k, v in SWEEP_MODES.items()}[m]

    def meas1(self, chain: int = 0) -> dict:
        m = LceMeas()
        self._ck(self.lib.lce_get_meas(self.h, chain, C.byref(m)))
        self._inflight = []
        return m.as_dict()

    def meas_batch(self) -> list:
        m = (LceMeas * len(self.params))()
        self._ck(self.lib.lce_get_meas_batch(self.h, m))
        return [x.as_dict() for x in m]

    def synchronize(self):
        self._ck(self.lib.lce_synchronize(self.h))
        self._inflight = []

    # ---- gauge fixing and measurements
    def landau_gauge(self, max_iters: int = 0, chain: int = 0):
        th, it = C.c_double(), C.c_int()
        self._ck(self.lib.lce_landau_gauge(self.h, chain, C.byref(th), C.byref(it), int(max_iters)))
        return th.value, it.value

    def gauge_fix_continue(self, max_iters: int = 0, chain: int = 0):
        th, it = C.c_double(), C.c_int()
        self._ck(self.lib.lce_gauge_fix_continue(self.h, chain, C.byref(th), C.byref(it), int(max_iters)))
        return th.value, it.value

    @staticmethod
    def _itgf_flags(fix_component: bool, ascend: bool, track: bool) -> int:
        return ((_lib.LCE_ITGF_FIX_COMPONENT if fix_component else 0) | (_lib.LCE_ITGF_ASCEND if ascend else 0)
                | (_lib.LCE_ITGF_TRACK if track else 0))

    def it_gauge_fixing(self, step: float = 0.0, fix_component: bool = False, ascend: bool = False,
                        track: bool = False, chain: int = 0) -> float:
        """One iteration of f/it_gauge_fixing.f on U_f, A_f; returns da1.
        step <= 0: the context's alpha (the reference's step).  Defaults are
        the reference as written; fix_component and ascend select the
        corrected steepest ascent (lce_it_gauge_fixing)."""
        da1 = C.c_double()
        self._ck(self.lib.lce_it_gauge_fixing(self.h, chain, float(step),
                                              self._itgf_flags(fix_component, ascend, track), C.byref(da1)))
        return da1.value

    def it_landau_gauge(self, step: float = 0.0, fix_component: bool = False, ascend: bool = False,
                        track: bool = False, max_iters: int = 0, chain: int = 0):
        """f/landau_gauge.f with it_gauge_fixing: copy, iterate and
        reunitarise until da1 <= limit_or.  Returns (da1, iterations)."""
        da1, it = C.c_double(), C.c_int()
        self._ck(self.lib.lce_it_landau_gauge(self.h, chain, float(step),
                                              self._itgf_flags(fix_component, ascend, track), C.byref(da1),
                                              C.byref(it), int(max_iters)))
        return da1.value, it.value

    def landau_gauge_from(self, start: str = "identity", max_iters: int = 0, chain: int = 0):
        """Gauge fixing tracking the transform G; start 'identity' or 'transform'
        (the current G).  Returns (theta_start, theta, iterations)."""
        ts, th, it = C.c_double(), C.c_double(), C.c_int()
        code = {"identity": _lib.LCE_GF_START_IDENTITY, "transform": _lib.LCE_GF_START_TRANSFORM}[start]
        self._ck(self.lib.lce_landau_gauge_from(self.h, chain, code, C.byref(ts), C.byref(th), C.byref(it),
                                                int(max_iters)))
        return ts.value, th.value, it.value

    def landau_gauge_warm(self, net=None, use_net: bool = True, judge: bool = True, record: bool = False,
                          fourier: bool = False, max_iters: int = 0, chain: int = 0, cg: bool = False):
        """Tracked gauge fixing from a warm start (the previous transform, or the
        network's correction of it; with judge the start of largest gauge
        functional among identity / previous / network).  Returns
        (start, functionals[3], theta, iterations); start is 'identity',
        'transform' or 'net'."""
        flags = ((_lib.LCE_WARM_NET if (use_net and net is not None) else 0) |
                 (_lib.LCE_WARM_JUDGE if judge else 0) | (_lib.LCE_WARM_RECORD if record else 0) |
                 (_lib.LCE_WARM_FOURIER if fourier else 0) | (_lib.LCE_WARM_CG if cg else 0))
        su, th, it = C.c_int(), C.c_double(), C.c_int()
        F = (C.c_double * 3)()
        self._ck(self.lib.lce_landau_gauge_warm(self.h, chain, net.h if net is not None else None, flags,
                                                C.byref(su), F, C.byref(th), C.byref(it), int(max_iters)))
        return ["identity", "transform", "net"][su.value], list(F), th.value, it.value

    def landau_gauge_fourier(self, start: str = "identity", step: float = 1.0, theta_switch: float = 0.0,
                             max_iters: int = 0, chain: int = 0):
        """Fourier-accelerated gauge fixing (tracking G) to theta_switch, then the
        plain iteration to limit_or.  Returns (theta, fourier_iters, plain_iters)."""
        th, itf, itp = C.c_double(), C.c_int(), C.c_int()
        code = {"identity": _lib.LCE_GF_START_IDENTITY, "transform": _lib.LCE_GF_START_TRANSFORM}[start]
        self._ck(self.lib.lce_landau_gauge_fourier(self.h, chain, code, float(step), float(theta_switch),
                                                   C.byref(th), C.byref(itf), C.byref(itp), int(max_iters)))
        return th.value, itf.value, itp.value

    def landau_gauge_fourier_cg(self, start: str = "identity", theta_switch: float = 0.0, max_iters: int = 0,
                                chain: int = 0):
        """The conjugate-gradient form of landau_gauge_fourier (lce_landau_gauge_fourier_cg).
        Returns (theta, fourier_iters, plain_iters)."""
        th, itf, itp = C.c_double(), C.c_int(), C.c_int()
        code = {"identity": _lib.LCE_GF_START_IDENTITY, "transform": _lib.LCE_GF_START_TRANSFORM}[start]
        self._ck(self.lib.lce_landau_gauge_fourier_cg(self.h, chain, code, float(theta_switch), C.byref(th),
                                                      C.byref(itf), C.byref(itp), int(max_iters)))
        return th.value, itf.value, itp.value

    def debug_fourier_step(self, step: float = 1.0, chain: int = 0) -> np.ndarray:
        """Preconditioned direction omega [2][V/2][3] (a3, Re b, Im b) of the current U_f."""
        om = np.zeros((2, self.nh(chain), 3), np.float64)
        self._ck(self.lib.lce_debug_fourier_step(self.h, chain, float(step), _ptr(om)))
        return om

    def apply_transform(self, chain: int = 0):
        self._ck(self.lib.lce_apply_transform(self.h, chain))

    def get_transform(self, chain: int = 0) -> np.ndarray:
        g = np.zeros((2, self.nh(chain), 4), np.float32)
        self._ck(self.lib.lce_get_transform(self.h, chain, _ptr(g), self.nh(chain)))
        return g

    def set_transform(self, g: np.ndarray, chain: int = 0):
        gg = np.ascontiguousarray(g, np.float32).reshape(2, self.nh(chain), 4)
        self._ck(self.lib.lce_set_transform(self.h, chain, _ptr(gg), self.nh(chain)))

    def gauge_functional(self, chain: int = 0) -> float:
        v = C.c_double()
        self._ck(self.lib.lce_gauge_functional(self.h, chain, C.byref(v)))
        return v.value

    def theta(self, chain: int = 0) -> float:
        v = C.c_double()
        self._ck(self.lib.lce_theta(self.h, chain, C.byref(v)))
        return v.value

    def correlator(self, chain: int = 0):
        L3 = self.params[chain].L[2]
        ca, cu, c3, af = np.zeros(L3), np.zeros(L3), np.zeros(L3), np.zeros(3)
        self._ck(self.lib.lce_correlator(self.h, chain, _ptr(ca), _ptr(cu), _ptr(c3), _ptr(af)))
        return ca, cu, c3, af

    def meas2(self, chain: int = 0):
        return self.correlator(chain)[3]

    def polyakov(self, chain: int = 0):
        L3 = self.params[chain].L[2]
        sl, co, m = np.zeros(L3), np.zeros(L3), C.c_double()
        self._ck(self.lib.lce_polyakov(self.h, chain, _ptr(sl), _ptr(co), C.byref(m)))
        return sl, co, m.value

    def scalarcorr(self, chain: int = 0):
        L3 = self.params[chain].L[2]
        sl, co, m = np.zeros(L3), np.zeros(L3), C.c_double()
        self._ck(self.lib.lce_scalarcorr(self.h, chain, _ptr(sl), _ptr(co), C.byref(m)))
        return sl, co, m.value

    def plaquette(self, chain: int = 0) -> float:
        v = C.c_double()
        self._ck(self.lib.lce_plaquette(self.h, chain, C.byref(v)))
        return v.value

    def debug_staple(self, eo: int, mu: int) -> np.ndarray:
        out = np.zeros((self.nh(), 4))
        self._ck(self.lib.lce_debug_staple(self.h, eo, mu, _ptr(out)))
        return out

    def debug_force(self, eo: int) -> np.ndarray:
        out = np.zeros((self.nh(), 3))
        self._ck(self.lib.lce_debug_force(self.h, eo, _ptr(out)))
        return out

    # ---- timing
    def flush_l2(self):
        self._ck(self.lib.lce_flush_l2(self.h))

    def profile_sweep(self, measflag: int = 0, max_passes: int = 64, with_finalize: bool = False):
        """Per-pass durations (ms) of one sweep run as a graph with timing
        events hung off the pass kernels; with_finalize appends the finalize
        kernel's."""
        ms = np.zeros(max_passes + 1, np.float32)
        n = self._ck(self.lib.lce_profile_sweep(self.h, measflag, _ptr(ms), max_passes + 1))
        return ms[:n + 1 if with_finalize else n].astype(np.float64)

    def timer_start(self):
        self._ck(self.lib.lce_timer_start(self.h))

    def timer_stop(self) -> float:
        ms = C.c_float()
        self._ck(self.lib.lce_timer_stop(self.h, C.byref(ms)))
        return ms.value


class GaugeNet:
    """The warm-start network of lce_landau_gauge_warm (4 layers, 16 channels,
    3x3x3 periodic kernels, BF16 on the tensor cores; no reference
    counterpart).  Parameters per layer: weights [27][16 out][16 in], then 16
    biases; offset k = 9 (dx+1) + 3 (dy+1) + (dz+1)."""

    LAYERS, CHANNELS, OFFSETS, OUT = 4, 16, 27, 4

    def __init__(self, device: int = 0, seed: int = 1):
        self.lib = load()
        h = self.lib.lce_net_create(int(device), int(seed))
        if not h:
            raise _lib.LceError(_lib.LCE_ERR_CUDA, "lce_net_create: " + self.lib.lce_last_error(None).decode())
        self.h = C.c_void_p(h)
        self.nparam = self.lib.lce_net_num_params(self.h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.lce_net_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def params(self) -> np.ndarray:
        w = np.empty(self.nparam, np.float32)
        check(self.lib.lce_net_get_params(self.h, _ptr(w)))
        return w

    def set_params(self, w: np.ndarray):
        w = np.ascontiguousarray(w, np.float32)
        assert w.size == self.nparam
        check(self.lib.lce_net_set_params(self.h, _ptr(w)))

    def save(self, path: str):
        check(self.lib.lce_net_save(self.h, path.encode()))

    def load(self, path: str):
        check(self.lib.lce_net_load(self.h, path.encode()))

    def eval(self, L, feat: np.ndarray, target: np.ndarray):
        """(raw output [V][4], gradient [nparam], loss) on caller data in the
        parity-split site order: feat [V][16], target [V][4]."""
        feat = np.ascontiguousarray(feat, np.float32)
        target = np.ascontiguousarray(target, np.float32)
        V = L[0] * L[1] * L[2]
        assert feat.shape == (V, 16) and target.shape == (V, 4)
        out = np.empty((V, 4), np.float32)
        grad = np.empty(self.nparam, np.float32)
        loss = C.c_double()
        check(self.lib.lce_net_eval(self.h, int(L[0]), int(L[1]), int(L[2]), _ptr(feat), _ptr(target), _ptr(out),
                                    _ptr(grad), C.byref(loss)))
        return out, grad, loss.value

    def num_pairs(self) -> int:
        return check(self.lib.lce_net_num_pairs(self.h))

    def clear_pairs(self):
        check(self.lib.lce_net_clear_pairs(self.h))

    def train(self, epochs: int = 1, lr: float = 1e-3) -> float:
        loss = C.c_double()
        check(self.lib.lce_net_train(self.h, int(epochs), float(lr), C.byref(loss)))
        return loss.value


class SlabLattice:
    """A lattice split along z into slabs on one or more GPUs (lce_slabs_*:
    the reference's domain decomposition with a halo exchange after every
    pass).  A sweep reproduces the fields of an undecomposed Lattice with
    the same parameters bit for bit; measurements are the whole lattice's."""

    def __init__(self, L=(16, 16, 16), nslabs=2, devices=None, beta=9.0, x=0.1, y=0.5, **kw):
        self.lib = load()
        self.params = Params(L=tuple(L), beta=beta, x=x, y=y, **kw)
        devs = list(devices) if devices is not None else [self.params.device] * nslabs
        if len(devs) != nslabs:
            raise ValueError("one device per slab")
        arr = (C.c_int * nslabs)(*devs)
        p = self.params.to_c()
        h = self.lib.lce_slabs_create(C.byref(p), nslabs, arr)
        if not h:
            raise _lib.LceError(_lib.LCE_ERR_INVALID, "lce_slabs_create: " + self.lib.lce_last_error(None).decode())
        self.h = C.c_void_p(h)
        self.nh = L[0] * L[1] * L[2] // 2
        self.dtype = np.float64 if self.params.precision == "f64" else np.float32

    def _ck(self, rc):
        if rc < 0:
            raise _lib.LceError(rc, f"{self.lib.lce_strerror(rc).decode()}: {self.lib.lce_last_error(None).decode()}")
        return rc

    def upload(self, u, a):
        f64 = np.asarray(u).dtype == np.float64
        dt = np.float64 if f64 else np.float32
        uu = np.ascontiguousarray(u, dt).reshape(3, 2, self.nh, 4)
        aa = np.ascontiguousarray(a, dt).reshape(2, self.nh, 3)
        fn = self.lib.lce_slabs_upload_f64 if f64 else self.lib.lce_slabs_upload
        self._ck(fn(self.h, _ptr(uu), _ptr(aa), self.nh))

    def download(self, dtype=None, fixed: bool = False):
        """u, a of the whole lattice (fixed: the gauge-fixed u_f, a_f)."""
        dt = dtype or self.dtype
        u = np.zeros((3, 2, self.nh, 4), dt)
        a = np.zeros((2, self.nh, 3), dt)
        if fixed:
            fn = self.lib.lce_slabs_download_fixed_f64 if dt == np.float64 else self.lib.lce_slabs_download_fixed
        else:
            fn = self.lib.lce_slabs_download_f64 if dt == np.float64 else self.lib.lce_slabs_download
        self._ck(fn(self.h, _ptr(u), _ptr(a), self.nh))
        return u, a

    def sweep(self, measflag: int = 1) -> dict:
        m = LceMeas()
        self._ck(self.lib.lce_slabs_sweep(self.h, measflag, C.byref(m)))
        return m.as_dict()

    def set_rng_stream(self, u: np.ndarray):
        """Validation mode (rng="stream", precision="f64"): the whole lattice's
        uniform stream in the reference's consumption order."""
        self._stream = np.ascontiguousarray(u, np.float64)
        self._ck(self.lib.lce_slabs_set_rng_stream(self.h, _ptr(self._stream), self._stream.size))

    def landau_gauge(self, max_iters: int = 0):
        """The overrelaxed Landau gauge fixing of Lattice.landau_gauge on the
        slabs; returns (theta, iterations)."""
        th, it = C.c_double(), C.c_int()
        self._ck(self.lib.lce_slabs_landau_gauge(self.h, C.byref(th), C.byref(it), int(max_iters)))
        return th.value, it.value

    def landau_gauge_from(self, start: str = "identity", max_iters: int = 0):
        """Lattice.landau_gauge_from on the slabs (the transform G tracked;
        start 'identity' or 'transform'); returns (theta, iterations)."""
        th, it = C.c_double(), C.c_int()
        code = {"identity": _lib.LCE_GF_START_IDENTITY, "transform": _lib.LCE_GF_START_TRANSFORM}[start]
        self._ck(self.lib.lce_slabs_landau_gauge_from(self.h, code, C.byref(th), C.byref(it), int(max_iters)))
        return th.value, it.value

    def it_landau_gauge(self, step: float = 0.0, fix_component: bool = False, ascend: bool = False,
                        track: bool = False, max_iters: int = 0):
        """Lattice.it_landau_gauge (f/it_gauge_fixing.f) on the slabs.
        Returns (da1, iterations)."""
        flags = ((_lib.LCE_ITGF_FIX_COMPONENT if fix_component else 0) | (_lib.LCE_ITGF_ASCEND if ascend else 0) |
                 (_lib.LCE_ITGF_TRACK if track else 0))
        da1, it = C.c_double(), C.c_int()
        self._ck(self.lib.lce_slabs_it_landau_gauge(self.h, float(step), flags, C.byref(da1), C.byref(it),
                                                    int(max_iters)))
        return da1.value, it.value

    def landau_gauge_fourier_cg(self, start: str = "identity", theta_switch: float = 0.0, max_iters: int = 0):
        """Lattice.landau_gauge_fourier_cg on the slabs.  Returns (theta,
        fourier_iters, plain_iters)."""
        th, itf, itp = C.c_double(), C.c_int(), C.c_int()
        code = {"identity": _lib.LCE_GF_START_IDENTITY, "transform": _lib.LCE_GF_START_TRANSFORM}[start]
        self._ck(self.lib.lce_slabs_landau_gauge_fourier_cg(self.h, code, float(theta_switch), C.byref(th),
                                                            C.byref(itf), C.byref(itp), int(max_iters)))
        return th.value, itf.value, itp.value

    def landau_gauge_fourier(self, start: str = "identity", step: float = 1.0, theta_switch: float = 0.0,
                             max_iters: int = 0):
        """Lattice.landau_gauge_fourier on the slabs.  Returns (theta,
        fourier_iters, plain_iters)."""
        th, itf, itp = C.c_double(), C.c_int(), C.c_int()
        code = {"identity": _lib.LCE_GF_START_IDENTITY, "transform": _lib.LCE_GF_START_TRANSFORM}[start]
        self._ck(self.lib.lce_slabs_landau_gauge_fourier(self.h, code, float(step), float(theta_switch),
                                                         C.byref(th), C.byref(itf), C.byref(itp), int(max_iters)))
        return th.value, itf.value, itp.value

    def correlator(self):
        L3 = self.params.L[2]
        ca, cu, c3, af = np.zeros(L3), np.zeros(L3), np.zeros(L3), np.zeros(3)
        self._ck(self.lib.lce_slabs_correlator(self.h, _ptr(ca), _ptr(cu), _ptr(c3), _ptr(af)))
        return ca, cu, c3, af

    def polyakov(self):
        L3 = self.params.L[2]
        sl, co, m = np.zeros(L3), np.zeros(L3), C.c_double()
        self._ck(self.lib.lce_slabs_polyakov(self.h, _ptr(sl), _ptr(co), C.byref(m)))
        return sl, co, m.value

    def scalarcorr(self):
        L3 = self.params.L[2]
        sl, co, m = np.zeros(L3), np.zeros(L3), C.c_double()
        self._ck(self.lib.lce_slabs_scalarcorr(self.h, _ptr(sl), _ptr(co), C.byref(m)))
        return sl, co, m.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.lce_slabs_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Lattice(_Context):
    """One chain on one GPU (the drop-in for the reference's single lattice)."""

    def __init__(self, L=(16, 16, 16), beta=9.0, x=0.1, y=0.5, **kw):
        super().__init__([Params(L=tuple(L), beta=beta, x=x, y=y, **kw)])


class Ensemble(_Context):
    """Many independent chains (uneven volumes and couplings) advanced together."""

    def __init__(self, params_list):
        super().__init__(params_list)


# ------------------------------------------------------------------ inputfile
INPUTFILE_KEYS = [
    ("n_lattice", 3, int), ("dimproc", 3, int), ("nproc", 1, int), ("init", 1, int), ("rand", 1, int),
    ("save", 1, int), ("confstart", 1, int), ("beta", 1, float), ("x", 1, float), ("y", 1, float),
    ("lambda", 1, float), ("alpha", 1, float), ("limit_or", 1, float), ("limit_it", 1, float),
    ("inorm", 1, int), ("nsweep_flag", 1, int), ("ntime", 1, int), ("nsweep", 1, int), ("imeas", 1, int),
    ("imode", 1, int),
]


def read_inputfile(path: str) -> dict:
    """The 20-line positional inputfile of f/paraminit.f:82-101 (list-directed
    reads: the leading values of each line, the rest is a comment).  Raises
    ValueError where the reference would abort()."""
    with open(path) as f:
        lines = f.read().splitlines()
    if len(lines) < len(INPUTFILE_KEYS):
        raise ValueError(f"inputfile {path}: {len(lines)} lines, need {len(INPUTFILE_KEYS)}")
    out = {}
    for (key, n, typ), line in zip(INPUTFILE_KEYS, lines):
        tok = line.replace(",", " ").split()
        try:
            vals = [typ(float(t)) if typ is int else float(t.replace("d", "e").replace("D", "E"))
                    for t in tok[:n]]
        except ValueError as e:
            raise ValueError(f"inputfile {path}: bad value for {key}: {line!r}") from e
        if len(vals) < n:
            raise ValueError(f"inputfile {path}: missing value for {key}")
        out[key] = vals if n > 1 else vals[0]
    return out


def params_from_inputfile(cfg: dict, **kw) -> Params:
    return Params(L=tuple(cfg["n_lattice"]), beta=cfg["beta"], x=cfg["x"], y=cfg["y"], lam=cfg["lambda"],
                  alpha=cfg["alpha"], limit_or=cfg["limit_or"], imode=cfg["imode"], **kw)
