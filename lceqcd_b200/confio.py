"""Host-side reader/writer of the reference's configuration files (numpy).

f/confsave.f:57-233 and f/confget.f:349-526 store configurations as
unformatted direct-access files in single precision: the links as one record
per (mu, eo, z) -- an xy slice of one parity in half-row order, each site
COMPLEX(2) = (Re a, Im a, Re b, Im b) -- and the Higgs field as one record
per (eo, z) of REAL(3).  The declared record lengths are twice the payload
(u_rl = 16*2*L1*L2/2, a_rl = 8*3*L1*L2/2 bytes); the payload comes first.
Arrays use the reference order u[mu, eo, site, 4], a[eo, site, 3].
"""
from __future__ import annotations

import numpy as np


def _geom(L):
    L1, L2, L3 = (int(v) for v in L)
    nxy = L1 * L2 // 2
    return L1, L2, L3, nxy, nxy * L3


def write_conf(u_path: str, a_path: str, u: np.ndarray, a: np.ndarray, L) -> None:
    L1, L2, L3, nxy, nh = _geom(L)
    u = np.asarray(u, np.float32).reshape(3, 2, L3, nxy, 4)
    a = np.asarray(a, np.float32).reshape(2, L3, nxy, 3)
    urec = np.zeros((3, 2, L3, 2 * nxy * 4), np.float32)
    urec[..., : nxy * 4] = u.reshape(3, 2, L3, nxy * 4)
    arec = np.zeros((2, L3, 2 * nxy * 3), np.float32)
    arec[..., : nxy * 3] = a.reshape(2, L3, nxy * 3)
    urec.tofile(u_path)
    arec.tofile(a_path)


def read_conf(u_path: str, a_path: str, L):
    L1, L2, L3, nxy, nh = _geom(L)
    ub = np.fromfile(u_path, np.float32)
    ab = np.fromfile(a_path, np.float32)
    nu, na = 3 * 2 * L3 * 2 * nxy * 4, 2 * L3 * 2 * nxy * 3
    # the last record may stop after its payload
    if ub.size < nu - nxy * 4 or ab.size < na - nxy * 3:
        raise ValueError("configuration file shorter than the lattice")
    ub = np.concatenate([ub, np.zeros(max(0, nu - ub.size), np.float32)])[:nu]
    ab = np.concatenate([ab, np.zeros(max(0, na - ab.size), np.float32)])[:na]
    u = ub.reshape(3, 2, L3, 2 * nxy * 4)[..., : nxy * 4].reshape(3, 2, nh, 4)
    a = ab.reshape(2, L3, 2 * nxy * 3)[..., : nxy * 3].reshape(2, nh, 3)
    return u.copy(), a.copy()
