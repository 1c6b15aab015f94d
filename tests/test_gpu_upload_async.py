"""lce_upload_async: the host-to-device copy on the context's copy stream,
then a device copy into the fields on the context stream.

The update calls queued after it must see exactly the uploaded fields, and a
pipelined client (step k+1's upload queued before step k's measurements are
read) must get the same results as one that uploads and sweeps in turn.
"""
import numpy as np
import pytest
import torch

from lceqcd_b200 import _lib
from lceqcd_b200.lattice import Lattice

pytestmark = pytest.mark.gpu

L = (32, 16, 24)
KW = dict(beta=12.0, x=0.09, y=0.3, seed=11, sweep_mode="passes")


def _configs(n):
    g = Lattice(L, **KW)
    out = []
    for k in range(n):
        g.init_hot(100 + k)
        g.sweeps(2, 0)
        out.append(g.download())
    g.close()
    return out


def _pinned(u, a):
    pu = torch.empty(u.shape, dtype=torch.float32, pin_memory=True).numpy()
    pa = torch.empty(a.shape, dtype=torch.float32, pin_memory=True).numpy()
    pu[...] = u
    pa[...] = a
    return pu, pa


def test_upload_async_equals_upload():
    (u, a), = _configs(1)
    res = []
    for mode in ("sync", "async"):
        g = Lattice(L, **KW)
        g.init_hot(1)
        if mode == "sync":
            g.upload(u, a)
        else:
            g.upload_async(*_pinned(u, a))
        got = g.download()
        np.testing.assert_array_equal(got[0], u)
        np.testing.assert_array_equal(got[1], a)
        ms = g.sweep(1)
        res.append((g.download(), ms))
        g.close()
    np.testing.assert_array_equal(res[0][0][0], res[1][0][0])
    np.testing.assert_array_equal(res[0][0][1], res[1][0][1])
    assert res[0][1] == res[1][1]


def test_pipelined_client_matches_sequential():
    """Four configurations streamed through one context: upload k+1 queued
    before reading step k's measurements."""
    cfgs = _configs(4)
    seq = []
    g = Lattice(L, **KW)
    for u, a in cfgs:
        g.upload(u, a)
        seq.append((g.sweep(1), g.download()))
    g.close()
    pins = [_pinned(u, a) for u, a in cfgs]
    g = Lattice(L, **KW)
    pipe = []
    g.upload_async(*pins[0])
    for k in range(4):
        g.sweeps(1, 1)
        if k + 1 < 4:
            g.upload_async(*pins[k + 1])
        pipe.append(g.meas1())
    g.close()
    # the Philox counters advance identically in both clients
    for (m_seq, _), m_pipe in zip(seq, pipe):
        assert m_seq == m_pipe


def test_streaming_client_two_slots_matches_sequential():
    """lce_upload_stage two steps ahead, lce_upload_apply behind each sweep:
    every step sweeps its own configuration."""
    cfgs = _configs(5)
    seq = []
    g = Lattice(L, **KW)
    for u, a in cfgs:
        g.upload(u, a)
        seq.append(g.sweep(1))
    g.close()
    pins = [_pinned(u, a) for u, a in cfgs]
    g = Lattice(L, **KW)
    got = []
    g.upload_stage(*pins[0])
    g.upload_apply()
    g.upload_stage(*pins[1])
    for k in range(5):
        g.sweeps(1, 1)
        got.append(g.meas1())
        if k + 1 < 5:
            g.upload_apply()
        if k + 2 < 5:
            g.upload_stage(*pins[k + 2])
    with pytest.raises(_lib.LceError):
        g.upload_apply()  # nothing staged
    g.close()
    assert got == seq


def test_upload_stage_refuses_a_third_pending_upload():
    (u, a), = _configs(1)
    g = Lattice(L, **KW)
    p = _pinned(u, a)
    g.upload_stage(*p)
    g.upload_stage(*p)
    with pytest.raises(_lib.LceError):
        g.upload_stage(*p)
    g.upload_apply()
    g.upload_apply()
    np.testing.assert_array_equal(g.download()[0], u)
    g.close()


def test_upload_async_fp64_context_unsupported():
    g = Lattice((8, 8, 8), beta=9.0, x=0.1, y=0.5, precision="f64", seed=2)
    u, a = g.download()
    with pytest.raises(_lib.LceError):
        g.upload_async(u.astype(np.float32), a.astype(np.float32))
    g.close()
