"""The oracle's RANLUX restatement against the reference's only golden
vectors: the expected output of the luxtst program (f/luxtst.f:88-162),
captured in tests/golden/ranlux_luxtst.json by tests/golden/make_golden.py."""
import json
import os

import numpy as np
import pytest

from oracle.oracle import Ranlux, philox4x32, reference_stream

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ranlux_luxtst.json")))
TOL = 5.1e-9  # the reference prints F12.8


def _check(got, want):
    np.testing.assert_allclose(np.asarray(got, np.float64)[:5], want, rtol=0, atol=TOL)


def test_default_initialisation():
    r = Ranlux()
    r.reset_default()
    _check(r.ranlux(100), GOLD["cases"][0]["first"])
    _check(r.ranlux(100), GOLD["cases"][0]["second"])


@pytest.mark.parametrize("idx,args", [(1, (0, 0)), (2, (389, 1)), (3, (75, 0))])
def test_rluxgo_levels(idx, args):
    r = Ranlux()
    r.rluxgo(*args)
    _check(r.ranlux(100), GOLD["cases"][idx]["first"])
    _check(r.ranlux(100), GOLD["cases"][idx]["second"])


def test_restart_vector_and_roundtrip():
    r = Ranlux()
    r.rluxgo(75, 0)
    r.ranlux(100)
    r.ranlux(100)
    st = r.rluxut()
    assert list(st) == GOLD["restart"]
    a1, a2 = r.ranlux(100), r.ranlux(100)
    _check(a1, GOLD["cases"][4]["first"])
    _check(a2, GOLD["cases"][4]["second"])
    r.rluxin(st)
    b1, b2 = r.ranlux(100), r.ranlux(100)
    np.testing.assert_array_equal(a1, b1)
    np.testing.assert_array_equal(a2, b2)
    _check(b1, GOLD["cases"][5]["first"])


def test_rluxat_and_skip_restart():
    """rluxgo(lux, ins, k1, k2) restarts at a break point given by rluxat
    (f/luxury.f:264-300): skipping must land on the same numbers."""
    r = Ranlux()
    r.rluxgo(4, 7674985, 0, 0)
    for _ in range(10):
        r.ranlux(1000)
    lout, inout, k1, k2 = r.rluxat()
    assert (lout, inout, k2) == (4, 7674985, 0)
    want = r.ranlux(200)
    r.rluxgo(lout, inout, k1, k2)
    got = r.ranlux(200)
    np.testing.assert_array_equal(got, want)


def test_reference_seeding_stream_is_in_open_interval():
    u = reference_stream(10000, seed=314159)
    assert u.min() > 0.0 and u.max() < 1.0


# Philox4x32-10 known-answer vectors published with the Random123 library
# (Salmon et al., SC'11), kat_vectors: (counter, key) -> output.
KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_philox_known_answers(ctr, key, out):
    assert tuple(int(v) for v in philox4x32(ctr, key)) == out
