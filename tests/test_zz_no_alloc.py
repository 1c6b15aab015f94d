"""The allocation-free plaquette entry point (lce_plaquette_noalloc).

It exists for callers that cannot let the library allocate device memory (a
driver whose GPU memory belongs to another allocator, or code between
asynchronous launches where cudaMalloc/cudaFree could synchronise the
device).  The caller owns the input field and the output; the scratch is a
fixed __device__ array shared by all calls.  This file is collected last so a
run that stops at the first failure has already run every other test.

Checked through the C ABI against the context-based lce_plaquette on the same
configuration, on two calls in a row, at the 1e-12 relative tolerance the FP64
reductions are held to elsewhere; and the size limit of the fixed scratch.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
lce = pytest.importorskip("lceqcd_b200")
torch = pytest.importorskip("torch")

TOL = 1e-12


@pytest.mark.parametrize("L", [(8, 8, 8), (16, 12, 10), (32, 32, 32)])
def test_noalloc_plaquette_matches_context_entry_point(L):
    from lceqcd_b200 import Lattice
    lib = lce.load()
    lat = Lattice(L, beta=9.0, x=0.1, y=0.45, precision="f32")
    lat.init_hot(7)
    ref = lat.plaquette()
    u, _ = lat.download()                        # reference order, FP32
    nh = u.shape[2]
    ud = torch.from_numpy(np.ascontiguousarray(u)).cuda()
    out = torch.full((1,), -1.0, dtype=torch.float64, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        rc = lib.lce_plaquette_noalloc(C.c_void_p(ud.data_ptr()), nh, L[0], L[1], L[2],
                                       C.c_void_p(out.data_ptr()), stream)
        assert rc == 0, lib.lce_last_error(None)
        torch.cuda.synchronize()
        assert abs(out.item() - ref) <= TOL * max(1.0, abs(ref))
    # a second configuration through the same shared scratch
    lat.sweeps(3, 0)
    ref2 = lat.plaquette()
    u2, _ = lat.download()
    ud.copy_(torch.from_numpy(np.ascontiguousarray(u2)))
    rc = lib.lce_plaquette_noalloc(C.c_void_p(ud.data_ptr()), nh, L[0], L[1], L[2],
                                   C.c_void_p(out.data_ptr()), stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert abs(out.item() - ref2) <= TOL * max(1.0, abs(ref2))
    lat.close()


def test_noalloc_rejects_sizes_beyond_scratch():
    lib = lce.load()
    dummy = torch.zeros(16, dtype=torch.float32, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.lce_plaquette_noalloc(C.c_void_p(dummy.data_ptr()), 1 << 30, 258, 256, 256,
                                   C.c_void_p(out.data_ptr()), None)
    assert rc == lce._lib.LCE_ERR_INVALID
    assert b"scratch capacity" in lib.lce_last_error(None)
    rc = lib.lce_plaquette_noalloc(C.c_void_p(dummy.data_ptr()), 4, 4, 4, 5,
                                   C.c_void_p(out.data_ptr()), None)
    assert rc == lce._lib.LCE_ERR_INVALID
