"""The allocation-free measurement entry point, called through the C ABI.

glac_measure_noalloc serves callers that cannot allocate device memory (a host
framework that owns all GPU memory through its own pool, or a phase where a
driver allocation would stall other streams): they hand over the field and the
output vector in device memory they already own.  Here those buffers come from
torch, the entry point itself allocates nothing, and its result must match the
context path (glac_measure) to FP64 rounding on two calls in a row, which also
checks that the shared scratch array carries nothing over between calls.
This file sorts last so a stop-at-first-failure run has done everything else.
"""
import ctypes

import numpy as np
import pytest

from conftest import assert_obs_close

pytestmark = pytest.mark.gpu


def _lib():
    import glac_b200
    L = glac_b200.lib()
    L.glac_measure_noalloc.argtypes = [ctypes.c_int * 4, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.glac_measure_noalloc.restype = ctypes.c_int
    L.glac_noalloc_error.restype = ctypes.c_char_p
    return L


def test_measure_noalloc_matches_context_path(oracle):
    import torch
    import glac_b200 as g

    L = _lib()
    fields = [((8, 8, 8, 16), 501), ((6, 4, 6, 8), 502)]
    for dims, seed in fields:
        links = oracle.haar_field(dims, seed)
        with g.Lattice(dims, precision="fp64") as lat:
            lat.set_links(links)
            want = lat.measure()
        assert_obs_close(want, oracle.observables(dims, links), 1e-12, f"{dims} context path vs oracle")
        dev_links = torch.from_numpy(links.reshape(-1)).cuda()
        dev_obs = torch.zeros(3 + dims[3], dtype=torch.float64, device="cuda")
        for call in range(2):
            dev_obs.fill_(np.nan)
            st = L.glac_measure_noalloc((ctypes.c_int * 4)(*dims), dev_links.data_ptr(), dev_obs.data_ptr(), None)
            assert st == 0, L.glac_noalloc_error().decode()
            torch.cuda.synchronize()
            got = dev_obs.cpu().numpy()
            assert np.all(np.isfinite(got)), (dims, call)
            assert_obs_close(got, want, 1e-12, f"{dims} call {call} vs glac_measure")
            assert_obs_close(got, oracle.observables(dims, links), 1e-12, f"{dims} call {call} vs oracle")


def test_measure_noalloc_rejects_oversize():
    L = _lib()
    dummy = ctypes.c_void_p(16)
    st = L.glac_measure_noalloc((ctypes.c_int * 4)(4, 4, 4, 5000), dummy, dummy, None)
    assert st == 1
    assert "scratch capacity" in L.glac_noalloc_error().decode()


def test_measure_noalloc_rejects_misaligned_buffers():
    # the field is read as 16-byte words and the output written as doubles:
    # buffers off those boundaries are refused on the host, before any launch
    import torch

    L = _lib()
    dims = (4, 4, 4, 4)
    buf = torch.zeros(4 * 256 * 18 + 2, dtype=torch.float64, device="cuda")
    obs = torch.zeros(3 + 4 + 1, dtype=torch.float64, device="cuda")
    assert buf.data_ptr() % 16 == 0
    st = L.glac_measure_noalloc((ctypes.c_int * 4)(*dims), buf.data_ptr() + 8, obs.data_ptr(), None)
    assert st == 1 and "16-byte" in L.glac_noalloc_error().decode()
    st = L.glac_measure_noalloc((ctypes.c_int * 4)(*dims), buf.data_ptr(), obs.data_ptr() + 4, None)
    assert st == 1 and "8-byte" in L.glac_noalloc_error().decode()


def test_measure_noalloc_rejects_volume_overflow():
    # extents whose product wraps a 64-bit integer are refused before it is formed
    L = _lib()
    dummy = ctypes.c_void_p(256)
    st = L.glac_measure_noalloc((ctypes.c_int * 4)(1 << 21, 1 << 21, 1 << 21, 2), dummy, dummy, None)
    assert st == 1 and "too large" in L.glac_noalloc_error().decode()
