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

from conftest import rel_err

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
        dev_links = torch.from_numpy(links.reshape(-1)).cuda()
        dev_obs = torch.zeros(3 + dims[3], dtype=torch.float64, device="cuda")
        for call in range(2):
            dev_obs.fill_(np.nan)
            st = L.glac_measure_noalloc((ctypes.c_int * 4)(*dims), dev_links.data_ptr(), dev_obs.data_ptr(), None)
            assert st == 0, L.glac_noalloc_error().decode()
            torch.cuda.synchronize()
            got = dev_obs.cpu().numpy()
            assert np.all(np.isfinite(got)), (dims, call)
            assert rel_err(got, want) < 1e-12, (dims, call)


def test_measure_noalloc_rejects_oversize():
    L = _lib()
    dummy = ctypes.c_void_p(16)
    st = L.glac_measure_noalloc((ctypes.c_int * 4)(4, 4, 4, 5000), dummy, dummy, None)
    assert st == 1
    assert "scratch capacity" in L.glac_noalloc_error().decode()
