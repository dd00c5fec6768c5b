"""The allocation-free conservation sums (lbm_b200_moments_noalloc).

Callers that cannot call cudaMalloc -- code that runs while another component
owns the device allocator, or that may only use the device buffers its host
application hands it -- get the same FP64 mass/momentum sums as
lbm_b200_moments_device, with the reduction scratch held in a fixed array in
the library instead of a per-call allocation. This test calls both entry
points through the C ABI on the same device field, twice in a row on two
different states (the shared scratch keeps the previous call's contents), and
checks that sizes beyond the fixed scratch are refused. The output buffers
belong to the caller; here torch provides them.

Kept in a file of its own, collected last, so that a run stopping at the
first failure has run every other test before this one.
"""
import ctypes

import numpy as np
import pytest

import lbmb200
from lbm_cases import random_pdfs

pytestmark = pytest.mark.gpu


def _state(inst):
    pdfs, ncells, nfluid, stream = ctypes.c_void_p(), ctypes.c_longlong(), ctypes.c_int(), ctypes.c_void_p()
    rc = lbmb200.lib().lbm_b200_device_state(inst.kdp, ctypes.byref(pdfs), ctypes.byref(ncells),
                                             ctypes.byref(nfluid), ctypes.byref(stream))
    assert rc == 0
    return pdfs, ncells, nfluid, stream


def test_noalloc_moments_match_allocating_entry_point():
    import torch
    L = lbmb200.lib()
    lat = lbmb200.geometry("pipe", (24, 20, 22), (1, 0, 0))
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat)
    try:
        inst.set_field(random_pdfs(lat.mask.size, 21))
        inst.run(lbmb200.case(omega=1.3, xforce=2e-4, iterations=4))
        for call in range(2):
            if call == 1:
                # a second state, so that stale scratch from the first call would show
                inst.run(lbmb200.case(omega=0.9, xforce=-1e-4, iterations=6))
            pdfs, ncells, nfluid, stream = _state(inst)
            want = torch.zeros(4, dtype=torch.float64, device="cuda")
            got = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            assert L.lbm_b200_moments_device(pdfs, ncells, nfluid, ctypes.c_void_p(want.data_ptr()), stream) == 0
            assert L.lbm_b200_moments_noalloc(pdfs, ncells, nfluid, ctypes.c_void_p(got.data_ptr()), stream) == 0
            torch.cuda.synchronize()
            w, g = want.cpu().numpy(), got.cpu().numpy()
            assert np.all(np.isfinite(g))
            np.testing.assert_allclose(g, w, rtol=1e-12, atol=1e-12 * abs(w[0]))
    finally:
        inst.deinit()


def test_noalloc_moments_refuses_more_nodes_than_its_scratch():
    L = lbmb200.lib()
    lat = lbmb200.geometry("fluid", (8, 8, 8), (1, 1, 1))
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat)
    try:
        pdfs, _, _, stream = _state(inst)
        import torch
        out = torch.zeros(4, dtype=torch.float64, device="cuda")
        too_many = 65536 * 256 + 1
        # refused before anything is launched
        rc = L.lbm_b200_moments_noalloc(pdfs, ctypes.c_longlong(too_many), too_many,
                                        ctypes.c_void_p(out.data_ptr()), stream)
        assert rc == -2
    finally:
        inst.deinit()
