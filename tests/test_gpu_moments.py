"""FP64 conservation sums on the GPU (lbm_b200_moments_device) against the
host sums of the same field read back through GetNode."""
import ctypes

import numpy as np
import pytest

import lbmb200
from lbm_cases import CX, CY, CZ, random_pdfs

pytestmark = pytest.mark.gpu


def _device_sums(inst):
    import torch
    L = lbmb200.lib()
    pdfs = ctypes.c_void_p()
    ncells = ctypes.c_longlong()
    nfluid = ctypes.c_int()
    stream = ctypes.c_void_p()
    assert L.lbm_b200_device_state(inst.kdp, ctypes.byref(pdfs), ctypes.byref(ncells), ctypes.byref(nfluid),
                                   ctypes.byref(stream)) == 0
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = L.lbm_b200_moments_device(pdfs, ncells, nfluid, ctypes.c_void_p(out.data_ptr()), stream)
    assert rc == 0
    return out.cpu().numpy()


@pytest.mark.parametrize("kname", ["cuda-list-aa-pv-soa", "cuda-list-pull-split-nt-1s-soa"])
@pytest.mark.parametrize("geo,dims,per", [("pipe", (20, 18, 17), (0, 0, 0)), ("fluid", (33, 7, 40), (1, 1, 1))])
def test_moments_match_host_sums(kname, geo, dims, per):
    lat = lbmb200.geometry(geo, dims, per)
    inst = lbmb200.kernel(kname).init(lat)
    try:
        inst.set_field(random_pdfs(lat.mask.size, 5))
        inst.run(lbmb200.case(omega=1.4, xforce=3e-4, iterations=6))
        got = _device_sums(inst)
        f = inst.get_field()[lat.mask != 0]
    finally:
        inst.deinit()
    want = np.array([f.sum(), (f * CX).sum(), (f * CY).sum(), (f * CZ).sum()])
    assert abs(got[0] - want[0]) / want[0] < 1e-12
    scale = np.abs(f).sum()
    assert np.all(np.abs(got[1:] - want[1:]) / scale < 1e-12)


def test_moments_deterministic():
    lat = lbmb200.geometry("fluid", (40, 30, 20), (1, 1, 1))
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat)
    try:
        inst.set_field(random_pdfs(lat.mask.size, 9))
        inst.run(lbmb200.case(omega=1.0, xforce=0.0, iterations=2))
        a = _device_sums(inst)
        b = _device_sums(inst)
    finally:
        inst.deinit()
    assert np.array_equal(a, b)


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_reduced_storage_instance_moments(prec):
    """lbm_b200_instance_moments on FP32/FP16 storage: FP64 sums of the stored
    deviations plus the node count, against the host sums of the field the
    instance hands back through GetNode (weights plus the same deviations)."""
    lat, _ = lbmb200.spheres((28, 24, 20), 4, 0.5, 2.0, 4.0, 3000)
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=["-precision", prec])
    try:
        rng = np.random.default_rng(2)
        inst.set_field(lbmb200.W[None, :] * (1.0 + 0.05 * (rng.random((lat.mask.size, 19)) - 0.5)))
        inst.run(lbmb200.case(omega=1.2, xforce=3e-4, iterations=6))
        got = np.array(inst.moments())
        f = inst.get_field()[lat.mask != 0]
    finally:
        inst.deinit()
    want = np.array([f.sum(), (f * CX).sum(), (f * CY).sum(), (f * CZ).sum()])
    assert abs(got[0] - want[0]) / want[0] < 1e-12
    scale = np.abs(f).sum()
    assert np.all(np.abs(got[1:] - want[1:]) / scale < 1e-12)
