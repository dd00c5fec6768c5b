"""Reduced-storage list AA (-precision fp32 / fp16) against the FP64 oracle.

The FP32 form stores f_i - w_i as float, the FP16 form stores
(f_i - w_i) * 2^k_i as half; both relax in FP32 on these deviations.
Tolerances (absolute, on PDFs of size ~w_i, after 20 steps from a seeded 5 %
perturbation): FP32 1e-7, FP16 5e-5."""
import numpy as np
import pytest

import lbmb200
from lbm_cases import random_pdfs

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-7, "fp16": 5e-5}


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
@pytest.mark.parametrize("geo,dims,per", [("pipe", (14, 12, 13), (0, 0, 0)), ("blocks-2", (13, 11, 12), (0, 1, 0)),
                                          ("fluid", (9, 8, 7), (1, 1, 1))])
def test_reduced_storage_close_to_fp64_oracle(oracle, prec, geo, dims, per):
    lat = lbmb200.geometry(geo, dims, per)
    init = random_pdfs(lat.mask.size, 17)
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=["-precision", prec, "-lambda", "3/16"])
    try:
        inst.set_field(init)
        inst.run(lbmb200.case(omega=1.3, xforce=2e-4, iterations=20))
        g = inst.get_field()
    finally:
        inst.deinit()
    o = oracle.run("list-aa", dims, lat.periodic, lat.mask, omega=1.3, lam=3.0 / 16.0, xforce=2e-4,
                   iterations=20, init="pdfs", init_pdfs=init)
    m = lat.mask != 0
    err = np.max(np.abs(g[m] - o[m]))
    assert err < TOL[prec], err


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_reduced_storage_conserves_mass(prec):
    lat = lbmb200.geometry("fluid", (24, 20, 16), (1, 1, 1))
    init = random_pdfs(lat.mask.size, 11)
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=["-precision", prec])
    try:
        inst.set_field(init)
        start = inst.get_field().sum()  # the stored (rounded) start
        inst.run(lbmb200.case(omega=1.5, xforce=0.0, iterations=200))
        end = inst.get_field().sum()
    finally:
        inst.deinit()
    assert abs(end - start) / start < (1e-9 if prec == "fp32" else 1e-4)
