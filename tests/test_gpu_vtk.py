"""VTK output of the CUDA rows' Kernel (cd->VtkOutput, the -vtk flag): the
files a run writes, their labels, and their bytes, against the same writer
fed with oracle states (FP64 kernels are bit-identical to the oracle, so the
files are byte-identical)."""
import os

import numpy as np
import pytest

import lbmb200

pytestmark = pytest.mark.gpu

DIMS, GEO, ITERS, MOD = (10, 9, 8), "blocks-2", 6, 2

# label -> steps done when the CUDA rows write it: after each step pair (AA
# forms) or step (pull) whose first step index is a multiple of the modulus
CASES = [("cuda-aa-soa", "aa", {-1: 0, 0: 2, 2: 4, 4: 6, 6: 6}),
         ("cuda-list-aa-pv-soa", "list-aa", {-1: 0, 0: 2, 2: 4, 4: 6, 6: 6}),
         ("cuda-list-pull-split-nt-1s-soa", "list-pull", {-1: 0, 0: 1, 2: 3, 4: 5, 6: 6})]


@pytest.mark.parametrize("kname,okernel,sched", CASES)
def test_kernel_writes_reference_vtk_files(tmp_path, monkeypatch, oracle, kname, okernel, sched):
    lat = lbmb200.geometry(GEO, DIMS, (0, 0, 0))
    monkeypatch.chdir(tmp_path)
    inst = lbmb200.kernel(kname).init(lat)
    try:
        inst.run(lbmb200.case(xforce=1e-5, iterations=ITERS, vtk=MOD))
    finally:
        inst.deinit()
    names = sorted(os.listdir(tmp_path / "vtk"))
    assert names == sorted("file-%04d.vtk" % k for k in sched)
    for label, steps in sched.items():
        f = oracle.run(okernel, DIMS, lat.periodic, lat.mask, xforce=1e-5, iterations=steps, init="zero")
        want = str(tmp_path / ("want_%d.vtk" % label))
        lbmb200.write_vtk_field(lat, f, 1e-5, label, want)
        got = tmp_path / "vtk" / ("file-%04d.vtk" % label)
        assert got.read_bytes() == open(want, "rb").read(), (kname, label)


def test_instance_write_vtk_matches_field_writer(tmp_path, oracle):
    lat = lbmb200.geometry("pipe", (12, 10, 11), (0, 0, 0))
    init = np.random.default_rng(5).uniform(0.01, 0.1, (lat.mask.size, 19))
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat)
    try:
        inst.set_field(init)
        cd = lbmb200.case(xforce=2e-5, iterations=8)
        inst.run(cd)
        inst.write_vtk(cd, 8, str(tmp_path / "a.vtk"))
    finally:
        inst.deinit()
    f = oracle.run("list-aa", lat.dims, lat.periodic, lat.mask, xforce=2e-5, iterations=8, init="pdfs",
                   init_pdfs=init)
    lbmb200.write_vtk_field(lat, f, 2e-5, 8, str(tmp_path / "b.vtk"))
    assert (tmp_path / "a.vtk").read_bytes() == (tmp_path / "b.vtk").read_bytes()
