"""One AA-pattern lattice split into x-slabs (lbm_aa_slab_*, lbmb200.slabs),
full-array (cuda-aa-soa) and list (cuda-list-aa-pv-soa) layouts: slabs in
one process on one GPU, halo messages through device buffers on one stream,
against the single-instance kernel -- bit for bit after every pair. (With one
slab per GPU the messages travel through torch.distributed instead; that
transport is tested on CPU ranks in test_slabs_gloo.py.)"""
import numpy as np
import pytest

import lbmb200
from lbm_cases import random_pdfs
from lbmb200 import slabs as sl

pytestmark = pytest.mark.gpu

CASES = [
    ("fluid", (24, 10, 12), (1, 1, 1), 2),
    ("box", (12, 9, 8), (0, 1, 1), 3),       # x closed, y/z periodic: edge links wrap to the other x end
    ("fluid", (5, 6, 7), (0, 1, 1), 5),
    ("fluid", (9, 8, 7), (0, 1, 0), 3),
    ("fluid", (25, 9, 11), (1, 1, 1), 3),    # uneven slabs, periodic ring
    ("fluid", (9, 8, 7), (1, 0, 1), 4),      # thin slabs, corner links wrap on several axes
    ("fluid", (6, 7, 8), (1, 1, 0), 3),      # two-plane slabs, open z faces
    ("channel", (30, 12, 14), (0, 0, 0), 3), # closed x faces on the end slabs
    ("box", (20, 10, 12), (0, 1, 1), 2),
    ("blocks-2", (26, 11, 12), (1, 0, 1), 3),
    ("fluid", (9, 8, 7), (0, 0, 0), 2),      # all faces open
]


def _run_slabs(lat, parts, init, cd, pairs, layout="full", kargs=("-lambda", "3/16"), overlap=False):
    import torch
    work = torch.cuda.Stream()  # an explicit stream orders all slabs' operations
    stream = work.cuda_stream
    ring = sl.is_ring(lat.periodic)
    ranges = sl.partition(lat.dims[0], parts)
    slabs = [sl.Slab(lat, x0, x1, *sl.halo_flags(r, parts, ring), kernel_args=list(kargs), layout=layout)
             for r, (x0, x1) in enumerate(ranges)]
    try:
        sl.scatter_field(slabs, lat, init)
        tr = sl.LocalTransport(slabs, ring, stream,
                               lambda n: torch.empty(n, dtype=torch.float64, device="cuda"))
        sl.step_pairs(slabs, tr, cd, pairs, stream, overlap=overlap)
        torch.cuda.synchronize()
        return sl.gather_field(slabs, lat)
    finally:
        for s in slabs:
            s.close()


@pytest.mark.parametrize("geo,dims,per,parts", CASES)
def test_slabs_equal_whole_lattice(geo, dims, per, parts):
    lat = lbmb200.geometry(geo, dims, per)
    init = random_pdfs(lat.mask.size, 31)
    cd = lbmb200.case(omega=1.2, xforce=2e-4, iterations=10)
    inst = lbmb200.kernel("cuda-aa-soa").init(lat, kernel_args=["-lambda", "3/16"])
    try:
        inst.set_field(init)
        inst.run(cd)
        whole = inst.get_field()
    finally:
        inst.deinit()
    got = _run_slabs(lat, parts, init, cd, 5)
    m = lat.mask != 0
    assert np.array_equal(got[m], whole[m])


def test_slab_refuses_halo_on_closed_boundary():
    lat = lbmb200.geometry("fluid", (12, 8, 8), (0, 0, 0))
    with pytest.raises(RuntimeError, match="periodic"):
        sl.Slab(lat, 0, 6, True, True)


def test_slabrun_single_process(capsys):
    from lbmb200 import slabrun
    slabrun.main(["--dims", "32x16x16", "--pairs", "2", "--warmup", "1"])
    out = capsys.readouterr().out.strip().splitlines()[-1]
    import json
    rec = json.loads(out)
    assert rec["ranks"] == 1 and rec["fluid_nodes"] == 32 * 16 * 16 and rec["mflups"] > 0


LIST_CASES = CASES + [
    ("spheres", (30, 24, 24), (1, 1, 1), 3),
    ("spheres", (16, 16, 16), (1, 1, 1), 8),  # slabs of two planes
]


def _lattice(geo, dims, per):
    if geo == "spheres":
        return lbmb200.spheres(dims, 42, 0.45, 2.0, 4.0, 4000)[0]
    return lbmb200.geometry(geo, dims, per)


@pytest.mark.parametrize("geo,dims,per,parts", LIST_CASES)
def test_list_slabs_equal_whole_lattice(geo, dims, per, parts):
    lat = _lattice(geo, dims, per)
    init = random_pdfs(lat.mask.size, 37)
    cd = lbmb200.case(omega=1.1, xforce=2e-4, iterations=10)
    kargs = ["-lambda", "3/16", "-pad", "no"]
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=kargs)
    try:
        inst.set_field(init)
        inst.run(cd)
        whole = inst.get_field()
    finally:
        inst.deinit()
    got = _run_slabs(lat, parts, init, cd, 5, layout="list", kargs=kargs)
    m = lat.mask != 0
    assert np.array_equal(got[m], whole[m])


def test_list_slab_moments_sum_to_whole_lattice():
    """FP64 conservation sums of the slabs' owned nodes add up to the whole
    lattice's (the sums a multi-GPU run all-reduces)."""
    lat = _lattice("spheres", (24, 20, 20), (1, 1, 1))
    init = random_pdfs(lat.mask.size, 5)
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=["-lambda", "3/16"])
    try:
        inst.set_field(init)
        whole = np.array(inst.moments())
    finally:
        inst.deinit()
    ring = sl.is_ring(lat.periodic)
    slabs = [sl.Slab(lat, x0, x1, *sl.halo_flags(r, 3, ring), kernel_args=["-lambda", "3/16"], layout="list")
             for r, (x0, x1) in enumerate(sl.partition(lat.dims[0], 3))]
    try:
        sl.scatter_field(slabs, lat, init)
        parts = np.sum([np.array(s.inst.moments()) for s in slabs], axis=0)
    finally:
        for s in slabs:
            s.close()
    assert np.allclose(parts, whole, rtol=1e-12, atol=1e-12)


def test_slabrun_list_layout_single_process(capsys):
    from lbmb200 import slabrun
    slabrun.main(["--dims", "32x24x24", "--geometry", "spheres:7:0.5:2:4", "--layout", "list",
                  "--pairs", "2", "--warmup", "1"])
    import json
    rec = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert rec["layout"] == "list" and rec["mflups"] > 0
    # the flow starts at rest with f = w: the mass is one per fluid node
    assert abs(rec["sum_rho"] - rec["fluid_nodes"]) < 1e-9 * rec["fluid_nodes"]
    assert rec["sum_jx"] > 0 and rec["permeability"] > 0


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
@pytest.mark.parametrize("geo,dims,per,parts", [
    ("spheres", (30, 24, 24), (1, 1, 1), 3),
    ("channel", (30, 12, 14), (0, 0, 0), 3),
    ("fluid", (9, 8, 7), (0, 1, 0), 3),
])
def test_reduced_storage_list_slabs_equal_whole_lattice(prec, geo, dims, per, parts):
    """FP32 / FP16 list slabs: halo messages carry the stored elements bit for
    bit, so the slabs equal the single reduced-storage instance exactly."""
    lat = _lattice(geo, dims, per)
    rng = np.random.default_rng(3)
    w = lbmb200.W
    init = w[None, :] * (1.0 + 0.05 * (rng.random((lat.mask.size, 19)) - 0.5))
    cd = lbmb200.case(omega=1.1, xforce=2e-4, iterations=10)
    kargs = ["-lambda", "3/16", "-precision", prec]
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=kargs)
    try:
        inst.set_field(init)
        inst.run(cd)
        whole = inst.get_field()
    finally:
        inst.deinit()
    got = _run_slabs(lat, parts, init, cd, 5, layout="list", kargs=kargs)
    m = lat.mask != 0
    assert np.array_equal(got[m], whole[m])


def test_slabrun_list_fp32_single_process(capsys):
    from lbmb200 import slabrun
    slabrun.main(["--dims", "32x24x24", "--geometry", "spheres:7:0.5:2:4", "--layout", "list",
                  "--precision", "fp32", "--pairs", "2", "--warmup", "1", "--overlap"])
    import json
    rec = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert rec["precision"] == "fp32" and rec["overlap"] and rec["mflups"] > 0
    assert abs(rec["sum_rho"] - rec["fluid_nodes"]) < 1e-6 * rec["fluid_nodes"]
    assert rec["sum_jx"] > 0 and rec["permeability"] > 0


@pytest.mark.parametrize("layout,kargs,geo,dims,per,parts", [
    ("full", ["-lambda", "3/16"], "fluid", (25, 9, 11), (1, 1, 1), 3),
    ("full", ["-lambda", "3/16"], "channel", (30, 12, 14), (0, 0, 0), 3),
    ("list", ["-lambda", "3/16", "-pad", "no"], "spheres", (30, 24, 24), (1, 1, 1), 3),
    ("list", ["-lambda", "3/16", "-precision", "fp32"], "spheres", (30, 24, 24), (1, 1, 1), 2),
    ("list", ["-lambda", "3/16", "-precision", "fp16"], "spheres", (30, 24, 24), (1, 1, 1), 2),  # even step whole
    ("list", ["-lambda", "3/16", "-blk", "4"], "fluid", (16, 12, 12), (1, 1, 1), 2),  # no inner tile range
])
def test_overlapped_steps_equal_whole_lattice(layout, kargs, geo, dims, per, parts):
    """The odd step in two parts around the phase-0 exchange and the next
    even step in two parts around the phase-1 exchange
    (lbm_aa_slab_odd_part / lbm_aa_slab_even_part) leave the single
    instance's bits."""
    lat = _lattice(geo, dims, per)
    rng = np.random.default_rng(8)
    init = lbmb200.W[None, :] * (1.0 + 0.05 * (rng.random((lat.mask.size, 19)) - 0.5))
    cd = lbmb200.case(omega=1.1, xforce=2e-4, iterations=10)
    kname = "cuda-aa-soa" if layout == "full" else "cuda-list-aa-pv-soa"
    inst = lbmb200.kernel(kname).init(lat, kernel_args=kargs)
    try:
        inst.set_field(init)
        inst.run(cd)
        whole = inst.get_field()
    finally:
        inst.deinit()
    got = _run_slabs(lat, parts, init, cd, 5, layout=layout, kargs=kargs, overlap=True)
    m = lat.mask != 0
    assert np.array_equal(got[m], whole[m])
