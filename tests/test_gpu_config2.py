"""The list kernels on the seeded periodic sphere packing (the indirect-
addressing workload: a periodic box of solid spheres, radius uniform in
[6, 12], porosity 0.40, body force along x, omega 1, 500 steps), pinned to
the reference itself:

* layout: the CUDA rows' grid, adjacency and nCells equal the reference's
  own list-aa-pv-soa and list-pull-split-nt Init
  (src/BenchKernelD3Q19ListAaPvCommon.c:471-823,
  src/BenchKernelD3Q19ListPullSplitNtCommon.c:422-779) bit for bit;
* fields: after 500 steps the FP64 fields are within 1e-12 relative of the
  reference's list-aa-pv-soa and list-pull-split-nt-{1s,2s}-soa
  (src/BenchKernelD3Q19ListAaPv.c:45-851,
  src/BenchKernelD3Q19ListPullSplitNt.c:51-478), which fix Lambda at 1/12
  (src/BenchKernelD3Q19ListAaPv.c:177); and equal to the oracle bit for bit
  at Lambda = 3/16.

A 64^3 packing runs against the reference build live (oracle/_ref). The full
256^3 packing with the bench's seed (6.7M fluid nodes) runs in the same
`-m gpu` pass under the extra marker `big` (deselect with -m "gpu and not
big") against fixtures that the reference build wrote
(tests/golden/make_packing_golden.py): its VERIFICATION list kernels take
tens of minutes for 500 steps at that size on a host's cores."""
import hashlib
import json
import os

import numpy as np
import pytest

import lbmb200
from lbm_cases import random_pdfs

pytestmark = pytest.mark.gpu

ROWS = [("cuda-list-aa-pv-soa", "list-aa-pv-soa", 0),
        ("cuda-list-pull-split-nt-1s-soa", "list-pull-split-nt-1s-soa", 1),
        ("cuda-list-pull-split-nt-2s-soa", "list-pull-split-nt-2s-soa", 1)]

REL_TOL = 1e-12  # FP64 fields against the reference's SIMD-order list kernels
STEPS = 500
XFORCE = 1e-5
PACKING_SEED = 20251203  # the bench's 256^3 packing
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _packing(edge, seed):
    lat, st = lbmb200.spheres((edge,) * 3, seed, 0.40, 6.0, 12.0)
    assert abs(st["porosity"] - 0.40) < 0.02  # spheres of radius up to 12 make 64^3 coarse
    return lat


def _gpu_run(kname, lat, init, lam):
    inst = lbmb200.kernel(kname).init(lat, kernel_args=["-lambda", lam])
    try:
        inst.set_field(init)
        inst.run(lbmb200.case(omega=1.0, xforce=XFORCE, iterations=STEPS))
        return inst.get_field(), inst.list_layout()
    finally:
        inst.deinit()


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _max_rel(a, b):
    return float(np.max(np.abs(a - b) / np.abs(b)))


def _check_against_reference(reference, lat, init):
    m = lat.mask != 0
    report = []
    for kname, rkernel, _ in ROWS:
        g, (grid, adj, nf, nc) = _gpu_run(kname, lat, init, "1/12")
        rg, radj, rnf, rnc = reference.list_layout(rkernel, lat.dims, lat.periodic, lat.mask)
        assert (nf, nc) == (rnf, rnc) and nf == lat.n_fluid
        assert np.array_equal(grid, rg), kname + ": grid differs from the reference"
        assert np.array_equal(adj, radj), kname + ": adjacency differs from the reference"
        r = reference.run(rkernel, lat.dims, lat.periodic, lat.mask, omega=1.0, xforce=XFORCE,
                          iterations=STEPS, init="pdfs", init_pdfs=init)
        rel = _max_rel(g[m], r[m])
        report.append("%s vs %s: max rel %.3e" % (kname, rkernel, rel))
        assert rel <= REL_TOL, report[-1]
    print("; ".join(report))


def test_packing_64_against_reference(reference):
    lat = _packing(64, PACKING_SEED)
    init = random_pdfs(lat.mask.size, 64)
    reference.set_threads(os.cpu_count() or 1)
    try:
        _check_against_reference(reference, lat, init)
    finally:
        reference.set_threads(min(4, os.cpu_count() or 1))


@pytest.mark.parametrize("kname,rkernel", [("cuda-list-push-soa", "list-push-soa"),
                                           ("cuda-list-pull-soa", "list-pull-soa")])
def test_packing_64_two_grid_list_rows_equal_reference(reference, kname, rkernel):
    # the two-grid list rows (src/BenchKernelD3Q19List.c) on the packing, 500
    # forced steps: bit for bit against the reference's scalar kernels
    lat = _packing(64, PACKING_SEED)
    init = random_pdfs(lat.mask.size, 66)
    g, _ = _gpu_run(kname, lat, init, "1/12")
    reference.set_threads(os.cpu_count() or 1)
    try:
        r = reference.run(rkernel, lat.dims, lat.periodic, lat.mask, omega=1.0, xforce=XFORCE, iterations=STEPS,
                          init="pdfs", init_pdfs=init)
    finally:
        reference.set_threads(min(4, os.cpu_count() or 1))
    m = lat.mask != 0
    assert np.array_equal(g[m], r[m])


@pytest.mark.parametrize("kname,okernel", [("cuda-list-aa-pv-soa", "list-aa"),
                                           ("cuda-list-pull-split-nt-1s-soa", "list-pull")])
def test_packing_64_lambda_3_16_equals_oracle(oracle, kname, okernel):
    lat = _packing(64, PACKING_SEED + 1)
    init = random_pdfs(lat.mask.size, 65)
    g, _ = _gpu_run(kname, lat, init, "3/16")
    o = oracle.run(okernel, lat.dims, lat.periodic, lat.mask, omega=1.0, lam=3.0 / 16.0, xforce=XFORCE,
                   iterations=STEPS, init="pdfs", init_pdfs=init)
    m = lat.mask != 0
    assert np.array_equal(g[m], o[m])


@pytest.mark.big
@pytest.mark.parametrize("kname,rkernel,pull", ROWS)
def test_packing_256_against_reference_fixture(kname, rkernel, pull):
    # the bench's domain: 256^3, seed 20251203, ~6.7M fluid nodes, equilibrium
    # start (f_i = w_i), 500 steps. The reference's side was written by the
    # reference build (tests/golden/make_packing_golden.py): layout hashes,
    # 1024 sampled cells and per-plane sums of every direction's PDFs.
    with open(os.path.join(GOLDEN, "packing256.json")) as f:
        meta = json.load(f)
    ref = np.load(os.path.join(GOLDEN, "packing256.npz"))
    lat = _packing(meta["edge"], meta["seed"])
    assert lat.n_fluid == meta["n_fluid"]
    assert _sha(lat.mask) == meta["mask_sha256"]
    init = np.ascontiguousarray(np.broadcast_to(lbmb200.W, (lat.mask.size, 19)))
    g, (grid, adj, nf, nc) = _gpu_run(kname, lat, init, "1/12")
    lay = meta["layouts"]["pull" if pull else "push"]
    assert (nf, nc) == (lay["n_fluid"], lay["n_cells"])
    assert _sha(grid) == lay["grid_sha256"], kname + ": grid differs from the reference"
    assert _sha(adj) == lay["adj_sha256"], kname + ": adjacency differs from the reference"
    key = rkernel.replace("-", "_")
    cells = ref["sample_cells"]
    rel = _max_rel(g[cells], ref["sample_" + key])
    g[lat.mask == 0] = 0.0
    nx, ny, nz = lat.dims
    f = g.reshape(nz, ny, nx, 19)
    planes = np.stack([f.sum(axis=(0, 1)), f.sum(axis=(0, 2)), f.sum(axis=(1, 2))])
    rel_planes = _max_rel(planes, ref["planes_" + key])
    print("%s vs %s (256^3, 500 steps): sampled cells max rel %.3e, plane sums max rel %.3e"
          % (kname, rkernel, rel, rel_planes))
    assert rel <= REL_TOL and rel_planes <= REL_TOL
