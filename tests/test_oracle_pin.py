"""Pins the CPU oracle (oracle/lbm_oracle.c) to the reference.

Against the reference itself (oracle/_ref, compiled from the reference sources;
skipped when absent) and against the committed fixtures in tests/golden/ and
the reference's known -verify answers.
"""
import hashlib
import json
import os
import zlib

import numpy as np
import pytest

from lbm_cases import FIELD_CASES, random_pdfs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
GEOMS = ["box", "channel", "pipe", "blocks", "blocks-3", "fluid"]
PERIODIC = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 1), (1, 1, 1), (0, 0, 1)]
DIMS = [(16, 16, 16), (17, 9, 13), (7, 9, 8)]


def _geom_cases():
    for g in GEOMS:
        for p in PERIODIC:
            for d in DIMS:
                bs = 8 if g == "blocks" else (3 if g == "blocks-3" else 0)
                if bs and bs > min(d) // 2:
                    continue
                yield g, p, d


@pytest.mark.parametrize("geo,per,dims", list(_geom_cases()))
def test_geometry_matches_reference(oracle, reference, geo, per, dims):
    a, ia = oracle.geometry(geo, dims, per)
    b, ib = reference.geometry(geo, dims, per)
    assert np.array_equal(a, b)
    assert ia == ib


def _sha(*arrs):
    h = hashlib.sha256()
    for a in arrs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_geometry_golden(oracle):
    with open(os.path.join(GOLDEN, "geometry.json")) as f:
        gold = json.load(f)
    assert len(gold) > 50
    for key, rec in gold.items():
        geo, per, dims = rec["geo"], tuple(rec["periodic"]), tuple(rec["dims"])
        lat, info = oracle.geometry(geo, dims, per)
        assert _sha(lat) == rec["sha256"], key
        assert info["nFluid"] == rec["nFluid"] and list(info["ldPeriodic"]) == rec["ldPeriodic"], key


LAYOUT_CASES = [
    ("box", (16, 16, 16), (1, 1, 0), []),
    ("channel", (12, 10, 9), (0, 0, 0), []),
    ("fluid", (9, 8, 7), (1, 0, 1), []),
    ("pipe", (10, 12, 11), (0, 0, 0), ["-blk", "7"]),
    ("blocks-2", (13, 11, 12), (0, 1, 0), ["-pad", "no"]),
    ("box", (16, 16, 16), (1, 1, 0), ["-blk-x", "3", "-blk-z", "5"]),
]


def _kargs_to_oracle(kargs):
    blk = [0, 0, 0]
    pad = 0
    i = 0
    while i < len(kargs):
        a = kargs[i]
        if a == "-blk":
            blk = [int(kargs[i + 1])] * 3
        elif a.startswith("-blk-"):
            blk["xyz".index(a[-1])] = int(kargs[i + 1])
        elif a == "-pad":
            pad = {"no": 1, "auto": 0}.get(kargs[i + 1], 2)
        i += 2
    return tuple(blk), pad


@pytest.mark.parametrize("pull", [0, 1])
@pytest.mark.parametrize("geo,dims,per,kargs", LAYOUT_CASES)
def test_list_layout_matches_reference(oracle, reference, pull, geo, dims, per, kargs):
    lat, _ = reference.geometry(geo, dims, per)
    kernel = "list-pull-split-nt-1s-soa" if pull else "list-aa-pv-soa"
    blk, pad = _kargs_to_oracle(kargs)
    g1, a1, nf1, nc1 = reference.list_layout(kernel, dims, per, lat, kargs)
    g2, a2, nf2, nc2 = oracle.list_layout(pull, dims, per, lat, blk, pad)
    assert (nf1, nc1) == (nf2, nc2)
    assert np.array_equal(g1, g2)
    assert np.array_equal(a1, a2)


def test_pad_cells_known_values(oracle):
    # auto padding of the reference (src/Padding.c:24-41): 2 MiB-page and L2-set offsets
    assert oracle.pad_cells(3584) == 3584 + 260624
    assert oracle.pad_cells(1) > 1
    assert oracle.pad_cells(1000, pad_mode=1) == 1000


@pytest.mark.parametrize("kernel,pull", [("list-push-soa", 0), ("list-pull-soa", 2), ("list-aa-soa", 0),
                                         ("list-aa-ria-soa", 0)])
@pytest.mark.parametrize("geo,dims,per,kargs", LAYOUT_CASES[:4])
def test_other_list_layouts_match_reference(oracle, reference, kernel, pull, geo, dims, per, kargs):
    # the two-grid list kernels and the other list-AA variants share the
    # numbering and adjacency rules; two-grid pull has no cache-line pad
    lat, _ = reference.geometry(geo, dims, per)
    blk, pad = _kargs_to_oracle(kargs)
    g1, a1, nf1, nc1 = reference.list_layout(kernel, dims, per, lat, kargs)
    g2, a2, nf2, nc2 = oracle.list_layout(pull, dims, per, lat, blk, pad)
    assert (nf1, nc1) == (nf2, nc2)
    assert np.array_equal(g1, g2) and np.array_equal(a1, a2)


@pytest.mark.parametrize("kernel,okernel,exact", [
    ("aa-soa", "aa", True),
    ("list-pull-split-nt-1s-soa", "list-pull", False),
    ("list-pull-split-nt-2s-soa", "list-pull", False),
    ("list-aa-pv-soa", "list-aa", False),
    ("list-aa-soa", "list-aa", True),
    ("list-aa-ria-soa", "list-aa", True),
    ("list-push-soa", "list-push2", True),
    ("list-pull-soa", "list-pull2", True),
    ("push-soa", "push-fa", True),
    ("pull-soa", "pull-fa", True),
])
@pytest.mark.parametrize("geo,dims,per", FIELD_CASES)
def test_fields_match_reference(oracle, reference, kernel, okernel, exact, geo, dims, per):
    lat, _ = reference.geometry(geo, dims, per)
    init = random_pdfs(lat.size, seed=zlib.crc32(repr((geo, dims, per)).encode()) % 1000)
    kw = dict(omega=1.3, xforce=2e-4, iterations=20, init="pdfs", init_pdfs=init)
    r = reference.run(kernel, dims, per, lat, **kw)
    o = oracle.run(okernel, dims, per, lat, lam=1.0 / 12.0, **kw)
    m = lat != 0
    if exact:
        assert np.array_equal(r[m], o[m])
    else:
        # the reference's SIMD paths sum in a different order than its scalar
        # path: rounding-level differences only
        assert np.max(np.abs(r[m] - o[m]) / np.abs(r[m])) < 1e-13


@pytest.mark.parametrize("okernel", ["aa", "list-aa", "list-pull", "list-push2", "list-pull2", "push-fa", "pull-fa"])
def test_verify_known_answer_lambda_1_12(oracle, okernel):
    # reference -verify (16^3 box, periodic x/y, 1000 steps): 4.561374e-02
    dims, per = (16, 16, 16), (1, 1, 0)
    lat, _ = oracle.geometry("box", dims, per)
    f = oracle.run(okernel, dims, per, lat, lam=1.0 / 12.0, iterations=1000, init="verify")
    assert "%e" % oracle.verify_error(dims, lat, f) == "4.561374e-02"


@pytest.mark.parametrize("okernel", ["aa", "list-aa", "list-pull", "list-push2", "list-pull2", "push-fa", "pull-fa"])
def test_verify_known_answer_lambda_3_16(oracle, okernel):
    # reference with Lambda = 3/16 at the -verify preset: 7.855978e-02
    dims, per = (16, 16, 16), (1, 1, 0)
    lat, _ = oracle.geometry("box", dims, per)
    f = oracle.run(okernel, dims, per, lat, lam=3.0 / 16.0, iterations=1000, init="verify")
    assert "%e" % oracle.verify_error(dims, lat, f) == "7.855978e-02"


def test_fields_golden(oracle):
    """Fixtures written by the reference itself (tests/golden/make_golden.py)."""
    with open(os.path.join(GOLDEN, "fields.json")) as f:
        gold = json.load(f)
    for key, rec in gold.items():
        dims, per = tuple(rec["dims"]), tuple(rec["periodic"])
        lat, _ = oracle.geometry(rec["geo"], dims, per)
        init = random_pdfs(lat.size, seed=rec["seed"])
        o = oracle.run(rec["okernel"], dims, per, lat, omega=rec["omega"], lam=1.0 / 12.0,
                       xforce=rec["xforce"], iterations=rec["iterations"], init="pdfs", init_pdfs=init)
        ref = np.load(os.path.join(GOLDEN, rec["file"]))
        m = lat != 0
        if rec["exact"]:
            assert np.array_equal(o[m], ref[m]), key
        else:
            assert np.max(np.abs(o[m] - ref[m]) / np.abs(ref[m])) < 1e-13, key


@pytest.mark.parametrize("kernel,okernel,exact", [("aa-soa", "aa", True), ("push-soa", "push-fa", True),
                                                  ("pull-soa", "pull-fa", True),
                                                  ("list-aa-pv-soa", "list-aa", False)])
@pytest.mark.parametrize("dims,seed", [((30, 26, 28), 3), ((9, 13, 140), 8)])
def test_fields_match_reference_periodic_packing(oracle, reference, kernel, okernel, exact, dims, seed):
    # sphere packings periodic on every axis, obstacles on every face: links
    # that wrap through x, y and z into obstacle cells (the GPU parity test
    # runs the same lattices against the oracle)
    import lbmb200
    lat, _ = lbmb200.spheres(dims, seed, 0.45, 2.0, 4.0)
    per = (1, 1, 1)
    init = random_pdfs(lat.mask.size, seed=seed)
    kw = dict(omega=1.3, xforce=2e-4, iterations=20, init="pdfs", init_pdfs=init)
    r = reference.run(kernel, dims, per, lat.mask, **kw)
    o = oracle.run(okernel, dims, per, lat.mask, lam=1.0 / 12.0, **kw)
    m = lat.mask != 0
    if exact:
        assert np.array_equal(r[m], o[m])
    else:
        assert np.max(np.abs(r[m] - o[m]) / np.abs(r[m])) < 1e-13
