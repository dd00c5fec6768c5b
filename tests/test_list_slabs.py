"""List-AA slabs on the CPU: the host-built slab layouts (owned nodes, ghost
nodes, halo slot lists of lbm_aa_list_slab_layout) driven by the oracle's
list AA half steps, with the two-phase halo exchange done in numpy. After
every even/odd pair the slabs' owned nodes must hold the undivided lattice's
oracle run bit for bit. Ghost slots start as NaN, so a ghost value that the
exchange failed to deliver poisons the result instead of passing unnoticed.

Also: the oracle's half-step form against its own full run, the layout's
invariants (each remote slot listed once, the two sides of a face agree), and
the refusal of a link that leaves through a face without a halo."""
import numpy as np
import pytest

import lbmb200
from lbmb200 import slabs as sl
from slab_emu import LAM, NONE, OMEGA, XF, init_field as _init_field, run_slabs


CASES = [
    # (geometry, dims, periodic, parts, kernel args)
    ("channel", (12, 7, 6), (1, 1, 0), 3, ()),
    ("fluid", (6, 5, 4), (1, 1, 1), 2, ("-pad", "no")),        # two slabs on a ring: both faces to one peer
    ("box", (10, 6, 5), (0, 0, 0), 3, ("-pad", "no")),          # closed x ends, no ring
    ("fluid", (9, 6, 5), (0, 1, 0), 3, ("-pad", "no")),         # non-periodic x, periodic y: the wrap ring
    ("fluid", (9, 5, 6), (0, 0, 1), 2, ("-blk", "2")),          # periodic z only, blocked numbering
    ("blocks-2", (8, 8, 8), (1, 0, 1), 4, ("-pad", "no")),
    ("fluid", (5, 4, 4), (1, 1, 1), 4, ("-pad", "no")),         # slabs of one and two planes
    ("fluid", (3, 4, 5), (1, 0, 0), 3, ("-pad", "no")),         # one plane per slab, periodic x only
    ("channel", (10, 7, 6), (1, 1, 0), 3, ("-precision", "fp32")),  # reduced-storage layout: whole 1024-node tiles
]


@pytest.mark.parametrize("geo,dims,per,parts,kargs", CASES)
def test_list_slabs_match_undivided_run(oracle, geo, dims, per, parts, kargs):
    lat = lbmb200.geometry(geo, dims, per)
    init = _init_field(lat, 7)
    pairs = 3
    want = oracle.run("list-aa", lat.dims, lat.periodic, lat.mask, omega=OMEGA, lam=LAM, xforce=XF,
                      iterations=2 * pairs, init="pdfs", init_pdfs=init)
    got, _ = run_slabs(oracle, lat, parts, pairs, init, kargs)
    fl = lat.mask != 0
    assert np.all(np.isfinite(got[fl]))
    assert np.array_equal(got[fl], want[fl])


def test_list_slabs_sphere_packing(oracle):
    lat, _ = lbmb200.spheres((14, 12, 12), 99, 0.5, 2.0, 3.5, 2000)
    init = _init_field(lat, 3)
    want = oracle.run("list-aa", lat.dims, lat.periodic, lat.mask, omega=OMEGA, lam=LAM, xforce=XF,
                      iterations=4, init="pdfs", init_pdfs=init)
    got, slabs = run_slabs(oracle, lat, 3, 2, init, ("-pad", "no"))
    fl = lat.mask != 0
    assert np.array_equal(got[fl], want[fl])
    assert sum(s.lay["n_owned"] for s in slabs) == lat.n_fluid


def test_oracle_half_steps_equal_full_run(oracle):
    """The pinned oracle run against the half-step form on the undivided
    lattice's own layout."""
    lat = lbmb200.geometry("channel", (8, 6, 7), (1, 1, 0))
    init = _init_field(lat, 11)
    grid, adj, nf, nc = oracle.list_layout(0, lat.dims, lat.periodic, lat.mask)
    f = np.zeros(19 * nc)
    cells = np.nonzero(grid != NONE)[0]
    nodes = grid[cells].astype(np.int64)
    for d in range(19):
        f[d * nc + nodes] = init[cells, d]
    for _ in range(3):
        oracle.list_aa_half(0, nf, nc, adj, f, OMEGA, LAM, XF)
        oracle.list_aa_half(1, nf, nc, adj, f, OMEGA, LAM, XF)
    want = oracle.run("list-aa", lat.dims, lat.periodic, lat.mask, omega=OMEGA, lam=LAM, xforce=XF,
                      iterations=6, init="pdfs", init_pdfs=init)
    got = np.zeros_like(init)
    for d in range(19):
        got[cells, d] = f[d * nc + nodes]
    assert np.array_equal(got[cells], want[cells])


def test_layout_invariants():
    lat = lbmb200.geometry("fluid", (7, 5, 4), (1, 1, 1))
    parts = 3
    lays = []
    for r, (x0, x1) in enumerate(sl.partition(7, parts)):
        lo, hi = sl.halo_flags(r, parts, True)
        lays.append(sl.list_slab_layout(lat, x0, x1, lo, hi, ("-pad", "no")))
    for r, lay in enumerate(lays):
        n_own, n_ghost, nc = lay["n_owned"], lay["n_ghost"], lay["n_cells"]
        assert n_own == (sl.partition(7, parts)[r][1] - sl.partition(7, parts)[r][0]) * 5 * 4
        assert nc >= n_own + n_ghost
        adj = lay["adj"].reshape(-1, 18)
        node = adj % nc
        # every ghost slot an owned link reaches appears in exactly one ghost list
        reached = np.sort(adj[node >= n_own])
        listed = np.sort(np.concatenate([g for g in lay["ghost"] if g is not None]))
        assert np.array_equal(reached, listed)
        # own lists name owned slots, each once per face
        for s in (0, 1):
            own = lay["own"][s]
            assert np.all(own % nc < n_own)
            assert np.unique(own).size == own.size
        # a fully periodic box of fluid: 5 links per face cell and face
        for s in (0, 1):
            assert lay["ghost"][s].size == lay["own"][s].size == 5 * 5 * 4


def test_closed_face_refuses_crossing_link():
    lat = lbmb200.geometry("fluid", (6, 4, 4), (1, 1, 1))
    with pytest.raises(RuntimeError, match="without a halo"):
        sl.list_slab_layout(lat, 0, 3, False, True)


def test_reduced_storage_layout_pads_to_tiles():
    lat = lbmb200.geometry("fluid", (9, 6, 5), (1, 1, 1))
    for r, (x0, x1) in enumerate(sl.partition(9, 3)):
        lo, hi = sl.halo_flags(r, 3, True)
        lay = sl.list_slab_layout(lat, x0, x1, lo, hi, ("-precision", "fp16"))
        assert lay["n_cells"] % 1024 == 0 and lay["n_cells"] >= lay["n_owned"] + lay["n_ghost"]


def test_transport_word_counts():
    """Messages of 2-, 4- and 8-byte PDF elements travel in whole 8-byte
    words; both sides of a face compute the same word count."""
    class S:
        def __init__(self, eb, n):
            self.elem_bytes, self.n = eb, n

        def message(self, side, phase, send):
            return self.n

    assert sl.message(S(8, 5), 0, 0, True) == 5
    assert sl.message(S(4, 5), 0, 0, True) == 3
    assert sl.message(S(2, 5), 0, 0, True) == 2
    assert sl.message(S(2, 8), 0, 0, True) == 2
    assert sl.message(S(2, -1), 0, 0, True) == -1


@pytest.mark.parametrize("geo,dims,per,parts,kargs", [
    ("channel", (24, 16, 16), (1, 1, 0), 3, ()),
    ("fluid", (20, 12, 12), (1, 1, 1), 2, ("-pad", "no")),
    ("box", (24, 12, 12), (0, 0, 0), 3, ("-pad", "no")),
    ("fluid", (9, 5, 6), (0, 0, 1), 2, ("-blk", "2")),   # blocked numbering: no inner range
])
def test_overlapped_odd_step_matches_undivided_run(oracle, geo, dims, per, parts, kargs):
    """The odd step split into the inner tiles (run while the phase-0 messages
    travel) and the rest (after they arrive) leaves the same bits."""
    lat = lbmb200.geometry(geo, dims, per)
    init = _init_field(lat, 13)
    want = oracle.run("list-aa", lat.dims, lat.periodic, lat.mask, omega=OMEGA, lam=LAM, xforce=XF,
                      iterations=6, init="pdfs", init_pdfs=init)
    got, slabs = run_slabs(oracle, lat, parts, 3, init, kargs, overlap=True)
    fl = lat.mask != 0
    assert np.array_equal(got[fl], want[fl])
    if "-blk" not in kargs:
        assert any(s.lay["inner"][1] > s.lay["inner"][0] for s in slabs)


def test_inner_tiles_link_to_no_ghost():
    lat, _ = lbmb200.spheres((24, 12, 12), 5, 0.5, 2.0, 3.0, 2000)
    for r, (x0, x1) in enumerate(sl.partition(24, 2)):
        lo, hi = sl.halo_flags(r, 2, True)
        lay = sl.list_slab_layout(lat, x0, x1, lo, hi, ("-pad", "no"))
        t0, t1 = lay["inner"]
        assert 0 < t0 < t1
        adj = lay["adj"].reshape(-1, 18)
        inner = adj[t0 * 256: min(t1 * 256, lay["n_owned"])]
        assert np.all(inner % lay["n_cells"] < lay["n_owned"])
        # no slot of an inner node travels in a message
        for own in lay["own"]:
            if own is not None:
                node = own % lay["n_cells"]
                assert not np.any((node >= t0 * 256) & (node < t1 * 256))
