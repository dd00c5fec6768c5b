"""The slab transport over torch.distributed on CPU ranks (gloo): each rank
holds a stand-in slab whose pack writes a recognisable message; after an
exchange every halo face has received exactly its neighbour's message for
that face and phase -- two ranks on a periodic ring (both messages between
the same pair), three ranks, and closed x ends."""
import json
import os
import subprocess
import sys
import textwrap

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = textwrap.dedent("""
    import json, os, sys
    sys.path.insert(0, os.path.join(%(root)r, "lbm-benchmark-kernels_b200"))
    import torch
    import torch.distributed as dist
    from lbmb200.ranks import Ranks
    from lbmb200 import slabs as sl

    class FakeSlab:
        count = 6
        def __init__(self, rank):
            self.rank, self.got = rank, {}
        def pack(self, side, phase, buf, stream=None):
            buf.copy_(torch.tensor([1000 * self.rank + 100 * side + 10 * phase + k for k in range(6)],
                                   dtype=torch.float64))
        def unpack(self, side, phase, buf, stream=None):
            self.got["%%d/%%d" %% (side, phase)] = [float(v) for v in buf]

    r = Ranks(backend="gloo", timeout_s=30)
    periodic = int(sys.argv[1])
    slab = FakeSlab(r.rank)
    tr = sl.DistTransport(slab, r.rank, r.world, sl.is_ring((periodic, 0, 0)), dist,
                          lambda n: torch.zeros(n, dtype=torch.float64))
    tr.exchange(0)
    tr.exchange(1)
    with open(os.path.join(%(out)r, "slab%%d.json" %% r.rank), "w") as f:
        json.dump({"rank": r.rank, "left": tr.left, "right": tr.right, "got": slab.got}, f)
    r.close()
""")


@pytest.mark.parametrize("world,periodic", [(2, 1), (3, 1), (3, 0)])
def test_dist_transport_pairs_faces(tmp_path, world, periodic):
    script = tmp_path / "slab_probe.py"
    script.write_text(SCRIPT % {"root": ROOT, "out": str(tmp_path)})
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % world,
           "--master-addr=127.0.0.1", "--master-port=%d" % (29531 + world + 10 * periodic), str(script),
           str(periodic)]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=180, env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stderr[-2000:]
    recs = {r: json.loads((tmp_path / ("slab%d.json" % r)).read_text()) for r in range(world)}
    for r, rec in recs.items():
        exp_left = (r - 1) % world if (r > 0 or periodic) else None
        exp_right = (r + 1) % world if (r < world - 1 or periodic) else None
        assert (rec["left"], rec["right"]) == (exp_left, exp_right)
        for phase in (0, 1):
            # the left face receives what the left neighbour packed for its right face, and vice versa
            if exp_left is not None:
                want = [1000 * exp_left + 100 * 1 + 10 * phase + k for k in range(6)]
                assert rec["got"]["0/%d" % phase] == want
            else:
                assert "0/%d" % phase not in rec["got"]
            if exp_right is not None:
                want = [1000 * exp_right + 100 * 0 + 10 * phase + k for k in range(6)]
                assert rec["got"]["1/%d" % phase] == want
            else:
                assert "1/%d" % phase not in rec["got"]


LIST_SCRIPT = textwrap.dedent("""
    import json, os, sys
    sys.path[:0] = [os.path.join(%(root)r, "lbm-benchmark-kernels_b200"), os.path.join(%(root)r, "tests"),
                    os.path.join(%(root)r, "oracle")]
    import numpy as np
    import torch
    import torch.distributed as dist
    import lbmb200
    from lbmb200.ranks import Ranks
    from lbmb200 import slabs as sl
    from oracle import Oracle
    from slab_emu import EmuSlab, SteppedEmuSlab, init_field

    r = Ranks(backend="gloo", timeout_s=60)
    geo, dims, per, pairs = sys.argv[1], tuple(int(v) for v in sys.argv[2].split("x")), \\
        tuple(int(c) for c in sys.argv[3]), int(sys.argv[4])
    lat = lbmb200.geometry(geo, dims, per)
    ring = sl.is_ring(lat.periodic)
    x0, x1 = sl.partition(dims[0], r.world)[r.rank]
    lo, hi = sl.halo_flags(r.rank, r.world, ring)
    slab = EmuSlab(lat, x0, x1, lo, hi, ("-pad", "no"))
    slab.set_field(init_field(lat, 5))
    tr = sl.DistTransport(slab, r.rank, r.world, ring, dist, lambda n: torch.zeros(n, dtype=torch.float64))
    overlap = len(sys.argv) > 5 and sys.argv[5] == "1"
    # the library's own step sequence (serial or overlapped) drives the slab
    sl.step_pairs([SteppedEmuSlab(slab, Oracle())], tr, None, pairs, None, overlap=overlap)
    out = np.zeros((lat.mask.size, 19))
    slab.get_field(out)
    np.save(os.path.join(%(out)r, "part%%d.npy" %% r.rank), out[slab.gcells])
    np.save(os.path.join(%(out)r, "cells%%d.npy" %% r.rank), slab.gcells)
    r.close()
""")


@pytest.mark.parametrize("world,geo,dims,per,overlap", [(2, "fluid", "6x5x4", "111", 0),
                                                         (3, "channel", "9x6x5", "110", 0),
                                                         (2, "box", "8x5x5", "000", 0),
                                                         (2, "fluid", "20x12x12", "111", 1),
                                                         (3, "channel", "24x16x16", "110", 1)])
def test_list_slabs_over_gloo_match_undivided_run(tmp_path, oracle, world, geo, dims, per, overlap):
    """List-AA slabs as gloo ranks: the layout from the library, the steps
    from the oracle, the step sequence from lbmb200.slabs.step_pairs and the
    halo messages through DistTransport's asynchronous start/finish (with
    `overlap`, the phase-0 messages are posted, the inner tiles step, then
    the messages are awaited and the other tiles step); the gathered field
    equals the undivided oracle run bit for bit."""
    sys.path[:0] = [os.path.join(ROOT, "tests")]
    import numpy as np
    import lbmb200
    from slab_emu import LAM, OMEGA, XF, init_field
    script = tmp_path / "list_slab_probe.py"
    script.write_text(LIST_SCRIPT % {"root": ROOT, "out": str(tmp_path)})
    pairs = 3
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % world,
           "--master-addr=127.0.0.1", "--master-port=%d" % (29571 + world + 7 * len(geo) + 50 * overlap),
           str(script), geo, dims, per, str(pairs), str(overlap)]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=240, env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stderr[-3000:]
    d = tuple(int(v) for v in dims.split("x"))
    lat = lbmb200.geometry(geo, d, tuple(int(c) for c in per))
    init = init_field(lat, 5)
    want = oracle.run("list-aa", lat.dims, lat.periodic, lat.mask, omega=OMEGA, lam=LAM, xforce=XF,
                      iterations=2 * pairs, init="pdfs", init_pdfs=init)
    seen = 0
    for rank in range(world):
        cells = np.load(tmp_path / ("cells%d.npy" % rank))
        part = np.load(tmp_path / ("part%d.npy" % rank))
        assert np.array_equal(part, want[cells])
        seen += cells.size
    assert seen == lat.n_fluid
