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
