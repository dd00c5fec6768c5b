"""The multi-rank plumbing on CPU: two gloo ranks (world size 2) exchange
the timing max / sum and split a request stream without overlap."""
import os
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = textwrap.dedent("""
    import json, os, sys
    sys.path.insert(0, os.path.join(%(root)r, "lbm-benchmark-kernels_b200"))
    from lbmb200.ranks import Ranks
    from lbmb200.serving import make_requests
    r = Ranks(backend="gloo", timeout_s=30)
    r.barrier()
    mx = r.max(10.0 + r.rank)
    sm = r.sum(1 + r.rank)
    mine = [q.id for q in r.share(make_requests(7, rate=2.0, seed=5))]
    with open(os.path.join(%(out)r, "rank%%d.json" %% r.rank), "w") as f:
        json.dump({"rank": r.rank, "max": mx, "sum": sm, "mine": mine}, f)
    r.close()
""")


def test_two_gloo_ranks(tmp_path):
    script = tmp_path / "ranks_probe.py"
    script.write_text(SCRIPT % {"root": ROOT, "out": str(tmp_path)})
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", "--master-port=29517", str(script)]
    env = dict(os.environ, OMP_NUM_THREADS="1")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=180, env=env)
    assert out.returncode == 0, out.stderr[-2000:]
    import json
    recs = [json.loads((tmp_path / ("rank%d.json" % r)).read_text()) for r in range(2)]
    assert len(recs) == 2
    for rec in recs:
        assert rec["max"] == 11.0 and rec["sum"] == 3.0
    ids = sorted(recs[0]["mine"] + recs[1]["mine"])
    assert ids == list(range(7)) and not set(recs[0]["mine"]) & set(recs[1]["mine"])
