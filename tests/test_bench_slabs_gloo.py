"""bench.py's one-lattice slab section (section_slabs) as two gloo ranks on
CPU: the section's own partition, transport, timing and reduction code runs
unchanged; the slabs are oracle-stepped stand-ins (tests/slab_emu.py) and
the clock is the host's. Checks that the "slabs" key carries both modes with
their MFLUP/s and exchange share over the whole lattice."""
import json
import os
import subprocess
import sys
import textwrap

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = textwrap.dedent("""
    import argparse, json, os, sys, time
    sys.path[:0] = [%(root)r, os.path.join(%(root)r, "lbm-benchmark-kernels_b200"), os.path.join(%(root)r, "tests"),
                    os.path.join(%(root)r, "oracle")]
    import torch
    import torch.distributed as dist
    import bench
    import lbmb200
    from lbmb200 import slabs as sl
    from lbmb200.ranks import Ranks
    from oracle import Oracle
    from slab_emu import EmuSlab, SteppedEmuSlab, init_field

    class EmuBackend:
        stream = None
        def __init__(self, lat):
            self.lat, self.orc = lat, Oracle()
        def slab(self, lat, x0, x1, lo, hi, kargs):
            emu = EmuSlab(lat, x0, x1, lo, hi, ("-pad", "no"))
            emu.set_field(init_field(lat, 5))
            s = SteppedEmuSlab(emu, self.orc)
            s.local = argparse.Namespace(n_fluid=emu.lay["n_owned"])
            return s
        def transport(self, slab, rank, world, ring):
            return sl.DistTransport(slab, rank, world, ring, dist, lambda n: torch.zeros(n, dtype=torch.float64))
        def mark(self):
            return time.perf_counter()
        def sync(self):
            pass
        @staticmethod
        def ms(a, b):
            return (b - a) * 1e3
        def close(self, slab):
            pass

    r = Ranks(backend="gloo", timeout_s=60)
    lat = lbmb200.geometry("fluid", (20, 10, 8), (1, 1, 1))
    args = argparse.Namespace(edge=20, seed=1, porosity=1.0)
    out = bench.section_slabs(args, r, backend=EmuBackend(lat), lat=lat, pairs=2, warmup=1)
    if r.rank == 0:
        with open(os.path.join(%(out)r, "slabs.json"), "w") as f:
            json.dump(out, f)
    r.close()
""")


def test_bench_slab_section_over_gloo(tmp_path):
    script = tmp_path / "bench_slabs.py"
    script.write_text(SCRIPT % {"root": ROOT, "out": str(tmp_path)})
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", "--master-port=29611", str(script)]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=240, env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stderr[-3000:]
    rec = json.loads((tmp_path / "slabs.json").read_text())
    assert rec["scaling"] == "strong" and rec["fluid_nodes"] == 20 * 10 * 8
    for mode in ("serial", "overlapped"):
        m = rec[mode]
        assert m["ms"] > 0 and m["mflups"] > 0 and abs(m["mflups_per_rank"] * 2 - m["mflups"]) < 0.2
        assert 0.0 <= m["exchange_share"] <= 1.0
