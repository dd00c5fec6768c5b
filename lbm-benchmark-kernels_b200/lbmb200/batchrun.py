"""Command-line run of the batched form: N seeded porous domains (sphere
packings, edge U{lo..hi}, porosity U[0.3, 0.6], radii U[3, 8], omega
U[0.8, 1.6]) advanced together for a number of steps; prints the aggregate
MFLUP/s measured with CUDA events (lbm_batch_time_steps).

    python -m lbmb200.batchrun --domains 32 --steps 20 --storage fp32 [--tune]

(run with lbm-benchmark-kernels_b200 on the Python path). The batched
counterpart of the C driver bin/lbmbenchk-b200, which runs one domain.
"""
import argparse
import json

import numpy as np

from . import Batch, spheres


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--domains", type=int, default=32)
    p.add_argument("--edge-min", type=int, default=32)
    p.add_argument("--edge-max", type=int, default=128)
    p.add_argument("--storage", choices=["fp32", "fp16"], default="fp32")
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--seed", type=int, default=7000)
    p.add_argument("--tune", action="store_true", help="run the launch autotuner first")
    p.add_argument("--budget-gb", type=float, default=150.0)
    a = p.parse_args(argv)

    rng = np.random.default_rng(a.seed)
    b = Batch(a.storage, budget_gb=a.budget_gb, max_domains=a.domains)
    nodes = 0
    try:
        for i in range(a.domains):
            edge = int(rng.integers(a.edge_min, a.edge_max + 1))
            por, omega = float(rng.uniform(0.3, 0.6)), float(rng.uniform(0.8, 1.6))
            lat, _ = spheres((edge,) * 3, a.seed * 1000 + i, por, 3.0, 8.0)
            if b.add(lat, omega=omega, lam=3.0 / 16.0, xforce=1e-5) < 0:
                raise SystemExit("domain %d does not fit the budget" % i)
            nodes += lat.n_fluid
        if a.tune:
            b.tune(trial_steps=6)
        b.time_steps(2)  # warm up
        ms = b.time_steps(a.steps)
        b.sync()
        print(json.dumps({"domains": a.domains, "fluid_nodes": nodes, "storage": a.storage, "steps": a.steps,
                          "ms": round(ms, 4), "mflups": round(nodes * a.steps / (ms / 1e3) / 1e6, 1),
                          "launch": b.launch()}))
    finally:
        b.close()


if __name__ == "__main__":
    main()
