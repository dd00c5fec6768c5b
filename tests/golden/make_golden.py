"""Writes the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where oracle/_ref has been built from the reference sources
(make -C oracle ref):  python tests/golden/make_golden.py
The fixtures let the oracle pin run where the reference build is absent.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.dirname(HERE))

from oracle import Reference  # noqa: E402
from lbm_cases import random_pdfs  # noqa: E402

GEOMS = ["box", "channel", "pipe", "blocks", "blocks-3", "fluid"]
PERIODIC = [(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 1), (1, 1, 1), (0, 0, 1)]
DIMS = [(16, 16, 16), (17, 9, 13), (7, 9, 8)]

FIELDS = [
    # key: (reference kernel, oracle kernel, exact, geo, dims, periodic, omega, xforce, iterations, seed)
    ("aa_channel_open", "aa-soa", "aa", True, "channel", (8, 6, 5), (0, 0, 0), 1.2, 1e-4, 10, 11),
    ("aa_box_verify", "aa-soa", "aa", True, "box", (8, 6, 5), (1, 1, 0), 1.0, 1e-5, 10, 12),
    ("listaa_blocks", "list-aa-pv-soa", "list-aa", False, "blocks-1", (8, 6, 5), (1, 0, 1), 0.8, 1e-4, 10, 13),
    ("pull_pipe", "list-pull-split-nt-1s-soa", "list-pull", False, "pipe", (8, 8, 8), (0, 0, 0), 1.6, 1e-4, 9, 14),
]


def main():
    ref = Reference("verify")
    ref.set_threads(1)
    geo = {}
    for g in GEOMS:
        for p in PERIODIC:
            for d in DIMS:
                bs = 8 if g == "blocks" else (3 if g == "blocks-3" else 0)
                if bs and bs > min(d) // 2:
                    continue
                lat, info = ref.geometry(g, d, p)
                geo["%s|%s|%s" % (g, p, d)] = {
                    "geo": g, "periodic": list(p), "dims": list(d),
                    "sha256": hashlib.sha256(lat.tobytes()).hexdigest(),
                    "nFluid": info["nFluid"], "ldPeriodic": list(info["ldPeriodic"])}
    with open(os.path.join(HERE, "geometry.json"), "w") as f:
        json.dump(geo, f, indent=1, sort_keys=True)

    fields = {}
    for key, rk, ok, exact, g, d, p, om, fx, it, seed in FIELDS:
        lat, _ = ref.geometry(g, d, p)
        init = random_pdfs(lat.size, seed=seed)
        out = ref.run(rk, d, p, lat, omega=om, xforce=fx, iterations=it, init="pdfs", init_pdfs=init)
        fn = "field_%s.npy" % key
        np.save(os.path.join(HERE, fn), out)
        fields[key] = {"kernel": rk, "okernel": ok, "exact": exact, "geo": g, "dims": list(d),
                       "periodic": list(p), "omega": om, "xforce": fx, "iterations": it,
                       "seed": seed, "file": fn}
    with open(os.path.join(HERE, "fields.json"), "w") as f:
        json.dump(fields, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
