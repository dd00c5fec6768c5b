"""Writes tests/golden/packing256.json and packing256.npz from the reference
itself: its list layouts and its 500-step FP64 fields on the seeded 256^3
sphere packing (the indirect-addressing throughput workload).

Run in a checkout where oracle/_ref has been built from the reference sources
(make -C oracle ref) and liblbmb200.so is built (the packing generator is its
host-side C code; no GPU is used):

    python tests/golden/make_packing_golden.py [threads]

The reference's VERIFICATION list kernels need tens of minutes for 3 x 500
steps at this size on a few host cores, which is why the GPU test reads these
fixtures instead of running the reference at full size. What is kept:

* sha256 of the packing mask, and of the reference's Grid and AdjList for the
  push (list-aa-pv-soa) and pull (list-pull-split-nt) layouts, with nFluid and
  nCells: the layout pins are bit for bit;
* per reference kernel (list-aa-pv-soa, list-pull-split-nt-1s-soa,
  list-pull-split-nt-2s-soa; Lambda 1/12, fixed by the reference): the
  logical PDFs of 1024 seeded fluid cells, and the sums of every direction's
  PDFs over each x, y and z plane (3 x 256 x 19 values) -- a whole-field
  fingerprint that a wrong node anywhere moves.

The run: omega 1, F_x = 1e-5, 500 steps, equilibrium start f_i = w_i.
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "oracle"), os.path.join(ROOT, "lbm-benchmark-kernels_b200")):
    sys.path.insert(0, p)

import lbmb200  # noqa: E402
from oracle import Reference  # noqa: E402

EDGE, SEED, POROSITY, RMIN, RMAX = 256, 20251203, 0.40, 6.0, 12.0
STEPS, OMEGA, XFORCE = 500, 1.0, 1e-5
N_SAMPLE, SAMPLE_SEED = 1024, 7
KERNELS = ["list-aa-pv-soa", "list-pull-split-nt-1s-soa", "list-pull-split-nt-2s-soa"]
LAYOUTS = {"push": "list-aa-pv-soa", "pull": "list-pull-split-nt-1s-soa"}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def plane_sums(field, dims):
    """field: (nCells, 19), cells x fastest -> (3, edge, 19) sums over the
    x, y and z planes (obstacle cells hold zeros)."""
    nx, ny, nz = dims
    f = field.reshape(nz, ny, nx, 19)
    return np.stack([f.sum(axis=(0, 1)), f.sum(axis=(0, 2)), f.sum(axis=(1, 2))])


def sample_cells(mask):
    fluid = np.flatnonzero(mask != 0)
    rng = np.random.default_rng(SAMPLE_SEED)
    return np.sort(rng.choice(fluid, N_SAMPLE, replace=False)).astype(np.int64)


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    lat, st = lbmb200.spheres((EDGE,) * 3, SEED, POROSITY, RMIN, RMAX)
    ref = Reference("verify")
    ref.set_threads(threads)
    meta = {"edge": EDGE, "seed": SEED, "porosity_target": POROSITY, "radius": [RMIN, RMAX],
            "porosity": st["porosity"], "n_fluid": lat.n_fluid, "mask_sha256": sha(lat.mask),
            "steps": STEPS, "omega": OMEGA, "xforce": XFORCE, "lambda": "1/12 (fixed by the reference)",
            "init": "equilibrium f_i = w_i", "n_sample": N_SAMPLE, "sample_seed": SAMPLE_SEED,
            "layouts": {}, "kernels": {}}
    for key, rk in LAYOUTS.items():
        grid, adj, nf, nc = ref.list_layout(rk, lat.dims, lat.periodic, lat.mask)
        meta["layouts"][key] = {"kernel": rk, "n_fluid": nf, "n_cells": nc, "grid_sha256": sha(grid),
                                "adj_sha256": sha(adj)}
    cells = sample_cells(lat.mask)
    arrays = {"sample_cells": cells}
    init = np.ascontiguousarray(np.broadcast_to(lbmb200.W, (lat.mask.size, 19)))
    for rk in KERNELS:
        t0 = time.time()
        out = ref.run(rk, lat.dims, lat.periodic, lat.mask, omega=OMEGA, xforce=XFORCE, iterations=STEPS,
                      init="pdfs", init_pdfs=init)
        out[lat.mask == 0] = 0.0
        key = rk.replace("-", "_")
        arrays["sample_" + key] = out[cells]
        arrays["planes_" + key] = plane_sums(out, lat.dims)
        meta["kernels"][rk] = {"seconds": round(time.time() - t0, 1), "threads": threads}
        print(rk, meta["kernels"][rk], flush=True)
        del out
    np.savez_compressed(os.path.join(HERE, "packing256.npz"), **arrays)
    with open(os.path.join(HERE, "packing256.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
