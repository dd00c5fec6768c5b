"""Command-line run of one AA-pattern lattice split into x-slabs, one slab
per GPU, halo messages through torch.distributed (NCCL):

    python -m torch.distributed.run --nproc-per-node 4 --master-addr 127.0.0.1 \\
        -m lbmb200.slabrun --dims 1024x256x256 --geometry fluid --periodic xyz --pairs 50
    ... -m lbmb200.slabrun --layout list --dims 512x256x256 \\
        --geometry spheres:20251203:0.4:6:12 --pairs 50

(run with lbm-benchmark-kernels_b200 on the Python path). Every rank builds the
same lattice, takes its slab -- full array (cuda-aa-soa kernels) or fluid-node
list (cuda-list-aa-pv-soa kernels) -- and runs `pairs` even/odd step pairs;
rank 0 prints the aggregate MFLUP/s (device-timed per rank with CUDA events,
max over ranks). List slabs (any --precision) also report the FP64
conservation sums of the whole lattice (per-slab sums all-reduced) and the
permeability they give. --overlap sends each phase's halo messages while
the cells they do not concern take their step (Slab.odd_part/even_part).
With one process, the lattice runs as one slab without halos.
"""
import argparse
import json

import numpy as np


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    p.add_argument("--dims", default="256x256x256")
    p.add_argument("--geometry", default="fluid")
    p.add_argument("--periodic", default="xyz", help="periodic axes, e.g. xyz or x")
    p.add_argument("--pairs", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--omega", type=float, default=1.0)
    p.add_argument("--lambda", dest="lam", default="3/16")
    p.add_argument("--layout", default="full", choices=("full", "list"))
    p.add_argument("--precision", default="fp64", choices=("fp64", "fp32", "fp16"),
                   help="PDF storage of list slabs")
    p.add_argument("--overlap", action="store_true",
                   help="send the phase-0 halo messages while the inner cells take their odd step")
    a = p.parse_args(argv)

    import torch
    import torch.distributed as dist

    import lbmb200
    from lbmb200 import slabs as sl
    from lbmb200.ranks import Ranks

    ranks = Ranks()
    try:
        dims = tuple(int(v) for v in a.dims.split("x"))
        per = tuple(int(c in a.periodic) for c in "xyz")
        lat = lbmb200.geometry(a.geometry, dims, per)
        x0, x1 = sl.partition(dims[0], ranks.world)[ranks.rank]
        ring = sl.is_ring(lat.periodic)
        lo, hi = sl.halo_flags(ranks.rank, ranks.world, ring)
        lbmb200.lib().lbm_b200_set_device(ranks.local)
        torch.cuda.set_device(ranks.local)
        if a.precision != "fp64" and a.layout != "list":
            raise SystemExit("--precision fp32/fp16 needs --layout list")
        kargs = ["-lambda", a.lam] + (["-precision", a.precision] if a.layout == "list" else [])
        slab = sl.Slab(lat, x0, x1, lo, hi, kernel_args=kargs, layout=a.layout)
        if a.layout == "list":
            slab.inst.set_field(np.broadcast_to(lbmb200.W, (slab.local.mask.size, 19)))
        # an explicit stream, current for torch.distributed too: kernels,
        # packs, the library's sends/receives and unpacks run in one order
        work = torch.cuda.Stream()
        torch.cuda.set_stream(work)
        stream = work.cuda_stream
        tr = sl.DistTransport(slab, ranks.rank, ranks.world, ring, dist,
                              lambda n: torch.empty(n, dtype=torch.float64, device="cuda"), stream=stream)
        cd = lbmb200.case(omega=a.omega, xforce=1e-5)
        sl.step_pairs([slab], tr, cd, a.warmup, stream, overlap=a.overlap)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ranks.barrier()
        e0.record()
        sl.step_pairs([slab], tr, cd, a.pairs, stream, overlap=a.overlap)
        e1.record()
        torch.cuda.synchronize()
        ms = ranks.max(e0.elapsed_time(e1))
        nodes = ranks.sum(slab.local.n_fluid)
        rec = {"dims": dims, "geometry": a.geometry, "layout": a.layout, "precision": a.precision,
               "overlap": a.overlap, "ranks": ranks.world,
               "fluid_nodes": nodes, "pairs": a.pairs, "ms": round(ms, 3),
               "mflups": round(nodes * 2 * a.pairs / (ms / 1e3) / 1e6, 1)}
        if a.layout == "list":
            from lbmb200.porous import permeability
            rho, jx, jy, jz = ranks.sum_vec(slab.inst.moments())
            rec.update({"sum_rho": rho, "sum_jx": jx, "sum_jy": jy, "sum_jz": jz,
                        "permeability": permeability(jx, nodes, dims[0] * dims[1] * dims[2], a.omega, cd.XForce)})
        if ranks.rank == 0:
            print(json.dumps(rec))
        slab.close()
    finally:
        ranks.close()


if __name__ == "__main__":
    main()
