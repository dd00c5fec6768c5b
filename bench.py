#!/usr/bin/env python
"""Throughput benchmark of the B200 D3Q19 TRT kernels.

Workload (N=1, per rank for N>1): a 256^3 fully periodic box filled with a
seeded packing of solid spheres (radius uniform in [6, 12], porosity 0.40,
about 6.7M fluid nodes), FP64 PDFs, TRT with Lambda = 3/16, omega = 1, body
force along x. The headline kernel is the list AA kernel
("cuda-list-aa-pv-soa", the drop-in for the reference's list-aa-pv-soa). A
"step" is one time step over all fluid nodes.

  value     MFLUP/s over exactly K device-timed steps (CUDA events on the
            kernel stream), inputs resident in HBM (1.3 GB of PDFs, larger than
            the 126 MB L2), max over ranks
  e2e       the same metric through the reference-facing C ABI: one Kernel()
            call of the configuration's 500 steps with the PDF field uploaded
            from the pinned host mirror before and downloaded after
  roofline  the dominant kernel (the odd, adjacency-driven step): algorithmic
            bytes per launch / mean launch time, against the measured HBM copy
            bandwidth in MEASURED_PEAKS.json
  cpu_baseline  the reference's own list-aa-pv-soa (compiled from its sources
            into oracle/_ref) on this host's cores, a bounded sample of the
            same domain

`--impl reference` times the reference's CPU kernel alone on the same
workload and prints its own line. For N>1 every rank runs its own domain (seed
+ rank): no data moves between ranks, scaling is weak. Beside that headline,
N>1 also reports "slabs": the one 256^3 lattice split into x-slabs over the
ranks with halo messages over NCCL (strong scaling), serial and overlapped;
the single-GPU sections (secondary kernel lines, batched, serving,
precision, CPU baseline) run at N=1 only.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "lbm-benchmark-kernels_b200")
sys.path.insert(0, PKG)

L2_BYTES = 126 * 1024 * 1024
B_PER_FLUP = {"even": 2 * 19 * 8, "aa": 2 * 19 * 8}


def adjacency_bytes_per_node(lbmb200, inst, n_fluid):
    """Adjacency bytes per node that one adjacency-driven launch reads (run
    records for the list AA odd and list push steps, whole tiles for pull)."""
    L = lbmb200.lib()
    L.lbm_b200_adjacency_bytes.restype = ctypes.c_longlong
    return L.lbm_b200_adjacency_bytes(inst.kdp) / max(1, n_fluid)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=500)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--edge", type=int, default=256)
    p.add_argument("--porosity", type=float, default=0.40)
    p.add_argument("--seed", type=int, default=20251203)
    p.add_argument("--no-extra", action="store_true", help="skip the secondary kernel lines")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    p.add_argument("--batched", type=int, default=512, help="domains of the batched form (0 = skip)")
    p.add_argument("--serving", type=int, default=100, help="requests of the serving form (0 = skip)")
    p.add_argument("--precision-steps", type=int, default=20000, help="steps of the precision study (0 = skip)")
    p.add_argument("--no-slabs", action="store_true",
                   help="N>1: skip the one-lattice x-slab split (strong scaling) beside the replicas")
    return p.parse_args()


# ---------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------

def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(kernel_key):
    """DRAM bytes per launch from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        t = json.load(f)
    rec = t.get(kernel_key)
    return None if rec is None else rec.get("bytes_per_launch_full")


def sphere_lattice(lbmb200, edge, porosity, seed):
    L = lbmb200.lib()
    L.lbm_geo_spheres.argtypes = [ctypes.c_int * 3, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, ctypes.POINTER(lbmb200.LatticeDesc),
                                  ctypes.POINTER(ctypes.c_double)]
    ld = lbmb200.LatticeDesc()
    st = (ctypes.c_double * 4)()
    dims = (edge, edge, edge)
    rc = L.lbm_geo_spheres((ctypes.c_int * 3)(*dims), seed, porosity, 6.0, 12.0, 20000, ctypes.byref(ld), st)
    if rc:
        raise RuntimeError("sphere packing failed")
    import numpy as np
    n = edge ** 3
    mask = np.ctypeslib.as_array(ld.Lattice, shape=(n,)).copy()
    ctypes.CDLL(None).free(ctypes.cast(ld.Lattice, ctypes.c_void_p))
    lat = lbmb200.Lattice(mask, dims, (1, 1, 1), "spheres")
    stats = {"porosity": round(st[0], 6), "spheres_rsa": int(st[1]), "spheres_overlap": int(st[2]),
             "jam_porosity": round(st[3], 4)}
    return lat, stats


def equilibrium_field(lbmb200, lat):
    import numpy as np
    return np.broadcast_to(lbmb200.W, (lat.mask.size, 19))


def time_kernel(lbmb200, kname, lat, steps, warmup, kargs, dist, odd_key):
    """Device-timed steps of one kernel instance; returns timing dict."""
    import numpy as np
    inst = lbmb200.kernel(kname).init(lat, kernel_args=kargs)
    try:
        inst.set_field(np.ascontiguousarray(equilibrium_field(lbmb200, lat)))
        cd = lbmb200.case(omega=1.0, xforce=1e-5, iterations=steps)
        L = lbmb200.lib()
        tot = ctypes.c_double(0.0)
        if warmup > 0:
            rc = L.lbm_b200_time_steps(inst.kdp, ctypes.byref(cd), warmup, ctypes.byref(tot), None)
            if rc:
                raise RuntimeError(L.lbm_b200_last_error().decode())
        pairs = (steps + 1) // 2
        cap = inst.launches_for(steps)
        per = (ctypes.c_double * cap)()
        dist.barrier()
        rc = L.lbm_b200_time_steps(inst.kdp, ctypes.byref(cd), steps, ctypes.byref(tot), per)
        if rc:
            raise RuntimeError(L.lbm_b200_last_error().decode())
        dist.barrier()
        n_launch = inst.last_launches
        per = list(per)[:n_launch]
        res = {"ms": tot.value, "launches": n_launch,
               "steps_run": steps if ("pull" in kname or "push" in kname) else 2 * pairs,
               "per_launch_ms": per, "inst": inst,
               "launches_per_pair": inst.launches_for(2)}
        return res
    except Exception:
        inst.deinit()
        raise


class _StdoutToStderr:
    """Sends C-level stdout to stderr (the reference prints its progress there),
    so that stdout carries only the JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *exc):
        ctypes.CDLL(None).fflush(None)
        os.dup2(self.saved, 1)
        os.close(self.saved)


_HOST_CPUS = None


def host_cpus():
    """One logical CPU per physical core among the CPUs this process may run
    on (the first sibling of each core, from the sysfs topology), and a
    description of the host's processor. Taken once, before any pinning."""
    global _HOST_CPUS
    if _HOST_CPUS is None:
        _HOST_CPUS = _host_cpus()
    return _HOST_CPUS


def _host_cpus():
    allowed = sorted(os.sched_getaffinity(0))
    seen, phys = set(), []
    for c in allowed:
        try:
            with open("/sys/devices/system/cpu/cpu%d/topology/thread_siblings_list" % c) as f:
                key = f.read().strip()
        except OSError:
            key = str(c)
        if key not in seen:
            seen.add(key)
            phys.append(c)
    return phys, {"model": cpu_model(), "logical_cpus": len(allowed), "physical_cores": len(phys)}


def cpu_reference(lat, iterations, threads=None, variant=None, kernel="list-aa-pv-soa"):
    """A reference kernel (benchmark build; list-aa-pv-soa by default) on this
    host's physical cores, one OpenMP thread pinned per core (the reference's
    -t <cores> -pin <list>)."""
    with _StdoutToStderr():
        return _cpu_reference(lat, iterations, threads, variant, kernel)


def _cpu_reference(lat, iterations, threads=None, variant=None, kernel="list-aa-pv-soa"):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference, reference_available
    if variant is None:
        flags = open("/proc/cpuinfo").read()
        variant = "bench-avx512" if " avx512f" in flags and reference_available("bench-avx512") else "bench-avx2"
    if not reference_available(variant):
        return None
    ref = Reference(variant)
    phys, desc = host_cpus()
    cpus = phys[:threads] if threads else phys
    threads = ref.set_threads(len(cpus))
    # the OpenMP master is this thread: pinning it for the reference's run
    # must not confine the rest of the process (host threads of the serving
    # and batched sections start from its affinity), so it is restored after
    saved = os.sched_getaffinity(0)
    try:
        pin_failed = ref.pin(cpus[:threads])
        ref.run(kernel, lat.dims, lat.periodic, lat.mask, omega=1.0, xforce=1e-5,
                iterations=iterations, init="zero", want_pdfs=False)
    finally:
        os.sched_setaffinity(0, saved)
    dur = ref.last_duration
    it = iterations + (iterations % 2)  # the AA loop runs whole pairs
    return {"mflups": lat.n_fluid * it / dur / 1e6, "seconds": dur, "iterations": it, "threads": threads,
            "variant": variant, "pinned": "%d threads pinned one per physical core (cpus %s)%s"
            % (threads, _cpu_ranges(cpus[:threads]), "" if pin_failed == 0 else ", %d pinnings failed" % pin_failed),
            "host": desc}


def _cpu_ranges(cpus):
    out, i = [], 0
    while i < len(cpus):
        j = i
        while j + 1 < len(cpus) and cpus[j + 1] == cpus[j] + 1:
            j += 1
        out.append(str(cpus[i]) if i == j else "%d-%d" % (cpus[i], cpus[j]))
        i = j + 1
    return ",".join(out)


def aa_line(lbmb200, fl, args, kargs, dist, peak):
    """Device-timed cuda-aa-soa steps on lattice `fl`: MFLUP/s, HBM fraction,
    per-launch split of each even/odd pair, and the reference's fastest
    full-array CPU kernel (aa-vec-soa) on the same lattice beside it."""
    ta = time_kernel(lbmb200, "cuda-aa-soa", fl, min(args.steps, 200), 4, kargs, dist, "aa")
    ta["inst"].deinit()
    per, lpp = ta["per_launch_ms"], ta["launches_per_pair"]
    # per pair: even step, then the odd step's launches (interior blocks without
    # and with reversed links, face shell)
    pairs = [per[k:k + lpp] for k in range(0, len(per) - lpp + 1, lpp)]
    ev = statistics.mean(p[0] for p in pairs)
    od = statistics.mean(sum(p[1:]) for p in pairs)
    am = (ev + od) / 2
    out = {"fluid_nodes": fl.n_fluid, "mflups": round(fl.n_fluid / (am / 1e3) / 1e6, 1),
           "achieved_gbs": round(B_PER_FLUP["aa"] * fl.n_fluid / (am / 1e3) / 1e9, 1),
           "frac": round(B_PER_FLUP["aa"] * fl.n_fluid / (am / 1e3) / 1e9 / peak, 4),
           "even_ms": round(ev, 5), "odd_ms": round(od, 5),
           "odd_launch_ms": [round(statistics.mean(p[k] for p in pairs), 5) for k in range(1, lpp)]}
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu:
        probe = cpu_reference(fl, 2, kernel="aa-vec-soa")
        if probe is not None:
            iters = int(max(2, min(200, 5.0 * probe["mflups"] * 1e6 / fl.n_fluid)))
            r = cpu_reference(fl, iters + iters % 2, kernel="aa-vec-soa")
            out["cpu_reference"] = {"mflups": round(r["mflups"], 1), "cores": r["threads"],
                                    "sample": "%d steps, reference aa-vec-soa (%s build), %s"
                                              % (r["iterations"], r["variant"], r["pinned"])}
    return out


def cpu_model():
    """The processor's name with its family/model/stepping (a virtual machine
    may report only a generic name) and, where sysfs has it, the socket count."""
    info = {}
    try:
        for line in open("/proc/cpuinfo"):
            k, _, v = line.partition(":")
            k = k.strip()
            if k in ("model name", "cpu family", "model", "stepping") and k not in info:
                info[k] = v.strip()
    except OSError:
        return "unknown"
    sockets = set()
    for c in sorted(os.sched_getaffinity(0)):
        try:
            with open("/sys/devices/system/cpu/cpu%d/topology/physical_package_id" % c) as f:
                sockets.add(f.read().strip())
        except OSError:
            pass
    return "%s (family %s, model %s, stepping %s%s)" % (
        info.get("model name", "unknown"), info.get("cpu family", "?"), info.get("model", "?"),
        info.get("stepping", "?"), ", %d socket(s)" % len(sockets) if sockets else "")


# ---------------------------------------------------------------------------
# the batched (512 domains), served and reduced-precision workloads

def _batch_domains(n, seed, edge_range=(32, 128), threads=16):
    """n seeded porous domains: edge U{32..128}, r ~ U[3,8], porosity U[0.3,0.6],
    omega U[0.8,1.6]; sphere packings generated on host threads (C)."""
    import concurrent.futures

    import numpy as np

    import lbmb200
    rng = np.random.default_rng(seed)
    specs = [(int(rng.integers(edge_range[0], edge_range[1] + 1)), float(rng.uniform(0.3, 0.6)),
              float(rng.uniform(0.8, 1.6)), seed * 1000 + i) for i in range(n)]
    with concurrent.futures.ThreadPoolExecutor(threads) as pool:
        lats = list(pool.map(lambda sp: lbmb200.spheres((sp[0],) * 3, sp[3], sp[1], 3.0, 8.0)[0], specs))
    return lats, [sp[2] for sp in specs]


def section_batched(args, dist, peak):
    """512 domains in one batch (FP32), autotuned, 100-step CUDA graphs, against
    the same kernel family run one domain at a time."""
    import time

    import numpy as np

    import lbmb200
    L = lbmb200.lib()
    lats, omegas = _batch_domains(args.batched, 7000 + dist.rank)
    b = lbmb200.Batch("fp32", budget_gb=150.0, max_domains=args.batched)
    try:
        slots = [b.add(l, omega=o, lam=3.0 / 16.0, xforce=1e-5) for l, o in zip(lats, omegas)]
        if min(slots) < 0:
            raise RuntimeError("the domains do not fit the HBM budget")
        nodes = sum(l.n_fluid for l in lats)
        rows = b.tune(trial_steps=6)
        print("batched tuner rows {which, threads, nodes/thread, blocks (0 = one per tile), ms}:\n"
              + "\n".join(" ".join("%g" % v for v in r) for r in rows), file=sys.stderr)
        cfg = b.launch()
        b.step(100, graph=True)  # capture and warm the graph
        b.sync()
        reps = 3
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(reps):
            b.step(100, graph=True)
        b.sync()
        wall = dist.max(time.perf_counter() - t0)
        ms_direct = b.time_steps(100)
        agg = nodes * 100 * reps / wall / 1e6
        agg_direct = nodes * 100 / (ms_direct / 1e3) / 1e6
    finally:
        b.close()
    # one at a time: a seeded subset of the same domains, each alone with the
    # single-domain FP32 list kernel (device-timed 100 steps each)
    sub = list(range(0, len(lats), max(1, len(lats) // 64)))[:64]
    tot_nodes_steps, tot_s = 0, 0.0
    for i in sub:
        lat = lats[i]
        inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=["-precision", "fp32", "-lambda", "3/16"])
        try:
            inst.set_field(np.ascontiguousarray(equilibrium_field(lbmb200, lat)))
            cd = lbmb200.case(omega=omegas[i], xforce=1e-5, iterations=100)
            tot = ctypes.c_double(0.0)
            L.lbm_b200_time_steps(inst.kdp, ctypes.byref(cd), 4, ctypes.byref(tot), None)
            L.lbm_b200_time_steps(inst.kdp, ctypes.byref(cd), 100, ctypes.byref(tot), None)
            tot_s += tot.value / 1e3
            tot_nodes_steps += lat.n_fluid * 100
        finally:
            inst.deinit()
    one = tot_nodes_steps / tot_s / 1e6
    return {"domains": len(lats), "fluid_nodes": nodes, "storage": "fp32",
            "mflups_graph": round(dist.sum(agg), 1), "mflups_direct_launch": round(dist.sum(agg_direct), 1),
            "mflups_one_at_a_time": round(dist.sum(one), 1), "speedup_vs_one_at_a_time": round(agg / one, 2),
            "one_at_a_time_sample": "%d of %d domains, single-domain FP32 kernel, 100 device-timed steps each"
                                    % (len(sub), len(lats)),
            "autotuned": cfg, "tuner_candidates": int(len(rows)),
            "timing": "wall clock around 3 synchronised replays of a 100-step CUDA graph"}


def section_serving(args, dist, peak):
    """Continuous batching (FP32) against the plain FP64 kernel one request at a
    time, on the same seeded open-loop stream at 80 % of measured capacity.
    Both servers prepare packings on the same number of host threads (one per
    physical core but the serving loop's) from each request's arrival on, so
    the ratio compares the GPU work, not host preparation."""
    from lbmb200 import serving
    n = args.serving
    om = (0.8, 1.6)
    # host preparation (sphere packings, in C) on one thread per physical core
    # but the one the serving loop itself runs on, alike for both servers
    prep = max(1, len(host_cpus()[0]) - 1)
    # capacity: the batched server with every request available at t = 0
    cap_reqs = serving.make_requests(n, rate=0.0, seed=900 + dist.rank, omega_range=om)
    cap_sum, _ = serving.serve_batched(cap_reqs, closed_loop=True, prep_threads=prep)
    rate = 0.8 * cap_sum["solves_per_s"]
    reqs = serving.make_requests(n, rate=rate, seed=901 + dist.rank, omega_range=om)
    batched, recs = serving.serve_batched(reqs, prep_threads=prep)
    fp64, recs64 = serving.serve_fp64_sequential(reqs, prep_threads=prep)
    by_id = {r["id"]: r for r in recs64}
    both = [r for r in recs if r["k"] is not None and by_id[r["id"]]["k"] is not None]
    kerr = max((abs(r["k"] - by_id[r["id"]]["k"]) / abs(by_id[r["id"]]["k"]) for r in both), default=None)
    return {"requests": n, "arrivals": "Poisson, %.3f/s (0.8 x measured capacity %.3f/s)"
                                      % (rate, cap_sum["solves_per_s"]),
            "domain": "edge U{32..192}, porosity U[0.3,0.6], r U[3,8], omega U[0.8,1.6], F_x=1e-5, "
                      "tol 1e-6 per 100 steps, cap 20000",
            "preparation": "both servers: packings built on %d host threads (one per physical core but the "
                           "serving loop's) from each request's arrival on" % prep,
            "p99_note": "p99 over %d latency samples" % batched["latency_samples"],
            "batched_fp32": batched, "fp64_one_at_a_time": fp64,
            "solves_per_s_ratio": round(batched["solves_per_s"] / fp64["solves_per_s"], 3),
            "max_rel_permeability_diff_fp32_vs_fp64": kerr}


def section_precision(args, dist, peak):
    """The 256^3 packing for N steps in FP64, FP32 and FP16-deviation storage."""
    import lbmb200
    from lbmb200 import porous
    lat, _ = lbmb200.spheres((args.edge,) * 3, args.seed, args.porosity, 6.0, 12.0)
    res = porous.precision_study(lat, steps=args.precision_steps, xforce=1e-5)
    res["steps"] = args.precision_steps
    return res


# ---------------------------------------------------------------------------
# one lattice over the ranks (x-slabs, strong scaling)

class CudaSlabBackend:
    """Slabs on this rank's GPU: the library's list-layout slab, an explicit
    stream that is also torch's current stream, NCCL messages through
    DistTransport, CUDA events for the timing."""

    def __init__(self, dist):
        import torch
        self.torch = torch
        torch.cuda.set_device(dist.local)
        self.work = torch.cuda.Stream()
        torch.cuda.set_stream(self.work)
        self.stream = self.work.cuda_stream

    def slab(self, lat, x0, x1, lo, hi, kargs):
        import numpy as np

        import lbmb200
        from lbmb200 import slabs as sl
        s = sl.Slab(lat, x0, x1, lo, hi, kernel_args=kargs, layout="list")
        s.inst.set_field(np.broadcast_to(lbmb200.W, (s.local.mask.size, 19)))
        return s

    def transport(self, slab, rank, world, ring):
        import torch.distributed
        from lbmb200 import slabs as sl
        return sl.DistTransport(slab, rank, world, ring, torch.distributed,
                                lambda n: self.torch.empty(n, dtype=self.torch.float64, device="cuda"),
                                stream=self.stream)

    def mark(self):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.work)
        return e

    def sync(self):
        self.torch.cuda.synchronize()

    @staticmethod
    def ms(a, b):
        return a.elapsed_time(b)

    def close(self, slab):
        slab.close()
        self.torch.cuda.synchronize()
        self.torch.cuda.set_stream(self.torch.cuda.default_stream())


class _TimedTransport:
    """Marks the stream around each exchange operation of a transport (the
    packs, the posting, the wait and the unpacks), so that the share of the
    run spent on messages can be read off afterwards; nothing is skipped."""

    def __init__(self, tr, backend):
        self.tr, self.b, self.spans = tr, backend, []

    def _timed(self, fn, phase):
        m0 = self.b.mark()
        fn(phase)
        self.spans.append((m0, self.b.mark()))

    def exchange(self, phase):
        self._timed(self.tr.exchange, phase)

    def start(self, phase):
        self._timed(self.tr.start, phase)

    def finish(self, phase):
        self._timed(self.tr.finish, phase)


def section_slabs(args, dist, backend=None, lat=None, pairs=20, warmup=3):
    """The indirect-addressing workload's lattice (list layout, FP64) split
    into x-slabs, one per rank, halo messages between neighbouring ranks:
    serial (exchange after each half step) and overlapped (messages travel
    while the inner tiles step). Every rank builds the same lattice (the
    headline seed, not seed + rank) and takes its slab; times are the max
    over ranks of the device-timed pairs."""
    from lbmb200 import slabs as sl
    import lbmb200
    backend = backend or CudaSlabBackend(dist)
    if lat is None:
        lat, _ = sphere_lattice(lbmb200, args.edge, args.porosity, args.seed)
    x0, x1 = sl.partition(lat.dims[0], dist.world)[dist.rank]
    ring = sl.is_ring(lat.periodic)
    lo, hi = sl.halo_flags(dist.rank, dist.world, ring)
    slab = backend.slab(lat, x0, x1, lo, hi, ["-lambda", "3/16"])
    try:
        tr = _TimedTransport(backend.transport(slab, dist.rank, dist.world, ring), backend)
        cd = lbmb200.case(omega=1.0, xforce=1e-5)
        nodes = dist.sum(slab.local.n_fluid)
        out = {"workload": "%d^3 sphere packing (seed %d), list layout, FP64, split in x over %d ranks"
                           % (args.edge, args.seed, dist.world),
               "scaling": "strong", "fluid_nodes": nodes, "pairs": pairs,
               "slab_planes": [x0, x1], "layout": "list"}
        for overlap in (False, True):
            sl.step_pairs([slab], tr, cd, warmup, backend.stream, overlap=overlap)
            backend.sync()
            tr.spans = []
            dist.barrier()
            e0 = backend.mark()
            sl.step_pairs([slab], tr, cd, pairs, backend.stream, overlap=overlap)
            e1 = backend.mark()
            backend.sync()
            own = backend.ms(e0, e1)
            exch = sum(backend.ms(a, b) for a, b in tr.spans)
            ms = dist.max(own)
            key = "overlapped" if overlap else "serial"
            out[key] = {"ms": round(ms, 4), "mflups": round(nodes * 2 * pairs / (ms / 1e3) / 1e6, 1),
                        "mflups_per_rank": round(nodes * 2 * pairs / (ms / 1e3) / 1e6 / dist.world, 1),
                        "exchange_share": round(dist.max(exch / own if own > 0 else 0.0), 4)}
        out["exchange_share_note"] = ("time of the stream between the marks around each exchange operation "
                                      "(packs, posting, waiting, unpacks) over the pairs' time, max over ranks")
        return out
    finally:
        backend.close(slab)


# ---------------------------------------------------------------------------

def headline_config(args, stats, lat, n_cells, dist):
    """The workload of the headline line, the same for both arms."""
    return {"workload": "%d^3 periodic sphere packing, porosity %.4f, r~U[6,12], seed %d+rank; "
                        "list AA (list-aa-pv-soa), FP64, Lambda=3/16, omega=1, F_x=1e-5"
                        % (args.edge, stats["porosity"], args.seed),
            "fluid_nodes_per_rank": lat.n_fluid, "packing": stats,
            "l2": "inputs larger than L2 (%.2f GB of PDFs per rank)" % (19 * 8 * n_cells / 1e9),
            "parallelism": "replicas" if dist.world > 1 else "single GPU"}


def run_reference_arm(args, dist):
    metric = "MFLUP/s & % HBM roofline at 256^3"
    if dist.rank != 0:
        return 0
    import lbmb200
    lat, stats = sphere_lattice(lbmb200, args.edge, args.porosity, args.seed)
    if args.warmup > 0:
        cpu_reference(lat, max(2, args.warmup))
    r = cpu_reference(lat, args.steps)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref is missing"}))
        return 0
    line = {"impl": "reference", "metric": metric, "value": round(r["mflups"], 3), "unit": "MFLUP/s",
            "n_gpus": args.gpus, "steps": r["iterations"], "warmup": args.warmup,
            "ms_per_step": round(1e3 * r["seconds"] / r["iterations"], 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": headline_config(args, stats, lat, lbmb200.lib().lbmh_pad_cells(lat.n_fluid, 8, None), dist),
            "kernel": "reference list-aa-pv-soa (%s build; its Lambda is fixed at 1/12, which does not change "
                      "the work per step)" % r["variant"],
            "cpu_baseline": {"value": round(r["mflups"], 3), "unit": "MFLUP/s", "cores": r["threads"],
                             "kind": "reference", "sample": "%d steps of the full domain, %s"
                                                            % (r["iterations"], r["pinned"]),
                             "cpu": r["host"]},
            "e2e": {"value": round(r["mflups"], 3), "unit": "MFLUP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args, dist):
    import numpy as np

    import lbmb200
    L = lbmb200.lib()
    if L.lbm_b200_set_device(dist.local) != 0:
        raise RuntimeError("cannot select CUDA device %d: %s" % (dist.local, L.lbm_b200_last_error().decode()))
    peak, peak_kind = measured_peaks()
    lat, stats = sphere_lattice(lbmb200, args.edge, args.porosity, args.seed + dist.rank)
    kargs = ["-lambda", "3/16"]

    clocks = ClockSampler(dist.local)
    clocks.start()
    t = time_kernel(lbmb200, "cuda-list-aa-pv-soa", lat, args.steps, max(3, args.warmup), kargs, dist, "odd")
    inst = t["inst"]
    adj_node = adjacency_bytes_per_node(lbmb200, inst, lat.n_fluid)
    odd_bpf = B_PER_FLUP["even"] + adj_node
    try:
        # e2e: the reference-facing Kernel() call, mirror uploaded and downloaded
        cd = lbmb200.case(omega=1.0, xforce=1e-5, iterations=500)
        L.lbm_b200_mark_mirror_dirty(inst.kdp)
        dist.barrier()
        w0 = time.perf_counter()
        inst.run(cd)
        e2e_s = time.perf_counter() - w0
        e2e_s = dist.max(e2e_s)
        h2d, d2h = inst.last_copy_bytes()
        e2e_iters = 500
        n_cells = inst.list_layout()[3]
    finally:
        inst.deinit()
    clk = clocks.stop()

    nf_total = dist.sum(lat.n_fluid)
    ms = dist.max(t["ms"])
    steps_run = t["steps_run"]
    value = nf_total * steps_run / (ms / 1e3) / 1e6
    per = t["per_launch_ms"]
    even = per[0::2]
    odd = per[1::2]
    odd_ms = statistics.mean(odd)
    even_ms = statistics.mean(even)
    achieved = odd_bpf * lat.n_fluid / (odd_ms / 1e3) / 1e9
    traffic = profile_traffic("list_odd_fp64")
    line = {
        "metric": "MFLUP/s & % HBM roofline at 256^3", "value": round(value, 3), "unit": "MFLUP/s",
        "n_gpus": dist.world, "steps": steps_run, "warmup": max(3, args.warmup),
        "ms_per_step": round(ms / steps_run, 5), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(args, stats, lat, n_cells, dist),
        "roofline": {"bound": "hbm", "kernel": "k_list_odd_fp64 (adjacency-driven odd step)",
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
                     "bytes_per_flup": round(odd_bpf, 2),
                     "adjacency": "run-compressed: %.2f B per node (72 uncompressed)" % adj_node,
                     "launch_ms": round(odd_ms, 5),
                     "traffic": traffic,
                     "even_step": {"bytes_per_flup": B_PER_FLUP["even"], "launch_ms": round(even_ms, 5),
                                   "achieved": round(B_PER_FLUP["even"] * lat.n_fluid / (even_ms / 1e3) / 1e9, 1)}},
        "e2e": {"value": round(nf_total * e2e_iters / e2e_s / 1e6, 3), "unit": "MFLUP/s",
                "h2d_bytes_per_step": int(round(h2d / e2e_iters)), "d2h_bytes_per_step": int(round(d2h / e2e_iters)),
                "h2d_bytes_per_call": int(h2d), "d2h_bytes_per_call": int(d2h), "steps_per_call": e2e_iters,
                "call": "one Kernel() call of %d time steps: the PDF field uploaded from the pinned host mirror "
                        "before the steps and downloaded after them (the bytes per step are the call's bytes "
                        "over its steps)" % e2e_iters},
        "gpu_launches": t["launches"],
        "clocks": clk,
    }

    # with several ranks the line carries the replica headline and the slab
    # split; the secondary kernel lines, batched and serving sections are
    # single-GPU measurements (every rank would repeat them on its own GPU)
    if not args.no_extra and dist.world == 1:
        extra = {}
        # pull kernel on the same domain
        tp = time_kernel(lbmb200, "cuda-list-pull-split-nt-1s-soa", lat, min(args.steps, 200), 3, kargs, dist, "pull")
        bpf = B_PER_FLUP["even"] + adjacency_bytes_per_node(lbmb200, tp["inst"], lat.n_fluid)
        tp["inst"].deinit()
        pm = statistics.mean(tp["per_launch_ms"])
        extra["cuda-list-pull-split-nt-1s-soa"] = {
            "mflups": round(lat.n_fluid / (pm / 1e3) / 1e6, 1), "launch_ms": round(pm, 5),
            "bytes_per_flup": round(bpf, 2),
            "achieved_gbs": round(bpf * lat.n_fluid / (pm / 1e3) / 1e9, 1),
            "frac": round(bpf * lat.n_fluid / (pm / 1e3) / 1e9 / peak, 4)}
        # the two-grid list rows on the same domain (304 B of PDFs plus the adjacency each reads per node update)
        for kname in ("cuda-list-push-soa", "cuda-list-pull-soa"):
            tq = time_kernel(lbmb200, kname, lat, min(args.steps, 200), 3, kargs, dist, "pull")
            bpf = B_PER_FLUP["even"] + adjacency_bytes_per_node(lbmb200, tq["inst"], lat.n_fluid)
            tq["inst"].deinit()
            qm = statistics.mean(tq["per_launch_ms"])
            extra[kname] = {"mflups": round(lat.n_fluid / (qm / 1e3) / 1e6, 1), "launch_ms": round(qm, 5),
                            "bytes_per_flup": round(bpf, 2),
                            "achieved_gbs": round(bpf * lat.n_fluid / (qm / 1e3) / 1e9, 1),
                            "frac": round(bpf * lat.n_fluid / (qm / 1e3) / 1e9 / peak, 4)}
        # full-array AA at 256^3: the reference's -geometry fluid with -periodic-x -periodic-y
        # -periodic-z, and -geometry channel (x periodic, walls in y and z)
        for key, geo, per_flags in (("cuda-aa-soa", "fluid", (1, 1, 1)), ("cuda-aa-soa/channel", "channel", (0, 0, 0))):
            fl = lbmb200.geometry(geo, (args.edge,) * 3, per_flags)
            extra[key] = aa_line(lbmb200, fl, args, kargs, dist, peak)
            extra[key]["workload"] = "%d^3 %s" % (args.edge, "fully periodic fluid box" if geo == "fluid"
                                                  else "channel, periodic x, walls in y and z")
        # the two-grid full-array rows on the fluid box (304 B per node update)
        fl = lbmb200.geometry("fluid", (args.edge,) * 3, (1, 1, 1))
        for kname in ("cuda-push-soa", "cuda-pull-soa"):
            tq = time_kernel(lbmb200, kname, fl, min(args.steps, 100), 3, kargs, dist, "aa")
            tq["inst"].deinit()
            qm = statistics.mean(tq["per_launch_ms"])
            extra[kname] = {"workload": "%d^3 fully periodic fluid box" % args.edge,
                            "mflups": round(fl.n_fluid / (qm / 1e3) / 1e6, 1), "launch_ms": round(qm, 5),
                            "achieved_gbs": round(B_PER_FLUP["aa"] * fl.n_fluid / (qm / 1e3) / 1e9, 1),
                            "frac": round(B_PER_FLUP["aa"] * fl.n_fluid / (qm / 1e3) / 1e9 / peak, 4)}
        # reduced storage list AA on the porous domain (FP32 arithmetic)
        for prec, pb in (("fp32", 4), ("fp16", 2)):
            tl = time_kernel(lbmb200, "cuda-list-aa-pv-soa", lat, min(args.steps, 200), 4,
                             kargs + ["-precision", prec], dist, "odd")
            # mean of the even (38 s) and odd (38 s + adjacency) steps
            bpf = 2 * 19 * pb + adjacency_bytes_per_node(lbmb200, tl["inst"], lat.n_fluid) / 2
            tl["inst"].deinit()
            m = statistics.mean(tl["per_launch_ms"])
            extra["cuda-list-aa-pv-soa/" + prec] = {
                "mflups": round(lat.n_fluid / (m / 1e3) / 1e6, 1), "bytes_per_flup": round(bpf, 2),
                "achieved_gbs": round(bpf * lat.n_fluid / (m / 1e3) / 1e9, 1),
                "frac": round(bpf * lat.n_fluid / (m / 1e3) / 1e9 / peak, 4),
                "even_ms": round(statistics.mean(tl["per_launch_ms"][0::2]), 5),
                "odd_ms": round(statistics.mean(tl["per_launch_ms"][1::2]), 5)}
        line["kernels"] = extra

    for name, fn, enabled in (("batched", section_batched, args.batched > 0 and dist.world == 1),
                              ("serving", section_serving, args.serving > 0 and dist.world == 1),
                              ("precision", section_precision, args.precision_steps > 0 and dist.world == 1),
                              ("slabs", lambda a, d, p: section_slabs(a, d), dist.world > 1 and not args.no_slabs)):
        if not enabled:
            continue
        try:
            line[name] = fn(args, dist, peak)
        except Exception as e:  # a failing extra must not lose the headline line
            line[name] = {"error": "%s: %s" % (type(e).__name__, e)}

    if dist.rank == 0 and dist.world == 1 and not args.no_cpu:
        probe = cpu_reference(lat, 2)
        if probe is not None:
            # size the sample to about 10 s of CPU work
            iters = int(max(4, min(400, 10.0 * probe["mflups"] * 1e6 / lat.n_fluid)))
            r = cpu_reference(lat, iters)
            line["cpu_baseline"] = {"value": round(r["mflups"], 3), "unit": "MFLUP/s", "cores": r["threads"],
                                    "kind": "reference",
                                    "sample": "%d steps of the same domain, reference list-aa-pv-soa (%s build), %s"
                                              % (r["iterations"], r["variant"], r["pinned"]),
                                    "cpu": r["host"]}
    if dist.rank == 0:
        print(json.dumps(line))
    return 0


def main():
    args = parse()
    from lbmb200.ranks import Ranks
    dist = Ranks(timeout_s=120)
    try:
        if args.impl == "reference":
            return run_reference_arm(args, dist)
        return run_ours(args, dist)
    finally:
        dist.close()


if __name__ == "__main__":
    sys.exit(main())
