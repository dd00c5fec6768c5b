"""Continuous-batching server for permeability solves (no counterpart in the
reference).

Requests (a seeded porous domain each) arrive over time. Each one is
prepared on a host worker thread (sphere packing, in C), then admitted into
the running batch as soon as a slot and the HBM budget allow; admitted
domains keep their PDFs on the device and advance together, one persistent
launch per step for all of them (lbm_batch_*, replayed from a captured CUDA
graph in chunks of `check_every` steps). After every chunk the FP64
per-domain sums decide which domains are done (porous.py's stopping rule:
converged, not converged within the step cap, or diverged -- non-finite
sums retire a domain at its next check instead of holding its slot and HBM
until the cap); those return their status and permeability and leave,
freeing memory for the next arrivals while the others keep running.

The baseline serves the same stream one request at a time with the plain FP64
list AA kernel. Both servers prepare requests the same way: each request's
packing is built on a pool of host threads from its arrival on, so host
preparation overlaps the GPU work in both and neither's service time counts
packing that the other hides.
"""
import collections
import concurrent.futures
import time

import numpy as np

from . import Batch
from .porous import DIVERGED, mean_ux, permeability, request_domain, solve_fp64, stop_status

Request = collections.namedtuple("Request", "id arrival seed edge porosity omega")


def make_requests(n, rate, seed=1, edge_range=(32, 192), porosity_range=(0.3, 0.6), omega_range=(1.0, 1.0)):
    """n requests with Poisson arrivals at `rate` per second (seeded)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        out.append(Request(i, t, int(rng.integers(1, 2 ** 31)), int(rng.integers(edge_range[0], edge_range[1] + 1)),
                           float(rng.uniform(*porosity_range)), float(rng.uniform(*omega_range))))
    return out


def _summary(records, wall):
    lat = np.array([r["done"] - r["arrival"] for r in records])
    status = collections.Counter(r["status"] for r in records)
    return {"solves": len(records), "wall_s": wall, "solves_per_s": len(records) / wall if wall > 0 else None,
            "p50_latency_s": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_latency_s": float(np.percentile(lat, 99)) if len(lat) else None,
            "latency_samples": int(len(lat)),
            "mean_steps": float(np.mean([r["steps"] for r in records])) if records else None,
            "status": dict(sorted(status.items()))}


def serve_batched(requests, storage="fp32", budget_gb=150.0, max_active=256, lam=3.0 / 16.0, xforce=1e-5,
                  check_every=100, tol=1e-6, cap=20000, prep_threads=8, closed_loop=False, initial_field=None):
    """Serves `requests` with continuous batching; returns (summary, records).
    closed_loop: every request is available at time 0 (capacity measurement).
    initial_field(request, lattice): PDFs to start a request from (None =
    equilibrium)."""
    b = Batch(storage, budget_gb=budget_gb, max_domains=max_active)
    pool = concurrent.futures.ThreadPoolExecutor(prep_threads)
    pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
    preparing = {}   # future -> request
    ready = collections.deque()  # (request, lattice)
    active = {}      # slot -> state
    records = []
    start = time.perf_counter()
    try:
        while pending or preparing or ready or active:
            now = time.perf_counter() - start
            while pending and (closed_loop or pending[0].arrival <= now):
                r = pending.popleft()
                preparing[pool.submit(request_domain, r.seed, r.edge, r.porosity)] = r
            for fut in [f for f in preparing if f.done()]:
                r = preparing.pop(fut)
                ready.append((r, fut.result()[0]))
            while ready:
                r, lat = ready[0]
                slot = b.add(lat, omega=r.omega, lam=lam, xforce=xforce)
                if slot < 0:
                    break  # wait for memory or a slot to free up
                ready.popleft()
                f0 = initial_field(r, lat) if initial_field else None
                if f0 is not None:
                    b.set_field(slot, f0)
                active[slot] = {"req": r, "lat": lat, "steps": 0, "prev": None,
                                "admit": time.perf_counter() - start}
            if not active:
                if preparing:
                    concurrent.futures.wait(list(preparing), timeout=0.05,
                                            return_when=concurrent.futures.FIRST_COMPLETED)
                elif pending:
                    time.sleep(max(0.0, min(0.05, pending[0].arrival - (time.perf_counter() - start))))
                continue
            b.step(check_every, graph=True)
            mom = b.moments()  # synchronises
            t_now = time.perf_counter() - start
            for slot in list(active):
                st = active[slot]
                st["steps"] += check_every
                lat = st["lat"]
                u = mean_ux(mom[slot][1], lat.n_fluid, xforce)
                status = stop_status(u, st["prev"], st["steps"], tol, cap)
                st["prev"] = u
                if status:
                    r = st["req"]
                    k = None if status == DIVERGED else permeability(mom[slot][1], lat.n_fluid, lat.mask.size,
                                                                     r.omega, xforce)
                    records.append({"id": r.id, "arrival": 0.0 if closed_loop else r.arrival, "admit": st["admit"],
                                    "done": t_now, "steps": st["steps"], "edge": r.edge, "porosity": r.porosity,
                                    "omega": r.omega, "fluid_nodes": lat.n_fluid, "status": status, "k": k})
                    b.remove(slot)
                    del active[slot]
        wall = time.perf_counter() - start
        return _summary(records, wall), records
    finally:
        pool.shutdown(wait=True)
        b.close()


def _prepare_on_arrival(r, start, closed_loop):
    """Host preparation of one request, started no earlier than its arrival."""
    if not closed_loop:
        wait = start + r.arrival - time.perf_counter()
        if wait > 0:
            time.sleep(wait)
    return request_domain(r.seed, r.edge, r.porosity)[0]


def serve_fp64_sequential(requests, lam=3.0 / 16.0, xforce=1e-5, check_every=100, tol=1e-6, cap=20000,
                          closed_loop=False, prep_threads=8, initial_field=None):
    """The same stream served one request at a time by the plain FP64 kernel.
    Packings are prepared as in serve_batched: on `prep_threads` host threads,
    each from its request's arrival on, so that the next request's packing is
    usually ready when the GPU frees up."""
    records = []
    ordered = sorted(requests, key=lambda q: q.arrival)
    pool = concurrent.futures.ThreadPoolExecutor(prep_threads)
    start = time.perf_counter()
    try:
        futs = [pool.submit(_prepare_on_arrival, r, start, closed_loop) for r in ordered]
        for r, fut in zip(ordered, futs):
            lat = fut.result()
            f0 = initial_field(r, lat) if initial_field else None
            res = solve_fp64(lat, omega=r.omega, lam=lam, xforce=xforce, check_every=check_every, tol=tol, cap=cap,
                             initial_field=f0)
            records.append({"id": r.id, "arrival": 0.0 if closed_loop else r.arrival,
                            "done": time.perf_counter() - start, "steps": res["steps"], "k": res["k"],
                            "status": res["status"], "edge": r.edge, "porosity": r.porosity, "omega": r.omega,
                            "fluid_nodes": lat.n_fluid})
        wall = time.perf_counter() - start
        return _summary(records, wall), records
    finally:
        pool.shutdown(wait=True, cancel_futures=True)
