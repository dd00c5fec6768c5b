"""Permeability solves on seeded porous domains (no counterpart in the
reference, which benchmarks fixed-length runs only).

A solve drives the flow with a body force F along x until the mean velocity
settles: it stops when the relative change of the mean x velocity over the
last `check_every` steps drops below `tol` (status "converged"), after `cap`
steps ("not_converged"), or as soon as the FP64 sums are not finite
("diverged": an unstable relaxation rate or a corrupt initial field; the
domain then holds NaN or Inf and would never meet the tolerance). Mass and
momentum are summed on the GPU in FP64 (lbm_b200_moments_device for the FP64
kernel, the batch's per-domain sums for reduced storage).

Permeability (lattice units), Darcy's law with the body force per unit mass
F: k = nu * q / F, with the superficial velocity q = sum_fluid u_x / N_total
and u_x = j_x + F/2 per node (the half-force correction the reference also
applies to its velocity profile, src/Kernel.c:488-493), nu = (1/omega - 1/2)/3.
"""
import ctypes
import math
import time

import numpy as np

from . import Batch, case, kernel, lib, spheres


def viscosity(omega):
    return (1.0 / omega - 0.5) / 3.0


def mean_ux(jx_sum, n_fluid, xforce):
    return (jx_sum + n_fluid * 0.5 * xforce) / n_fluid


def permeability(jx_sum, n_fluid, n_total, omega, xforce):
    q = (jx_sum + n_fluid * 0.5 * xforce) / n_total
    return viscosity(omega) * q / xforce


CONVERGED, NOT_CONVERGED, DIVERGED = "converged", "not_converged", "diverged"


def stop_status(u, prev, steps, tol, cap):
    """The stopping rule after a check: None (keep going) or the status."""
    if not math.isfinite(u):
        return DIVERGED
    if prev is not None and abs(u - prev) <= tol * abs(u):
        return CONVERGED
    if steps >= cap:
        return NOT_CONVERGED
    return None


def request_domain(seed, edge, porosity, rmin=3.0, rmax=8.0):
    lat, stats = spheres((edge, edge, edge), seed, porosity, rmin, rmax)
    return lat, stats


class _Fp64Solver:
    """The plain FP64 list AA kernel, one domain at a time."""

    def __init__(self, lattice, omega, lam, xforce):
        self.lat, self.omega, self.xforce = lattice, omega, xforce
        self.inst = kernel("cuda-list-aa-pv-soa").init(lattice, kernel_args=["-lambda", repr(lam)])
        self.inst.set_field(np.broadcast_to(_W, (lattice.mask.size, 19)))
        self.cd = case(omega=omega, xforce=xforce, iterations=0)
        self.out = (ctypes.c_double * 4)()

    def step(self, n):
        self.inst.step_device(self.cd, n)

    def jx(self):
        rc = lib().lbm_b200_instance_moments(self.inst.kdp, self.out)
        if rc:
            raise RuntimeError("moments failed: %d" % rc)
        return float(self.out[1])

    def close(self):
        self.inst.deinit()


from . import W as _W  # noqa: E402


def solve_fp64(lattice, omega=1.0, lam=3.0 / 16.0, xforce=1e-5, check_every=100, tol=1e-6, cap=20000,
               initial_field=None):
    """Steady-state permeability with the FP64 kernel; returns dict with the
    status (k is None for a diverged solve). initial_field: PDFs to start
    from instead of the equilibrium f_i = w_i."""
    s = _Fp64Solver(lattice, omega, lam, xforce)
    try:
        if initial_field is not None:
            s.inst.set_field(initial_field)
        prev, steps, t0 = None, 0, time.perf_counter()
        while True:
            s.step(check_every)
            steps += check_every
            jx = s.jx()
            u = mean_ux(jx, lattice.n_fluid, xforce)
            status = stop_status(u, prev, steps, tol, cap)
            if status:
                break
            prev = u
        k = None if status == DIVERGED else permeability(jx, lattice.n_fluid, lattice.mask.size, omega, xforce)
        return {"k": k, "steps": steps, "u": u, "status": status, "seconds": time.perf_counter() - t0}
    finally:
        s.close()


def solve_batched(lattices, storage="fp32", omegas=None, lam=3.0 / 16.0, xforce=1e-5, check_every=100, tol=1e-6,
                  cap=20000, budget_gb=150.0, initial_fields=None):
    """Steady-state permeabilities of several domains solved together in one
    batch; returns one dict per domain (same stopping rule as solve_fp64).
    initial_fields: optional list of PDF fields (None = equilibrium)."""
    omegas = omegas or [1.0] * len(lattices)
    b = Batch(storage, budget_gb=budget_gb, max_domains=max(1, len(lattices)))
    try:
        slots = [b.add(l, omega=o, lam=lam, xforce=xforce) for l, o in zip(lattices, omegas)]
        if min(slots) < 0:
            raise RuntimeError("domains do not fit the batch")
        for s, f in zip(slots, initial_fields or []):
            if f is not None:
                b.set_field(s, f)
        live = {s: i for i, s in enumerate(slots)}
        prev, steps, res = {}, 0, [None] * len(lattices)
        while live:
            b.step(check_every)
            steps += check_every
            mom = b.moments()
            for s in list(live):
                i = live[s]
                lat = lattices[i]
                u = mean_ux(mom[s][1], lat.n_fluid, xforce)
                status = stop_status(u, prev.get(s), steps, tol, cap)
                prev[s] = u
                if status:
                    k = None if status == DIVERGED else permeability(mom[s][1], lat.n_fluid, lat.mask.size,
                                                                     omegas[i], xforce)
                    res[i] = {"k": k, "steps": steps, "u": u, "status": status}
                    b.remove(s)
                    del live[s]
        return res
    finally:
        b.close()


_CX = np.array([0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0], dtype=np.float64)
_CY = np.array([1, -1, 0, 0, 1, -1, 1, -1, 0, 1, 0, 0, -1, 0, -1, 1, 0, 0, 0], dtype=np.float64)
_CZ = np.array([0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, 0], dtype=np.float64)


def velocity_field(pdfs, mask, xforce):
    """Per fluid node (u_x, u_y, u_z) = sum_i c_i f_i + (F/2, 0, 0)."""
    f = pdfs[mask != 0]
    u = np.stack([f @ _CX, f @ _CY, f @ _CZ], axis=1)
    u[:, 0] += 0.5 * xforce
    return u


def precision_study(lattice, steps=20000, omega=1.0, lam=3.0 / 16.0, xforce=1e-5, storages=("fp32", "fp16")):
    """Runs the same domain for `steps` steps with FP64 PDFs and with each
    reduced storage; reports the relative L2 error of the velocity field and
    the relative permeability error against the FP64 run."""
    out = {}
    s = _Fp64Solver(lattice, omega, lam, xforce)
    try:
        t0 = time.perf_counter()
        for done in range(0, steps, 1000):
            s.step(min(1000, steps - done))
        jx = s.jx()
        t64 = time.perf_counter() - t0
        s.inst.sync_mirror()
        u64 = velocity_field(s.inst.get_field(), lattice.mask, xforce)
    finally:
        s.close()
    k64 = permeability(jx, lattice.n_fluid, lattice.mask.size, omega, xforce)
    out["fp64"] = {"k": k64, "seconds": t64}
    norm = np.sqrt((u64 ** 2).sum())
    for st in storages:
        b = Batch(st, budget_gb=8.0, max_domains=1)
        try:
            slot = b.add(lattice, omega=omega, lam=lam, xforce=xforce)
            t0 = time.perf_counter()
            for done in range(0, steps, 1000):
                b.step(min(1000, steps - done))
            mom = b.moments()
            t = time.perf_counter() - t0
            u = velocity_field(b.get_field(slot), lattice.mask, xforce)
        finally:
            b.close()
        k = permeability(mom[slot][1], lattice.n_fluid, lattice.mask.size, omega, xforce)
        out[st] = {"k": k, "k_rel_err": abs(k - k64) / abs(k64),
                   "u_l2_rel_err": float(np.sqrt(((u - u64) ** 2).sum()) / norm), "seconds": t}
    return out
