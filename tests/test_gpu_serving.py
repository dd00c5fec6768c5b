"""Permeability solves: batched FP32 against the plain FP64 kernel, the same
result alone and in a mix, and the continuous-batching server end to end."""
import numpy as np
import pytest

import lbmb200
from lbmb200 import porous, serving

pytestmark = pytest.mark.gpu

TOL = 1e-6  # relative change of the mean velocity over 100 steps


def _lat(seed, edge, por):
    return porous.request_domain(seed, edge, por)[0]


def test_fp32_permeability_within_1e4_of_fp64():
    lat = _lat(11, 28, 0.45)
    k64 = porous.solve_fp64(lat, omega=1.0, xforce=1e-5, tol=TOL)
    k32 = porous.solve_batched([lat], storage="fp32", xforce=1e-5, tol=TOL)[0]
    assert k64["steps"] < 20000 and k32["steps"] < 20000
    assert abs(k32["k"] - k64["k"]) / k64["k"] < 1e-4
    assert k64["k"] > 0


def test_same_result_alone_and_in_the_mix():
    lats = [_lat(20 + i, e, p) for i, (e, p) in enumerate([(24, 0.4), (32, 0.55), (20, 0.35), (36, 0.5)])]
    omegas = [1.0, 1.3, 0.9, 1.5]
    alone = porous.solve_batched([lats[1]], omegas=[omegas[1]], tol=TOL)[0]
    mix = porous.solve_batched(lats, omegas=omegas, tol=TOL)
    assert mix[1]["steps"] == alone["steps"]
    assert mix[1]["k"] == alone["k"]  # bit for bit: the domain's arithmetic does not see its neighbours


def test_server_completes_stream_under_tight_budget():
    reqs = serving.make_requests(8, rate=0.0, seed=3, edge_range=(20, 36))
    # a budget that holds only a few of these domains at a time: admission has to wait
    summary, recs = serving.serve_batched(reqs, budget_gb=0.006, max_active=8, tol=TOL, closed_loop=True,
                                          prep_threads=4)
    assert summary["solves"] == 8
    assert sorted(r["id"] for r in recs) == list(range(8))
    # each result equals the request solved alone
    for r in recs[:3]:
        q = reqs[r["id"]]
        lat = _lat(q.seed, q.edge, q.porosity)
        alone = porous.solve_batched([lat], omegas=[q.omega], tol=TOL)[0]
        assert alone["k"] == r["k"] and alone["steps"] == r["steps"]


def _poisoned(field_of):
    """initial_field hook: equilibrium everywhere, NaN in one PDF of the first
    fluid cell of the requests in `field_of` (a host-side injection through
    SetNode-equivalent field upload; no device fault is involved)."""
    def init(req, lat):
        if req.id not in field_of:
            return None
        f = np.array(np.broadcast_to(lbmb200.W, (lat.mask.size, 19)))
        f[int(np.flatnonzero(lat.mask)[0]), 2] = np.nan
        return f
    return init


def test_diverged_request_retires_at_its_first_check():
    reqs = serving.make_requests(4, rate=0.0, seed=5, edge_range=(20, 32), omega_range=(0.8, 1.6))
    summary, recs = serving.serve_batched(reqs, max_active=4, tol=TOL, closed_loop=True, prep_threads=2,
                                          initial_field=_poisoned({1}))
    by_id = {r["id"]: r for r in recs}
    assert summary["solves"] == 4 and summary["status"].get("diverged") == 1
    bad = by_id[1]
    assert bad["status"] == "diverged" and bad["k"] is None and bad["steps"] == 100
    # the others are untouched by their poisoned neighbour: bit for bit their solo results
    for i in (0, 2, 3):
        q = reqs[i]
        alone = porous.solve_batched([_lat(q.seed, q.edge, q.porosity)], omegas=[q.omega], tol=TOL)[0]
        assert by_id[i]["status"] == alone["status"] == "converged"
        assert by_id[i]["k"] == alone["k"] and by_id[i]["steps"] == alone["steps"]


def test_fp64_solver_reports_divergence():
    lat = _lat(11, 24, 0.45)
    f = np.array(np.broadcast_to(lbmb200.W, (lat.mask.size, 19)))
    f[int(np.flatnonzero(lat.mask)[0]), 5] = np.inf
    res = porous.solve_fp64(lat, tol=TOL, initial_field=f)
    assert res["status"] == "diverged" and res["k"] is None and res["steps"] == 100
    ok = porous.solve_fp64(lat, tol=TOL)
    assert ok["status"] == "converged" and ok["k"] > 0


def test_sequential_fp64_server_statuses():
    reqs = serving.make_requests(3, rate=0.0, seed=9, edge_range=(20, 28), omega_range=(0.8, 1.6))
    summary, recs = serving.serve_fp64_sequential(reqs, tol=TOL, closed_loop=True, prep_threads=2,
                                                  initial_field=_poisoned({2}))
    by_id = {r["id"]: r for r in recs}
    assert summary["latency_samples"] == 3
    assert by_id[2]["status"] == "diverged" and by_id[0]["status"] == by_id[1]["status"] == "converged"
