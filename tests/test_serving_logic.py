"""Host logic of the permeability solves and the server (no GPU): the
stopping rule with its three outcomes, the request stream, the summary."""
import math

from lbmb200 import porous, serving


def test_stop_status():
    assert porous.stop_status(1.0, None, 100, 1e-6, 20000) is None
    assert porous.stop_status(1.0, 1.0 + 1e-7, 200, 1e-6, 20000) == porous.CONVERGED
    assert porous.stop_status(1.0, 1.1, 200, 1e-6, 20000) is None
    assert porous.stop_status(1.0, 1.1, 20000, 1e-6, 20000) == porous.NOT_CONVERGED
    # a non-finite mean velocity retires the solve at once, before the cap
    for u in (math.nan, math.inf, -math.inf):
        assert porous.stop_status(u, 1.0, 100, 1e-6, 20000) == porous.DIVERGED
        assert porous.stop_status(u, None, 100, 1e-6, 20000) == porous.DIVERGED


def test_requests_draw_omega_from_the_range():
    reqs = serving.make_requests(200, rate=5.0, seed=1, omega_range=(0.8, 1.6))
    om = [r.omega for r in reqs]
    assert min(om) >= 0.8 and max(om) <= 1.6 and max(om) - min(om) > 0.6
    assert all(b.arrival >= a.arrival for a, b in zip(reqs, reqs[1:]))
    assert all(32 <= r.edge <= 192 for r in reqs)


def test_summary_counts_statuses_and_samples():
    recs = [{"arrival": 0.0, "done": 1.0 + i, "steps": 100 * (i + 1), "status": s}
            for i, s in enumerate(["converged", "diverged", "converged", "not_converged"])]
    s = serving._summary(recs, 8.0)
    assert s["solves"] == 4 and s["latency_samples"] == 4 and s["solves_per_s"] == 0.5
    assert s["status"] == {"converged": 2, "diverged": 1, "not_converged": 1}
