"""Batched domains: one persistent launch per step over many independent
porous domains (lbm_batch_*), against the single-domain reduced-storage list
AA kernel, alone versus in a mix, graph replay versus direct launches."""
import numpy as np
import pytest

import lbmb200
from lbm_cases import CX, CY, CZ, random_pdfs

pytestmark = pytest.mark.gpu


def _domains(n, seed0=100):
    rng = np.random.default_rng(seed0)
    out = []
    for i in range(n):
        edge = int(rng.integers(16, 41))
        por = float(rng.uniform(0.35, 0.6))
        lat, _ = lbmb200.spheres((edge, edge, edge), seed0 + i, por, 3.0, 8.0)
        out.append((lat, float(rng.uniform(0.8, 1.6))))
    return out


def _single(lat, omega, init, steps, prec):
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=["-precision", prec, "-lambda", "3/16"])
    try:
        inst.set_field(init)
        inst.run(lbmb200.case(omega=omega, xforce=2e-5, iterations=steps))
        return inst.get_field()
    finally:
        inst.deinit()


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_batch_matches_single_domain_kernel(prec):
    doms = _domains(5)
    b = lbmb200.Batch(prec, budget_gb=4.0, max_domains=16)
    try:
        slots, inits = [], []
        for k, (lat, om) in enumerate(doms):
            s = b.add(lat, omega=om, lam=3.0 / 16.0, xforce=2e-5)
            assert s >= 0
            init = random_pdfs(lat.mask.size, 40 + k, amp=0.02)
            b.set_field(s, init)
            slots.append(s)
            inits.append(init)
        b.step(24, graph=True)
        b.sync()
        for s, (lat, om), init in zip(slots, doms, inits):
            got = b.get_field(s)
            want = _single(lat, om, init, 24, prec)
            m = lat.mask != 0
            # the single-domain kernels relax pairs on packed FP32x2
            # instructions, the batched ones pair by pair: the two agree to
            # FP32 rounding, carried through the storage format (one FP16
            # rounding step can flip; each stays within 1e-7 / 5e-5 of FP64)
            assert np.max(np.abs(got[m] - want[m])) <= (1e-6 if prec == "fp32" else 5e-5)
    finally:
        b.close()


def test_domain_alone_equals_domain_in_mix():
    doms = _domains(6, seed0=300)
    lat0, om0 = doms[0]
    init0 = random_pdfs(lat0.mask.size, 7, amp=0.02)
    alone = lbmb200.Batch("fp32", budget_gb=4.0, max_domains=8)
    mix = lbmb200.Batch("fp32", budget_gb=4.0, max_domains=8)
    try:
        s = alone.add(lat0, omega=om0)
        alone.set_field(s, init0)
        # in the mix the domain is admitted third, after others, into a different slot and tile range
        for lat, om in doms[1:3]:
            mix.add(lat, omega=om)
        sm = mix.add(lat0, omega=om0)
        mix.set_field(sm, init0)
        for lat, om in doms[3:]:
            mix.add(lat, omega=om)
        alone.step(40)
        mix.step(40)
        alone.sync()
        mix.sync()
        a, m_ = alone.get_field(s), mix.get_field(sm)
        mask = lat0.mask != 0
        assert np.array_equal(a[mask], m_[mask])
        ma, mm = alone.moments()[s], mix.moments()[sm]
        assert np.array_equal(ma, mm)
    finally:
        alone.close()
        mix.close()


def test_graph_replay_equals_direct_launches_and_survives_membership_changes():
    doms = _domains(4, seed0=500)
    g = lbmb200.Batch("fp32", budget_gb=4.0, max_domains=8)
    d = lbmb200.Batch("fp32", budget_gb=4.0, max_domains=8)
    try:
        sg = [g.add(lat, omega=om) for lat, om in doms[:3]]
        sd = [d.add(lat, omega=om) for lat, om in doms[:3]]
        g.step(20, graph=True)
        d.step(20, graph=False)
        # admit a fourth domain and retire the first: the captured graph is reused
        g.add(doms[3][0], omega=doms[3][1])
        d.add(doms[3][0], omega=doms[3][1])
        g.remove(sg[0])
        d.remove(sd[0])
        g.step(20, graph=True)
        d.step(20, graph=False)
        g.sync()
        d.sync()
        for a, b_ in zip(sg[1:], sd[1:]):
            assert np.array_equal(g.get_field(a), d.get_field(b_), equal_nan=True)
    finally:
        g.close()
        d.close()


def test_batch_moments_match_host_sums():
    doms = _domains(3, seed0=700)
    b = lbmb200.Batch("fp32", budget_gb=4.0, max_domains=4)
    try:
        slots = [b.add(lat, omega=om, xforce=1e-4) for lat, om in doms]
        b.step(30)
        mom = b.moments()
        # FP32 storage holds the deviations delta_i = f_i - w_i; the device
        # sums them in FP64 and reports rho = 1 + sum(delta) per node
        for s, (lat, _) in zip(slots, doms):
            f = b.get_field(s)[lat.mask != 0]
            dlt = f - lbmb200.W[None, :]
            want = [lat.n_fluid + dlt.sum(), (dlt * CX).sum(), (dlt * CY).sum(), (dlt * CZ).sum()]
            assert abs(mom[s][0] - want[0]) / want[0] < 1e-12
            assert np.all(np.abs(mom[s][1:] - want[1:]) < 1e-12 * want[0])
            assert mom[s][1] > 0  # the force drives +x flow
    finally:
        b.close()


def test_admission_respects_hbm_budget_and_slot_reuse():
    lat, _ = lbmb200.spheres((32, 32, 32), 9, 0.5, 3.0, 8.0)
    b = lbmb200.Batch("fp32", budget_gb=0.004, max_domains=4)  # room for about one 32^3 domain
    try:
        s0 = b.add(lat)
        assert s0 >= 0
        assert b.add(lat) == -1  # over budget
        used = b.bytes_used
        assert used > 0
        assert b.remove(s0) == 0
        assert b.bytes_used == 0
        s1 = b.add(lat)
        assert s1 == s0
        f = b.get_field(s1)[lat.mask != 0]
        assert np.array_equal(f, np.broadcast_to(lbmb200.W, f.shape))  # a re-admitted slot starts at rest
    finally:
        b.close()


def test_autotuner_picks_a_candidate():
    doms = _domains(3, seed0=900)
    b = lbmb200.Batch("fp32", budget_gb=4.0, max_domains=4)
    try:
        for lat, om in doms:
            b.add(lat, omega=om)
        rows = b.tune(trial_steps=4)
        assert len(rows) >= 10
        cfg = b.launch()
        for which in ("even", "odd"):
            c = cfg[which]
            assert c["threads"] in (64, 128, 256) and c["threads"] * c["nodes_per_thread"] == 256
        b.step(10)
        b.sync()
    finally:
        b.close()
