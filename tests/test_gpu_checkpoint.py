"""Checkpoint / restart (lbm_b200_checkpoint_*, lbm_batch_checkpoint_*): a
run continued from a checkpoint equals the uninterrupted run bit for bit;
files of another lattice or kernel, and damaged files, are refused."""
import numpy as np
import pytest

import lbmb200
from lbm_cases import random_pdfs

pytestmark = pytest.mark.gpu

CASES = [("cuda-aa-soa", []), ("cuda-list-aa-pv-soa", []), ("cuda-list-pull-split-nt-1s-soa", []),
         ("cuda-list-aa-pv-soa", ["-precision", "fp32"]), ("cuda-list-aa-pv-soa", ["-precision", "fp16"])]


@pytest.mark.parametrize("kname,kargs", CASES)
def test_restart_continues_bit_for_bit(tmp_path, kname, kargs):
    lat = lbmb200.geometry("blocks-2", (14, 12, 10), (1, 0, 1))
    init = random_pdfs(lat.mask.size, 21, amp=0.02) if kargs else random_pdfs(lat.mask.size, 21)
    cd = lbmb200.case(omega=1.2, xforce=3e-5, iterations=10)
    a = lbmb200.kernel(kname).init(lat, kernel_args=["-lambda", "3/16"] + kargs)
    b = lbmb200.kernel(kname).init(lat, kernel_args=["-lambda", "3/16"] + kargs)
    try:
        a.set_field(init)
        a.run(cd)
        a.checkpoint(str(tmp_path / "s.ckpt"))
        a.run(cd)
        want = a.get_field()
        b.restore(str(tmp_path / "s.ckpt"))
        b.run(cd)
        got = b.get_field()
    finally:
        a.deinit()
        b.deinit()
    m = lat.mask != 0
    assert np.array_equal(got[m], want[m])


def test_mismatched_and_damaged_files_are_refused(tmp_path):
    lat = lbmb200.geometry("pipe", (12, 10, 11), (0, 0, 0))
    other = lbmb200.geometry("pipe", (12, 10, 12), (0, 0, 0))
    a = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat)
    b = lbmb200.kernel("cuda-list-aa-pv-soa").init(other)
    c = lbmb200.kernel("cuda-list-pull-split-nt-1s-soa").init(lat)
    try:
        a.run(lbmb200.case(iterations=4))
        path = tmp_path / "s.ckpt"
        a.checkpoint(str(path))
        before = a.get_field()
        for inst in (b, c):
            with pytest.raises(RuntimeError, match=r"\(-2\)"):
                inst.restore(str(path))
        data = bytearray(path.read_bytes())
        data[-5] ^= 0x40
        (tmp_path / "bad.ckpt").write_bytes(bytes(data))
        with pytest.raises(RuntimeError, match=r"\(-3\)"):
            a.restore(str(tmp_path / "bad.ckpt"))
        (tmp_path / "short.ckpt").write_bytes(bytes(data[: len(data) // 2]))
        with pytest.raises(RuntimeError, match=r"\(-1\)"):
            a.restore(str(tmp_path / "short.ckpt"))
        m = lat.mask != 0
        assert np.array_equal(a.get_field()[m], before[m])  # a refused file leaves the state alone
    finally:
        for inst in (a, b, c):
            inst.deinit()


def test_batch_domain_restart(tmp_path):
    lat, _ = lbmb200.spheres((24, 24, 24), 4, 0.5, 3.0, 6.0)
    other, _ = lbmb200.spheres((20, 20, 20), 5, 0.5, 3.0, 6.0)
    b = lbmb200.Batch("fp16", budget_gb=1.0, max_domains=4)
    try:
        s0 = b.add(lat, omega=1.1, xforce=2e-5)
        s1 = b.add(other, omega=0.9)
        b.step(20)
        b.checkpoint(s0, str(tmp_path / "d.ckpt"))
        b.step(20)
        b.sync()
        want = b.get_field(s0)
        b.remove(s0)
        s2 = b.add(lat, omega=1.1, xforce=2e-5)
        with pytest.raises(RuntimeError, match=r"\(-2\)"):
            b.restore(s1, str(tmp_path / "d.ckpt"))
        b.restore(s2, str(tmp_path / "d.ckpt"))
        b.step(20)
        b.sync()
        got = b.get_field(s2)
        m = lat.mask != 0
        assert np.array_equal(got[m], want[m])
    finally:
        b.close()


def test_checkpoint_of_another_geometry_with_equal_counts_is_refused(tmp_path):
    # two masks with the same dimensions, periodicity and fluid count that
    # differ in where one obstacle cell sits: the lattice hash tells them apart
    dims = (10, 8, 9)
    m1 = np.ones(int(np.prod(dims)), dtype=np.int32)
    m2 = m1.copy()
    m1[123] = 0
    m2[321] = 0
    a = lbmb200.kernel("cuda-list-aa-pv-soa").init(lbmb200.Lattice(m1, dims, (1, 1, 1)))
    b = lbmb200.kernel("cuda-list-aa-pv-soa").init(lbmb200.Lattice(m2, dims, (1, 1, 1)))
    try:
        a.run(lbmb200.case(iterations=2))
        a.checkpoint(str(tmp_path / "a.ckpt"))
        with pytest.raises(RuntimeError, match=r"\(-2\)"):
            b.restore(str(tmp_path / "a.ckpt"))
        a.restore(str(tmp_path / "a.ckpt"))  # its own file still loads
    finally:
        a.deinit()
        b.deinit()


def test_lost_device_state_is_refused_until_a_state_is_uploaded():
    # the error word a bounded wait sets when it gives up, written from the
    # host (no kernel faults): steps, downloads and checkpoints refuse until
    # set_field uploads a state again
    import ctypes
    L = lbmb200.lib()
    lat = lbmb200.geometry("blocks-2", (14, 12, 10), (1, 0, 1))
    init = random_pdfs(lat.mask.size, 31)
    cd = lbmb200.case(omega=1.2, xforce=3e-5, iterations=4)
    inst = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=["-lambda", "3/16"])
    ref = lbmb200.kernel("cuda-list-aa-pv-soa").init(lat, kernel_args=["-lambda", "3/16"])
    try:
        inst.set_field(init)
        inst.step_device(cd, 4)
        inst.sync_mirror()
        good = inst.get_field()
        assert L.lbm_b200_inject_device_error(inst.kdp, 1) == 0
        assert L.lbm_b200_sync_mirror(inst.kdp) == -4
        m = lat.mask != 0
        assert np.array_equal(inst.get_field()[m], good[m])  # the mirror keeps the last good state
        assert L.lbm_b200_step_device(inst.kdp, ctypes.byref(cd), 2) == -4
        tot = ctypes.c_double(0.0)
        assert L.lbm_b200_time_steps(inst.kdp, ctypes.byref(cd), 2, ctypes.byref(tot), None) == -4
        out = (ctypes.c_double * 4)()
        assert L.lbm_b200_instance_moments(inst.kdp, out) == -4
        # a state upload clears it: the run continues exactly as a clean instance
        inst.set_field(init)
        inst.step_device(cd, 4)
        inst.sync_mirror()
        ref.set_field(init)
        ref.step_device(cd, 4)
        ref.sync_mirror()
        assert np.array_equal(inst.get_field()[m], ref.get_field()[m])
    finally:
        inst.deinit()
        ref.deinit()
