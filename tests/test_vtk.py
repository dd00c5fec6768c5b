"""The legacy VTK writer of the CUDA rows (lbm_vtk_write_file, host C):
file format and contents against the reference's own VtkWrite
(src/Vtk.c:51-245, built with VTK_OUTPUT into oracle/_ref/lbmbenchk-vtk), fed
with oracle states. No GPU needed."""
import os
import struct
import subprocess

import numpy as np
import pytest

import lbmb200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_VTK = os.path.join(ROOT, "oracle", "_ref", "lbmbenchk-vtk")

DIMS, GEO, ITERS, MOD = (10, 9, 8), "blocks-2", 6, 2


def parse_vtk(path):
    """(header lines, flags u8, density f64, velocity f64 (n, 3)) of a binary
    legacy VTK file in the reference's layout."""
    data = open(path, "rb").read()
    lines, pos = [], 0
    for _ in range(10):
        end = data.index(b"\n", pos)
        lines.append(data[pos:end].decode())
        pos = end + 1
    nx, ny, nz = (int(v) for v in lines[4].split()[1:])
    n = nx * ny * nz
    flags = np.frombuffer(data, np.uint8, n, pos)
    pos += n
    for tag in (b"SCALARS Density double\n", b"LOOKUP_TABLE default\n"):
        assert data[pos:pos + len(tag)] == tag
        pos += len(tag)
    rho = np.frombuffer(data, ">f8", n, pos).astype(np.float64)
    pos += 8 * n
    tag = b"VECTORS VelocityVectors double\n"
    assert data[pos:pos + len(tag)] == tag
    pos += len(tag)
    u = np.frombuffer(data, ">f8", 3 * n, pos).astype(np.float64).reshape(n, 3)
    assert pos + 24 * n == len(data)
    return lines, flags, rho, u


def expected_moments(field, mask, xforce):
    """Density and velocity per cell, summed in the reference's order."""
    n = mask.size
    rho, u = np.zeros(n), np.zeros((n, 3))
    E, W, N, S, T, B = 2, 3, 0, 1, 8, 13
    NE, SE, NW, SW, TN, TE, TW, TS, BS, BN, BW, BE = 4, 5, 6, 7, 9, 10, 11, 12, 14, 15, 16, 17
    for c in np.flatnonzero(mask != 0):
        p = [float(v) for v in field[c]]
        r = 0.0
        for v in p:
            r += v
        ux = p[E] + p[NE] + p[SE] + p[TE] + p[BE] - p[W] - p[NW] - p[SW] - p[TW] - p[BW]
        uy = p[N] + p[NE] + p[NW] + p[TN] + p[BN] - p[S] - p[SE] - p[SW] - p[TS] - p[BS]
        uz = p[T] + p[TE] + p[TW] + p[TN] + p[TS] - p[B] - p[BE] - p[BW] - p[BN] - p[BS]
        rho[c], u[c] = r, (ux + 0.5 * xforce, uy, uz)
    return rho, u


def test_writer_contents_and_layout(tmp_path, oracle):
    lat = lbmb200.geometry(GEO, DIMS, (0, 0, 0))
    f = oracle.run("list-aa", DIMS, lat.periodic, lat.mask, xforce=1e-5, iterations=4, init="zero")
    path = str(tmp_path / "a.vtk")
    lbmb200.write_vtk_field(lat, f, 1e-5, 4, path)
    lines, flags, rho, u = parse_vtk(path)
    assert lines[1] == "Comment: lid driven cavity, iteration    4"
    assert lines[2:5] == ["BINARY", "DATASET STRUCTURED_POINTS", "DIMENSIONS 10 9 8"]
    assert np.array_equal(flags, lat.mask.astype(np.uint8))
    er, eu = expected_moments(f, lat.mask, 1e-5)
    assert np.array_equal(rho, er) and np.array_equal(u, eu)


def _reference_files(tmp_path, rkernel):
    if not os.path.exists(REF_VTK):
        pytest.skip("reference VTK build oracle/_ref/lbmbenchk-vtk not present")
    d = tmp_path / rkernel
    d.mkdir()
    subprocess.run([REF_VTK, "-dims", "x".join(map(str, DIMS)), "-geometry", GEO, "-iterations", str(ITERS),
                    "-vtk", str(MOD), "-kernel", rkernel, "-t", "1"], cwd=d, check=True, capture_output=True)
    return {int(name[5:-4]): str(d / "vtk" / name) for name in os.listdir(d / "vtk")}


# label -> steps done, per the reference's loops (AA: in-loop dumps follow the
# even step only, so just the first and the last are compared)
SCHEDULES = {
    "list-aa-pv-soa": ("list-aa", {-1: 0, 0: 2, 2: 4, 4: 6, 6: 6}),
    "list-pull-split-nt-1s-soa": ("list-pull", {-1: 0, 0: 1, 2: 3, 4: 5, 6: 6}),
    "aa-soa": ("aa", {-1: 0, 6: 6}),
}


@pytest.mark.parametrize("rkernel", list(SCHEDULES))
def test_writer_matches_reference_vtk_files(tmp_path, oracle, rkernel):
    okernel, sched = SCHEDULES[rkernel]
    files = _reference_files(tmp_path, rkernel)
    assert set(files) == {-1, 0, 2, 4, 6}
    lat = lbmb200.geometry(GEO, DIMS, (0, 0, 0))
    for label, steps in sched.items():
        f = oracle.run(okernel, DIMS, lat.periodic, lat.mask, xforce=1e-5, iterations=steps, init="zero")
        ours = str(tmp_path / ("ours_%d.vtk" % label))
        lbmb200.write_vtk_field(lat, f, 1e-5, label, ours)
        ref = files[label]
        if rkernel == "aa-soa" or steps == 0:
            # the scalar AA kernel and the zero start are bit-identical states
            assert open(ours, "rb").read() == open(ref, "rb").read()
        else:
            # the reference's SIMD list loops round differently (<= 1e-13)
            lo, fo, ro, uo = parse_vtk(ours)
            lr, fr, rr, ur = parse_vtk(ref)
            assert lo == lr and np.array_equal(fo, fr)
            assert np.allclose(ro, rr, rtol=1e-13, atol=1e-20)
            assert np.allclose(uo, ur, rtol=1e-11, atol=1e-17)
