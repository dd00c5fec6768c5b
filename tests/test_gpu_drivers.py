"""The drop-in boundary exercised end to end through command-line drivers:

* oracle/_ref/lbmbenchk-cuda: the reference's own main() (src/Main.c:537-643:
  kernel lookup by name, Init, -verify initialisation through SetNode,
  kd->Kernel, KernelVerifiy through GetNode, the P: line, Deinit) with the
  CUDA rows added to its kernel table as INTEGRATION.md shows, linked against
  liblbmb200.so (oracle/Makefile target `cuda`);
* lbm-benchmark-kernels_b200/bin/lbmbenchk-b200: this repository's own driver
  with the reference's flags.

The -verify preset (16^3 box, periodic x/y, walls in z, omega 1, F = 1e-5,
1000 steps, src/Main.c:232-265) has the known answers 4.561374e-02 at
Lambda = 1/12 and 7.855978e-02 at Lambda = 3/16 (the reference build's own
output)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_CUDA = os.path.join(ROOT, "oracle", "_ref", "lbmbenchk-cuda")
OWN = os.path.join(ROOT, "lbm-benchmark-kernels_b200", "bin", "lbmbenchk-b200")
CUDA_ROWS = ["cuda-aa-soa", "cuda-list-aa-pv-soa", "cuda-list-pull-split-nt-1s-soa",
             "cuda-list-pull-split-nt-2s-soa", "cuda-list-aa-soa", "cuda-list-aa-ria-soa", "cuda-list-push-soa",
             "cuda-list-pull-soa", "cuda-push-soa", "cuda-pull-soa"]
P_LINE = re.compile(r"^P:\s+([0-9.]+) MFLUP/s\s+t: (\d+)\s+d: ([0-9.]+) s\s+iter: (\d+)\s+fnodes: ([0-9.]+) x1e6\s+"
                    r"geo: (\S+)\s+kernel: (\S+)\s+(VERIFICATION|B)\s+dp$", re.M)


def _need(path):
    if not os.path.exists(path):
        pytest.skip("%s is not built" % os.path.relpath(path, ROOT))


def _run(cmd, cwd):
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, timeout=600)
    return r.returncode, r.stdout


def test_reference_driver_lists_cuda_rows(tmp_path):
    # -list returns before any kernel runs: no GPU is touched
    _need(REF_CUDA)
    rc, out = _run([REF_CUDA, "-list"], str(tmp_path))
    listed = [ln.strip() for ln in out.splitlines() if ln.startswith("   ")]
    assert "list-aa-pv-soa" in listed and "aa-soa" in listed  # the reference's own rows stay
    for name in CUDA_ROWS:
        assert name in listed, name


@pytest.mark.gpu
@pytest.mark.parametrize("kname", CUDA_ROWS)
@pytest.mark.parametrize("lam,expect", [("1/12", "4.561374e-02"), ("3/16", "7.855978e-02")])
def test_reference_driver_verify(tmp_path, kname, lam, expect):
    _need(REF_CUDA)
    rc, out = _run([REF_CUDA, "-verify", "-kernel", kname, "--", "-lambda", lam], str(tmp_path))
    assert rc == 0, out[-2000:]
    assert "# VERIFICATION: deviation from analytical solution: %s" % expect in out, out[-2000:]
    assert "# VERIFICATION SUCCEEDED." in out
    m = P_LINE.search(out)
    assert m and m.group(7) == kname and m.group(8) == "VERIFICATION" and int(m.group(4)) == 1000, out[-1000:]
    assert float(m.group(1)) > 0.0


@pytest.mark.gpu
def test_reference_driver_channel_run(tmp_path):
    # a plain benchmark-style run through the reference's main(): the P: line
    # reports the fluid nodes of the reference's own channel geometry
    _need(REF_CUDA)
    rc, out = _run([REF_CUDA, "-dims", "40x24x20", "-geometry", "channel", "-periodic-x", "-iterations", "20",
                    "-kernel", "cuda-list-aa-pv-soa", "--", "-lambda", "3/16"], str(tmp_path))
    assert rc == 0, out[-2000:]
    m = P_LINE.search(out)
    assert m and m.group(6) == "channel" and m.group(7) == "cuda-list-aa-pv-soa"
    assert abs(float(m.group(5)) - 40 * 22 * 18 / 1e6) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("kname", ["cuda-aa-soa", "cuda-list-aa-pv-soa", "cuda-list-pull-split-nt-2s-soa"])
def test_own_driver_verify_and_p_line(tmp_path, kname):
    _need(OWN)
    rc, out = _run([OWN, "-verify", "-kernel", kname, "--", "-lambda", "3/16"], str(tmp_path))
    assert rc == 0, out[-2000:]
    assert "# VERIFICATION: deviation from analytical solution: 7.855978e-02" in out
    m = P_LINE.search(out)
    assert m and m.group(6) == "box" and m.group(7) == kname and m.group(8) == "VERIFICATION"
    assert int(m.group(4)) == 1000 and abs(float(m.group(5)) - 16 * 16 * 14 / 1e6) < 1e-6
    assert float(m.group(1)) > 0.0


def test_own_driver_lists_rows(tmp_path):
    _need(OWN)
    rc, out = _run([OWN, "-list"], str(tmp_path))
    assert rc == 0
    listed = [ln.strip() for ln in out.splitlines() if ln.startswith("   ")]
    assert listed == CUDA_ROWS
