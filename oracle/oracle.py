"""ctypes wrappers for the oracle -- TEST INFRASTRUCTURE ONLY.

Two checkers live here:

* ``Oracle``: the plain-C restatement of the reference's D3Q19 TRT path
  (oracle/lbm_oracle.c, built into oracle/_build/liblbmoracle.so).
* ``Reference``: the reference implementation itself, compiled from its own
  sources by oracle/Makefile into oracle/_ref/libreflbm-<variant>.so and driven
  through its own kernel table by oracle/ref_harness.c.

Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() import this
module, and only to check or time against the product; the product never does.

Arrays are numpy arrays with the reference's lattice order: cell index
``z*nX*nY + y*nX + x`` (x fastest) and, for PDF fields, 19 doubles per cell in
the reference's direction order N,S,E,W,NE,SE,NW,SW,T,TN,TE,TW,TS,B,BS,BN,BW,BE,C.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

GEO = {"box": 0, "channel": 1, "pipe": 2, "blocks": 3, "fluid": 4}
KERNEL = {"aa": 0, "list-aa": 1, "list-pull": 2, "list-push2": 3, "list-pull2": 4, "push-fa": 5, "pull-fa": 6}

_i3 = ctypes.c_int * 3


def _p(a, t):
    return a.ctypes.data_as(ctypes.POINTER(t)) if a is not None else None


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


class Oracle:
    def __init__(self):
        path = os.path.join(BUILD, "liblbmoracle.so")
        if not os.path.exists(path):
            build_oracle()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.orc_run.restype = ctypes.c_int
        L.orc_verify_error.restype = ctypes.c_double

    def geometry(self, name, dims, periodic=(0, 0, 0)):
        """Returns (mask int32[nZ,nY,nX] flattened x-fastest, info dict)."""
        base = name.split("-")[0]
        bs = 8
        if base == "blocks" and len(name) > 7:
            bs = int(name[7:])
        lat = np.zeros(int(np.prod(dims)), dtype=np.int32)
        info = np.zeros(8, dtype=np.int32)
        self.lib.orc_geometry(GEO[base], bs, _i3(*dims), _i3(*periodic),
                              _p(lat, ctypes.c_int), _p(info, ctypes.c_int))
        return lat, _info(info)

    def pad_cells(self, n, pad_mode=0):
        return self.lib.orc_pad_cells(n, 8, pad_mode, 0, None, None)

    def list_layout(self, pull, dims, periodic, lat, blk=(0, 0, 0), pad_mode=0):
        nf = int(np.count_nonzero(lat))
        grid = np.zeros(lat.size, dtype=np.uint32)
        adj = np.zeros(max(nf, 1) * 18, dtype=np.uint32)
        counts = np.zeros(2, dtype=np.int32)
        rc = self.lib.orc_list_layout(int(pull), _i3(*dims), _i3(*periodic), _p(lat, ctypes.c_int),
                                      _i3(*blk), pad_mode, 0, None, None,
                                      _p(grid, ctypes.c_uint32), _p(adj, ctypes.c_uint32),
                                      _p(counts, ctypes.c_int))
        assert rc == 0
        return grid, adj[: nf * 18], int(counts[0]), int(counts[1])

    def run(self, kernel, dims, periodic, lat, omega=1.0, lam=1.0 / 12.0, xforce=1e-5,
            rho_in=1.0, rho_out=1.0, iterations=10, init="verify", init_pdfs=None,
            blk=(0, 0, 0), pad_mode=0):
        out = np.full(lat.size * 19, np.nan)
        mode = {"zero": 0, "verify": 1, "pdfs": 2}[init]
        if init_pdfs is not None:
            init_pdfs = np.ascontiguousarray(init_pdfs, dtype=np.float64).reshape(-1)
        rc = self.lib.orc_run(KERNEL[kernel], _i3(*dims), _i3(*periodic), _p(lat, ctypes.c_int),
                              ctypes.c_double(omega), ctypes.c_double(lam), ctypes.c_double(xforce),
                              ctypes.c_double(rho_in), ctypes.c_double(rho_out), iterations, mode,
                              _p(init_pdfs, ctypes.c_double), _p(out, ctypes.c_double),
                              _i3(*blk), pad_mode)
        assert rc == 0
        return out.reshape(-1, 19)

    def list_aa_half(self, odd, n_nodes, n_cells, adj, f, omega=1.0, lam=1.0 / 12.0, xforce=1e-5):
        """One half of a list AA step pair in place on f (float64, 19 *
        n_cells) through adj (uint32, n_nodes * 18): orc_list_aa_half."""
        assert f.dtype == np.float64 and f.flags.c_contiguous and f.size >= 19 * n_cells
        adj = np.ascontiguousarray(adj, dtype=np.uint32)
        rc = self.lib.orc_list_aa_half(int(odd), int(n_nodes), int(n_cells), _p(adj, ctypes.c_uint32),
                                       _p(f, ctypes.c_double), ctypes.c_double(omega), ctypes.c_double(lam),
                                       ctypes.c_double(xforce))
        assert rc == 0

    def list_aa_half_range(self, odd, n0, n1, n_cells, adj, f, omega=1.0, lam=1.0 / 12.0, xforce=1e-5):
        """list_aa_half over nodes [n0, n1) only: orc_list_aa_half_range."""
        assert f.dtype == np.float64 and f.flags.c_contiguous and f.size >= 19 * n_cells
        adj = np.ascontiguousarray(adj, dtype=np.uint32)
        rc = self.lib.orc_list_aa_half_range(int(odd), int(n0), int(n1), int(n_cells), _p(adj, ctypes.c_uint32),
                                             _p(f, ctypes.c_double), ctypes.c_double(omega), ctypes.c_double(lam),
                                             ctypes.c_double(xforce))
        assert rc == 0

    def verify_error(self, dims, lat, pdfs, omega=1.0, xforce=1e-5):
        pdfs = np.ascontiguousarray(pdfs, dtype=np.float64).reshape(-1)
        return self.lib.orc_verify_error(_i3(*dims), _p(lat, ctypes.c_int), _p(pdfs, ctypes.c_double),
                                         ctypes.c_double(omega), ctypes.c_double(xforce))


def _info(info):
    return {"nFluid": int(info[0]), "nObst": int(info[1]), "nInlet": int(info[2]),
            "nOutlet": int(info[3]), "ldPeriodic": tuple(int(v) for v in info[4:7]),
            "geoPeriodicBits": int(info[7])}


def reference_available(variant="verify"):
    return os.path.exists(os.path.join(REF, "libreflbm-%s.so" % variant))


def reference_binary(variant):
    return os.path.join(REF, "lbmbenchk-%s" % variant)


class Reference:
    """The reference's own kernels (oracle/_ref), through oracle/ref_harness.c."""

    def __init__(self, variant="verify"):
        self.lib = ctypes.CDLL(os.path.join(REF, "libreflbm-%s.so" % variant))
        self.lib.refh_kernel_name.restype = ctypes.c_char_p

    def set_threads(self, n):
        return self.lib.refh_set_threads(int(n))

    def pin(self, cpus):
        """Pins the OpenMP threads to `cpus` (thread i to cpus[i]) with the
        reference's own pinning code; returns the number of failures."""
        return self.lib.refh_pin(",".join(str(int(c)) for c in cpus).encode())

    def kernels(self):
        return [self.lib.refh_kernel_name(i).decode() for i in range(self.lib.refh_kernel_count())]

    def geometry(self, name, dims, periodic=(0, 0, 0)):
        lat = np.zeros(int(np.prod(dims)), dtype=np.int32)
        info = np.zeros(8, dtype=np.int32)
        self.lib.refh_geometry(name.encode(), _i3(*dims), _i3(*periodic), _p(lat, ctypes.c_int),
                               _p(info, ctypes.c_int))
        return lat, _info(info)

    @staticmethod
    def _kargs(kargs):
        kargs = list(kargs or [])
        arr = (ctypes.c_char_p * max(1, len(kargs)))(*[k.encode() for k in kargs])
        return len(kargs), arr

    def run(self, kernel, dims, periodic, lat, omega=1.0, xforce=1e-5, rho_in=1.0, rho_out=1.0,
            iterations=10, init="verify", init_pdfs=None, kargs=None, want_pdfs=True):
        lat = np.ascontiguousarray(lat, dtype=np.int32)
        out = np.full(lat.size * 19, np.nan) if want_pdfs else None
        mode = {"zero": 0, "verify": 1, "pdfs": 2}[init]
        if init_pdfs is not None:
            init_pdfs = np.ascontiguousarray(init_pdfs, dtype=np.float64).reshape(-1)
        nk, ka = self._kargs(kargs)
        dur = ctypes.c_double(0.0)
        rc = self.lib.refh_run(kernel.encode(), _i3(*dims), _i3(*periodic), _p(lat, ctypes.c_int),
                               ctypes.c_double(omega), ctypes.c_double(xforce), ctypes.c_double(rho_in),
                               ctypes.c_double(rho_out), iterations, mode,
                               _p(init_pdfs, ctypes.c_double), _p(out, ctypes.c_double), nk, ka,
                               ctypes.byref(dur))
        assert rc == 0, "unknown reference kernel %s" % kernel
        self.last_duration = dur.value
        return out.reshape(-1, 19) if want_pdfs else None

    def list_layout(self, kernel, dims, periodic, lat, kargs=None):
        lat = np.ascontiguousarray(lat, dtype=np.int32)
        nf = int(np.count_nonzero(lat))
        grid = np.zeros(lat.size, dtype=np.uint32)
        adj = np.zeros(max(nf, 1) * 18, dtype=np.uint32)
        counts = np.zeros(2, dtype=np.int32)
        nk, ka = self._kargs(kargs)
        rc = self.lib.refh_list_layout(kernel.encode(), _i3(*dims), _i3(*periodic), _p(lat, ctypes.c_int),
                                       nk, ka, _p(grid, ctypes.c_uint32), _p(adj, ctypes.c_uint32),
                                       _p(counts, ctypes.c_int))
        assert rc == 0
        return grid, adj[: nf * 18], int(counts[0]), int(counts[1])
