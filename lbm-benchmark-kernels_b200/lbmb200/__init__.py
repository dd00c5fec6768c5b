"""Python mirror of the reference benchmark's kernel-table API over the B200
C ABI (include/lbm_b200.h, liblbmb200.so).

The flow is the one src/Main.c follows::

    ld = geometry("box", (16, 16, 16), periodic=(1, 1, 0))     # GeoCreateByStr
    kf = kernel("cuda-aa-soa")                                  # g_kernels lookup
    kd = kf.init(ld, kernel_args=["-lambda", "3/16"])           # kf->Init
    kd.set_initial_density(cd); kd.set_initial_velocity(cd)     # -verify init
    kd.run(cd)                                                  # kd->Kernel
    err = kd.verify(cd)                                         # KernelVerifiy
    kd.deinit()                                                 # kf->Deinit

Kernel names follow the reference's (src/KernelFunctions.h:56-188) with a
"cuda-" prefix; lookups are case-insensitive as in src/Main.c:543. There is no
CPU fallback: loading fails loudly when the library is missing, and running a
kernel without a GPU fails in the CUDA runtime.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "liblbmb200.so")

Q = 19
W = np.array([1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4 + [1 / 3])


class LatticeDesc(ctypes.Structure):
    _fields_ = [("Dims", ctypes.c_int * 3), ("Lattice", ctypes.POINTER(ctypes.c_int)),
                ("nCells", ctypes.c_int), ("nFluid", ctypes.c_int), ("nObst", ctypes.c_int),
                ("nInlet", ctypes.c_int), ("nOutlet", ctypes.c_int), ("PeriodicX", ctypes.c_int),
                ("PeriodicY", ctypes.c_int), ("PeriodicZ", ctypes.c_int), ("Name", ctypes.c_char_p)]


class CaseData(ctypes.Structure):
    _fields_ = [("Omega", ctypes.c_double), ("RhoIn", ctypes.c_double), ("RhoOut", ctypes.c_double),
                ("Ux", ctypes.c_double), ("Uy", ctypes.c_double), ("Uz", ctypes.c_double),
                ("XForce", ctypes.c_double), ("MaxIterations", ctypes.c_int), ("VtkOutput", ctypes.c_int),
                ("VtkModulus", ctypes.c_int), ("StatisticsModulus", ctypes.c_int)]


class KernelData(ctypes.Structure):
    pass


_GETNODE = ctypes.CFUNCTYPE(None, ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            ctypes.POINTER(ctypes.c_double))
_KERNEL = ctypes.CFUNCTYPE(None, ctypes.POINTER(LatticeDesc), ctypes.POINTER(KernelData),
                           ctypes.POINTER(CaseData))
_BCGET = ctypes.CFUNCTYPE(None, ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.POINTER(ctypes.c_double))
_BCSET = ctypes.CFUNCTYPE(None, ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                          ctypes.c_int, ctypes.c_double)

KernelData._fields_ = [
    ("Pdfs", ctypes.POINTER(ctypes.c_double) * 2), ("SrcPdfs", ctypes.POINTER(ctypes.c_double)),
    ("DstPdfs", ctypes.POINTER(ctypes.c_double)), ("PdfsActive", ctypes.POINTER(ctypes.c_double)),
    ("Dims", ctypes.c_int * 3), ("GlobalDims", ctypes.c_int * 3), ("Offsets", ctypes.c_int * 3),
    ("ObstIndices", ctypes.POINTER(ctypes.c_int)), ("nObstIndices", ctypes.c_int),
    ("BounceBackPdfsSrc", ctypes.POINTER(ctypes.c_int)), ("BounceBackPdfsDst", ctypes.POINTER(ctypes.c_int)),
    ("nBounceBackPdfs", ctypes.c_int), ("LoopBalance", ctypes.c_double), ("Duration", ctypes.c_double),
    ("BoundaryConditionsGetPdf", _BCGET), ("BoundaryConditionsSetPdf", _BCSET),
    ("GetNode", _GETNODE), ("SetNode", _GETNODE), ("Kernel", _KERNEL)]


class Parameters(ctypes.Structure):
    _fields_ = [("nArgs", ctypes.c_int), ("Args", ctypes.POINTER(ctypes.c_char_p)),
                ("nKernelArgs", ctypes.c_int), ("KernelArgs", ctypes.POINTER(ctypes.c_char_p))]


_INIT = ctypes.CFUNCTYPE(None, ctypes.POINTER(LatticeDesc), ctypes.POINTER(ctypes.POINTER(KernelData)),
                         ctypes.POINTER(Parameters))
_DEINIT = ctypes.CFUNCTYPE(None, ctypes.POINTER(LatticeDesc), ctypes.POINTER(ctypes.POINTER(KernelData)))


class _KF(ctypes.Structure):
    _fields_ = [("Name", ctypes.c_char * 128), ("Init", _INIT), ("Deinit", _DEINIT)]


_lib = None


def lib():
    """The loaded liblbmb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("liblbmb200.so is not built (run: make -C lbm-benchmark-kernels_b200)")
        L = ctypes.CDLL(LIB_PATH)
        L.lbm_b200_kernels.restype = ctypes.POINTER(_KF)
        L.lbm_b200_kernels.argtypes = [ctypes.POINTER(ctypes.c_int)]
        L.lbm_b200_last_device_ms.restype = ctypes.c_double
        L.lbm_b200_last_launches.restype = ctypes.c_long
        L.lbm_b200_launches_for.restype = ctypes.c_long
        L.lbm_b200_last_error.restype = ctypes.c_char_p
        L.lbm_verify.restype = ctypes.c_double
        L.lbm_density.restype = ctypes.c_double
        L.lbm_geo_create.argtypes = [ctypes.c_char_p, ctypes.c_int * 3, ctypes.c_int * 3,
                                     ctypes.POINTER(LatticeDesc)]
        _lib = L
    return _lib


def kernel_names():
    n = ctypes.c_int(0)
    t = lib().lbm_b200_kernels(ctypes.byref(n))
    return [t[i].Name.decode() for i in range(n.value)]


class Lattice:
    """A LatticeDesc plus the numpy array that owns its mask."""

    def __init__(self, mask, dims, periodic, name="custom"):
        self.mask = np.ascontiguousarray(mask, dtype=np.int32).reshape(-1)
        self.dims = tuple(int(v) for v in dims)
        assert self.mask.size == self.dims[0] * self.dims[1] * self.dims[2]
        self._name = name.encode()
        d = LatticeDesc()
        for i in range(3):
            d.Dims[i] = self.dims[i]
        d.Lattice = self.mask.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        d.nCells = int(self.mask.size)
        d.nObst = int(np.count_nonzero(self.mask == 0))
        d.nFluid = int(self.mask.size - d.nObst)
        d.nInlet = int(np.count_nonzero(self.mask == 2))
        d.nOutlet = int(np.count_nonzero(self.mask == 4))
        d.PeriodicX, d.PeriodicY, d.PeriodicZ = (int(v) for v in periodic)
        d.Name = self._name
        self.desc = d

    @property
    def periodic(self):
        return (self.desc.PeriodicX, self.desc.PeriodicY, self.desc.PeriodicZ)

    @property
    def n_fluid(self):
        return self.desc.nFluid


def geometry(name, dims, periodic=(0, 0, 0)):
    """GeoCreateByStr through the library (src/Geometry.c:37-281)."""
    d = (ctypes.c_int * 3)(*dims)
    p = (ctypes.c_int * 3)(*periodic)
    ld = LatticeDesc()
    rc = lib().lbm_geo_create(name.encode(), d, p, ctypes.byref(ld))
    if rc != 0:
        raise ValueError("geometry %r rejected" % name)
    n = dims[0] * dims[1] * dims[2]
    mask = np.ctypeslib.as_array(ld.Lattice, shape=(n,)).copy()
    ctypes.CDLL(None).free(ctypes.cast(ld.Lattice, ctypes.c_void_p))
    lat = Lattice(mask, dims, (ld.PeriodicX, ld.PeriodicY, ld.PeriodicZ), ld.Name.decode())
    lat.geo_periodic = tuple(p)  # the flags after the geometry forced its own
    return lat


def case(omega=1.0, xforce=1e-5, iterations=10, rho_in=1.0, rho_out=1.0, vtk=0):
    """CaseData with the reference's defaults (src/Main.c:140-147); vtk=n > 0
    asks Kernel for VTK files every n steps (the -vtk n flag)."""
    cd = CaseData()
    cd.Omega, cd.XForce, cd.MaxIterations = omega, xforce, iterations
    cd.RhoIn, cd.RhoOut = rho_in, rho_out
    cd.VtkModulus = cd.StatisticsModulus = 100
    if vtk:
        cd.VtkOutput, cd.VtkModulus = 1, int(vtk)
    return cd


def write_vtk_field(lattice, field, xforce, iteration, path):
    """lbm_vtk_write_file on a logical PDF field held on the host (cells x
    fastest, 19 per cell): the VTK writer of the CUDA rows, fed through a
    GetNode that reads `field`."""
    f = np.ascontiguousarray(field, dtype=np.float64).reshape(-1, Q)
    nx, ny, _ = lattice.dims

    def get_node(_kd, x, y, z, out):
        row = f[x + nx * (y + ny * z)]
        for d in range(Q):
            out[d] = row[d]

    kd = KernelData()
    cb = _GETNODE(get_node)
    kd.GetNode = cb
    cd = case(xforce=xforce)
    rc = lib().lbm_vtk_write_file(ctypes.byref(lattice.desc), ctypes.byref(kd), ctypes.byref(cd), int(iteration),
                                  os.fsencode(path))
    if rc:
        raise RuntimeError("writing %s failed" % path)


class Kernel:
    """One row of the kernel table: {Name, Init, Deinit}."""

    def __init__(self, row):
        self.name = row.Name.decode()
        self._row = row

    def init(self, lattice, kernel_args=()):
        args = [a.encode() for a in kernel_args]
        arr = (ctypes.c_char_p * max(1, len(args)))(*args)
        p = Parameters(0, None, len(args), arr)
        kdp = ctypes.POINTER(KernelData)()
        self._row.Init(ctypes.byref(lattice.desc), ctypes.byref(kdp), ctypes.byref(p))
        return Instance(self, lattice, kdp)


def kernel(name):
    n = ctypes.c_int(0)
    t = lib().lbm_b200_kernels(ctypes.byref(n))
    for i in range(n.value):
        if t[i].Name.decode().lower() == name.lower():
            return Kernel(t[i])
    raise KeyError("requested kernel %r not found; available: %s" % (name, ", ".join(kernel_names())))


class Instance:
    """An initialised kernel (the KernelData an Init returned)."""

    def __init__(self, kf, lattice, kdp):
        self.kf, self.lattice, self.kdp = kf, lattice, kdp

    @property
    def kd(self):
        return self.kdp.contents

    def set_initial_density(self, cd):
        lib().lbm_set_initial_density(ctypes.byref(self.lattice.desc), self.kdp, ctypes.byref(cd))

    def set_initial_velocity(self, cd):
        lib().lbm_set_initial_velocity(ctypes.byref(self.lattice.desc), self.kdp, ctypes.byref(cd))

    def run(self, cd):
        """kd->Kernel: cd.MaxIterations steps; returns the kernel's Duration."""
        self.kd.Kernel(ctypes.byref(self.lattice.desc), self.kdp, ctypes.byref(cd))
        return self.kd.Duration

    def launches_for(self, n):
        """Kernel launches that n time steps take on this instance."""
        return int(lib().lbm_b200_launches_for(self.kdp, int(n)))

    def write_vtk(self, cd, iteration, path):
        """lbm_vtk_write_file: the current state as a legacy VTK file."""
        if lib().lbm_vtk_write_file(ctypes.byref(self.lattice.desc), self.kdp, ctypes.byref(cd), int(iteration),
                                    os.fsencode(path)):
            raise RuntimeError("writing %s failed" % path)

    def checkpoint(self, path):
        """lbm_b200_checkpoint_save: the state, bit for bit, into `path`."""
        rc = lib().lbm_b200_checkpoint_save(self.kdp, os.fsencode(path))
        if rc:
            raise RuntimeError("checkpoint failed (%d): %s" % (rc, lib().lbm_b200_last_error().decode()))

    def restore(self, path):
        """lbm_b200_checkpoint_load: continue from a checkpoint of an
        instance of the same kernel, storage, lattice and Lambda."""
        rc = lib().lbm_b200_checkpoint_load(self.kdp, os.fsencode(path))
        if rc:
            raise RuntimeError("restore failed (%d): %s" % (rc, lib().lbm_b200_last_error().decode()))

    def step_device(self, cd, n):
        rc = lib().lbm_b200_step_device(self.kdp, ctypes.byref(cd), int(n))
        if rc:
            raise RuntimeError(lib().lbm_b200_last_error().decode())

    def sync_mirror(self):
        rc = lib().lbm_b200_sync_mirror(self.kdp)
        if rc:
            raise RuntimeError(lib().lbm_b200_last_error().decode())

    def get_node(self, x, y, z):
        out = (ctypes.c_double * Q)()
        self.kd.GetNode(self.kdp, x, y, z, out)
        return np.array(out[:])

    def set_node(self, x, y, z, pdfs):
        arr = (ctypes.c_double * Q)(*[float(v) for v in pdfs])
        self.kd.SetNode(self.kdp, x, y, z, arr)

    def get_field(self):
        out = np.full(self.lattice.mask.size * Q, np.nan)
        lib().lbm_b200_get_field(self.kdp, ctypes.byref(self.lattice.desc),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out.reshape(-1, Q)

    def set_field(self, pdfs):
        pdfs = np.ascontiguousarray(pdfs, dtype=np.float64).reshape(-1)
        lib().lbm_b200_set_field(self.kdp, ctypes.byref(self.lattice.desc),
                                 pdfs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))

    def verify(self, cd, write_file=False):
        """KernelVerifiy through GetNode on the host mirror (lbm_verify)."""
        return lib().lbm_verify(ctypes.byref(self.lattice.desc), self.kdp, ctypes.byref(cd), int(write_file))

    def verify_device(self, cd, write_file=False):
        """The same check on the device (lbm_b200_verify_device): only the
        x-velocity slice and the error come back to the host."""
        err = ctypes.c_double(0.0)
        rc = lib().lbm_b200_verify_device(ctypes.byref(self.lattice.desc), self.kdp, ctypes.byref(cd),
                                          int(write_file), ctypes.byref(err))
        if rc:
            raise RuntimeError("device verify failed (%d): %s" % (rc, lib().lbm_b200_last_error().decode()))
        return err.value

    def density(self):
        return lib().lbm_density(self.kdp, ctypes.byref(self.lattice.desc))

    def moments(self):
        """lbm_b200_instance_moments: FP64 (sum rho, sum j_x, sum j_y, sum j_z)
        over the instance's fluid nodes (list kernels, any storage)."""
        out = (ctypes.c_double * 4)()
        rc = lib().lbm_b200_instance_moments(self.kdp, out)
        if rc:
            raise RuntimeError("moments failed (%d): %s" % (rc, lib().lbm_b200_last_error().decode()))
        return tuple(out)

    def list_layout(self):
        g = ctypes.POINTER(ctypes.c_uint32)()
        a = ctypes.POINTER(ctypes.c_uint32)()
        nf, nc = ctypes.c_int(0), ctypes.c_int(0)
        rc = lib().lbm_b200_list_layout(self.kdp, ctypes.byref(g), ctypes.byref(a), ctypes.byref(nf),
                                        ctypes.byref(nc))
        if rc:
            raise ValueError("not a list kernel")
        grid = np.ctypeslib.as_array(g, shape=(self.lattice.mask.size,)).copy()
        adj = np.ctypeslib.as_array(a, shape=(max(nf.value, 1) * 18,))[: nf.value * 18].copy()
        return grid, adj, nf.value, nc.value

    @property
    def last_device_ms(self):
        return lib().lbm_b200_last_device_ms(self.kdp)

    @property
    def last_launches(self):
        return lib().lbm_b200_last_launches(self.kdp)

    def last_copy_bytes(self):
        h, d = ctypes.c_size_t(0), ctypes.c_size_t(0)
        lib().lbm_b200_last_copy_bytes(self.kdp, ctypes.byref(h), ctypes.byref(d))
        return h.value, d.value

    def deinit(self):
        if self.kdp:
            self.kf._row.Deinit(ctypes.byref(self.lattice.desc), ctypes.byref(self.kdp))
            self.kdp = ctypes.POINTER(KernelData)()


def list_build(lattice, pull, blk=(0, 0, 0), pad=None):
    """Host list layout without a GPU: (grid, adj, nFluid, nCells)."""
    L = lib()
    n_cells = L.lbmh_pad_cells(lattice.n_fluid, 8, pad.encode() if pad else None)
    if n_cells < 0:
        raise ValueError("bad padding string %r" % pad)
    if pull:
        n_cells = n_cells + (8 - n_cells % 8)
    grid = np.zeros(lattice.mask.size, dtype=np.uint32)
    adj = np.zeros(max(lattice.n_fluid, 1) * 18, dtype=np.uint32)
    b = (ctypes.c_int * 3)(*blk)
    nf = L.lbmh_list_build(ctypes.byref(lattice.desc), int(bool(pull)), b, n_cells,
                           grid.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), None,
                           adj.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    return grid, adj[: nf * 18], nf, n_cells


def list_build_device(lattice, pull, blk=(0, 0, 0), pad=None):
    """lbm_b200_list_build: the same layout built on the GPU."""
    L = lib()
    n_cells = L.lbmh_pad_cells(lattice.n_fluid, 8, pad.encode() if pad else None)
    if n_cells < 0:
        raise ValueError("bad padding string %r" % pad)
    if pull:
        n_cells = n_cells + (8 - n_cells % 8)
    grid = np.zeros(lattice.mask.size, dtype=np.uint32)
    adj = np.zeros(max(lattice.n_fluid, 1) * 18, dtype=np.uint32)
    b = (ctypes.c_int * 3)(*blk)
    nf = L.lbm_b200_list_build(ctypes.byref(lattice.desc), int(bool(pull)), b, n_cells,
                               grid.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                               adj.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)))
    if nf < 0:
        raise RuntimeError("device list build failed (%d)" % nf)
    return grid, adj[: nf * 18], nf, n_cells


# ---------------------------------------------------------------------------
# Batched domains (lbm_batch_* in include/lbm_b200.h)

STORAGE = {"fp32": 1, "fp16": 2}


def _batch_lib():
    L = lib()
    if not getattr(L, "_batch_sigs", False):
        L.lbm_batch_create.restype = ctypes.c_void_p
        L.lbm_batch_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int]
        for name in ("lbm_batch_destroy", "lbm_batch_add", "lbm_batch_remove", "lbm_batch_reset", "lbm_batch_step",
                     "lbm_batch_sync", "lbm_batch_moments", "lbm_batch_get_field", "lbm_batch_set_field",
                     "lbm_batch_set_launch", "lbm_batch_get_launch", "lbm_batch_time_steps", "lbm_batch_tune",
                     "lbm_batch_bytes_used", "lbm_batch_launches", "lbm_batch_active_domains",
                     "lbm_batch_fluid_nodes", "lbm_batch_checkpoint_save", "lbm_batch_checkpoint_load"):
            getattr(L, name).argtypes = None
        L.lbm_batch_add.argtypes = [ctypes.c_void_p, ctypes.POINTER(LatticeDesc), ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double]
        L.lbm_batch_bytes_used.restype = ctypes.c_size_t
        L.lbm_batch_launches.restype = ctypes.c_longlong
        L.lbm_batch_last_error.restype = ctypes.c_char_p
        L._batch_sigs = True
    return L


class Batch:
    """Many independent domains advanced by one persistent launch per step."""

    def __init__(self, storage="fp32", budget_gb=150.0, max_domains=1024):
        self.L = _batch_lib()
        self.max_domains = max_domains
        self.h = self.L.lbm_batch_create(STORAGE[storage], ctypes.c_double(budget_gb), max_domains)
        if not self.h:
            raise RuntimeError(self.L.lbm_batch_last_error().decode())
        self.h = ctypes.c_void_p(self.h)
        self.lattices = {}

    def add(self, lattice, omega=1.0, lam=3.0 / 16.0, xforce=1e-5):
        slot = self.L.lbm_batch_add(self.h, ctypes.byref(lattice.desc), omega, lam, xforce)
        if slot >= 0:
            self.lattices[slot] = lattice
        return slot

    def remove(self, slot):
        rc = self.L.lbm_batch_remove(self.h, slot)
        self.lattices.pop(slot, None)
        return rc

    def step(self, n, graph=True):
        rc = self.L.lbm_batch_step(self.h, int(n), int(bool(graph)))
        if rc:
            raise RuntimeError("batch step failed: %s" % self.L.lbm_batch_last_error().decode())

    def sync(self):
        rc = self.L.lbm_batch_sync(self.h)
        if rc:
            raise RuntimeError("batch sync failed: %s" % self.L.lbm_batch_last_error().decode())

    def moments(self):
        out = np.zeros(self.max_domains * 4)
        rc = self.L.lbm_batch_moments(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if rc:
            raise RuntimeError("batch moments failed: %s" % self.L.lbm_batch_last_error().decode())
        return out.reshape(-1, 4)

    def get_field(self, slot):
        lat = self.lattices[slot]
        out = np.full(lat.mask.size * Q, np.nan)
        rc = self.L.lbm_batch_get_field(self.h, slot, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert rc == 0
        return out.reshape(-1, Q)

    def set_field(self, slot, pdfs):
        pdfs = np.ascontiguousarray(pdfs, dtype=np.float64).reshape(-1)
        rc = self.L.lbm_batch_set_field(self.h, slot, pdfs.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        assert rc == 0

    def checkpoint(self, slot, path):
        """lbm_batch_checkpoint_save: one resident domain, bit for bit."""
        rc = self.L.lbm_batch_checkpoint_save(self.h, int(slot), os.fsencode(path))
        if rc:
            raise RuntimeError("checkpoint failed (%d): %s" % (rc, self.L.lbm_batch_last_error().decode()))

    def restore(self, slot, path):
        """lbm_batch_checkpoint_load into a slot admitted from the same
        lattice with the same relaxation parameters."""
        rc = self.L.lbm_batch_checkpoint_load(self.h, int(slot), os.fsencode(path))
        if rc:
            raise RuntimeError("restore failed (%d): %s" % (rc, self.L.lbm_batch_last_error().decode()))

    def time_steps(self, n):
        ms = ctypes.c_double(0.0)
        rc = self.L.lbm_batch_time_steps(self.h, int(n), ctypes.byref(ms))
        if rc:
            raise RuntimeError(self.L.lbm_batch_last_error().decode())
        return ms.value

    def tune(self, trial_steps=10):
        rows = np.zeros((64, 5))
        n = self.L.lbm_batch_tune(self.h, int(trial_steps), rows.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 64)
        return rows[:n]

    def launch(self):
        out = (ctypes.c_int * 6)()
        self.L.lbm_batch_get_launch(self.h, out)
        return {"even": {"threads": out[0], "nodes_per_thread": out[1], "blocks": out[2]},
                "odd": {"threads": out[3], "nodes_per_thread": out[4], "blocks": out[5]}}

    def set_launch(self, which, threads, blocks):
        assert self.L.lbm_batch_set_launch(self.h, {"even": 0, "odd": 1, "both": 2}[which], threads, blocks) == 0

    @property
    def bytes_used(self):
        return self.L.lbm_batch_bytes_used(self.h)

    def fluid_nodes(self, slot):
        return self.L.lbm_batch_fluid_nodes(self.h, slot)

    def close(self):
        if self.h:
            self.L.lbm_batch_destroy(self.h)
            self.h = None


def spheres(dims, seed, porosity, rmin, rmax, rsa_attempts=20000):
    """Seeded periodic sphere packing (lbm_geo_spheres): (Lattice, stats)."""
    L = lib()
    L.lbm_geo_spheres.argtypes = [ctypes.c_int * 3, ctypes.c_uint64, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_int, ctypes.POINTER(LatticeDesc),
                                  ctypes.POINTER(ctypes.c_double)]
    ld = LatticeDesc()
    st = (ctypes.c_double * 4)()
    rc = L.lbm_geo_spheres((ctypes.c_int * 3)(*dims), int(seed), porosity, rmin, rmax, rsa_attempts,
                           ctypes.byref(ld), st)
    if rc:
        raise ValueError("sphere packing rejected its arguments")
    n = dims[0] * dims[1] * dims[2]
    mask = np.ctypeslib.as_array(ld.Lattice, shape=(n,)).copy()
    ctypes.CDLL(None).free(ctypes.cast(ld.Lattice, ctypes.c_void_p))
    lat = Lattice(mask, dims, (1, 1, 1), "spheres")
    return lat, {"porosity": st[0], "spheres_rsa": int(st[1]), "spheres_overlap": int(st[2]),
                 "jam_porosity": st[3]}
