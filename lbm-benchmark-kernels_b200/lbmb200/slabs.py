"""One full-array AA lattice split into x-slabs: one slab per GPU (one process
per GPU, torch.distributed for the halo messages), or several slabs in one
process on one GPU (tests, and the same arithmetic without a second GPU).

A step pair of the AA pattern on a slab:

1. even step on every slab (local to each cell, no exchange);
2. phase-0 exchange: each halo face sends the face plane's five PDFs that the
   neighbour's cells read and write in the odd step; the neighbour stores them
   in its ghost plane;
3. odd step on every slab: face cells read and write the ghost plane as if it
   were the neighbour's plane;
4. phase-1 exchange: each slab sends what its cells wrote into the ghost plane
   back; the neighbour stores it in its face plane.

Every slot is read and written by exactly one cell in the odd step, so after
the pair the slabs hold the whole lattice's state bit for bit (tested against
the single-instance kernel). Messages are 5 x nY x nZ doubles per face and
phase (lbm_aa_halo_count).

Transports: ``LocalTransport`` (all slabs in this process: device-to-device
through shared device buffers, every operation on one stream) and
``DistTransport`` (one slab per rank: paired isend/irecv through
torch.distributed -- NCCL on GPUs, gloo on CPU for the host-side tests).
The slabs close into a ring (the first and last slab exchange too) when any
axis is periodic (``is_ring``).
"""
import ctypes

import numpy as np

from . import Instance, Lattice, KernelData, LatticeDesc, Parameters, lib


def partition(nx, parts):
    """x ranges [x0, x1) of `parts` slabs of nearly equal thickness."""
    if not 1 <= parts <= nx:
        raise ValueError("cannot split %d planes into %d slabs" % (nx, parts))
    edges = [nx * k // parts for k in range(parts + 1)]
    return list(zip(edges[:-1], edges[1:]))


def is_ring(periodic):
    """Whether the slabs close into a ring: with a periodic x axis, and also
    with only y or z periodic, since a link that leaves through the x boundary
    and a periodic face at once wraps every crossed axis to the other x end
    (the reference's rule, src/BenchKernelD3Q19AaCommon.c:522-578)."""
    return any(bool(p) for p in periodic)


def halo_flags(rank, parts, ring):
    """(halo at the x0 face, halo at the x1-1 face) of slab `rank`."""
    if parts == 1:
        return False, False
    return (rank > 0 or bool(ring)), (rank < parts - 1 or bool(ring))


def neighbours(rank, parts, ring):
    """(left, right) neighbour slab of `rank` (None at a closed x face)."""
    lo, hi = halo_flags(rank, parts, ring)
    return ((rank - 1) % parts if lo else None), ((rank + 1) % parts if hi else None)


def _sigs(L):
    if not getattr(L, "_slab_sigs", False):
        L.lbm_aa_slab_init.restype = ctypes.POINTER(KernelData)
        L.lbm_aa_slab_init.argtypes = [ctypes.POINTER(LatticeDesc), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.POINTER(Parameters)]
        L.lbm_aa_halo_count.restype = ctypes.c_longlong
        for name in ("lbm_aa_halo_pack", "lbm_aa_halo_unpack"):
            getattr(L, name).argtypes = [ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p]
        L.lbm_aa_slab_step.argtypes = [ctypes.POINTER(KernelData), ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L._slab_sigs = True
    return L


def _ptr(buf):
    """Device address of a buffer: a torch tensor or an integer address."""
    return buf.data_ptr() if hasattr(buf, "data_ptr") else int(buf)


class Slab:
    """The x range [x0, x1) of `lattice` as an AA instance on the current
    device (cuda-aa-soa kernels; kernel_args as for its Init)."""

    def __init__(self, lattice, x0, x1, halo_lo, halo_hi, kernel_args=()):
        self.L = _sigs(lib())
        nx, ny, nz = lattice.dims
        self.x0, self.x1 = x0, x1
        mask = lattice.mask.reshape(nz, ny, nx)[:, :, x0:x1]
        self.local = Lattice(mask.reshape(-1), (x1 - x0, ny, nz), lattice.periodic, "slab")
        args = [a.encode() for a in kernel_args]
        self._argv = (ctypes.c_char_p * max(1, len(args)))(*args)
        p = Parameters()
        p.nArgs, p.Args, p.nKernelArgs, p.KernelArgs = 0, None, len(args), self._argv
        self._global = lattice  # keeps the lattice's mask alive for the call
        kdp = self.L.lbm_aa_slab_init(ctypes.byref(lattice.desc), x0, x1, int(halo_lo), int(halo_hi),
                                      ctypes.byref(p))
        if not kdp:
            raise RuntimeError("slab init failed: %s" % self.L.lbm_b200_last_error().decode())
        self.inst = Instance(None, self.local, kdp)
        self.kdp = kdp
        self.count = int(self.L.lbm_aa_halo_count(kdp))

    def step(self, cd, half, stream=None):
        rc = self.L.lbm_aa_slab_step(self.kdp, ctypes.byref(cd), int(half), stream)
        if rc:
            raise RuntimeError("slab step failed (%d)" % rc)

    def pack(self, side, phase, buf, stream=None):
        rc = self.L.lbm_aa_halo_pack(self.kdp, int(side), int(phase), _ptr(buf), stream)
        if rc:
            raise RuntimeError("halo pack failed (%d)" % rc)

    def unpack(self, side, phase, buf, stream=None):
        rc = self.L.lbm_aa_halo_unpack(self.kdp, int(side), int(phase), _ptr(buf), stream)
        if rc:
            raise RuntimeError("halo unpack failed (%d)" % rc)

    def close(self):
        if self.kdp:
            self.L.lbm_aa_slab_deinit(self.kdp)
            self.kdp = None


class LocalTransport:
    """All slabs of the lattice in this process, on one device: messages go
    through device buffers, and every step, pack and unpack is enqueued on
    one stream, so they run in program order. The stream must be an explicit
    one: the library puts operations given a null stream on each instance's
    own stream, which would not order the slabs' operations."""

    def __init__(self, slabs, ring, stream, alloc):
        if not stream:
            raise ValueError("LocalTransport needs an explicit (non-null) stream")
        self.slabs, self.stream = slabs, stream
        n = len(slabs)
        # faces between slab r (side 1) and its right-hand neighbour (side 0)
        self.faces = [(r, (r + 1) % n) for r in range(n) if neighbours(r, n, ring)[1] is not None]
        self.bufs = {f: (alloc(slabs[f[0]].count), alloc(slabs[f[0]].count)) for f in self.faces}

    def exchange(self, phase):
        for (r, q) in self.faces:
            to_right, to_left = self.bufs[(r, q)]
            self.slabs[r].pack(1, phase, to_right, self.stream)
            self.slabs[q].unpack(0, phase, to_right, self.stream)
            self.slabs[q].pack(0, phase, to_left, self.stream)
            self.slabs[r].unpack(1, phase, to_left, self.stream)


class DistTransport:
    """One slab per rank: paired isend/irecv with the left and right
    neighbours through torch.distributed. Sends are posted right face first,
    receives left face first, so that two messages between the same pair of
    ranks (two slabs on a periodic ring) match in order."""

    def __init__(self, slab, rank, world, ring, dist, make_buf, stream=None):
        self.slab, self.dist, self.stream = slab, dist, stream
        self.left, self.right = neighbours(rank, world, ring)
        self.send = {s: make_buf(slab.count) for s in (0, 1)}
        self.recv = {s: make_buf(slab.count) for s in (0, 1)}

    def exchange(self, phase, sync=None):
        d = self.dist
        for side in (1, 0):
            if (self.right if side else self.left) is not None:
                self.slab.pack(side, phase, self.send[side], self.stream)
        if sync:
            sync()  # the packed buffers are complete before the library sends them
        ops = []
        for side, peer in ((1, self.right), (0, self.left)):
            if peer is not None:
                ops.append(d.P2POp(d.isend, self.send[side], peer))
        for side, peer in ((0, self.left), (1, self.right)):
            if peer is not None:
                ops.append(d.P2POp(d.irecv, self.recv[side], peer))
        if ops:
            for req in d.batch_isend_irecv(ops):
                req.wait()
        for side in (0, 1):
            if (self.right if side else self.left) is not None:
                self.slab.unpack(side, phase, self.recv[side], self.stream)


def step_pairs(slabs, transport, cd, pairs, stream=None):
    """`pairs` even/odd step pairs of a slab-decomposed lattice."""
    for _ in range(pairs):
        for s in slabs:
            s.step(cd, 0, stream)
        transport.exchange(0)
        for s in slabs:
            s.step(cd, 1, stream)
        transport.exchange(1)


def gather_field(slabs, lattice):
    """The whole lattice's logical PDFs (cells x fastest, 19 per cell) from
    the slabs' mirrors (call after the slabs' streams are synchronised)."""
    nx, ny, nz = lattice.dims
    out = np.full((nz, ny, nx, 19), np.nan)
    for s in slabs:
        s.inst.sync_mirror()
        f = s.inst.get_field().reshape(nz, ny, s.x1 - s.x0, 19)
        out[:, :, s.x0:s.x1, :] = f
    return out.reshape(-1, 19)


def scatter_field(slabs, lattice, field):
    """Sets each slab's PDFs from a whole-lattice field."""
    nx, ny, nz = lattice.dims
    f = np.asarray(field, dtype=np.float64).reshape(nz, ny, nx, 19)
    for s in slabs:
        s.inst.set_field(np.ascontiguousarray(f[:, :, s.x0:s.x1, :]).reshape(-1, 19))
