"""One AA-pattern lattice split into x-slabs: one slab per GPU (one process
per GPU, torch.distributed for the halo messages), or several slabs in one
process on one GPU (tests, and the same arithmetic without a second GPU).
Two layouts: the full array (cuda-aa-soa kernels) and the fluid-node list
(cuda-list-aa-pv-soa kernels, FP64), whose slabs keep ghost nodes for the
neighbours' fluid cells that their links reach.

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
phase for full-array slabs, one PDF element (8, 4 or 2 bytes: the list's
storage) per link through the face for list slabs (``Slab.message``); the
transports carry them in buffers of 8-byte words.

Transports: ``LocalTransport`` (all slabs in this process: device-to-device
through shared device buffers, every operation on one stream) and
``DistTransport`` (one slab per rank: paired isend/irecv through
torch.distributed -- NCCL on GPUs, gloo on CPU for the host-side tests).
The slabs close into a ring (the first and last slab exchange too) when any
axis is periodic (``is_ring``).
"""
import contextlib
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
        L.lbm_aa_list_slab_init.restype = ctypes.POINTER(KernelData)
        L.lbm_aa_list_slab_init.argtypes = L.lbm_aa_slab_init.argtypes
        L.lbm_aa_halo_count.restype = ctypes.c_longlong
        L.lbm_aa_halo_message.restype = ctypes.c_longlong
        L.lbm_aa_halo_message.argtypes = [ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.lbm_aa_halo_elem_bytes.argtypes = [ctypes.POINTER(KernelData)]
        L.lbm_aa_list_slab_layout.argtypes = [ctypes.POINTER(LatticeDesc), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.POINTER(Parameters),
                                              ctypes.POINTER(ctypes.c_longlong)] + [ctypes.c_void_p] * 6
        for name in ("lbm_aa_halo_pack", "lbm_aa_halo_unpack"):
            getattr(L, name).argtypes = [ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p]
        L.lbm_aa_slab_step.argtypes = [ctypes.POINTER(KernelData), ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.lbm_aa_slab_odd_part.argtypes = [ctypes.POINTER(KernelData), ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_void_p]
        L.lbm_aa_slab_even_part.argtypes = L.lbm_aa_slab_odd_part.argtypes
        L._slab_sigs = True
    return L


def _ptr(buf):
    """Device address of a buffer: a torch tensor or an integer address."""
    return buf.data_ptr() if hasattr(buf, "data_ptr") else int(buf)


def _params(kernel_args):
    args = [a.encode() for a in kernel_args]
    argv = (ctypes.c_char_p * max(1, len(args)))(*args)
    p = Parameters()
    p.nArgs, p.Args, p.nKernelArgs, p.KernelArgs = 0, None, len(args), argv
    return p, argv


class Slab:
    """The x range [x0, x1) of `lattice` as an AA-pattern instance on the
    current device: layout "full" (cuda-aa-soa kernels) or "list"
    (cuda-list-aa-pv-soa kernels, FP64); kernel_args as for the kernel's
    Init."""

    def __init__(self, lattice, x0, x1, halo_lo, halo_hi, kernel_args=(), layout="full"):
        if layout not in ("full", "list"):
            raise ValueError("layout must be 'full' or 'list'")
        self.L = _sigs(lib())
        nx, ny, nz = lattice.dims
        self.x0, self.x1, self.layout = x0, x1, layout
        mask = lattice.mask.reshape(nz, ny, nx)[:, :, x0:x1]
        self.local = Lattice(mask.reshape(-1), (x1 - x0, ny, nz), lattice.periodic, "slab")
        p, self._argv = _params(kernel_args)
        self._global = lattice  # keeps the lattice's mask alive for the call
        init = self.L.lbm_aa_slab_init if layout == "full" else self.L.lbm_aa_list_slab_init
        kdp = init(ctypes.byref(lattice.desc), x0, x1, int(halo_lo), int(halo_hi), ctypes.byref(p))
        if not kdp:
            raise RuntimeError("slab init failed: %s" % self.L.lbm_b200_last_error().decode())
        self.inst = Instance(None, self.local, kdp)
        self.kdp = kdp
        self.elem_bytes = int(self.L.lbm_aa_halo_elem_bytes(kdp))
        self.count = int(self.L.lbm_aa_halo_count(kdp))

    def message(self, side, phase, send):
        """PDF elements (elem_bytes each) this slab sends (send=True) or
        receives through `side` in `phase` (-1: no halo on that face)."""
        return int(self.L.lbm_aa_halo_message(self.kdp, int(side), int(phase), int(bool(send))))

    def step(self, cd, half, stream=None):
        rc = self.L.lbm_aa_slab_step(self.kdp, ctypes.byref(cd), int(half), stream)
        if rc:
            raise RuntimeError("slab step failed (%d)" % rc)

    def odd_part(self, cd, part, stream=None):
        """Part 0 (cells that touch no halo slot) or part 1 (the rest) of the
        odd step: lbm_aa_slab_odd_part."""
        rc = self.L.lbm_aa_slab_odd_part(self.kdp, ctypes.byref(cd), int(part), stream)
        if rc:
            raise RuntimeError("slab odd step part failed (%d)" % rc)

    def even_part(self, cd, part, stream=None):
        """Part 0 (cells whose slots no message carries) or part 1 (the rest)
        of the even step: lbm_aa_slab_even_part."""
        rc = self.L.lbm_aa_slab_even_part(self.kdp, ctypes.byref(cd), int(part), stream)
        if rc:
            raise RuntimeError("slab even step part failed (%d)" % rc)

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


def message(slab, side, phase, send):
    """Length of a slab's message through `side` in `phase`, in 8-byte words
    (the transports' buffers hold doubles; a message of 4- or 2-byte PDF
    elements fills the words' leading bytes): the slab's own ``message``
    method, else its fixed ``count``; -1 without a halo."""
    m = getattr(slab, "message", None)
    n = m(side, phase, send) if m else slab.count
    return n if n < 0 else words(slab, n)


def words(slab, n):
    """8-byte words holding n PDF elements of the slab's storage."""
    eb = getattr(slab, "elem_bytes", 8)
    return (n * eb + 7) // 8


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
        for (r, q) in self.faces:
            for phase in (0, 1):
                if (message(slabs[r], 1, phase, True) != message(slabs[q], 0, phase, False)
                        or message(slabs[q], 0, phase, True) != message(slabs[r], 1, phase, False)):
                    raise ValueError("slabs %d and %d disagree on their shared face's messages" % (r, q))
        self.bufs = {f: (alloc(max(1, words(slabs[f[0]], slabs[f[0]].count))),
                         alloc(max(1, words(slabs[f[1]], slabs[f[1]].count)))) for f in self.faces}

    def exchange(self, phase):
        for (r, q) in self.faces:
            to_right, to_left = self.bufs[(r, q)]
            self.slabs[r].pack(1, phase, to_right, self.stream)
            self.slabs[q].unpack(0, phase, to_right, self.stream)
            self.slabs[q].pack(0, phase, to_left, self.stream)
            self.slabs[r].unpack(1, phase, to_left, self.stream)

    # all slabs share one stream, so a started exchange is already complete
    # in stream order
    def start(self, phase):
        self.exchange(phase)

    def finish(self, phase):
        pass


class DistTransport:
    """One slab per rank: paired isend/irecv with the left and right
    neighbours through torch.distributed. Sends are posted right face first,
    receives left face first, so that two messages between the same pair of
    ranks (two slabs on a periodic ring) match in order.

    Stream order (NCCL): a posted send waits for torch's current stream, and
    ``req.wait()`` makes only the current stream wait for the received
    data. With an explicit `stream` (the slab's packs, unpacks and steps run
    there), ``start`` and ``finish`` make that stream torch's current one for
    their duration, so the sends follow the packs and the unpacks follow the
    receives whatever stream the caller has current."""

    def __init__(self, slab, rank, world, ring, dist, make_buf, stream=None):
        self.slab, self.dist, self.stream = slab, dist, stream
        self.left, self.right = neighbours(rank, world, ring)
        # one buffer per face and direction; each phase's message is a prefix
        self.send = {s: make_buf(max(1, max(message(slab, s, p, True) for p in (0, 1)))) for s in (0, 1)}
        self.recv = {s: make_buf(max(1, max(message(slab, s, p, False) for p in (0, 1)))) for s in (0, 1)}
        self._reqs, self._inc = [], {}

    def exchange(self, phase, sync=None):
        self.start(phase, sync)
        self.finish(phase)

    def _on_stream(self):
        if not self.stream:
            return contextlib.nullcontext()
        import torch
        return torch.cuda.stream(torch.cuda.ExternalStream(self.stream))

    def start(self, phase, sync=None):
        """Packs this slab's messages and posts the sends and receives; they
        travel while the caller enqueues more work (with NCCL the library's
        stream waits for the packs, then runs beside the slab's stream)."""
        with self._on_stream():
            self._start(phase, sync)

    def _start(self, phase, sync):
        d = self.dist
        faces = [s for s in (1, 0) if (self.right if s else self.left) is not None]
        out = {s: self.send[s][:message(self.slab, s, phase, True)] for s in faces}
        self._inc = {s: self.recv[s][:message(self.slab, s, phase, False)] for s in faces}
        for side in faces:
            self.slab.pack(side, phase, out[side], self.stream)
        if sync:
            sync()  # the packed buffers are complete before the library sends them
        ops = []
        for side, peer in ((1, self.right), (0, self.left)):
            if peer is not None:
                ops.append(d.P2POp(d.isend, out[side], peer))
        for side, peer in ((0, self.left), (1, self.right)):
            if peer is not None:
                ops.append(d.P2POp(d.irecv, self._inc[side], peer))
        self._reqs = d.batch_isend_irecv(ops) if ops else []

    def finish(self, phase):
        """Waits for the posted messages (on NCCL: the slab's stream waits)
        and unpacks the received ones."""
        with self._on_stream():
            self._finish(phase)

    def _finish(self, phase):
        for req in self._reqs:
            req.wait()
        self._reqs = []
        for side in (0, 1):
            if (self.right if side else self.left) is not None:
                self.slab.unpack(side, phase, self._inc[side], self.stream)


def list_slab_layout(lattice, x0, x1, halo_lo, halo_hi, kernel_args=()):
    """The layout of a list slab, built on the host (no CUDA call): a dict
    with n_owned, n_ghost, n_cells, grid (slab cells, x fastest), adj
    (n_owned x 18), the slot lists own / ghost per side (None: no halo) and
    the inner tile range (256-node tiles that link to no ghost node)."""
    L = _sigs(lib())
    nx, ny, nz = lattice.dims
    p, argv = _params(kernel_args)
    counts = (ctypes.c_longlong * 9)()
    args = (ctypes.byref(lattice.desc), x0, x1, int(halo_lo), int(halo_hi), ctypes.byref(p), counts)
    rc = L.lbm_aa_list_slab_layout(*args, None, None, None, None, None, None)
    if rc:
        raise RuntimeError("list slab layout failed (%d): %s" % (rc, L.lbm_b200_last_error().decode()))
    n_owned = counts[0]
    grid = np.zeros((x1 - x0) * ny * nz, dtype=np.uint32)
    adj = np.zeros(max(1, n_owned) * 18, dtype=np.uint32)
    lists = [np.zeros(max(1, counts[3 + k]), dtype=np.uint32) for k in range(4)]
    ptr = [a.ctypes.data for a in [grid, adj] + lists]
    rc = L.lbm_aa_list_slab_layout(*args, *ptr)
    if rc:
        raise RuntimeError("list slab layout failed (%d)" % rc)
    cut = [lists[k][:counts[3 + k]] if counts[3 + k] >= 0 else None for k in range(4)]
    return {"n_owned": n_owned, "n_ghost": counts[1], "n_cells": counts[2], "grid": grid,
            "adj": adj[: n_owned * 18], "own": (cut[0], cut[2]), "ghost": (cut[1], cut[3]),
            "inner": (counts[7], counts[8])}


def step_pairs(slabs, transport, cd, pairs, stream=None, overlap=False):
    """`pairs` even/odd step pairs of a slab-decomposed lattice. With
    `overlap`, each exchange travels while the cells that its messages do not
    concern take a step: the phase-0 messages during the odd step of the
    inner cells (Slab.odd_part 0), the phase-1 messages during the next
    pair's even step of the inner cells (Slab.even_part 0); the other cells
    follow the unpack."""
    if not overlap:
        for _ in range(pairs):
            for s in slabs:
                s.step(cd, 0, stream)
            transport.exchange(0)
            for s in slabs:
                s.step(cd, 1, stream)
            transport.exchange(1)
        return
    if pairs <= 0:
        return
    for s in slabs:
        s.step(cd, 0, stream)
    for k in range(pairs):
        transport.start(0)
        for s in slabs:
            s.odd_part(cd, 0, stream)
        transport.finish(0)
        for s in slabs:
            s.odd_part(cd, 1, stream)
        transport.start(1)
        last = k + 1 == pairs
        if not last:
            for s in slabs:
                s.even_part(cd, 0, stream)
        transport.finish(1)
        if not last:
            for s in slabs:
                s.even_part(cd, 1, stream)


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
