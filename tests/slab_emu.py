"""A list-AA slab held in numpy and stepped by the oracle's half steps --
test infrastructure for the decomposed list layout (lbm_aa_list_slab_layout):
the layout under test is the library's, the arithmetic the oracle's. Used by
the in-process and the gloo (multi-process) slab tests."""
import numpy as np

from lbmb200 import slabs as sl

OMEGA, LAM, XF = 1.0, 3.0 / 16.0, 1.3e-5
NONE = 0xFFFFFFFF


def init_field(lat, seed):
    """Seeded PDFs near the weights on fluid cells, zeros on obstacles."""
    rng = np.random.default_rng(seed)
    w = np.array([1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4 + [1 / 3])
    f = w[None, :] * (1.0 + 0.1 * (rng.random((lat.mask.size, 19)) - 0.5))
    f[lat.mask == 0] = 0.0
    return f


class EmuSlab:
    """One list slab held in numpy and stepped by the oracle."""

    def __init__(self, lat, x0, x1, lo, hi, kargs):
        nx, ny, nz = lat.dims
        self.x0, self.x1 = x0, x1
        self.lay = sl.list_slab_layout(lat, x0, x1, lo, hi, kargs)
        self.nc = self.lay["n_cells"]
        self.f = np.full(19 * self.nc, np.nan)
        g = self.lay["grid"].reshape(nz, ny, x1 - x0)
        self.cells = np.nonzero(g.reshape(-1) != NONE)[0]
        zz, yy, xx = np.unravel_index(self.cells, (nz, ny, x1 - x0))
        self.gcells = (zz * ny + yy) * nx + xx + x0          # global cell of each owned slab cell
        self.nodes = g.reshape(-1)[self.cells].astype(np.int64)

    def set_field(self, field):
        for d in range(19):
            self.f[d * self.nc + self.nodes] = field[self.gcells, d]

    def get_field(self, out):
        for d in range(19):
            out[self.gcells, d] = self.f[d * self.nc + self.nodes]

    def half(self, oracle, odd):
        oracle.list_aa_half(odd, self.lay["n_owned"], self.nc, self.lay["adj"], self.f, OMEGA, LAM, XF)

    def _part(self, oracle, odd, part):
        t0, t1 = self.lay["inner"]
        no = self.lay["n_owned"]
        if t1 > t0:
            ranges = [(t0 * 256, min(t1 * 256, no))] if part == 0 else [(0, t0 * 256), (min(t1 * 256, no), no)]
        else:
            ranges = [] if part == 0 else [(0, no)]
        for n0, n1 in ranges:
            if n1 > n0:
                oracle.list_aa_half_range(odd, n0, n1, self.nc, self.lay["adj"], self.f, OMEGA, LAM, XF)

    def odd_part(self, oracle, part):
        """Part 0 (the inner tiles) or part 1 (the rest) of the odd step, by
        the library's inner tile range."""
        self._part(oracle, 1, part)

    def even_part(self, oracle, part):
        """The same split of the even step."""
        self._part(oracle, 0, part)

    def idx(self, side, phase, pack):
        own = (phase == 0) == pack
        return (self.lay["own"] if own else self.lay["ghost"])[side]

    # the slab interface of lbmb200.slabs' transports, on CPU torch tensors
    def message(self, side, phase, send):
        i = self.idx(side, phase, send)
        return -1 if i is None else int(i.size)

    def pack(self, side, phase, buf, stream=None):
        import torch
        buf.copy_(torch.from_numpy(self.f[self.idx(side, phase, True)]))

    def unpack(self, side, phase, buf, stream=None):
        self.f[self.idx(side, phase, False)] = buf.numpy()


class SteppedEmuSlab:
    """An EmuSlab behind the library slab's step interface (step, odd_part,
    even_part with lbmb200.slabs.Slab's signatures; cd and stream unused), so
    that lbmb200.slabs.step_pairs drives the oracle-stepped slab exactly as
    it drives a GPU slab."""

    def __init__(self, emu, oracle):
        self.emu, self.oracle = emu, oracle

    def step(self, cd, half, stream=None):
        self.emu.half(self.oracle, half)

    def odd_part(self, cd, part, stream=None):
        self.emu.odd_part(self.oracle, part)

    def even_part(self, cd, part, stream=None):
        self.emu.even_part(self.oracle, part)

    def message(self, side, phase, send):
        return self.emu.message(side, phase, send)

    def pack(self, side, phase, buf, stream=None):
        self.emu.pack(side, phase, buf, stream)

    def unpack(self, side, phase, buf, stream=None):
        self.emu.unpack(side, phase, buf, stream)


def exchange(slabs, faces, phase):
    """The two-phase exchange between in-process slabs: faces are (r, q)
    pairs, q the right-hand neighbour of r."""
    for r, q in faces:
        a, b = slabs[r], slabs[q]
        b.f[b.idx(0, phase, False)] = a.f[a.idx(1, phase, True)]
        a.f[a.idx(1, phase, False)] = b.f[b.idx(0, phase, True)]


def run_slabs(oracle, lat, parts, pairs, init, kargs=(), overlap=False):
    """`pairs` step pairs of `lat` split into `parts` slabs in this process;
    returns the gathered logical field and the slabs. With `overlap`, each
    phase's messages are packed, then the inner tiles take the next step
    (odd after phase 0, the next even after phase 1), then the messages are
    unpacked and the other tiles follow."""
    nx = lat.dims[0]
    ring = sl.is_ring(lat.periodic)
    slabs = []
    for r, (x0, x1) in enumerate(sl.partition(nx, parts)):
        lo, hi = sl.halo_flags(r, parts, ring)
        s = EmuSlab(lat, x0, x1, lo, hi, kargs)
        s.set_field(init)
        slabs.append(s)
    faces = [(r, (r + 1) % parts) for r in range(parts) if sl.neighbours(r, parts, ring)[1] is not None]
    for r, q in faces:
        for phase in (0, 1):
            assert slabs[r].idx(1, phase, True).size == slabs[q].idx(0, phase, False).size
            assert slabs[q].idx(0, phase, True).size == slabs[r].idx(1, phase, False).size
    def send(phase):  # the packed messages, before any step that follows
        return [(a.f[a.idx(1, phase, True)].copy(), b.f[b.idx(0, phase, True)].copy())
                for a, b in ((slabs[r], slabs[q]) for r, q in faces)]

    def receive(phase, sent):
        for (r, q), (to_right, to_left) in zip(faces, sent):
            slabs[q].f[slabs[q].idx(0, phase, False)] = to_right
            slabs[r].f[slabs[r].idx(1, phase, False)] = to_left

    if overlap:
        for s in slabs:
            s.half(oracle, 0)
        for k in range(pairs):
            sent = send(0)
            for s in slabs:
                s.odd_part(oracle, 0)
            receive(0, sent)
            for s in slabs:
                s.odd_part(oracle, 1)
            sent = send(1)
            if k + 1 < pairs:
                for s in slabs:
                    s.even_part(oracle, 0)
            receive(1, sent)
            if k + 1 < pairs:
                for s in slabs:
                    s.even_part(oracle, 1)
    else:
        for _ in range(pairs):
            for s in slabs:
                s.half(oracle, 0)
            exchange(slabs, faces, 0)
            for s in slabs:
                s.half(oracle, 1)
            exchange(slabs, faces, 1)
    out = np.zeros_like(init)
    for s in slabs:
        s.get_field(out)
    return out, slabs
