"""The run-compressed adjacency the list steps read (lbm_b200_run_records):
decoded in numpy, every node's 18 links equal its full adjacency row (the
reference's encoding, lbm_b200_list_layout), for push and pull layouts,
blocked numbering and padding; the header's prefix counts match the mask."""
import ctypes

import numpy as np
import pytest

import lbmb200

pytestmark = pytest.mark.gpu


def _decode(offs, rec, n_fluid):
    out = np.zeros((n_fluid, 18), dtype=np.int64)
    for t in range(len(offs) - 1):
        r = rec[offs[t] * 4: offs[t + 1] * 4]
        mask = r[:8]
        heads = [k for k in range(256) if (int(mask[k >> 5]) >> (k & 31)) & 1]
        for w in range(8):
            before = sum(bin(int(m)).count("1") for m in mask[:w])
            assert (int(r[8 + (w >> 2)]) >> (8 * (w & 3))) & 0xFF == before
        assert r[10] == 0 and r[11] == 0
        h2 = (len(heads) + 1) & ~1
        assert len(r) == 12 + 18 * h2
        rows = r[12:].reshape(-1, 18).astype(np.int64)
        for k in range(256):
            n = t * 256 + k
            if n >= n_fluid:
                break
            rank = sum(1 for h in heads if h <= k) - 1
            out[n] = rows[rank] + (k - heads[rank])
    return out


@pytest.mark.parametrize("kname,kargs", [
    ("cuda-list-aa-pv-soa", ["-pad", "no"]),
    ("cuda-list-aa-pv-soa", ["-blk", "4"]),
    ("cuda-list-pull-split-nt-1s-soa", []),
    ("cuda-list-push-soa", ["-pad", "no"]),
])
def test_run_records_decode_to_full_adjacency(kname, kargs):
    lat, _ = lbmb200.spheres((24, 20, 18), 11, 0.45, 2.0, 4.0, 3000)
    inst = lbmb200.kernel(kname).init(lat, kernel_args=kargs)
    try:
        grid, adj, nf, nc = inst.list_layout()
        L = lbmb200.lib()
        L.lbm_b200_adjacency_bytes.restype = ctypes.c_longlong
        nbytes = L.lbm_b200_adjacency_bytes(inst.kdp)
        tiles = (nf + 255) // 256
        offs = np.zeros(tiles + 1, dtype=np.uint32)
        rec = np.zeros(nbytes // 4, dtype=np.uint32)
        assert L.lbm_b200_run_records(inst.kdp, offs.ctypes.data_as(ctypes.c_void_p),
                                      rec.ctypes.data_as(ctypes.c_void_p)) == 0
        assert int(offs[-1]) * 16 == nbytes
        got = _decode(offs.astype(np.int64), rec, nf)
        assert np.array_equal(got, adj.reshape(-1, 18).astype(np.int64))
        # fewer bytes than the full rows at this packing
        assert nbytes < nf * 72
    finally:
        inst.deinit()
