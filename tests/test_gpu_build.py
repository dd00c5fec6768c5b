"""The list layout built on the GPU (lbm_b200_list_build, used by the list
rows' Init and by lbm_batch_add) against the host builder and the oracle,
bit for bit: numbering (blocked orders included) and push/pull adjacency."""
import numpy as np
import pytest

import lbmb200
from lbm_cases import FIELD_CASES

pytestmark = pytest.mark.gpu

CASES = FIELD_CASES + [("fluid", (3, 3, 3), (1, 1, 1)), ("box", (1, 4, 5), (1, 1, 1)),
                       ("channel", (40, 9, 37), (0, 0, 0)), ("box", (7, 6, 5), (0, 1, 0))]


@pytest.mark.parametrize("pull", [0, 1])
@pytest.mark.parametrize("geo,dims,per", CASES)
def test_device_build_equals_host_build(geo, dims, per, pull):
    lat = lbmb200.geometry(geo, dims, per)
    g1, a1, n1, c1 = lbmb200.list_build(lat, pull)
    g2, a2, n2, c2 = lbmb200.list_build_device(lat, pull)
    assert (n1, c1) == (n2, c2) == (lat.n_fluid, c1)
    assert np.array_equal(g1, g2) and np.array_equal(a1, a2)


@pytest.mark.parametrize("blk", [(4, 4, 4), (3, 5, 7), (1, 1, 2), (0, 3, 0)])
def test_device_build_blocked_numbering(oracle, blk):
    lat = lbmb200.geometry("blocks-2", (13, 11, 12), (0, 1, 0))
    g1, a1, _, _ = lbmb200.list_build(lat, 0, blk=blk)
    g2, a2, _, _ = lbmb200.list_build_device(lat, 0, blk=blk)
    assert np.array_equal(g1, g2) and np.array_equal(a1, a2)
    g3, a3, _, _ = oracle.list_layout(0, lat.dims, lat.periodic, lat.mask, blk=blk)
    assert np.array_equal(g2, g3) and np.array_equal(a2, a3)


def test_device_build_large_packing():
    lat, _ = lbmb200.spheres((96, 80, 72), 3, 0.45, 3.0, 8.0)
    g1, a1, n1, _ = lbmb200.list_build(lat, 0)
    g2, a2, n2, _ = lbmb200.list_build_device(lat, 0)
    assert n1 == n2 == lat.n_fluid
    assert np.array_equal(g1, g2) and np.array_equal(a1, a2)
