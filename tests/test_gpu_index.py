"""GPU index construction vs the oracle: bit-exact neighbour lists, halos, retro lists, transposes."""
import numpy as np
import pytest

import systems
from cq_oracle import OracleSystem

pytestmark = pytest.mark.gpu

GEOM = ["n_parts", "ngnode", "nm_group", "ig_prim", "lab_cell", "lab_cover", "n_ing_cover", "icover_ibeg",
        "ig_cover", "iprim_group"]
RANGE = ["n_nab", "i_acc", "i_nd_acc", "ndimi", "onsite", "i_part", "i_seq", "ndimj", "npxyz", "bind", "halo_sizes",
         "nh_part", "j_beg", "lab_hcell", "lab_hcover", "j_seq", "halo_ndimj", "i_halo", "i_h2d", "t_i_prim", "t_i_beg",
         "t_i_nd_beg", "t_n_hnab", "itran_addr"]


def _pair(coords, cell, nsf, rc):
    import cq_b200
    return OracleSystem(coords, cell, nsf, rc), cq_b200.System(coords, cell, nsf, rc)


@pytest.fixture(scope="module")
def cfg1():
    coords, cell, nsf, rc = systems.config1()
    return _pair(coords, cell, nsf, rc)


@pytest.fixture(scope="module")
def cfg2():
    coords, cell, nsf = systems.config2()
    return _pair(coords, cell, nsf, list(systems.lnv_ranges().values()))


@pytest.mark.parametrize("name", GEOM)
def test_geometry_arrays(cfg1, name):
    o, g = cfg1
    assert np.array_equal(o.geti(name), g.geti(name))


def test_cover_dims(cfg2):
    o, g = cfg2
    assert np.array_equal(o.geti("cover_dims")[:8], g.geti("cover_dims"))


def test_blocklists_identical(cfg2):
    """The product's layout description equals the oracle's, so generated inputs are identical."""
    import systems as _s
    o, g = cfg2
    coords, cell, _ = _s.config2()
    for r in range(len(o.rcuts)):
        a, b = o.blocklist(r, coords, cell), g.blocklist(r, coords, cell)
        for k in ("ig_i", "ig_j", "shift", "radius", "nd_i", "nd_j", "elem_off"):
            assert np.array_equal(getattr(a, k), getattr(b, k)), (r, k)


@pytest.mark.parametrize("cfg", ["cfg1", "cfg2"])
def test_range_arrays_bit_exact(cfg, request):
    o, g = request.getfixturevalue(cfg)
    for r in range(len(o.rcuts)):
        assert o.length(r) == g.length(r)
        for name in RANGE:
            a, b = o.geti(name, r), g.geti(name, r)
            assert a.shape == b.shape and np.array_equal(a, b), (cfg, r, name)
        assert np.array_equal(o.getd("radius", r), g.radius(r))
