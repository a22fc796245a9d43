"""Device-side synthetic S and H against the host generators of cq_b200.inputs.

The generators are integer hashing plus one exp() per block; the hash is bit-identical and exp()
may differ from numpy's in the last place, so the comparison allows 2 ulp relative.
"""
import numpy as np
import pytest

import systems
from cq_b200 import inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nsf", [4, 13])
def test_generated_S_H_match_host(nsf):
    import torch
    import cq_b200
    coords, cell, _ = systems.config2(ncell=2, sigma=0.1, seed=3)
    n = len(coords)
    g = cq_b200.System(coords, cell, np.full(n, nsf, np.int32), [10.0, 12.0])
    for r, which in ((0, 0), (1, 1)):
        bl = g.blocklist(r, coords, cell)
        host = inputs.overlap_S(bl) if which == 0 else inputs.hamiltonian_H(bl, seed=7)
        dev = torch.full((g.length(r),), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()      # torch's stream and the library's stream are different
        g.generate_SH(r, which, 7, dev)
        g.synchronize()
        got = dev.cpu().numpy()
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, host, rtol=4.5e-16, atol=0.0)
        # the onsite blocks carry no exp() and are bit-identical
        onsite = (bl.ig_i == bl.ig_j) & np.all(bl.shift == 0, axis=1)
        for q in np.nonzero(onsite)[0]:
            s = slice(bl.elem_off[q], bl.elem_off[q] + nsf * nsf)
            assert np.array_equal(got[s], host[s])
