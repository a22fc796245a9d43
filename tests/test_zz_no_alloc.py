"""cq_exact_dots_noalloc: exact traces for callers that cannot allocate device memory (a host that
has handed the whole device to its own pool, or a loop that must not synchronise the device in
cudaMalloc/cudaFree).  Its scratch is a static device array; the values must be bit-identical to
the library's allocating entry point, cq_matrix_product_trace, on two calls in a row (the second
call must not see what the first left in the shared array)."""
import numpy as np
import pytest

import systems

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sysL():
    import cq_b200
    coords, cell, nsf = systems.config2(ncell=2, sigma=0.1, seed=9)
    g = cq_b200.System(coords, cell, nsf, [10.0, 16.0])
    return g


def _rand(n, seed, scale=1.0):
    import torch
    r = np.random.default_rng(seed).uniform(-1.0, 1.0, n) * scale
    return torch.tensor(r, dtype=torch.float64, device="cuda")


def test_noalloc_matches_product_trace_twice(sysL):
    import torch
    import cq_b200
    g = sysL
    n = g.length(1)
    a, b = _rand(n, 1), _rand(n, 2, 1e3)
    ones = torch.ones(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()     # the library works on its own stream
    ref = [g.product_trace(1, a, b), g.product_trace(1, a, a), g.product_trace(1, b, ones)]
    got = cq_b200.exact_dots_noalloc([a, a, b], [b, a, None])
    assert got == ref
    # second call in a row: other data, fewer sums, a zero vector and a tiny-magnitude one
    c, d = _rand(n, 3, 1e-200), torch.zeros(n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    ref2 = [g.product_trace(1, c, ones), g.product_trace(1, d, a)]
    got2 = cq_b200.exact_dots_noalloc([c, d], [None, a])
    assert got2 == ref2
    assert got2[1] == 0.0


def test_noalloc_rejects_too_many_sums(sysL):
    import torch
    import cq_b200
    a = _rand(sysL.length(0), 4)
    ones = torch.ones_like(a)
    torch.cuda.synchronize()
    with pytest.raises(cq_b200.CQError) as e:
        cq_b200.exact_dots_noalloc([a] * (cq_b200.NOALLOC_MAX_SUMS + 1))
    assert e.value.code == cq_b200.CQ_ERR_ARG
    assert "CQ_NOALLOC_MAX_SUMS" in str(e.value)
    # the maximum itself is accepted
    vals = cq_b200.exact_dots_noalloc([a] * cq_b200.NOALLOC_MAX_SUMS)
    assert len(set(vals)) == 1 and vals[0] == sysL.product_trace(0, a, ones)
