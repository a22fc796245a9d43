"""Batched FP64 products: many independent products (different systems, sizes, block sizes and
mult types) in one persistent launch over the concatenation of their output-block lists
(cq_mat_mult_batch), against the same products launched one at a time.  Every output element is
computed with the same operations either way, so the results must be identical bit for bit; the
single launches are themselves bit-exact against the oracle (test_gpu_mult.py)."""
import numpy as np
import pytest

import systems
from cq_b200 import inputs

pytestmark = pytest.mark.gpu


def _systems():
    import cq_b200
    out = []
    rng = systems.lnv_ranges(8.0, 9.0, 10.0, 8.0)
    ridx = {k: i for i, k in enumerate(rng)}
    # 64-atom periodic SZ cell, a 44-atom DZP cluster, a 64-atom cell with 4- and 13-orbital atoms
    c1, cell1 = inputs.diamond_si(2, sigma=0.1, seed=31)
    c2, cell2 = inputs.si_cluster(44, sigma=0.1, seed=32)
    c3, cell3 = inputs.diamond_si(2, sigma=0.05, seed=33)
    nsf3 = np.where(np.arange(len(c3)) % 3 == 0, 13, 4).astype(np.int32)
    for c, cell, nsf in ((c1, cell1, np.full(len(c1), 4, np.int32)), (c2, cell2, np.full(len(c2), 13, np.int32)),
                         (c3, cell3, nsf3)):
        out.append((cq_b200.System(c, cell, nsf, list(rng.values())), c, cell))
    return out, ridx


PRODUCTS = [(1, "L", "S", "LS"), (1, "LS", "L", "LSL"), (2, "L", "LS", "LSL"), (2, "H", "LS", "LSL"),
            (1, "T", "H", "TH"), (2, "L", "T", "TL")]


def _operands(g, ridx, t, ra, rb, rc, seed):
    import torch
    dev = torch.device("cuda", 0)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    mk = lambda r: (torch.rand(g.length(ridx[r]), dtype=torch.float64, device=dev, generator=gen) - 0.5)
    a, b, c = mk(ra), mk(rb), mk(rc)
    return a, b, c


@pytest.mark.parametrize("precision_name", ["PREC_FP64", "PREC_FP64_FMA"])
def test_batched_products_equal_separate_launches(precision_name):
    import torch
    import cq_b200
    prec = getattr(cq_b200, precision_name)
    torch.cuda.set_device(0)
    syss, ridx = _systems()
    batch, separate = [], []
    seed = 100
    # 3 systems x 6 products, repeated 6 times with fresh operands: 108 products, more than one launch's table
    for rep in range(6):
        for (g, _, _) in syss:
            for (t, ra, rb, rc) in PRODUCTS:
                seed += 1
                a, b, c = _operands(g, ridx, t, ra, rb, rc, seed)
                out_b = (torch.full_like(c, float("nan")) if t == 1 else torch.full_like(a, float("nan")))
                out_s = out_b.clone()
                if t == 1:
                    batch.append((g, 1, ridx[ra], ridx[rb], ridx[rc], a, b, out_b, prec))
                    separate.append((g, 1, ridx[ra], ridx[rb], ridx[rc], a, b, out_s, prec))
                else:
                    batch.append((g, 2, ridx[ra], ridx[rb], ridx[rc], out_b, b, c, prec))
                    separate.append((g, 2, ridx[ra], ridx[rb], ridx[rc], out_s, b, c, prec))
    torch.cuda.synchronize()
    for (g, t, ra, rb, rc, a, b, c, p) in separate:
        g.mat_mult(t, ra, rb, rc, a, b, c, precision=p)
    for (g, _, _) in syss:
        g.synchronize()
    cq_b200.mat_mult_batch(batch)
    for (g, _, _) in syss:
        g.synchronize()
    assert len(batch) > 96
    for bt, sp in zip(batch, separate):
        ob = bt[7] if bt[1] == 1 else bt[5]
        os_ = sp[7] if sp[1] == 1 else sp[5]
        assert not torch.isnan(ob).any()
        assert torch.equal(ob, os_)
    for (g, _, _) in syss:
        g.close()


def test_batch_rejects_split_precision():
    import torch
    import cq_b200
    syss, ridx = _systems()
    g = syss[0][0]
    a, b, c = _operands(g, ridx, 1, "L", "S", "LS", 7)
    with pytest.raises(cq_b200.CQError):
        cq_b200.mat_mult_batch([(g, 1, ridx["L"], ridx["S"], ridx["LS"], a, b, c, cq_b200.PREC_BF16X3)])
    for (g, _, _) in syss:
        g.close()
