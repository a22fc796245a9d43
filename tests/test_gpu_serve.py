"""Serving loop on the GPU: every result is the same alone and in the mix.

Each solve is deterministic (exact reductions, fixed kernels), so the energy, electron count and
work of a request are compared bit for bit between a one-slot server (requests run one after
another) and a four-slot server (all requests overlap on the device), and against the direct
LNV entry point fed with the same device-generated S and H.
"""
import numpy as np
import pytest

import cq_b200
from cq_b200 import inputs

pytestmark = pytest.mark.gpu

RANGES = (8.0, 9.0, 10.0, 8.0)


def _requests():
    out = []
    c, cell = inputs.si_cluster(40, sigma=0.1, seed=11)
    out.append((c, cell, 4, float(len(c)), 101, False))
    c, cell = inputs.diamond_si(2, sigma=0.1, seed=12)
    out.append((c, cell, 4, float(len(c)), 102, False))
    c, cell = inputs.si_cluster(30, sigma=0.1, seed=13)
    out.append((c, cell, 13, 2.0 * len(c), 103, False))
    c, cell = inputs.si_cluster(52, sigma=0.1, seed=14)
    out.append((c, cell, 4, float(len(c)), 104, True))
    c, cell = inputs.diamond_si(1, sigma=0.1, seed=15)
    out.append((c, cell, 13, 2.0 * len(c), 105, True))
    return out


def _run(server, reqs, ranges=RANGES):
    ids = [server.submit(c, cell, nsf, *ranges, ne, seed=seed, mixed=mx) for c, cell, nsf, ne, seed, mx in reqs]
    return [server.wait(i, timeout=600) for i in ids]


def _key(r):
    return (r["energy"], r["electrons"], r["n_products"], r["flops"], r["n_products_mixed"], r["converged"])


def test_batched_products_alone_equals_mix():
    """Four slots whose FP64 products are gathered into shared persistent launches (batch_products)
    give the same bits as a one-slot server without gathering: the gathered launches compute every
    output block exactly as a product of its own."""
    reqs = _requests()
    alone = cq_b200.Server(n_slots=1, max_outer=3)
    ra = _run(alone, reqs)
    alone.close()
    mix = cq_b200.Server(n_slots=4, max_outer=3, batch_products=True, batch_window_us=100.0)
    rm = _run(mix, reqs)
    mix.close()
    for a, m in zip(ra, rm):
        assert a["status"] == 0 and m["status"] == 0, (a["message"], m["message"])
        assert _key(a) == _key(m)


def test_alone_equals_mix():
    reqs = _requests()
    alone = cq_b200.Server(n_slots=1, max_outer=3)
    ra = _run(alone, reqs)
    alone.close()
    mix = cq_b200.Server(n_slots=4, max_outer=3)
    rm = _run(mix, reqs)
    mix.close()
    for a, m in zip(ra, rm):
        assert a["status"] == 0 and m["status"] == 0, (a["message"], m["message"])
        assert a["n_products"] > 0
        assert _key(a) == _key(m)
    # the four-slot run overlapped solves
    ev = sorted([(r["t_admit"], 1) for r in rm] + [(r["t_done"], -1) for r in rm])
    cur = best = 0
    for _, d in ev:
        cur += d
        best = max(best, cur)
    assert best >= 2
    for r in ra + rm:
        assert 0 < r["bytes_peak"] <= r["bytes_estimate"]


def test_server_equals_direct_solver():
    import torch
    c, cell, nsf, ne, seed, mixed = _requests()[1]
    srv = cq_b200.Server(n_slots=2, max_outer=2)
    r = _run(srv, [(c, cell, nsf, ne, seed, mixed)])[0]
    srv.close()
    rng = cq_b200.lnv_ranges(*RANGES)
    g = cq_b200.System(c, cell, np.full(len(c), nsf, np.int32), list(rng.values()))
    ridx = {n: i for i, n in enumerate(rng)}
    S = torch.zeros(g.length(ridx["S"]), dtype=torch.float64, device="cuda")
    H = torch.zeros(g.length(ridx["H"]), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()          # torch's stream and the library's stream are different
    g.generate_SH(ridx["S"], 0, seed, S)
    g.generate_SH(ridx["H"], 1, seed, H)
    g.synchronize()
    lnv = cq_b200.LNV(g, ridx, ne, max_outer=2)
    lnv.set_SH(S, H)
    d = lnv.solve()
    assert (d["energy"], d["electrons"], d["n_products"]) == (r["energy"], r["electrons"], r["n_products"])


@pytest.mark.parametrize("split_parts", [2, 3])
def test_mixed_request_accuracy(split_parts):
    """Split-precision phase then FP64 continuation: same minimum as the FP64 solve within 1e-8 Ha/atom
    (a 30-atom DZP cluster with L and T ranges beyond its diameter, so the minimum is well defined), for
    the two-part (hand-over at 1e-6) and three-part (hand-over at 1e-8) splits.

    Both solves stop at a residual of 1e-9: at the default 1e-7 two solves of the same problem from
    different starting points already differ by about 1e-7 Ha/atom, whatever their arithmetic."""
    c, cell = inputs.si_cluster(30, sigma=0.1, seed=16)
    n = len(c)
    diam = float(np.max(np.linalg.norm(c[:, None] - c[None], axis=-1)))
    rg = (10.0, 12.0, diam + 1.0, diam + 1.0)
    srv = cq_b200.Server(n_slots=2, tolerance=1e-9, split_parts=split_parts)
    fp = _run(srv, [(c, cell, 13, 2.0 * n, 7, False)], rg)[0]
    mx = _run(srv, [(c, cell, 13, 2.0 * n, 7, True)], rg)[0]
    srv.close()
    assert fp["converged"] == 1 and mx["converged"] == 1
    assert mx["n_products_mixed"] > 0
    assert abs(mx["energy"] - fp["energy"]) / n < 1e-8
    assert abs(mx["electrons"] - fp["electrons"]) < 1e-6


def test_mixed_vs_fp64_truncated_dzp216():
    """The precision form on a config-3-shaped system: a truncated 216-atom DZP supercell (3x3x3 cells,
    sigma 0.1 bohr, 13x13 blocks, S/H/L/T 10/12/16/10 bohr, 432 electrons), FP64 and mixed (three-part
    split products to residual 1e-8 within four passes, then FP64) both to residual 1e-8 within 12
    passes.  Measured on B200: see the printed |dE| per atom; the bound is 4x the band that the
    FP64 path's own rounding spans at that stop."""
    c, cell = inputs.diamond_si(3, sigma=0.1, seed=77)
    srv = cq_b200.Server(n_slots=2, max_outer=12, tolerance=1e-8)
    ids = [srv.submit(c, cell, 13, 10.0, 12.0, 16.0, 10.0, 2.0 * len(c), seed=777, mixed=m) for m in (False, True)]
    fp, mx = [srv.wait(i, timeout=1200) for i in ids]
    srv.close()
    assert fp["status"] == 0 and mx["status"] == 0, (fp["message"], mx["message"])
    de = abs(mx["energy"] - fp["energy"]) / len(c)
    print("216-atom DZP: FP64 E = %.12f (converged %d, residual %.3g), mixed E = %.12f (converged %d, residual %.3g), "
          "|dE| = %.3g Ha/atom, split-precision products %d of %d" %
          (fp["energy"], fp["converged"], fp["residual"], mx["energy"], mx["converged"], mx["residual"], de,
           mx["n_products_mixed"], mx["n_products"]))
    assert fp["converged"] and mx["converged"]
    assert mx["n_products_mixed"] > 0
    # at this stop the FP64 path with fused multiply-add instead of separate multiply and add already
    # ends 6.2e-8 Ha/atom from it (measured on B200), and a 1e-9 stop is not reached by either arm on
    # this truncated system; the mixed form measured 1.65e-7
    assert de <= 2.5e-7
