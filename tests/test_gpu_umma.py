"""Split-precision block products on the tcgen05 tensor cores (dense 128 x 128 tiles, TMEM
accumulators) against the oracle's FP64 default kernel.

Every operand value is split into two bf16 parts (hi + lo, about 16 significant bits) and a block
product is hi.hi + hi.lo + lo.hi with FP32 accumulation, so per output element
    |got - ref| <= 2^-14 * sum |a| |b| over the element's terms
(the same bound as the per-block mma.sync kernel).  The output is fully overwritten: blocks with no
terms come out as zeros, never as the NaNs the output held before.
"""
import numpy as np
import pytest

import blockmaps as bm
import systems
from cq_b200 import inputs
from cq_oracle import OracleSystem

pytestmark = pytest.mark.gpu

TOL = 2.0 ** -14


def _run(o, g, t, ia, ib, ic, bls_a, bls_b, bls_c, seed, kernel=0, precision=None):
    """One product on both sides; returns (got, ref, sum |a||b| bound)."""
    import cq_b200
    g.set_mixed_kernel(kernel)
    prec = cq_b200.PREC_BF16X3 if precision is None else precision
    b = inputs.random_blocks(bls_b, seed, inputs.TAG_RANDOM_B)
    if t == 1:
        a = inputs.random_blocks(bls_a, seed, inputs.TAG_RANDOM_A)
        ref = np.zeros(bls_c.length); o.mat_mult(1, ia, ib, ic, a, b, ref)
        bound = np.zeros(bls_c.length); o.mat_mult(1, ia, ib, ic, np.abs(a), np.abs(b), bound)
        got = np.full(bls_c.length, np.nan)
        g.mat_mult_host(1, ia, ib, ic, a, b, got, precision=prec)
    else:
        c = inputs.random_blocks(bls_c, seed + 1, inputs.TAG_RANDOM_A)
        ref = np.zeros(bls_a.length); o.mat_mult(2, ia, ib, ic, ref, b, c)
        bound = np.zeros(bls_a.length); o.mat_mult(2, ia, ib, ic, bound, np.abs(b), np.abs(c))
        got = np.full(bls_a.length, np.nan)
        g.mat_mult_host(2, ia, ib, ic, got, b, c, precision=prec)
    return got, ref, bound


def _assert_bound(got, ref, bound, tol=TOL):
    assert not np.any(np.isnan(got)), "output blocks left unwritten"
    err = np.abs(got - ref)
    worst = np.max(err / np.maximum(bound, 1e-300))
    assert np.all(err <= tol * bound + 1e-300), "worst error / sum|a||b| = %.3g" % worst
    assert err.max() > 0          # it really ran in reduced precision
    return worst


@pytest.fixture(scope="module")
def cfg1():
    import cq_b200
    coords, cell, nsf, rc = systems.config1()
    o = OracleSystem(coords, cell, nsf, rc)
    g = cq_b200.System(coords, cell, nsf, rc)
    bls = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    return o, g, bls


@pytest.fixture(scope="module")
def cfg2():
    import cq_b200
    coords, cell, nsf = systems.config2()
    rng = systems.lnv_ranges()
    names = list(rng.keys())
    o = OracleSystem(coords, cell, nsf, list(rng.values()))
    g = cq_b200.System(coords, cell, nsf, list(rng.values()))
    bls = {n: bm.oracle_blocklist(o, i, coords, cell) for i, n in enumerate(names)}
    return o, g, bls, {n: i for i, n in enumerate(names)}


@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("mult_type", [1, 2])
def test_dzp_products_within_split_bound(cfg1, mult_type, kernel):
    """216-atom Si, 13x13 blocks, A 8 / B 12 / C 20 bohr: tcgen05 tiles (0) and per-block mma.sync (1)."""
    o, g, bls = cfg1
    got, ref, bound = _run(o, g, mult_type, 0, 1, 2, bls[0], bls[1], bls[2], 41 + mult_type, kernel)
    _assert_bound(got, ref, bound)


def test_tile_plan_accounts_for_the_work(cfg1):
    """The tiles cover the product: the issued tensor work is at least the three split terms of every
    useful triple, and the plan is usable for 13x13 blocks."""
    o, g, bls = cfg1
    tiles, issued, usable = g.product_tensor_work(1, 0, 1, 2)
    triples, flops = g.product_work(1, 0, 1, 2)
    assert usable and tiles > 0
    assert issued >= 3 * flops
    # 128 x 128 tiles, K padded to 32: the tile count bounds the issued work from above
    assert issued <= 3 * 2 * 128 * 128 * tiles * (triples * 13 // max(tiles, 1) + 32 * tiles)


SZ_PRODUCTS = [(1, "L", "S", "LS"), (1, "LS", "L", "LSL"), (2, "L", "LS", "LSL"), (2, "H", "LS", "LSL"),
               (1, "LS", "S", "SLS"), (2, "L", "T", "TL")]


@pytest.mark.parametrize("prod", SZ_PRODUCTS)
def test_sz_products_within_split_bound(cfg2, prod):
    """512-atom Si, 4x4 blocks (32 atoms per 128-row tile), products of the LNV chain, both mult types."""
    o, g, bls, idx = cfg2
    t, ra, rb, rc = prod
    got, ref, bound = _run(o, g, t, idx[ra], idx[rb], idx[rc], bls[ra], bls[rb], bls[rc], 51)
    _assert_bound(got, ref, bound)
    assert g.product_tensor_work(t, idx[ra], idx[rb], idx[rc])[2]


@pytest.mark.parametrize("mult_type", [1, 2])
def test_mixed_block_sizes_within_split_bound(mult_type):
    """Atoms with 4 and 13 orbitals in one system: atoms of both sizes packed into the same tiles."""
    import cq_b200
    coords, cell = inputs.diamond_si(2, sigma=0.05, seed=21)
    nsf = np.where(np.arange(len(coords)) % 3 == 0, 13, 4).astype(np.int32)
    rc = [6.0, 8.0, 14.0]
    o = OracleSystem(coords, cell, nsf, rc)
    g = cq_b200.System(coords, cell, nsf, rc)
    bls = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    got, ref, bound = _run(o, g, mult_type, 0, 1, 2, bls[0], bls[1], bls[2], 61)
    _assert_bound(got, ref, bound)


def test_repeatable_bits(cfg1):
    """The tiles accumulate in a fixed order: two launches give the same bits."""
    o, g, bls = cfg1
    got1, _, _ = _run(o, g, 1, 0, 1, 2, bls[0], bls[1], bls[2], 71)
    got2, _, _ = _run(o, g, 1, 0, 1, 2, bls[0], bls[1], bls[2], 71)
    assert np.array_equal(got1, got2)


def test_bounded_wait_reports_timeout_and_context_survives(cfg1):
    """A tensor-core product whose bulk-copy thread stops after taking its first tile (test hook): the
    MMA thread's bounded wait runs out after about a second, the kernel drains and releases its tensor
    memory, and the host reports CQ_ERR_TIMEOUT.  The next product on the same context is correct."""
    import cq_b200
    o, g, bls = cfg1
    g.set_mixed_kernel(0)
    a = inputs.random_blocks(bls[0], 81, inputs.TAG_RANDOM_A)
    b = inputs.random_blocks(bls[1], 81, inputs.TAG_RANDOM_B)
    out = np.zeros(bls[2].length)
    g.test_stall_next_tensor_product()
    with pytest.raises(cq_b200.CQError) as ei:
        g.mat_mult_host(1, 0, 1, 2, a, b, out, precision=cq_b200.PREC_BF16X3)
    assert ei.value.code == cq_b200.CQ_ERR_TIMEOUT
    got, ref, bound = _run(o, g, 1, 0, 1, 2, bls[0], bls[1], bls[2], 82)
    _assert_bound(got, ref, bound)


# Three-part split (BF16x6): v = hi + mid + lo, six products per block pair, each pair's 16 x 16 x 16
# product rounded to FP32 once and the pairs summed in FP64.  The omitted products and split
# remainders are below 2^-23 |a||b| per element product and the FP32 rounding of a pair's product
# adds at most a few 2^-24 of its magnitude, so 2^-20 sum |a||b| bounds the error with margin.
TOL6 = 2.0 ** -20


@pytest.mark.parametrize("mult_type", [1, 2])
def test_three_part_split_dzp_within_bound(cfg1, mult_type):
    """216-atom Si, 13x13 blocks: the three-part split against the FP64 default kernel, and at least
    2^6 times more accurate than the two-part split on the same product."""
    import cq_b200
    o, g, bls = cfg1
    got6, ref, bound = _run(o, g, mult_type, 0, 1, 2, bls[0], bls[1], bls[2], 91 + mult_type,
                            precision=cq_b200.PREC_BF16X6)
    w6 = _assert_bound(got6, ref, bound, TOL6)
    got3, _, _ = _run(o, g, mult_type, 0, 1, 2, bls[0], bls[1], bls[2], 91 + mult_type, kernel=1)
    w3 = _assert_bound(got3, ref, bound)
    print("worst error / sum|a||b|: three-part %.3g, two-part %.3g" % (w6, w3))
    assert w6 * 64 < w3


@pytest.mark.parametrize("prod", SZ_PRODUCTS[:3])
def test_three_part_split_sz_within_bound(cfg2, prod):
    """512-atom Si, 4x4 blocks (padded to 16 x 16), products of the LNV chain."""
    import cq_b200
    o, g, bls, idx = cfg2
    t, ra, rb, rc = prod
    got, ref, bound = _run(o, g, t, idx[ra], idx[rb], idx[rc], bls[ra], bls[rb], bls[rc], 93,
                           precision=cq_b200.PREC_BF16X6)
    _assert_bound(got, ref, bound, TOL6)


def test_three_part_split_mixed_sizes_within_bound():
    """Atoms with 4 and 13 orbitals in one system."""
    import cq_b200
    coords, cell = inputs.diamond_si(2, sigma=0.05, seed=21)
    nsf = np.where(np.arange(len(coords)) % 3 == 0, 13, 4).astype(np.int32)
    rc = [6.0, 8.0, 14.0]
    o = OracleSystem(coords, cell, nsf, rc)
    g = cq_b200.System(coords, cell, nsf, rc)
    bls = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    for t in (1, 2):
        got, ref, bound = _run(o, g, t, 0, 1, 2, bls[0], bls[1], bls[2], 95, precision=cq_b200.PREC_BF16X6)
        _assert_bound(got, ref, bound, TOL6)


@pytest.mark.parametrize("precision_name", ["PREC_BF16X3", "PREC_BF16X6"])
def test_split_group_sizes_give_the_same_bits(cfg1, precision_name):
    """The mma.sync split kernels with 1, 2, 4 (and 8) output blocks per warp: the same bits."""
    import cq_b200
    o, g, bls = cfg1
    prec = getattr(cq_b200, precision_name)
    sizes = [1, 2, 4, 8] if prec == cq_b200.PREC_BF16X3 else [1, 2, 4]
    outs = []
    try:
        for gs in sizes:
            g.set_split_group(gs)
            for t in (1, 2):
                got, _, _ = _run(o, g, t, 0, 1, 2, bls[0], bls[1], bls[2], 97, kernel=1, precision=prec)
                outs.append((gs, t, got))
    finally:
        g.set_split_group(-1)
    for t in (1, 2):
        ref = [x for gs, tt, x in outs if tt == t]
        for x in ref[1:]:
            assert np.array_equal(x, ref[0])


# FP64 on the tensor cores (DMMA): FP64 products and sums in another order than the reference kernel,
# so per element |got - ref| is a few units of 2^-53 sum |a||b| (bounded here by 1e-14).
TOL_TC = 1e-14


@pytest.mark.parametrize("mult_type", [1, 2])
def test_fp64_tensor_dzp_within_bound(cfg1, mult_type):
    """216-atom Si, 13x13 blocks (two 8 x 8 tiles per dimension, the second partly padding)."""
    import cq_b200
    o, g, bls = cfg1
    got, ref, bound = _run(o, g, mult_type, 0, 1, 2, bls[0], bls[1], bls[2], 101 + mult_type,
                           precision=cq_b200.PREC_FP64_TC)
    assert not np.any(np.isnan(got))
    err = np.abs(got - ref)
    print("FP64 tensor cores: worst error / sum|a||b| = %.3g" % np.max(err / np.maximum(bound, 1e-300)))
    assert np.all(err <= TOL_TC * bound + 1e-300)


@pytest.mark.parametrize("prod", SZ_PRODUCTS[:3])
def test_fp64_tensor_sz_within_bound(cfg2, prod):
    """512-atom Si, 4x4 blocks (one 8 x 8 tile per block, mostly padding)."""
    import cq_b200
    o, g, bls, idx = cfg2
    t, ra, rb, rc = prod
    got, ref, bound = _run(o, g, t, idx[ra], idx[rb], idx[rc], bls[ra], bls[rb], bls[rc], 103,
                           precision=cq_b200.PREC_FP64_TC)
    assert not np.any(np.isnan(got))
    assert np.all(np.abs(got - ref) <= TOL_TC * bound + 1e-300)


def test_fp64_tensor_mixed_sizes_within_bound():
    """Atoms with 4 and 13 orbitals in one system: tiles of different counts per block."""
    import cq_b200
    coords, cell = inputs.diamond_si(2, sigma=0.05, seed=21)
    nsf = np.where(np.arange(len(coords)) % 3 == 0, 13, 4).astype(np.int32)
    rc = [6.0, 8.0, 14.0]
    o = OracleSystem(coords, cell, nsf, rc)
    g = cq_b200.System(coords, cell, nsf, rc)
    bls = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    for t in (1, 2):
        got, ref, bound = _run(o, g, t, 0, 1, 2, bls[0], bls[1], bls[2], 105, precision=cq_b200.PREC_FP64_TC)
        assert not np.any(np.isnan(got))
        assert np.all(np.abs(got - ref) <= TOL_TC * bound + 1e-300)


@pytest.mark.parametrize("mult_type", [1, 2])
def test_fp64_tensor_equals_fused_multiply_add_kernel(cfg1, mult_type):
    """Measured property of the B200 FP64 tensor cores: an m8n8k4 MMA sums its four products into the
    accumulator as a chain of fused multiply-adds in k order, so the DMMA product gives the bits of the
    CUDA-core FP64 kernels with fused multiply-add (variants 4 and 0 forced) and of the oracle's default
    kernel with fused multiply-add, which take the same terms in the same order."""
    import cq_b200
    o, g, bls = cfg1
    tc, _, _ = _run(o, g, mult_type, 0, 1, 2, bls[0], bls[1], bls[2], 107, precision=cq_b200.PREC_FP64_TC)
    outs = []
    try:
        for v in (4, 0):      # the CUDA-core kernels (register tiles; one lane per element)
            g.set_mult_variant(v)
            fma, _, _ = _run(o, g, mult_type, 0, 1, 2, bls[0], bls[1], bls[2], 107, precision=cq_b200.PREC_FP64_FMA)
            outs.append(fma)
    finally:
        g.set_mult_variant(-1)
    for fma in outs:
        assert np.array_equal(tc, fma)
    # and the oracle's default kernel with each multiply-add fused, the terms in the reference's order
    b = inputs.random_blocks(bls[1], 107, inputs.TAG_RANDOM_B)
    if mult_type == 1:
        a = inputs.random_blocks(bls[0], 107, inputs.TAG_RANDOM_A)
        ref = np.zeros(bls[2].length); o.mat_mult(1, 0, 1, 2, a, b, ref, kernel="default_fma")
    else:
        c = inputs.random_blocks(bls[2], 108, inputs.TAG_RANDOM_A)
        ref = np.zeros(bls[0].length); o.mat_mult(2, 0, 1, 2, ref, b, c, kernel="default_fma")
    assert np.array_equal(tc, ref)
