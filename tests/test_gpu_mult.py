"""GPU mat_mult, drop-in kernels and algebra vs the oracle.

FP64 with exact=True keeps the default kernel's separate multiply and add per
term in the same order, so results must equal the oracle bit for bit.  The
fused variant (exact=False) must stay within 1e-12 relative per element,
measured against sum |a||b| of the element's terms.
"""
import numpy as np
import pytest

import blockmaps as bm
import dropin_driver
import systems
from cq_b200 import inputs
from cq_oracle import OracleSystem

pytestmark = pytest.mark.gpu


def _sys(coords, cell, nsf, rc):
    import cq_b200
    return OracleSystem(coords, cell, nsf, rc), cq_b200.System(coords, cell, nsf, rc)


@pytest.fixture(scope="module")
def cfg1():
    coords, cell, nsf, rc = systems.config1()
    o, g = _sys(coords, cell, nsf, rc)
    bls = [bm.oracle_blocklist(o, r, coords, cell) for r in range(len(rc))]
    return o, g, bls


@pytest.fixture(scope="module")
def cfg2():
    coords, cell, nsf = systems.config2()
    rng = systems.lnv_ranges()
    names = list(rng.keys())
    o, g = _sys(coords, cell, nsf, list(rng.values()))
    bls = {n: bm.oracle_blocklist(o, i, coords, cell) for i, n in enumerate(names)}
    idx = {n: i for i, n in enumerate(names)}
    return o, g, bls, idx


def _abs_bound(o, mult_type, ra, rb, rc, a, b, c):
    """sum |a||b| per output element, from the oracle run on absolute values."""
    aa, bb, cc = np.abs(a), np.abs(b), np.abs(c)
    if mult_type == 1:
        out = np.zeros_like(c)
        o.mat_mult(1, ra, rb, rc, aa, bb, out)
    else:
        out = np.zeros_like(a)
        o.mat_mult(2, ra, rb, rc, out, bb, cc)
    return out


@pytest.mark.parametrize("variant", [-1, 0, 4])
def test_type1_dzp_bit_exact(cfg1, variant):
    o, g, bls = cfg1
    g.set_mult_variant(variant)
    a = inputs.random_blocks(bls[0], 11, inputs.TAG_RANDOM_A)
    b = inputs.random_blocks(bls[1], 11, inputs.TAG_RANDOM_B)
    c_ref = np.zeros(bls[2].length)
    o.mat_mult(1, 0, 1, 2, a, b, c_ref)
    c = np.full(bls[2].length, np.nan)
    g.mat_mult_host(1, 0, 1, 2, a, b, c, exact=True)
    assert np.array_equal(c, c_ref)
    c2 = np.zeros(bls[2].length)
    g.mat_mult_host(1, 0, 1, 2, a, b, c2, exact=False)
    bound = _abs_bound(o, 1, 0, 1, 2, a, b, c_ref)
    assert np.all(np.abs(c2 - c_ref) <= 1e-12 * bound + 1e-300)
    # algorithmic work matches the triple count of the default kernel
    t, f = g.product_work(1, 0, 1, 2)
    assert f == 2 * 13 ** 3 * t and t > 0


@pytest.mark.parametrize("mult_type", [1, 2])
def test_bf16x3_tensor_core_products(cfg1, mult_type):
    """Split-precision products: per element within 2^-14 of sum |a||b| (about 16 bits per term)."""
    import cq_b200
    o, g, bls = cfg1
    b = inputs.random_blocks(bls[1], 13, inputs.TAG_RANDOM_B)
    if mult_type == 1:
        a = inputs.random_blocks(bls[0], 13, inputs.TAG_RANDOM_A)
        ref = np.zeros(bls[2].length); o.mat_mult(1, 0, 1, 2, a, b, ref)
        got = np.zeros(bls[2].length); g.mat_mult_host(1, 0, 1, 2, a, b, got, precision=cq_b200.PREC_BF16X3)
        bound = _abs_bound(o, 1, 0, 1, 2, a, b, ref)
    else:
        cin = inputs.random_blocks(bls[2], 14, inputs.TAG_RANDOM_A)
        ref = np.zeros(bls[0].length); o.mat_mult(2, 0, 1, 2, ref, b, cin)
        got = np.zeros(bls[0].length); g.mat_mult_host(2, 0, 1, 2, got, b, cin, precision=cq_b200.PREC_BF16X3)
        bound = _abs_bound(o, 2, 0, 1, 2, ref, b, cin)
    err = np.abs(got - ref)
    assert np.all(err <= 2.0 ** -14 * bound + 1e-300)
    assert err.max() > 0          # it really ran in reduced precision


@pytest.mark.parametrize("variant", [-1, 0, 4])
def test_type2_dzp_bit_exact(cfg1, variant):
    o, g, bls = cfg1
    g.set_mult_variant(variant)
    b = inputs.random_blocks(bls[1], 12, inputs.TAG_RANDOM_B)
    cin = inputs.random_blocks(bls[2], 12, inputs.TAG_RANDOM_A)
    out_ref = np.zeros(bls[0].length)
    o.mat_mult(2, 0, 1, 2, out_ref, b, cin)
    out = np.full(bls[0].length, np.nan)
    g.mat_mult_host(2, 0, 1, 2, out, b, cin, exact=True)
    assert np.array_equal(out, out_ref)


@pytest.mark.parametrize("variant", [0, 4])
@pytest.mark.parametrize("mult_type", [1, 2])
def test_mixed_block_sizes_bit_exact(variant, mult_type):
    """Atoms with 4 and 13 orbitals in one system: every block shape (4x4, 4x13, 13x4, 13x13)."""
    import cq_b200
    coords, cell = inputs.diamond_si(2, sigma=0.05, seed=21)
    nsf = np.where(np.arange(len(coords)) % 3 == 0, 13, 4).astype(np.int32)
    rc = [6.0, 8.0, 14.0]
    o = OracleSystem(coords, cell, nsf, rc)
    g = cq_b200.System(coords, cell, nsf, rc)
    g.set_mult_variant(variant)
    bls = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    b = inputs.random_blocks(bls[1], 31, inputs.TAG_RANDOM_B)
    if mult_type == 1:
        a = inputs.random_blocks(bls[0], 31, inputs.TAG_RANDOM_A)
        ref = np.zeros(bls[2].length); o.mat_mult(1, 0, 1, 2, a, b, ref)
        got = np.full(bls[2].length, np.nan); g.mat_mult_host(1, 0, 1, 2, a, b, got)
    else:
        cin = inputs.random_blocks(bls[2], 32, inputs.TAG_RANDOM_A)
        ref = np.zeros(bls[0].length); o.mat_mult(2, 0, 1, 2, ref, b, cin)
        got = np.full(bls[0].length, np.nan); g.mat_mult_host(2, 0, 1, 2, got, b, cin)
    assert np.array_equal(got, ref)


LNV_PRODUCTS = [  # (type, a range, b range, c range) in mat_mult roles, from the product table of mult_module.f90
    (1, "L", "S", "LS"), (1, "L", "H", "LH"), (1, "LH", "S", "LSL"), (2, "L", "LS", "LSL"), (1, "LS", "S", "SLS"),
    (2, "L", "LS", "SLS"), (1, "LS", "L", "LSL"), (2, "H", "LS", "LSL"), (1, "T", "L", "TL"), (2, "L", "T", "TL"),
    (1, "T", "S", "TS"), (1, "T", "H", "TH"), (2, "L", "T", "TH"), (2, "T", "T", "TS"),
]


@pytest.mark.parametrize("variant", [-1, 0, 1, 2, 3, 5, 6])
@pytest.mark.parametrize("prod", LNV_PRODUCTS)
def test_lnv_products_sz_bit_exact(cfg2, prod, variant):
    o, g, bls, idx = cfg2
    g.set_mult_variant(variant)
    t, ra, rb, rc = prod
    ia, ib, ic = idx[ra], idx[rb], idx[rc]
    a = inputs.random_blocks(bls[ra], 21, inputs.TAG_RANDOM_A)
    b = inputs.random_blocks(bls[rb], 21, inputs.TAG_RANDOM_B)
    c = inputs.random_blocks(bls[rc], 22, inputs.TAG_RANDOM_A)
    if t == 1:
        ref = np.zeros(bls[rc].length); o.mat_mult(1, ia, ib, ic, a, b, ref)
        got = np.full(bls[rc].length, np.nan); g.mat_mult_host(1, ia, ib, ic, a, b, got)
    else:
        ref = np.zeros(bls[ra].length); o.mat_mult(2, ia, ib, ic, ref, b, c)
        got = np.full(bls[ra].length, np.nan); g.mat_mult_host(2, ia, ib, ic, got, b, c)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("deferred", [False, True])
@pytest.mark.parametrize("mult_type", [1, 2])
def test_dropin_kernels_match_default(cfg2, mult_type, deferred):
    """mat_mult's partition loop calling cq_m_kern_max / cq_m_kern_min reproduces the default kernel,
    completing every call or (deferred) enqueuing the loop's calls and completing at the last partition."""
    o, g, bls, idx = cfg2
    ra, rb, rc = ("L", "S", "LS") if mult_type == 1 else ("L", "LS", "SLS")
    ia, ib, ic = idx[ra], idx[rb], idx[rc]
    a = inputs.random_blocks(bls[ra], 31, inputs.TAG_RANDOM_A)
    b = inputs.random_blocks(bls[rb], 31, inputs.TAG_RANDOM_B)
    c = inputs.random_blocks(bls[rc], 32, inputs.TAG_RANDOM_A)
    if mult_type == 1:
        ref = np.zeros(bls[rc].length); o.mat_mult(1, ia, ib, ic, a, b, ref)
        got = np.zeros(bls[rc].length); dropin_driver.mat_mult_dropin(o, 1, ia, ib, ic, a, b, got, deferred)
    else:
        ref = np.zeros(bls[ra].length); o.mat_mult(2, ia, ib, ic, ref, b, c)
        got = np.zeros(bls[ra].length); dropin_driver.mat_mult_dropin(o, 2, ia, ib, ic, got, b, c, deferred)
    assert np.array_equal(got, ref)


def test_algebra_matches_oracle(cfg2):
    import torch
    o, g, bls, idx = cfg2
    dev = torch.device("cuda:0")
    L = inputs.random_blocks(bls["L"], 41, 1)
    S = inputs.random_blocks(bls["S"], 41, 2)
    LSL = inputs.random_blocks(bls["LSL"], 41, 3)
    tL, tS, tLSL = (torch.tensor(x, device=dev) for x in (L, S, LSL))
    # torch works on its default stream and the library on its own: synchronise between them
    sync = torch.cuda.synchronize
    # same range: scal + axpy
    ref = L.copy(); ref = ref * 0.5; ref = ref + (-2.0 * L)
    t = tL.clone(); sync(); g.matrix_sum(idx["L"], t, 0.5, idx["L"], tL, -2.0); g.synchronize()
    assert np.array_equal(t.cpu().numpy(), ref)
    # shorter destination (prune) and longer destination (partial update)
    ref = S.copy(); o.matrix_add(0.0, ref, idx["S"], 3.0, LSL, idx["LSL"])
    t = tS.clone(); sync(); g.matrix_sum(idx["S"], t, 0.0, idx["LSL"], tLSL, 3.0); g.synchronize()
    assert np.array_equal(t.cpu().numpy(), ref)
    ref = L.copy(); o.matrix_add(1.0, ref, idx["L"], -0.25, S, idx["S"])
    t = tL.clone(); sync(); g.matrix_sum(idx["L"], t, 1.0, idx["S"], tS, -0.25); g.synchronize()
    assert np.array_equal(t.cpu().numpy(), ref)
    # transpose, traces
    for r in ("L", "LS", "LSL"):
        x = inputs.random_blocks(bls[r], 43, 5)
        tx = torch.tensor(x, device=dev); tt = torch.empty_like(tx)
        sync()
        g.transpose(idx[r], tx, tt); g.synchronize()
        assert np.array_equal(tt.cpu().numpy(), o.transpose(idx[r], x))
    assert abs(g.trace(idx["L"], tL) - o.trace(idx["L"], L)) < 1e-12 * abs(o.trace(idx["L"], L)) + 1e-14
    dot_ref = float(np.dot(L, L))
    assert abs(g.product_trace(idx["L"], tL, tL) - dot_ref) < 1e-12 * dot_ref


def test_matrices_by_id_match_oracle(cfg2):
    """Matrices by id (cq_matrix_*): host arrays bound to ids, uploaded, multiplied (both mult
    types), summed (same and different ranges), transposed and traced on the system-owned device
    copies, downloaded; bit for bit against the oracle and the pointer-based entries."""
    o, g, bls, idx = cfg2
    g.set_mult_variant(-1)
    L = inputs.random_blocks(bls["L"], 51, inputs.TAG_RANDOM_A)
    S = inputs.random_blocks(bls["S"], 51, inputs.TAG_RANDOM_B)
    T = inputs.random_blocks(bls["T"], 52, inputs.TAG_RANDOM_B)
    TS = inputs.random_blocks(bls["TS"], 52, inputs.TAG_RANDOM_A)
    hL, hS, hLS = L.copy(), S.copy(), np.full(bls["LS"].length, np.nan)
    hT, hTS, hTo = T.copy(), TS.copy(), np.full(bls["T"].length, np.nan)
    hL2 = np.full(bls["L"].length, np.nan)
    for mid, r, h in ((1, "L", hL), (2, "S", hS), (3, "LS", hLS), (4, "T", hT), (5, "TS", hTS), (6, "T", hTo),
                      (7, "L", hL2)):
        g.bind(mid, idx[r], h)
    for mid in (1, 2, 4, 5):
        g.upload(mid)
    # type 1: LS = L . S
    g.product_id(1, 1, 2, 3)
    ref = np.zeros(bls["LS"].length); o.mat_mult(1, idx["L"], idx["S"], idx["LS"], L, S, ref)
    assert np.array_equal(g.download(3), ref)
    # type 2: T_out = TS . T^T
    g.product_id(2, 6, 4, 5)
    ref2 = np.zeros(bls["T"].length); o.mat_mult(2, idx["T"], idx["T"], idx["TS"], ref2, T, TS)
    assert np.array_equal(g.download(6), ref2)
    # transpose into a second L-range matrix, then sums of equal and of different ranges
    g.transpose_id(1, 7)
    assert np.array_equal(g.download(7), o.transpose(idx["L"], L))
    g.sum_id(7, 0.5, 1, -2.0)
    ref3 = o.transpose(idx["L"], L) * 0.5 + (-2.0 * L)
    assert np.array_equal(g.download(7), ref3)
    g.sum_id(2, 0.0, 3, 3.0)
    ref4 = S.copy(); o.matrix_add(0.0, ref4, idx["S"], 3.0, ref, idx["LS"])
    assert np.array_equal(g.download(2), ref4)
    # product trace by id equals the pointer-based entry on the same device arrays
    p1, n1 = g.device_ptr(1)
    p7, _ = g.device_ptr(7)
    assert n1 == bls["L"].length
    assert g.product_trace_id(1, 7) == g.product_trace(idx["L"], p1, p7)
    # an id binds once; unbound ids are rejected
    import cq_b200
    with pytest.raises(cq_b200.CQError):
        g.bind(1, idx["L"], hL)
    for mid in range(1, 8):
        g.unbind(mid)
    with pytest.raises(cq_b200.CQError):
        g.upload(1)


def test_unbind_after_stream_switch_keeps_inflight_inputs(cfg2):
    """Matrices bound on the system's own stream, then a switch to a torch stream: a product by id is
    enqueued there, its inputs are unbound while it may still run, and new ids bound and filled
    at once (allocations that may reuse the released memory).  The release happens on the current
    stream, after the product, so the product still reads its own inputs: bit for bit against the
    oracle."""
    import torch
    o, g, bls, idx = cfg2
    g.set_mult_variant(-1)
    L = inputs.random_blocks(bls["L"], 61, inputs.TAG_RANDOM_A)
    S = inputs.random_blocks(bls["S"], 61, inputs.TAG_RANDOM_B)
    hL, hS, hLS = L.copy(), S.copy(), np.full(bls["LS"].length, np.nan)
    g.bind(11, idx["L"], hL); g.bind(12, idx["S"], hS); g.bind(13, idx["LS"], hLS)
    g.upload(11); g.upload(12)
    g.synchronize()
    st = torch.cuda.Stream()
    g.set_stream(st.cuda_stream)
    try:
        junkL, junkS = np.full(bls["L"].length, 7.0), np.full(bls["S"].length, -3.0)
        for _ in range(3):
            g.product_id(1, 11, 12, 13)
        g.unbind(11); g.unbind(12)
        g.bind(14, idx["L"], junkL); g.bind(15, idx["S"], junkS)
        g.upload(14); g.upload(15)
        ref = np.zeros(bls["LS"].length)
        o.mat_mult(1, idx["L"], idx["S"], idx["LS"], L, S, ref)
        assert np.array_equal(g.download(13), ref)
        for mid in (13, 14, 15):
            g.unbind(mid)
        g.synchronize()
    finally:
        g.set_stream(None)
