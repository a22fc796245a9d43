"""CPU checks of the oracle itself (no GPU): known-answer tests that pin the restatement.

The reference ships no golden vectors for mat_mult, so the oracle is pinned by
independent constructions: explicit periodic-image arithmetic for the products
and the transpose, brute-force neighbour enumeration for the index, and the
invariants of the Hilbert ordering.
"""
import itertools

import numpy as np
import pytest

import blockmaps as bm
import systems
from cq_b200 import inputs
from cq_oracle import OracleSystem


@pytest.fixture(scope="module")
def sz_small():
    coords, cell = inputs.diamond_si(2, sigma=0.1, seed=3)
    rc = [5.0, 8.0, 12.0, 20.0]
    return coords, cell, OracleSystem(coords, cell, np.full(len(coords), 4), rc)


@pytest.fixture(scope="module")
def dzp_cfg1():
    coords, cell, nsf, rc = systems.config1()
    return coords, cell, OracleSystem(coords, cell, nsf, rc)


def brute_neighbours(coords, cell, rcut):
    """All (i, j, image) with |r_i - r_j - image| < rcut (squared test with RD_ERR), by explicit image loops."""
    xw = bm.wrapped(coords, cell)
    n = len(xw)
    out = {}
    nimg = [int(np.ceil(rcut / cell[d])) + 1 for d in range(3)]
    shifts = np.array(list(itertools.product(*[range(-m, m + 1) for m in nimg])))
    for i in range(n):
        d = xw[None, :, :] + (shifts[:, None, :] * cell[None, None, :]) - xw[i][None, None, :]
        d2 = (d ** 2).sum(-1)
        s_idx, j_idx = np.nonzero(d2 < rcut * rcut - 1e-8)
        out[i] = set((int(j), tuple(int(v) for v in shifts[s])) for s, j in zip(s_idx, j_idx))
    return out


def test_hilbert_partitions_cover_all_atoms(dzp_cfg1):
    coords, cell, o = dzp_cfg1
    nm = o.geti("nm_group")
    assert nm.sum() == len(coords)
    assert sorted(o.geti("ig_prim").tolist()) == list(range(1, len(coords) + 1))
    # every cover partition of the covering set appears once
    lab = o.geti("lab_cover")
    assert len(set(lab.tolist())) == len(lab)


@pytest.mark.parametrize("r", [0, 1, 2, 3])
def test_neighbour_lists_match_bruteforce(sz_small, r):
    coords, cell, o = sz_small
    bl = bm.oracle_blocklist(o, r, coords, cell)
    brute = brute_neighbours(coords, cell, o.rcuts[r])
    got = {}
    for q in range(len(bl.ig_i)):
        got.setdefault(int(bl.ig_i[q]), set()).add((int(bl.ig_j[q]), tuple(int(v) for v in bl.shift[q])))
    for i in range(len(coords)):
        assert got[i] == brute[i]
    # radius is the image distance
    xw = bm.wrapped(coords, cell)
    d = np.linalg.norm(xw[bl.ig_j] + bl.shift * cell - xw[bl.ig_i], axis=1)
    np.testing.assert_allclose(bl.radius, d, rtol=0, atol=1e-12)


def test_type1_matches_image_arithmetic_dzp(dzp_cfg1):
    coords, cell, o = dzp_cfg1
    blA, blB, blC = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    a = inputs.random_blocks(blA, 101, inputs.TAG_RANDOM_A)
    b = inputs.random_blocks(blB, 101, inputs.TAG_RANDOM_B)
    c = np.zeros(blC.length)
    o.mat_mult(1, 0, 1, 2, a, b, c)
    ck = bm.kat_type1(blA, a, blB, b, blC)
    err = np.abs(c - ck) / (np.abs(ck).max())
    assert err.max() < 1e-13


def test_type2_and_ompgemm_sz(sz_small):
    coords, cell, o = sz_small
    blO, blB, blI = [bm.oracle_blocklist(o, r, coords, cell) for r in (1, 2, 3)]
    b = inputs.random_blocks(blB, 5, inputs.TAG_RANDOM_B)
    cin = inputs.random_blocks(blI, 5, inputs.TAG_RANDOM_A)
    out = np.zeros(blO.length)
    o.mat_mult(2, 1, 2, 3, out, b, cin)
    ck = bm.kat_type2(blO, blB, b, blI, cin)
    assert np.abs(out - ck).max() < 1e-13 * np.abs(ck).max()
    out2 = np.zeros(blO.length)
    o.mat_mult(2, 1, 2, 3, out2, b, cin, kernel="ompGemm", nthreads=2)
    assert np.abs(out2 - out).max() < 1e-12 * np.abs(ck).max()
    # type 1 with ompGemm against default
    a = inputs.random_blocks(blO, 6, inputs.TAG_RANDOM_A)
    c1 = np.zeros(blI.length); c2 = np.zeros(blI.length)
    o.mat_mult(1, 1, 2, 3, a, b, c1)
    o.mat_mult(1, 1, 2, 3, a, b, c2, kernel="ompGemm", nthreads=3)
    assert np.abs(c1 - c2).max() < 1e-12 * np.abs(c1).max()


def test_ompdoii_is_bit_identical_to_default(sz_small):
    coords, cell, o = sz_small
    blO, blB, blI = [bm.oracle_blocklist(o, r, coords, cell) for r in (1, 2, 3)]
    a = inputs.random_blocks(blO, 16, 1)
    b = inputs.random_blocks(blB, 16, 2)
    c1 = np.zeros(blI.length); c2 = np.zeros(blI.length)
    o.mat_mult(1, 1, 2, 3, a, b, c1)
    o.mat_mult(1, 1, 2, 3, a, b, c2, kernel="ompDoii", nthreads=4)
    assert np.array_equal(c1, c2)
    cin = inputs.random_blocks(blI, 17, 3)
    o1 = np.zeros(blO.length); o2 = np.zeros(blO.length)
    o.mat_mult(2, 1, 2, 3, o1, b, cin)
    o.mat_mult(2, 1, 2, 3, o2, b, cin, kernel="ompDoii", nthreads=3)
    assert np.array_equal(o1, o2)


def test_transpose_matches_image_arithmetic(sz_small):
    coords, cell, o = sz_small
    for r in range(4):
        bl = bm.oracle_blocklist(o, r, coords, cell)
        a = inputs.random_blocks(bl, 9, 3)
        assert np.array_equal(o.transpose(r, a), bm.kat_transpose(bl, a))


def test_matrix_add_nested_ranges(sz_small):
    coords, cell, o = sz_small
    blS, blL = bm.oracle_blocklist(o, 1, coords, cell), bm.oracle_blocklist(o, 3, coords, cell)
    s = inputs.random_blocks(blS, 1, 1)
    l = inputs.random_blocks(blL, 1, 2)
    dL = bm.block_dict(blL)
    # short += long (prune): every short block updated
    s2 = s.copy()
    o.matrix_add(0.5, s2, 1, 2.0, l, 3)
    exp = s.copy()
    for q in range(len(blS.ig_i)):
        key = (int(blS.ig_i[q]), int(blS.ig_j[q])) + tuple(int(v) for v in blS.shift[q])
        off, ni, nj = dL[key]
        o0 = blS.elem_off[q]
        exp[o0:o0 + ni * nj] = 0.5 * s[o0:o0 + ni * nj] + 2.0 * l[off:off + ni * nj]
    np.testing.assert_array_equal(s2, exp)
    # long += short: only the shared blocks change, the others keep their old values
    l2 = l.copy()
    o.matrix_add(3.0, l2, 3, -1.0, s, 1)
    dS = bm.block_dict(blS)
    exp = l.copy()
    for q in range(len(blL.ig_i)):
        key = (int(blL.ig_i[q]), int(blL.ig_j[q])) + tuple(int(v) for v in blL.shift[q])
        if key in dS:
            off, ni, nj = dS[key]
            o0 = blL.elem_off[q]
            exp[o0:o0 + ni * nj] = 3.0 * l[o0:o0 + ni * nj] - 1.0 * s[off:off + ni * nj]
    np.testing.assert_array_equal(l2, exp)


def test_trace_is_onsite_diagonal(sz_small):
    coords, cell, o = sz_small
    bl = bm.oracle_blocklist(o, 1, coords, cell)
    a = inputs.random_blocks(bl, 4, 4)
    tr = 0.0
    for q in range(len(bl.ig_i)):
        if bl.ig_i[q] == bl.ig_j[q] and not bl.shift[q].any():
            blk = a[bl.elem_off[q]:bl.elem_off[q] + 16].reshape(4, 4)
            tr += np.trace(blk)
    assert abs(o.trace(1, a) - tr) < 1e-12


@pytest.mark.parametrize("case", ["one_atom", "two_atoms_mixed_sizes"])
def test_tiny_cells_match_image_arithmetic(case):
    """Edge cases: a one-atom cell whose neighbours are all its own periodic images, and a
    two-atom cell with 4x4 and 13x13 blocks in an orthorhombic box; both mult types against
    explicit image arithmetic."""
    if case == "one_atom":
        coords, cell, nsf = np.array([[0.3, 0.2, 0.1]]), np.array([5.0, 5.0, 5.0]), [4]
    else:
        coords, cell, nsf = np.array([[0.0, 0.0, 0.0], [2.5, 2.5, 2.5]]), np.array([5.0, 6.0, 7.0]), [4, 13]
    o = OracleSystem(coords, cell, np.array(nsf), [4.0, 6.0, 10.0])
    bls = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    assert len(bls[0].ig_i) == len(coords)           # range 4 < every image distance: onsite only
    a = inputs.random_blocks(bls[0], 7, inputs.TAG_RANDOM_A)
    b = inputs.random_blocks(bls[1], 7, inputs.TAG_RANDOM_B)
    c = np.zeros(bls[2].length)
    o.mat_mult(1, 0, 1, 2, a, b, c)
    ck = bm.kat_type1(bls[0], a, bls[1], b, bls[2])
    assert np.abs(c - ck).max() < 1e-13 * np.abs(ck).max()
    cin = inputs.random_blocks(bls[2], 8, inputs.TAG_RANDOM_A)
    out = np.zeros(bls[0].length)
    o.mat_mult(2, 0, 1, 2, out, b, cin)
    ck2 = bm.kat_type2(bls[0], bls[1], b, bls[2], cin)
    assert np.abs(out - ck2).max() < 1e-13 * np.abs(ck2).max()


def test_default_kernel_with_fused_multiply_add(dzp_cfg1):
    """The oracle's default kernel with each multiply-add fused ("default_fma", the order of the GPU's
    fused-multiply-add and FP64 tensor-core products): the same sums to FP64 rounding (a few 2^-53 of
    sum |a||b|), and really different roundings (not the same bits as the separate multiply and add)."""
    coords, cell, o = dzp_cfg1
    blA, blB, blC = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    a = inputs.random_blocks(blA, 111, inputs.TAG_RANDOM_A)
    b = inputs.random_blocks(blB, 111, inputs.TAG_RANDOM_B)
    for t in (1, 2):
        if t == 1:
            c0 = np.zeros(blC.length); c1 = np.zeros(blC.length); bound = np.zeros(blC.length)
            o.mat_mult(1, 0, 1, 2, a, b, c0)
            o.mat_mult(1, 0, 1, 2, a, b, c1, kernel="default_fma")
            o.mat_mult(1, 0, 1, 2, np.abs(a), np.abs(b), bound)
        else:
            cin = inputs.random_blocks(blC, 112, inputs.TAG_RANDOM_A)
            c0 = np.zeros(blA.length); c1 = np.zeros(blA.length); bound = np.zeros(blA.length)
            o.mat_mult(2, 0, 1, 2, c0, b, cin)
            o.mat_mult(2, 0, 1, 2, c1, b, cin, kernel="default_fma")
            o.mat_mult(2, 0, 1, 2, bound, np.abs(b), np.abs(cin))
        assert np.all(np.abs(c1 - c0) <= 1e-14 * bound)
        assert not np.array_equal(c1, c0)
