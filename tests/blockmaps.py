"""Layout-independent views of block-sparse matrices for the tests.

A stored block is identified by (global row atom, global column atom, periodic
image of the column atom relative to its wrapped position).  These helpers turn
the index arrays exported by the oracle or by the CUDA library into that view,
build the generator's BlockList, and run dictionary-based known-answer products
that do not use halos, partitions or i_h2d at all.
"""
from __future__ import annotations

import numpy as np

from cq_b200.inputs import BlockList


def wrapped(coords, cell):
    c = np.asarray(coords, float)
    return c - np.floor((c + 1e-6) / cell) * cell


def oracle_blocklist(osys, r, coords, cell):
    """BlockList of range r from the oracle's exported index (reference layout)."""
    nnab = osys.geti("n_nab", r)
    ig_prim = osys.geti("ig_prim")
    i_part = osys.geti("i_part", r)
    i_seq = osys.geti("i_seq", r)
    icb = osys.geti("icover_ibeg")
    ig_cover = osys.geti("ig_cover")
    xcov = osys.getd("xcover").reshape(-1, 3)
    ndimi = osys.geti("ndimi", r)
    ndimj = osys.geti("ndimj", r)
    rad = osys.getd("radius", r)
    ca = icb[i_part - 1] + i_seq - 1 - 1  # 0-based cover atom
    ig_i = np.repeat(ig_prim, nnab) - 1
    ig_j = ig_cover[ca] - 1
    xw = wrapped(coords, cell)
    shift = np.rint((xcov[ca] - xw[ig_j]) / cell).astype(np.int64)
    nd_i = np.repeat(ndimi, nnab)
    sizes = nd_i * ndimj
    off = np.concatenate([[0], np.cumsum(sizes)[:-1]])
    return BlockList(ig_i, ig_j, shift, rad, nd_i, ndimj, off, int(sizes.sum()))


def block_dict(bl):
    """(ig_i, ig_j, sx, sy, sz) -> (elem offset, nd_i, nd_j)."""
    d = {}
    for q in range(len(bl.ig_i)):
        key = (int(bl.ig_i[q]), int(bl.ig_j[q]), int(bl.shift[q, 0]), int(bl.shift[q, 1]), int(bl.shift[q, 2]))
        d[key] = (int(bl.elem_off[q]), int(bl.nd_i[q]), int(bl.nd_j[q]))
    return d


def rows_of(bl):
    rows = {}
    for q in range(len(bl.ig_i)):
        rows.setdefault(int(bl.ig_i[q]), []).append(q)
    return rows


def kat_type1(blA, a, blB, b, blC):
    """C = A.B restricted to C's blocks, by explicit image arithmetic (no halos)."""
    c = np.zeros(blC.length)
    dC = block_dict(blC)
    rowsB = rows_of(blB)
    for qa in range(len(blA.ig_i)):
        i, k = int(blA.ig_i[qa]), int(blA.ig_j[qa])
        sk = blA.shift[qa]
        ndi, ndk = int(blA.nd_i[qa]), int(blA.nd_j[qa])
        A = a[blA.elem_off[qa]:blA.elem_off[qa] + ndi * ndk].reshape(ndk, ndi).T
        for qb in rowsB.get(k, []):
            j = int(blB.ig_j[qb])
            s = sk + blB.shift[qb]
            key = (i, j, int(s[0]), int(s[1]), int(s[2]))
            if key not in dC:
                continue
            off, _, ndj = dC[key]
            B = b[blB.elem_off[qb]:blB.elem_off[qb] + ndk * ndj].reshape(ndj, ndk).T
            c[off:off + ndi * ndj] += (A @ B).T.ravel()
    return c


def kat_type2(blOut, blB, b, blIn, cin):
    """out_ik = sum_j In_ij . B_kj^T over out's blocks (type-2 mat_mult), by image arithmetic."""
    out = np.zeros(blOut.length)
    dIn = block_dict(blIn)
    rowsB = rows_of(blB)
    for qo in range(len(blOut.ig_i)):
        i, k = int(blOut.ig_i[qo]), int(blOut.ig_j[qo])
        sk = blOut.shift[qo]
        ndi, ndk = int(blOut.nd_i[qo]), int(blOut.nd_j[qo])
        acc = np.zeros((ndi, ndk))
        for qb in rowsB.get(k, []):
            j = int(blB.ig_j[qb])
            s = sk + blB.shift[qb]
            key = (i, j, int(s[0]), int(s[1]), int(s[2]))
            if key not in dIn:
                continue
            off, _, ndj = dIn[key]
            X = cin[off:off + ndi * ndj].reshape(ndj, ndi).T
            B = b[blB.elem_off[qb]:blB.elem_off[qb] + ndk * ndj].reshape(ndj, ndk).T
            acc += X @ B.T
        out[blOut.elem_off[qo]:blOut.elem_off[qo] + ndi * ndk] = acc.T.ravel()
    return out


def kat_transpose(bl, a):
    """AT(j, i image -s) = A(i, j image s)^T over the same range."""
    at = np.zeros(bl.length)
    d = block_dict(bl)
    for q in range(len(bl.ig_i)):
        i, j = int(bl.ig_i[q]), int(bl.ig_j[q])
        s = -bl.shift[q]
        off, ndj, ndi = d[(j, i, int(s[0]), int(s[1]), int(s[2]))]
        ndI, ndJ = int(bl.nd_i[q]), int(bl.nd_j[q])
        A = a[bl.elem_off[q]:bl.elem_off[q] + ndI * ndJ].reshape(ndJ, ndI).T
        at[off:off + ndJ * ndI] = A.ravel()  # A row-major is A^T column-major
    return at


def dense(bl, v, n, nd):
    """Dense (n nd) x (n nd) matrix of a range's values v (blocks of a cluster with no periodic images
    in range; image blocks of one pair would be summed)."""
    M = np.zeros((n * nd, n * nd))
    for q in range(len(bl.ig_i)):
        i, j = bl.ig_i[q], bl.ig_j[q]
        M[i * nd:(i + 1) * nd, j * nd:(j + 1) * nd] += v[bl.elem_off[q]:bl.elem_off[q] + nd * nd].reshape(nd, nd).T
    return M
