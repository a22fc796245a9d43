"""Seeded synthetic inputs for the block-sparse multiply and the LNV solver.

Geometry: diamond-cubic Si supercells (a = 10.263 bohr) with seeded Gaussian
displacements, and spherical clusters carved from the same lattice.

Matrix values are a pure function of (seed, matrix tag, global atom i, global
atom j, periodic image of j, element), so they do not depend on the storage
order of any implementation: the CUDA path and the CPU oracle receive
bit-identical inputs once both have laid out the same neighbour lists.

Generators (per image-resolved atom pair at distance r, blocks nd_i x nd_j):
  * random blocks: uniform[-1, 1] * exp(-r / 3)                 (mat_mult KAT)
  * S: onsite 1.0 * I, offsite 0.3 * exp(-r / 2) * w every entry (overlap)
  * H: onsite diagonal uniform[-0.5, 0], offsite -0.2 * exp(-r / 2) * w
with the block weight w = min(1, 4 / sqrt(nd_i nd_j)).  For 4 x 4 (SZ) blocks w = 1 and the entries
are the stated ones; for larger blocks an offsite block whose every entry equals 0.3 exp(-r/2) has
a row sum nd_j times larger, and with 13 x 13 (DZP) blocks the overlap of diamond Si is no longer
diagonally dominant (nor positive definite), so the weight keeps the row sums of the SZ case.
"""
from __future__ import annotations

import numpy as np

A_SI = 10.263  # bohr, conventional cubic cell of Si used by the reference's matrix_multiply benchmarks

_FCC = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]])
_BASIS = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]])


def diamond_si(ncell, a=A_SI, sigma=0.0, seed=0):
    """Diamond-cubic Si supercell of ncell^3 conventional cells -> (coords (N,3), cell (3,))."""
    nc = (ncell, ncell, ncell) if np.isscalar(ncell) else tuple(ncell)
    frac = []
    for ix in range(nc[0]):
        for iy in range(nc[1]):
            for iz in range(nc[2]):
                for f in _FCC:
                    for b in _BASIS:
                        frac.append((np.array([ix, iy, iz], float) + f + b))
    coords = np.array(frac) * a
    rng = np.random.default_rng(seed)
    if sigma > 0:
        coords = coords + rng.normal(0.0, sigma, size=coords.shape)
    cell = np.array(nc, float) * a
    return coords, cell


def si_cluster(n_target, a=A_SI, sigma=0.1, seed=0, vacuum=30.0):
    """Spherical Si cluster of about n_target atoms carved from the diamond lattice, centred in a box
    with `vacuum` bohr of empty space on each side (no periodic neighbours within any range used here)."""
    ncell = int(np.ceil((n_target / 8.0) ** (1.0 / 3.0))) + 2
    coords, _ = diamond_si(ncell, a, 0.0, 0)
    centre = coords.mean(axis=0)
    d = np.linalg.norm(coords - centre, axis=1)
    order = np.argsort(d, kind="stable")
    sel = np.sort(order[:n_target])
    c = coords[sel] - coords[sel].min(axis=0)
    rng = np.random.default_rng(seed)
    if sigma > 0:
        c = c + rng.normal(0.0, sigma, size=c.shape)
    c = c - c.min(axis=0) + vacuum
    cell = c.max(axis=0) + vacuum
    return c, cell


# --------------------------------------------------------------------------
# counter-based hashing (splitmix64 finaliser) -> uniform [0, 1)
# --------------------------------------------------------------------------
_M = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix(x):
    x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return x ^ (x >> np.uint64(31))


def hash_uniform(seed, tag, ig_i, ig_j, sx, sy, sz, elem):
    """Uniform [0,1) from the integer key (all arguments broadcast; int64 arrays)."""
    with np.errstate(over="ignore"):
        k = _mix(np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15) + np.uint64(tag))
        for v, c in ((ig_i, 0xD1B54A32D192ED03), (ig_j, 0xABC98388FB8FAC03), (sx, 0x8CB92BA72F3D8DD7),
                     (sy, 0xC2B2AE3D27D4EB4F), (sz, 0x165667B19E3779F9), (elem, 0x27D4EB2F165667C5)):
            k = _mix(k ^ (np.asarray(v).astype(np.int64).astype(np.uint64) * np.uint64(c)))
    return (k >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


TAG_RANDOM_A, TAG_RANDOM_B, TAG_H_ONSITE = 11, 12, 21


class BlockList:
    """Layout-agnostic description of a block matrix: one row per stored block."""

    def __init__(self, ig_i, ig_j, shift, radius, nd_i, nd_j, elem_off, length):
        self.ig_i = np.asarray(ig_i, np.int64)
        self.ig_j = np.asarray(ig_j, np.int64)
        self.shift = np.asarray(shift, np.int64).reshape(-1, 3)
        self.radius = np.asarray(radius, np.float64)
        self.nd_i = np.asarray(nd_i, np.int64)
        self.nd_j = np.asarray(nd_j, np.int64)
        self.elem_off = np.asarray(elem_off, np.int64)
        self.length = int(length)


def _fill(bl, blockfn):
    out = np.zeros(bl.length, dtype=np.float64)
    for ndi in np.unique(bl.nd_i):
        for ndj in np.unique(bl.nd_j):
            sel = np.nonzero((bl.nd_i == ndi) & (bl.nd_j == ndj))[0]
            if sel.size == 0:
                continue
            ne = int(ndi * ndj)
            e = np.arange(ne, dtype=np.int64)
            vals = blockfn(sel, int(ndi), int(ndj), e)  # (nsel, ne), column-major within block
            idx = bl.elem_off[sel][:, None] + e[None, :]
            out[idx.ravel()] = vals.ravel()
    return out


def random_blocks(bl, seed, tag, decay=3.0):
    """uniform[-1,1] * exp(-r/decay) per element of each image-resolved block."""
    def fn(sel, ndi, ndj, e):
        u = hash_uniform(seed, tag, bl.ig_i[sel][:, None], bl.ig_j[sel][:, None], bl.shift[sel, 0][:, None],
                         bl.shift[sel, 1][:, None], bl.shift[sel, 2][:, None], e[None, :])
        return (2.0 * u - 1.0) * np.exp(-bl.radius[sel] / decay)[:, None]
    return _fill(bl, fn)


def _onsite_mask(bl, sel):
    return (bl.ig_i[sel] == bl.ig_j[sel]) & np.all(bl.shift[sel] == 0, axis=1)


def block_weight(ndi, ndj):
    """Offsite weight of an nd_i x nd_j block: 1 for SZ blocks, 4 / sqrt(nd_i nd_j) for larger ones."""
    return min(1.0, 4.0 / np.sqrt(float(ndi) * float(ndj)))


def overlap_S(bl):
    """S: 1.0 * I on the onsite block, 0.3 * exp(-r/2) * w on every entry of an offsite block."""
    def fn(sel, ndi, ndj, e):
        v = np.repeat((0.3 * block_weight(ndi, ndj) * np.exp(-bl.radius[sel] / 2.0))[:, None], e.size, axis=1)
        on = _onsite_mask(bl, sel)
        if on.any():
            eye = (e % ndi == e // ndi).astype(np.float64)
            v[on] = eye[None, :]
        return v
    return _fill(bl, fn)


def hamiltonian_H(bl, seed):
    """H: onsite block diagonal with orbital energies uniform[-0.5, 0], offsite -0.2 * exp(-r/2) * w per entry.

    The onsite block is kept diagonal (hence symmetric): with uniform off-diagonal onsite entries as
    well, the Gershgorin-type estimate of the McWeeny initialisation (onsite |H| added to both
    bounds, McWeeny.f90:1060-1075) lies above the lowest eigenvalue and the initial L is not a
    valid starting point.
    """
    def fn(sel, ndi, ndj, e):
        v = np.repeat((-0.2 * block_weight(ndi, ndj) * np.exp(-bl.radius[sel] / 2.0))[:, None], e.size, axis=1)
        on = _onsite_mask(bl, sel)
        if on.any():
            r_, c_ = e % ndi, e // ndi
            ig = bl.ig_i[sel][on][:, None]
            u = hash_uniform(seed, TAG_H_ONSITE, ig, ig, 0, 0, 0, r_[None, :])
            v[on] = np.where((r_ == c_)[None, :], -0.5 * u, 0.0)
        return v
    return _fill(bl, fn)
