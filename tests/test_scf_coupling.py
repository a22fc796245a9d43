"""Mixed-L self-consistency (minE.MixedLSelfConsistent, DMMinModule.f90:894-907, 1138-1149) in the
oracle chain: lateDM rebuilds H from K of the current L.  A linear density feedback H = H0 + g K
stands in for the grid rebuild of H (get_electronic_density + get_H_matrix).

Known answers on a cluster with no truncation: the converged L is the ground state of the last H
(band energy = twice the sum of the lowest ne generalised eigenvalues of (H, S)), and H is
self-consistent with the final K.  With g = 0 the coupled chain takes the plain chain's steps.
"""
import numpy as np
import pytest
import scipy.linalg as sla

import blockmaps as bm
import cq_b200
from cq_b200 import inputs
from cq_oracle import OracleSystem
from lnv_oracle import OracleLNV, Params


def _cluster(n_atoms):
    coords, cell = inputs.si_cluster(n_atoms, sigma=0.1, seed=4)
    n = len(coords)
    diam = np.max(np.linalg.norm(coords[:, None] - coords[None], axis=-1))
    rng = cq_b200.lnv_ranges(10.0, 12.0, diam + 1, diam + 1)
    ridx = {k: i for i, k in enumerate(rng)}
    o = OracleSystem(coords, cell, np.full(n, 4), list(rng.values()))
    blS = bm.oracle_blocklist(o, ridx["S"], coords, cell)
    blH = bm.oracle_blocklist(o, ridx["H"], coords, cell)
    S = inputs.overlap_S(blS)
    H = inputs.hamiltonian_H(blH, seed=5)
    return n, o, ridx, blS, blH, S, H


def _solve(n, o, ridx, S, H, feedback, tolerance=1.0e-7):
    lnv = OracleLNV(o, ridx, S, H, float(n), 4.0 * n, Params(tolerance=tolerance))
    H0 = np.array(H, dtype=np.float64)
    if feedback is not None:
        lnv.h_rebuild = lambda K: H0 + feedback * K
    lnv.iter_hott_invs()
    E, N = lnv.find_min_dm(max_outer=40)
    return lnv, E, N


def test_zero_feedback_takes_the_plain_steps():
    n, o, ridx, blS, blH, S, H = _cluster(16)
    plain, E0, N0 = _solve(n, o, ridx, S, H, None)
    coupled, E1, N1 = _solve(n, o, ridx, S, H, 0.0)
    late_entries = sum(1 for x in coupled.log if x[0] == "lateDM" and x[1] == 1)
    late_iters = sum(1 for x in coupled.log if x[0] == "lateDM")
    assert coupled.h_rebuilds == late_entries + late_iters > 0
    assert (E1, N1) == (E0, N0)
    assert np.array_equal(coupled.L.v, plain.L.v)


@pytest.mark.parametrize("g", [-0.05, -0.1])
def test_coupled_minimum_is_ground_state_of_last_h(g):
    """Negative feedback (it lowers the occupied levels and opens the gap).  The chain stops on the
    DM residual of the current H while H still drifts with K, so the energy error of the stopped
    chain tracks the tolerance: at 1e-11 it is below 1e-9 relative."""
    n, o, ridx, blS, blH, S, H = _cluster(16)
    lnv, E, N = _solve(n, o, ridx, S, H, g, tolerance=1.0e-11)
    assert lnv.converged and lnv.h_rebuilds > 1
    ev = sla.eigh(bm.dense(blH, lnv.H.v, n, 4), bm.dense(blS, S, n, 4), eigvals_only=True)
    exact = 2.0 * ev[:n].sum()
    assert abs(E - exact) < 1e-9 * abs(exact)
    assert abs(N - 2.0 * n) < 1e-8
    # the chain stops right after a rebuild, with no step of L since: H is built from the final K
    assert np.array_equal(lnv.H.v, np.asarray(H) + g * lnv.K.v)
    # the feedback moved the answer
    _, E0, _ = _solve(n, o, ridx, S, H, None)
    assert abs(E - E0) > 1e-3
