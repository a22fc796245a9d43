"""Known answers for the pieces of the oracle's density-matrix chain, on a 16-atom Si cluster whose
T and L ranges exceed the cluster (no truncation):

* Hotelling S^-1 (Iter_Hott_InvS, S_matrix_module.f90:746-963) gives T S = I;
* the McWeeny start and purification (InitMcW / McWMin, McWeeny.f90:107-570) give an L that is
  idempotent in the S metric, holds ne electrons per spin, and whose band energy is the dense
  generalised ground state of (H, S).
"""
import numpy as np
import scipy.linalg as sla

import blockmaps as bm
from cq_b200 import inputs
from lnv_oracle import OracleLNV, Params
from test_scf_coupling import _cluster


def _chain():
    n, o, ridx, blS, blH, S, H = _cluster(16)
    coords, cell = inputs.si_cluster(16, sigma=0.1, seed=4)
    lnv = OracleLNV(o, ridx, S, H, float(n), 4.0 * n, Params())
    dense = {r: (lambda v, r=r: bm.dense(bm.oracle_blocklist(o, ridx[r], coords, cell), v, n, 4))
             for r in ("S", "H", "L", "T")}
    return n, lnv, dense, S, H


def test_hotelling_inverse_of_untruncated_overlap():
    n, lnv, dense, S, H = _chain()
    omega = lnv.iter_hott_invs()
    TS = dense["T"](lnv.T.v) @ dense["S"](S)
    assert omega < 1e-12
    assert np.abs(TS - np.eye(4 * n)).max() < 1e-12


def test_mcweeny_start_is_the_ground_state_density():
    n, lnv, dense, S, H = _chain()
    lnv.iter_hott_invs()
    lnv.transpose(lnv.T, lnv.Ttran)
    lnv.init_mcw()
    lnv.mcw_min(lnv.p.n_L_iterations)
    Ld, Sd, Hd = dense["L"](lnv.L.v), dense["S"](S), dense["H"](H)
    assert np.abs(Ld @ Sd @ Ld - Ld).max() < 1e-10            # idempotent: L S L = L
    assert abs(np.trace(Ld @ Sd) - n) < 1e-9                  # ne = n electrons per spin
    ev = sla.eigh(Hd, Sd, eigvals_only=True)
    exact = 2.0 * ev[:n].sum()
    assert abs(2.0 * np.trace(Ld @ Hd) - exact) < 1e-10 * abs(exact)


def test_solve_cubic_roots():
    """SolveCubic (DMMinModule.f90:2072-2143): a real root of x^3 + a x^2 + b x + c; with three real
    roots the one of least magnitude.  Cardano's formula loses a few digits where its two cube
    roots cancel, so roots are compared at 1e-6 relative."""
    rs = np.random.default_rng(1)
    for _ in range(2000):
        a, b, c = rs.normal(size=3) * rs.choice([0.1, 1.0, 10.0], 3)
        x = OracleLNV.solve_cubic(a, b, c, 1.0e6)
        r = np.roots([1.0, a, b, c])
        real = r[np.abs(r.imag) < 1e-9].real
        tol = 1e-6 * max(1.0, abs(x))
        assert np.min(np.abs(real - x)) < tol
        if len(real) == 3:
            assert abs(abs(x) - np.min(np.abs(real))) < tol


def test_electron_number_correction_restores_ne():
    """correct_electron_number (DMMinModule.f90:1676-1817) brings a perturbed L back to ne electrons."""
    n, lnv, dense, S, H = _chain()
    lnv.iter_hott_invs()
    lnv.transpose(lnv.T, lnv.Ttran)
    lnv.init_mcw()
    lnv.mcw_min(lnv.p.n_L_iterations)
    rs = np.random.default_rng(1)
    lnv.L.v[:] += rs.normal(size=lnv.L.v.size) * 1e-3
    lnv.symmetrise_L()
    before, _ = lnv.lnv(dophi=True, phi=lnv.phi)
    lnv.correct_electron_number()
    after, _ = lnv.lnv(dophi=True, phi=lnv.phi)
    assert abs(before - n) > 1e-4
    assert abs(after - n) < 1e-9
