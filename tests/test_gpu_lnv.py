"""GPU LNV / McWeeny chain vs the oracle chain and vs the exact dense answer.

Tolerances: band energy and electron count within 1e-10 of the
oracle for the FP64 path.
"""
import hashlib
import json
import os

import numpy as np
import pytest
import scipy.linalg as sla

import blockmaps as bm
import systems
from cq_b200 import inputs
from cq_oracle import OracleSystem
from lnv_oracle import OracleLNV, Params

pytestmark = pytest.mark.gpu


def _setup(coords, cell, nsf, ne_spin, rs=10.0, rh=12.0, rl=16.0, rt=10.0, **params):
    import cq_b200
    rng = cq_b200.lnv_ranges(rs, rh, rl, rt)
    names = list(rng)
    ridx = {n: i for i, n in enumerate(names)}
    o = OracleSystem(coords, cell, nsf, list(rng.values()))
    g = cq_b200.System(coords, cell, nsf, list(rng.values()))
    blS = bm.oracle_blocklist(o, ridx["S"], coords, cell)
    blH = bm.oracle_blocklist(o, ridx["H"], coords, cell)
    S, H = inputs.overlap_S(blS), inputs.hamiltonian_H(blH, seed=5)
    olnv = OracleLNV(o, ridx, S, H, ne_spin, float(np.sum(nsf)),
                     Params(**{k: v for k, v in params.items() if k not in ("max_outer", "graphs")}))
    glnv = cq_b200.LNV(g, ridx, ne_spin, **params)
    return o, g, ridx, S, H, olnv, glnv


_dense = bm.dense


def test_cluster_matches_dense_eigh():
    """No truncation (ranges exceed the cluster): the LNV minimum is the exact ground state."""
    coords, cell = inputs.si_cluster(64, sigma=0.1, seed=4)
    n = len(coords)
    diam = np.max(np.linalg.norm(coords[:, None] - coords[None], axis=-1))
    ne_spin = 64.0
    o, g, ridx, S, H, olnv, glnv = _setup(coords, cell, np.full(n, 4), ne_spin, rl=diam + 1, rt=diam + 1)
    res, L, K = glnv.solve_host(S, H, want_L=True, want_K=True)
    blS = bm.oracle_blocklist(o, ridx["S"], coords, cell); blH = bm.oracle_blocklist(o, ridx["H"], coords, cell)
    ev = sla.eigh(_dense(blH, H, n, 4), _dense(blS, S, n, 4), eigvals_only=True)
    exact = 2.0 * ev[:int(ne_spin)].sum()
    assert res["converged"] == 1
    assert abs(res["energy"] - exact) < 1e-9 * abs(exact)
    assert abs(res["electrons"] - 2 * ne_spin) < 1e-8


GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lnv_chain_si64.json")))


@pytest.mark.parametrize("case", sorted(GOLDEN["cases"]))
def test_periodic_matches_oracle_chain(case):
    """Periodic Si (2x2x2 cells, SZ, truncated ranges): GPU chain vs the oracle chain's fixture.

    Products are bit-exact and every reduction is an exact, order-independent sum on both
    sides, so the two chains take the same steps: the same number of products, the same final
    L to the bit, E and Ne within 1e-10.  The short-range case stalls above the tolerance (as
    the reference would) and is compared after its pass limit.
    """
    gold = GOLDEN["cases"][case]
    coords, cell = inputs.diamond_si(2, sigma=0.1, seed=2)
    n = len(coords)
    rs, rh, rl, rt = gold["ranges"]
    o, g, ridx, S, H, olnv, glnv = _setup(coords, cell, np.full(n, 4), float(n), rs, rh, rl, rt,
                                          max_outer=gold["max_outer"])
    res, L, K = glnv.solve_host(S, H, want_L=True)
    assert res["converged"] == int(gold["converged"])
    assert res["n_products"] == gold["n_products"]
    assert abs(res["energy"] - gold["energy"]) <= 1e-10 * max(1.0, abs(gold["energy"]))
    assert abs(res["electrons"] - gold["electrons"]) <= 1e-10 * max(1.0, abs(gold["electrons"]))
    assert hashlib.sha256(np.ascontiguousarray(L, np.float64).tobytes()).hexdigest() == gold["L_sha256"]


def test_graph_replay_matches_direct_launches():
    """LNV_matrix_multiply calls replayed from CUDA graphs give the same bits as direct launches."""
    gold = GOLDEN["cases"]["r8_9_10_8"]
    coords, cell = inputs.diamond_si(2, sigma=0.1, seed=2)
    n = len(coords)
    out = []
    for graphs in (0, 1):
        o, g, ridx, S, H, olnv, glnv = _setup(coords, cell, np.full(n, 4), float(n), *gold["ranges"],
                                              max_outer=gold["max_outer"], graphs=graphs)
        res, L, K = glnv.solve_host(S, H, want_L=True)
        out.append((res, L))
    (r0, L0), (r1, L1) = out
    assert r0["graph_launches"] == 0 and r1["graph_launches"] > 0
    assert (r0["energy"], r0["electrons"], r0["n_products"]) == (r1["energy"], r1["electrons"], r1["n_products"])
    assert np.array_equal(L0, L1)
    assert hashlib.sha256(np.ascontiguousarray(L1, np.float64).tobytes()).hexdigest() == gold["L_sha256"]


def test_force_matrices_match_oracle():
    """M12 (S range) and M4 (H range) of a given L: the doM1 + doM2 and doM4 branches of
    LNV_matrix_multiply, bit for bit against the oracle on the same L."""
    coords, cell = inputs.diamond_si(2, sigma=0.1, seed=2)
    n = len(coords)
    o, g, ridx, S, H, olnv, glnv = _setup(coords, cell, np.full(n, 4), float(n), 8.0, 9.0, 10.0, 8.0)
    glnv.set_SH(S, H)
    rs = np.random.default_rng(17)
    Lr = rs.uniform(-0.05, 0.05, g.length(ridx["L"]))
    glnv.put("L", Lr)
    olnv.L.v[:] = Lr
    M12, M4 = glnv.force_matrices()
    oM12, oM4 = olnv.force_matrices()
    assert np.array_equal(M12, oM12)
    assert np.array_equal(M4, oM4)
    assert np.abs(M12).max() > 0 and np.abs(M4).max() > 0


def test_matrix_file_round_trip(tmp_path):
    """L written in the reference's binary matrix-file format (dump_matrix2) and read back
    (grab_matrix2): the records parse as Fortran unformatted sequential records with the
    reference's layout, and the grabbed matrix equals the dumped one bit for bit."""
    import torch
    from scipy.io import FortranFile
    coords, cell = inputs.diamond_si(2, sigma=0.1, seed=2)
    n = len(coords)
    o, g, ridx, S, H, olnv, glnv = _setup(coords, cell, np.full(n, 4), float(n), 8.0, 9.0, 10.0, 8.0, max_outer=1)
    glnv.solve_host(S, H)
    L = glnv.get("L")
    dev = torch.tensor(L, device="cuda")
    torch.cuda.synchronize()
    path = str(tmp_path / "Lmatrix2.i00.p000001")
    rl = ridx["L"]
    g.dump_matrix(rl, dev, path, inode=1)
    # the record layout of store_matrix_module.f90:375-415
    f = FortranFile(path, "r")
    inode, nprim = f.read_ints(np.int32)
    assert (inode, nprim) == (1, n)
    nsf_i = f.read_ints(np.int32); jmax = f.read_ints(np.int32); jbeta = f.read_ints(np.int32)
    assert f.read_ints(np.int32)[0] == 1
    assert np.all(nsf_i == 4) and np.array_equal(jmax, g.geti("n_nab", rl))
    ig_prim = g.geti("ig_prim"); ig_j = g.geti("ig_j", rl)
    start = 0
    for p in range(n):
        assert f.read_ints(np.int32)[0] == ig_prim[p]
        beta = f.read_ints(np.int32); idj = f.read_ints(np.int32)
        assert np.all(beta == 4) and jbeta[p] == beta.sum()
        assert np.array_equal(idj, ig_j[start:start + jmax[p]])
        for _ in range(jmax[p]):
            assert f.read_reals(np.float64).shape == (3,)
        for _ in range(jbeta[p] * nsf_i[p]):
            f.read_reals(np.float64)
        start += jmax[p]
    f.close()
    back = torch.zeros_like(dev)
    torch.cuda.synchronize()
    matched = g.grab_matrix(rl, back, path)
    assert matched == g.n_blocks(rl)
    assert np.array_equal(back.cpu().numpy(), L)


GOLDEN_SCF = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lnv_scf_si64.json")))


@pytest.mark.parametrize("case", sorted(GOLDEN_SCF["cases"]))
def test_mixed_l_self_consistency_matches_oracle(case):
    """lateDM with the H rebuild callback (mixed-L self-consistency): H = H0 + g K rebuilt on the
    device through cq_matrix_sum at lateDM's start and after every Pulay step.  The same number
    of rebuilds as the oracle chain, L and the final H to the bit, E and Ne within 1e-10."""
    import torch
    gold = GOLDEN_SCF["cases"][case]
    coords, cell = inputs.diamond_si(2, sigma=0.1, seed=2)
    n = len(coords)
    o, g, ridx, S, H, olnv, glnv = _setup(coords, cell, np.full(n, 4), float(n), *gold["ranges"],
                                          max_outer=gold["max_outer"])
    rH = ridx["H"]
    H0 = torch.tensor(H, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    calls = []

    def rebuild(k, h, length, stream):
        calls.append(length)
        g.matrix_sum(rH, h, 0.0, rH, H0.data_ptr(), 1.0)
        g.matrix_sum(rH, h, 1.0, rH, k, gold["feedback"])
        return 0

    glnv.set_h_rebuild(rebuild)
    glnv.set_SH(S, H)
    res = glnv.solve()
    L, Hf = glnv.get("L"), glnv.get("H")
    assert len(calls) == gold["h_rebuilds"] and set(calls) == {g.length(rH)}
    assert res["converged"] == int(gold["converged"])
    assert res["n_products"] == gold["n_products"]
    assert abs(res["energy"] - gold["energy"]) <= 1e-10 * max(1.0, abs(gold["energy"]))
    assert abs(res["electrons"] - gold["electrons"]) <= 1e-10 * max(1.0, abs(gold["electrons"]))
    assert hashlib.sha256(np.ascontiguousarray(L, np.float64).tobytes()).hexdigest() == gold["L_sha256"]
    assert hashlib.sha256(np.ascontiguousarray(Hf, np.float64).tobytes()).hexdigest() == gold["H_sha256"]


def test_failing_h_rebuild_ends_the_solve_and_leaves_the_solver_usable():
    """A nonzero status from the callback ends the solve with CQ_ERR_CALLBACK; with the coupling
    switched off the same solver then reproduces the plain chain's fixture."""
    import cq_b200
    gold = GOLDEN["cases"]["r8_9_10_8"]
    coords, cell = inputs.diamond_si(2, sigma=0.1, seed=2)
    n = len(coords)
    o, g, ridx, S, H, olnv, glnv = _setup(coords, cell, np.full(n, 4), float(n), *gold["ranges"],
                                          max_outer=gold["max_outer"])
    glnv.set_h_rebuild(lambda k, h, length, stream: 3)
    glnv.set_SH(S, H)
    with pytest.raises(cq_b200.CQError) as err:
        glnv.solve()
    assert err.value.code == cq_b200.CQ_ERR_CALLBACK
    glnv.set_h_rebuild(None)
    res = glnv.solve()
    L = glnv.get("L")
    assert res["n_products"] == gold["n_products"]
    assert hashlib.sha256(np.ascontiguousarray(L, np.float64).tobytes()).hexdigest() == gold["L_sha256"]


def test_system_outlives_its_solvers():
    """cq_system_destroy refuses while a solver of the system is alive; System.close() destroys the
    system's solvers first, so finalising the Python objects in either order is safe."""
    import ctypes
    import cq_b200
    coords, cell = inputs.diamond_si(1, sigma=0.1, seed=2)
    n = len(coords)
    o, g, ridx, S, H, olnv, glnv = _setup(coords, cell, np.full(n, 4), float(n), 8.0, 9.0, 10.0, 8.0)
    glnv.set_SH(S, H)
    assert cq_b200.lib().cq_system_destroy(g.handle) == cq_b200.CQ_ERR_STATE
    assert g.length(ridx["L"]) > 0                  # the system is untouched
    g.close()                                       # destroys the solver, then the system
    assert not g.handle.value
    glnv.close()                                    # nothing left to destroy
    assert not glnv._h.value


GOLDEN512_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lnv_chain_si512.json")


def test_benchmark_workload_matches_oracle_chain():
    """The benchmark workload itself (512-atom Si supercell, 4x4 blocks, S/H/L/T ranges 10/12/16/10 bohr,
    1024 electrons, 50 LNV iterations, tolerance 1e-7): the GPU solve against the oracle chain's fixture.
    Products are bit-exact and every reduction exact on both sides, so the chains take the same steps:
    the same number of products, the same final L to the bit, E and Ne within 1e-10."""
    import cq_b200
    gold = json.load(open(GOLDEN512_PATH))["cases"]["r10_12_16_10"]
    coords, cell = inputs.diamond_si(4, sigma=0.1, seed=2)
    n = len(coords)
    rng = cq_b200.lnv_ranges(*gold["ranges"])
    ridx = {k: i for i, k in enumerate(rng)}
    g = cq_b200.System(coords, cell, np.full(n, 4, np.int32), list(rng.values()))
    S = inputs.overlap_S(g.blocklist(ridx["S"], coords, cell))
    H = inputs.hamiltonian_H(g.blocklist(ridx["H"], coords, cell), seed=5)
    solver = cq_b200.LNV(g, ridx, gold["ne_spin"], exact=1, max_outer=gold["max_outer"])
    res, L, _ = solver.solve_host(S, H, want_L=True)
    assert res["converged"] == int(gold["converged"])
    assert res["n_products"] == gold["n_products"]
    assert L.size == gold["L_length"]
    assert hashlib.sha256(np.ascontiguousarray(L, np.float64).tobytes()).hexdigest() == gold["L_sha256"]
    assert abs(res["energy"] - gold["energy"]) <= 1e-10 * abs(gold["energy"])
    assert abs(res["electrons"] - gold["electrons"]) <= 1e-10 * abs(gold["electrons"])
    solver.close()
