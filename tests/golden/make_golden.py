"""Generate the LNV-chain fixtures of tests/golden from the CPU oracle.

    python tests/golden/make_golden.py

For each case (periodic 64-atom Si, SZ blocks, two range sets) the oracle chain (Hotelling
T = S^-1, then FindMinDM from the McWeeny start) is run on the seeded synthetic S and H, and the
band energy, electron count, number of products and a SHA-256 of the final L (the raw float64
bytes in the storage order of the oracle, which is the storage order of the library) are written
to lnv_chain_si64.json (with the pass limit and whether the chain converged).  The GPU tests compare against these numbers bit for bit.

lnv_scf_si64.json holds the same quantities for the chain with mixed-L self-consistency
(minE.MixedLSelfConsistent): lateDM rebuilds H = H0 + g K from K of the current L at its start and
after every Pulay step, a linear density feedback standing in for the grid rebuild of H, plus the
number of rebuilds and a SHA-256 of the final H.

lnv_chain_si512.json holds the same quantities for the benchmark workload: the 512-atom Si supercell
(4x4x4 cells, sigma 0.1 bohr, seed 2), SZ blocks, S/H/L/T ranges 10/12/16/10 bohr, 1024 electrons,
50 LNV iterations, tolerance 1e-7, solved to convergence.  It takes several minutes on the CPU.

    python tests/golden/make_golden.py [chain|scf|bench]      (default: chain and scf)
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "conquest-release_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

# name: (S, H, L, T ranges in bohr, FindMinDM pass limit).  With the short ranges the residual stalls
# above the tolerance (the reference would loop for ever), so that case stops after two passes and
# checks the iterates, not the minimum.
CASES = {"r8_9_10_8": ((8.0, 9.0, 10.0, 8.0), 2), "r10_12_16_10": ((10.0, 12.0, 16.0, 10.0), 40)}


def run_case(ranges, max_outer, feedback=None, ncell=2):
    import blockmaps as bm
    import cq_b200
    from cq_b200 import inputs
    from cq_oracle import OracleSystem
    from lnv_oracle import OracleLNV, Params
    coords, cell = inputs.diamond_si(ncell, sigma=0.1, seed=2)
    n = len(coords)
    rng = cq_b200.lnv_ranges(*ranges)
    ridx = {k: i for i, k in enumerate(rng)}
    o = OracleSystem(coords, cell, np.full(n, 4), list(rng.values()))
    S = inputs.overlap_S(bm.oracle_blocklist(o, ridx["S"], coords, cell))
    H = inputs.hamiltonian_H(bm.oracle_blocklist(o, ridx["H"], coords, cell), seed=5)
    lnv = OracleLNV(o, ridx, S, H, float(n), 4.0 * n, Params())
    extra = {}
    if feedback is not None:
        H0 = np.array(H, dtype=np.float64)
        lnv.h_rebuild = lambda K: H0 + feedback * K
    lnv.iter_hott_invs()
    E, N = lnv.find_min_dm(max_outer=max_outer)
    if feedback is not None:
        extra = {"feedback": feedback, "h_rebuilds": int(lnv.h_rebuilds),
                 "H_sha256": hashlib.sha256(np.ascontiguousarray(lnv.H.v, np.float64).tobytes()).hexdigest()}
    return {**extra,"ranges": list(ranges), "max_outer": max_outer, "converged": bool(lnv.converged), "atoms": n, "ne_spin": float(n), "energy": E, "electrons": N,
            "n_products": int(lnv.n_products),
            "L_sha256": hashlib.sha256(np.ascontiguousarray(lnv.L.v, np.float64).tobytes()).hexdigest(),
            "L_length": int(lnv.L.v.size)}


# name: (S, H, L, T ranges, pass limit, feedback g of H = H0 + g K)
SCF_CASES = {"r8_9_10_8_gm005": ((8.0, 9.0, 10.0, 8.0), 1, -0.05)}


def main(which=("chain", "scf")):
    if "bench" in which:
        out = {"system": "diamond Si 4x4x4 cells (512 atoms), sigma 0.1 bohr, seed 2; S overlap_S, H hamiltonian_H "
                         "seed 5; 4x4 blocks; ne_spin = 512 (1024 electrons); the benchmark workload", "cases": {}}
        t = time.time()
        out["cases"]["r10_12_16_10"] = run_case((10.0, 12.0, 16.0, 10.0), 40, ncell=4)
        out["cases"]["r10_12_16_10"]["oracle_seconds"] = round(time.time() - t, 1)
        print("si512", out["cases"]["r10_12_16_10"]["energy"], "%.1f s" % (time.time() - t), flush=True)
        json.dump(out, open(os.path.join(HERE, "lnv_chain_si512.json"), "w"), indent=1)
    if "scf" in which:
        out = {"system": "diamond Si 2x2x2 cells (64 atoms), sigma 0.1 bohr, seed 2; S overlap_S, H0 hamiltonian_H "
                         "seed 5; 4x4 blocks; ne_spin = 64; H = H0 + g K rebuilt by lateDM", "cases": {}}
        for name, (rg, mo, gfb) in SCF_CASES.items():
            t = time.time()
            out["cases"][name] = run_case(rg, mo, gfb)
            print(name, out["cases"][name]["energy"], "%.1f s" % (time.time() - t), flush=True)
        json.dump(out, open(os.path.join(HERE, "lnv_scf_si64.json"), "w"), indent=1)
    if "chain" not in which:
        return
    out = {"system": "diamond Si 2x2x2 cells (64 atoms), sigma 0.1 bohr, seed 2; S overlap_S, H hamiltonian_H seed 5; "
                     "4x4 blocks; ne_spin = 64", "cases": {}}
    for name, (rg, mo) in CASES.items():
        t = time.time()
        out["cases"][name] = run_case(rg, mo)
        print(name, out["cases"][name]["energy"], "%.1f s" % (time.time() - t), flush=True)
    json.dump(out, open(os.path.join(HERE, "lnv_chain_si64.json"), "w"), indent=1)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("chain", "scf"))
