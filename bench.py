#!/usr/bin/env python
"""Benchmark of the B200 LNV / McWeeny density-matrix solver (libcqb200.so).

Workload (N=1 default): plain FP64 LNV + McWeeny density-matrix minimisation on a
512-atom diamond Si supercell (4x4x4 conventional cells, a = 10.263 bohr, seeded
displacements sigma = 0.1 bohr), 4x4 (SZ) blocks, S range 10, H range 12,
L range 16, T range 10 bohr, 1024 electrons, DM.LVariations = 50, tolerance 1e-7.
One step = one complete solve on device-resident S and H: T = S^-1 by Hotelling
iterations, then FindMinDM from the McWeeny initial L.  Synthetic seeded inputs.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): independent replicas, one solve per rank
per step, no collectives on the data path (weak scaling); time is the max over
ranks.  `--impl reference` times the CPU restatement of the reference's
multiply_kernel_ompGemm chain on the host cores instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "conquest-release_b200"))

METRIC = "LNV solves/s (FP64, 512-atom Si SZ)"
WORKLOAD = "lnv512_si_sz_fp64"
CFG = dict(ncell=4, sigma=0.1, seed=2, rs=10.0, rh=12.0, rl=16.0, rt=10.0, nsf=4, ne_per_atom=2.0, h_seed=5)
SAMPLE_S = 5.0     # seconds of CPU chain per timed sample (reference arm step, cpu_baseline leg)


def build_problem(cq_b200):
    """System, solver and host S/H of the workload (setup, untimed)."""
    from cq_b200 import inputs
    coords, cell = inputs.diamond_si(CFG["ncell"], sigma=CFG["sigma"], seed=CFG["seed"])
    n = len(coords)
    rng = cq_b200.lnv_ranges(CFG["rs"], CFG["rh"], CFG["rl"], CFG["rt"])
    names = list(rng)
    ridx = {k: i for i, k in enumerate(names)}
    sysm = cq_b200.System(coords, cell, np.full(n, CFG["nsf"], np.int32), list(rng.values()))
    blS = sysm.blocklist(ridx["S"], coords, cell)
    blH = sysm.blocklist(ridx["H"], coords, cell)
    S = inputs.overlap_S(blS)
    H = inputs.hamiltonian_H(blH, seed=CFG["h_seed"])
    ne_spin = CFG["ne_per_atom"] * n / 2.0
    solver = cq_b200.LNV(sysm, ridx, ne_spin, exact=1)
    return dict(coords=coords, cell=cell, n=n, ridx=ridx, system=sysm, S=S, H=H, solver=solver, ne_spin=ne_spin)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


def fp64_peak_tflops(dev):
    """FP64 reference peak on this GPU, measured here: cuBLAS DGEMM (torch.matmul float64) 8192^3,
    best of 5 after 2 warm-ups (CUDA events)."""
    import torch
    n = 8192
    a = torch.rand(n, n, dtype=torch.float64, device=dev)
    b = torch.rand(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    best = 1e30
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best / 1e3) / 1e12


def load_traffic():
    """DRAM bytes of one captured launch of the dominant kernel, from the committed ncu summary:
    (bytes, description of the launch, its algorithmic bytes), or (None, None, None) if absent."""
    p = os.path.join(ROOT, "profiles", "lnv512_mult_traffic.json")
    if os.path.exists(p):
        try:
            d = json.load(open(p))
            return (d.get("dram_bytes_per_launch"), "%s on %s" % (d.get("kernel"), d.get("launch")),
                    d.get("algorithmic_bytes_of_launch"))
        except Exception:
            pass
    return None, None, None


def work_record_path():
    return os.path.join(ROOT, "profiles", "lnv512_solve_work.json")


def lnv_call_products():
    """The products of one LNV_matrix_multiply(doM3, dophi, doE) call (mult_module.f90:1557-1700), mat_mult roles."""
    return [(1, "L", "S", "LS"), (1, "L", "H", "LH"), (1, "LH", "S", "LSL"), (1, "LH", "S", "LSL"),
            (2, "L", "LS", "LSL"), (1, "LS", "S", "SLS"), (2, "L", "LS", "SLS"), (1, "LS", "L", "LSL"),
            (2, "H", "LS", "LSL")]


class _SampleDone(Exception):
    pass


def cpu_chain_setup(coords, cell, ridx, S, H, ne_spin, nthreads):
    """The oracle's restatement of the chain with the ompGemm kernel on `nthreads` host threads, set up to the
    point where FindMinDM's iterations start: T = S^-1 (Hotelling) and the McWeeny initial L (untimed).
    Returns (chain, L after the McWeeny start, its energy change)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ["OMP_NUM_THREADS"] = str(nthreads)
    from cq_oracle import OracleSystem
    from lnv_oracle import OracleLNV, Params
    import cq_b200
    rng = cq_b200.lnv_ranges(CFG["rs"], CFG["rh"], CFG["rl"], CFG["rt"])
    n = len(coords)
    o = OracleSystem(coords, cell, np.full(n, CFG["nsf"]), list(rng.values()))
    lnv = OracleLNV(o, ridx, S, H, ne_spin, float(CFG["nsf"] * n), Params(), kernel="ompGemm", nthreads=nthreads)
    lnv.iter_hott_invs()
    lnv.transpose(lnv.T, lnv.Ttran)
    lnv.init_mcw()
    de = lnv.mcw_min(lnv.p.n_L_iterations)
    return lnv, lnv.L.v.copy(), de


def cpu_chain_sample(lnv, L0, de0, budget_s):
    """One timed sample of the CPU chain: FindMinDM iterations (early and late DM, line searches, electron
    number corrections, Pulay steps: every product, sum, transpose and trace of the chain) from the McWeeny
    start, stopped before the first product that begins after `budget_s` seconds.
    Returns (seconds, algorithmic flops of the products run, products run)."""
    lnv.L.v[:] = L0
    lnv.delta_e = de0
    f0, p0 = lnv.flops, lnv.n_products
    t0 = time.perf_counter()

    def stop(_):
        if time.perf_counter() - t0 > budget_s:
            raise _SampleDone()
    lnv.before_product = stop
    try:
        lnv.find_min_dm(resetL=False)
    except _SampleDone:
        pass
    finally:
        lnv.before_product = None
    return time.perf_counter() - t0, lnv.flops - f0, lnv.n_products - p0


def cpu_record():
    """The committed record of one complete CPU solve of the workload timed on the GPU box's host cores
    (profiles/cpu_solve_lnv512.json), or None."""
    p = os.path.join(ROOT, "profiles", "cpu_solve_lnv512.json")
    return json.load(open(p)) if os.path.exists(p) else None


def cpu_full_solve(path):
    """One complete solve of the workload on the CPU chain (T = S^-1, McWeeny start, FindMinDM to
    convergence), the oracle's restatement with the ompGemm kernel on every host core, timed end to end."""
    from cq_b200 import inputs
    import cq_b200
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from cq_oracle import OracleSystem
    from lnv_oracle import OracleLNV, Params
    coords, cell = inputs.diamond_si(CFG["ncell"], sigma=CFG["sigma"], seed=CFG["seed"])
    n = len(coords)
    rng = cq_b200.lnv_ranges(CFG["rs"], CFG["rh"], CFG["rl"], CFG["rt"])
    ridx = {k: i for i, k in enumerate(rng)}
    o = OracleSystem(coords, cell, np.full(n, CFG["nsf"]), list(rng.values()))
    S = inputs.overlap_S(o.blocklist(ridx["S"], coords, cell))
    H = inputs.hamiltonian_H(o.blocklist(ridx["H"], coords, cell), seed=CFG["h_seed"])
    nth = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(nth)
    lnv = OracleLNV(o, ridx, S, H, CFG["ne_per_atom"] * n / 2.0, float(CFG["nsf"] * n), Params(), kernel="ompGemm",
                    nthreads=nth)
    t0 = time.perf_counter()
    lnv.iter_hott_invs()
    E, N = lnv.find_min_dm()
    t = time.perf_counter() - t0
    rec = {"workload": WORKLOAD, "what": "one complete solve on the CPU chain (oracle restatement, ompGemm kernel, "
                                         "OpenBLAS dgemm with one thread per OpenMP thread)",
           "cores": nth, "seconds": t, "energy": E, "electrons": N, "products": int(lnv.n_products),
           "flops": int(lnv.flops), "converged": bool(lnv.converged),
           "command": "python bench.py --cpu-full-solve " + os.path.relpath(path, ROOT)}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    json.dump(rec, open(path, "w"), indent=1)
    emit(rec)


def fixture_parity(res):
    """The timed solve against the oracle chain's committed fixture of this workload
    (tests/golden/lnv_chain_si512.json): energy, electron count and product count."""
    p = os.path.join(ROOT, "tests", "golden", "lnv_chain_si512.json")
    if not os.path.exists(p):
        return None
    gold = json.load(open(p))["cases"]["r10_12_16_10"]
    return {"fixture": "tests/golden/lnv_chain_si512.json", "oracle_energy": gold["energy"],
            "oracle_electrons": gold["electrons"], "oracle_products": gold["n_products"],
            "energy_identical": res["energy"] == gold["energy"],
            "energy_rel_diff": abs(res["energy"] - gold["energy"]) / abs(gold["energy"]),
            "electrons_rel_diff": abs(res["electrons"] - gold["electrons"]) / abs(gold["electrons"]),
            "products_identical": res["n_products"] == gold["n_products"]}


def config_of(n, ne_spin, ws):
    return {"workload": WORKLOAD, "atoms": n, "blocks": "4x4", "ranges_bohr": {"S": 10, "H": 12, "L": 16, "T": 10},
            "electrons": int(2 * ne_spin), "n_L_iterations": 50, "tolerance": 1e-7,
            "l2": "flushed (256 MB write) before every timed step", "parallelism": "replicas x%d" % ws}


def flops_of_lnv_call(system, ridx):
    tot = 0
    for (t, a, b, c) in lnv_call_products():
        tot += system.product_work(t, ridx[a], ridx[b], ridx[c])[1]
    return tot


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x, dist=None, device=None):
    """The largest value of x over all ranks (replicas are timed by their slowest rank); x itself
    without a process group."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank, world_size, seconds):
    """Whole-job throughput of independent replicas: every rank processed units_per_rank in at most `seconds`."""
    return world_size * units_per_rank / seconds


def emit(line):
    print(json.dumps(line), flush=True)


def reference_main(args, ws, rank):
    """CPU arm: the oracle's restatement of the reference's chain with the ompGemm kernel (OpenMP over all host
    cores, OpenBLAS dgemm with one thread), rank 0 only.

    Set-up (untimed, once): geometry, indices, S, H, T = S^-1 and the McWeeny start.  Each step then times a
    bounded sample of the solve, FindMinDM's iterations from the McWeeny start for about SAMPLE_S seconds, and
    counts the algorithmic flops of the products it ran.  solves/s = that flop rate / the flops of one complete
    solve (counted from the same chain's products, profiles/lnv512_solve_work.json).  A complete CPU solve timed
    once on the same host is reported beside it (profiles/cpu_solve_lnv512.json).
    """
    if rank != 0:
        return
    from cq_b200 import inputs
    import cq_b200
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from cq_oracle import OracleSystem
    rec = json.load(open(work_record_path()))
    coords, cell = inputs.diamond_si(CFG["ncell"], sigma=CFG["sigma"], seed=CFG["seed"])
    n = len(coords)
    rng = cq_b200.lnv_ranges(CFG["rs"], CFG["rh"], CFG["rl"], CFG["rt"])
    ridx = {k: i for i, k in enumerate(rng)}
    o = OracleSystem(coords, cell, np.full(n, CFG["nsf"]), list(rng.values()))
    S = inputs.overlap_S(o.blocklist(ridx["S"], coords, cell))
    H = inputs.hamiltonian_H(o.blocklist(ridx["H"], coords, cell), seed=CFG["h_seed"])
    ne_spin = CFG["ne_per_atom"] * n / 2.0
    nth = os.cpu_count() or 1
    lnv, L0, de0 = cpu_chain_setup(coords, cell, ridx, S, H, ne_spin, nth)
    for _ in range(min(args.warmup, 1)):
        cpu_chain_sample(lnv, L0, de0, 1.0)
    secs, flops, prods = [], [], []
    for _ in range(args.steps):
        t, f, pr = cpu_chain_sample(lnv, L0, de0, SAMPLE_S)
        secs.append(t); flops.append(f); prods.append(pr)
    rate = sum(flops) / sum(secs)                     # flop/s of the chain on the host cores
    full = cpu_record()
    est_s = (full["flops"] if full else rec["flops_per_solve"]) / rate
    if full and int(full["cores"]) == nth:
        solve_s, basis = float(full["seconds"]), "the complete solve timed on these host cores"
    else:
        solve_s, basis = est_s, "the sample's flop rate over the CPU chain's flops per solve"
    value = 1.0 / solve_s
    sample = ("timed: FindMinDM iterations of the workload from its McWeeny start (T = S^-1 and the start set up "
              "once, untimed), about %.0f s per step, %d steps: %d products, %.3g flop in %.1f s on %d threads "
              "(%.3g flop/s, %.0f s per solve at that rate); solves/s from %s (%.0f s per solve)" %
              (SAMPLE_S, args.steps, sum(prods), sum(flops), sum(secs), nth, rate, est_s, basis, solve_s))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": solve_s * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Si supercell, S/H generators)",
            "config": config_of(n, ne_spin, ws),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nth, "kind": "port", "sample": sample,
                             "sample_ms_per_step": 1e3 * float(np.mean(secs)), "sample_estimate_s_per_solve": est_s,
                             "full_solve_timed": full},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    emit(line)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mixed-sample-only", action="store_true",
                    help="run only the mixed-precision vs FP64 comparison on the DZP sample (with --tol, --max-outer)")
    ap.add_argument("--mixed-handover", type=float, default=None,
                    help="mixed-sample: residual at which the split-precision phase hands over to FP64 (default 1e-6)")
    ap.add_argument("--no-mixed-sample", action="store_true",
                    help="skip the mixed-precision vs FP64 comparison on the bounded DZP sample")
    ap.add_argument("--workload", default="lnv512",
                    choices=["lnv512", "batch", "serve", "mult216", "mult512", "mult216dzp", "mult4096", "forms216"],
                    help="lnv512: the plain FP64 512-atom solve (default); batch / serve: mixed-precision solves of "
                         "many systems on concurrent slots vs the FP64 path one at a time; mult216 / mult512 / "
                         "mult216dzp / mult4096: single block products (216-atom DZP C=A.B; the products of one LNV "
                         "call on the 512-atom SZ, 216-atom DZP and 4096-atom DZP cells); forms216: one 216-atom "
                         "DZP solve in each precision form")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fma", "bf16x3", "bf16x6", "fp64tc"])
    ap.add_argument("--variant", type=int, default=None, help="FP64 4x4 product kernel variant (-1 autotuned, 0..3, 5, 6)")
    ap.add_argument("--mixed-kernel", type=int, default=-1, choices=[-1, 0, 1],
                    help="split-precision products: -1 = chosen per product by the tile plan's useful fraction "
                         "(default), 0 = tcgen05 tiles, 1 = one block per mma.sync warp")
    ap.add_argument("--work-record", default=None,
                    help="write the workload's per-solve work (flops, products, energy) as JSON to this path")
    ap.add_argument("--cpu-full-solve", default=None, metavar="PATH",
                    help="time one complete solve of the workload on the CPU chain (the oracle's ompGemm restatement, "
                         "all host cores; several minutes) and write the record as JSON to PATH")
    ap.add_argument("--one-solve", action="store_true",
                    help="run exactly one solve of the workload and print its result (for launch lists under ncu)")
    ap.add_argument("--forms-cell", default="3,77,777", metavar="NCELL,SEED,SH_SEED",
                    help="forms216: the periodic Si cell (cells per side, displacement seed, S/H generator seed)")
    ap.add_argument("--forms", default=None, help="forms216: comma list of the forms to run (default all)")
    ap.add_argument("--history-stride", type=int, default=4, help="forms216: every n-th iteration in the history")
    ap.add_argument("--requests", type=int, default=32)
    ap.add_argument("--nmin", type=int, default=64)
    ap.add_argument("--nmax", type=int, default=1000)
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--batch-products", action="store_true",
                    help="batch / serve: gather the slots' FP64 products into shared persistent launches")
    ap.add_argument("--fp64-slots", action="store_true",
                    help="batch / serve: also run the FP64 path on the slots, without and with gathered products")
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--tol", type=float, default=None, help="batch/serve: residual tolerance of both arms")
    ap.add_argument("--max-outer", type=int, default=None, help="batch/serve: FindMinDM pass limit per request")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if args.workload == "forms216" and args.impl == "ours":
        return forms_main(args)
    if args.workload in ("mult216", "mult512", "mult216dzp", "mult4096") and args.impl == "ours":
        if rank == 0:
            mult_main(args)
        return
    if args.workload != "lnv512" and args.impl == "ours":
        if rank == 0:
            serve_main(args)
        return
    if args.impl == "reference":
        return reference_main(args, ws, rank)
    if args.mixed_sample_only:
        import torch
        import cq_b200
        torch.cuda.set_device(local)
        emit({"mixed_vs_fp64": mixed_vs_fp64(cq_b200, args.tol, args.max_outer, args.mixed_handover)})
        return
    if args.cpu_full_solve:
        if rank == 0:
            cpu_full_solve(args.cpu_full_solve)
        return
    import torch
    import cq_b200
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    prob = build_problem(cq_b200)
    system, solver = prob["system"], prob["solver"]
    if args.variant is not None:
        system.set_mult_variant(args.variant)
    # a dedicated stream: the library enqueues on it and the CUDA events are recorded on it (torch's
    # default stream handle is 0, which the library reads as "its own stream")
    stream = torch.cuda.Stream(device=torch.device("cuda", local))
    torch.cuda.set_stream(stream)
    system.set_stream(stream.cuda_stream)
    dev = torch.device("cuda", local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # 256 MB > 126 MB L2
    solver.set_SH(prob["S"], prob["H"])
    if args.one_solve:
        r = solver.solve()
        torch.cuda.synchronize()
        emit({"one_solve": {k: r[k] for k in ("energy", "electrons", "converged", "n_products")},
              "gpu_launches": system.launch_count()})
        return
    for _ in range(args.warmup):
        res = solver.solve()
    torch.cuda.synchronize()
    # ---- timed region: K solves on device-resident S, H (no per-kernel events inside)
    launches0 = system.launch_count()
    step_ms = []
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev_all0, ev_all1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev_all0.record(stream)
        for _ in range(args.steps):
            flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            res = solver.solve()
            e1.record(stream)
            step_ms.append((e0, e1))
        ev_all1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    total_ms = ev_all0.elapsed_time(ev_all1)
    steps_ms = [a.elapsed_time(b) for a, b in step_ms]
    launches = system.launch_count() - launches0
    # ---- one more solve with CUDA events around every product launch (kernel-level numbers)
    system.profile(True)
    flush.zero_()
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    solver.solve()
    p1.record(stream)
    torch.cuda.synchronize()
    prof_step_ms = p0.elapsed_time(p1)
    prof = system.profile_read()
    system.profile(False)
    t_max = max_over_ranks(total_ms, dist, dev)
    value = replica_rate(args.steps, ws, t_max / 1e3)
    # ---- end to end through the host-memory C ABI call (pinned host S, H in; L, K out)
    pinS = torch.from_numpy(prob["S"]).pin_memory()
    pinH = torch.from_numpy(prob["H"]).pin_memory()
    nL = system.length(prob["ridx"]["L"]); nK = system.length(prob["ridx"]["H"])
    pinL = torch.empty(nL, dtype=torch.float64).pin_memory()
    pinK = torch.empty(nK, dtype=torch.float64).pin_memory()
    e2e_steps = max(1, min(args.steps, 3))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        solve_host_pinned(solver, pinS, pinH, pinL, pinK)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    e2e_value = replica_rate(e2e_steps, ws, e2e_s)
    if rank == 0:
        peak, peak_kind = load_peaks()
        achieved = prof["bytes"] / (prof["ms"] / 1e3) / 1e9 if prof["ms"] > 0 else 0.0
        traffic = load_traffic()
        dgemm = fp64_peak_tflops(dev)
        per_solve_flops = res["flops"]
        fl_call = flops_of_lnv_call(system, prob["ridx"])
        rec = {"workload": WORKLOAD, "flops_per_solve": per_solve_flops, "products_per_solve": res["n_products"],
               "flops_per_lnv_call": fl_call, "energy": res["energy"], "electrons": res["electrons"]}
        if args.work_record:
            os.makedirs(os.path.dirname(os.path.abspath(args.work_record)), exist_ok=True)
            json.dump(rec, open(args.work_record, "w"), indent=1)
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            nth = os.cpu_count() or 1
            lnv_c, L0, de0 = cpu_chain_setup(prob["coords"], prob["cell"], prob["ridx"], prob["S"], prob["H"],
                                             prob["ne_spin"], nth)
            t_c, f_c, p_c = cpu_chain_sample(lnv_c, L0, de0, 2 * SAMPLE_S)
            rate_c = f_c / t_c
            full = cpu_record()
            est_s = (full["flops"] if full else per_solve_flops) / rate_c
            solve_s = float(full["seconds"]) if full and int(full["cores"]) == nth else est_s
            cpu = {"value": 1.0 / solve_s, "unit": "solves/s", "cores": nth, "kind": "port",
                   "sample": "timed: FindMinDM iterations of this solve on the oracle's ompGemm chain from the McWeeny "
                             "start (set up untimed): %d products, %.3g flop in %.1f s on %d threads (%.0f s per solve "
                             "at that rate); solves/s from %s (%.0f s per solve)" %
                             (p_c, f_c, t_c, nth, est_s,
                              "the complete solve timed on these host cores" if solve_s != est_s else "that rate",
                              solve_s),
                   "full_solve_timed": full}
        clocks = clk.summary()
        mixed = None
        if ws == 1 and not args.no_mixed_sample:
            torch.cuda.synchronize()
            mixed = mixed_vs_fp64(cq_b200)
        srt = sorted(steps_ms)
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Si supercell, S/H generators)",
            "config": config_of(prob["n"], prob["ne_spin"], ws),
            "latency_ms": {"p50": float(np.percentile(srt, 50)), "p99": float(np.percentile(srt, 99))},
            "solve": {"energy": res["energy"], "electrons": res["electrons"], "products": res["n_products"],
                      "flops": per_solve_flops, "late_iters": res["late_iters"], "early_iters": res["early_iters"],
                      "mcw_sweeps": res["mcw_sweeps"], "converged": res["converged"]},
            "parity": fixture_parity(res),
            "mixed_vs_fp64": mixed,
            "block_mult_tflops": (prof["flops"] / (prof["ms"] / 1e3) / 1e12) if prof["ms"] > 0 else None,
            "roofline": {"bound": "hbm", "kernel": "FP64 4x4 block products (autotuned k_mult_nd4_warp / k_mult_nd4_quad)", "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic[0], "traffic_launch": traffic[1],
                         "traffic_launch_algorithmic_bytes": traffic[2], "launches": prof["launches"],
                         "avg_launch_ms": prof["ms"] / max(1, prof["launches"]),
                         "algorithmic_bytes_per_launch": prof["bytes"] / max(1, prof["launches"]),
                         "share_of_step": prof["ms"] / prof_step_ms if prof_step_ms > 0 else None,
                         "measured_in": "one extra solve with CUDA events around every product launch"},
            "roofline_fp64": {"bound": "fp64", "achieved": (prof["flops"] / (prof["ms"] / 1e3) / 1e12) if prof["ms"] > 0 else None,
                              "peak": dgemm, "peak_kind": "measured here: cuBLAS DGEMM 8192^3", "unit": "TFLOP/s",
                              "frac": ((prof["flops"] / (prof["ms"] / 1e3) / 1e12) / dgemm) if prof["ms"] > 0 else None},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": 8 * (prob["S"].size + prob["H"].size),
                    "d2h_bytes_per_step": 8 * (nL + nK)},
            "gpu_launches": launches,
            "gpu_launches_per_step": launches / max(1, args.steps),
            "clocks": clocks,
        }
        emit(line)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ----------------------------------------------------------------------------
# batched / served solves (the Batching-with-serving form)
# ----------------------------------------------------------------------------
SERVE_RANGES = (10.0, 12.0, 16.0, 10.0)   # S, H, L, T (bohr), as the 512-atom workload
# residual at which both arms stop: at the default 1e-7 two FP64 solves of one problem from different
# starting points differ by ~1e-7 Ha/atom, so the 1e-8 Ha/atom comparison needs a tighter stop
SERVE_TOL = 1e-9
SERVE_MAX_OUTER = 4        # FindMinDM passes per request (a stalled residual stops there)


def request_set(n_req, nmin, nmax, seed):
    """Seeded systems of the batched/served workloads: atom counts log-uniform in [nmin, nmax],
    alternately clusters carved from the Si lattice and periodic supercells, 4x4 and 13x13 blocks
    alternating in pairs, sigma = 0.1 bohr, per-request generator seed."""
    from cq_b200 import inputs
    rs = np.random.default_rng(seed)
    out = []
    for k in range(n_req):
        n = int(round(np.exp(rs.uniform(np.log(nmin), np.log(nmax)))))
        if k % 2 == 0:
            c, cell = inputs.si_cluster(n, sigma=0.1, seed=1000 + k)
        else:
            m = int(np.clip(round((n / 8.0) ** (1.0 / 3.0)), 2, 10))
            c, cell = inputs.diamond_si(m, sigma=0.1, seed=1000 + k)
        # 4x4 and 13x13 blocks alternate in pairs up to 1000 atoms (the batched configuration's range);
        # larger systems of the served range use 4x4 blocks (a 13x13 system of several thousand atoms
        # needs some 25 GB per matrix of its 42-bohr range)
        nsf = 4 if ((k // 2) % 2 == 0 or len(c) > 1000) else 13
        ne = float(len(c)) if nsf == 4 else 2.0 * len(c)
        out.append(dict(coords=c, cell=cell, nsf=nsf, ne=ne, seed=5000 + k, n=len(c)))
    return out


def run_server(cq_b200, reqs, n_slots, mixed, rate=None, seed=0, batch_products=False, **lnv):
    """Submit the requests (all at once, or as a Poisson stream of `rate` per second) and wait for all.
    batch_products: the slots' FP64 products are gathered into shared persistent launches; lnv: further
    solver parameters (cq_lnv_params fields)."""
    srv = cq_b200.Server(n_slots=n_slots, hbm_budget=int(0.8 * torch_total_mem()), tolerance=SERVE_TOL,
                         batch_products=batch_products,
                         max_outer=SERVE_MAX_OUTER, **lnv)
    t_arr = np.zeros(len(reqs))
    if rate:
        t_arr = np.cumsum(np.random.default_rng(seed).exponential(1.0 / rate, size=len(reqs)))
    t0 = srv.now()
    ids = []
    for r, ta in zip(reqs, t_arr):
        while srv.now() - t0 < ta:
            time.sleep(min(0.002, max(0.0, ta - (srv.now() - t0))))
        ids.append(srv.submit(r["coords"], r["cell"], r["nsf"], *SERVE_RANGES, r["ne"], seed=r["seed"], mixed=mixed,
                              t_arrival=t0 + ta))
    res = [srv.wait(i) for i in ids]
    t1 = max(x["t_done"] for x in res)
    srv.close()
    return res, t1 - t0


def mixed_sample_requests():
    """Bounded DZP sample of the mixed-precision comparison in the default bench line: four periodic Si
    supercells of 64 atoms (2x2x2 cells, sigma 0.1 bohr, different seeds), 13x13 blocks, 2 electrons per
    atom, ranges as the 512-atom workload, per-request generator seeds."""
    from cq_b200 import inputs
    out = []
    for k in range(4):
        c, cell = inputs.diamond_si(2, sigma=0.1, seed=2000 + k)
        out.append(dict(coords=c, cell=cell, nsf=13, ne=2.0 * len(c), seed=6000 + k, n=len(c)))
    return out


MIXED_SAMPLE_TOL = 1e-8    # residual at which both arms of the mixed-precision comparison stop
MIXED_SAMPLE_MAX_OUTER = 12


def mixed_vs_fp64(cq_b200, tol=None, max_outer=None, handover=None):
    """The precision form against the plain FP64 path on the bounded DZP sample: FP64 solves one at a
    time, mixed-precision solves on 4 concurrent slots; both stop at residual `tol` (pass limit
    `max_outer`).  Solves/s of both arms, their ratio, and |dE| per atom of every request."""
    global SERVE_TOL, SERVE_MAX_OUTER
    saved = (SERVE_TOL, SERVE_MAX_OUTER)
    SERVE_TOL = MIXED_SAMPLE_TOL if tol is None else tol
    SERVE_MAX_OUTER = MIXED_SAMPLE_MAX_OUTER if max_outer is None else max_outer
    try:
        reqs = mixed_sample_requests()
        fp, t_fp = run_server(cq_b200, reqs, 1, False)
        extra = {} if handover is None else {"mixed_tolerance": float(handover)}
        mx, t_mx = run_server(cq_b200, reqs, 4, True, **extra)
        tol_used, mo_used = SERVE_TOL, SERVE_MAX_OUTER
    finally:
        SERVE_TOL, SERVE_MAX_OUTER = saved
    per = [{"n": a["n_atoms"], "fp64_converged": int(a["converged"]), "mixed_converged": int(b["converged"]),
            "fp64_residual": a["residual"], "mixed_residual": b["residual"],
            "fp64_electrons": a["electrons"], "mixed_electrons": b["electrons"],
            "dE_per_atom_Ha": (b["energy"] - a["energy"]) / a["n_atoms"], "fp64_s": a["t_done"] - a["t_admit"],
            "mixed_s": b["t_done"] - b["t_admit"], "split_restart": b["split_restarts"]}
           for a, b in zip(fp, mx) if a["status"] == 0 and b["status"] == 0]
    both = [abs(r["dE_per_atom_Ha"]) for r in per if r["fp64_converged"] and r["mixed_converged"]]
    return {"sample": "4 periodic DZP (13x13) Si supercells of 64 atoms; S/H/L/T 10/12/16/10 bohr; both arms stop at "
                      "residual %g (pass limit %d)" % (tol_used, mo_used),
            "fp64": {"solves_per_s": len(reqs) / t_fp, "seconds": t_fp, "slots": 1},
            "mixed": {"solves_per_s": len(reqs) / t_mx, "seconds": t_mx, "slots": 4,
                      "precision": "bf16x6 split products (three bf16 parts, tensor cores, FP64 sums over block "
                                   "pairs), FP64 traces, line search, Hotelling, McWeeny start and FP64 continuation "
                                   "from residual %g" % (max(tol_used, 1e-8) if handover is None else handover)},
            "ratio": t_fp / t_mx,
            "max_abs_dE_per_atom_Ha_converged": max(both) if both else None,
            "per_request": per,
            "failed": sum(1 for r in fp + mx if r["status"] != 0),
            "target": "mixed >= 5x the FP64 solves/s at <= 1e-8 Ha/atom"}


def torch_total_mem():
    import torch
    return torch.cuda.get_device_properties(0).total_memory


def serve_main(args):
    """Batched (all requests at t=0) or served (Poisson arrivals) density-matrix solves, mixed precision on
    n_slots concurrent slots, against the plain FP64 path run one request at a time on the same set."""
    import torch
    import cq_b200
    torch.cuda.set_device(0)
    global SERVE_TOL, SERVE_MAX_OUTER
    if args.tol is not None:
        SERVE_TOL = args.tol
    if args.max_outer is not None:
        SERVE_MAX_OUTER = args.max_outer
    reqs = request_set(args.requests, args.nmin, args.nmax, seed=7)
    rate = args.rate if args.workload == "serve" else None
    warm = request_set(2, 64, 64, seed=99)
    run_server(cq_b200, warm, 2, True)
    with ClockSampler(0) as clk:
        fp, t_fp = run_server(cq_b200, reqs, 1, False)
        mx, t_mx = run_server(cq_b200, reqs, args.slots, True, rate=rate, seed=11, batch_products=args.batch_products)
        fps = fpb = None
        if args.fp64_slots:
            # the FP64 path on the same slots: products launched per solve, then gathered across the slots
            fps, t_fps = run_server(cq_b200, reqs, args.slots, False, rate=rate, seed=11)
            fpb, t_fpb = run_server(cq_b200, reqs, args.slots, False, rate=rate, seed=11, batch_products=True)
    bad = [r for r in fp + mx if r["status"] != 0]
    ok = [(a, b) for a, b in zip(fp, mx) if a["status"] == 0 and b["status"] == 0 and a["converged"] and b["converged"]]
    err = max([abs(a["energy"] - b["energy"]) / a["n_atoms"] for a, b in ok], default=None)
    lat = np.array([r["latency"] for r in mx]) * 1e3
    atoms = sum(r["n"] for r in reqs)
    flops_fp64 = sum(r["flops"] for r in fp)
    line = {
        "metric": "LNV solves/s (%s, mixed precision, %d slots)" % ("served" if rate else "batched", args.slots),
        "value": len(reqs) / t_mx, "unit": "solves/s", "n_gpus": 1, "higher_is_better": True,
        "dtype": "bf16x6+f64", "data": "synthetic (seeded Si clusters and supercells, S/H generators)",
        "config": {"workload": "lnv_%s_si_mixed" % args.workload, "requests": len(reqs),
                   "atoms": [args.nmin, args.nmax], "atoms_total": atoms, "blocks": "4x4 and 13x13",
                   "ranges_bohr": dict(zip("SHLT", SERVE_RANGES)), "arrival_rate_per_s": rate,
                   "slots": args.slots, "tolerance": SERVE_TOL, "max_outer": SERVE_MAX_OUTER},
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "fp64_path": {"value": len(reqs) / t_fp, "unit": "solves/s", "slots": 1,
                      "latency_ms_p50": float(np.percentile([r["latency"] * 1e3 for r in fp], 50)),
                      "block_mult_flops": flops_fp64},
        "speedup_vs_fp64_path": t_fp / t_mx,
        "fp64_on_slots": None if fps is None else {
            "slots": args.slots, "solves_per_s": len(reqs) / t_fps,
            "products_gathered_solves_per_s": len(reqs) / t_fpb,
            "identical_results_gathered": all(a["energy"] == b["energy"] and a["n_products"] == b["n_products"]
                                              for a, b in zip(fps, fpb) if a["status"] == 0 and b["status"] == 0)},
        "batch_products": bool(args.batch_products),
        "max_energy_error_per_atom": err,
        "failed": len(bad), "converged": sum(r["converged"] for r in mx),
        "failures": [{"n_atoms": r["n_atoms"], "mixed": r["mixed"], "message": r["message"]} for r in bad][:8],
        "per_request": [{"n": a["n_atoms"], "nsf": q["nsf"], "fp64_s": a["t_done"] - a["t_admit"],
                         "mixed_s": b["t_done"] - b["t_admit"], "conv": [a["converged"], b["converged"]],
                         "dE_per_atom": (b["energy"] - a["energy"]) / a["n_atoms"],
                         "products": [a["n_products"], b["n_products"]],
                         "flops": [a["flops"], b["flops"]], "flops_split_mixed": b["flops_mixed"],
                         "split_restart": b["split_restarts"]}
                        for a, b, q in zip(fp, mx, reqs)],
        "bytes_peak_max": max(r["bytes_peak"] for r in mx),
        "clocks": clk.summary(),
    }
    emit(line)


# ----------------------------------------------------------------------------
# precision forms of one DZP solve
# ----------------------------------------------------------------------------
FORMS = [("fp64", dict(exact=1)),
         ("fp64_fma", dict(exact=0)),
         ("fp64_tensor", dict(mixed=1, split_parts=0)),
         ("bf16x6+fp64_tensor", dict(mixed=1)),
         ("bf16x6+fp64", dict(mixed=1, fp64_tensor=0)),
         ("bf16x3+fp64", dict(mixed=1, split_parts=2, fp64_tensor=0))]


def forms_main(args):
    """One 216-atom DZP solve (3x3x3 Si cells, sigma 0.1 bohr, seed 77; 13x13 blocks; S/H/L/T 10/12/16/10
    bohr; 432 electrons; S and H from the device generators with seed 777) in each precision form: the
    plain FP64 path, FP64 with fused multiply-add on the CUDA cores and on the FP64 tensor cores, and the
    mixed forms.  Every solve stops at residual --tol (default 1e-8) within 16 passes; one untimed solve
    of the plain and of the default mixed form first builds and tunes the plans."""
    import torch
    import cq_b200
    from cq_b200 import inputs
    torch.cuda.set_device(0)
    tol = args.tol if args.tol is not None else 1e-8
    ncell, cseed, shseed = (int(x) for x in args.forms_cell.split(","))
    coords, cell = inputs.diamond_si(ncell, sigma=0.1, seed=cseed)
    n = len(coords)
    rng = cq_b200.lnv_ranges(10.0, 12.0, 16.0, 10.0)
    ridx = {k: i for i, k in enumerate(rng)}
    g = cq_b200.System(coords, cell, np.full(n, 13, np.int32), list(rng.values()))
    dev = torch.device("cuda", 0)
    S = torch.empty(g.length(ridx["S"]), dtype=torch.float64, device=dev)
    H = torch.empty(g.length(ridx["H"]), dtype=torch.float64, device=dev)
    g.generate_SH(ridx["S"], 0, shseed, S)
    g.generate_SH(ridx["H"], 1, shseed, H)
    torch.cuda.synchronize()

    def solve(kw):
        sol = cq_b200.LNV(g, ridx, float(n), tolerance=tol, max_outer=16, **kw)
        sol.set_SH(S, H)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = sol.solve()
        dt = time.perf_counter() - t0
        h = sol.residual_history()
        sol.close()
        return r, dt, h

    forms = [f for f in FORMS if not args.forms or f[0] in args.forms.split(",")]
    for kw in (FORMS[0][1], FORMS[3][1]):
        solve(kw)
    out, ref = [], None
    with ClockSampler(0) as clk:
        for name, kw in forms:
            r, dt, h = solve(kw)
            if ref is None:
                ref = r
            split_rows = [x for x in h if x[3] == 1]
            out.append({"form": name, "seconds": dt, "speedup_vs_fp64": None if not out else out[0]["seconds"] / dt,
                        "energy": r["energy"], "dE_per_atom_vs_fp64": (r["energy"] - ref["energy"]) / n,
                        "converged": r["converged"], "residual": r["residual"], "products": r["n_products"],
                        "products_split": r["n_products_mixed"], "iterations": len(h),
                        "seconds_to_first_iteration": float(h[0][4]) if len(h) else None,
                        "split_phase_end": None if not split_rows else
                        {"residual": float(split_rows[-1][0]), "seconds": float(split_rows[-1][4]),
                         "products": int(split_rows[-1][2])},
                        "history": [[float("%.3g" % x[0]), int(x[2]), int(x[3]), round(float(x[4]), 2)]
                                    for x in h[::args.history_stride]]})
    if out:
        out[0]["speedup_vs_fp64"] = 1.0
    emit({"metric": "one DZP LNV solve per precision form (seconds)", "value": out[-1]["seconds"], "unit": "s",
          "n_gpus": 1, "higher_is_better": False, "dtype": "f64 / bf16x6+f64 / bf16x3+f64", "data": "synthetic",
          "config": {"workload": "forms216", "system": "%d-atom Si DZP (13x13), %dx%dx%d cells, sigma 0.1, seed %d, "
                                                     "S/H seed %d" % (n, ncell, ncell, ncell, cseed, shseed),
                     "ranges_bohr": {"S": 10.0, "H": 12.0, "L": 16.0, "T": 10.0}, "electrons": 2 * n,
                     "tolerance": tol, "max_outer": 16},
          "forms": out, "clocks": clk.summary()})


# ----------------------------------------------------------------------------
# single products: config 1 (216-atom DZP mat_mult) and the products of one LNV call
# ----------------------------------------------------------------------------
def mult_main(args):
    """Time block products on device-resident operands with CUDA events (L2 flushed before each launch).

    mult216: C = A.B on a 216-atom Si supercell (3x3x3 cells, sigma 0.05), 13x13 blocks, A range 8,
             B range 12, C range 20, entries uniform[-1,1] exp(-r/3).
    mult512 / mult216dzp / mult4096: the nine products of one LNV_matrix_multiply(M3, phi, E) call on the
             512-atom SZ workload, on a 216-atom DZP cell (3x3x3 cells, sigma 0.1, seed 77) and on the
             4096-atom DZP cell (8x8x8 cells).
    """
    import torch
    import cq_b200
    from cq_b200 import inputs
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(device=dev)      # the library's stream, where the events are recorded
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    prec = {"fp64": cq_b200.PREC_FP64, "fma": cq_b200.PREC_FP64_FMA, "bf16x3": cq_b200.PREC_BF16X3,
            "bf16x6": cq_b200.PREC_BF16X6, "fp64tc": cq_b200.PREC_FP64_TC}[args.precision]
    if args.workload == "mult216":
        coords, cell = inputs.diamond_si(3, sigma=0.05, seed=1)
        n = len(coords)
        g = cq_b200.System(coords, cell, np.full(n, 13, np.int32), [8.0, 12.0, 20.0])
        a = torch.from_numpy(inputs.random_blocks(g.blocklist(0, coords, cell), 1, inputs.TAG_RANDOM_A)).to(dev)
        b = torch.from_numpy(inputs.random_blocks(g.blocklist(1, coords, cell), 1, inputs.TAG_RANDOM_B)).to(dev)
        c = torch.zeros(g.length(2), dtype=torch.float64, device=dev)
        prods = [("A.B->C", 1, 0, 1, 2, a, b, c)]
        desc = "216-atom Si DZP (13x13), A 8 / B 12 / C 20 bohr"
    else:
        from cq_b200 import inputs as _inp
        ncell, nsf = {"mult512": (4, 4), "mult216dzp": (3, 13)}.get(args.workload, (8, 13))
        coords, cell = _inp.diamond_si(ncell, sigma=0.1, seed=77 if args.workload == "mult216dzp" else 2)
        n = len(coords)
        rng = cq_b200.lnv_ranges(CFG["rs"], CFG["rh"], CFG["rl"], CFG["rt"])
        ridx = {k: i for i, k in enumerate(rng)}
        g = cq_b200.System(coords, cell, np.full(n, nsf, np.int32), list(rng.values()))
        gen = torch.Generator(device=dev)
        gen.manual_seed(3)
        mats = {k: (torch.rand(g.length(ridx[k]), dtype=torch.float64, device=dev, generator=gen) - 0.5) * 0.2
                for k in ("S", "H", "L", "LS", "LH", "LSL", "SLS")}
        prods = []
        for (t, x, y, z) in lnv_call_products():
            prods.append(("%s_%s_%s/%d" % (x, y, z, t), t, ridx[x], ridx[y], ridx[z], mats[x], mats[y], mats[z]))
        desc = "%d-atom Si %s, S/H/L/T ranges 10/12/16/10 bohr: the nine products of one LNV call" % (
            n, "SZ (4x4)" if nsf == 4 else "DZP (13x13)")
    torch.cuda.synchronize()
    g.set_stream(stream.cuda_stream)
    if args.variant is not None:
        g.set_mult_variant(args.variant)
    g.set_mixed_kernel(args.mixed_kernel)
    out = []
    with ClockSampler(0) as clk:
        for (name, t, ra, rb, rc, A, B, C) in prods:
            triples, flops = g.product_work(t, ra, rb, rc)
            for _ in range(args.warmup):
                g.mat_mult(t, ra, rb, rc, A, B, C, precision=prec)
            torch.cuda.synchronize()
            ms = []
            for _ in range(args.steps):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                g.mat_mult(t, ra, rb, rc, A, B, C, precision=prec)
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            m = float(np.median(ms))
            nbytes = 8.0 * (g.length(ra) + g.length(rb) + g.length(rc))
            tv, tms = g.product_tuning(t, ra, rb, rc, mixed=(args.precision in ("bf16x3", "bf16x6")))
            tensor = None
            if args.precision == "bf16x3" and args.mixed_kernel != 1:
                nt, issued, usable = g.product_tensor_work(t, ra, rb, rc)
                tensor = {"tiles": nt, "issued_tflop": issued / 1e12, "useful_fraction": 3.0 * flops / max(issued, 1),
                          "issued_tflops": issued / (m / 1e3) / 1e12}
            out.append({"product": name, "triples": triples, "flops": flops, "ms": m, "tuned_variant": tv,
                        "tune_ms": tms, "tensor": tensor,
                        "tflops": flops / (m / 1e3) / 1e12, "gbs_algorithmic": nbytes / (m / 1e3) / 1e9})
    tot_fl = sum(o["flops"] for o in out)
    tot_ms = sum(o["ms"] for o in out)
    emit({"metric": "block-mult TFLOP/s (%s)" % args.precision, "value": tot_fl / (tot_ms / 1e3) / 1e12,
          "unit": "TFLOP/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
          "dtype": {"fp64": "f64", "fma": "f64", "bf16x3": "bf16x3", "bf16x6": "bf16x6", "fp64tc": "f64"}[args.precision],
          "data": "synthetic", "config": {"workload": args.workload, "system": desc, "variant": args.variant,
                                          "mixed_kernel": args.mixed_kernel,
                                          "l2": "flushed (256 MB write) before every timed launch"},
          "products": out, "clocks": clk.summary()})


def solve_host_pinned(solver, pinS, pinH, pinL, pinK):
    """cq_lnv_solve_host with pinned host buffers: S, H copied in, L and K copied out."""
    import ctypes
    import cq_b200
    r = cq_b200.LNVResult()
    P = ctypes.POINTER(ctypes.c_double)
    cq_b200.check(cq_b200.lib().cq_lnv_solve_host(
        solver._h, ctypes.cast(pinS.data_ptr(), P), ctypes.cast(pinH.data_ptr(), P), ctypes.cast(pinL.data_ptr(), P),
        ctypes.cast(pinK.data_ptr(), P), ctypes.byref(r)))
    return r.as_dict()


if __name__ == "__main__":
    main()
