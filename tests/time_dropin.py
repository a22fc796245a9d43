"""Timing of the drop-in kernel pair on the 216-atom DZP product (13x13 blocks, A range 8, B range 12,
C range 20 bohr: C = A.B), beside the mat_mult-level entries, on one GPU.

    python tests/time_dropin.py            (prints one JSON line)

The drop-in path is driven as a Fortran build with MULT_KERN=gpu would drive it: mat_mult's partition
loop (tests/dropin_driver.py, with the reference-layout index arrays the oracle exports) calling
cq_m_kern_max once per A-halo partition, either completing every call or deferred (cq_m_kern_defer).
Times are wall-clock seconds of whole products with host arrays in and out (median of 5 after 1
warm-up); cq_mat_mult on device-resident operands is timed with CUDA events.
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "conquest-release_b200"))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
sys.path.insert(0, HERE)


def main():
    import torch
    import cq_b200
    import blockmaps as bm
    import dropin_driver
    import systems
    from cq_b200 import inputs
    from cq_oracle import OracleSystem
    torch.cuda.set_device(0)
    coords, cell, nsf, rc = systems.config1()
    o = OracleSystem(coords, cell, nsf, rc)
    g = cq_b200.System(coords, cell, nsf, rc)
    bls = [bm.oracle_blocklist(o, r, coords, cell) for r in range(3)]
    a = inputs.random_blocks(bls[0], 1, inputs.TAG_RANDOM_A)
    b = inputs.random_blocks(bls[1], 1, inputs.TAG_RANDOM_B)
    ref = np.zeros(bls[2].length)
    o.mat_mult(1, 0, 1, 2, a, b, ref)

    def wall(f, reps=5):
        f()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            f()
            ts.append(time.perf_counter() - t0)
        return float(np.median(ts))

    out = {}
    c1 = np.zeros(bls[2].length)
    out["dropin_per_call_s"] = wall(lambda: dropin_driver.mat_mult_dropin(o, 1, 0, 1, 2, a, b, c1, False))
    c2 = np.zeros(bls[2].length)
    out["dropin_deferred_s"] = wall(lambda: dropin_driver.mat_mult_dropin(o, 1, 0, 1, 2, a, b, c2, True))
    c3 = np.zeros(bls[2].length)
    out["mat_mult_host_s"] = wall(lambda: g.mat_mult_host(1, 0, 1, 2, a, b, c3))
    da, db = torch.tensor(a, device="cuda"), torch.tensor(b, device="cuda")
    dc = torch.zeros(bls[2].length, dtype=torch.float64, device="cuda")
    g.mat_mult(1, 0, 1, 2, da, db, dc)
    g.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st = torch.cuda.current_stream()
    g.set_stream(st.cuda_stream)
    e0.record(st)
    for _ in range(5):
        g.mat_mult(1, 0, 1, 2, da, db, dc)
    e1.record(st)
    torch.cuda.synchronize()
    g.set_stream(None)
    out["mat_mult_device_s"] = e0.elapsed_time(e1) / 5 / 1e3
    # the partition loop the drop-in calls see
    out["partitions"] = int(len(o.geti("lab_hcell", 0)))
    out["bit_exact"] = bool(np.array_equal(c1, ref) and np.array_equal(c2, ref) and np.array_equal(c3, ref)
                            and np.array_equal(dc.cpu().numpy(), ref))
    out["workload"] = "216-atom Si DZP (13x13), A 8 / B 12 / C 20 bohr, C = A.B"
    print(json.dumps(out))


if __name__ == "__main__":
    main()
