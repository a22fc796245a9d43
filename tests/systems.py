"""Standard seeded test systems (shapes of the benchmark configurations, smaller where noted)."""
import numpy as np

from cq_b200 import inputs

# range order used by the LNV tests: S, H, L, T and the products of the chain
# (rcut(LSrange) = L + S etc., src/dimens_module.f90:338-355)
def lnv_ranges(rs=10.0, rh=12.0, rl=16.0, rt=10.0):
    return {"S": rs, "H": rh, "L": rl, "T": rt, "LS": rl + rs, "LH": rl + rh, "LSL": 2 * rl + rs,
            "SLS": 2 * rs + rl, "TS": rt + rs, "TH": rt + rh, "TL": rt + rl}


def config1(ncell=3, sigma=0.05, seed=1):
    """mat_mult KAT system: diamond Si, 13x13 blocks, A range 8, B range 12, C range 20."""
    coords, cell = inputs.diamond_si(ncell, sigma=sigma, seed=seed)
    return coords, cell, np.full(len(coords), 13, np.int32), [8.0, 12.0, 20.0]


def config2(ncell=4, sigma=0.1, seed=2):
    """LNV system: diamond Si, 4x4 blocks."""
    coords, cell = inputs.diamond_si(ncell, sigma=sigma, seed=seed)
    return coords, cell, np.full(len(coords), 4, np.int32)
