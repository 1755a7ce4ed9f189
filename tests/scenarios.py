"""Seeded test scenarios shared by the CPU and GPU tests."""
import json

import numpy as np

from icempm_multi_b200 import make_block, parse_json
from icempm_multi_b200._lib import STATUS_CRUSHED, STATUS_DISABLED, STATUS_LIQUID


def params_for(grid_x, grid_y, h, dt, **kw):
    cfg = {
        "InputRawPoints": "synthetic", "nPartitions": 1, "GridHaloSize": kw.pop("halo", 8),
        "InitialTimeStep": dt, "GridX": grid_x, "GridY": grid_y, "GridXDimension": grid_x * h,
        "YoungsModulus": 1e9, "PoissonsRatio": 0.3, "Density": 980, "Gravity": 9.81,
        "DP_phi": 62, "DP_threshold_p": 0, "GrainVariability": 0.5,
        "IndDiameter": 2.0, "IndVelocity": 1.0, "IndDepth": 0.5, "SetupType": 0,
    }
    cfg.update(kw)
    p, _ = parse_json(json.dumps(cfg))
    return p


def standard(n_cells_x=32, n_cells_y=8, seed=1, h=0.25, grid=(96, 48), dt=1e-4, **kw):
    """The small config of the reference's first benchmark shape: an ice block
    on the floor, 4 points per cell, indenter of radius 1 m at 1 m/s."""
    p = params_for(grid[0], grid[1], h, dt, **kw)
    soa = make_block(p, n_cells_x * h, n_cells_y * h, ppc=4, seed=seed, n_grains=12)
    return p, soa


def stress(seed=7, n_cells_x=24, n_cells_y=10, h=0.25, grid=(80, 48), dt=1e-4):
    """Every branch of the hot path: weak ice and a fast indenter (crushing and
    the SVD return mapping), perturbed initial velocities / Fe / Bp, pre-crushed,
    liquid and disabled points."""
    p = params_for(grid[0], grid[1], h, dt, IndVelocity=10.0, IndDepth=0.8,
                   IceCompressiveStrength=2e6, IceTensileStrength=2e5, IceTensileStrength2=1.5e5,
                   IceShearStrength=1e5, DP_phi=45, DP_threshold_p=50, GrainVariability=0.6)
    soa = make_block(p, n_cells_x * h, n_cells_y * h, ppc=4, seed=seed, n_grains=20)
    rng = np.random.default_rng(seed)
    n = soa.size
    soa.vel[:] = rng.normal(0.0, 0.3, size=(2, n))
    soa.Fe[:] += rng.normal(0.0, 1.5e-4, size=(4, n))
    soa.Bp[:] = rng.normal(0.0, 0.05, size=(4, n))
    u = soa.utility
    r = rng.random(n)
    u[r < 0.05] |= STATUS_CRUSHED
    liq = (r >= 0.05) & (r < 0.08)
    u[liq] |= STATUS_LIQUID
    soa.Jp_inv[liq] = 1.0 + rng.normal(0.0, 1e-3, size=liq.sum())
    u[(r >= 0.08) & (r < 0.10)] |= STATUS_DISABLED
    p.nPtsTotal = int(((u & STATUS_DISABLED) == 0).sum())
    return p, soa


def comparable_bits(soa):
    """HSSOA bits with the fields the reference leaves undefined masked out:
    P and Q of liquid points are read from an uninitialised icy::Point on
    record steps (simulation/kernels.cuh:317,410-414)."""
    import numpy as np
    b = soa.buf[:, :soa.size].view(np.int64).copy()
    liq = soa.liquid()
    b[1:3, liq] = 0
    return b


def randomized(seed):
    """A seeded random floe-indentation scene: grid, cell size, block, points
    per cell, material (E, nu, friction angle, cohesion, strengths, grain
    variability), indenter (speed, depth, diameter) and time step drawn from
    ranges that keep every point inside the grid for the steps the tests run."""
    rng = np.random.default_rng(1000 + seed)
    h = float(rng.choice([0.1, 0.2, 0.25, 0.5]))
    gx, gy = int(rng.integers(48, 160)), int(rng.integers(32, 80))
    bw, bh = int(rng.integers(8, max(9, gx // 2))), int(rng.integers(4, max(5, gy // 3)))
    E = float(rng.uniform(5e8, 3e9))
    rho = 980.0
    c = np.sqrt(E / rho)
    dt = float(0.3 * h / c)                     # CFL number 0.3
    p = params_for(gx, gy, h, dt, YoungsModulus=E, PoissonsRatio=float(rng.uniform(0.2, 0.4)),
                   DP_phi=float(rng.uniform(30, 70)), DP_threshold_p=float(rng.choice([0.0, 50.0, 500.0])),
                   GrainVariability=float(rng.uniform(0.0, 0.8)), IndVelocity=float(rng.uniform(0.5, 8.0)),
                   IndDepth=float(rng.uniform(0.1, 0.6)) * bh * h, IndDiameter=float(rng.uniform(0.5, 3.0)),
                   IceCompressiveStrength=float(rng.uniform(2e6, 1e8)),
                   IceTensileStrength=float(rng.uniform(2e5, 5e6)), IceShearStrength=float(rng.uniform(1e5, 3e6)))
    soa = make_block(p, bw * h, bh * h, ppc=int(rng.choice([2, 4, 6, 9])), seed=seed,
                     n_grains=int(rng.integers(0, 40)))
    return p, soa
