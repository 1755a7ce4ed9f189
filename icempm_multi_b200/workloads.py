"""Seeded synthetic floe-indentation workloads.

The reference reads point clouds from HDF5 files (simulation/snapshotmanager.cpp:29-60),
which cannot be read here; these generators produce blocks with the same
placement rules (see icy_scene_block) and the parameter values of the
benchmark scenarios, passed through the reference's JSON keys.
"""
import json

from .hssoa import make_block
from .params import parse_json

# the single large instance: grid 4096 x 2048 at h = 0.05 m, 150 m x 40 m block at
# 4 points per cell (9.6 M points), dt = 2e-5 s
LARGE = dict(grid_x=4096, grid_y=2048, h=0.05, block_w=150.0, block_h=40.0, ppc=4, dt=2e-5,
             E=1e9, nu=0.3, rho=980.0, phi=62.0, cohesion=0.0, ind_radius=1.0, ind_velocity=1.0,
             ind_depth=0.5, seed=1, n_grains=64)

# a profiling-size instance on the same grid: 100 m x 30 m block (4.8 M points); its
# FP32 state (173 MB) is still larger than L2
MEDIUM = dict(LARGE, block_w=100.0, block_h=30.0)

# the CPU-runnable small instance: grid 512 x 256 at h = 0.25 m, 64 m x 16 m block
# (65,536 points), dt = 1e-4 s, 1000 steps
SMALL = dict(grid_x=512, grid_y=256, h=0.25, block_w=64.0, block_h=16.0, ppc=4, dt=1e-4,
             E=1e9, nu=0.3, rho=980.0, phi=62.0, cohesion=0.0, ind_radius=1.0, ind_velocity=1.0,
             ind_depth=0.5, seed=1, n_grains=16)


def workload_params(w, halo=8):
    cfg = {
        "InputRawPoints": "synthetic", "nPartitions": 1, "GridHaloSize": halo,
        "InitialTimeStep": w["dt"], "GridX": w["grid_x"], "GridY": w["grid_y"],
        "GridXDimension": w["grid_x"] * w["h"], "YoungsModulus": w["E"], "PoissonsRatio": w["nu"],
        "Density": w["rho"], "Gravity": 9.81, "DP_phi": w["phi"], "DP_threshold_p": w["cohesion"],
        "IndDiameter": 2 * w["ind_radius"], "IndVelocity": w["ind_velocity"], "IndDepth": w["ind_depth"],
        "SetupType": 0,
    }
    if "strengths" in w:   # ice strengths (Pa): compressive, tensile, shear, second tensile
        c, t, sh, t2 = w["strengths"]
        cfg.update({"IceCompressiveStrength": c, "IceTensileStrength": t, "IceShearStrength": sh,
                    "IceTensileStrength2": t2})
    p, _ = parse_json(json.dumps(cfg))
    return p


def make_workload(w, pinned=False):
    p = workload_params(w)
    soa = make_block(p, w["block_w"], w["block_h"], ppc=w["ppc"], seed=w["seed"], n_grains=w["n_grains"],
                     pinned=pinned)
    return p, soa


# ---------------------------------------------------------------- many scenarios
# grids available to served scenarios (cells), smallest that fits first
GRIDS = [(128, 128), (256, 128), (256, 256), (512, 256), (512, 512), (1024, 512), (2048, 512), (2048, 1024)]
# the batched workload's grids: 128 x 128 to 1024 x 512
GRIDS_BATCH = [g for g in GRIDS if g[0] <= 1024 and g[1] <= 512]


def wave_speed(E, nu, rho):
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    return ((lam + 2 * mu) / rho) ** 0.5


def cfl_dt(E, nu, rho, h, courant=0.4):
    """Explicit time step with c dt / h = courant (c: P-wave speed), rounded
    down to 2 significant digits."""
    import math
    dt = courant * h / wave_speed(E, nu, rho)
    e = math.floor(math.log10(dt))
    return math.floor(dt / 10 ** (e - 1)) * 10 ** (e - 1)


def floe_scenario(n_points, E, phi, v_ind, seed, h=0.1, aspect=4.0, ppc=4, nu=0.3, rho=980.0, grids=GRIDS):
    """A floe-indentation scenario of about n_points points: a block of
    aspect:1 cells at ppc points per cell on the smallest grid of `grids` that
    leaves room around it (the largest grid, with the block cut to fit, if
    none does), dt from the CFL condition."""
    import math
    cells = max(n_points // ppc, 16)
    ch = max(4, int(round(math.sqrt(cells / aspect))))
    cw = max(4, cells // ch)
    for gx, gy in grids:
        if cw + 24 <= gx and ch + 16 <= gy:
            break
    else:
        gx, gy = grids[-1]
        cw, ch = min(cw, gx - 24), min(ch, gy - 16)
    w = dict(grid_x=gx, grid_y=gy, h=h, block_w=cw * h, block_h=ch * h, ppc=ppc,
             dt=cfl_dt(E, nu, rho, h), E=E, nu=nu, rho=rho, phi=phi, cohesion=0.0,
             ind_radius=1.0, ind_velocity=v_ind, ind_depth=0.5, seed=seed, n_grains=16)
    return w


def batch_scenarios(n_instances=256, seed=7, n_min=10_000, n_max=500_000):
    """The batched workload: particle counts log-uniform in [n_min, n_max],
    E uniform 5e8-2e9 Pa, friction angle uniform 45-70 deg, indenter speed
    uniform 0.5-3 m/s (seeded)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_instances):
        n = int(round(np.exp(rng.uniform(np.log(n_min), np.log(n_max)))))
        out.append(floe_scenario(n, E=float(rng.uniform(5e8, 2e9)), phi=float(rng.uniform(45, 70)),
                                 v_ind=float(rng.uniform(0.5, 3.0)), seed=seed * 1000 + k, grids=GRIDS_BATCH))
    return out
