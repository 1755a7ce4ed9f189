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
    p, _ = parse_json(json.dumps(cfg))
    return p


def make_workload(w, pinned=False):
    p = workload_params(w)
    soa = make_block(p, w["block_w"], w["block_h"], ppc=w["ppc"], seed=w["seed"], n_grains=w["n_grains"],
                     pinned=pinned)
    return p, soa
