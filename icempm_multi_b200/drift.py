"""FP32 split precision against FP64 over a long high-deformation run.

The fracture stress case: indenter of radius 1 m at 10 m/s, cohesion 0,
friction angle 30 deg, a block of `cells_x` x `cells_y` cells at 4 points per
cell on a 2048 x 1024 grid (default 1600 x 625 cells = 4 M points at
h = 0.05 m), dt from the CFL condition.  The ice strengths are 3 % of the
reference's defaults (SimParams::Reset, simulation/parameters_sim.cpp:31-34:
compressive 3 MPa, tensile 0.3 MPa, shear 0.18 MPa, second tensile 0.15 MPa)
so that the case fractures: on a 64,000-point block 43 % of the points are
crushed after 10,000 steps (at the default strengths 4 %), and the
crushed-point return mapping runs at every step for most of them.  The same initial state runs on the
FP64 path and on the FP32 split path of the same GPU, side by side; every
`every` steps both are downloaded and compared:

    pos       ||X32 - X64|| / ||X64||  over all points
    pos_max_h max |X32 - X64| / h
    Jp        ||Jp32 - Jp64|| / ||Jp64 - 1||  (relative to the plastic change)
    mom_x/y   total momentum sum(m v) of each run, and their difference
    mass      total mass of each run (constant by construction)
    crushed   fraction of points whose crushed bit differs

The FP64 path itself is held to the FP64 oracle by the GPU parity tests.
With `floor=True` a third run, FP64 on the one-thread-per-item kernels
(global atomics in another summation order), is compared with the tiled
FP64 run in the same way (keys with the suffix `_64`): the divergence that
round-off alone produces in this case, the floor against which the FP32
figures are read.

    python -m icempm_multi_b200.drift [--steps 20000] [--every 2000] [--cells 1600 625]
"""
import argparse
import json
import time

import numpy as np

from ._lib import PRECISION_FP32_SPLIT, PRECISION_FP64
from .hssoa import make_block
from .model import GPUImplementation
from .workloads import cfl_dt, workload_params


# ice strengths of the fracture case (Pa): compressive, tensile, shear, second tensile
FRACTURE_STRENGTHS = (3e6, 3e5, 1.8e5, 1.5e5)


def fracture_case(cells_x=1600, cells_y=625, h=0.05, grid=(2048, 1024), seed=5, strengths=FRACTURE_STRENGTHS):
    dt = cfl_dt(1e9, 0.3, 980.0, h)
    w = dict(grid_x=grid[0], grid_y=grid[1], h=h, block_w=cells_x * h, block_h=cells_y * h, ppc=4, dt=dt,
             E=1e9, nu=0.3, rho=980.0, phi=30.0, cohesion=0.0, ind_radius=1.0, ind_velocity=10.0,
             ind_depth=0.5, seed=seed, n_grains=64, strengths=strengths)
    p = workload_params(w)
    soa = make_block(p, w["block_w"], w["block_h"], ppc=4, seed=seed, n_grains=64)
    return p, soa, w


def compare(p, a, b):
    """Differences of the FP32 run a against the FP64 run b (host HSSOAs)."""
    m = ~b.disabled()
    dx = a.pos[:, m] - b.pos[:, m]
    mass = np.where(b.liquid()[m], p.WaterParticleMass, p.ParticleMass)
    jp_dev = np.linalg.norm(b.Jp_inv[m] - 1.0)
    out = {
        "pos": float(np.linalg.norm(dx) / np.linalg.norm(b.pos[:, m])),
        "pos_max_h": float(np.max(np.abs(dx)) / p.cellsize),
        "Jp": float(np.linalg.norm(a.Jp_inv[m] - b.Jp_inv[m]) / (jp_dev if jp_dev > 0 else 1.0)),
        "mom64": [float((mass * b.vel[0, m]).sum()), float((mass * b.vel[1, m]).sum())],
        "mom32": [float((mass * a.vel[0, m]).sum()), float((mass * a.vel[1, m]).sum())],
        "mass64": float(mass.sum()),
        "mass32": float(np.where(a.liquid()[~a.disabled()], p.WaterParticleMass, p.ParticleMass).sum()),
        "crushed_diff": float(np.mean(a.crushed()[m] != b.crushed()[m])),
        "crushed64": float(np.mean(b.crushed()[m])),
    }
    out["mom_diff_rel"] = float(np.hypot(out["mom32"][0] - out["mom64"][0], out["mom32"][1] - out["mom64"][1]) /
                                max(np.hypot(*out["mom64"]), 1e-300))
    return out


def run(steps=20000, every=2000, cells=(1600, 625), device=0, out=print, floor=False):
    p, soa, w = fracture_case(*cells)
    runs = {}
    legs = [("fp64", PRECISION_FP64), ("fp32", PRECISION_FP32_SPLIT)] + ([("fp64b", PRECISION_FP64)] if floor else [])
    for name, prec in legs:
        s = soa.clone(pinned=True)
        g = GPUImplementation(p, s, device=device, precision=prec)
        if name == "fp64b":
            g.set_option("tiled", 0)
        g.update_constants()
        g.transfer_ponts_to_device()
        runs[name] = [g, s, 0.0]
    out(json.dumps({"case": "fracture", "points": soa.size, "dt": p.InitialTimeStep, "h": p.cellsize,
                    "grid": [p.GridXTotal, p.GridY], "steps": steps, "every": every,
                    "indenter_speed": p.IndVelocity, "phi_deg": w["phi"]}))
    done = 0
    t0 = time.time()
    while done < steps:
        k = min(every, steps - done)
        for name in runs:
            g, s, t = runs[name]
            runs[name][2] = g.run_steps(done, k, t)
        done += k
        for name in runs:
            runs[name][0].transfer_from_device()
        assert runs["fp64"][2] == runs["fp32"][2]
        row = {"step": done, "t": runs["fp64"][2], "wall_s": round(time.time() - t0, 2)}
        row.update(compare(p, runs["fp32"][1], runs["fp64"][1]))
        if floor:
            c = compare(p, runs["fp64b"][1], runs["fp64"][1])
            row.update({k + "_64": c[k] for k in ("pos", "pos_max_h", "Jp", "crushed_diff", "mom_diff_rel")})
        out(json.dumps(row))
    for g, _, _ in runs.values():
        g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--every", type=int, default=2000)
    ap.add_argument("--cells", type=int, nargs=2, default=[1600, 625])
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--floor", action="store_true", help="also compare FP64 one-thread kernels with tiled FP64")
    a = ap.parse_args()
    run(a.steps, a.every, tuple(a.cells), a.device, out=lambda s: print(s, flush=True), floor=a.floor)


if __name__ == "__main__":
    main()
